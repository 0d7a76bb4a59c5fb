// heom_dynamics: drop-in for the reference's CPU_dynamics executable
// (etoheom-cpu/src/CPU_dynamics.cpp:14-50; GPU_dynamics.cu:23-46 is its FP32 GPU twin).
//
//   heom_dynamics <file.key> [--sites 1,2] [--device D]
//
// Reads a population-dynamics key file (param::param_dynamics), propagates the HEOM from
// site 1 excited on the bit-exact FP64 path and prints CPU_dynamics' report byte for
// byte: the three header lines, then for each site "site i population: ", a blank line,
// one population per line in iostream's default format and a blank line.  The
// population vector has CPU_dynamics' length, (t_end - t_start) / print_step + 1 in
// float arithmetic.  Errors go to stderr with a non-zero exit status.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "heom.h"

static int die(const char *what, int rc) {
  std::fprintf(stderr, "heom_dynamics: %s failed (%d): %s\n", what, rc, heom_last_error());
  return 1;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <file.key> [--sites 1,2] [--device D]\n", argv[0]);
    return 2;
  }
  std::vector<int> sites = {1, 2}; // CPU_dynamics.cpp:26
  int device = 0;
  for (int a = 2; a < argc; a++) {
    if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--sites") && a + 1 < argc) {
      sites.clear();
      std::stringstream ss(argv[++a]);
      for (std::string t; std::getline(ss, t, ',');)
        if (!t.empty()) sites.push_back(std::atoi(t.c_str()));
    } else {
      std::fprintf(stderr, "heom_dynamics: unknown option '%s'\n", argv[a]);
      return 2;
    }
  }
  heom_problem *prob = nullptr;
  int rc = heom_problem_from_key(argv[1], HEOM_KEY_DYNAMICS, &prob);
  if (rc) return die("reading the key file", rc);
  heom_problem_info info;
  heom_problem_info_get(prob, &info);
  heom_opts opts{};
  opts.precision = HEOM_FP64_EXACT;
  opts.device = device;
  opts.max_points = 1;
  heom_plan *plan = nullptr;
  rc = heom_plan_create(prob, &opts, &plan);
  if (rc) return die("creating the device plan", rc);
  const int cap = info.n_record > 0 ? info.n_record : 1;
  std::vector<double> pop((size_t)sites.size() * cap, 0.0);
  int n = 0;
  rc = heom_run_populations(plan, sites.data(), (int)sites.size(), pop.data(), cap, &n);
  if (rc) return die("propagating", rc);
  // CPU_dynamics.cpp:27: population vectors of (t_end - t_start) / print_step + 1 entries
  const float lenf = (info.t_end - info.t_start) / info.print_step + 1;
  const size_t len = lenf > 0 ? (size_t)lenf : 0;
  std::cout << "Now is CPU version" << '\n';
  std::cout << "Running " << argv[1] << '\n';
  std::cout << "The bath type is " << "" << '\n'; // param_dynamics never sets bath_type
  for (size_t i = 0; i < sites.size(); i++) {
    std::cout << "site" << " " << i + 1 << " " << "population: " << '\n' << '\n';
    for (size_t j = 0; j < len; j++) std::cout << (j < (size_t)n ? pop[i * cap + j] : 0.0) << '\n';
    std::cout << '\n';
  }
  heom_plan_destroy(plan);
  heom_problem_destroy(prob);
  return 0;
}
