// heom_2des: drop-in for the reference's CPU_2DES / GPU_2DES executables
// (etoheom-cpu/src/CPU_2DES.cpp:14-97, etoheom-gpu/src/GPU_2DES.cu:25-88).
//
//   heom_2des <file.key> [--precision fp64-exact|fp64|fp32-bulk] [--full-precision]
//             [--device D]
//
// Reads the same key file and prints P(t) = mean over samples of p111 - p110 - p101,
// one "re im" line per recorded point, in the reference's format
// (scientific, 6 digits; --full-precision prints 17).  Errors go to stderr with a
// non-zero exit status instead of a crash.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "heom.h"

static int die(const char *what, int rc) {
  std::fprintf(stderr, "heom_2des: %s failed (%d): %s\n", what, rc, heom_last_error());
  return 1;
}

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <file.key> [--precision fp64-exact|fp64|fp32-bulk] [--full-precision] [--device D]\n",
                 argv[0]);
    return 2;
  }
  int precision = HEOM_FP64_EXACT, device = 0, digits = 6;
  for (int a = 2; a < argc; a++) {
    if (!std::strcmp(argv[a], "--full-precision")) digits = 17;
    else if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--precision") && a + 1 < argc) {
      std::string p = argv[++a];
      if (p == "fp64-exact") precision = HEOM_FP64_EXACT;
      else if (p == "fp64") precision = HEOM_FP64;
      else if (p == "fp32-bulk") precision = HEOM_FP32_BULK;
      else { std::fprintf(stderr, "heom_2des: unknown precision '%s'\n", p.c_str()); return 2; }
    } else {
      std::fprintf(stderr, "heom_2des: unknown option '%s'\n", argv[a]);
      return 2;
    }
  }
  heom_problem *prob = nullptr;
  int rc = heom_problem_from_key(argv[1], 0, &prob);
  if (rc) return die("reading the key file", rc);
  heom_problem_info info;
  heom_problem_info_get(prob, &info);
  // The first sample's draws happen before the plan exists, as in CPU_2DES.cpp:50-60.
  rc = heom_problem_prepare_sample(prob);
  if (rc) return die("preparing sample 1", rc);
  heom_opts opts{};
  opts.precision = precision;
  opts.device = device;
  opts.max_points = 1;
  heom_plan *plan = nullptr;
  rc = heom_plan_create(prob, &opts, &plan);
  if (rc) return die("creating the device plan", rc);
  const int cap = info.n_record > 0 ? info.n_record : 1;
  std::vector<double> P(2 * (size_t)cap, 0.0), p(2 * (size_t)cap, 0.0);
  int n = 0;
  for (int s = 0; s < info.n_sample; s++) {
    if (s > 0) {
      rc = heom_problem_prepare_sample(prob);
      if (rc) return die("preparing a sample", rc);
      rc = heom_plan_update(plan, prob);
      if (rc) return die("uploading a sample", rc);
    }
    if (precision == HEOM_FP64_EXACT) {
      rc = heom_run_2des(plan, p.data(), nullptr, cap, &n);
      if (rc) return die("propagating", rc);
    } else {
      heom_scan_point pt{info.tau[0], info.tau[1], info.tau[2], info.t_end, 0};
      long long off = 0, total = 0;
      int cnt = 0;
      heom_scan_layout(plan, &pt, 1, &off, &cnt, &total);
      rc = heom_run_scan(plan, &pt, 1, p.data(), &off, &cnt);
      if (rc) return die("propagating", rc);
      n = cnt;
    }
    for (int j = 0; j < 2 * n; j++) P[j] += p[j] / info.n_sample; // CPU_2DES.cpp:83-89
  }
  std::cout << std::scientific << std::setprecision(digits);
  for (int j = 0; j < n; j++) std::cout << P[2 * j] << " " << P[2 * j + 1] << '\n';
  heom_plan_destroy(plan);
  heom_problem_destroy(prob);
  return 0;
}
