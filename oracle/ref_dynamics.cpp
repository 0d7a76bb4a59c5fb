// Reference population-dynamics driver (test infrastructure only).
//
// Links the reference's own, unmodified CPU library sources (compiled in place against
// the GSL-API shim by oracle/Makefile) and runs the flow of
// etoheom-cpu/src/CPU_dynamics.cpp:14-50 -- param_dynamics, construct_ADO_set,
// dynamics_solver -- for the sites given, printing the populations at full precision.
//
// Usage:  ref_dynamics <file.key> [site ...]      (default sites: 1 2, as CPU_dynamics)
// Output: #site <s> <n> then n rows "%.17e" (population vector sized as CPU_dynamics
//         sizes it: (t_end - t_start) / print_step + 1 in float arithmetic).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "param.h"
#include "utilize.h"
#include "dynamics.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <file.key> [site ...]\n", argv[0]);
    return 2;
  }
  param k;
  k.param_dynamics(argv[1]);
  construct_ADO_set(k);
  std::vector<int> sites;
  for (int a = 2; a < argc; a++) sites.push_back(std::atoi(argv[a]));
  if (sites.empty()) sites = {1, 2};
  std::vector<std::vector<double>> population(sites.size(),
                                              std::vector<double>((k.t_end - k.t_start) / k.print_step + 1, 0.0));
  dynamics_solver(k, k.Hal, sites, population);
  for (size_t i = 0; i < sites.size(); i++) {
    std::printf("#site %d %zu\n", sites[i], population[i].size());
    for (double v : population[i]) std::printf("%.17e\n", v);
  }
  k.param_free();
  return 0;
}
