// Reference driver (test infrastructure only).
//
// Links the reference's own, unmodified CPU library sources
// (etoheom-cpu/lib/{param,utilize,dynamics,TD_hamiltonian,polar,constant}.cpp,
// compiled in place against the GSL-API shim by oracle/Makefile) and runs the
// same flow as etoheom-cpu/src/CPU_2DES.cpp:14-91, but prints at full
// precision and also prints every trajectory (masks 111, 110, 101) so parity
// can be checked per trajectory and on the combined output.
//
// Usage:  ref_driver <file.key> [--dump]
// Output (text):
//   [--dump]  setup section: sizes, ADO multi-indices, H, X[0..3], bath, pulses
//   #traj <sample> <npoints>      then rows: p111r p111i p110r p110i p101r p101i
//   #combined <npoints>           then rows: Pr Pi   (mean over samples)
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "param.h"
#include "utilize.h"
#include "dynamics.h"
#include "polar.h"

static void dump_matrix(const char* name, const gsl_matrix_complex* m) {
  std::printf("#matrix %s %zu %zu\n", name, m->size1, m->size2);
  for (size_t i = 0; i < m->size1; i++)
    for (size_t j = 0; j < m->size2; j++) {
      gsl_complex z = gsl_matrix_complex_get(m, i, j);
      std::printf("%.17e %.17e\n", GSL_REAL(z), GSL_IMAG(z));
    }
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <file.key> [--dump]\n", argv[0]);
    return 2;
  }
  bool dump = argc > 2 && std::strcmp(argv[2], "--dump") == 0;
  param k;
  k.param_2des(argv[1]);
  construct_ADO_set(k);

  gsl_rng_env_setup();
  gsl_rng* r = gsl_rng_alloc(gsl_rng_default);
  gsl_rng_set(r, k.seed);

  if (dump) {
    std::printf("#sizes %d %d %d %d %d %zu\n", k.single_size, k.sys_size, k.K, k.K_m, k.L, k.ado.size());
    std::printf("#ado %zu %d\n", k.ado.size(), k.K * k.K_m);
    for (const std::string& s : k.ado) {
      for (size_t q = 0; q < s.size(); q++) std::printf("%d%c", (int)s[q], q + 1 < s.size() ? ' ' : '\n');
    }
    std::printf("#bath %d %d\n", k.K, k.K_m);
    for (int j = 0; j < k.K; j++)
      for (int m = 0; m < k.K_m; m++)
        std::printf("%.17e %.17e %.17e %.17e\n", GSL_REAL(k.alpha[j][m]), GSL_IMAG(k.alpha[j][m]),
                    GSL_REAL(k.gamma[j][m]), GSL_IMAG(k.gamma[j][m]));
    std::printf("#pulses\n");
    for (int p = 0; p < 3; p++)
      std::printf("%.17e %.17e %.17e %.17e\n", k.pulses[p].E0, k.pulses[p].tau0, k.pulses[p].taup, k.pulses[p].w0);
    std::printf("#time %.9e %.9e %.9e %.9e\n", k.t_start, k.t_end, k.step_size, k.print_step);
  }

  int N = k.sys_size;
  gsl_matrix_complex* H = gsl_matrix_complex_alloc(N, N);
  std::vector<std::vector<gsl_complex>> combined;
  for (int s = 0; s < k.n_sample; s++) {
    gsl_matrix_complex_set_all(H, gsl_complex_rect(0.0, 0.0));
    construct_Hal(k, H, r);
    polar_mat_set(k);
    polar_mat_ranrot(k, r);
    compute_pulse_interaction(k);
    if (dump) {
      dump_matrix("H", H);
      for (int q = 0; q < 4; q++) dump_matrix(("X" + std::to_string(q)).c_str(), k.X[q]);
    }
    std::vector<gsl_complex> p1, p2, p3;
    twoD_spectrum_solver(k, H, 1, 1, 1, p1);
    twoD_spectrum_solver(k, H, 1, 1, 0, p2);
    twoD_spectrum_solver(k, H, 1, 0, 1, p3);
    std::printf("#traj %d %zu\n", s, p1.size());
    std::vector<gsl_complex> pi;
    for (size_t j = 0; j < p1.size(); j++) {
      std::printf("%.17e %.17e %.17e %.17e %.17e %.17e\n", GSL_REAL(p1[j]), GSL_IMAG(p1[j]), GSL_REAL(p2[j]),
                  GSL_IMAG(p2[j]), GSL_REAL(p3[j]), GSL_IMAG(p3[j]));
      // Same combine as CPU_2DES.cpp:73-79.
      double re = GSL_REAL(p1[j]) - GSL_REAL(p2[j]) - GSL_REAL(p3[j]);
      double im = GSL_IMAG(p1[j]) - GSL_IMAG(p2[j]) - GSL_IMAG(p3[j]);
      pi.push_back(gsl_complex_rect(re, im));
    }
    combined.push_back(pi);
  }
  // Mean over samples, CPU_2DES.cpp:83-89.
  std::vector<gsl_complex> P(combined.empty() ? 0 : combined[0].size(), gsl_complex_rect(0.0, 0.0));
  for (size_t s = 0; s < combined.size(); s++)
    for (size_t j = 0; j < combined[s].size(); j++) {
      P[j].dat[0] += GSL_REAL(combined[s][j]) / k.n_sample;
      P[j].dat[1] += GSL_IMAG(combined[s][j]) / k.n_sample;
    }
  std::printf("#combined %zu\n", P.size());
  for (const gsl_complex& z : P) std::printf("%.17e %.17e\n", GSL_REAL(z), GSL_IMAG(z));
  gsl_matrix_complex_free(H);
  gsl_rng_free(r);
  k.param_free();
  return 0;
}
