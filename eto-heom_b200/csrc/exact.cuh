// Bit-exact FP64 right-hand side of the HEOM (the reference's operation order).
//
// total_ADO_dynamics_Ht (etoheom-cpu/lib/dynamics.cpp:117-179) evaluates, for ADO n,
//   zgemm(i, rho_n, V, 0)          -> C[r][c]  = sum_l (i rho[r][l]) V[l][c]
//   zgemm(-i, V, rho_n, 1)         -> C[r][c] += sum_l (-i V[r][l]) rho[l][c]
//   zaxpy(x_n, rho_n)              -> C[r][c] += x_n rho[r][c]            (n != 0)
//   per (site j, line k), up then down neighbours: zgemm with the one-hot S_j,
// with every product and sum rounded separately (baseline x86-64 has no FMA).
// Reference-BLAS zgemm forms temp = alpha*A[i][l] once and then adds temp*B[l][j],
// so every contribution to an element has the form  C += a (x) z  with
//   (a (x) z).re = fl(fl(a.re z.re) - fl(a.im z.im)),
//   (a (x) z).im = fl(fl(a.re z.im) + fl(a.im z.re)),
// and the one-hot S contributions reduce to a single such term on row or column
// s = j+1 (the other terms add exact zeros).  This header evaluates exactly that
// sequence, so results are bit-identical to the reference CPU build.
#pragma once
#include <cstdint>

namespace heom_dev {

struct Op {            // mirrors heom::CouplingOp
  int32_t kind, s, nb, pad;
  double cr, ci;
};

__device__ __forceinline__ void cmac(double &cr, double &ci, double ar, double ai, double zr, double zi) {
  const double d = __dsub_rn(__dmul_rn(ar, zr), __dmul_rn(ai, zi));
  const double e = __dadd_rn(__dmul_rn(ar, zi), __dmul_rn(ai, zr));
  cr = __dadd_rn(cr, d);
  ci = __dadd_rn(ci, e);
}

// k[e] for element (n, r, c).  rho is the whole state (n_ado x N x N, interleaved)
// and is read for neighbour elements; rn is ADO n's own N x N block (it may be a
// shared-memory copy); V is N x N.
__device__ __forceinline__ double2 rhs_exact(const double2 *__restrict__ rho, const double2 *__restrict__ rn,
                                             const double2 *__restrict__ V, int N, int n, int r, int c,
                                             double2 damp, const Op *__restrict__ ops, int op_begin, int op_end) {
  const int nn = N * N;
  double cr = 0.0, ci = 0.0;
  // i * rho[r][l] = (0*re - 1*im, 0*im + 1*re) = (-im, re) exactly
  for (int l = 0; l < N; l++) {
    const double2 a = rn[r * N + l];
    const double2 v = V[l * N + c];
    cmac(cr, ci, -a.y, a.x, v.x, v.y);
  }
  // -i * V[r][l] = (0*re + 1*im, 0*im - 1*re) = (im, -re) exactly
  for (int l = 0; l < N; l++) {
    const double2 v = V[r * N + l];
    const double2 z = rn[l * N + c];
    cmac(cr, ci, v.y, -v.x, z.x, z.y);
  }
  if (n != 0) {
    const double2 z = rn[r * N + c];
    cmac(cr, ci, damp.x, damp.y, z.x, z.y);
  }
  for (int q = op_begin; q < op_end; q++) {
    const Op o = ops[q];
    const bool hit = (o.kind == 0) ? (c == o.s) : (r == o.s);
    if (hit) {
      const double2 z = rho[(size_t)o.nb * nn + r * N + c];
      cmac(cr, ci, o.cr, o.ci, z.x, z.y);
    }
  }
  return make_double2(cr, ci);
}

// y + fl(a*x) per component: cblas_zaxpy with a real alpha (alpha.im * x = +-0).
__device__ __forceinline__ double2 axpy_exact(double2 y, double a, double2 x) {
  return make_double2(__dadd_rn(y.x, __dmul_rn(a, x.x)), __dadd_rn(y.y, __dmul_rn(a, x.y)));
}

// V[t] for element t: H - e1 X0 - e2 X1^T - e3 X2^T for the pulses switched on
// (gsl_matrix_complex_scale, then gsl_matrix_complex_sub; dynamics.cpp:348-363).
__device__ __forceinline__ double2 build_v(const double2 *H, const double2 *Xs, int nn, int t, unsigned flags,
                                           const double2 *e) {
  double vr = H[t].x, vi = H[t].y;
  for (int q = 0; q < 3; q++)
    if (flags & (1u << q)) {
      const double2 a = Xs[q * nn + t];
      const double mr = __dsub_rn(__dmul_rn(a.x, e[q].x), __dmul_rn(a.y, e[q].y));
      const double mi = __dadd_rn(__dmul_rn(a.x, e[q].y), __dmul_rn(a.y, e[q].x));
      vr = __dsub_rn(vr, mr);
      vi = __dsub_rn(vi, mi);
    }
  return make_double2(vr, vi);
}

// P_jj = sum_l (1*rho0[j][l]) X3[l][j], from zero, in l order (dynamics.cpp:369).
__device__ __forceinline__ double2 trace_row_exact(const double2 *rho0, const double2 *X3, int N, int j) {
  double pr = 0.0, pi = 0.0;
  for (int l = 0; l < N; l++) {
    const double2 a = rho0[j * N + l];
    // ONE * a = (1*re - 0*im, 1*im + 0*re) = (re, im)
    const double2 x = X3[l * N + j];
    cmac(pr, pi, a.x, a.y, x.x, x.y);
  }
  return make_double2(pr, pi);
}

} // namespace heom_dev
