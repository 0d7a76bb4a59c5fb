// Adjoint (reverse-mode) gradient of a delay scan: discrete adjoint of the RK4 scheme with
// V frozen per step, in the mixed-difference basis, FP64, checkpointed.
//
// Forward step i (Horner form of RK4, see scan.cu):
//   w4 = rho_i;  w3 = rho_i + (h/4) L w4;  w2 = rho_i + (h/3) L w3;  w1 = rho_i + (h/2) L w2;
//   rho_{i+1} = rho_i + h L w1,          P_i = Tr(X3 (Q_i - R_i)) before the step.
// For a real objective J with dJ/dP_i = g_i (complex gradient convention
// g = dJ/dRe + i dJ/dIm) the adjoint lambda_i = dJ/drho_i obeys, per step,
//   u = lambda_{i+1};  acc = lambda_{i+1}
//   for (c, w) in (h, w1), (h/2, w2), (h/3, w3), (h/4, w4):
//       dJ/dtheta += Re <u, c (dL/dtheta) w>;   u = c L^H u;   acc += u
//   lambda_i = acc + dP_i/drho_i^H g_i,
// where L^H is the conjugate transpose of the four-component Liouvillian (sources run
// backwards: R <- D2, D3 and D2, D3 <- Q).  States between checkpoints (every
// ceil(sqrt(steps)) steps) are recomputed segment by segment, and the stage vectors of a
// step are recomputed from rho_i.
//
// Parameter derivatives:
//  * Hamiltonian parameters (site energies, couplings): dL/dtheta w = -i [D, w] with
//    D = dH/dtheta, so Re <g, c(-i[D, w])> = Re(-i sum_rl D_rl Mc_lr) with
//    Mc = c (w g^H - g^H w) accumulated over components, ADOs, stages and steps;
//  * bath amplitude scale s_jk: the up and down couplings of offset o = j + k K scale
//    as s^(1/2), so dL/ds w = (1/2s) (bath terms of offset o).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/heom.h"
#include "heom_host.h"
#include "sg.cuh"

namespace heom_dev {

namespace {
thread_local std::string adj_err;
size_t a256(size_t v) { return (v + 255) & ~(size_t)255; }

struct AdjArgs {
  int N, n_ado, M, K, Km, E_pt, S_max, apc;
  double h;
  const double *Hd;
  const double2 *Hoff, *Xs, *X3, *damp, *alpha;
  const double *xc, *yc;
  const int *up, *dn;
  const unsigned char *flags;
  const int *rec, *nsteps;
  const double2 *field;
  const long long *offsets;
};

__device__ __forceinline__ void cmadd(double &xr, double &xi, double2 a, double2 z) {
  xr = fma(a.x, z.x, fma(-a.y, z.y, xr));
  xi = fma(a.x, z.y, fma(a.y, z.x, xi));
}
__device__ __forceinline__ double2 conjd(double2 a) { return make_double2(a.x, -a.y); }

// Component operators of step i for point p into shared memory: A[q] (q = 0..3),
// S2 = V'_2, S3 = V'_3 (V'_q = -e_q X~_q where pulse q is on).
__device__ void build_ops(const AdjArgs &a, int p, int i, double2 *A, int *on) {
  const int N = a.N, NN = N * N;
  const size_t si = (size_t)p * a.S_max + i;
  const unsigned f = a.flags[si];
  double2 ef[3];
  for (int q = 0; q < 3; q++) {
    on[q] = (f >> q) & 1;
    ef[q] = a.field[si * 3 + q];
  }
  for (int t = threadIdx.x; t < NN; t += blockDim.x) {
    double vr[3], vi[3];
    for (int q = 0; q < 3; q++) {
      const double2 x = a.Xs[q * NN + t];
      vr[q] = on[q] ? -(x.x * ef[q].x - x.y * ef[q].y) : 0.0;
      vi[q] = on[q] ? -(x.x * ef[q].y + x.y * ef[q].x) : 0.0;
    }
    const double br = a.Hoff[t].x + vr[0], bi = a.Hoff[t].y + vi[0];
    A[t] = make_double2(br, bi);
    A[NN + t] = make_double2(br + vr[1], bi + vi[1]);
    A[2 * NN + t] = make_double2(br + vr[2], bi + vi[2]);
    A[3 * NN + t] = make_double2(br + vr[1] + vr[2], bi + vi[1] + vi[2]);
    A[4 * NN + t] = make_double2(vr[1], vi[1]);
    A[5 * NN + t] = make_double2(vr[2], vi[2]);
  }
}

} // namespace

// out = base + c * L w, for step i (identity copy of base where the point has ended).
__global__ void adj_fwd(AdjArgs a, const double2 *__restrict__ w, const double2 *__restrict__ base,
                       double2 *__restrict__ out, double c, int i) {
  extern __shared__ double2 smd[];
  const int p = blockIdx.z, cq = blockIdx.y, N = a.N, NN = N * N, nado = a.n_ado, M = a.M, K = a.K;
  const size_t pb = (size_t)p * a.E_pt;
  const int n0 = blockIdx.x * a.apc;
  if (i >= a.nsteps[p]) {
    for (int t = threadIdx.x; t < a.apc * NN; t += blockDim.x) {
      const int n = n0 + t / NN;
      if (n < nado) out[pb + (size_t)(cq * nado + n) * NN + t % NN] = base[pb + (size_t)(cq * nado + n) * NN + t % NN];
    }
    return;
  }
  double2 *A = smd;
  __shared__ int on[3];
  int onl[3];
  build_ops(a, p, i, A, onl);
  if (threadIdx.x == 0) for (int q = 0; q < 3; q++) on[q] = onl[q];
  __syncthreads();
  const double2 *Ac = A + cq * NN;
  const bool src = (on[1] || on[2]) && cq > 0;
  for (int t = threadIdx.x; t < a.apc * NN; t += blockDim.x) {
    const int n = n0 + t / NN;
    if (n >= nado) continue;
    const int rc = t % NN, r = rc / N, c2 = rc % N;
    const double2 *wn = w + pb + (size_t)(cq * nado + n) * NN;
    double xr = 0, xi = 0; // X = A w - w A
    for (int l = 0; l < N; l++) {
      cmadd(xr, xi, Ac[r * N + l], wn[l * N + c2]);
      cmadd(xr, xi, make_double2(-wn[r * N + l].x, -wn[r * N + l].y), Ac[l * N + c2]);
    }
    if (src)
      for (int s2 = 0; s2 < 2; s2++) {
        int from = -1, op = 0;
        if (cq == 1 && s2 == 0 && on[1]) { from = 0; op = 4; }
        if (cq == 2 && s2 == 0 && on[2]) { from = 0; op = 5; }
        if (cq == 3 && s2 == 0 && on[1]) { from = 2; op = 4; }
        if (cq == 3 && s2 == 1 && on[2]) { from = 1; op = 5; }
        if (from < 0) continue;
        const double2 *S = A + op * NN, *wf = w + pb + (size_t)(from * nado + n) * NN;
        for (int l = 0; l < N; l++) {
          cmadd(xr, xi, S[r * N + l], wf[l * N + c2]);
          cmadd(xr, xi, make_double2(-wf[r * N + l].x, -wf[r * N + l].y), S[l * N + c2]);
        }
      }
    double kr = xi, ki = -xr;
    for (int pass = 0; pass < 2; pass++) {
      const int s = pass == 0 ? r : c2;
      if (s < 1 || s > K || (pass == 1 && c2 == r)) continue;
      const int j = s - 1, dr = (r == s), dc = (c2 == s);
      for (int k = 0; k < a.Km; k++) {
        const int o = n * M + j + k * K, u = a.up[o], d = a.dn[o];
        if (u >= 0 && dr != dc) {
          const double x = a.xc[o] * (dc - dr);
          const double2 z = w[pb + (size_t)(cq * nado + u) * NN + rc];
          kr = fma(x, z.y, kr);
          ki = fma(-x, z.x, ki);
        }
        if (d >= 0) {
          const double y = a.yc[o];
          const double2 al = a.alpha[k];
          const double cr = -al.y * (dr + dc) * y, ci = al.x * (dr - dc) * y;
          const double2 z = w[pb + (size_t)(cq * nado + d) * NN + rc];
          kr = fma(cr, z.x, fma(-ci, z.y, kr));
          ki = fma(cr, z.y, fma(ci, z.x, ki));
        }
      }
    }
    const size_t idx = pb + (size_t)(cq * nado + n) * NN + rc;
    const double2 wv = w[idx], dmp = a.damp[n];
    const double gr = dmp.x, gi = dmp.y - (a.Hd[r] - a.Hd[c2]);
    kr = fma(gr, wv.x, fma(-gi, wv.y, kr));
    ki = fma(gr, wv.y, fma(gi, wv.x, ki));
    const double2 b = base[idx];
    out[idx] = make_double2(fma(c, kr, b.x), fma(c, ki, b.y));
  }
}

// u_out = c L^H u; acc += u_out; gradient contributions Re<u, c dL/dtheta w>.
__global__ void adj_bwd(AdjArgs a, const double2 *__restrict__ u, const double2 *__restrict__ w,
                        double2 *__restrict__ uo, double2 *__restrict__ acc, double c, int i,
                        double2 *__restrict__ gM, double *__restrict__ gB) {
  extern __shared__ double2 smd[];
  const int p = blockIdx.z, cq = blockIdx.y, N = a.N, NN = N * N, nado = a.n_ado, M = a.M, K = a.K;
  const size_t pb = (size_t)p * a.E_pt;
  const int n0 = blockIdx.x * a.apc;
  if (i >= a.nsteps[p]) {
    for (int t = threadIdx.x; t < a.apc * NN; t += blockDim.x) {
      const int n = n0 + t / NN;
      if (n < nado) uo[pb + (size_t)(cq * nado + n) * NN + t % NN] = make_double2(0.0, 0.0);
    }
    return;
  }
  double2 *A = smd;                 // 6 NN
  double2 *sM = smd + 6 * NN;       // NN partial M
  double *sB = (double *)(sM + NN); // M partial bath sums
  __shared__ int on[3];
  int onl[3];
  build_ops(a, p, i, A, onl);
  if (threadIdx.x == 0) for (int q = 0; q < 3; q++) on[q] = onl[q];
  for (int t = threadIdx.x; t < NN; t += blockDim.x) sM[t] = make_double2(0.0, 0.0);
  for (int t = threadIdx.x; t < M; t += blockDim.x) sB[t] = 0.0;
  __syncthreads();
  const double2 *Ac = A + cq * NN;
  for (int t = threadIdx.x; t < a.apc * NN; t += blockDim.x) {
    const int n = n0 + t / NN;
    if (n >= nado) continue;
    const int rc = t % NN, r = rc / N, c2 = rc % N;
    const double2 *un = u + pb + (size_t)(cq * nado + n) * NN;
    const double2 *wn = w + pb + (size_t)(cq * nado + n) * NN;
    // X' = A^H u - u A^H,  (A^H)_{rl} = conj(A_{lr})
    double xr = 0, xi = 0;
    for (int l = 0; l < N; l++) {
      cmadd(xr, xi, conjd(Ac[l * N + r]), un[l * N + c2]);
      cmadd(xr, xi, make_double2(-un[r * N + l].x, -un[r * N + l].y), conjd(Ac[c2 * N + l]));
    }
    // adjoint sources: R <- P2^H D2 + P3^H D3;  D2 <- P3^H Q;  D3 <- P2^H Q
    for (int s2 = 0; s2 < 2; s2++) {
      int from = -1, op = 0;
      if (cq == 0 && s2 == 0 && on[1]) { from = 1; op = 4; }
      if (cq == 0 && s2 == 1 && on[2]) { from = 2; op = 5; }
      if (cq == 1 && s2 == 0 && on[2]) { from = 3; op = 5; }
      if (cq == 2 && s2 == 0 && on[1]) { from = 3; op = 4; }
      if (from < 0) continue;
      const double2 *S = A + op * NN, *uf = u + pb + (size_t)(from * nado + n) * NN;
      for (int l = 0; l < N; l++) {
        cmadd(xr, xi, conjd(S[l * N + r]), uf[l * N + c2]);
        cmadd(xr, xi, make_double2(-uf[r * N + l].x, -uf[r * N + l].y), conjd(S[c2 * N + l]));
      }
    }
    double kr = -xi, ki = xr; // i X'
    // adjoint bath: gathers from the ADOs whose couplings land on this one
    for (int pass = 0; pass < 2; pass++) {
      const int s = pass == 0 ? r : c2;
      if (s < 1 || s > K || (pass == 1 && c2 == r)) continue;
      const int j = s - 1, dr = (r == s), dc = (c2 == s);
      for (int k = 0; k < a.Km; k++) {
        const int oo = j + k * K, o = n * M + oo;
        const int na = a.dn[o], nb = a.up[o];
        if (na >= 0 && dr != dc) { // adjoint of na's up-coupling: conj(-i x f) = i x f
          const double x = a.xc[(size_t)na * M + oo] * (dc - dr);
          const double2 z = u[pb + (size_t)(cq * nado + na) * NN + rc];
          kr = fma(-x, z.y, kr);
          ki = fma(x, z.x, ki);
        }
        if (nb >= 0) { // adjoint of nb's down-coupling: conj(y (-b(dr+dc), a(dr-dc)))
          const double y = a.yc[(size_t)nb * M + oo];
          const double2 al = a.alpha[k];
          const double cr = -al.y * (dr + dc) * y, ci = -al.x * (dr - dc) * y;
          const double2 z = u[pb + (size_t)(cq * nado + nb) * NN + rc];
          kr = fma(cr, z.x, fma(-ci, z.y, kr));
          ki = fma(cr, z.y, fma(ci, z.x, ki));
        }
      }
    }
    const size_t idx = pb + (size_t)(cq * nado + n) * NN + rc;
    const double2 uv = u[idx], dmp = a.damp[n];
    // conj(d_n) + i (Hd_r - Hd_c)
    const double gr = dmp.x, gi = -dmp.y + (a.Hd[r] - a.Hd[c2]);
    kr = fma(gr, uv.x, fma(-gi, uv.y, kr));
    ki = fma(gr, uv.y, fma(gi, uv.x, ki));
    const double2 o2 = make_double2(c * kr, c * ki);
    uo[idx] = o2;
    const double2 av = acc[idx];
    acc[idx] = make_double2(av.x + o2.x, av.y + o2.y);
    // ---- gradients with g = u, w = forward stage vector
    // M_{rc} (thread's element) = sum_k w[r][k] conj(g[c][k]) - conj(g[k][r]) w[k][c]
    double mr = 0, mi = 0;
    for (int k = 0; k < N; k++) {
      cmadd(mr, mi, wn[r * N + k], conjd(un[c2 * N + k]));
      const double2 gk = conjd(un[k * N + r]);
      cmadd(mr, mi, make_double2(-gk.x, -gk.y), wn[k * N + c2]);
    }
    atomicAdd(&sM[rc].x, c * mr);
    atomicAdd(&sM[rc].y, c * mi);
    // bath offsets: Re(conj(g_rc) * c * term_o) with the forward term of offset o
    for (int pass = 0; pass < 2; pass++) {
      const int s = pass == 0 ? r : c2;
      if (s < 1 || s > K || (pass == 1 && c2 == r)) continue;
      const int j = s - 1, dr = (r == s), dc = (c2 == s);
      for (int k = 0; k < a.Km; k++) {
        const int oo = j + k * K, o = n * M + oo, uu = a.up[o], d = a.dn[o];
        double tr = 0, ti = 0;
        if (uu >= 0 && dr != dc) {
          const double x = a.xc[o] * (dc - dr);
          const double2 z = w[pb + (size_t)(cq * nado + uu) * NN + rc];
          tr += x * z.y;
          ti -= x * z.x;
        }
        if (d >= 0) {
          const double y = a.yc[o];
          const double2 al = a.alpha[k];
          const double cr = -al.y * (dr + dc) * y, ci = al.x * (dr - dc) * y;
          const double2 z = w[pb + (size_t)(cq * nado + d) * NN + rc];
          tr += cr * z.x - ci * z.y;
          ti += cr * z.y + ci * z.x;
        }
        if (tr != 0.0 || ti != 0.0) atomicAdd(&sB[oo], c * (uv.x * tr + uv.y * ti));
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < NN; t += blockDim.x) {
    atomicAdd(&gM[(size_t)p * NN + t].x, sM[t].x);
    atomicAdd(&gM[(size_t)p * NN + t].y, sM[t].y);
  }
  for (int t = threadIdx.x; t < M; t += blockDim.x)
    if (sB[t] != 0.0) atomicAdd(&gB[(size_t)p * M + t], sB[t]);
}

// Forward readout P_i = Tr(X3 (Q - R)) of every point recorded at step i.
__global__ void adj_record_fwd(AdjArgs a, const double2 *__restrict__ rho, int i, double2 *__restrict__ P) {
  const int p = blockIdx.x;
  if (i >= a.nsteps[p]) return;
  const int rec = a.rec[(size_t)p * a.S_max + i];
  if (rec < 0 || threadIdx.x >= 32) return;
  const int N = a.N, NN = N * N;
  const size_t pb = (size_t)p * a.E_pt;
  double sr = 0, si = 0;
  for (int t = threadIdx.x; t < NN; t += 32) {
    const int jr = t / N, l = t % N;
    const double2 q = rho[pb + (size_t)3 * a.n_ado * NN + t], r0 = rho[pb + t];
    const double2 v = make_double2(q.x - r0.x, q.y - r0.y), x = a.X3[l * N + jr];
    sr += v.x * x.x - v.y * x.y;
    si += v.x * x.y + v.y * x.x;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_down_sync(0xffffffffu, sr, o);
    si += __shfl_down_sync(0xffffffffu, si, o);
  }
  if (threadIdx.x == 0) P[a.offsets[p] + rec] = make_double2(sr, si);
}

// acc += dP_i/drho^H g_i: Q block of ADO 0 gets conj(X3^T) g, R block gets -conj(X3^T) g.
__global__ void adj_record_bwd(AdjArgs a, double2 *__restrict__ acc, int i, const double2 *__restrict__ g) {
  const int p = blockIdx.x;
  if (i >= a.nsteps[p]) return;
  const int rec = a.rec[(size_t)p * a.S_max + i];
  if (rec < 0) return;
  const int N = a.N, NN = N * N;
  const size_t pb = (size_t)p * a.E_pt;
  const double2 gp = g[a.offsets[p] + rec];
  for (int t = threadIdx.x; t < NN; t += blockDim.x) {
    const int jr = t / N, l = t % N;
    const double2 x = conjd(a.X3[l * N + jr]);
    const double vr = x.x * gp.x - x.y * gp.y, vi = x.x * gp.y + x.y * gp.x;
    double2 *q = acc + pb + (size_t)3 * a.n_ado * NN + t, *r0 = acc + pb + t;
    *q = make_double2(q->x + vr, q->y + vi);
    *r0 = make_double2(r0->x - vr, r0->y - vi);
  }
}

__global__ void adj_init(double2 *rho, long long total, int E_pt) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x)
    rho[e] = make_double2((e % E_pt) == 0 ? 1.0 : 0.0, 0.0);
}

const char *adj_last_error() { return adj_err.c_str(); }

// Host driver: see the header comment.  P (host, `total` points) receives the forward
// readout, grad (host, n_params) the gradient of Re sum conj(g) P.
int adjoint_scan(const heom::Problem &p, const heom_scan_point *pts, int n, const long long *offsets, long long total,
                 const double *g_host, double *P_host, double *grad, long long *launches, cudaStream_t st) {
#define ACK(call)                                                                                   \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) { adj_err = std::string(#call) + ": " + cudaGetErrorString(e_); rc = HEOM_ERR_CUDA; goto done; } \
  } while (0)
  int rc = HEOM_OK;
  const int N = p.N(), NN = N * N, nado = p.n_ado, M = p.M;
  const int E_pt = 4 * nado * NN;
  const long long E = (long long)n * E_pt;
  const size_t SB = a256(16 * (size_t)E);
  std::vector<int> nsteps(n);
  int S_max = 1;
  for (int q = 0; q < n; q++) { nsteps[q] = heom::steps_for(p, pts[q].t_end); S_max = std::max(S_max, nsteps[q]); }
  const int Kc = std::max(1, (int)std::ceil(std::sqrt((double)S_max)));
  const int nck = (S_max + Kc - 1) / Kc;
  const size_t NS = (size_t)n * S_max;
  std::vector<unsigned char> flags(NS, 0);
  std::vector<int> rec(NS, -1);
  std::vector<double> field(6 * NS, 0.0);
  for (int q = 0; q < n; q++) {
    const double tau[3] = {pts[q].tau1, pts[q].tau2, pts[q].tau3};
    const int nv[3] = {1, 1, 1};
    heom::Schedule sc = heom::make_schedule(p, tau, pts[q].t_end, nv);
    for (int i = 0; i < sc.n_steps; i++) {
      flags[(size_t)q * S_max + i] = sc.flags[i] & 7;
      rec[(size_t)q * S_max + i] = sc.rec_idx[i];
      for (int k = 0; k < 3; k++) {
        field[2 * (((size_t)q * S_max + i) * 3 + k)] = sc.field[2 * ((size_t)k * sc.n_steps + i)];
        field[2 * (((size_t)q * S_max + i) * 3 + k) + 1] = sc.field[2 * ((size_t)k * sc.n_steps + i) + 1];
      }
    }
  }
  // tables (FP64 staged layout)
  std::vector<double> hd(N), hoff(2 * NN, 0.0), xs(6 * NN), x3(2 * NN), xc((size_t)nado * M), yc((size_t)nado * M);
  std::vector<int> up(p.up.begin(), p.up.end()), dn(p.dn.begin(), p.dn.end());
  for (int r = 0; r < N; r++)
    for (int c = 0; c < N; c++) {
      const size_t t = (size_t)r * N + c, tt = (size_t)c * N + r;
      if (r == c) { hd[r] = p.H[2 * t]; hoff[2 * t + 1] = p.H[2 * t + 1]; }
      else { hoff[2 * t] = p.H[2 * t]; hoff[2 * t + 1] = p.H[2 * t + 1]; }
      xs[2 * t] = p.X[0][2 * t]; xs[2 * t + 1] = p.X[0][2 * t + 1];
      xs[2 * (NN + t)] = p.X[1][2 * tt]; xs[2 * (NN + t) + 1] = p.X[1][2 * tt + 1];
      xs[2 * (2 * NN + t)] = p.X[2][2 * tt]; xs[2 * (2 * NN + t) + 1] = p.X[2][2 * tt + 1];
      x3[2 * t] = p.X[3][2 * t]; x3[2 * t + 1] = p.X[3][2 * t + 1];
    }
  for (int q = 0; q < nado; q++)
    for (int o = 0; o < M; o++) { xc[(size_t)q * M + o] = heom::coupling_x(p, q, o); yc[(size_t)q * M + o] = heom::coupling_y(p, q, o); }
  unsigned char *dev = nullptr;
  double2 *gM = nullptr;
  double *gB = nullptr;
  AdjArgs a{};
  // device layout
  const size_t o_hd = 0, o_hoff = a256(o_hd + 8 * N), o_xs = a256(o_hoff + 16 * NN), o_x3 = a256(o_xs + 48 * NN);
  const size_t o_damp = a256(o_x3 + 16 * NN), o_alpha = a256(o_damp + 16 * (size_t)nado);
  const size_t o_xc = a256(o_alpha + 16 * (size_t)p.K_m), o_yc = a256(o_xc + 8 * xc.size());
  const size_t o_up = a256(o_yc + 8 * yc.size()), o_dn = a256(o_up + 4 * up.size()), o_fl = a256(o_dn + 4 * dn.size());
  const size_t o_rec = a256(o_fl + NS), o_field = a256(o_rec + 4 * NS), o_ns = a256(o_field + 48 * NS);
  const size_t o_off = a256(o_ns + 4 * (size_t)n), o_g = a256(o_off + 8 * (size_t)n), o_P = a256(o_g + 16 * (size_t)total);
  const size_t o_st = a256(o_P + 16 * (size_t)total);
  const int nbuf = 10 + nck + Kc; // rho_a, rho_b, w1, w2, w3, lam, acc, u_a, u_b, spare, ckpt[nck], seg[Kc]
  const size_t bytes = o_st + SB * (size_t)nbuf;
  const int apc = std::max(1, 256 / NN) * NN > 1024 ? 1 : std::max(1, 256 / NN);
  const int threads = std::min(1024, ((apc * NN + 31) / 32) * 32);
  const size_t smem_f = 16 * 6 * (size_t)NN, smem_b = 16 * 7 * (size_t)NN + 8 * (size_t)M + 16;
  const dim3 grid((nado + apc - 1) / apc, 4, n);
  double2 *rho_a, *rho_b, *w1, *w2, *w3, *lam, *acc, *ua, *ub;
  std::vector<double2 *> ck(nck), seg(Kc);
  std::vector<double> gMh((size_t)n * NN * 2), gBh((size_t)n * M);
  long long nl = 0;
  const double h = (double)p.step_size;
  ACK(cudaMalloc(&dev, bytes));
  ACK(cudaMalloc(&gM, 16 * (size_t)n * NN));
  ACK(cudaMalloc(&gB, 8 * (size_t)n * M));
  ACK(cudaMemsetAsync(gM, 0, 16 * (size_t)n * NN, st));
  ACK(cudaMemsetAsync(gB, 0, 8 * (size_t)n * M, st));
  ACK(cudaMemcpyAsync(dev + o_hd, hd.data(), 8 * hd.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_hoff, hoff.data(), 8 * hoff.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_xs, xs.data(), 8 * xs.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_x3, x3.data(), 8 * x3.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_damp, p.damp.data(), 16 * (size_t)nado, cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_alpha, p.alpha.data(), 16 * (size_t)p.K_m, cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_xc, xc.data(), 8 * xc.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_yc, yc.data(), 8 * yc.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_up, up.data(), 4 * up.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_dn, dn.data(), 4 * dn.size(), cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_fl, flags.data(), NS, cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_rec, rec.data(), 4 * NS, cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_field, field.data(), 48 * NS, cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_ns, nsteps.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_off, offsets, 8 * (size_t)n, cudaMemcpyHostToDevice, st));
  ACK(cudaMemcpyAsync(dev + o_g, g_host, 16 * (size_t)total, cudaMemcpyHostToDevice, st));
  ACK(cudaMemsetAsync(dev + o_P, 0, 16 * (size_t)total, st));
  a.N = N; a.n_ado = nado; a.M = M; a.K = p.K; a.Km = p.K_m; a.E_pt = E_pt; a.S_max = S_max; a.apc = apc; a.h = h;
  a.Hd = (const double *)(dev + o_hd);
  a.Hoff = (const double2 *)(dev + o_hoff);
  a.Xs = (const double2 *)(dev + o_xs);
  a.X3 = (const double2 *)(dev + o_x3);
  a.damp = (const double2 *)(dev + o_damp);
  a.alpha = (const double2 *)(dev + o_alpha);
  a.xc = (const double *)(dev + o_xc);
  a.yc = (const double *)(dev + o_yc);
  a.up = (const int *)(dev + o_up);
  a.dn = (const int *)(dev + o_dn);
  a.flags = dev + o_fl;
  a.rec = (const int *)(dev + o_rec);
  a.field = (const double2 *)(dev + o_field);
  a.nsteps = (const int *)(dev + o_ns);
  a.offsets = (const long long *)(dev + o_off);
  {
    double2 *bufs[10];
    for (int b = 0; b < 10; b++) bufs[b] = (double2 *)(dev + o_st + SB * b);
    rho_a = bufs[0]; rho_b = bufs[1]; w1 = bufs[2]; w2 = bufs[3]; w3 = bufs[4];
    lam = bufs[5]; acc = bufs[6]; ua = bufs[7]; ub = bufs[8];
    for (int k = 0; k < nck; k++) ck[k] = (double2 *)(dev + o_st + SB * (10 + k));
    for (int k = 0; k < Kc; k++) seg[k] = (double2 *)(dev + o_st + SB * (10 + nck + k));
  }
  // ---- forward with checkpoints
  adj_init<<<1024, 256, 0, st>>>(rho_a, E, E_pt);
  nl++;
  for (int i = 0; i < S_max; i++) {
    if (i % Kc == 0) ACK(cudaMemcpyAsync(ck[i / Kc], rho_a, 16 * (size_t)E, cudaMemcpyDeviceToDevice, st));
    adj_record_fwd<<<n, 32, 0, st>>>(a, rho_a, i, (double2 *)(dev + o_P));
    adj_fwd<<<grid, threads, smem_f, st>>>(a, rho_a, rho_a, w3, h / 4, i);
    adj_fwd<<<grid, threads, smem_f, st>>>(a, w3, rho_a, w2, h / 3, i);
    adj_fwd<<<grid, threads, smem_f, st>>>(a, w2, rho_a, w1, h / 2, i);
    adj_fwd<<<grid, threads, smem_f, st>>>(a, w1, rho_a, rho_b, h, i);
    std::swap(rho_a, rho_b);
    nl += 5;
  }
  ACK(cudaGetLastError());
  ACK(cudaMemcpyAsync(P_host, dev + o_P, 16 * (size_t)total, cudaMemcpyDeviceToHost, st));
  // ---- backward
  ACK(cudaMemsetAsync(lam, 0, 16 * (size_t)E, st));
  for (int sgi = nck - 1; sgi >= 0; sgi--) {
    const int i0 = sgi * Kc, i1 = std::min(S_max, i0 + Kc);
    ACK(cudaMemcpyAsync(seg[0], ck[sgi], 16 * (size_t)E, cudaMemcpyDeviceToDevice, st));
    for (int t = 1; t < i1 - i0; t++) {
      const int i = i0 + t - 1;
      adj_fwd<<<grid, threads, smem_f, st>>>(a, seg[t - 1], seg[t - 1], w3, h / 4, i);
      adj_fwd<<<grid, threads, smem_f, st>>>(a, w3, seg[t - 1], w2, h / 3, i);
      adj_fwd<<<grid, threads, smem_f, st>>>(a, w2, seg[t - 1], w1, h / 2, i);
      adj_fwd<<<grid, threads, smem_f, st>>>(a, w1, seg[t - 1], seg[t], h, i);
      nl += 4;
    }
    for (int i = i1 - 1; i >= i0; i--) {
      double2 *ri = seg[i - i0];
      adj_fwd<<<grid, threads, smem_f, st>>>(a, ri, ri, w3, h / 4, i);
      adj_fwd<<<grid, threads, smem_f, st>>>(a, w3, ri, w2, h / 3, i);
      adj_fwd<<<grid, threads, smem_f, st>>>(a, w2, ri, w1, h / 2, i);
      ACK(cudaMemcpyAsync(acc, lam, 16 * (size_t)E, cudaMemcpyDeviceToDevice, st));
      adj_bwd<<<grid, threads, smem_b, st>>>(a, lam, w1, ua, acc, h, i, gM, gB);
      adj_bwd<<<grid, threads, smem_b, st>>>(a, ua, w2, ub, acc, h / 2, i, gM, gB);
      adj_bwd<<<grid, threads, smem_b, st>>>(a, ub, w3, ua, acc, h / 3, i, gM, gB);
      adj_bwd<<<grid, threads, smem_b, st>>>(a, ua, ri, ub, acc, h / 4, i, gM, gB);
      adj_record_bwd<<<n, 64, 0, st>>>(a, acc, i, (const double2 *)(dev + o_g));
      std::swap(lam, acc);
      nl += 8;
    }
    ACK(cudaGetLastError());
  }
  ACK(cudaMemcpyAsync(gMh.data(), gM, 16 * (size_t)n * NN, cudaMemcpyDeviceToHost, st));
  ACK(cudaMemcpyAsync(gBh.data(), gB, 8 * (size_t)n * M, cudaMemcpyDeviceToHost, st));
  ACK(cudaStreamSynchronize(st));
  {
    // assemble: H parameters Re(-i sum_rl D_rl M_lr); bath scales (1/2s) sum
    const int np = heom::n_params(p), nh = np - p.K * p.K_m;
    std::vector<double> Msum(2 * (size_t)NN, 0.0);
    for (int q = 0; q < n; q++)
      for (int t = 0; t < 2 * NN; t++) Msum[t] += gMh[(size_t)q * 2 * NN + t];
    heom::cbuf D;
    for (int k = 0; k < nh; k++) {
      heom::param_dH(p, k, D);
      double sre = 0.0;
      for (int r = 0; r < N; r++)
        for (int l = 0; l < N; l++) {
          const double dr = D[2 * ((size_t)r * N + l)], di = D[2 * ((size_t)r * N + l) + 1];
          const double mr = Msum[2 * ((size_t)l * N + r)], mi = Msum[2 * ((size_t)l * N + r) + 1];
          // Re(-i (d m)) = Im(d m)
          sre += dr * mi + di * mr;
        }
      grad[k] = sre;
    }
    for (int j = 0; j < p.K; j++)
      for (int k = 0; k < p.K_m; k++) {
        const int oo = j + k * p.K;
        double sB = 0.0;
        for (int q = 0; q < n; q++) sB += gBh[(size_t)q * M + oo];
        grad[nh + j * p.K_m + k] = sB * 0.5 / p.bath_scale[(size_t)j * p.K_m + k];
      }
  }
  if (launches) *launches += nl;
done:
  if (dev) cudaFree(dev);
  if (gM) cudaFree(gM);
  if (gB) cudaFree(gB);
  return rc;
#undef ACK
}

} // namespace heom_dev
