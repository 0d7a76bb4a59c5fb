// General-size propagation path: see sg.cuh.
//
// Arithmetic per element (r, c) of ADO n in component q, for Horner stage m (w is the
// previous stage's iterate, w = rho at the first stage of a step):
//   k = -i (H_rr - H_cc) w + d_n w                                   (FP64)
//     + -i [A_q, w] + sources_q + bath couplings of rows/columns 1..K (FP32 or FP64)
//   w' = rho + (h/m) k,   rho <- w' after m = 1,
// with A_q = off-diagonal H plus the pulse operators switched on for component q, and
// the mixed-difference sources D2 <- P2 R, D3 <- P3 R, Q <- P2 D3 + P3 D2 (see scan.cu).
// P = Tr(X3 (Q - R)) (C = 4) or Tr(X3 rho) (C = 1) is recorded before each step, from
// the FP64 state, exactly where the reference records it (dynamics.cpp:367-381).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "sg.cuh"

namespace heom_dev {

namespace {
thread_local std::string sg_err;

template <class T> struct Vec2;
template <> struct Vec2<float> { using t = float2; };
template <> struct Vec2<double> { using t = double2; };
template <class T> __device__ __forceinline__ typename Vec2<T>::t to2(double x, double y);
template <> __device__ __forceinline__ float2 to2<float>(double x, double y) { return make_float2((float)x, (float)y); }
template <> __device__ __forceinline__ double2 to2<double>(double x, double y) { return make_double2(x, y); }

size_t a256(size_t v) { return (v + 255) & ~(size_t)255; }

struct SgArgs {
  int N, n_ado, M, K, Km, C, E_pt, S_max, apc, mask[3];
  double h;
  const double *Hd;
  const double2 *Hoff, *Xs, *X3, *damp, *alpha;
  const double *xc, *yc;
  const int *up, *dn;
  const unsigned char *flags;
  const int *rec, *nsteps;
  const double2 *field;
  const long long *offsets;
  double2 *rho, *w64a, *w64b;
  void *w32a, *w32b;
  double2 *P;
  unsigned char *ops;    // per (point, component): the step's operators and their ranges
  long long ops_stride;  // bytes per (point, component)
};

// Table layout in one allocation (byte offsets, 256-aligned sections).
struct SgTab {
  size_t Hd, Hoff, Xs, X3, damp, alpha, xc, yc, up, dn, total;
  SgTab(int N, int n_ado, int M, int Km) {
    const size_t NN = (size_t)N * N, nM = (size_t)n_ado * M;
    Hd = 0;
    Hoff = a256(Hd + 8 * N);
    Xs = a256(Hoff + 16 * NN);
    X3 = a256(Xs + 48 * NN);
    damp = a256(X3 + 16 * NN);
    alpha = a256(damp + 16 * (size_t)n_ado);
    xc = a256(alpha + 16 * (size_t)Km);
    yc = a256(xc + 8 * nM);
    up = a256(yc + 8 * nM);
    dn = a256(up + 4 * nM);
    total = a256(dn + 4 * nM);
  }
};

} // namespace

const char *sg_last_error() { return sg_err.c_str(); }

// Shared-memory geometry of sg_stage.  Blocks are stored with rows padded to Np (a
// multiple of 4) plus 2, so that a thread's 4-wide column strip is one or two 16-byte
// loads and the rows of a warp's tile fall in different banks.
__host__ __device__ inline int sg_np(int N) { return (N + 3) & ~3; }
__host__ __device__ inline int sg_stride(int N) { return sg_np(N) + 2; }
// Strip slots per ADO: N rows x Np/4 strips, laid out linearly for Np <= 16 and in warp
// tiles of 8 rows x 4 strips (conflict-free strip loads) for wider blocks.
__host__ __device__ inline int sg_slots_per_ado(int N) {
  const int spr = sg_np(N) / 4;
  return spr <= 4 ? N * spr : ((N + 7) / 8) * ((spr + 3) / 4) * 32;
}
// T2 elements of dynamic shared memory: own operator, P2, P3 (N x S each), the own and
// up to two source blocks of apc ADOs (N x S each), the commutator of apc ADOs (N x N).
__host__ __device__ inline size_t sg_smem_elems(int N, int apc) {
  return (size_t)(3 + 3 * apc) * N * sg_stride(N) + (size_t)apc * N * N;
}

constexpr int kSgMaxN = 32;
// Bytes of one (point, component) entry of the operator buffer: own operator, P2, P3
// (N x S each, T2) and int ranges [3][4][kSgMaxN] (row lo/hi, column lo/hi).
__host__ __device__ inline size_t sg_ops_bytes(int N, size_t tsz) {
  return ((3 * (size_t)N * sg_stride(N) * tsz + 3 * 4 * kSgMaxN * sizeof(int)) + 255) & ~(size_t)255;
}

template <typename T> struct Quad;
template <> struct Quad<float> {
  static __device__ __forceinline__ void load(const float2 *p, float2 (&v)[4]) {
    const float4 u = *reinterpret_cast<const float4 *>(p), w = *reinterpret_cast<const float4 *>(p + 2);
    v[0] = make_float2(u.x, u.y);
    v[1] = make_float2(u.z, u.w);
    v[2] = make_float2(w.x, w.y);
    v[3] = make_float2(w.z, w.w);
  }
};
template <> struct Quad<double> {
  static __device__ __forceinline__ void load(const double2 *p, double2 (&v)[4]) {
    for (int e = 0; e < 4; e++) v[e] = p[e];
  }
};

// The operators of one step, once per (component, point): own operator A_q (off-diagonal
// H plus the pulses on for component q), P2 and P3 (the source operators), padded to
// rows of S, and for each the range [lo, hi) of nonzero entries of every row and
// column (lo = 32767, hi = 0 when empty).  Rows and columns outside the ranges hold
// exact zeros, so the stage kernel's commutator loops skip them without changing any
// partial sum.
template <typename T>
__global__ void __launch_bounds__(256) sg_ops(SgArgs a, int step_local, const int *__restrict__ base) {
  using T2 = typename Vec2<T>::t;
  const int cq = blockIdx.x, p = blockIdx.y;
  const int i = *base + step_local;
  if (i >= a.nsteps[p]) return;
  const int N = a.N, NN = N * N, S = sg_stride(N), NS = N * S;
  const int tid = threadIdx.x, bs = blockDim.x;
  extern __shared__ __align__(16) unsigned char smraw[];
  T2 *Om = (T2 *)smraw;
  unsigned char *gb = a.ops + (size_t)(p * a.C + cq) * a.ops_stride;
  T2 *Og = (T2 *)gb;
  int *Rg = (int *)(gb + 3 * (size_t)NS * sizeof(T2));
  const size_t si = (size_t)p * a.S_max + i;
  const unsigned f = a.flags[si];
  int on[3];
  double2 ef[3];
  for (int q = 0; q < 3; q++) {
    on[q] = (f >> q) & 1;
    if (a.C == 1) on[q] = on[q] && a.mask[q];
    ef[q] = a.field[si * 3 + q];
  }
  const T2 zero = to2<T>(0.0, 0.0);
  for (int t = tid; t < NS; t += bs) {
    const int r = t / S, c = t - r * S;
    T2 own = zero, p2 = zero, p3 = zero;
    if (c < N) {
      const int e = r * N + c;
      double vr[3], vi[3];
      for (int q = 0; q < 3; q++) {
        const double2 x = a.Xs[q * NN + e];
        vr[q] = on[q] ? -(x.x * ef[q].x - x.y * ef[q].y) : 0.0;
        vi[q] = on[q] ? -(x.x * ef[q].y + x.y * ef[q].x) : 0.0;
      }
      const double br = a.Hoff[e].x + vr[0], bi = a.Hoff[e].y + vi[0];
      if (a.C == 1 || cq == 3) own = to2<T>(br + vr[1] + vr[2], bi + vi[1] + vi[2]);
      else if (cq == 1) own = to2<T>(br + vr[1], bi + vi[1]);
      else if (cq == 2) own = to2<T>(br + vr[2], bi + vi[2]);
      else own = to2<T>(br, bi);
      p2 = to2<T>(vr[1], vi[1]);
      p3 = to2<T>(vr[2], vi[2]);
    }
    Om[t] = own;
    Om[NS + t] = p2;
    Om[2 * NS + t] = p3;
    Og[t] = own;
    Og[NS + t] = p2;
    Og[2 * NS + t] = p3;
  }
  __syncthreads();
  for (int t = tid; t < 3 * 2 * kSgMaxN; t += bs) {
    const int o = t / (2 * kSgMaxN), kind = (t / kSgMaxN) & 1, j = t % kSgMaxN;
    int lo = 32767, hi = 0;
    if (j < N)
      for (int l = 0; l < N; l++) {
        const T2 v = kind == 0 ? Om[o * NS + j * S + l] : Om[o * NS + l * S + j];
        if (v.x != (T)0 || v.y != (T)0) {
          lo = min(lo, l);
          hi = l + 1;
        }
      }
    Rg[(o * 4 + 2 * kind) * kSgMaxN + j] = lo;
    Rg[(o * 4 + 2 * kind + 1) * kSgMaxN + j] = hi;
  }
}

// One Horner stage over (ADO tile, component, point).  Phase 1: each thread forms the
// commutator -- own operator plus sources, operators from sg_ops -- of a 1 x 4 strip
// (r, c0..c0+3) of one ADO block from shared memory, over the nonzero rows/columns of
// each operator only.  Phase 2: element-per-thread (coalesced) bath couplings, FP64
// diagonal and damping, and the Horner update.
// Phase-1 products for precision studies of a tensor-core commutator (FP32 state copies):
// TF = 0: FP32 products; TF = 1: both factors rounded to TF32 (cvt.rna.tf32.f32) first,
// the product exact in FP32 and accumulated in FP32, as one TF32 tensor-core MMA does;
// TF = 3: the 3xTF32 split a = a_hi + a_lo, z = z_hi + z_lo, accumulating
// a_lo z_hi + a_hi z_lo + a_hi z_hi (a_lo z_lo dropped).
__device__ __forceinline__ float tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
template <typename T, int TF> __device__ __forceinline__ T sg_mac(T acc, T a, T z) {
  if constexpr (TF == 0 || sizeof(T) != 4) {
    return fma(a, z, acc);
  } else if constexpr (TF == 1) {
    return fma(tf32_rna(a), tf32_rna(z), acc);
  } else {
    const float ah = tf32_rna(a), al = tf32_rna(a - ah), zh = tf32_rna(z), zl = tf32_rna(z - zh);
    acc = fma(al, zh, acc);
    acc = fma(ah, zl, acc);
    return fma(ah, zh, acc);
  }
}

template <typename T, int TF = 0>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) sg_stage(SgArgs a, int m, int step_local, const int *__restrict__ base) {
  using T2 = typename Vec2<T>::t;
  const int p = blockIdx.z, cq = blockIdx.y;
  const int i = *base + step_local;
  if (i >= a.nsteps[p]) return;
  const int N = a.N, NN = N * N, nado = a.n_ado, M = a.M, K = a.K, Km = a.Km;
  const int S = sg_stride(N), NS = N * S, spr = sg_np(N) / 4;
  const int tid = threadIdx.x, bs = blockDim.x;
  const int apc = a.apc;
  extern __shared__ __align__(16) unsigned char smraw[];
  T2 *Am = (T2 *)smraw;         // [3][N][S]: own operator, P2, P3
  T2 *Wm = Am + 3 * NS;         // [3][apc][N][S]: own blocks, first and second source blocks
  T2 *Xm = Wm + 3 * apc * NS;   // [apc][N][N]: commutator
  const int g = 4 * i + (4 - m);   // global stage index: buffers alternate every stage
  const double2 *w64_in = (g & 1) ? a.w64b : a.w64a;
  double2 *w64_out = (g & 1) ? a.w64a : a.w64b;
  const T2 *w32_in = (const T2 *)((g & 1) ? a.w32b : a.w32a);
  T2 *w32_out = (T2 *)((g & 1) ? a.w32a : a.w32b);
  const size_t pb = (size_t)p * a.E_pt;
  const size_t si = (size_t)p * a.S_max + i;
  const unsigned f = a.flags[si];
  int on[3];
  for (int q = 0; q < 3; q++) on[q] = (f >> q) & 1;
  // mixed-difference sources of this component: D2 <- P2 R, D3 <- P3 R, Q <- P2 D3 + P3 D2
  // (operator index in Am, source component) of source 1 and source 2
  int nsrc = 0, op1 = 0, from1 = 0, op2 = 0, from2 = 0;
  if (a.C == 4) {
    if (cq == 1 && on[1]) { op1 = 1; from1 = 0; nsrc = 1; }
    if (cq == 2 && on[2]) { op1 = 2; from1 = 0; nsrc = 1; }
    if (cq == 3) {
      if (on[1]) { op1 = 1; from1 = 2; nsrc = 1; }
      if (on[2]) {
        if (nsrc == 0) { op1 = 2; from1 = 1; }
        else { op2 = 2; from2 = 1; }
        nsrc++;
      }
    }
  }
  const T2 zero = to2<T>(0.0, 0.0);
  __shared__ int s_rng[3 * 4 * kSgMaxN];
  {
    const unsigned char *gb = a.ops + (size_t)(p * a.C + cq) * a.ops_stride;
    const int *Rg = (const int *)(gb + 3 * (size_t)NS * sizeof(T2));
    for (int t = tid; t < 3 * 4 * kSgMaxN; t += bs) s_rng[t] = Rg[t];
    const int nv = NS * (int)sizeof(T2) / 16; // 16-byte vectors per operator
    for (int b = 0; b <= nsrc; b++) {
      const int o = b == 0 ? 0 : b == 1 ? op1 : op2;
      const uint4 *src = (const uint4 *)(gb + (size_t)o * NS * sizeof(T2));
      uint4 *dst = (uint4 *)(Am + (size_t)o * NS);
      for (int t = tid; t < nv; t += bs) dst[t] = src[t];
    }
  }
  const int n0 = blockIdx.x * apc;
  for (int b = 0; b <= nsrc; b++) {
    const int comp = b == 0 ? cq : b == 1 ? from1 : from2;
    T2 *Wb = Wm + (size_t)b * apc * NS;
    for (int t = tid; t < apc * NS; t += bs) {
      const int nl = t / NS, rc = t - nl * NS, r = rc / S, c = rc - r * S;
      const int n = n0 + nl;
      Wb[t] = (n < nado && c < N) ? w32_in[pb + (size_t)(comp * nado + n) * NN + r * N + c] : zero;
    }
  }
  __syncthreads();
  // P before the step, from the FP64 state of ADO 0 (first stage of the step only)
  if (m == 4 && cq == 0 && blockIdx.x == 0) {
    const int rec = a.rec[si];
    if (rec >= 0 && tid < 32) {
      double sr = 0.0, sim = 0.0;
      for (int t = tid; t < NN; t += 32) {
        const int jr = t / N, l = t - jr * N;
        double2 v = a.rho[pb + t];
        if (a.C == 4) {
          const double2 qv = a.rho[pb + (size_t)3 * nado * NN + t];
          v = make_double2(qv.x - v.x, qv.y - v.y);
        }
        const double2 x = a.X3[l * N + jr];
        sr += v.x * x.x - v.y * x.y;
        sim += v.x * x.y + v.y * x.x;
      }
      for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_down_sync(0xffffffffu, sr, o);
        sim += __shfl_down_sync(0xffffffffu, sim, o);
      }
      if (tid == 0) a.P[a.offsets[p] + rec] = make_double2(sr, sim);
    }
  }
  // phase 1: X = sum over (operator O, block Z) of O Z - Z O, one 1 x 4 strip per slot
  const int per_ado = sg_slots_per_ado(N);
  const int cg = (spr + 3) / 4;
  for (int s = tid; s < apc * per_ado; s += bs) {
    const int nl = s / per_ado, u = s - nl * per_ado;
    int r, cs;
    if (spr <= 4) {
      r = u / spr;
      cs = u - r * spr;
    } else {
      const int tile = u >> 5, lane = u & 31;
      r = (tile / cg) * 8 + (lane >> 2);
      cs = (tile % cg) * 4 + (lane & 3);
      if (r >= N || cs >= spr) continue;
    }
    const int c0 = 4 * cs;
    T xr[4] = {0, 0, 0, 0}, xi[4] = {0, 0, 0, 0};
    for (int b = 0; b <= nsrc; b++) {
      const int o = b == 0 ? 0 : b == 1 ? op1 : op2;
      const T2 *Ab = Am + o * NS;
      const T2 *Wb = Wm + ((size_t)b * apc + nl) * NS;
      const int *rg = s_rng + o * 4 * kSgMaxN;
      // A W: the nonzero entries of row r of A
      for (int l = rg[r], le = rg[kSgMaxN + r]; l < le; l++) {
        const T2 a1 = Ab[r * S + l];
        T2 z1[4];
        Quad<T>::load(Wb + l * S + c0, z1);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          xr[e] = sg_mac<T, TF>(xr[e], a1.x, z1[e].x);
          xr[e] = sg_mac<T, TF>(xr[e], -a1.y, z1[e].y);
          xi[e] = sg_mac<T, TF>(xi[e], a1.x, z1[e].y);
          xi[e] = sg_mac<T, TF>(xi[e], a1.y, z1[e].x);
        }
      }
      // - W A: the nonzero entries of columns c0..c0+3 of A
      int lo = rg[2 * kSgMaxN + c0], hi = rg[3 * kSgMaxN + c0];
#pragma unroll
      for (int e = 1; e < 4; e++) {
        lo = min(lo, rg[2 * kSgMaxN + c0 + e]);
        hi = max(hi, rg[3 * kSgMaxN + c0 + e]);
      }
      for (int l = lo; l < hi; l++) {
        const T2 z2 = Wb[r * S + l];
        T2 a2[4];
        Quad<T>::load(Ab + l * S + c0, a2);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          xr[e] = sg_mac<T, TF>(xr[e], -z2.x, a2[e].x);
          xr[e] = sg_mac<T, TF>(xr[e], z2.y, a2[e].y);
          xi[e] = sg_mac<T, TF>(xi[e], -z2.x, a2[e].y);
          xi[e] = sg_mac<T, TF>(xi[e], -z2.y, a2[e].x);
        }
      }
    }
    T2 *Xr = Xm + (size_t)nl * NN + r * N;
#pragma unroll
    for (int e = 0; e < 4; e++)
      if (c0 + e < N) {
        T2 v;
        v.x = xr[e];
        v.y = xi[e];
        Xr[c0 + e] = v;
      }
  }
  __syncthreads();
  // phase 2: k = -i X + bath couplings + FP64 diagonal/damping; Horner update
  const double cm = a.h / m;
  for (int t = tid; t < apc * NN; t += bs) {
    const int nl = t / NN, n = n0 + nl;
    if (n >= nado) continue;
    const int rc = t - nl * NN, r = rc / N, c = rc - r * N;
    const T2 x = Xm[t];
    T kr = x.y, ki = -x.x; // -i X
    for (int pass = 0; pass < 2; pass++) {
      const int s = pass == 0 ? r : c;
      if (s < 1 || s > K || (pass == 1 && c == r)) continue;
      const int j = s - 1, dr = (r == s), dc = (c == s);
      for (int k = 0; k < Km; k++) {
        const int o = n * M + j + k * K;
        const int u = a.up[o], d = a.dn[o];
        if (u >= 0 && dr != dc) {
          const T xx = (T)a.xc[o] * (T)(dc - dr);
          const T2 z = w32_in[pb + (size_t)(cq * nado + u) * NN + rc];
          kr = fma(xx, z.y, kr);
          ki = fma(-xx, z.x, ki);
        }
        if (d >= 0) {
          const T y = (T)a.yc[o];
          const double2 al = a.alpha[k];
          const T cr = -(T)al.y * (T)(dr + dc) * y, ci = (T)al.x * (T)(dr - dc) * y;
          const T2 z = w32_in[pb + (size_t)(cq * nado + d) * NN + rc];
          kr = fma(cr, z.x, fma(-ci, z.y, kr));
          ki = fma(cr, z.y, fma(ci, z.x, ki));
        }
      }
    }
    const size_t idx = pb + (size_t)(cq * nado + n) * NN + rc;
    const double2 wv = w64_in[idx], dmp = a.damp[n];
    const double gr = dmp.x, gi = dmp.y - (a.Hd[r] - a.Hd[c]);
    const double k_r = fma(gr, wv.x, fma(-gi, wv.y, (double)kr));
    const double k_i = fma(gr, wv.y, fma(gi, wv.x, (double)ki));
    const double2 r0 = a.rho[idx];
    const double2 wn = make_double2(fma(cm, k_r, r0.x), fma(cm, k_i, r0.y));
    w64_out[idx] = wn;
    if (!std::is_same<T, double>::value) w32_out[idx] = to2<T>(wn.x, wn.y);
    if (m == 1) a.rho[idx] = wn;
  }
}

template <typename T> __global__ void sg_init_state(SgArgs a, long long total) {
  using T2 = typename Vec2<T>::t;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const double v = (e % a.E_pt) == 0 ? 1.0 : 0.0; // R = |0><0| on ADO 0 of every point
    a.rho[e] = make_double2(v, 0.0);
    a.w64a[e] = make_double2(v, 0.0);
    if (!std::is_same<T, double>::value) ((T2 *)a.w32a)[e] = to2<T>(v, 0.0);
  }
}

__global__ void sg_bump(int *base, int by) { *base += by; }

// ------------------------------------------------------------------ host
namespace {


int fail(int code, const std::string &m) {
  sg_err = m;
  return code;
}
#define SGCK(call)                                                                      \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) return fail(HEOM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

} // namespace

int sg_init(SgState &s, const heom::Problem &p, int precision, cudaStream_t st) {
  s = SgState();
  s.precision = precision == HEOM_FP64_EXACT ? HEOM_FP64 : precision;
  s.N = p.N();
  s.n_ado = p.n_ado;
  s.M = p.M;
  s.K = p.K;
  s.K_m = p.K_m;
  s.t_start = p.t_start;
  s.dt = p.step_size;
  s.stride = p.print_stride();
  s.h = (double)p.step_size;
  const int NN = s.N * s.N;
  // about 256 strip slots per CTA (one ADO for N > 16), at most 256 threads
  const int slots = sg_slots_per_ado(s.N);
  s.apc = std::max(1, 256 / slots);
  s.threads = std::min(256, ((s.apc * slots + 31) / 32) * 32);
  const size_t tsz = s.precision == HEOM_FP64 ? 16 : 8;
  s.smem = tsz * sg_smem_elems(s.N, s.apc);
  int max_smem = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (NN > 1024 || s.smem > (size_t)max_smem) return fail(HEOM_ERR_UNSUPPORTED, "system too large for the staged path");
  SGCK(cudaFuncSetAttribute(sg_stage<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem));
  // precision study of a tensor-core commutator: HEOM_SG_CONTRACTION=tf32 | tf32x3 rounds
  // the FP32-bulk phase-1 products as TF32 MMAs would (see sg_mac)
  if (const char *v = std::getenv("HEOM_SG_CONTRACTION")) {
    if (!std::strcmp(v, "tf32")) s.tf = 1;
    else if (!std::strcmp(v, "tf32x3")) s.tf = 3;
    else if (std::strcmp(v, "fp32")) return fail(HEOM_ERR_ARG, std::string("HEOM_SG_CONTRACTION: unknown value ") + v);
  }
  SGCK(cudaFuncSetAttribute(sg_stage<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem));
  SGCK(cudaFuncSetAttribute(sg_stage<float, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem));
  SGCK(cudaFuncSetAttribute(sg_stage<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem));
  const int ops_smem = (int)(3 * (size_t)s.N * sg_stride(s.N) * tsz);
  SGCK(cudaFuncSetAttribute(sg_ops<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, ops_smem));
  SGCK(cudaFuncSetAttribute(sg_ops<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ops_smem));
  SgTab tl(s.N, s.n_ado, s.M, s.K_m);
  s.tab_bytes = tl.total;
  SGCK(cudaMalloc(&s.d_tab, tl.total));
  SGCK(cudaMalloc(&s.d_base, sizeof(int) * 4));
  std::vector<unsigned char> tb(tl.total, 0);
  const size_t nM = (size_t)p.n_ado * p.M;
  double *xc = (double *)(tb.data() + tl.xc), *yc = (double *)(tb.data() + tl.yc);
  int *up = (int *)(tb.data() + tl.up), *dn = (int *)(tb.data() + tl.dn);
  for (size_t q = 0; q < nM; q++) {
    const int n = (int)(q / p.M), o = (int)(q % p.M);
    up[q] = p.up[q];
    dn[q] = p.dn[q];
    xc[q] = heom::coupling_x(p, n, o);
    yc[q] = heom::coupling_y(p, n, o);
  }
  std::memcpy(tb.data() + tl.damp, p.damp.data(), sizeof(double) * 2 * p.n_ado);
  std::memcpy(tb.data() + tl.alpha, p.alpha.data(), sizeof(double) * 2 * p.K_m);
  SGCK(cudaMemcpy(s.d_tab, tb.data(), tl.total, cudaMemcpyHostToDevice));
  return sg_upload_system(s, p, st);
}

int sg_upload_system(SgState &s, const heom::Problem &p, cudaStream_t st) {
  const int N = s.N, NN = N * N;
  SgTab tl(s.N, s.n_ado, s.M, s.K_m);
  std::vector<double> hd(N), hoff(2 * NN, 0.0), xs(6 * NN), x3(2 * NN);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      const size_t t = (size_t)i * N + j, tt = (size_t)j * N + i;
      if (i == j) {
        hd[i] = p.H[2 * t];
        hoff[2 * t + 1] = p.H[2 * t + 1];
      } else {
        hoff[2 * t] = p.H[2 * t];
        hoff[2 * t + 1] = p.H[2 * t + 1];
      }
      xs[2 * t] = p.X[0][2 * t];
      xs[2 * t + 1] = p.X[0][2 * t + 1];
      xs[2 * (NN + t)] = p.X[1][2 * tt];
      xs[2 * (NN + t) + 1] = p.X[1][2 * tt + 1];
      xs[2 * (2 * NN + t)] = p.X[2][2 * tt];
      xs[2 * (2 * NN + t) + 1] = p.X[2][2 * tt + 1];
      x3[2 * t] = p.X[3][2 * t];
      x3[2 * t + 1] = p.X[3][2 * t + 1];
    }
  unsigned char *b = (unsigned char *)s.d_tab;
  SGCK(cudaMemcpyAsync(b + tl.Hd, hd.data(), 8 * hd.size(), cudaMemcpyHostToDevice, st));
  SGCK(cudaMemcpyAsync(b + tl.Hoff, hoff.data(), 8 * hoff.size(), cudaMemcpyHostToDevice, st));
  SGCK(cudaMemcpyAsync(b + tl.Xs, xs.data(), 8 * xs.size(), cudaMemcpyHostToDevice, st));
  SGCK(cudaMemcpyAsync(b + tl.X3, x3.data(), 8 * x3.size(), cudaMemcpyHostToDevice, st));
  SGCK(cudaStreamSynchronize(st));
  return HEOM_OK;
}

int sg_run(SgState &s, const heom::Problem &p, int C, const int mask[3], const heom_scan_point *pts, int n,
           double *P, const long long *offsets, long long total, cudaStream_t st) {
  if (n <= 0) return HEOM_OK;
  const int NN = s.N * s.N;
  // host schedules: float time, gating and glibc field factors as in dynamics.cpp:344-367
  std::vector<int> nsteps(n);
  int S_max = 0;
  for (int q = 0; q < n; q++) {
    nsteps[q] = heom::steps_for(p, pts[q].t_end);
    S_max = std::max(S_max, nsteps[q]);
  }
  S_max = std::max(S_max, 1);
  const size_t NS = (size_t)n * S_max;
  std::vector<unsigned char> flags(NS, 0);
  std::vector<int> rec(NS, -1);
  std::vector<double> field(2 * 3 * NS, 0.0);
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
  const size_t off_flags = 0, off_rec = a256(off_flags + NS), off_field = a256(off_rec + 4 * NS);
  const size_t off_ns = a256(off_field + 48 * NS), off_off = a256(off_ns + 4 * (size_t)n);
  const size_t sched_bytes = a256(off_off + 8 * (size_t)n);
  if (sched_bytes > s.sched_bytes) {
    if (s.d_sched) cudaFree(s.d_sched);
    s.d_sched = nullptr;
    s.sched_bytes = 0;
    SGCK(cudaMalloc(&s.d_sched, sched_bytes));
    s.sched_bytes = sched_bytes;
  }
  unsigned char *sb = (unsigned char *)s.d_sched;
  SGCK(cudaMemcpyAsync(sb + off_flags, flags.data(), NS, cudaMemcpyHostToDevice, st));
  SGCK(cudaMemcpyAsync(sb + off_rec, rec.data(), 4 * NS, cudaMemcpyHostToDevice, st));
  SGCK(cudaMemcpyAsync(sb + off_field, field.data(), 48 * NS, cudaMemcpyHostToDevice, st));
  SGCK(cudaMemcpyAsync(sb + off_ns, nsteps.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, st));
  SGCK(cudaMemcpyAsync(sb + off_off, offsets, 8 * (size_t)n, cudaMemcpyHostToDevice, st));
  // state
  const int E_pt = C * s.n_ado * NN;
  const long long E = (long long)n * E_pt;
  const bool d = s.precision == HEOM_FP64;
  // rho and the FP64 iterate w64 (16 B each), plus: FP64 path -- a second w64 buffer,
  // read by neighbours while the other is written; FP32-bulk -- two FP32 copies for the
  // neighbours and shared blocks, w64 then being read and written only by its own
  // element's thread, in place.
  const size_t state_bytes = a256(16 * E) * (d ? 3 : 2) + (d ? 0 : a256(8 * E) * 2);
  if (state_bytes > s.state_bytes) {
    if (s.d_state) cudaFree(s.d_state);
    s.d_state = nullptr;
    s.state_bytes = 0;
    cudaError_t e = cudaMalloc(&s.d_state, state_bytes);
    if (e != cudaSuccess) return fail(HEOM_ERR_NOMEM, "staged path state: out of device memory");
    s.state_bytes = state_bytes;
  }
  const size_t ops_stride = sg_ops_bytes(s.N, d ? 16 : 8);
  const size_t ops_bytes = ops_stride * (size_t)n * C;
  if (ops_bytes > s.ops_bytes) {
    if (s.d_ops) cudaFree(s.d_ops);
    s.d_ops = nullptr;
    s.ops_bytes = 0;
    SGCK(cudaMalloc(&s.d_ops, ops_bytes));
    s.ops_bytes = ops_bytes;
  }
  if (total > s.P_cap || !s.d_P) { // allocated even when nothing is recorded
    if (s.d_P) cudaFree(s.d_P);
    s.d_P = nullptr;
    s.P_cap = 0;
    SGCK(cudaMalloc(&s.d_P, sizeof(double2) * std::max<long long>(total, 1)));
    s.P_cap = total;
  }
  SgTab tl(s.N, s.n_ado, s.M, s.K_m);
  unsigned char *tb = (unsigned char *)s.d_tab, *stb = (unsigned char *)s.d_state;
  SgArgs a{};
  a.N = s.N;
  a.n_ado = s.n_ado;
  a.M = s.M;
  a.K = s.K;
  a.Km = s.K_m;
  a.C = C;
  a.E_pt = E_pt;
  a.S_max = S_max;
  a.apc = s.apc;
  for (int q = 0; q < 3; q++) a.mask[q] = mask ? mask[q] : 1;
  a.h = s.h;
  a.Hd = (const double *)(tb + tl.Hd);
  a.Hoff = (const double2 *)(tb + tl.Hoff);
  a.Xs = (const double2 *)(tb + tl.Xs);
  a.X3 = (const double2 *)(tb + tl.X3);
  a.damp = (const double2 *)(tb + tl.damp);
  a.alpha = (const double2 *)(tb + tl.alpha);
  a.xc = (const double *)(tb + tl.xc);
  a.yc = (const double *)(tb + tl.yc);
  a.up = (const int *)(tb + tl.up);
  a.dn = (const int *)(tb + tl.dn);
  a.flags = sb + off_flags;
  a.rec = (const int *)(sb + off_rec);
  a.field = (const double2 *)(sb + off_field);
  a.nsteps = (const int *)(sb + off_ns);
  a.offsets = (const long long *)(sb + off_off);
  a.rho = (double2 *)stb;
  a.w64a = (double2 *)(stb + a256(16 * E));
  a.w64b = d ? (double2 *)(stb + 2 * a256(16 * E)) : a.w64a;
  a.w32a = d ? (void *)a.w64a : (void *)(stb + 2 * a256(16 * E));
  a.w32b = d ? (void *)a.w64b : (void *)(stb + 2 * a256(16 * E) + a256(8 * E));
  a.P = s.d_P;
  a.ops = (unsigned char *)s.d_ops;
  a.ops_stride = (long long)ops_stride;
  SGCK(cudaMemsetAsync(s.d_P, 0, sizeof(double2) * std::max<long long>(total, 1), st));
  if (d) sg_init_state<double><<<1024, 256, 0, st>>>(a, E);
  else sg_init_state<float><<<1024, 256, 0, st>>>(a, E);
  SGCK(cudaMemsetAsync(s.d_base, 0, sizeof(int), st));
  s.launches += 1;
  // Graph of one chunk of steps (the stage launches read the step index from *d_base).
  // Its arguments (buffer offsets, masks, batch shape) belong to this run, so it is
  // built per run and replayed S_max / chunk times.
  if (s.gexec) { cudaGraphExecDestroy(s.gexec); s.gexec = nullptr; }
  cudaGraph_t graph;
  SGCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  dim3 grid((s.n_ado + s.apc - 1) / s.apc, C, n);
  const dim3 ogrid(C, n);
  const size_t osmem = 3 * (size_t)s.N * sg_stride(s.N) * (d ? 16 : 8);
  for (int k = 0; k < s.g_chunk; k++) {
    if (d) sg_ops<double><<<ogrid, 256, osmem, st>>>(a, k, s.d_base);
    else sg_ops<float><<<ogrid, 256, osmem, st>>>(a, k, s.d_base);
    for (int m = 4; m >= 1; m--) {
      if (d) sg_stage<double><<<grid, s.threads, s.smem, st>>>(a, m, k, s.d_base);
      else if (s.tf == 1) sg_stage<float, 1><<<grid, s.threads, s.smem, st>>>(a, m, k, s.d_base);
      else if (s.tf == 3) sg_stage<float, 3><<<grid, s.threads, s.smem, st>>>(a, m, k, s.d_base);
      else sg_stage<float><<<grid, s.threads, s.smem, st>>>(a, m, k, s.d_base);
    }
  }
  sg_bump<<<1, 1, 0, st>>>(s.d_base, s.g_chunk);
  cudaError_t le = cudaGetLastError();
  cudaError_t ce = cudaStreamEndCapture(st, &graph);
  if (le != cudaSuccess) return fail(HEOM_ERR_CUDA, std::string("capture staged chunk: ") + cudaGetErrorString(le));
  if (ce != cudaSuccess) return fail(HEOM_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ce));
  cudaError_t ie = cudaGraphInstantiate(&s.gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) return fail(HEOM_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ie));
  const int reps = (S_max + s.g_chunk - 1) / s.g_chunk;
  for (int r = 0; r < reps; r++) SGCK(cudaGraphLaunch(s.gexec, st));
  s.launches += (long long)reps * (5LL * s.g_chunk + 1);
  if (total > 0) SGCK(cudaMemcpyAsync(P, s.d_P, sizeof(double2) * total, cudaMemcpyDeviceToHost, st));
  SGCK(cudaStreamSynchronize(st));
  for (long long q = 0; q < 2 * total; q++)
    if (!std::isfinite(P[q])) return fail(HEOM_ERR_NUMERIC, "non-finite P(t): the propagation diverged");
  return HEOM_OK;
}

void sg_release(SgState &s) {
  if (s.gexec) cudaGraphExecDestroy(s.gexec);
  if (s.d_tab) cudaFree(s.d_tab);
  if (s.d_state) cudaFree(s.d_state);
  if (s.d_sched) cudaFree(s.d_sched);
  if (s.d_P) cudaFree(s.d_P);
  if (s.d_ops) cudaFree(s.d_ops);
  if (s.d_base) cudaFree(s.d_base);
  s = SgState();
}

} // namespace heom_dev
