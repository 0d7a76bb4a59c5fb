// Bit-exact FP64 trajectory kernels (HEOM_FP64_EXACT).
//
// Replace twoD_spectrum_solver + total_ADO_dynamics_Ht (etoheom-cpu/lib/dynamics.cpp:
// 117-200, 298-432; GPU: etoheom-gpu/lib/HEOM_dynamics.cu:190-287, 489-658).  The RK4
// stage sequence is the reference's in-place one:
//   k1 = F(rho);  rho += h/2 k1
//   k2 = F(rho);  rho -= h/2 k1;  rho += h/2 k2
//   k3 = F(rho);  rho -= h/2 k2;  rho += h k3
//   k4 = F(rho);  rho -= h k3;    rho += h b0 k1; += h b1 k2; += h b2 k3; += h b3 k4
// with V = H - sum_q e_q(t) X_q frozen over the four stages, and P = Tr(rho_0 X3)
// recorded before the step.  Each element's update only reads that element, so the
// "rho" of consecutive stages ping-pongs between two buffers (A at step start, B
// after stages 1 and 3) and one barrier per stage suffices.
//
// Two launch forms:
//  * exact_traj_smem: one CTA owns one trajectory for all its steps, with the state
//    (A, B, k1, k2, k3) resident in shared memory; for small hierarchies.
//  * exact_stage: one launch per RK4 stage over all ADOs of all trajectories, state in
//    global memory (L2-resident), replayed from a CUDA graph in chunks of steps
//    (exact_stage_wide for blocks whose tiles do not fit in shared memory).
#include <cuda_runtime.h>
#include <cstdint>

#include "exact.cuh"
#include "kernels.h"

namespace heom_dev {

__global__ void __launch_bounds__(512) exact_traj_smem(ExactArgs a, const ExactTraj *__restrict__ trajs) {
  extern __shared__ double2 sm[];
  const ExactTraj tj = trajs[blockIdx.x];
  const int N = a.N, nn = N * N, tot = a.n_ado * nn;
  double2 *A = sm, *B = A + tot, *K1 = B + tot, *K2 = K1 + tot, *K3 = K2 + tot;
  double2 *V = K3 + tot, *Pt = V + nn;
  const int tid = threadIdx.x, bs = blockDim.x;
  for (int e = tid; e < tot; e += bs) A[e] = make_double2(e == 0 ? 1.0 : 0.0, 0.0); // reset_rho

  for (int i = 0; i < tj.n_steps; i++) {
    const unsigned f = tj.flags[i];
    double2 ef[3];
    for (int q = 0; q < 3; q++) ef[q] = tj.field[(size_t)q * tj.n_steps + i];
    for (int t = tid; t < nn; t += bs) V[t] = build_v(a.H, a.Xs, nn, t, f, ef);
    __syncthreads();
    const int rec = tj.rec_idx[i];
    if (rec >= 0) {
      for (int j = tid; j < N; j += bs) Pt[j] = trace_row_exact(A, tj.X3 ? tj.X3 : a.X3, N, j);
      __syncthreads();
      if (tid == 0) {
        double tr = 0.0, ti = 0.0;
        for (int j = 0; j < N; j++) { tr = __dadd_rn(tr, Pt[j].x); ti = __dadd_rn(ti, Pt[j].y); }
        tj.P[rec] = make_double2(tr, ti);
      }
    }
    // stage 1
    for (int e = tid; e < tot; e += bs) {
      const int n = e / nn, rc = e - n * nn, r = rc / N, c = rc - r * N;
      const double2 k = rhs_exact(A, A + (size_t)n * nn, V, N, n, r, c, a.damp[n], a.ops, a.op_start[n], a.op_start[n + 1]);
      K1[e] = k;
      B[e] = axpy_exact(A[e], a.h2, k);
    }
    __syncthreads();
    // stage 2
    for (int e = tid; e < tot; e += bs) {
      const int n = e / nn, rc = e - n * nn, r = rc / N, c = rc - r * N;
      const double2 k = rhs_exact(B, B + (size_t)n * nn, V, N, n, r, c, a.damp[n], a.ops, a.op_start[n], a.op_start[n + 1]);
      K2[e] = k;
      A[e] = axpy_exact(axpy_exact(B[e], -a.h2, K1[e]), a.h2, k);
    }
    __syncthreads();
    // stage 3
    for (int e = tid; e < tot; e += bs) {
      const int n = e / nn, rc = e - n * nn, r = rc / N, c = rc - r * N;
      const double2 k = rhs_exact(A, A + (size_t)n * nn, V, N, n, r, c, a.damp[n], a.ops, a.op_start[n], a.op_start[n + 1]);
      K3[e] = k;
      B[e] = axpy_exact(axpy_exact(A[e], -a.h2, K2[e]), a.h, k);
    }
    __syncthreads();
    // stage 4 and the final combination
    for (int e = tid; e < tot; e += bs) {
      const int n = e / nn, rc = e - n * nn, r = rc / N, c = rc - r * N;
      const double2 k = rhs_exact(B, B + (size_t)n * nn, V, N, n, r, c, a.damp[n], a.ops, a.op_start[n], a.op_start[n + 1]);
      double2 y = axpy_exact(B[e], -a.h, K3[e]);
      y = axpy_exact(y, a.hb[0], K1[e]);
      y = axpy_exact(y, a.hb[1], K2[e]);
      y = axpy_exact(y, a.hb[2], K3[e]);
      A[e] = axpy_exact(y, a.hb[3], k);
    }
    __syncthreads();
  }
  if (tj.final_state)
    for (int e = tid; e < tot; e += bs) tj.final_state[e] = A[e];
}

// Shared-memory rows of exact_stage are padded to S = Np + 1 (Np = N rounded up to 4):
// the rows a warp reads at one column then fall in distinct banks.  A thread owns a
// tile of 1 row x 4 columns, the columns strided by Np/4, so that the Np/4 lanes of a
// row read consecutive elements.
constexpr int kExTileMaxN = 96; // row-trace buffer of exact_stage; wider blocks take exact_stage_wide
__host__ __device__ inline int ex_np(int N) { return (N + 3) & ~3; }
__host__ __device__ inline int ex_stride(int N) { return ex_np(N) + 1; }
__host__ __device__ inline int ex_tiles(int N) { return N * (ex_np(N) / 4); }
__host__ __device__ inline int ex_apc(int N) { return ex_tiles(N) >= 256 ? 1 : 256 / ex_tiles(N); }
__host__ __device__ inline size_t ex_smem_elems(int N, int apc) {
  return (size_t)(1 + apc) * N * ex_stride(N) + (size_t)apc * N * N;
}

// One RK4 stage of every trajectory: block (tile of apc ADOs, trajectory).  V and the
// ADOs' own blocks are staged in shared memory.  Phase 1 forms, per element, the two
// zgemm sums and the damping term in the reference's order (a 1 x 4 element tile per
// thread); phase 2 adds the neighbour terms (read from L2) and applies the stage update,
// one element per thread.
__global__ void __launch_bounds__(256, 4) exact_stage(ExactArgs a, const ExactTraj *__restrict__ trajs, int stage,
                                                   int step_local, const int *__restrict__ base) {
  extern __shared__ double2 sm[];
  const ExactTraj tj = trajs[blockIdx.y];
  const int i = *base + step_local;
  if (i >= tj.n_steps) return;
  const int N = a.N, nn = N * N, tot = a.n_ado * nn, nado = a.n_ado;
  const int S = ex_stride(N), NS = N * S, q4 = ex_np(N) / 4, tiles = ex_tiles(N), apc = ex_apc(N);
  const int n0 = blockIdx.x * apc, tid = threadIdx.x, bs = blockDim.x;
  double2 *A = tj.work, *B = A + tot, *K1 = B + tot, *K2 = K1 + tot, *K3 = K2 + tot;
  const double2 *src = (stage == 1 || stage == 3) ? A : B;
  double2 *V = sm, *own = sm + NS, *X = own + (size_t)apc * NS;
  __shared__ double2 Pt[kExTileMaxN];
  const unsigned f = tj.flags[i];
  double2 ef[3];
  for (int q = 0; q < 3; q++) ef[q] = tj.field[(size_t)q * tj.n_steps + i];
  for (int t = tid; t < NS; t += bs) {
    const int r = t / S, c = t - r * S;
    V[t] = c < N ? build_v(a.H, a.Xs, nn, r * N + c, f, ef) : make_double2(0.0, 0.0);
  }
  for (int t = tid; t < apc * NS; t += bs) {
    const int nl = t / NS, rc = t - nl * NS, r = rc / S, c = rc - r * S;
    own[t] = (n0 + nl < nado && c < N) ? src[(size_t)(n0 + nl) * nn + r * N + c] : make_double2(0.0, 0.0);
  }
  if (stage == 1 && n0 == 0) {
    const int rec = tj.rec_idx[i];
    if (rec >= 0) {
      for (int j = tid; j < N; j += bs) Pt[j] = trace_row_exact(src, tj.X3 ? tj.X3 : a.X3, N, j);
      __syncthreads();
      if (tid == 0) {
        double tr = 0.0, ti = 0.0;
        for (int j = 0; j < N; j++) { tr = __dadd_rn(tr, Pt[j].x); ti = __dadd_rn(ti, Pt[j].y); }
        tj.P[rec] = make_double2(tr, ti);
      }
    }
  }
  __syncthreads();
  for (int s = tid; s < apc * tiles; s += bs) {
    const int nl = s / tiles, u = s - nl * tiles, r = u / q4, j = u - r * q4;
    const int n = n0 + nl;
    if (n >= nado) continue;
    const double2 *ow = own + (size_t)nl * NS;
    double cr[4], ci[4];
#pragma unroll
    for (int e = 0; e < 4; e++) cr[e] = ci[e] = 0.0;
    // zgemm(i, rho_n, V, 0): C[r][c] = sum_l (i rho[r][l]) V[l][c], i rho = (-im, re)
    for (int l = 0; l < N; l++) {
      const double2 a0 = ow[r * S + l];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const double2 v = V[l * S + j + e * q4];
        cmac(cr[e], ci[e], -a0.y, a0.x, v.x, v.y);
      }
    }
    // zgemm(-i, V, rho_n, 1): C[r][c] += sum_l (-i V[r][l]) rho[l][c], -i V = (im, -re)
    for (int l = 0; l < N; l++) {
      const double2 v0 = V[r * S + l];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const double2 z = ow[l * S + j + e * q4];
        cmac(cr[e], ci[e], v0.y, -v0.x, z.x, z.y);
      }
    }
    double2 *Xn = X + (size_t)nl * nn;
    const double2 dmp = a.damp[n];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int c = j + e * q4;
      if (c >= N) continue;
      double xr = cr[e], xi = ci[e];
      if (n != 0) { // zaxpy(x_n, rho_n)
        const double2 z = ow[r * S + c];
        cmac(xr, xi, dmp.x, dmp.y, z.x, z.y);
      }
      Xn[r * N + c] = make_double2(xr, xi);
    }
  }
  __syncthreads();
  for (int t = tid; t < apc * nn; t += bs) {
    const int nl = t / nn, rc = t - nl * nn, n = n0 + nl;
    if (n >= nado) continue;
    const int r = rc / N, c = rc - r * N;
    const size_t e = (size_t)n * nn + rc;
    double cr = X[t].x, ci = X[t].y;
    for (int q = a.op_start[n]; q < a.op_start[n + 1]; q++) {
      const Op o = a.ops[q];
      const bool hit = (o.kind == 0) ? (c == o.s) : (r == o.s);
      if (hit) {
        const double2 z = src[(size_t)o.nb * nn + rc];
        cmac(cr, ci, o.cr, o.ci, z.x, z.y);
      }
    }
    const double2 k = make_double2(cr, ci);
    if (stage == 1) {
      K1[e] = k;
      B[e] = axpy_exact(A[e], a.h2, k);
    } else if (stage == 2) {
      K2[e] = k;
      A[e] = axpy_exact(axpy_exact(B[e], -a.h2, K1[e]), a.h2, k);
    } else if (stage == 3) {
      K3[e] = k;
      B[e] = axpy_exact(axpy_exact(A[e], -a.h2, K2[e]), a.h, k);
    } else {
      double2 y = axpy_exact(B[e], -a.h, K3[e]);
      y = axpy_exact(y, a.hb[0], K1[e]);
      y = axpy_exact(y, a.hb[1], K2[e]);
      y = axpy_exact(y, a.hb[2], K3[e]);
      A[e] = axpy_exact(y, a.hb[3], k);
    }
  }
}

// The same stage for blocks too wide for exact_stage's tiles in shared memory (N above
// about 69): block (n, trajectory), one element per thread, the ADO's own block and V
// in shared memory, neighbour elements from L2.
__global__ void __launch_bounds__(256) exact_stage_wide(ExactArgs a, const ExactTraj *__restrict__ trajs, int stage,
                                                   int step_local, const int *__restrict__ base) {
  extern __shared__ double2 sm[];
  const ExactTraj tj = trajs[blockIdx.y];
  const int i = *base + step_local;
  if (i >= tj.n_steps) return;
  const int N = a.N, nn = N * N, tot = a.n_ado * nn;
  const int n = blockIdx.x, tid = threadIdx.x, bs = blockDim.x;
  double2 *A = tj.work, *B = A + tot, *K1 = B + tot, *K2 = K1 + tot, *K3 = K2 + tot;
  const double2 *src = (stage == 1 || stage == 3) ? A : B;
  double2 *V = sm, *own = sm + nn, *Pt = own + nn;
  const unsigned f = tj.flags[i];
  double2 ef[3];
  for (int q = 0; q < 3; q++) ef[q] = tj.field[(size_t)q * tj.n_steps + i];
  for (int t = tid; t < nn; t += bs) {
    V[t] = build_v(a.H, a.Xs, nn, t, f, ef);
    own[t] = src[(size_t)n * nn + t];
  }
  __syncthreads();
  if (stage == 1 && n == 0) {
    const int rec = tj.rec_idx[i];
    if (rec >= 0) {
      for (int j = tid; j < N; j += bs) Pt[j] = trace_row_exact(own, tj.X3 ? tj.X3 : a.X3, N, j);
      __syncthreads();
      if (tid == 0) {
        double tr = 0.0, ti = 0.0;
        for (int j = 0; j < N; j++) { tr = __dadd_rn(tr, Pt[j].x); ti = __dadd_rn(ti, Pt[j].y); }
        tj.P[rec] = make_double2(tr, ti);
      }
    }
  }
  const double2 dmp = a.damp[n];
  const int ob = a.op_start[n], oe = a.op_start[n + 1];
  for (int rc = tid; rc < nn; rc += bs) {
    const int r = rc / N, c = rc - r * N;
    const size_t e = (size_t)n * nn + rc;
    const double2 k = rhs_exact(src, own, V, N, n, r, c, dmp, a.ops, ob, oe);
    if (stage == 1) {
      K1[e] = k;
      B[e] = axpy_exact(A[e], a.h2, k);
    } else if (stage == 2) {
      K2[e] = k;
      A[e] = axpy_exact(axpy_exact(B[e], -a.h2, K1[e]), a.h2, k);
    } else if (stage == 3) {
      K3[e] = k;
      B[e] = axpy_exact(axpy_exact(A[e], -a.h2, K2[e]), a.h, k);
    } else {
      double2 y = axpy_exact(B[e], -a.h, K3[e]);
      y = axpy_exact(y, a.hb[0], K1[e]);
      y = axpy_exact(y, a.hb[1], K2[e]);
      y = axpy_exact(y, a.hb[2], K3[e]);
      A[e] = axpy_exact(y, a.hb[3], k);
    }
  }
}

__global__ void exact_init(const ExactTraj *__restrict__ trajs, int tot) {
  const ExactTraj tj = trajs[blockIdx.y];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += gridDim.x * blockDim.x)
    tj.work[e] = make_double2(e == 0 ? 1.0 : 0.0, 0.0);
}

__global__ void bump_base(int *base, int by) { *base += by; }

} // namespace heom_dev

// ---------------------------------------------------------------- host launchers
namespace heom_dev {

size_t exact_smem_bytes(int N, int n_ado) {
  const size_t nn = (size_t)N * N;
  return sizeof(double2) * (5 * n_ado * nn + nn + N);
}

cudaError_t launch_exact_smem(const ExactArgs &a, const ExactTraj *d_trajs, int n_traj, cudaStream_t s) {
  const size_t bytes = exact_smem_bytes(a.N, a.n_ado);
  cudaError_t err = cudaFuncSetAttribute(exact_traj_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err != cudaSuccess) return err;
  const int tot = a.n_ado * a.N * a.N;
  const int threads = tot >= 512 ? 512 : ((tot + 31) / 32) * 32;
  exact_traj_smem<<<n_traj, threads, bytes, s>>>(a, d_trajs);
  return cudaGetLastError();
}

cudaError_t launch_exact_staged_chunk(const ExactArgs &a, const ExactTraj *d_trajs, int n_traj, int chunk,
                                      int *d_base, cudaStream_t s) {
  int dev = 0, max_smem = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const int apc = ex_apc(a.N);
  const size_t bytes = sizeof(double2) * ex_smem_elems(a.N, apc);
  if (a.N > kExTileMaxN || bytes + sizeof(double2) * kExTileMaxN > (size_t)max_smem) { // wide blocks
    const int nn = a.N * a.N;
    const size_t wbytes = sizeof(double2) * (2 * nn + a.N);
    cudaError_t err = cudaFuncSetAttribute(exact_stage_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wbytes);
    if (err != cudaSuccess) return err;
    dim3 grid(a.n_ado, n_traj);
    for (int st = 0; st < chunk; st++)
      for (int stage = 1; stage <= 4; stage++)
        exact_stage_wide<<<grid, 256, wbytes, s>>>(a, d_trajs, stage, st, d_base);
    bump_base<<<1, 1, 0, s>>>(d_base, chunk);
    return cudaGetLastError();
  }
  cudaError_t err = cudaFuncSetAttribute(exact_stage, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err != cudaSuccess) return err;
  const int slots = apc * ex_tiles(a.N);
  const int threads = slots >= 256 ? 256 : ((slots + 31) / 32) * 32;
  dim3 grid((a.n_ado + apc - 1) / apc, n_traj);
  for (int st = 0; st < chunk; st++)
    for (int stage = 1; stage <= 4; stage++)
      exact_stage<<<grid, threads, bytes, s>>>(a, d_trajs, stage, st, d_base);
  bump_base<<<1, 1, 0, s>>>(d_base, chunk);
  return cudaGetLastError();
}

cudaError_t launch_exact_init(const ExactTraj *d_trajs, int n_traj, int tot, cudaStream_t s) {
  dim3 grid((tot + 255) / 256 < 1024 ? (tot + 255) / 256 : 1024, n_traj);
  exact_init<<<grid, 256, 0, s>>>(d_trajs, tot);
  return cudaGetLastError();
}

} // namespace heom_dev
