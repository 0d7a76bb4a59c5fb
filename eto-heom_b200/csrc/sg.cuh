// General-size propagation path (HEOM_FP64 / HEOM_FP32_BULK for any N): host state.
//
// The state of a batch of points lives in global memory (L2-resident for the configured
// sizes): one kernel launch per Horner stage over (ADO tile, component, point), with
// the same arithmetic as the shared-memory scan kernel -- mixed-difference basis for a
// 2DES point (4 components) or a single pulse mask (1 component), FP64 state and
// Horner accumulator, FP32 (or FP64) contractions.  Launch sequences of a chunk of steps
// are captured into a CUDA graph and replayed; the step index lives in device memory.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/heom.h"
#include "heom_host.h"

namespace heom_dev {

struct SgState {
  int precision = HEOM_FP32_BULK;
  int N = 0, n_ado = 0, M = 0, K = 0, K_m = 0;
  int apc = 1, threads = 32;          // ADOs per CTA, threads per CTA
  int tf = 0;                         // FP32-bulk phase-1 products: 0 FP32, 1 TF32, 3 3xTF32 (study)
  size_t smem = 0;
  // problem tables (device)
  void *d_tab = nullptr;              // Hd, Hoff, Xs, X3, damp, alpha, xc, yc, up, dn
  size_t tab_bytes = 0;
  // per-run buffers (device), grown on demand
  void *d_state = nullptr;            // rho, w64[2], w32[2]
  size_t state_bytes = 0;
  void *d_sched = nullptr;            // flags, rec, field, nsteps, offsets
  size_t sched_bytes = 0;
  double2 *d_P = nullptr;
  long long P_cap = 0;
  void *d_ops = nullptr;              // per (point, component): the step's operators
  size_t ops_bytes = 0;
  int *d_base = nullptr;
  // graph of one chunk of steps of the current run
  cudaGraphExec_t gexec = nullptr;
  int g_chunk = 8;
  float t_start = 0, dt = 0;
  int stride = 1;
  double h = 0;
  long long launches = 0;
};

int sg_init(SgState &s, const heom::Problem &p, int precision, cudaStream_t st);
int sg_upload_system(SgState &s, const heom::Problem &p, cudaStream_t st);
// Propagate n points.  C = 4: 2DES points in the mixed-difference basis, output
// P = p111 - p110 - p101; C = 1: one trajectory per point with pulse mask `mask`,
// output Tr(X3 rho).  pts give the pulse times and end time of each point; P (host)
// receives the recorded points at offsets[i] (counts from heom::count_records).
int sg_run(SgState &s, const heom::Problem &p, int C, const int mask[3], const heom_scan_point *pts, int n,
           double *P, const long long *offsets, long long total, cudaStream_t st);
void sg_release(SgState &s);
const char *sg_last_error();

// Adjoint of a delay scan (adjoint.cu): forward readout into P_host and the gradient of
// Re sum_i conj(g_i) P_i with respect to heom::n_params(p) parameters into grad.
int adjoint_scan(const heom::Problem &p, const heom_scan_point *pts, int n, const long long *offsets, long long total,
                 const double *g_host, double *P_host, double *grad, long long *launches, cudaStream_t st);
const char *adj_last_error();

} // namespace heom_dev
