// Kernel argument blocks and launchers shared by the plan (plan.cu) and the kernel
// translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace heom_dev {

struct Op;

// Problem-wide data for the bit-exact FP64 path (device pointers).
struct ExactArgs {
  int N, n_ado;
  const double2 *H;      // N x N
  const double2 *Xs;     // 3 x N x N: X[0], X[1]^T, X[2]^T (pulse operators)
  const double2 *X3;     // N x N readout operator
  const double2 *damp;   // n_ado: -sum n gamma
  const Op *ops;         // coupling ops, reference order
  const int *op_start;   // n_ado + 1
  double h2, h, hb[4];   // h/2, h, h*b[m] (b = 1/6, 2/6, 2/6, 1/6)
};

// One trajectory (device pointers).
struct ExactTraj {
  const uint8_t *flags;  // n_steps: bit q = pulse q+1 on
  const double2 *field;  // 3 x n_steps field factors
  const int *rec_idx;    // n_steps: output slot of P recorded before step i, or -1
  double2 *P;            // recorded points
  double2 *work;         // staged form: A, B, k1, k2, k3 (5 x n_ado x N x N)
  double2 *final_state;  // optional copy of the final state (n_ado x N x N)
  const double2 *X3;     // readout operator of this trajectory (nullptr: ExactArgs::X3)
  int n_steps, pad;
};

size_t exact_smem_bytes(int N, int n_ado);
cudaError_t launch_exact_smem(const ExactArgs &a, const ExactTraj *d_trajs, int n_traj, cudaStream_t s);
cudaError_t launch_exact_staged_chunk(const ExactArgs &a, const ExactTraj *d_trajs, int n_traj, int chunk,
                                      int *d_base, cudaStream_t s);
cudaError_t launch_exact_init(const ExactTraj *d_trajs, int n_traj, int tot, cudaStream_t s);

} // namespace heom_dev
