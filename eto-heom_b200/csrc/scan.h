// Batched 2DES delay-scan path (HEOM_FP64 / HEOM_FP32_BULK): host state and entry points.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/heom.h"
#include "heom_host.h"

namespace heom_dev {

struct ScanState {
  int precision = HEOM_FP32_BULK;
  int N = 0, n_ado = 0, M = 0, K = 0, K_m = 0, E = 0, max_points = 0;
  bool supported = false;
  std::string why;
  // launch shape (autotuned)
  int variant = 0, ept = 8, threads = 0, grid = 0, sm_count = 0;
  int wcap = 0;                  // pulse-field window table length (whole-ADO form)
  int ado0 = 0;                  // index of ADO 0 in the whole-ADO form's order
  size_t smem = 0;
  float tune_ms = 0;
  bool pinned = false;           // launch shape fixed by HEOM_SCAN_VARIANT
  // problem constants
  float t_start = 0, dt = 0;
  int stride = 1;
  double E0[3] = {0, 0, 0}, taup[3] = {0, 0, 0}, w0[3] = {0, 0, 0}, h = 0;
  // device buffers
  void *d_tables = nullptr;      // packed read-only tables (see scan.cu)
  size_t tables_bytes = 0;
  double *d_sys = nullptr;       // Hd, Hoff, Xs, X3 (re-uploaded per sample)
  size_t sys_doubles = 0;
  heom_scan_point *d_pts = nullptr;
  long long *d_offsets = nullptr;
  double *d_P = nullptr;
  long long P_cap = 0;
  int *d_order = nullptr, *d_counter = nullptr, *d_status = nullptr;
  // pinned staging for the host-buffer entry point
  heom_scan_point *h_pts = nullptr;
  long long *h_offsets = nullptr;
  double *h_P = nullptr;
  long long hP_cap = 0;
  // copy-out straight into a caller buffer from heom_host_alloc: the finiteness check
  // runs on the device (flag d_bad, read back into h_bad)
  int *d_bad = nullptr, *h_bad = nullptr;
  long long check_launches = 0;
  // staged scan (scan_slots.cuh): shared R/D2 per (tau1, tau2), per-point pulse-3 window,
  // pulse-free tails as products with the dual rows
  bool staged = false;           // chosen for heom_run_scan / heom_run_scan_device
  bool rstat = false;            // H couples level 0 to nothing (|0><0| stationary)
  bool r_row0 = false;           // R stays in row 0 and Tr X3 R = 0 (see scan_upload_system)
  int sl_threads = 0, sl_grid = 0, sl_wcap = 0;
  size_t sl_smem = 0;
  void *d_snap = nullptr;        // snapshots: 2 states per regular point
  size_t snap_cap = 0;
  void *d_jobs = nullptr, *d_saves = nullptr, *d_flags = nullptr;
  size_t jobs_cap = 0, saves_cap = 0, flags_cap = 0;
  int *err_pending = nullptr;    // error word of a run not yet checked
  // test hook (heom_plan_inject_wait_fault): the next staged run only
  unsigned long long inject_wait_ns = 0; // dependency wait limit (0: the default 30 s)
  bool inject_unmet = false;     // one consumer job waits for a flag value never set
  long long last_work = 0;       // component-steps propagated by the last staged run
  std::vector<float> t_grid;     // float time of each step (t_start + dt accumulated)
  int tail_n = 0;                // its positions (0: tails run on full blocks)
  void *d_tailpts = nullptr;     // the tail kernel's points, then its tiles
  size_t tailpts_cap = 0;
  // dual tails (scan_tail_dual): L^T of the pulse-free reduced system (CSR) and its
  // diagonal, w_k rows on the host and the device, the reduced positions
  std::vector<unsigned char> h_tables;
  std::vector<int> dual_start, dual_idx, dual_pos;
  std::vector<double> dual_coef, h_W;
  int W_rows = 0, W_dev_rows = 0;
  bool dual_pos_dirty = false;
  void *d_W = nullptr, *d_dualpos = nullptr;
  size_t W_cap = 0;
  // the dual rows on the device: CSR of L^T (start | idx | coef), its upload copy, an
  // auxiliary stream that overlaps the chain with the slot kernel, fork / join events
  bool dual_dirty = false, dual_on_aux = false;
  void *d_dcsr = nullptr;
  size_t dcsr_cap = 0, dcsr_idx = 0, dcsr_coef = 0;
  std::vector<unsigned char> h_dcsr;
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // jumps over pulse-free intervals: position blocks (jtab: count, positions per block,
  // first position, matrix offset, positions), dense L0 blocks, powers T0^(2^j) on device
  std::vector<int> jtab, jdims;
  std::vector<double> h_jL;
  long long jpow_elems = 0;
  size_t jblocks = 0;
  int jpow_n = 0, jpow_cap = 0; // d_jpow holds jpow_cap powers and one leg T0^jleg_formed after them
  int jleg_formed = 0;          // the leg formed for this sample (0: none)
  bool jL_dirty = false;
  void *d_jtab = nullptr, *d_jL = nullptr, *d_jpow = nullptr, *d_jtmp = nullptr, *d_jdims = nullptr;
  size_t jL_cap = 0, jtab_cap = 0, jmeta_offs = 0; // kept across samples while large enough
  std::vector<unsigned char> h_jmeta;            // jtab + per-block offsets, as uploaded
  std::vector<int> h_jdims;                      // block sizes as uploaded
  int jdims_cap = 0;
  std::vector<heom_scan_point> rb_pts; // points / offsets read back for heom_run_scan_device
  std::vector<long long> rb_off;
  long long staged_launches = 0;
  // replay of the last planned staged scan (staged_run): valid while the points, offsets,
  // output buffer, snapshot buffer and sample structure are unchanged; the kernel arguments are
  // kept as bytes (SlotArgs, DualArgs of scan_slots.cuh)
  std::vector<int> structure;    // what the planner reads of the sample (scan_upload_system)
  bool dual_launched = false;    // the last dual_rows call launched the chain kernel
  cudaGraphExec_t rp_graph = nullptr; // a steady-state replay as one graph (staged_replay)
  const void *rp_graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
  struct Replay {
    bool valid = false, tails = false;
    int n = 0, grid = 0, jpow_use = 0, jleg = 0, kmax = 0, tail_grid = 0, tail_grid_y = 0;
    size_t nflags = 0;
    long long work = 0;
    std::vector<int> structure;
    const void *d_P = nullptr, *snap = nullptr;
    std::vector<heom_scan_point> pts;
    std::vector<long long> offsets;
    alignas(16) unsigned char a[512];
    alignas(16) unsigned char da[128];
  } rp;
  // graph cache for heom_run_scan_device
  cudaGraphExec_t gexec = nullptr;
  const void *g_key[4] = {nullptr, nullptr, nullptr, nullptr};
  int g_n = -1;
};

int scan_init(ScanState &s, const heom::Problem &p, int precision, int max_points, bool autotune, cudaStream_t st,
              bool single_pass = false);
// Shape + packed tables without any device allocation (false: unsupported, s.why set).
bool scan_prepare(ScanState &s, const heom::Problem &p, int precision, int max_points,
                  std::vector<unsigned char> &tables);
// Packed system matrices of the problem's current sample (s.sys_doubles entries).
void scan_system_host(const heom::Problem &p, std::vector<double> &sys);
// Enqueue [order kernel, scan kernel] on st using the device pointers held in s.
cudaError_t scan_enqueue(const ScanState &s, const heom_scan_point *d_pts, int n, double *d_P,
                         const long long *d_offsets, cudaStream_t st);
int scan_upload_system(ScanState &s, const heom::Problem &p, cudaStream_t st);
int scan_run_host(ScanState &s, const heom_scan_point *pts, int n, double *P, const long long *offsets,
                  long long total, cudaStream_t st);
// Page-locked host buffers of heom_host_alloc, kept in a registry so that the host-buffer
// scan entry can recognise an output array that lies inside one of them.
int host_alloc(size_t bytes, void **p);
int host_free(void *p);
bool host_pinned_covers(const void *p, size_t bytes);
int scan_run_device(ScanState &s, const heom_scan_point *d_pts, int n, double *d_P, const long long *d_offsets,
                    cudaStream_t st);
// Waits for the stream and returns the status of the last staged run (HEOM_ERR_TIMEOUT
// when a dependency wait gave up, HEOM_ERR_CUDA when a device-side check failed).
int scan_sync(ScanState &s, cudaStream_t st);
void scan_release(ScanState &s);
std::string scan_describe(const ScanState &s);
const char *scan_last_error();
long long scan_launches_per_run(const ScanState &s);

} // namespace heom_dev
