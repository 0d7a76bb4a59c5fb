// C ABI implementation (include/heom.h): problem handles, device plans and the
// trajectory / 2DES / scan entry points.  Host code only; kernels live in exact.cu
// and scan.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/heom.h"
#include "exact.cuh"
#include "heom_host.h"
#include "kernels.h"
#include "scan.h"
#include "sg.cuh"

namespace {
thread_local std::string g_err;
int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}
} // namespace

int heom::set_error(int code, const std::string &msg) { return fail(code, msg); }

namespace {
int cuda_fail(cudaError_t e, const char *what) {
  return fail(HEOM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                                  \
  do {                                                            \
    cudaError_t e_ = (call);                                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);           \
  } while (0)

template <class T> struct DevBuf {
  T *ptr = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t want) {
    if (want <= n && ptr) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&ptr, sizeof(T) * std::max<size_t>(want, 1));
    if (e == cudaSuccess) n = want;
    return e;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
};
} // namespace

struct heom_plan {
  int device = 0, precision = HEOM_FP64_EXACT, max_points = 1024;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  heom::Problem prob; // snapshot of tables and the current sample
  long long launches = 0;
  // problem-wide device data
  DevBuf<double2> d_H, d_Xs, d_X3, d_damp;
  DevBuf<heom_dev::Op> d_ops;
  DevBuf<int> d_op_start;
  // exact path, up to three concurrent trajectories
  DevBuf<uint8_t> d_flags;
  DevBuf<double2> d_field, d_P, d_work;
  DevBuf<int> d_rec, d_base;
  DevBuf<heom_dev::ExactTraj> d_trajs;
  DevBuf<double2> d_X3pop; // per-site readout operators of heom_run_populations
  bool use_smem = true;
  int chunk = 8;
  static constexpr int kMaxTraj = 64; // concurrent exact-path trajectories per launch
  cudaGraphExec_t graph[kMaxTraj + 1] = {};
  heom_dev::ExactArgs args{};
  // scan path (shared-memory resident) and staged path (any size), the latter built on
  // first use
  heom_dev::ScanState scan;
  heom_dev::SgState sg;
  bool sg_ready = false;
  std::string desc;
  ~heom_plan() {
    for (auto &g : graph)
      if (g) cudaGraphExecDestroy(g);
    heom_dev::scan_release(scan);
    if (sg_ready) heom_dev::sg_release(sg);
    d_H.release(); d_Xs.release(); d_X3.release(); d_damp.release(); d_ops.release(); d_op_start.release();
    d_flags.release(); d_field.release(); d_P.release(); d_work.release(); d_rec.release(); d_base.release();
    d_trajs.release(); d_X3pop.release();
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

int upload_system(heom_plan *pl) {
  const heom::Problem &p = pl->prob;
  const int N = p.N(), nn = N * N;
  std::vector<double> xs(2 * 3 * (size_t)nn);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++) {
      const size_t t = (size_t)i * N + j, tt = (size_t)j * N + i;
      xs[2 * t] = p.X[0][2 * t];
      xs[2 * t + 1] = p.X[0][2 * t + 1];
      xs[2 * (nn + t)] = p.X[1][2 * tt];          // X[1]^T (dynamics.cpp:305-306)
      xs[2 * (nn + t) + 1] = p.X[1][2 * tt + 1];
      xs[2 * (2 * nn + t)] = p.X[2][2 * tt];      // X[2]^T
      xs[2 * (2 * nn + t) + 1] = p.X[2][2 * tt + 1];
    }
  CK(cudaMemcpyAsync(pl->d_H.ptr, p.H.data(), sizeof(double) * 2 * nn, cudaMemcpyHostToDevice, pl->stream));
  CK(cudaMemcpyAsync(pl->d_Xs.ptr, xs.data(), sizeof(double) * xs.size(), cudaMemcpyHostToDevice, pl->stream));
  CK(cudaMemcpyAsync(pl->d_X3.ptr, p.X[3].data(), sizeof(double) * 2 * nn, cudaMemcpyHostToDevice, pl->stream));
  CK(cudaStreamSynchronize(pl->stream));
  int rc = heom_dev::scan_upload_system(pl->scan, p, pl->stream);
  if (rc) return rc;
  if (pl->sg_ready) {
    rc = heom_dev::sg_upload_system(pl->sg, p, pl->stream);
    if (rc) return fail(rc, heom_dev::sg_last_error());
  }
  return HEOM_OK;
}

int ensure_sg(heom_plan *pl) {
  if (pl->sg_ready) return HEOM_OK;
  int rc = heom_dev::sg_init(pl->sg, pl->prob, pl->precision, pl->stream);
  if (rc) return fail(rc, heom_dev::sg_last_error());
  pl->sg_ready = true;
  return HEOM_OK;
}

// Staged path: n points of C components (see sg.cuh); P receives `total` points.
int run_sg(heom_plan *pl, int C, const int mask[3], const heom_scan_point *pts, int n, double *P,
           const long long *offsets, long long total) {
  int rc = ensure_sg(pl);
  if (rc) return rc;
  rc = heom_dev::sg_run(pl->sg, pl->prob, C, mask, pts, n, P, offsets, total, pl->stream);
  if (rc) return fail(rc, heom_dev::sg_last_error());
  return HEOM_OK;
}

heom_scan_point key_point(const heom::Problem &p) {
  return heom_scan_point{p.pulses[0].tau0, p.pulses[1].tau0, p.pulses[2].tau0, p.t_end, 0};
}

// Run up to kMaxTraj trajectories of the exact path concurrently (one CTA or block row
// each).  tau_in: pulse times (nullptr: the key's); X3s: per-trajectory device readout
// operators (nullptr: the problem's X3).
int run_exact(heom_plan *pl, const int (*masks)[3], int n_traj, std::vector<std::vector<double>> &out,
              const double *tau_in = nullptr, const double2 *const *X3s = nullptr) {
  const heom::Problem &p = pl->prob;
  if (n_traj < 1 || n_traj > heom_plan::kMaxTraj) return fail(HEOM_ERR_ARG, "trajectory count out of range");
  const double tau[3] = {tau_in ? tau_in[0] : p.pulses[0].tau0, tau_in ? tau_in[1] : p.pulses[1].tau0,
                         tau_in ? tau_in[2] : p.pulses[2].tau0};
  std::vector<heom::Schedule> sch;
  for (int t = 0; t < n_traj; t++) sch.push_back(heom::make_schedule(p, tau, p.t_end, masks[t]));
  const int ns = sch[0].n_steps, nrec = sch[0].n_record;
  const int N = p.N(), nn = N * N, tot = p.n_ado * nn;
  CK(pl->d_flags.ensure((size_t)n_traj * ns));
  CK(pl->d_field.ensure((size_t)n_traj * 3 * ns));
  CK(pl->d_rec.ensure((size_t)n_traj * ns));
  CK(pl->d_P.ensure((size_t)n_traj * std::max(nrec, 1)));
  CK(pl->d_trajs.ensure(n_traj));
  if (!pl->use_smem) CK(pl->d_work.ensure((size_t)n_traj * 5 * tot));
  std::vector<heom_dev::ExactTraj> tr(n_traj);
  for (int t = 0; t < n_traj; t++) {
    CK(cudaMemcpyAsync(pl->d_flags.ptr + (size_t)t * ns, sch[t].flags.data(), ns, cudaMemcpyHostToDevice, pl->stream));
    CK(cudaMemcpyAsync(pl->d_field.ptr + (size_t)t * 3 * ns, sch[t].field.data(), sizeof(double2) * 3 * ns,
                       cudaMemcpyHostToDevice, pl->stream));
    CK(cudaMemcpyAsync(pl->d_rec.ptr + (size_t)t * ns, sch[t].rec_idx.data(), sizeof(int) * ns, cudaMemcpyHostToDevice,
                       pl->stream));
    tr[t].flags = pl->d_flags.ptr + (size_t)t * ns;
    tr[t].field = pl->d_field.ptr + (size_t)t * 3 * ns;
    tr[t].rec_idx = pl->d_rec.ptr + (size_t)t * ns;
    tr[t].P = pl->d_P.ptr + (size_t)t * std::max(nrec, 1);
    tr[t].work = pl->use_smem ? nullptr : pl->d_work.ptr + (size_t)t * 5 * tot;
    tr[t].final_state = nullptr;
    tr[t].X3 = X3s ? X3s[t] : nullptr;
    tr[t].n_steps = ns;
  }
  CK(cudaMemcpyAsync(pl->d_trajs.ptr, tr.data(), sizeof(heom_dev::ExactTraj) * n_traj, cudaMemcpyHostToDevice,
                     pl->stream));
  if (pl->use_smem) {
    CK(heom_dev::launch_exact_smem(pl->args, pl->d_trajs.ptr, n_traj, pl->stream));
    pl->launches += 1;
  } else {
    CK(heom_dev::launch_exact_init(pl->d_trajs.ptr, n_traj, tot, pl->stream));
    CK(pl->d_base.ensure(1));
    CK(cudaMemsetAsync(pl->d_base.ptr, 0, sizeof(int), pl->stream));
    pl->launches += 1;
    cudaGraphExec_t &g = pl->graph[n_traj];
    if (!g) {
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(pl->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t le = heom_dev::launch_exact_staged_chunk(pl->args, pl->d_trajs.ptr, n_traj, pl->chunk,
                                                           pl->d_base.ptr, pl->stream);
      cudaError_t ce = cudaStreamEndCapture(pl->stream, &graph);
      if (le != cudaSuccess) return cuda_fail(le, "capture exact stage chunk");
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      cudaError_t ie = cudaGraphInstantiate(&g, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate");
    }
    const int reps = (ns + pl->chunk - 1) / pl->chunk;
    for (int r = 0; r < reps; r++) CK(cudaGraphLaunch(g, pl->stream));
    pl->launches += (long long)reps * (4LL * pl->chunk + 1);
  }
  out.assign(n_traj, std::vector<double>(2 * (size_t)nrec));
  for (int t = 0; t < n_traj; t++)
    if (nrec)
      CK(cudaMemcpyAsync(out[t].data(), tr[t].P, sizeof(double2) * nrec, cudaMemcpyDeviceToHost, pl->stream));
  CK(cudaStreamSynchronize(pl->stream));
  for (auto &v : out)
    for (double x : v)
      if (!std::isfinite(x)) return fail(HEOM_ERR_NUMERIC, "non-finite P(t): the propagation diverged");
  return HEOM_OK;
}

} // namespace

extern "C" {

const char *heom_last_error(void) { return g_err.c_str(); }
int heom_abi_version(void) { return HEOM_ABI_VERSION; }

int heom_problem_from_key(const char *path, int flags, heom_problem **out) {
  if (!path || !out) return fail(HEOM_ERR_ARG, "null argument");
  *out = nullptr;
  heom_problem *h = new (std::nothrow) heom_problem();
  if (!h) return fail(HEOM_ERR_NOMEM, "out of host memory");
  std::string err;
  int code = HEOM_ERR_PARSE;
  try {
    if (!heom::parse_key(path, flags, h->p, err, &code)) {
      delete h;
      return fail(code, err);
    }
  } catch (const std::bad_alloc &) {
    delete h;
    return fail(HEOM_ERR_NOMEM, "out of host memory while building the hierarchy");
  }
  *out = h;
  return HEOM_OK;
}

int heom_problem_info_get(const heom_problem *h, heom_problem_info *info) {
  if (!h || !info) return fail(HEOM_ERR_ARG, "null argument");
  const heom::Problem &p = h->p;
  std::memset(info, 0, sizeof *info);
  info->single_size = p.single_size;
  info->sys_size = p.sys_size;
  info->K = p.K;
  info->K_m = p.K_m;
  info->L = p.L;
  info->n_ado = p.n_ado;
  info->n_sample = p.n_sample;
  info->seed = p.seed;
  info->n_steps = p.n_steps();
  info->print_stride = p.print_stride();
  info->n_record = heom::count_records(p, p.dynamics ? -HUGE_VAL : p.pulses[2].tau0, p.t_end);
  info->t_start = p.t_start;
  info->t_end = p.t_end;
  info->step_size = p.step_size;
  info->print_step = p.print_step;
  for (int q = 0; q < 3; q++) {
    info->E0[q] = p.pulses[q].E0;
    info->tau[q] = p.pulses[q].tau0;
    info->taup[q] = p.pulses[q].taup;
    info->w0[q] = p.pulses[q].w0;
  }
  return HEOM_OK;
}

int heom_problem_scan_compatible(const heom_problem *a, const heom_problem *b) {
  if (!a || !b) return fail(HEOM_ERR_ARG, "null problem");
  const heom::Problem &x = a->p, &y = b->p;
  bool same = x.single_size == y.single_size && x.sys_size == y.sys_size && x.K == y.K && x.K_m == y.K_m &&
              x.L == y.L && x.n_sample == y.n_sample && x.seed == y.seed && x.single_manifold == y.single_manifold &&
              x.d_a == y.d_a && x.d_b == y.d_b && x.Hkey == y.Hkey && x.Dis == y.Dis && x.Xx == y.Xx &&
              x.Xy == y.Xy && x.Xz == y.Xz && x.have_polar == y.have_polar && x.have_dipole == y.have_dipole &&
              x.have_bath == y.have_bath && x.have_pulse == y.have_pulse && x.alpha == y.alpha &&
              x.alpha_t == y.alpha_t && x.gamma == y.gamma && x.bath_scale == y.bath_scale &&
              x.t_start == y.t_start && x.step_size == y.step_size && x.print_step == y.print_step;
  for (int q = 0; q < 4; q++) same = same && x.angle[q] == y.angle[q];
  for (int q = 0; q < 3; q++)
    same = same && x.pulses[q].E0 == y.pulses[q].E0 && x.pulses[q].taup == y.pulses[q].taup &&
           x.pulses[q].w0 == y.pulses[q].w0;
  return same ? 1 : 0;
}

int heom_problem_prepare_sample(heom_problem *h) {
  if (!h) return fail(HEOM_ERR_ARG, "null problem");
  heom::prepare_sample(h->p, true, true);
  return HEOM_OK;
}
int heom_problem_prepare_identity(heom_problem *h) {
  if (!h) return fail(HEOM_ERR_ARG, "null problem");
  heom::prepare_sample(h->p, false, false);
  return HEOM_OK;
}
int heom_problem_reset_rng(heom_problem *h) {
  if (!h) return fail(HEOM_ERR_ARG, "null problem");
  h->p.rng.seed(h->p.seed);
  return HEOM_OK;
}

static heom::cbuf *select_matrix(heom::Problem &p, int which) {
  switch (which) {
  case HEOM_MAT_H: return &p.H;
  case HEOM_MAT_X0: return &p.X[0];
  case HEOM_MAT_X1: return &p.X[1];
  case HEOM_MAT_X2: return &p.X[2];
  case HEOM_MAT_X3: return &p.X[3];
  case HEOM_MAT_HKEY: return &p.Hkey;
  default: return nullptr;
  }
}

int heom_problem_get_matrix(const heom_problem *h, int which, double *out) {
  if (!h || !out) return fail(HEOM_ERR_ARG, "null argument");
  heom::cbuf *m = select_matrix(const_cast<heom::Problem &>(h->p), which);
  if (!m) return fail(HEOM_ERR_ARG, "unknown matrix selector");
  std::memcpy(out, m->data(), sizeof(double) * m->size());
  return HEOM_OK;
}
int heom_problem_set_matrix(heom_problem *h, int which, const double *in) {
  if (!h || !in) return fail(HEOM_ERR_ARG, "null argument");
  heom::cbuf *m = select_matrix(h->p, which);
  if (!m) return fail(HEOM_ERR_ARG, "unknown matrix selector");
  std::memcpy(m->data(), in, sizeof(double) * m->size());
  return HEOM_OK;
}
int heom_problem_get_ado(const heom_problem *h, unsigned char *out) {
  if (!h || !out) return fail(HEOM_ERR_ARG, "null argument");
  std::memcpy(out, h->p.ado.data(), h->p.ado.size());
  return HEOM_OK;
}
void heom_problem_destroy(heom_problem *h) { delete h; }

int heom_plan_create(const heom_problem *h, const heom_opts *opts, heom_plan **out) {
  if (!h || !out) return fail(HEOM_ERR_ARG, "null argument");
  *out = nullptr;
  heom_opts o{};
  if (opts) o = *opts;
  if (o.precision < HEOM_FP64_EXACT || o.precision > HEOM_FP32_BULK) return fail(HEOM_ERR_ARG, "unknown precision");
  if (h->p.dynamics && o.precision != HEOM_FP64_EXACT)
    return fail(HEOM_ERR_UNSUPPORTED, "population-dynamics keys run on HEOM_FP64_EXACT plans");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(HEOM_ERR_CUDA, std::string("no CUDA device: ") + (e == cudaSuccess ? "count 0" : cudaGetErrorString(e)));
  if (o.device < 0 || o.device >= ndev) return fail(HEOM_ERR_ARG, "device ordinal out of range");
  CK(cudaSetDevice(o.device));
  std::unique_ptr<heom_plan> pl(new (std::nothrow) heom_plan());
  if (!pl) return fail(HEOM_ERR_NOMEM, "out of host memory");
  pl->device = o.device;
  pl->precision = o.precision;
  pl->max_points = o.max_points > 0 ? o.max_points : 1024;
  pl->prob = h->p;
  if (o.stream) {
    pl->stream = (cudaStream_t)o.stream;
  } else {
    CK(cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking));
    pl->own_stream = true;
  }
  const heom::Problem &p = pl->prob;
  const int N = p.N(), nn = N * N;
  CK(pl->d_H.ensure(nn));
  CK(pl->d_Xs.ensure(3 * (size_t)nn));
  CK(pl->d_X3.ensure(nn));
  CK(pl->d_damp.ensure(p.n_ado));
  CK(pl->d_ops.ensure(std::max<size_t>(p.ops.size(), 1)));
  CK(pl->d_op_start.ensure(p.n_ado + 1));
  CK(cudaMemcpyAsync(pl->d_damp.ptr, p.damp.data(), sizeof(double2) * p.n_ado, cudaMemcpyHostToDevice, pl->stream));
  if (!p.ops.empty())
    CK(cudaMemcpyAsync(pl->d_ops.ptr, p.ops.data(), sizeof(heom::CouplingOp) * p.ops.size(), cudaMemcpyHostToDevice,
                       pl->stream));
  CK(cudaMemcpyAsync(pl->d_op_start.ptr, p.op_start.data(), sizeof(int) * (p.n_ado + 1), cudaMemcpyHostToDevice,
                     pl->stream));
  static_assert(sizeof(heom::CouplingOp) == sizeof(heom_dev::Op), "op layout");
  heom_dev::ExactArgs &a = pl->args;
  a.N = N;
  a.n_ado = p.n_ado;
  a.H = pl->d_H.ptr;
  a.Xs = pl->d_Xs.ptr;
  a.X3 = pl->d_X3.ptr;
  a.damp = pl->d_damp.ptr;
  a.ops = pl->d_ops.ptr;
  a.op_start = pl->d_op_start.ptr;
  // dynamics.cpp:303,388-417: coefficients are float step_size promoted to double.
  const double hs = (double)p.step_size;
  const double b[4] = {1.0 / 6, 2.0 / 6, 2.0 / 6, 1.0 / 6};
  a.h2 = hs * 0.5;
  a.h = hs;
  for (int m = 0; m < 4; m++) a.hb[m] = hs * b[m];
  pl->use_smem = heom_dev::exact_smem_bytes(N, p.n_ado) <= 200 * 1024;
  int rc = 0;
  if (!p.dynamics) { // the batched paths put site j's S on level j+1 (2DES keys only)
    rc = heom_dev::scan_init(pl->scan, p, pl->precision, pl->max_points, o.autotune != 0, pl->stream,
                             o.single_pass != 0);
    if (rc) return fail(rc, heom_dev::scan_last_error());
  }
  rc = upload_system(pl.get());
  if (rc) return rc;
  char buf[256];
  std::snprintf(buf, sizeof buf, "exact: %s; scan: %s", pl->use_smem ? "one CTA per trajectory, state in SMEM"
                                                                      : "per-stage graph, state in L2",
                heom_dev::scan_describe(pl->scan).c_str());
  pl->desc = buf;
  *out = pl.release();
  return HEOM_OK;
}

int heom_plan_update(heom_plan *pl, const heom_problem *h) {
  if (!pl || !h) return fail(HEOM_ERR_ARG, "null argument");
  if (h->p.N() != pl->prob.N() || h->p.n_ado != pl->prob.n_ado) return fail(HEOM_ERR_ARG, "problem shape changed");
  CK(cudaSetDevice(pl->device));
  pl->prob.H = h->p.H;
  for (int q = 0; q < 4; q++) pl->prob.X[q] = h->p.X[q];
  return upload_system(pl);
}

int heom_run_traj(heom_plan *pl, int nv1, int nv2, int nv3, double *P, int cap, int *n_out) {
  if (!pl || !n_out) return fail(HEOM_ERR_ARG, "null argument");
  CK(cudaSetDevice(pl->device));
  if (pl->precision != HEOM_FP64_EXACT) {
    const heom_scan_point pt = key_point(pl->prob);
    const int n = heom::count_records(pl->prob, pt.tau3, pt.t_end);
    *n_out = n;
    if (n > cap || (!P && n > 0)) return fail(HEOM_ERR_CAPACITY, "output buffer too small");
    const int mask[3] = {nv1 == 1, nv2 == 1, nv3 == 1};
    const long long off = 0;
    std::vector<double> tmp(2 * (size_t)std::max(n, 1));
    int rc = run_sg(pl, 1, mask, &pt, 1, tmp.data(), &off, n);
    if (rc) return rc;
    if (n) std::memcpy(P, tmp.data(), sizeof(double) * 2 * n);
    return HEOM_OK;
  }
  const int m[1][3] = {{nv1, nv2, nv3}};
  std::vector<std::vector<double>> out;
  int rc = run_exact(pl, m, 1, out);
  if (rc) return rc;
  const int n = (int)(out[0].size() / 2);
  *n_out = n;
  if (n > cap || (!P && n > 0)) return fail(HEOM_ERR_CAPACITY, "output buffer too small");
  if (n) std::memcpy(P, out[0].data(), sizeof(double) * 2 * n);
  return HEOM_OK;
}

int heom_run_populations(heom_plan *pl, const int *sites, int n_sites, double *pop, int cap, int *n_out) {
  if (!pl || !sites || !n_out || n_sites < 1) return fail(HEOM_ERR_ARG, "bad argument");
  if (n_sites > heom_plan::kMaxTraj) return fail(HEOM_ERR_CAPACITY, "at most 64 sites per call");
  if (pl->precision != HEOM_FP64_EXACT)
    return fail(HEOM_ERR_UNSUPPORTED, "heom_run_populations needs a HEOM_FP64_EXACT plan");
  const heom::Problem &p = pl->prob;
  const int N = p.N(), nn = N * N;
  for (int k = 0; k < n_sites; k++) // dynamics.cpp:206-215
    if (sites[k] < 1 || sites[k] > N) return fail(HEOM_ERR_ARG, "site " + std::to_string(sites[k]) + " is out of range");
  CK(cudaSetDevice(pl->device));
  // One trajectory per site, all in one launch, each reading out Tr(rho_0 |l><l|): the
  // reference's trace arithmetic with a one-hot operator adds only exact zeros to
  // rho_0[l][l], so the readout is the population itself.
  std::vector<double> X(2 * (size_t)n_sites * nn, 0.0);
  for (int k = 0; k < n_sites; k++) {
    const int l = sites[k] - 1;
    X[2 * ((size_t)k * nn + (size_t)l * N + l)] = 1.0;
  }
  CK(pl->d_X3pop.ensure((size_t)n_sites * nn));
  CK(cudaMemcpyAsync(pl->d_X3pop.ptr, X.data(), sizeof(double) * X.size(), cudaMemcpyHostToDevice, pl->stream));
  std::vector<const double2 *> X3s(n_sites);
  for (int k = 0; k < n_sites; k++) X3s[k] = pl->d_X3pop.ptr + (size_t)k * nn;
  std::vector<int> masks(3 * (size_t)n_sites, 0);
  const double tau[3] = {p.pulses[0].tau0, p.pulses[1].tau0, -HUGE_VAL}; // record from t_start
  std::vector<std::vector<double>> out;
  int rc = run_exact(pl, reinterpret_cast<const int(*)[3]>(masks.data()), n_sites, out, tau, X3s.data());
  if (rc) return rc;
  const int n = (int)(out[0].size() / 2);
  *n_out = n;
  if (n > cap || (!pop && n > 0)) return fail(HEOM_ERR_CAPACITY, "output buffer too small");
  for (int k = 0; k < n_sites; k++)
    for (int j = 0; j < n; j++) pop[(size_t)k * cap + j] = out[k][2 * (size_t)j];
  return HEOM_OK;
}

int heom_run_2des(heom_plan *pl, double *P, double *p_traj, int cap, int *n_out) {
  if (!pl || !n_out) return fail(HEOM_ERR_ARG, "null argument");
  if (pl->prob.dynamics) return fail(HEOM_ERR_UNSUPPORTED, "a population-dynamics plan runs heom_run_populations only");
  CK(cudaSetDevice(pl->device));
  static const int masks[3][3] = {{1, 1, 1}, {1, 1, 0}, {1, 0, 1}}; // CPU_2DES.cpp:65-71
  if (pl->precision != HEOM_FP64_EXACT) {
    // combined output in the mixed-difference basis; the three trajectories on request
    const heom_scan_point pt = key_point(pl->prob);
    const int n = heom::count_records(pl->prob, pt.tau3, pt.t_end);
    *n_out = n;
    if (n > cap || (!P && n > 0)) return fail(HEOM_ERR_CAPACITY, "output buffer too small");
    const long long off = 0;
    std::vector<double> tmp(2 * (size_t)std::max(n, 1));
    int rc = run_sg(pl, 4, nullptr, &pt, 1, tmp.data(), &off, n);
    if (rc) return rc;
    if (n) std::memcpy(P, tmp.data(), sizeof(double) * 2 * n);
    if (p_traj)
      for (int t = 0; t < 3; t++) {
        rc = run_sg(pl, 1, masks[t], &pt, 1, tmp.data(), &off, n);
        if (rc) return rc;
        if (n) std::memcpy(p_traj + 2 * (size_t)t * cap, tmp.data(), sizeof(double) * 2 * n);
      }
    return HEOM_OK;
  }
  std::vector<std::vector<double>> out;
  int rc = run_exact(pl, masks, 3, out);
  if (rc) return rc;
  const int n = (int)(out[0].size() / 2);
  *n_out = n;
  if (n > cap || (!P && n > 0)) return fail(HEOM_ERR_CAPACITY, "output buffer too small");
  for (int j = 0; j < 2 * n; j++) P[j] = out[0][j] - out[1][j] - out[2][j]; // CPU_2DES.cpp:73-79
  if (p_traj)
    for (int t = 0; t < 3; t++) std::memcpy(p_traj + 2 * (size_t)t * cap, out[t].data(), sizeof(double) * 2 * n);
  return HEOM_OK;
}

int heom_scan_layout(const heom_plan *pl, const heom_scan_point *pts, int n, long long *offsets, int *counts,
                     long long *total) {
  if (!pl || (!pts && n > 0) || !offsets || !counts || n < 0) return fail(HEOM_ERR_ARG, "bad argument");
  if (pl->prob.dynamics) return fail(HEOM_ERR_UNSUPPORTED, "a population-dynamics plan runs heom_run_populations only");
  long long off = 0;
  for (int i = 0; i < n; i++) {
    offsets[i] = off;
    counts[i] = heom::count_records(pl->prob, pts[i].tau3, pts[i].t_end);
    off += counts[i];
  }
  if (total) *total = off;
  return HEOM_OK;
}

int heom_run_scan(heom_plan *pl, const heom_scan_point *pts, int n, double *P, const long long *offsets,
                  const int *counts) {
  if (!pl || (!pts && n > 0) || !P || !offsets || !counts || n < 0) return fail(HEOM_ERR_ARG, "bad argument");
  if (pl->prob.dynamics) return fail(HEOM_ERR_UNSUPPORTED, "a population-dynamics plan runs heom_run_populations only");
  if (n > pl->max_points) return fail(HEOM_ERR_CAPACITY, "more scan points than the plan's max_points");
  CK(cudaSetDevice(pl->device));
  long long total = 0;
  for (int i = 0; i < n; i++) total = std::max(total, offsets[i] + counts[i]);
  if (!pl->scan.supported) // hierarchy too large for one CTA: staged path
    return run_sg(pl, 4, nullptr, pts, n, P, offsets, total);
  const long long before = pl->scan.staged_launches, checks = pl->scan.check_launches;
  int rc = heom_dev::scan_run_host(pl->scan, pts, n, P, offsets, total, pl->stream);
  if (rc) return fail(rc, heom_dev::scan_last_error());
  pl->launches += pl->scan.staged ? pl->scan.staged_launches - before : heom_dev::scan_launches_per_run(pl->scan);
  pl->launches += pl->scan.check_launches - checks;
  return HEOM_OK;
}

int heom_host_alloc(size_t bytes, void **ptr) {
  if (!ptr) return fail(HEOM_ERR_ARG, "bad argument");
  int rc = heom_dev::host_alloc(bytes, ptr);
  if (rc) return fail(rc, heom_dev::scan_last_error());
  return HEOM_OK;
}

int heom_host_free(void *ptr) {
  if (!ptr) return HEOM_OK;
  int rc = heom_dev::host_free(ptr);
  if (rc) return fail(rc, heom_dev::scan_last_error());
  return HEOM_OK;
}

int heom_run_scan_device(heom_plan *pl, const heom_scan_point *d_pts, int n, double *d_P, const long long *d_offsets) {
  if (!pl || (!d_pts && n > 0) || !d_P || !d_offsets || n < 0) return fail(HEOM_ERR_ARG, "bad argument");
  if (pl->prob.dynamics) return fail(HEOM_ERR_UNSUPPORTED, "a population-dynamics plan runs heom_run_populations only");
  if (n > pl->max_points) return fail(HEOM_ERR_CAPACITY, "more scan points than the plan's max_points");
  CK(cudaSetDevice(pl->device));
  const long long before = pl->scan.staged_launches;
  int rc = heom_dev::scan_run_device(pl->scan, d_pts, n, d_P, d_offsets, pl->stream);
  if (rc) return fail(rc, heom_dev::scan_last_error());
  pl->launches += pl->scan.staged ? pl->scan.staged_launches - before : heom_dev::scan_launches_per_run(pl->scan);
  return HEOM_OK;
}

int heom_plan_sync(heom_plan *pl) {
  if (!pl) return fail(HEOM_ERR_ARG, "null plan");
  CK(cudaSetDevice(pl->device));
  if (pl->prob.dynamics || !pl->scan.supported) {
    CK(cudaStreamSynchronize(pl->stream));
    return HEOM_OK;
  }
  int rc = heom_dev::scan_sync(pl->scan, pl->stream);
  if (rc) return fail(rc, heom_dev::scan_last_error());
  return HEOM_OK;
}

int heom_plan_inject_wait_fault(heom_plan *pl, unsigned long long wait_ns, int unmet) {
  if (!pl) return fail(HEOM_ERR_ARG, "null plan");
  if (!pl->scan.supported || !pl->scan.staged) return fail(HEOM_ERR_UNSUPPORTED, "the plan does not run staged scans");
  if (wait_ns == 0 || wait_ns > 60ull * 1000 * 1000 * 1000) return fail(HEOM_ERR_ARG, "wait limit outside (0, 60 s]");
  pl->scan.inject_wait_ns = wait_ns;
  pl->scan.inject_unmet = unmet != 0;
  return HEOM_OK;
}

long long heom_plan_scan_work(const heom_plan *pl) {
  if (!pl) return fail(HEOM_ERR_ARG, "null plan");
  return pl->scan.staged ? pl->scan.last_work : 0;
}

int heom_problem_param_count(const heom_problem *h) {
  if (!h) return fail(HEOM_ERR_ARG, "null problem");
  return heom::n_params(h->p);
}

int heom_problem_param_dH(const heom_problem *h, int i, double *dH) {
  if (!h || !dH) return fail(HEOM_ERR_ARG, "null argument");
  if (i < 0 || i >= heom::n_params(h->p)) return fail(HEOM_ERR_ARG, "parameter index out of range");
  heom::cbuf D;
  heom::param_dH(h->p, i, D);
  std::memcpy(dH, D.data(), sizeof(double) * D.size());
  return HEOM_OK;
}

int heom_problem_set_bath_scale(heom_problem *h, int site, int line, double scale) {
  if (!h) return fail(HEOM_ERR_ARG, "null problem");
  heom::Problem &p = h->p;
  if (site < 0 || site >= p.K || line < 0 || line >= p.K_m || !(scale > 0)) return fail(HEOM_ERR_ARG, "bad site/line/scale");
  p.bath_scale[(size_t)site * p.K_m + line] = scale;
  heom::build_hierarchy(p);
  return HEOM_OK;
}

int heom_adjoint_scan(heom_plan *pl, const heom_scan_point *pts, int n, const long long *offsets, long long total,
                      const double *dLdP, double *P, double *grad) {
  if (!pl || (!pts && n > 0) || !offsets || !dLdP || !P || !grad || n < 0 || total < 0)
    return fail(HEOM_ERR_ARG, "bad argument");
  if (pl->prob.dynamics) return fail(HEOM_ERR_UNSUPPORTED, "a population-dynamics plan runs heom_run_populations only");
  CK(cudaSetDevice(pl->device));
  int rc = heom_dev::adjoint_scan(pl->prob, pts, n, offsets, total, dLdP, P, grad, &pl->launches, pl->stream);
  if (rc) return fail(rc, heom_dev::adj_last_error());
  for (long long q = 0; q < 2 * total; q++)
    if (!std::isfinite(P[q])) return fail(HEOM_ERR_NUMERIC, "non-finite P(t) in the adjoint forward pass");
  return HEOM_OK;
}

int heom_plan_describe(const heom_plan *pl, char *buf, int len) {
  if (!pl || !buf || len <= 0) return fail(HEOM_ERR_ARG, "bad argument");
  std::snprintf(buf, (size_t)len, "%s", pl->desc.c_str());
  return HEOM_OK;
}
long long heom_plan_launch_count(const heom_plan *pl) { return pl ? pl->launches : -1; }
void heom_plan_destroy(heom_plan *pl) {
  if (!pl) return;
  cudaSetDevice(pl->device);
  if (pl->stream) cudaStreamSynchronize(pl->stream);
  delete pl;
}

} // extern "C"
