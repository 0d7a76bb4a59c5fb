/* heom.h -- C ABI of the B200-native HEOM-ETO 2DES propagation library (libheom.so).
 *
 * Drop-in for the propagation path of KaiChengLiu/ETO-HEOM.  The reference exposes
 * that path as C++ functions over its `param` class (no C ABI):
 *   param::param_2des(string)            etoheom-cpu/lib/param.h:41, param.cpp:18-248
 *   construct_ADO_set(param&)            etoheom-cpu/lib/utilize.h:18, utilize.cpp:26-36
 *   construct_Hal(param&, H, rng)        etoheom-cpu/lib/dynamics.h:25, dynamics.cpp:3-51
 *   polar_mat_set/_ranrot, compute_pulse_interaction   etoheom-cpu/lib/polar.h:26-30
 *   twoD_spectrum_solver(param&, H, nv1, nv2, nv3, P)  etoheom-cpu/lib/dynamics.h:23,
 *                                        dynamics.cpp:298-432 (GPU: HEOM_dynamics.h:36)
 *   total_ADO_dynamics_Ht(param&, rho, drho, Ht)       etoheom-cpu/lib/dynamics.h:19
 *   CPU_2DES / GPU_2DES main             etoheom-cpu/src/CPU_2DES.cpp:14-91,
 *                                        etoheom-gpu/src/GPU_2DES.cu:25-88
 * Each entry point below names the reference function it replaces.
 *
 * Conventions: every function returns HEOM_OK (0) or a negative HEOM_ERR_* code and
 * never exits the process; heom_last_error() gives a thread-local message.  Complex
 * numbers are interleaved (re, im) doubles; matrices are row-major N x N.  Output
 * buffers are caller-owned host memory unless the name ends in _device.  A plan is
 * bound to one CUDA device and stream and is not thread-safe; distinct plans may run
 * concurrently.  There is no CPU fallback: without a usable CUDA device,
 * heom_plan_create fails with HEOM_ERR_CUDA. */
#ifndef HEOM_H
#define HEOM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define HEOM_ABI_VERSION 1

enum {
  HEOM_OK = 0,
  HEOM_ERR_ARG = -1,          /* bad argument / handle */
  HEOM_ERR_IO = -2,           /* key file unreadable */
  HEOM_ERR_PARSE = -3,        /* key file incomplete or inconsistent */
  HEOM_ERR_CUDA = -4,         /* CUDA runtime failure or no device */
  HEOM_ERR_NOMEM = -5,        /* host or device allocation failed */
  HEOM_ERR_CAPACITY = -6,     /* output buffer too small / size above a limit */
  HEOM_ERR_UNSUPPORTED = -7,  /* option not available for this problem */
  HEOM_ERR_NUMERIC = -8,      /* non-finite value in the propagated state */
  HEOM_ERR_TIMEOUT = -9       /* a bounded device-side wait expired */
};

/* Precision of the propagation. */
enum {
  HEOM_FP64_EXACT = 0, /* FP64, the reference's floating-point operation sequence:
                          bit-identical P(t) to the reference CPU build */
  HEOM_FP64 = 1,       /* FP64 everywhere, fused multiply-add, batched layout */
  HEOM_FP32_BULK = 2   /* commutator and neighbour contractions in FP32 (FP32
                          accumulation); state, RK4 accumulation, damping diagonal,
                          site-energy diagonal and P(t) trace in FP64 */
};

/* Matrix selectors for heom_problem_get_matrix / heom_problem_set_matrix. */
enum { HEOM_MAT_H = 0, HEOM_MAT_X0 = 1, HEOM_MAT_X1 = 2, HEOM_MAT_X2 = 3, HEOM_MAT_X3 = 4,
       HEOM_MAT_HKEY = 5 };

/* heom_problem_from_key flags. */
enum {
  HEOM_KEY_SINGLE_MANIFOLD = 1, /* no two-exciton block (also: MANIFOLD single) */
  HEOM_KEY_DYNAMICS = 2         /* a population-dynamics key (param::param_dynamics,
                                   param.cpp:250-348): SIZE levels, all of them sites,
                                   static H with the reorganisation shift, no disorder,
                                   dipoles or pulses; run with heom_run_populations */
};

typedef struct heom_problem heom_problem;
typedef struct heom_plan heom_plan;

typedef struct {
  int single_size, sys_size; /* SIZE and N = SIZE + (SIZE-1)(SIZE-2)/2 */
  int K, K_m, L, n_ado;      /* sites, bath lines per site, depth, C(K*K_m+L, L) */
  int n_sample;
  unsigned long seed;
  int n_steps;               /* RK4 steps of one trajectory (floor(nstep) + 1) */
  int print_stride;          /* (int)(print_step / step_size) */
  int n_record;              /* recorded P points of one trajectory */
  float t_start, t_end, step_size, print_step;
  double E0[3], tau[3], taup[3], w0[3]; /* pulses, E0 and w0 already divided by hbar */
} heom_problem_info;

/* Parse a key file with the reference CPU parser semantics (replaces
 * param::param_2des, param.cpp:18-248, plus construct_ADO_set, utilize.cpp:26-36,
 * and the RNG seeding of CPU_2DES.cpp:23-29). */
int heom_problem_from_key(const char *path, int flags, heom_problem **out);
int heom_problem_info_get(const heom_problem *p, heom_problem_info *info);
/* Next disorder/orientation sample, drawing from the problem's RNG stream exactly as
 * CPU_2DES.cpp:52-60 does: construct_Hal (dynamics.cpp:3-51), polar_mat_set,
 * polar_mat_ranrot, compute_pulse_interaction (polar.cpp:17-101). */
int heom_problem_prepare_sample(heom_problem *p);
/* 1 if the two problems' key files differ at most in the pulse central times and the end
 * time (the fields script/IO-scripts/gen_2d_data.sh:21-33 substitutes into
 * key.key-tmpl), 0 otherwise: such keys draw the same disorder/orientation samples
 * (same seed, CPU_2DES.cpp:23-29) and can run as one heom_run_scan batch.  No
 * counterpart in the reference, which runs one process per key. */
int heom_problem_scan_compatible(const heom_problem *a, const heom_problem *b);
/* Same without random draws: zero disorder and no orientational rotation. */
int heom_problem_prepare_identity(heom_problem *p);
int heom_problem_reset_rng(heom_problem *p);
int heom_problem_get_matrix(const heom_problem *p, int which, double *out);
int heom_problem_set_matrix(heom_problem *p, int which, const double *in);
/* ADO multi-indices, n_ado x (K*K_m) bytes, in the reference's order. */
int heom_problem_get_ado(const heom_problem *p, unsigned char *out);
void heom_problem_destroy(heom_problem *p);

typedef struct {
  int precision;    /* HEOM_FP64_EXACT / HEOM_FP64 / HEOM_FP32_BULK */
  int device;       /* CUDA device ordinal */
  void *stream;     /* cudaStream_t to run on; NULL = a stream owned by the plan */
  int max_points;   /* capacity of one heom_run_scan call (0 = 1024) */
  int autotune;     /* 1 = time candidate launch shapes at plan creation */
  int single_pass;  /* 1 = propagate every scan point from t_start in one pass; 0 = stage
                       the scan (shared R/D2 per (tau1, tau2) group, per-point pulse-3
                       windows, FP64 jumps over pulse-free gaps, pulse-free tails as FP64
                       dual dot products) where the problem allows it.  The two agree up
                       to rounding, not bit for bit: jumps and dual tails round
                       differently from step-by-step propagation */
} heom_opts;

/* Device plan: uploads H, X[0..3], the ADO neighbour tables and the bath
 * coefficients of the problem's current sample. */
int heom_plan_create(const heom_problem *p, const heom_opts *opts, heom_plan **out);
/* Re-upload H and X[0..3] after heom_problem_prepare_sample. */
int heom_plan_update(heom_plan *plan, const heom_problem *p);

/* One trajectory with pulse mask (nv1, nv2, nv3) (replaces twoD_spectrum_solver,
 * dynamics.cpp:298-432; HEOM_dynamics.cu:489-658).  P receives the recorded
 * Tr(rho_0 X[3]) points, *n_out their count. */
int heom_run_traj(heom_plan *plan, int nv1, int nv2, int nv3, double *P, int cap, int *n_out);

/* Population dynamics (replaces dynamics_solver, dynamics.cpp:202-295, and the
 * CPU_dynamics main, etoheom-cpu/src/CPU_dynamics.cpp:14-50): propagates rho from
 * |1><1| (site 1 excited) under the static H with no fields and records Re rho_0[s][s]
 * for each site s (1-based) every print_step from t_start.  HEOM_FP64_EXACT plans only
 * (bit-identical to the reference build); pop receives [n_sites][cap] values and *n_out
 * the number recorded per site.  Any key works; for a 2DES key the state stays |0><0|. */
int heom_run_populations(heom_plan *plan, const int *sites, int n_sites, double *pop, int cap, int *n_out);

/* One 2DES point of the current sample: trajectories 111, 110, 101 and
 * P = p111 - p110 - p101 (CPU_2DES.cpp:65-79).  p_traj (optional) receives the
 * three trajectories, [3][cap] complex. */
int heom_run_2des(heom_plan *plan, double *P, double *p_traj, int cap, int *n_out);

/* A 2DES delay scan: n independent points (pulse times and end time replace the
 * key file's) in one batched GPU run (replaces one CPU_2DES/GPU_2DES process per key
 * file, script/cpu-script/submit_jobs.sh:49-67).  The default staged form plans its
 * job queue on the host and then issues two plain launches: one persistent kernel over
 * the queue (shared stages, pulse windows and jumps) and the pulse-free tail kernel;
 * the per-sample block powers are formed on the first run after a sample changes.
 * With heom_opts.single_pass = 1 the scan is one persistent kernel launch (after an
 * ordering kernel) replayed from a CUDA graph.  A staged plan keeps its last job plan:
 * a scan with the same points and offsets into the same output buffer, on a sample of
 * the same structure (heom_plan_update between disorder samples), skips the host
 * planning and only resets the queue before its launches; once the sample's dual rows
 * exist, that run is one CUDA graph (captured on its first use, launched after).
 * Output of point i: counts[i] combined P points at P + 2*offsets[i].  heom_scan_layout
 * fills counts/offsets and returns the total number of complex points through *total. */
typedef struct { double tau1, tau2, tau3; float t_end; int flags; } heom_scan_point;
int heom_scan_layout(const heom_plan *plan, const heom_scan_point *pts, int n,
                     long long *offsets, int *counts, long long *total);
int heom_run_scan(heom_plan *plan, const heom_scan_point *pts, int n, double *P,
                  const long long *offsets, const int *counts);
/* Page-locked host memory for heom_run_scan's output (no counterpart in the reference,
 * which prints P).  When P lies inside one buffer from heom_host_alloc, a scan on the
 * batched path (N <= 15) copies the result into it by DMA and checks it for Inf/NaN on
 * the device.  Into any other memory it copies through the plan's own page-locked
 * staging buffer and checks on the host.  The general-size path (larger hierarchies)
 * copies into P directly and checks on the host either way.  The buffer serves any plan
 * on any device; heom_host_free(NULL) is a no-op and freeing an unknown pointer returns
 * HEOM_ERR_ARG. */
int heom_host_alloc(size_t bytes, void **ptr);
int heom_host_free(void *ptr);
/* heom_run_scan with every buffer already in device memory.  A staged scan reads the points and
 * offsets back once to plan its stages (one host synchronisation); a single-pass scan
 * does not synchronise.  Errors found on the device (a dependency wait that expired, a
 * failed device-side check) are deferred: the call returns once the work is queued, and
 * the status reaches the caller through heom_plan_sync, or else through the plan's next
 * scan call.  The outputs of a failed run hold NaN where they depend on the failure. */
int heom_run_scan_device(heom_plan *plan, const heom_scan_point *d_pts, int n, double *d_P,
                         const long long *d_offsets);
/* Waits for the plan's queued work and returns the deferred status of its last
 * heom_run_scan_device call: HEOM_ERR_TIMEOUT when a dependency wait of the staged scan
 * expired, HEOM_ERR_CUDA when a device-side check failed or the stream reports an error.
 * No counterpart in the reference, whose errors exit the process
 * (etoheom-gpu/lib/HEOM_utilize.h:23-38). */
int heom_plan_sync(heom_plan *plan);
/* Test hook for the bounded device-side waits; no counterpart in the reference.  For the
 * plan's next staged scan only, the dependency wait limit becomes wait_ns (default 30 s;
 * at most 60 s), and with unmet != 0 the first job that waits on another job waits for a
 * flag value that no producer sets.  That wait expires after wait_ns: the kernel writes
 * NaN to the job's first records and to the states it would have saved, releases the
 * jobs that wait on it, and the run reports HEOM_ERR_TIMEOUT.  Every memory access stays
 * in bounds; the next run plans afresh and is unaffected. */
int heom_plan_inject_wait_fault(heom_plan *plan, unsigned long long wait_ns, int unmet);

/* Delay scan that performs no device allocation, for callers that cannot let a library
 * allocate device memory (a service that reserves its whole budget at start-up in its own
 * pool or an ML framework's caching allocator, or an application that allows allocation
 * only during initialisation).  No counterpart in the reference.  Same computation as
 * the single-pass form of heom_run_scan_device (heom_opts.single_pass = 1; a staged plan
 * agrees with it to rounding) with the default launch shape, on the caller's current
 * device and the given stream (NULL = legacy default stream); inputs and outputs are the
 * caller's device buffers, the problem comes from the host handle.  Its scratch
 * (work-queue counter, point ordering, packed tables and system matrices) lives in one
 * 4 MiB file-scope device array that every GPU loading the library holds until exit: at
 * most 65536 points per call, and the problem's tables must fit (else
 * HEOM_ERR_CAPACITY).  All calls on a device share that array; calls whose GPU work
 * overlaps race and must be serialised by the caller.  The first call on a device
 * resolves the array's address.  The tables are uploaded from host memory that the call
 * owns (pageable copies), so the call waits for earlier work on the stream before it
 * returns, and it must not be captured into a CUDA graph.  The scan itself is queued
 * and runs asynchronously. */
int heom_run_scan_noalloc(const heom_problem *p, int precision, const heom_scan_point *d_pts, int n,
                          double *d_P, const long long *d_offsets, void *stream);

/* Gradient parameters of a problem, in this order: the site energies eps_1..eps_{s-1}
 * (cm^-1, HAMILTONIAN diagonal), the couplings J_ab for a < b (cm^-1, row-major), and the
 * bath amplitude scales s_jk (site j < K outer, line k < K_m inner; alpha_jk = s_jk alpha_k,
 * 1 as parsed -- the reference keeps alpha per site, param.h:70).  No counterpart in the
 * reference, which has no gradients. */
int heom_problem_param_count(const heom_problem *p);
/* dH/dtheta_i (N x N complex, fs^-1 per cm^-1) through construct_Hal's two-exciton block,
 * the diagonal sort held at the key's order; zero for bath scales. */
int heom_problem_param_dH(const heom_problem *p, int i, double *dH);
/* Set s_jk; plans created afterwards use it. */
int heom_problem_set_bath_scale(heom_problem *p, int site, int line, double scale);

/* Adjoint gradient of a delay scan (config-4 style fitting).  Runs the scan forward in FP64
 * (mixed-difference basis, P = p111 - p110 - p101 into P, layout of heom_scan_layout) and
 * the discrete adjoint of its RK4 steps backwards with checkpoints every ceil(sqrt(steps))
 * steps, and returns grad_i = d/dtheta_i Re sum_t conj(dLdP_t) P_t for the parameters of
 * heom_problem_param_count (dLdP: complex gradient of a real objective with respect to each
 * recorded P).  No counterpart in the reference. */
int heom_adjoint_scan(heom_plan *plan, const heom_scan_point *pts, int n, const long long *offsets,
                      long long total, const double *dLdP, double *P, double *grad);

/* Launch shape chosen by the autotuner for this plan ("threads/CTA, CTAs/SM"). */
int heom_plan_describe(const heom_plan *plan, char *buf, int len);
/* Component-steps propagated by the plan's last staged delay scan (one component-step =
 * one RK4 step of one n_ado x N x N state: a reference trajectory step costs the same),
 * or 0 when the last scan ran in a single pass.  Measurement utility; no counterpart in
 * the reference. */
long long heom_plan_scan_work(const heom_plan *plan);
/* Number of device kernel launches issued by this plan since creation. */
long long heom_plan_launch_count(const heom_plan *plan);
void heom_plan_destroy(heom_plan *plan);

const char *heom_last_error(void);
int heom_abi_version(void);

/* Measured FP32 (fp64 = 0) or FP64 (fp64 = 1) FMA throughput of a device in TFLOP/s
 * (2 flops per FMA) -- the roofline denominator for the propagation kernels, which run
 * on the CUDA-core FMA pipes.  Measurement utility; no counterpart in the reference. */
int heom_measure_fma_peak(int device, int fp64, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
