/* CPU oracle for the HEOM-ETO 2DES propagation path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64 restatement of the reference CPU path (KaiChengLiu/ETO-HEOM,
 * etoheom-cpu/).  Only tests/, the smoke check and bench.py's cpu_baseline leg
 * may load it, and only as the checker; the product never routes through it.
 *
 * Parity pin: every function reproduces the reference's floating-point
 * operation sequence, and tests check it bit-for-bit against oracle/_ref/
 * (the reference's own sources compiled against oracle/gslshim).  The GSL
 * random stream is restated from GSL's published algorithms and is unpinned
 * against a real GSL build (GSL is not installed here).
 *
 * Matrices are row-major N x N complex128, interleaved (re, im). */
#ifndef HEOM_ORACLE_H
#define HEOM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ho_problem ho_problem;

enum { HO_DENSE = 0, HO_STRUCTURED = 1 };
enum { HO_H = 0, HO_X0 = 1, HO_X1 = 2, HO_X2 = 3, HO_X3 = 4, HO_HKEY = 5 };

/* Parse a key file with the CPU parser semantics (param.cpp:102-332).
 * single_manifold != 0 drops the two-exciton block (sys_size = SIZE), the
 * extension used for linear-response runs on large single-manifold systems. */
int ho_load_key(const char *path, int single_manifold, ho_problem **out, char *err, int errlen);
void ho_free(ho_problem *p);

/* info[0..9] = single_size, sys_size, K, K_m, L, n_ado, n_sample, n_steps,
 * print_stride, seed (low 31 bits). */
void ho_info(const ho_problem *p, int *info);

void ho_rng_reset(ho_problem *p);       /* gsl_rng_set(r, seed)  (CPU_2DES.cpp:23-29) */
void ho_prepare_sample(ho_problem *p);  /* construct_Hal, polar_mat_set/ranrot, compute_pulse_interaction */
void ho_prepare_identity(ho_problem *p);/* same without disorder draws or rotation */

int ho_get_matrix(const ho_problem *p, int which, double *out);
int ho_set_matrix(ho_problem *p, int which, const double *in);
void ho_get_ado(const ho_problem *p, unsigned char *out); /* n_ado x (K*K_m) */
void ho_get_bath(const ho_problem *p, double *out);       /* K_m x (a, b, g, w) */

/* F(rho) of total_ADO_dynamics_Ht (dynamics.cpp:117-179) for a given V. */
void ho_rhs(ho_problem *p, const double *V, const double *rho, double *drho, int mode);

/* One twoD_spectrum_solver trajectory (dynamics.cpp:298-419).
 * P receives up to cap recorded points (interleaved); *npts the count.
 * max_steps > 0 stops after that many steps (truncated parity runs). */
int ho_traj(ho_problem *p, int nv1, int nv2, int nv3, int mode, int max_steps,
            double *P, int cap, int *npts);

/* The whole CPU_2DES flow (CPU_2DES.cpp:14-91): for every sample,
 * construct_Hal + orientation + 3 trajectories, combine, average.
 * traj (optional) receives [n_sample][3][cap] complex points. */
int ho_2des(ho_problem *p, int mode, int max_steps, double *P, int cap, int *npts, double *traj);

/* ho_2des with the propagation, trace and combination in IEEE binary128 on the
 * reference's double-precision problem data: the true result of the reference's
 * discrete scheme (~1e-24 relative on the combined output), rounded to double.
 * Same arguments as ho_2des (no mode: the RHS is the structured form). */
int ho_2des_q(ho_problem *p, int max_steps, double *P, int cap, int *npts, double *traj);
/* One binary128 trajectory (mask nv1 nv2 nv3) of the first sample, each value as a
 * (hi, lo) double pair, so that separately run trajectories combine exactly. */
int ho_traj_q_split(ho_problem *p, int nv1, int nv2, int nv3, int max_steps, double *P_hi, double *P_lo, int cap,
                    int *npts);

#ifdef __cplusplus
}
#endif
#endif
