// Host-side model of one HEOM-ETO 2DES problem: key-file contents, the current
// disorder/orientation sample, the auxiliary-density-operator (ADO) hierarchy and
// the per-step schedules the kernels consume.  No CUDA types here.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace heom {

// Interleaved complex128 storage, row-major N x N for matrices.
using cbuf = std::vector<double>;

struct Pulse {
  double E0 = 0, tau0 = 0, taup = 0, w0 = 0; // E0, w0 divided by hbar (param.cpp:319-320)
};

// MT19937 with GSL's seeding (gsl_rng_set) and the two distributions the
// reference draws from (gsl_ran_gaussian, gsl_ran_dir_3d).
struct Rng {
  unsigned long mt[624];
  int mti = 625;
  void seed(unsigned long s);
  unsigned long next();
  double uniform();
  double uniform_pos();
  double gaussian(double sigma);
  void dir3d(double *x, double *y, double *z);
};

// One coupling of an ADO to a hierarchy neighbour, in the reference's
// accumulation order (dynamics.cpp:143-179).  It adds coef * rho_nb[r][c] to the
// elements of row s (kind == kRow) or column s (kind == kCol).
struct CouplingOp {
  enum : int32_t { kCol = 0, kRow = 1 };
  int32_t kind, s, nb, pad;
  double cr, ci;
};

struct Problem {
  // --- key file (CPU parser semantics, param.cpp:102-332)
  int single_size = 0, sys_size = 0, K = 0, K_m = 0, L = 0, n_sample = 0;
  unsigned long seed = 0;
  bool single_manifold = false;
  // Population-dynamics key (param_dynamics): every level is a site and site j's
  // coupling operator S_j = |j><j|; 2DES keys put the ground state at level 0 and
  // S_j = |j+1><j+1|.  level0 is the level of site 1's S (0 or 1).
  bool dynamics = false;
  int level0 = 1;
  std::vector<int> d_a, d_b;    // two-exciton level -> (a, b) (param.cpp:127-135)
  cbuf Hkey, Dis, Xx, Xy, Xz;   // N x N
  double angle[4] = {0, 0, 0, 0};
  bool have_polar = false, have_dipole = false, have_bath = false, have_pulse = false;
  std::vector<double> alpha, alpha_t, gamma; // K_m complex (same for every site)
  // Per (site j, line k) amplitude scale: alpha_jk = bath_scale[j*K_m + k] * alpha_k.  The
  // reference stores alpha per site (param.h:70); its parser fills identical copies, i.e.
  // every scale is 1.  The scales are the ETO amplitude parameters of the adjoint.
  std::vector<double> bath_scale;
  Pulse pulses[3];
  float t_start = 0, t_end = 0, step_size = 0, print_step = 0;

  // --- current sample (construct_Hal + compute_pulse_interaction)
  cbuf H, X[4];
  Rng rng;

  // --- hierarchy (utilize.cpp:3-36)
  int M = 0, n_ado = 0;
  std::vector<uint8_t> ado;     // n_ado x M digits
  std::vector<int> up, dn;      // n_ado x M neighbour index, -1 if absent
  std::vector<int> depth;       // sum of digits per ADO
  std::vector<double> damp;     // n_ado complex: -sum n*gamma in reference order
  std::vector<int> op_start;    // n_ado + 1 offsets into ops
  std::vector<CouplingOp> ops;  // per-ADO coupling list

  int N() const { return sys_size; }
  int n_steps() const;          // floor(nstep) + 1 with float nstep (dynamics.cpp:344-347)
  int print_stride() const { return (int)(print_step / step_size); }
};

// Parse; on failure returns false and fills err.  Status code in *code.
bool parse_key(const std::string &path, int flags, Problem &p, std::string &err, int *code);

// Complex amplitude of line k on site j (alpha_jk).
void bath_alpha(const Problem &p, int j, int k, double *ar, double *ai);
// Up/down hierarchy coefficients of ADO n, offset o = j + k K, as the staged and scan
// kernels tabulate them: x = sqrt((n_o + 1) |alpha_jk|), y = sqrt(n_o / |alpha_jk|) *
// scale_jk (so that y * alpha_k = sqrt(n_o/|alpha_jk|) alpha_jk).
double coupling_x(const Problem &p, int n, int o);
double coupling_y(const Problem &p, int n, int o);

// Gradient parameters: site energies eps_1..eps_{s-1} (cm^-1), couplings J_ab (a < b,
// row-major, cm^-1), bath amplitude scales (j outer, k inner).
int n_params(const Problem &p);
// dH/dtheta_i (N x N complex) for the Hamiltonian parameters (zero for bath scales),
// through construct_Hal's two-exciton block with the diagonal sort permutation held
// fixed at the key's order.
void param_dH(const Problem &p, int i, cbuf &dH);
// Build ADO list, neighbour tables, damping scalars and coupling ops.
void build_hierarchy(Problem &p);
// construct_Hal (draw = true: disorder from the RNG) then orientation (rotate).
void prepare_sample(Problem &p, bool draw, bool rotate);

// Field factor of pulse q at float time t, exactly as build_V_matrix /
// build_V_dagger_matrix compute it (TD_hamiltonian.cpp:5-31).
void pulse_field(const Pulse &q, float t, bool dagger, double *er, double *ei);

// Per-step schedule of one trajectory (dynamics.cpp:344-367): for step i, bit q
// of flags[i] says pulse q+1 is on, bit 3 says P is recorded before the step;
// field[(q*n + i)*2] holds the complex field factor where pulse q+1 is on.
struct Schedule {
  int n_steps = 0, n_record = 0;
  std::vector<uint8_t> flags;
  std::vector<int> rec_idx;  // output slot of the P recorded before step i, or -1
  std::vector<double> field; // 3 x n_steps complex
};
Schedule make_schedule(const Problem &p, const double tau[3], float t_end, const int nv[3]);
int count_records(const Problem &p, double tau3, float t_end);
int steps_for(const Problem &p, float t_end);

// Sets the thread-local message returned by heom_last_error(); returns code.
int set_error(int code, const std::string &msg);

} // namespace heom

// The opaque handle of the C ABI.
struct heom_problem {
  heom::Problem p;
};
