// Key-file parser, hierarchy builder and sample preparation.
//
// Semantics follow the reference CPU build (etoheom-cpu/lib), which is the
// authoritative one (the GPU build reads DISORDER and HAMILTONIAN with other row
// counts, etoheom-gpu/lib/HEOM_param.cu:50,69).  Built with -ffp-contract=off:
// every coefficient computed here must round exactly as the reference does.
#include "heom_host.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>

#include "../../include/heom.h"

namespace heom {

static const double kHbar = 5.308e3;                                     // constant.cpp:9
static const double kPi = 3.141592653589793238462643383279502884L;       // constant.cpp:11

static inline double &re(cbuf &m, int N, int i, int j) { return m[2 * ((size_t)i * N + j)]; }
static inline double &im(cbuf &m, int N, int i, int j) { return m[2 * ((size_t)i * N + j) + 1]; }
static inline double re(const cbuf &m, int N, int i, int j) { return m[2 * ((size_t)i * N + j)]; }

// ------------------------------------------------------------------ RNG
void Rng::seed(unsigned long s) {
  if (s == 0) s = 4357; // gsl_rng_set maps seed 0 to the generator default
  mt[0] = s & 0xffffffffUL;
  for (int i = 1; i < 624; i++)
    mt[i] = (1812433253UL * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (unsigned long)i) & 0xffffffffUL;
  mti = 624;
}
unsigned long Rng::next() {
  if (mti >= 624) {
    for (int k = 0; k < 624; k++) {
      unsigned long y = (mt[k] & 0x80000000UL) | (mt[(k + 1) % 624] & 0x7fffffffUL);
      mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1UL) ? 0x9908b0dfUL : 0UL);
    }
    mti = 0;
  }
  unsigned long k = mt[mti++];
  k ^= k >> 11;
  k ^= (k << 7) & 0x9d2c5680UL;
  k ^= (k << 15) & 0xefc60000UL;
  k ^= k >> 18;
  return k & 0xffffffffUL;
}
double Rng::uniform() { return next() / 4294967296.0; }
double Rng::uniform_pos() {
  double x;
  do x = uniform(); while (x == 0);
  return x;
}
double Rng::gaussian(double sigma) { // polar (Marsaglia) method
  double x, y, r2;
  do {
    x = -1 + 2 * uniform_pos();
    y = -1 + 2 * uniform_pos();
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0);
  return sigma * y * std::sqrt(-2.0 * std::log(r2) / r2);
}
void Rng::dir3d(double *x, double *y, double *z) { // Knuth's method
  double s;
  do {
    *x = -1 + 2 * uniform();
    *y = -1 + 2 * uniform();
    s = (*x) * (*x) + (*y) * (*y);
  } while (s > 1.0);
  *z = -1 + 2 * s;
  double a = 2 * std::sqrt(1 - s);
  *x *= a;
  *y *= a;
}

// ------------------------------------------------------------------ parser
namespace {
struct Reader {
  std::ifstream f;
  std::string line;
  bool next() { return (bool)std::getline(f, line); }
};
} // namespace

// Population-dynamics key file: param::param_dynamics (param.cpp:250-348).  Every level
// is a site; the bath's reorganisation energy shifts the first K diagonal elements; the
// state starts in |1><1| (reset_rho) and evolves under the static H.
static bool parse_key_dynamics(const std::string &path, Problem &p, std::string &err, int *code) {
  Reader rd;
  rd.f.open(path);
  if (!rd.f) {
    err = "cannot open key file '" + path + "'";
    *code = HEOM_ERR_IO;
    return false;
  }
  p = Problem();
  p.dynamics = true;
  p.level0 = 0;
  p.single_manifold = true;
  bool saw_size = false, saw_ham = false, saw_time = false;
  std::string kw;
  auto fail = [&](const std::string &m) { err = m; *code = HEOM_ERR_PARSE; return false; };
  while (rd.next()) {
    const std::string &line = rd.line;
    if (line.empty() || line[0] == '#') continue;
    { std::istringstream iss(line); iss >> kw; }
    if (kw == "HEOM") {
      rd.next();
      std::istringstream v(rd.line);
      v >> p.K >> p.L;
    } else if (kw == "SIZE") {
      rd.next();
      std::istringstream v(rd.line);
      v >> p.single_size;
      if (p.single_size < 1 || p.single_size > 64) return fail("SIZE must be between 1 and 64");
      p.sys_size = p.single_size;
      p.d_a.assign(p.sys_size, 0);
      p.d_b.assign(p.sys_size, 0);
      saw_size = true;
    } else if (kw == "HAMILTONIAN") {
      if (!saw_size) return fail("HAMILTONIAN before SIZE");
      const int N = p.sys_size;
      p.Hkey.assign(2 * (size_t)N * N, 0.0);
      for (int i = 0; i < p.single_size; i++) {
        rd.next();
        std::istringstream row(rd.line);
        double x;
        for (int j = 0; row >> x; j++)
          if (j < N) re(p.Hkey, N, i, j) = x / kHbar;
      }
      saw_ham = true;
    } else if (kw == "TEMPERATURE") {
      rd.next(); // beta is not used by the propagation
    } else if (kw == "BATH") {
      if (!saw_ham) return fail("BATH before HAMILTONIAN (the reorganisation shift needs H)");
      rd.next();
      double l = 0;
      { std::istringstream v(rd.line); v >> l; }
      const int N = p.sys_size;
      if (p.K < 1 || p.K > N) return fail("HEOM K must be between 1 and SIZE");
      for (int i = 0; i < p.K; i++) { // param.cpp:309: H_ii <- Re H_ii + lambda
        re(p.Hkey, N, i, i) = re(p.Hkey, N, i, i) + l;
        im(p.Hkey, N, i, i) = 0.0;
      }
      rd.next();
      int nm = 0;
      { std::istringstream v(rd.line); v >> nm; }
      if (nm < 1 || nm > 64) return fail("BATH line count must be between 1 and 64");
      p.alpha.assign(2 * nm, 0.0);
      p.alpha_t.assign(2 * nm, 0.0);
      p.gamma.assign(2 * nm, 0.0);
      for (int k = 0; k < nm; k++) {
        rd.next();
        std::istringstream v(rd.line);
        double a = 0, b = 0, g = 0, w = 0;
        v >> a >> b >> g >> w;
        p.alpha[2 * k] = a; p.alpha[2 * k + 1] = b;
        p.alpha_t[2 * k] = a; p.alpha_t[2 * k + 1] = -b;
        p.gamma[2 * k] = g; p.gamma[2 * k + 1] = w;
      }
      p.K_m = nm;
      p.have_bath = true;
    } else if (kw == "TIME") {
      rd.next();
      std::istringstream v(rd.line);
      v >> p.t_start >> p.t_end >> p.step_size >> p.print_step;
      saw_time = true;
    }
  }
  if (!saw_size || !saw_ham) return fail("key file lacks SIZE or HAMILTONIAN");
  if (!p.have_bath) return fail("key file lacks a BATH block");
  if (!saw_time || !(p.step_size > 0) || p.print_stride() <= 0 || !(p.t_end >= p.t_start))
    return fail("TIME needs t_end >= t_start, step_size > 0 and print_step >= step_size");
  if (p.L < 0 || p.L > 32) return fail("HEOM depth L must be between 0 and 32");
  if (p.K * p.K_m > 255) return fail("K * K_m above 255");
  p.n_sample = 1;
  p.bath_scale.assign((size_t)p.K * p.K_m, 1.0);
  build_hierarchy(p);
  if (p.n_ado <= 0) return fail("empty hierarchy");
  p.H = p.Hkey;
  for (auto &X : p.X) X.assign(2 * (size_t)p.N() * p.N(), 0.0);
  for (Pulse &q : p.pulses) q.taup = 1.0;
  return true;
}

bool parse_key(const std::string &path, int flags, Problem &p, std::string &err, int *code) {
  if (flags & HEOM_KEY_DYNAMICS) return parse_key_dynamics(path, p, err, code);
  Reader rd;
  rd.f.open(path);
  if (!rd.f) {
    err = "cannot open key file '" + path + "'";
    *code = HEOM_ERR_IO;
    return false;
  }
  p = Problem();
  p.single_manifold = (flags & HEOM_KEY_SINGLE_MANIFOLD) != 0;
  bool saw_size = false, saw_ham = false, saw_dis = false, saw_time = false;
  // Unknown keywords are skipped; a whitespace-only line leaves the previous
  // keyword in place, as `iss >> key_word` does in param.cpp:106-109.
  std::string kw;
  auto fail = [&](const std::string &m) { err = m; *code = HEOM_ERR_PARSE; return false; };
  // MANIFOLD may appear anywhere; pre-scan so SIZE can size the matrices.
  {
    std::ifstream g(path);
    std::string ln, w, v;
    while (std::getline(g, ln)) {
      std::istringstream s(ln);
      if (s >> w && w == "MANIFOLD" && std::getline(g, ln)) {
        std::istringstream s2(ln);
        if (s2 >> v && v == "single") p.single_manifold = true;
      }
    }
  }
  while (rd.next()) {
    const std::string &line = rd.line;
    if (line.empty() || line[0] == '#') continue;
    { std::istringstream iss(line); iss >> kw; }
    if (kw == "HEOM") {
      rd.next();
      std::istringstream v(rd.line);
      v >> p.K >> p.L;
    } else if (kw == "SIZE") {
      rd.next();
      std::istringstream v(rd.line);
      v >> p.single_size;
      int s = p.single_size;
      if (s < 1 || s > 64) return fail("SIZE must be between 1 and 64");
      p.sys_size = p.single_manifold ? s : s + (s - 1) * (s - 2) / 2;
      p.d_a.assign(p.sys_size, 0);
      p.d_b.assign(p.sys_size, 0);
      if (!p.single_manifold) {
        int ct = s;
        for (int i = 1; i < s; i++)
          for (int j = i; j < s; j++)
            if (i != j) { p.d_a[ct] = i; p.d_b[ct] = j; ct++; }
      }
      saw_size = true;
    } else if (kw == "MANIFOLD") {
      rd.next(); // handled by the pre-scan
    } else if (kw == "DISORDER") {
      if (!saw_size) return fail("DISORDER before SIZE");
      rd.next();
      std::istringstream v(rd.line);
      v >> p.n_sample >> p.seed;
      int N = p.sys_size;
      p.Dis.assign(2 * (size_t)N * N, 0.0);
      for (int i = 0; i < N; i++) { // the CPU parser reads sys_size rows (param.cpp:145)
        rd.next();
        std::istringstream row(rd.line);
        double x;
        for (int j = 0; row >> x; j++)
          if (j < N) re(p.Dis, N, i, j) = x / kHbar;
      }
      saw_dis = true;
    } else if (kw == "HAMILTONIAN") {
      if (!saw_size) return fail("HAMILTONIAN before SIZE");
      int N = p.sys_size;
      p.Hkey.assign(2 * (size_t)N * N, 0.0);
      for (int i = 0; i < p.single_size; i++) {
        rd.next();
        std::istringstream row(rd.line);
        double x;
        for (int j = 0; row >> x; j++)
          if (j < N) re(p.Hkey, N, i, j) = x / kHbar;
      }
      saw_ham = true;
    } else if (kw == "DIPOLE") {
      if (!saw_size) return fail("DIPOLE before SIZE");
      rd.next();
      int nd = 0;
      { std::istringstream v(rd.line); v >> nd; }
      int N = p.sys_size;
      p.Xx.assign(2 * (size_t)N * N, 0.0);
      p.Xy.assign(2 * (size_t)N * N, 0.0);
      p.Xz.assign(2 * (size_t)N * N, 0.0);
      for (int k = 0; k < nd; k++) {
        rd.next();
        std::istringstream v(rd.line);
        int i = 0, j = 0;
        double x = 0, y = 0, z = 0;
        v >> i >> j >> x >> y >> z;
        if (i < 0 || j < 0 || i >= N || j >= N) return fail("DIPOLE index out of range");
        re(p.Xx, N, i, j) = x;
        re(p.Xy, N, i, j) = y;
        re(p.Xz, N, i, j) = z;
      }
      // Two-exciton columns from the ground-row dipoles (param.cpp:200-230).
      cbuf *XS[3] = {&p.Xx, &p.Xy, &p.Xz};
      for (cbuf *X : XS)
        for (int i = 0; i < N; i++)
          for (int j = p.single_size; j < N; j++) {
            int a = p.d_a[j], b = p.d_b[j];
            double x1 = re(*X, N, 0, a), x2 = re(*X, N, 0, b);
            re(*X, N, i, j) = (b == i ? 1.0 : 0.0) * x1 + (a == i ? 1.0 : 0.0) * x2;
            im(*X, N, i, j) = 0.0;
          }
      p.have_dipole = true;
    } else if (kw == "POLARIZATION") {
      rd.next();
      std::istringstream v(rd.line);
      double a[4] = {0, 0, 0, 0};
      v >> a[0] >> a[1] >> a[2] >> a[3];
      for (int i = 0; i < 4; i++) p.angle[i] = a[i] * kPi / 180;
      p.have_polar = true;
    } else if (kw == "TEMPERATURE") {
      rd.next(); // beta enters only a commented-out correction (dynamics.cpp:180-197)
    } else if (kw == "BATH") {
      if (!saw_ham) return fail("BATH before HAMILTONIAN (the reorganisation shift needs H)");
      rd.next();
      double l = 0;
      { std::istringstream v(rd.line); v >> l; }
      int N = p.sys_size;
      for (int i = 0; i < p.K; i++) // param.cpp:273: lambda on the single-excitation diagonal
        if (i + 1 < N) re(p.Hkey, N, i + 1, i + 1) = re(p.Hkey, N, i + 1, i + 1) + l;
      rd.next();
      int nm = 0;
      { std::istringstream v(rd.line); v >> nm; }
      if (nm < 1 || nm > 64) return fail("BATH line count must be between 1 and 64");
      p.alpha.assign(2 * nm, 0.0);
      p.alpha_t.assign(2 * nm, 0.0);
      p.gamma.assign(2 * nm, 0.0);
      for (int k = 0; k < nm; k++) {
        rd.next();
        std::istringstream v(rd.line);
        double a = 0, b = 0, g = 0, w = 0;
        v >> a >> b >> g >> w;
        p.alpha[2 * k] = a; p.alpha[2 * k + 1] = b;
        p.alpha_t[2 * k] = a; p.alpha_t[2 * k + 1] = -b;
        p.gamma[2 * k] = g; p.gamma[2 * k + 1] = w;
      }
      p.K_m = nm;
      p.have_bath = true;
    } else if (kw == "PULSE") {
      rd.next();
      int n = 0;
      { std::istringstream v(rd.line); v >> n; }
      if (n != 3) return fail("Only support 3 pulses simulation."); // param.cpp:311-314
      for (int i = 0; i < 3; i++) {
        rd.next();
        std::istringstream v(rd.line);
        Pulse &q = p.pulses[i];
        v >> q.E0 >> q.tau0 >> q.taup >> q.w0;
        q.w0 = q.w0 / kHbar;
        q.E0 = q.E0 / kHbar;
      }
      p.have_pulse = true;
    } else if (kw == "TIME") {
      rd.next();
      std::istringstream v(rd.line);
      v >> p.t_start >> p.t_end >> p.step_size >> p.print_step;
      saw_time = true;
    }
  }
  // Sections without which the reference crashes or exits (polar.cpp:75-78,
  // CPU_2DES.cpp:83 with n_sample = 0, dynamics.cpp:15 with no DISORDER).
  if (!saw_size || !saw_ham) return fail("key file lacks SIZE or HAMILTONIAN");
  if (!p.have_bath) return fail("key file lacks a BATH block");
  if (!saw_dis || p.n_sample <= 0) return fail("key file lacks a DISORDER block with n_sample > 0");
  if (!p.have_dipole) return fail("key file lacks DIPOLE");
  if (!p.have_polar) return fail("key file lacks POLARIZATION");
  if (!p.have_pulse) return fail("key file lacks PULSE");
  if (!saw_time || !(p.step_size > 0) || p.print_stride() <= 0 || !(p.t_end >= p.t_start))
    return fail("TIME needs t_end >= t_start, step_size > 0 and print_step >= step_size");
  if (p.K < 1 || p.K > p.single_size - 1) return fail("HEOM K must be between 1 and SIZE-1");
  if (p.L < 0 || p.L > 32) return fail("HEOM depth L must be between 0 and 32");
  if (p.K * p.K_m > 255) return fail("K * K_m above 255");
  p.bath_scale.assign((size_t)p.K * p.K_m, 1.0);
  build_hierarchy(p);
  if (p.n_ado <= 0) return fail("empty hierarchy");
  p.H.assign(2 * (size_t)p.N() * p.N(), 0.0);
  for (auto &X : p.X) X.assign(2 * (size_t)p.N() * p.N(), 0.0);
  p.rng.seed(p.seed);
  return true;
}

// ------------------------------------------------------------------ hierarchy
static long long binom(int n, int k) {
  long long r = 1;
  for (int i = 1; i <= k; i++) { r = r * (n - k + i) / i; if (r > (1LL << 40)) return r; }
  return r;
}

void build_hierarchy(Problem &p) {
  const int M = p.K * p.K_m, L = p.L;
  p.M = M;
  long long count = binom(M + L, L);
  if (count > 50000000LL) { p.n_ado = -1; return; }
  p.n_ado = (int)count;
  p.ado.assign((size_t)count * M, 0);
  // Lexicographic enumeration of digit strings with sum <= L, the order of the
  // recursion in Build_ADO (utilize.cpp:3-18): odometer with the last digit fastest.
  std::vector<uint8_t> cur(M, 0);
  int sum = 0;
  for (long long n = 0; n < count; n++) {
    std::copy(cur.begin(), cur.end(), p.ado.begin() + n * M);
    // Successor: bump the last digit while the sum allows, else carry leftwards.
    if (sum < L) { cur[M - 1]++; sum++; continue; }
    for (int pos = M - 1; pos > 0;) {
      sum -= cur[pos];
      cur[pos] = 0;
      pos--;
      if (sum < L) { cur[pos]++; sum++; break; }
    }
  }
  // Neighbour lookup by binary search over the sorted digit strings.
  auto find = [&](const uint8_t *key) -> int {
    long long lo = 0, hi = count - 1;
    while (lo <= hi) {
      long long mid = (lo + hi) / 2;
      int c = 0;
      const uint8_t *m = &p.ado[mid * M];
      for (int q = 0; q < M && c == 0; q++) c = (int)m[q] - (int)key[q];
      if (c == 0) return (int)mid;
      if (c < 0) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
  };
  p.up.assign((size_t)count * M, -1);
  p.dn.assign((size_t)count * M, -1);
  p.depth.assign(count, 0);
  std::vector<uint8_t> key(M);
  for (long long n = 0; n < count; n++) {
    const uint8_t *a = &p.ado[n * M];
    int d = 0;
    for (int o = 0; o < M; o++) d += a[o];
    p.depth[n] = d;
    for (int o = 0; o < M; o++) {
      std::copy(a, a + M, key.begin());
      if (d < L) { key[o]++; p.up[n * M + o] = find(key.data()); key[o]--; }
      if (a[o] > 0) { key[o]--; p.dn[n * M + o] = find(key.data()); }
    }
  }
  // Damping scalar x = sum over (site j, line k) of -(gamma_k * n) in the order of
  // dynamics.cpp:130-138, complex arithmetic written out as gsl_complex does it.
  const int K = p.K, Km = p.K_m;
  p.damp.assign(2 * count, 0.0);
  for (long long n = 1; n < count; n++) {
    const uint8_t *a = &p.ado[n * M];
    double xr = 0.0, xi = 0.0;
    for (int j = 0; j < K; j++)
      for (int k = 0; k < Km; k++) {
        int off = j + k * K;
        if ((int)a[off] == 0) continue;
        double gr = (double)(int)a[off] * p.gamma[2 * k], gi = (double)(int)a[off] * p.gamma[2 * k + 1];
        double yr = -1.0 * gr - 0.0 * gi, yi = -1.0 * gi + 0.0 * gr;  // MINUS_ONE * (gamma n)
        xr = xr + yr;
        xi = xi + yi;
      }
    p.damp[2 * n] = xr;
    p.damp[2 * n + 1] = xi;
  }
  // Coupling ops in the reference order: all up-neighbours (j outer, k inner;
  // column then row), then all down-neighbours (row then column).
  p.op_start.assign(count + 1, 0);
  p.ops.clear();
  for (long long n = 0; n < count; n++) {
    p.op_start[n] = (int)p.ops.size();
    const uint8_t *a = &p.ado[n * M];
    for (int j = 0; j < K; j++)
      for (int k = 0; k < Km; k++) {
        int off = j + k * K;
        if ((int)a[off] >= L) continue;
        int t = p.up[n * M + off];
        if (t < 0) continue;
        double ajr, aji;
        bath_alpha(p, j, k, &ajr, &aji);
        double x = std::sqrt(((double)a[off] + 1) * std::hypot(ajr, aji));
        // rho+ S_j: coefficient alpha = gsl_complex_mul_real(MINUS_ICNT, x) = (x*0, x*-1).
        const double a1r = x * 0.0, a1i = x * -1.0;
        // S_j rho+: alpha = (x*0, x*1); zgemm first forms temp = alpha * S[s][s].
        const double a2r = x * 0.0, a2i = x * 1.0;
        p.ops.push_back(CouplingOp{CouplingOp::kCol, j + p.level0, t, 0, a1r, a1i});
        p.ops.push_back(CouplingOp{CouplingOp::kRow, j + p.level0, t, 0, a2r * 1.0 - a2i * 0.0, a2r * 0.0 + a2i * 1.0});
      }
    if (n != 0)
      for (int j = 0; j < K; j++)
        for (int k = 0; k < Km; k++) {
          int off = j + k * K;
          if ((int)a[off] <= 0) continue;
          int t = p.dn[n * M + off];
          if (t < 0) continue;
          double ar, ai;
          bath_alpha(p, j, k, &ar, &ai);
          const double sc = p.bath_scale.empty() ? 1.0 : p.bath_scale[(size_t)j * Km + k];
          double y = std::sqrt((double)a[off] / std::hypot(ar, ai));
          double ur = y * ar, ui = y * ai;            // gsl_complex_mul_real(alpha, y)
          double x1r = 0.0 * ur - 1.0 * ui, x1i = 0.0 * ui + 1.0 * ur;   // ICNT * (.)
          double vr = y * (sc * p.alpha_t[2 * k]), vi = y * (sc * p.alpha_t[2 * k + 1]);
          double x2r = 0.0 * vr - (-1.0) * vi, x2i = 0.0 * vi + (-1.0) * vr; // MINUS_ICNT * (.)
          CouplingOp c1{CouplingOp::kRow, j + p.level0, t, 0, x1r * 1.0 - x1i * 0.0, x1r * 0.0 + x1i * 1.0};
          CouplingOp c2{CouplingOp::kCol, j + p.level0, t, 0, x2r, x2i};
          p.ops.push_back(c1);
          p.ops.push_back(c2);
        }
  }
  p.op_start[count] = (int)p.ops.size();
}

int Problem::n_steps() const {
  float nstep = (t_end - t_start) / step_size;
  int n = 0;
  for (int i = 0; i <= nstep; i++) n++;
  return n;
}

int steps_for(const Problem &p, float t_end) {
  float nstep = (t_end - p.t_start) / p.step_size;
  int n = 0;
  for (int i = 0; i <= nstep; i++) n++;
  return n;
}

// ------------------------------------------------------------------ sample
void prepare_sample(Problem &p, bool draw, bool rotate) {
  if (p.dynamics) return; // static H, no orientation: CPU_dynamics draws nothing
  const int N = p.N(), s = p.single_size;
  // construct_Hal (dynamics.cpp:3-51)
  cbuf dH(2 * (size_t)N * N, 0.0);
  for (int i = 0; i < s; i++)
    for (int j = 0; j < s; j++) {
      double sigma = re(p.Dis, N, i, j), t;
      if (std::fabs(sigma) < 1e-10 || !draw) t = 0;
      else t = p.rng.gaussian(sigma);
      re(dH, N, i, j) = t;
    }
  p.H = p.Hkey;
  for (size_t k = 0; k < p.H.size(); k++) p.H[k] += dH[k];
  std::vector<double> Ht(s, 0.0);
  for (int i = 1; i < s; i++) Ht[i] = re(p.H, N, i, i);
  std::sort(Ht.begin(), Ht.end()); // index 0 (= 0.0) takes part in the sort
  for (int i = 1; i < s; i++) { re(p.H, N, i, i) = Ht[i]; im(p.H, N, i, i) = 0.0; }
  if (!p.single_manifold)
    for (int i = s; i < N; i++)
      for (int j = s; j < N; j++) {
        int a = p.d_a[i], b = p.d_b[i];
        if (i == j) {
          double hr = re(p.H, N, a, a) + re(p.H, N, b, b);
          double hi = p.H[2 * ((size_t)a * N + a) + 1] + p.H[2 * ((size_t)b * N + b) + 1];
          re(p.H, N, i, i) = hr;
          im(p.H, N, i, i) = hi;
        } else {
          int c = p.d_a[j], d = p.d_b[j];
          double x1 = (double)(a == c) * (1 - (double)(b == d)) * re(p.H, N, b, d);
          double x2 = (double)(a == d) * (1 - (double)(b == c)) * re(p.H, N, b, c);
          double x3 = (double)(b == c) * (1 - (double)(a == d)) * re(p.H, N, a, d);
          double x4 = (double)(b == d) * (1 - (double)(a == c)) * re(p.H, N, a, c);
          re(p.H, N, i, j) = x1 + x2 + x3 + x4;
          im(p.H, N, i, j) = 0.0;
        }
      }
  // polar_mat_set / polar_mat_ranrot (polar.cpp:17-72)
  double pol[3][4][2];
  for (int i = 0; i < 4; i++) {
    pol[0][i][0] = 0.0; pol[0][i][1] = 0.0;
    pol[1][i][0] = std::sin(p.angle[i]); pol[1][i][1] = 0.0;
    pol[2][i][0] = std::cos(p.angle[i]); pol[2][i][1] = 0.0;
  }
  if (rotate) {
    double a[3] = {0, 0, 0}, b[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    auto norm = [](double *v) {
      double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      v[0] = v[0] / n; v[1] = v[1] / n; v[2] = v[2] / n;
    };
    p.rng.dir3d(c, c + 1, c + 2);
    norm(c);
    p.rng.dir3d(a, a + 1, a + 2);
    double prod = a[0] * c[0] + a[1] * c[1] + a[2] * c[2];
    a[0] = a[0] - prod * c[0]; a[1] = a[1] - prod * c[1]; a[2] = a[2] - prod * c[2];
    norm(a);
    b[0] = c[1] * a[2] - c[2] * a[1];
    b[1] = c[2] * a[0] - c[0] * a[2];
    b[2] = c[0] * a[1] - c[1] * a[0];
    const double R[3][3] = {{a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]}};
    // zgemm(ONE, R, pol, ZERO, tmp): temp = ONE*R[i][l] = (1*r - 0*0, 1*0 + 0*r)
    double tmp[3][4][2] = {};
    for (int i = 0; i < 3; i++)
      for (int l = 0; l < 3; l++) {
        const double tr = 1.0 * R[i][l] - 0.0 * 0.0, ti = 1.0 * 0.0 + 0.0 * R[i][l];
        if (tr == 0.0 && ti == 0.0) continue;
        for (int j = 0; j < 4; j++) {
          tmp[i][j][0] += tr * pol[l][j][0] - ti * pol[l][j][1];
          tmp[i][j][1] += tr * pol[l][j][1] + ti * pol[l][j][0];
        }
      }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 4; j++) { pol[i][j][0] = tmp[i][j][0]; pol[i][j][1] = tmp[i][j][1]; }
  }
  // compute_pulse_interaction (polar.cpp:74-101): X[i] = sum_j pol[j][i] * X_j
  const cbuf *XS[3] = {&p.Xx, &p.Xy, &p.Xz};
  const size_t nn = (size_t)N * N;
  for (int i = 0; i < 4; i++) {
    cbuf &X = p.X[i];
    X.assign(2 * nn, 0.0);
    for (int j = 0; j < 3; j++) {
      const double er = pol[j][i][0], ei = pol[j][i][1];
      const cbuf &S = *XS[j];
      for (size_t k = 0; k < nn; k++) {
        const double ar = S[2 * k], ai = S[2 * k + 1];
        const double mr = ar * er - ai * ei, mi = ar * ei + ai * er; // gsl_matrix_complex_scale
        X[2 * k] += mr;
        X[2 * k + 1] += mi;
      }
    }
  }
}

// ------------------------------------------------------------------ schedule
void pulse_field(const Pulse &q, float t, bool dagger, double *er, double *ei) {
  double E = q.E0 * std::exp(-2.77 * (t - q.tau0) * (t - q.tau0) / q.taup / q.taup);
  double th = dagger ? -q.w0 * (t - q.tau0) : q.w0 * (t - q.tau0);
  *er = E * std::cos(th); // gsl_complex_polar
  *ei = E * std::sin(th);
}

Schedule make_schedule(const Problem &p, const double tau[3], float t_end, const int nv[3]) {
  Schedule s;
  float nstep = (t_end - p.t_start) / p.step_size;
  int n = 0;
  for (int i = 0; i <= nstep; i++) n++;
  s.n_steps = n;
  s.flags.assign(n, 0);
  s.rec_idx.assign(n, -1);
  s.field.assign(2 * 3 * (size_t)n, 0.0);
  const int stride = p.print_stride();
  float t = p.t_start;
  for (int i = 0; i < n; i++) {
    uint8_t f = 0;
    for (int q = 0; q < 3; q++) {
      Pulse pq = p.pulses[q];
      pq.tau0 = tau[q];
      if (nv[q] == 1 && std::fabs(t - pq.tau0) <= pq.taup * 2) {
        f |= (uint8_t)(1u << q);
        pulse_field(pq, t, q > 0, &s.field[2 * ((size_t)q * n + i)], &s.field[2 * ((size_t)q * n + i) + 1]);
      }
    }
    if (t >= tau[2] && i % stride == 0) { f |= 8u; s.rec_idx[i] = s.n_record++; }
    s.flags[i] = f;
    t += p.step_size;
  }
  return s;
}

// ------------------------------------------------------------------ parameters
void bath_alpha(const Problem &p, int j, int k, double *ar, double *ai) {
  const double s = p.bath_scale.empty() ? 1.0 : p.bath_scale[(size_t)j * p.K_m + k];
  *ar = s * p.alpha[2 * k];
  *ai = s * p.alpha[2 * k + 1];
}

double coupling_x(const Problem &p, int n, int o) {
  if (p.up[(size_t)n * p.M + o] < 0) return 0.0;
  const int j = o % p.K, k = o / p.K;
  double ar, ai;
  bath_alpha(p, j, k, &ar, &ai);
  return std::sqrt((p.ado[(size_t)n * p.M + o] + 1.0) * std::hypot(ar, ai));
}

double coupling_y(const Problem &p, int n, int o) {
  if (p.dn[(size_t)n * p.M + o] < 0) return 0.0;
  const int j = o % p.K, k = o / p.K;
  double ar, ai;
  bath_alpha(p, j, k, &ar, &ai);
  const double s = p.bath_scale.empty() ? 1.0 : p.bath_scale[(size_t)j * p.K_m + k];
  return std::sqrt(p.ado[(size_t)n * p.M + o] / std::hypot(ar, ai)) * s;
}

int n_params(const Problem &p) {
  const int ns = p.single_size - 1;
  return ns + ns * (ns - 1) / 2 + p.K * p.K_m;
}

void param_dH(const Problem &p, int i, cbuf &dH) {
  const int N = p.N(), s = p.single_size, ns = s - 1;
  dH.assign(2 * (size_t)N * N, 0.0);
  std::vector<double> D((size_t)s * s, 0.0); // single block, fs^-1 per cm^-1
  if (i < ns) {
    // site energy eps_{i+1}: its diagonal lands where construct_Hal's sort puts it
    // (dynamics.cpp:24-27, index 0 = 0.0 included); the permutation is held fixed.
    std::vector<std::pair<double, int>> d(s);
    for (int a = 0; a < s; a++) d[a] = {a == 0 ? 0.0 : re(p.Hkey, N, a, a), a};
    std::stable_sort(d.begin(), d.end(), [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
      return x.first < y.first;
    });
    for (int pos = 1; pos < s; pos++)
      if (d[pos].second == i + 1) D[(size_t)pos * s + pos] = 1.0 / kHbar;
  } else if (i < ns + ns * (ns - 1) / 2) {
    int q = i - ns;
    for (int a = 1; a < s; a++)
      for (int b = a + 1; b < s; b++, q--)
        if (q == 0) D[(size_t)a * s + b] = D[(size_t)b * s + a] = 1.0 / kHbar;
  } else {
    return; // bath scale: H does not depend on it
  }
  for (int a = 0; a < s; a++)
    for (int b = 0; b < s; b++) re(dH, N, a, b) = D[(size_t)a * s + b];
  if (p.single_manifold) return;
  // two-exciton block, linear in the single block (dynamics.cpp:29-49)
  for (int x = s; x < N; x++)
    for (int y = s; y < N; y++) {
      const int a = p.d_a[x], b = p.d_b[x], c = p.d_a[y], d = p.d_b[y];
      double v;
      if (x == y) {
        v = D[(size_t)a * s + a] + D[(size_t)b * s + b];
      } else {
        v = (a == c) * (1 - (b == d)) * D[(size_t)b * s + d] + (a == d) * (1 - (b == c)) * D[(size_t)b * s + c] +
            (b == c) * (1 - (a == d)) * D[(size_t)a * s + d] + (b == d) * (1 - (a == c)) * D[(size_t)a * s + c];
      }
      re(dH, N, x, y) = v;
    }
}

int count_records(const Problem &p, double tau3, float t_end) {
  float nstep = (t_end - p.t_start) / p.step_size;
  const int stride = p.print_stride();
  float t = p.t_start;
  int c = 0;
  for (int i = 0; i <= nstep; i++) {
    if (t >= tau3 && i % stride == 0) c++;
    t += p.step_size;
  }
  return c;
}

} // namespace heom
