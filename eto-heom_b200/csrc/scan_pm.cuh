// Position-major scan kernel for a compile-time system size NT (included by scan.cu).
//
// Thread (c, g, n) owns rows [g*RPT, g*RPT + RPT) of the N x N block of ADO n in
// component c (RPT = NT: the whole block).  Shared arrays are position-major: element
// (r, col) of all SP = 4 n_ado blocks is contiguous (index pos * SP + block), so a warp's
// accesses to one element position of 32 consecutive blocks are bank-conflict free.  Per stage a thread reads the FP32 copy of its block, gathers the neighbour rows
// and columns it needs, keeps the FP64 Horner accumulator of its rows in registers and
// writes only the FP32 copy of the result (double-buffered: one barrier per stage).
// The FP64 state rho stays in shared memory, touched only by its owner.  (Keeping the
// accumulator in shared memory, splitting a block over two threads, padding the position
// stride, or unrolling the neighbour links branch-free over a zero block all measured
// slower on the dimer scan.)
//
// Sparse commutator.  The operator A of a component (off-diagonal H plus the pulse
// fields that are on) is the same for every thread of the CTA, and for an exciton
// system it is sparse: H couples levels only inside one excitation manifold and the
// dipoles only between neighbouring manifolds (construct_Hal, dynamics.cpp:22-45;
// polar.cpp:84-101).  Each step warp 0 builds A and a bit mask of its nonzero entries;
// the products [A, w] are then issued only for nonzero entries, through branches that
// every thread of a component takes the same way.  For the dimer with no pulse on, A has
// 2 nonzeros of 16.
//
// Pulse fields.  E_q(t) (TD_hamiltonian.cpp:5-31) depends on the point's pulse times;
// at the start of a point the CTA evaluates it once for every step of each pulse window
// into shared memory, so the per-step set-up is a table read.  A window longer than the
// table (possible only for pathological dt / taup) falls back to evaluating the field
// in the step.
//
// Neighbour links.  The ADOs of each component are ordered by depth, deepest first (the
// deepest tier has no up-neighbours), then by which down-neighbours exist, so the threads
// of a warp mostly share the same links.  Each (offset, ADO) link is one 16-byte record
// {x, y Im(alpha), y Re(alpha), up | down << 16} read with a single shared load.
//
// Dormant components.  A component is exactly zero until its source switches on: D2
// until pulse 2's window, D3 until pulse 3's, Q until pulse 2 meets a nonzero D3 or
// pulse 3 a nonzero D2; R stays exactly |0><0| until pulse 1 (the commutators, damping
// and bath terms of |0><0| on ADO 0 all vanish term by term).  Their stages are skipped
// until then, which leaves every result bit-identical and removes about a third of the
// block-stages of a delay scan.
#pragma once

// One neighbour link of the whole-ADO form in shared memory.
template <class T> struct PmLink;
template <> struct __align__(16) PmLink<float> { float x, by, ay; int ud; };
template <> struct __align__(16) PmLink<double> { double x, by, ay; int ud, pad; };

__host__ __device__ inline int pm_stride(int n_ado) { return 4 * n_ado; }

template <int NT> __host__ __device__ inline size_t pm_smem_bytes(size_t tsz, int n_ado, int M, int wcap) {
  constexpr int NN = NT * NT;
  const size_t nM = (size_t)n_ado * M;
  const size_t EP = (size_t)NN * pm_stride(n_ado);
  size_t b = 0;
  b += al16(16 * EP);                   // rho (FP64)
  b += al16(2 * 2 * tsz * EP);          // w copies, double-buffered
  b += al16(2 * tsz * 6 * NN);          // A[4], S2, S3
  b += al16(16 * (size_t)NN);           // X3
  b += al16(8 * (size_t)NN);            // Hd[r] - Hd[c]
  b += al16((tsz == 4 ? 16 : 32) * nM); // links ([o][n])
  b += al16(16 * (size_t)NN);           // off-diagonal H (FP64)
  b += al16(16 * 3 * (size_t)NN);       // X0, X1^T, X2^T (FP64)
  b += al16(16 * (size_t)n_ado);        // damping scalars
  b += al16(16 * 3 * (size_t)wcap);     // pulse-field windows
  return b;
}

// Pulse-window table length for pulse widths taup and step dt: every step with
// |t - tau| <= 2 taup, plus margin for the rounding of the float time grid.
__host__ inline int pm_window_cap(const double taup[3], float dt) {
  int w = 0;
  for (int q = 0; q < 3; q++) {
    const double n = std::ceil(4.0 * taup[q] / (double)dt);
    w = std::max(w, n < 1e6 ? (int)n + 16 : 1 << 21);
  }
  return w;
}

struct PmShared {
  int SP, nado, M, K, Km;
};

// Field of pulse q at time offset d = t - tau_q (build_V_matrix, TD_hamiltonian.cpp:5-17:
// pulse 1 carries e^{+i w0 d}, pulses 2 and 3 e^{-i w0 d}).
__device__ __forceinline__ double2 pm_field(const ScanArgs &a, int q, double d) {
  // select with constant indices: a runtime index into a kernel parameter array would
  // copy the array to local memory
  const double E0 = q == 0 ? a.E0[0] : q == 1 ? a.E0[1] : a.E0[2];
  const double tp = q == 0 ? a.taup[0] : q == 1 ? a.taup[1] : a.taup[2];
  const double w0 = q == 0 ? a.w0[0] : q == 1 ? a.w0[1] : a.w0[2];
  const double Eq = E0 * exp(-2.77 * d * d / tp / tp);
  double sn, cs;
  sincos(q == 0 ? w0 * d : -w0 * d, &sn, &cs);
  return make_double2(Eq * cs, Eq * sn);
}

// k += -i [A, z] for the rows R0 .. R0+RPT-1 of block `blk` (kr = X.im, ki = -X.re with
// X = A z - z A), issuing products only for the nonzero entries of A given by `mask`.
template <typename T, int NT, int RPT, int R0>
__device__ __forceinline__ void pm_commutator(unsigned mask, const typename V2<T>::t *__restrict__ A,
                                              const typename V2<T>::t *__restrict__ W, int SP, int blk,
                                              T (&kr)[RPT * NT], T (&ki)[RPT * NT]) {
  using T2 = typename V2<T>::t;
  constexpr int NN = NT * NT;
  T2 zb[NN]; // the whole block: rows l for A z, the thread's rows for z A
#pragma unroll
  for (int e = 0; e < NN; e++) zb[e] = W[e * SP + blk];
  // FP32: the operator in registers, so that no shared-memory latency sits inside the
  // masked products (FP64 keeps reading it from shared memory: registers are short there)
  constexpr bool kPre = sizeof(T) == 4;
  T2 av[kPre ? NN : 1];
  if constexpr (kPre) {
#pragma unroll
    for (int e = 0; e < NN; e++) av[e] = A[e];
  }
#pragma unroll
  for (int rr = 0; rr < RPT; rr++)
#pragma unroll
    for (int l = 0; l < NT; l++) {
      if (!(mask & (1u << ((R0 + rr) * NT + l)))) continue;
      const T2 a = kPre ? av[kPre ? (R0 + rr) * NT + l : 0] : A[(R0 + rr) * NT + l];
#pragma unroll
      for (int c = 0; c < NT; c++) { // X[r][c] += a * z[l][c]
        const int e = rr * NT + c;
        const T2 z = zb[l * NT + c];
        ki[e] = fma(-a.x, z.x, ki[e]);
        ki[e] = fma(a.y, z.y, ki[e]);
        kr[e] = fma(a.x, z.y, kr[e]);
        kr[e] = fma(a.y, z.x, kr[e]);
      }
    }
#pragma unroll
  for (int l = 0; l < NT; l++)
#pragma unroll
    for (int c = 0; c < NT; c++) {
      if (!(mask & (1u << (l * NT + c)))) continue;
      const T2 a = kPre ? av[kPre ? l * NT + c : 0] : A[l * NT + c];
#pragma unroll
      for (int rr = 0; rr < RPT; rr++) { // X[r][c] -= z[r][l] * a
        const int e = rr * NT + c;
        const T2 z = zb[(R0 + rr) * NT + l];
        ki[e] = fma(z.x, a.x, ki[e]);
        ki[e] = fma(-z.y, a.y, ki[e]);
        kr[e] = fma(-z.x, a.y, kr[e]);
        kr[e] = fma(-z.y, a.x, kr[e]);
      }
    }
}

// Up-link of level s: k_n += -i x [S_s, w_u] restricted to row s and column s (the
// one-hot S_j of dynamics.cpp:143-160 written out).  Wc: this component's blocks.
template <typename T, int NT, int RPT, int R0, int s>
__device__ __forceinline__ void pm_up(const typename V2<T>::t *__restrict__ Wc, int SP, int u, T x,
                                      T (&kr)[RPT * NT], T (&ki)[RPT * NT]) {
  using T2 = typename V2<T>::t;
  if (s >= R0 && s < R0 + RPT) { // row s: +i x w_u
#pragma unroll
    for (int c = 0; c < NT; c++) {
      if (c == s) continue;
      const T2 z = Wc[(s * NT + c) * SP + u];
      kr[(s - R0) * NT + c] = fma(-x, z.y, kr[(s - R0) * NT + c]);
      ki[(s - R0) * NT + c] = fma(x, z.x, ki[(s - R0) * NT + c]);
    }
  }
#pragma unroll
  for (int rr = 0; rr < RPT; rr++) { // column s: -i x w_u
    const int r = R0 + rr;
    if (r == s) continue;
    const T2 z = Wc[(r * NT + s) * SP + u];
    kr[rr * NT + s] = fma(x, z.y, kr[rr * NT + s]);
    ki[rr * NT + s] = fma(-x, z.x, ki[rr * NT + s]);
  }
}

// Down-link of level s: k_n += y i(alpha S_s w_d - alpha* w_d S_s) on row s and column s
// (dynamics.cpp:162-179), with by = y Im(alpha), ay = y Re(alpha).
template <typename T, int NT, int RPT, int R0, int s>
__device__ __forceinline__ void pm_down(const typename V2<T>::t *__restrict__ Wc, int SP, int d, T by, T ay,
                                        T (&kr)[RPT * NT], T (&ki)[RPT * NT]) {
  using T2 = typename V2<T>::t;
  if (s >= R0 && s < R0 + RPT) { // row s: (-b y, a y) w_d; diagonal (-2 b y, 0)
#pragma unroll
    for (int c = 0; c < NT; c++) {
      const T2 z = Wc[(s * NT + c) * SP + d];
      const T cr = c == s ? -2 * by : -by, ci = c == s ? (T)0 : ay;
      kr[(s - R0) * NT + c] = fma(cr, z.x, fma(-ci, z.y, kr[(s - R0) * NT + c]));
      ki[(s - R0) * NT + c] = fma(cr, z.y, fma(ci, z.x, ki[(s - R0) * NT + c]));
    }
  }
#pragma unroll
  for (int rr = 0; rr < RPT; rr++) { // column s: (-b y, -a y) w_d
    const int r = R0 + rr;
    if (r == s) continue;
    const T2 z = Wc[(r * NT + s) * SP + d];
    kr[rr * NT + s] = fma(-by, z.x, fma(ay, z.y, kr[rr * NT + s]));
    ki[rr * NT + s] = fma(-by, z.y, fma(-ay, z.x, ki[rr * NT + s]));
  }
}

// All links of level s (offsets o = s-1 + k K, k < K_m).
template <typename T, int NT, int RPT, int R0, int s>
__device__ __forceinline__ void pm_links(const typename V2<T>::t *__restrict__ Wc, int SP, int nado, int K, int Km,
                                         int n, const PmLink<T> *__restrict__ links, T (&kr)[RPT * NT],
                                         T (&ki)[RPT * NT]) {
  for (int k = 0; k < Km; k++) {
    const PmLink<T> L = links[((s - 1) + k * K) * nado + n];
    const unsigned u = (unsigned)L.ud & 0xffffu, d = (unsigned)L.ud >> 16;
    if (u != 0xffffu) pm_up<T, NT, RPT, R0, s>(Wc, SP, (int)u, L.x, kr, ki);
    if (d != 0xffffu) pm_down<T, NT, RPT, R0, s>(Wc, SP, (int)d, L.by, L.ay, kr, ki);
  }
}

// One Horner stage for the rows R0 .. R0+RPT-1 of the thread's block.  am: nonzero mask
// of this component's A; m2, m3: nonzero masks of the pulse-2 / pulse-3 operators.
template <typename T, int NT, int RPT, int R0>
__device__ __forceinline__ void pm_stage(const PmShared &g, int cc, int n, int tid, bool src, int on2, int on3,
                                         unsigned am, unsigned m2, unsigned m3,
                                         const typename V2<T>::t *__restrict__ W, typename V2<T>::t *__restrict__ Wn,
                                         const typename V2<T>::t *__restrict__ Aall, const double *__restrict__ Hdd,
                                         double2 *__restrict__ rho, const PmLink<T> *__restrict__ links, double2 dmp,
                                         double cm, bool last, double2 (&w64)[RPT * NT]) {
  using T2 = typename V2<T>::t;
  constexpr int NN = NT * NT;
  const int SP = g.SP, nado = g.nado, K = g.K, Km = g.Km;
  T kr[RPT * NT], ki[RPT * NT];
#pragma unroll
  for (int e = 0; e < RPT * NT; e++) { kr[e] = 0; ki[e] = 0; }
  if (am) pm_commutator<T, NT, RPT, R0>(am, Aall + cc * NN, W, SP, tid, kr, ki);
  if (src) {
    // pulse sources: D2 <- -i[V2, R], D3 <- -i[V3, R], Q <- -i[V2, D3] - i[V3, D2]
#pragma unroll 1
    for (int s2 = 0; s2 < 2; s2++) {
      int from = -1, op = 0;
      if (cc == 1 && s2 == 0 && on2) { from = 0; op = 4; }
      if (cc == 2 && s2 == 0 && on3) { from = 0; op = 5; }
      if (cc == 3 && s2 == 0 && on2) { from = 2; op = 4; }
      if (cc == 3 && s2 == 1 && on3) { from = 1; op = 5; }
      if (from < 0) continue;
      const unsigned sm = op == 4 ? m2 : m3;
      if (sm) pm_commutator<T, NT, RPT, R0>(sm, Aall + op * NN, W, SP, from * nado + n, kr, ki);
    }
  }
  // Bath couplings of site j (level s = j+1).
  const T2 *Wc = W + cc * nado;
  if (K >= 1) pm_links<T, NT, RPT, R0, 1>(Wc, SP, nado, K, Km, n, links, kr, ki);
  if (NT > 2 && K >= 2) pm_links<T, NT, RPT, R0, (NT > 2 ? 2 : 1)>(Wc, SP, nado, K, Km, n, links, kr, ki);
  if (NT > 3 && K >= 3) pm_links<T, NT, RPT, R0, (NT > 3 ? 3 : 1)>(Wc, SP, nado, K, Km, n, links, kr, ki);
  // FP64: damping + site-energy diagonal, Horner update w = rho + (h/m) k
#pragma unroll
  for (int rr = 0; rr < RPT; rr++)
#pragma unroll
    for (int c = 0; c < NT; c++) {
      const int q = (R0 + rr) * NT + c, e = rr * NT + c;
      const double gr = dmp.x, gi = dmp.y - Hdd[q];
      const double2 wv = w64[e];
      const double k_r = fma(gr, wv.x, fma(-gi, wv.y, (double)kr[e]));
      const double k_i = fma(gr, wv.y, fma(gi, wv.x, (double)ki[e]));
      const double2 r0v = rho[q * SP + tid];
      const double2 wn = make_double2(fma(cm, k_r, r0v.x), fma(cm, k_i, r0v.y));
      w64[e] = wn;
      Wn[q * SP + tid] = mk2<T>(wn.x, wn.y);
      if (last) rho[q * SP + tid] = wn;
    }
}

template <typename T, int NT, int RPT, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) scan_pm(ScanArgs a) {
  using T2 = typename V2<T>::t;
  constexpr int NN = NT * NT;
  static_assert(RPT == NT, "one thread per whole block");
  static_assert(NN <= 32, "warp 0 builds A with one lane per element");
  static_assert(NT <= 4, "levels 1..3 carry the bath couplings");
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ double2 s_tr[2];
  __shared__ unsigned s_mask[6];
  __shared__ int s_lo[3], s_cnt[3], s_point, s_rstat;
  const int M = a.M, nado = a.n_ado, K = a.K, Km = a.K_m, wcap = a.wcap, ado0 = a.ado0;
  const int S = 4 * nado, SP = pm_stride(nado);
  const size_t EP = (size_t)NN * SP;
  const int tid = threadIdx.x, bs = blockDim.x;
  const size_t nM = (size_t)nado * M;
  unsigned char *p = sm;
  double2 *rho = (double2 *)p;
  p += al16(16 * EP);
  T2 *w32 = (T2 *)p; // [2][NN][SP]
  p += al16(2 * sizeof(T2) * EP);
  T2 *Aall = (T2 *)p;
  p += al16(sizeof(T2) * 6 * NN);
  double2 *X3 = (double2 *)p;
  p += al16(16 * (size_t)NN);
  double *Hdd = (double *)p;
  p += al16(8 * (size_t)NN);
  PmLink<T> *links = (PmLink<T> *)p;
  p += al16(sizeof(PmLink<T>) * nM);
  double2 *Hoff = (double2 *)p;
  p += al16(16 * (size_t)NN);
  double2 *Xf = (double2 *)p; // X0, X1^T, X2^T
  p += al16(16 * 3 * (size_t)NN);
  double2 *sdamp = (double2 *)p; // damping scalar per ADO
  p += al16(16 * (size_t)nado);
  double2 *fwin = (double2 *)p; // [3][wcap]
  TableLayout tl(nado, M, Km);
  const PmLinkHost *g_link = (const PmLinkHost *)(a.tables + tl.plink);
  const double2 *g_damp = (const double2 *)(a.tables + tl.pdamp);
  for (size_t q = tid; q < nM; q += bs) {
    const PmLinkHost L = g_link[q];
    PmLink<T> v;
    v.x = (T)L.x;
    v.by = (T)L.by;
    v.ay = (T)L.ay;
    v.ud = L.ud;
    links[q] = v;
  }
  for (int q = tid; q < nado; q += bs) sdamp[q] = g_damp[q];
  const double *g_Hd = a.sys, *g_Hoff = a.sys + NT, *g_Xs = g_Hoff + 2 * NN, *g_X3 = g_Xs + 6 * NN;
  for (int q = tid; q < NN; q += bs) {
    X3[q] = make_double2(g_X3[2 * q], g_X3[2 * q + 1]);
    Hdd[q] = g_Hd[q / NT] - g_Hd[q % NT];
    Hoff[q] = make_double2(g_Hoff[2 * q], g_Hoff[2 * q + 1]);
  }
  for (int q = tid; q < 3 * NN; q += bs) Xf[q] = make_double2(g_Xs[2 * q], g_Xs[2 * q + 1]);
  if (tid == 0) { // |0><0| is stationary under H when H couples level 0 to nothing
    int z = 1;
    for (int j = 1; j < NT; j++)
      z &= g_Hoff[2 * j] == 0.0 && g_Hoff[2 * j + 1] == 0.0 && g_Hoff[2 * j * NT] == 0.0 &&
           g_Hoff[2 * j * NT + 1] == 0.0;
    s_rstat = z;
  }
  const PmShared gsh{SP, nado, M, K, Km};

  for (;;) {
    __syncthreads();
    if (tid == 0) s_point = atomicAdd(a.counter, 1);
    __syncthreads();
    const int idx = s_point;
    if (idx >= a.n_points) break;
    const int pi = a.use_order ? a.order[idx] : idx;
    const heom_scan_point pt = a.pts[pi];
    const long long off = a.offsets[pi];
    const float nstep = (pt.t_end - a.t_start) / a.dt;
    const int nsteps = nstep >= 0.0f ? (int)nstep + 1 : 0;
    const double tau[3] = {pt.tau1, pt.tau2, pt.tau3};
    // Pulse windows: one pass over the float time grid (the same sequence of roundings
    // as the step loop) finds the contiguous run of steps where each pulse is on and
    // records t - tau for the steps that fit the table.
    if (tid < 3) {
      const int q = tid;
      const double tq = q == 0 ? pt.tau1 : q == 1 ? pt.tau2 : pt.tau3;
      const double tw = 2 * (q == 0 ? a.taup[0] : q == 1 ? a.taup[1] : a.taup[2]);
      int lo = -1, cnt = 0;
      float t = a.t_start;
      for (int i = 0; i < nsteps; i++) {
        const double d = (double)t - tq;
        if (fabs(d) <= tw) {
          if (lo < 0) lo = i;
          if (cnt < wcap) fwin[q * wcap + cnt] = make_double2(d, 0.0);
          cnt++;
        } else if (lo >= 0) {
          break;
        }
        t += a.dt;
      }
      s_lo[q] = lo < 0 ? 0 : lo;
      s_cnt[q] = cnt;
    }
    // initial state: R = |0><0| on ADO 0, D2 = D3 = Q = 0 (both FP32 copies: a dormant
    // component never rewrites either)
    for (size_t e = tid; e < (size_t)NN * S; e += bs) {
      const size_t q = e / S, blk = e - q * S;
      const double v = (blk == (size_t)ado0 && q == 0) ? 1.0 : 0.0;
      rho[q * SP + blk] = make_double2(v, 0.0);
      w32[q * SP + blk] = mk2<T>(v, 0.0);
      w32[EP + q * SP + blk] = mk2<T>(v, 0.0);
    }
    __syncthreads();
    for (int q = 0; q < 3; q++) {
      const int c = min(s_cnt[q], wcap);
      for (int k = tid; k < c; k += bs) fwin[q * wcap + k] = pm_field(a, q, fwin[q * wcap + k].x);
    }
    const int lo1 = s_lo[0], lo2 = s_lo[1], lo3 = s_lo[2];
    const int cn1 = s_cnt[0], cn2 = s_cnt[1], cn3 = s_cnt[2];
    // First step at which each component can leave its initial value.
    constexpr int kNever = 0x7fffffff;
    const int wR = s_rstat ? (cn1 > 0 ? lo1 : kNever) : 0;
    const int wD2 = cn2 > 0 ? lo2 : kNever, wD3 = cn3 > 0 ? lo3 : kNever;
    int wQ = kNever;
    if (cn2 > 0 && wD3 != kNever && max(lo2, wD3) < lo2 + cn2) wQ = max(lo2, wD3);
    if (cn3 > 0 && wD2 != kNever && max(lo3, wD2) < lo3 + cn3) wQ = min(wQ, max(lo3, wD2));
    int buf = 0, rec = 0;
    float t = a.t_start;
    for (int i = 0; i < nsteps; i++) {
      const int on1 = (unsigned)(i - lo1) < (unsigned)cn1, on2 = (unsigned)(i - lo2) < (unsigned)cn2,
                on3 = (unsigned)(i - lo3) < (unsigned)cn3;
      const bool do_rec = t >= pt.tau3 && i % a.stride == 0;
      if (i == 0) __syncthreads(); // field tables complete
      if (tid < 32) {
        // warp 0: A of the four components, the two pulse operators and their masks;
        // P = Tr(X3 (Q - R)) on ADO 0 before the step, one element per lane (FP64)
        const int q = tid;
        bool nz[6] = {false, false, false, false, false, false};
        double2 cR = make_double2(0.0, 0.0), cQ = make_double2(0.0, 0.0);
        if (q < NN) {
          const int ons[3] = {on1, on2, on3}, los[3] = {lo1, lo2, lo3}, cns[3] = {cn1, cn2, cn3};
          double vr[3], vi[3];
#pragma unroll
          for (int s = 0; s < 3; s++) {
            double2 ef = make_double2(0.0, 0.0);
            if (ons[s]) {
              const int k = i - los[s];
              ef = cns[s] <= wcap ? fwin[s * wcap + k] : pm_field(a, s, (double)t - tau[s]);
            }
            const double2 x = Xf[s * NN + q];
            vr[s] = -(x.x * ef.x - x.y * ef.y);
            vi[s] = -(x.x * ef.y + x.y * ef.x);
          }
          const double2 h = Hoff[q];
          const double br = h.x + vr[0], bi = h.y + vi[0];
          const T2 v[6] = {mk2<T>(br, bi), mk2<T>(br + vr[1], bi + vi[1]), mk2<T>(br + vr[2], bi + vi[2]),
                           mk2<T>(br + vr[1] + vr[2], bi + vi[1] + vi[2]), mk2<T>(vr[1], vi[1]),
                           mk2<T>(vr[2], vi[2])};
#pragma unroll
          for (int s = 0; s < 6; s++) {
            Aall[s * NN + q] = v[s];
            nz[s] = v[s].x != (T)0 || v[s].y != (T)0;
          }
          if (do_rec) { // element (j, l) contributes rho[j][l] X3[l][j]
            const int j = q / NT, l = q - j * NT;
            const double2 x = X3[l * NT + j], r = rho[q * SP + ado0], z = rho[q * SP + 3 * nado + ado0];
            cR = make_double2(r.x * x.x - r.y * x.y, r.x * x.y + r.y * x.x);
            cQ = make_double2(z.x * x.x - z.y * x.y, z.x * x.y + z.y * x.x);
          }
        }
#pragma unroll
        for (int s = 0; s < 6; s++) {
          const unsigned b = __ballot_sync(0xffffffffu, nz[s]);
          if (q == 0) s_mask[s] = b;
        }
        if (do_rec) {
#pragma unroll
          for (int o = 16; o >= 1; o >>= 1) {
            cR.x += __shfl_xor_sync(0xffffffffu, cR.x, o);
            cR.y += __shfl_xor_sync(0xffffffffu, cR.y, o);
            cQ.x += __shfl_xor_sync(0xffffffffu, cQ.x, o);
            cQ.y += __shfl_xor_sync(0xffffffffu, cQ.y, o);
          }
          if (q == 0) {
            s_tr[0] = cR;
            s_tr[1] = cQ;
          }
        }
      }
      __syncthreads();
      if (do_rec) {
        if (tid == 0) a.P[off + rec] = make_double2(s_tr[1].x - s_tr[0].x, s_tr[1].y - s_tr[0].y);
        rec++;
      }
      // One thread per block of every awake component.  The Horner accumulator restarts
      // from rho each step (w = rho at the first stage), so no state crosses steps in
      // registers.  (Spreading one or two awake components over all threads, two per
      // block, measured slower: the duplicated block loads and the larger code cost
      // more than the shorter per-thread chains save.)
      const bool a0 = i >= wR, a1 = i >= wD2, a2 = i >= wD3, a3 = i >= wQ;
      int cc = -1, n = 0;
      if (tid < S) {
        const int c = tid / nado;
        const bool awake = c == 0 ? a0 : c == 1 ? a1 : c == 2 ? a2 : a3;
        if (awake) {
          cc = c;
          n = tid - c * nado;
        }
      }
      const int blk = cc >= 0 ? cc * nado + n : 0;
      const double2 dmp = cc >= 0 ? sdamp[n] : make_double2(0.0, 0.0);
      const unsigned am = cc >= 0 ? s_mask[cc] : 0u, m2 = s_mask[4], m3 = s_mask[5];
      const bool src = (on2 || on3) && cc > 0;
      double2 w64[NN];
#pragma unroll
      for (int e = 0; e < NN; e++) w64[e] = cc >= 0 ? rho[e * SP + blk] : make_double2(0.0, 0.0);
      for (int m = 4; m >= 1; m--) {
        const double cm = a.h / m;
        const T2 *W = w32 + (size_t)buf * EP;
        T2 *Wn = w32 + (size_t)(buf ^ 1) * EP;
        if (cc >= 0)
          pm_stage<T, NT, NT, 0>(gsh, cc, n, blk, src, on2, on3, am, m2, m3, W, Wn, Aall, Hdd, rho, links, dmp, cm,
                                 m == 1, w64);
        buf ^= 1;
        __syncthreads();
      }
      t += a.dt;
    }
  }
}
