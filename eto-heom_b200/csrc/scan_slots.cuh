// Staged delay scan: the slot kernel (included by scan.cu after scan_pm.cuh).
//
// The single-pass scan kernel propagates, for every point, the four mixed-difference
// components R, D2, D3, Q from t_start to the point's end.  Points of a scan share most
// of that work: R depends only on pulse 1's time, D2 only on pulses 1 and 2, and D3 and
// Q stay exactly zero until pulse 3's window (see scan_pm.cuh).  The staged scan runs
// one persistent launch of this kernel over a queue of jobs (scan.cu, staged_run):
//   1. per (tau1, tau2) group: R and D2 from t_start until the first two pulses are over,
//      jumping over the pulse-free gap between them, saving D2 (and R where a member
//      needs it) at the members' window starts or at the group's jump base;
//   2. jump jobs (mode 2), one per group: D2 carried from the group's base through its
//      jumped members' window starts in step order, each leg T0^(steps) through the
//      block powers of the pulse-free step map;
//   3. per point: its pulse-3 window (D2 and Q, or R, D2, D3 and Q), recording P and
//      saving the state at the window's end.
// The pulse-free tails after the windows run in scan_tail_dual (below) as FP64 dot
// products with the dual vectors w_k.
//
// A job whose inputs come from an earlier job waits on a per-point flag that the
// producer sets after its snapshot stores are visible.  Every producer was dequeued
// before its consumers, by a CTA that is resident and never waits on a later job, so
// each wait ends; it is still bounded in time, and a wait that gives up sets an error
// flag, writes NaN into its outputs and releases its own dependants.
//
// A job holds up to four "slots" (trajectories).  Slot s has an operator (off-diagonal
// H plus the pulses in its op mask, with the pulse times of its field set), up to two
// sources -i[V_q, state(src)] (the mixed-difference couplings), an active step range
// [wake, stop) outside which it keeps its state, and an initial state (zero, |0><0| on
// ADO 0, or a snapshot).  Layout, thread mapping and stage arithmetic are those of
// scan_pm (one thread per ADO block of a slot, position-major shared memory, Horner RK4
// with the FP64 diagonal).
#pragma once

struct SlotSpec {
  int op;          // bit q: pulse q+1 enters the operator
  int fset;        // field set (pulse times) of the operator and the sources
  int src[2];      // source slots (-1: none)
  int srcq[2];     // pulse of each source: 1 = pulse 2, 2 = pulse 3
  int wake, stop;  // active on steps [wake, stop)
  int init;        // 0: zero, 1: |0><0| on ADO 0, 2: the snapshot at init_ptr
  int pad;
  const double2 *init_ptr; // [NN][n_ado], position-major, the kernel's ADO order
};

struct SlotRec {   // P[rec0 + k] = Tr X3 slot q - Tr X3 slot r at the k-th recorded step
  int q, r;        // slots (-1: no recorder)
  int first, last; // steps of the point within the job
  int rec0, nrec;  // first record index, records made in [first, last)
  double tau3;
  double2 *P;      // the point's output
};

struct SlotJob {
  int first, last;       // steps [first, last)
  int save_begin, save_end;
  int wait[4], wait_val; // start once flags[wait[k]] >= wait_val (-1: no wait)
  int mode;              // 0: slots stepped on full blocks; 2: a jump (see sl_jump)
  double tau[2][3];      // pulse times of the two field sets
  SlotSpec slot[4];
  SlotRec rec[4];
};

static_assert(sizeof(SlotJob) % sizeof(int) == 0, "copied to shared memory word by word");

struct SlotSave {        // copy slot `slot` (minus slot `minus`, unless -1) before step `step`
  int step, slot, minus; // (step == job.last: after the job)
  int flag, fval;        // then set flags[flag] = fval (-1: none), once the copy is visible
  int pad;
  double2 *dst;          // [NN][n_ado]
};

struct SlotArgs {
  int N, n_ado, M, K, K_m, n_jobs, stride, wcap, ado0;
  float t_start, dt;
  double E0[3], taup[3], w0[3], h;
  const unsigned char *tables;
  const double *sys;
  const SlotJob *jobs;
  const SlotSave *saves;
  int *counter;
  int *flags;            // per-point readiness between stages
  int *err;              // set to 1 when a dependency wait gives up
  unsigned long long wait_ns;
  const int *jtab;       // jump blocks: count, positions per block, first position, offset, positions
  const double2 *jpow;   // T0^(2^j) of every block, jpow_stride elements per power
  long long jpow_stride;
  int jpow_n;            // powers available
  int jleg_delta;        // > 0: a jump of exactly this many steps is one product with jleg
  const double2 *jleg;   // T0^jleg_delta of every block, laid out as one power
};

constexpr int kTailMax = 8;
constexpr int kGapMin = 8; // shortest pulse-free gap a slot job jumps over (steps)
// Reduced-tail table (doubles): [0] = n positions (0: none), [1..kTailMax] = positions
// r*N + c, then C (kTailMax x kTailMax complex, row-major): X_e = sum_e' C[e][e'] w_e' is
// the commutator [H_off, w] restricted to the positions.
__host__ __device__ inline size_t tail_doubles() { return 1 + kTailMax + 2 * kTailMax * kTailMax; }

__device__ __forceinline__ double2 sl_field(const SlotArgs &a, int q, double d) {
  const double E0 = q == 0 ? a.E0[0] : q == 1 ? a.E0[1] : a.E0[2];
  const double tp = q == 0 ? a.taup[0] : q == 1 ? a.taup[1] : a.taup[2];
  const double w0 = q == 0 ? a.w0[0] : q == 1 ? a.w0[1] : a.w0[2];
  const double Eq = E0 * exp(-2.77 * d * d / tp / tp);
  double sn, cs;
  sincos(q == 0 ? w0 * d : -w0 * d, &sn, &cs);
  return make_double2(Eq * cs, Eq * sn);
}

template <int NT> __host__ __device__ inline size_t sl_smem_bytes(size_t tsz, int n_ado, int M, int wcap) {
  constexpr int NN = NT * NT;
  const size_t nM = (size_t)n_ado * M;
  const size_t EP = (size_t)NN * pm_stride(n_ado);
  size_t b = 0;
  b += al16(16 * EP);                   // rho (FP64)
  b += al16(2 * 2 * tsz * EP);          // w copies, double-buffered
  b += al16(2 * tsz * 8 * NN);          // A of 4 slots, V2/V3 of 2 field sets
  b += al16(16 * (size_t)NN);           // X3
  b += al16(8 * (size_t)NN);            // Hd[r] - Hd[c]
  b += al16((tsz == 4 ? 16 : 32) * nM); // links ([o][n])
  b += al16(16 * (size_t)NN);           // off-diagonal H (FP64)
  b += al16(16 * 3 * (size_t)NN);       // X0, X1^T, X2^T (FP64)
  b += al16(16 * (size_t)n_ado);        // damping scalars
  b += al16(16 * 6 * (size_t)wcap);     // pulse-field windows, 2 field sets x 3 pulses
  return b;
}

// One Horner stage of a slot's block: own operator plus up to two sources.
template <typename T, int NT>
__device__ __forceinline__ void sl_stage(const PmShared &g, int n, int blk, unsigned am, const typename V2<T>::t *A,
                                         int sb0, unsigned sm0, const typename V2<T>::t *S0, int sb1, unsigned sm1,
                                         const typename V2<T>::t *S1, const typename V2<T>::t *__restrict__ W,
                                         typename V2<T>::t *__restrict__ Wn, const double *__restrict__ Hdd,
                                         double2 *__restrict__ rho, const PmLink<T> *__restrict__ links, int slot,
                                         double2 dmp, double cm, bool last, double2 (&w64)[NT * NT]) {
  using T2 = typename V2<T>::t;
  const int SP = g.SP, nado = g.nado, K = g.K, Km = g.Km;
  T kr[NT * NT], ki[NT * NT];
#pragma unroll
  for (int e = 0; e < NT * NT; e++) { kr[e] = 0; ki[e] = 0; }
  if (am) pm_commutator<T, NT, NT, 0>(am, A, W, SP, blk, kr, ki);
#pragma unroll 1
  for (int k = 0; k < 2; k++) { // sources -i[V_q, state(src)], the same ADO of another slot
    const int sb = k == 0 ? sb0 : sb1;
    const unsigned sm = k == 0 ? sm0 : sm1;
    if (sb >= 0 && sm) pm_commutator<T, NT, NT, 0>(sm, k == 0 ? S0 : S1, W, SP, sb * nado + n, kr, ki);
  }
  const T2 *Wc = W + slot * nado;
  if (K >= 1) pm_links<T, NT, NT, 0, 1>(Wc, SP, nado, K, Km, n, links, kr, ki);
  if (NT > 2 && K >= 2) pm_links<T, NT, NT, 0, (NT > 2 ? 2 : 1)>(Wc, SP, nado, K, Km, n, links, kr, ki);
  if (NT > 3 && K >= 3) pm_links<T, NT, NT, 0, (NT > 3 ? 3 : 1)>(Wc, SP, nado, K, Km, n, links, kr, ki);
#pragma unroll
  for (int q = 0; q < NT * NT; q++) {
    const double gr = dmp.x, gi = dmp.y - Hdd[q];
    const double2 wv = w64[q];
    const double k_r = fma(gr, wv.x, fma(-gi, wv.y, (double)kr[q]));
    const double k_i = fma(gr, wv.y, fma(gi, wv.x, (double)ki[q]));
    const double2 r0v = rho[q * SP + blk];
    const double2 wn = make_double2(fma(cm, k_r, r0v.x), fma(cm, k_i, r0v.y));
    w64[q] = wn;
    Wn[q * SP + blk] = mk2<T>(wn.x, wn.y);
    if (last) rho[q * SP + blk] = wn;
  }
}

// One position block's rows of y = P x, both block-ordered: a warp takes RW rows at a time
// and lane l their columns l + 32 u (u < U, 32 U >= d), so each lane has RW * U
// independent loads of P in flight before its first FMA; the block's x stays in registers.
template <int U, int RW>
__device__ __forceinline__ void jump_rows(const double2 *__restrict__ P, const double2 *xb, double2 *yb, int d,
                                          int lane, int warp, int nw) {
  double2 xv[U];
#pragma unroll
  for (int u = 0; u < U; u++) {
    const int c = lane + 32 * u;
    xv[u] = c < d ? xb[c] : make_double2(0.0, 0.0);
  }
  for (int r0 = warp * RW; r0 < d; r0 += nw * RW) {
    double2 m[RW][U];
#pragma unroll
    for (int k = 0; k < RW; k++)
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int c = lane + 32 * u;
        m[k][u] = (r0 + k < d && c < d) ? __ldg(P + (size_t)(r0 + k) * d + c) : make_double2(0.0, 0.0);
      }
#pragma unroll
    for (int k = 0; k < RW; k++) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int u = 0; u < U; u++) {
        re = fma(m[k][u].x, xv[u].x, fma(-m[k][u].y, xv[u].y, re));
        im = fma(m[k][u].x, xv[u].y, fma(m[k][u].y, xv[u].x, im));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
      }
      if (lane == 0 && r0 + k < d) yb[r0 + k] = make_double2(re, im);
    }
  }
}

// Rows of a block wider than the register tiles: one row per warp, 8 loads per lane in flight.
__device__ __forceinline__ void jump_rows_wide(const double2 *__restrict__ P, const double2 *xb, double2 *yb, int d,
                                               int lane, int warp, int nw) {
  for (int r = warp; r < d; r += nw) {
    const double2 *Pr = P + (size_t)r * d;
    double re = 0.0, im = 0.0;
    for (int c0 = 0; c0 < d; c0 += 256) {
      double2 m[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int c = c0 + lane + 32 * u;
        m[u] = c < d ? __ldg(Pr + c) : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const int c = c0 + lane + 32 * u;
        const double2 z = c < d ? xb[c] : make_double2(0.0, 0.0);
        re = fma(m[u].x, z.x, fma(-m[u].y, z.y, re));
        im = fma(m[u].x, z.y, fma(m[u].y, z.x, im));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) yb[r] = make_double2(re, im);
  }
}

// T0^delta applied to the block-ordered state x (the positions of jtab's list, each with
// its n_ado ADOs; y: scratch of the same size) as one dense block mat-vec per set bit of
// delta, through the powers T0^(2^j), or as one product with T0^jleg_delta when delta is
// that leg (the step count between consecutive delays of a scan, prepared per sample).
// Every thread of the CTA calls it; returns the buffer that holds the result.  A failed check (powers not prepared, a block outside a
// power) skips the access, sets the error word and fills the result with NaN, so that
// every output depending on it reads NaN.  The checks read only values that are the same
// for every thread, so all threads take the same branch.
__device__ double2 *jump_apply(const SlotArgs &a, double2 *x, double2 *y, int delta, int NN, int tid, int bs) {
  const int nado = a.n_ado;
  const int nb = a.jtab[0];
  const int *np = a.jtab + 1, *pfirst = a.jtab + 1 + nb, *moff = a.jtab + 1 + 2 * nb;
  const int lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
  bool bad = false;
  const bool leg = a.jleg_delta > 0 && delta == a.jleg_delta;
  for (int j = 0; leg ? j == 0 : (delta >> j) != 0; j++) {
    if (!leg && !((delta >> j) & 1)) continue;
    if (!leg && j >= a.jpow_n) { // powers not prepared: give up (checked error, no access)
      if (tid == 0) atomicMax(a.err, 3);
      bad = true;
      break;
    }
    const double2 *Pj = leg ? a.jleg : a.jpow + (size_t)j * a.jpow_stride;
    for (int b = 0; b < nb; b++) {
      const int d = np[b] * nado, o = pfirst[b] * nado;
      if ((long long)moff[b] + (long long)d * d > a.jpow_stride || pfirst[b] + np[b] > NN) {
        if (tid == 0) atomicMax(a.err, 4);
        bad = true;
        continue;
      }
      const double2 *Pb = Pj + moff[b];
      if (d <= 96)
        jump_rows<3, 4>(Pb, x + o, y + o, d, lane, warp, nw);
      else if (d <= 160)
        jump_rows<5, 3>(Pb, x + o, y + o, d, lane, warp, nw);
      else if (d <= 288)
        jump_rows<9, 2>(Pb, x + o, y + o, d, lane, warp, nw);
      else
        jump_rows_wide(Pb, x + o, y + o, d, lane, warp, nw);
    }
    __syncthreads();
    double2 *t = x;
    x = y;
    y = t;
  }
  if (bad) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int e = tid; e < NN * nado; e += bs) x[e] = make_double2(nan, nan);
    __syncthreads();
  }
  return x;
}

// A jump job (mode 2): the state snapshot slot[0].init_ptr at step `first` carried with no
// field on through the job's saves in step order (each leg T0^(save.step - previous)); each
// save gets the state at its step and then raises its flag.  sbuf: 2 x n_ado * NN doubles2
// of scratch.
template <int NT>
__device__ void sl_jump(const SlotArgs &a, const SlotJob &J, double2 *sbuf, int tid, int bs) {
  constexpr int NN = NT * NT;
  const int nado = a.n_ado, cells = NN * nado;
  const int *plist = a.jtab + 1 + 3 * a.jtab[0];
  double2 *x = sbuf;
  for (int e = tid; e < cells; e += bs) {
    const int f = e / nado;
    x[e] = __ldcg(J.slot[0].init_ptr + plist[f] * nado + (e - f * nado));
  }
  __syncthreads();
  // the targets in step order: a group's jumped members, each carried from the previous
  int cur = J.first;
  for (int k = J.save_begin; k < J.save_end; k++) {
    const SlotSave &sv = a.saves[k];
    if (sv.step < cur && tid == 0) atomicMax(a.err, 8); // planner order violated: no jump back
    x = jump_apply(a, x, x == sbuf ? sbuf + cells : sbuf, max(0, sv.step - cur), NN, tid, bs);
    cur = max(cur, sv.step);
    for (int e = tid; e < cells; e += bs) {
      const int f = e / nado;
      __stcg(sv.dst + plist[f] * nado + (e - f * nado), x[e]);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0 && sv.flag >= 0) atomicMax(a.flags + sv.flag, sv.fval);
  }
}

template <typename T, int NT, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) scan_slots(SlotArgs a) {
  using T2 = typename V2<T>::t;
  constexpr int NN = NT * NT;
  static_assert(NN <= 32 && NT <= 4, "warp 0 builds A with one lane per element");
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ double2 s_tr[8];
  __shared__ unsigned s_mask[8];
  __shared__ SlotJob s_jobd;
  __shared__ int s_lo[6], s_cnt[6], s_job, s_ok;
  __shared__ float s_t0;
  const int M = a.M, nado = a.n_ado, K = a.K, Km = a.K_m, wcap = a.wcap;
  const int S = 4 * nado, SP = pm_stride(nado);
  const size_t EP = (size_t)NN * SP;
  const int tid = threadIdx.x, bs = blockDim.x;
  const size_t nM = (size_t)nado * M;
  unsigned char *p = sm;
  double2 *rho = (double2 *)p;
  p += al16(16 * EP);
  T2 *w32 = (T2 *)p; // [2][NN][SP]
  p += al16(2 * sizeof(T2) * EP);
  T2 *Aall = (T2 *)p; // [0..3]: slot operators; 4 + 2 f + (q-1): V_{q+1} of field set f
  p += al16(sizeof(T2) * 8 * NN);
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
  double2 *sdamp = (double2 *)p;
  p += al16(16 * (size_t)nado);
  double2 *fwin = (double2 *)p; // [2 field sets][3 pulses][wcap]
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
  const PmShared gsh{SP, nado, M, K, Km};

  for (;;) {
    __syncthreads();
    if (tid == 0) s_job = atomicAdd(a.counter, 1);
    __syncthreads();
    const int jx = s_job;
    if (jx >= a.n_jobs) break;
    { // the job descriptor in shared memory: the step loop reads it every step
      const int *src = (const int *)(a.jobs + jx);
      int *dst = (int *)&s_jobd;
      for (int w = tid; w < (int)(sizeof(SlotJob) / sizeof(int)); w += bs) dst[w] = src[w];
    }
    __syncthreads();
    const SlotJob &J = s_jobd;
    const int first = J.first, last = J.last;
    if (tid == 0) { // bounded wait for the producers of this job's initial states
      int ok = 1;
      if (J.wait[0] >= 0 || J.wait[1] >= 0 || J.wait[2] >= 0 || J.wait[3] >= 0) {
        unsigned long long t0;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
        for (int k = 0; k < 4 && ok; k++) {
          if (J.wait[k] < 0) continue;
          for (;;) {
            if (atomicAdd(a.flags + J.wait[k], 0) >= J.wait_val) break;
            unsigned long long t1;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            if (t1 - t0 > a.wait_ns) { ok = 0; break; }
            __nanosleep(2000);
          }
        }
        __threadfence();
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) { // give up: NaN outputs (first records, whole snapshots), release dependants, report
      const double nan = __longlong_as_double(0x7ff8000000000000LL);
      for (int k = J.save_begin; k < J.save_end; k++) {
        double2 *dst = a.saves[k].dst;
        for (size_t e = tid; e < (size_t)NN * nado; e += bs) __stcg(dst + e, make_double2(nan, nan));
      }
      __threadfence();
      __syncthreads();
      if (tid == 0) {
        atomicExch(a.err, 1);
        for (int r = 0; r < 4; r++)
          if (J.rec[r].q >= 0 && J.rec[r].nrec > 0) J.rec[r].P[J.rec[r].rec0] = make_double2(nan, nan);
        for (int k = J.save_begin; k < J.save_end; k++)
          if (a.saves[k].flag >= 0) atomicMax(a.flags + a.saves[k].flag, a.saves[k].fval);
      }
      continue;
    }
    if (J.mode == 2) { // jump: pulse-free steps [first, last) as powers of T0
      sl_jump<NT>(a, J, rho, tid, bs);
      continue;
    }
    // Pulse windows of both field sets (absolute step indices), and the float time at
    // step `first`, by the same sequence of roundings as a single-pass run.
    if (tid < 6) {
      const int f = tid / 3, q = tid - 3 * f;
      const double tq = J.tau[f][q];
      const double tw = 2 * (q == 0 ? a.taup[0] : q == 1 ? a.taup[1] : a.taup[2]);
      int lo = -1, cnt = 0;
      float t = a.t_start;
      for (int i = 0; i < last; i++) {
        const double d = (double)t - tq;
        if (fabs(d) <= tw) {
          if (lo < 0) lo = i;
          if (cnt < wcap) fwin[(f * 3 + q) * wcap + cnt] = make_double2(d, 0.0);
          cnt++;
        } else if (lo >= 0) {
          break;
        }
        t += a.dt;
      }
      s_lo[tid] = lo < 0 ? 0 : lo;
      s_cnt[tid] = cnt;
    } else if (tid == 6) {
      float t = a.t_start;
      for (int i = 0; i < first; i++) t += a.dt;
      s_t0 = t;
    }
    // initial states (both FP32 copies)
    for (size_t e = tid; e < (size_t)NN * S; e += bs) {
      const size_t q = e / S, blk = e - q * S;
      const int sl = (int)(blk / nado), n = (int)(blk - (size_t)sl * nado);
      const SlotSpec &ss = J.slot[sl];
      double2 v = make_double2(0.0, 0.0);
      if (ss.init == 1 && q == 0 && n == a.ado0) v.x = 1.0;
      else if (ss.init == 2) v = __ldcg(ss.init_ptr + q * nado + n);
      rho[q * SP + blk] = v;
      w32[q * SP + blk] = mk2<T>(v.x, v.y);
      w32[EP + q * SP + blk] = mk2<T>(v.x, v.y);
    }
    __syncthreads();
    for (int w = 0; w < 6; w++) {
      const int c = min(s_cnt[w], wcap);
      for (int k = tid; k < c; k += bs)
        fwin[w * wcap + k] = sl_field(a, w % 3, fwin[w * wcap + k].x);
    }
    int lo[6], cn[6];
#pragma unroll
    for (int w = 0; w < 6; w++) { lo[w] = s_lo[w]; cn[w] = s_cnt[w]; }
    // this thread's slot
    const int sl = tid < S ? tid / nado : -1;
    const int n = sl >= 0 ? tid - sl * nado : 0;
    const SlotSpec my = J.slot[sl >= 0 ? sl : 0];
    const double2 dmp = sl >= 0 ? sdamp[n] : make_double2(0.0, 0.0);
    int rcn[4] = {0, 0, 0, 0}; // records made so far by each recorder
    int sv = J.save_begin;
    int next_save = sv < J.save_end ? a.saves[sv].step : 0x7fffffff;
    int buf = 0;
    bool fieldfree = false; // the operators in shared memory were built for a step with no field on
    float t = s_t0;
    __syncthreads(); // field tables complete
    for (int i = first; i <= last; i++) {
      // snapshots due before step i (after the job at i == last)
      const int sv0 = sv;
      for (; next_save <= i; sv++, next_save = sv < J.save_end ? a.saves[sv].step : 0x7fffffff) {
        const SlotSave &s = a.saves[sv];
        for (size_t e = tid; e < (size_t)NN * nado; e += bs) {
          const size_t q = e / nado, nn = e - q * nado;
          double2 v = rho[q * SP + (size_t)s.slot * nado + nn];
          if (s.minus >= 0) {
            const double2 u = rho[q * SP + (size_t)s.minus * nado + nn];
            v = make_double2(v.x - u.x, v.y - u.y);
          }
          __stcg(s.dst + e, v);
        }
      }
      if (sv > sv0) { // publish: every thread's stores, then the flags
        __threadfence();
        __syncthreads();
        if (tid == 0)
          for (int k = sv0; k < sv; k++)
            if (a.saves[k].flag >= 0) atomicMax(a.flags + a.saves[k].flag, a.saves[k].fval);
      }
      if (i == last) break;
      // A pulse-free gap: no pulse of either field set on, and no save, slot wake or stop,
      // or record inside.  Every live slot then evolves under the pulse-free map alone, so
      // the slots jump over the gap as T0^(gap) (FP64 block powers) instead of stepping.
      if (J.mode == 0 && a.jpow_n > 0) {
        int ge = min(last, next_save);
        ge = min(ge, i + (1 << min(a.jpow_n, 30)) - 1);
#pragma unroll
        for (int w = 0; w < 6; w++)
          if (cn[w] > 0) {
            if ((unsigned)(i - lo[w]) < (unsigned)cn[w]) ge = i;
            else if (lo[w] > i) ge = min(ge, lo[w]);
          }
#pragma unroll
        for (int z = 0; z < 4; z++) {
          if (J.slot[z].wake > i) ge = min(ge, J.slot[z].wake);
          if (J.slot[z].stop > i) ge = min(ge, J.slot[z].stop);
          if (J.rec[z].q >= 0) {
            if (i >= J.rec[z].first && i < J.rec[z].last) ge = i;
            else if (J.rec[z].first > i) ge = min(ge, J.rec[z].first);
          }
        }
        if (ge - i >= kGapMin) {
          const int cells = NN * nado;
          const int *plist = a.jtab + 1 + 3 * a.jtab[0];
          double2 *gx = (double2 *)w32, *gy = gx + cells; // the FP32 copies are rebuilt below
          for (int z = 0; z < 4; z++) {
            if (!(J.slot[z].wake <= i && i < J.slot[z].stop)) continue;
            for (int e = tid; e < cells; e += bs) {
              const int f = e / nado;
              gx[e] = rho[plist[f] * SP + z * nado + (e - f * nado)];
            }
            __syncthreads();
            const double2 *r = jump_apply(a, gx, gy, ge - i, NN, tid, bs);
            for (int e = tid; e < cells; e += bs) {
              const int f = e / nado;
              rho[plist[f] * SP + z * nado + (e - f * nado)] = r[e];
            }
            __syncthreads();
          }
          for (size_t e = tid; e < EP; e += bs) {
            const double2 v = rho[e];
            w32[e] = mk2<T>(v.x, v.y);
            w32[EP + e] = mk2<T>(v.x, v.y);
          }
          __syncthreads();
          for (int k = i; k < ge; k++) t += a.dt;
          fieldfree = false;
          i = ge - 1;
          continue;
        }
      }
      bool on[6];
#pragma unroll
      for (int w = 0; w < 6; w++) on[w] = (unsigned)(i - lo[w]) < (unsigned)cn[w];
      bool rec[4];
#pragma unroll
      for (int r = 0; r < 4; r++)
        rec[r] = J.rec[r].q >= 0 && i >= J.rec[r].first && i < J.rec[r].last && t >= J.rec[r].tau3 &&
                 i % a.stride == 0;
      // With no pulse on and no record due, the operators and masks of the last field-free
      // step still hold: skip warp 0's rebuild and its barrier (uniform across the CTA).
      bool anyon = false;
#pragma unroll
      for (int w = 0; w < 6; w++) anyon = anyon || on[w];
      const bool rebuild = anyon || rec[0] || rec[1] || rec[2] || rec[3] || !fieldfree;
      fieldfree = !anyon;
      if (rebuild && tid < 32) {
        // warp 0: the slots' operators, the pulse-2/3 operators of both field sets and their
        // nonzero masks (one element per lane); warp 1 forms the recorders' traces meanwhile
        const int q = tid;
        bool nz[8] = {false, false, false, false, false, false, false, false};
        if (q < NN) {
          double vr[6], vi[6];
#pragma unroll
          for (int w = 0; w < 6; w++) {
            double2 ef = make_double2(0.0, 0.0);
            if (on[w]) {
              const int k = i - lo[w];
              ef = cn[w] <= wcap ? fwin[w * wcap + k] : sl_field(a, w % 3, (double)t - J.tau[w / 3][w % 3]);
            }
            const double2 x = Xf[(w % 3) * NN + q];
            vr[w] = -(x.x * ef.x - x.y * ef.y);
            vi[w] = -(x.x * ef.y + x.y * ef.x);
          }
          const double2 h = Hoff[q];
#pragma unroll
          for (int s = 0; s < 4; s++) {
            const int op = J.slot[s].op, f = J.slot[s].fset;
            double br = h.x, bi = h.y;
            // the same sums, in the same order, as the single-pass kernel
            if (op & 1) { br += f ? vr[3] : vr[0]; bi += f ? vi[3] : vi[0]; }
            if (op & 2) { br += f ? vr[4] : vr[1]; bi += f ? vi[4] : vi[1]; }
            if (op & 4) { br += f ? vr[5] : vr[2]; bi += f ? vi[5] : vi[2]; }
            const T2 v = mk2<T>(br, bi);
            Aall[s * NN + q] = v;
            nz[s] = v.x != (T)0 || v.y != (T)0;
          }
#pragma unroll
          for (int f = 0; f < 2; f++)
#pragma unroll
            for (int k = 0; k < 2; k++) {
              const T2 v = mk2<T>(vr[3 * f + 1 + k], vi[3 * f + 1 + k]);
              Aall[(4 + 2 * f + k) * NN + q] = v;
              nz[4 + 2 * f + k] = v.x != (T)0 || v.y != (T)0;
            }
        }
#pragma unroll
        for (int s = 0; s < 8; s++) {
          const unsigned b = __ballot_sync(0xffffffffu, nz[s]);
          if (q == 0) s_mask[s] = b;
        }
      } else if (rebuild && tid < 64 && (rec[0] || rec[1] || rec[2] || rec[3])) {
        // warp 1: Tr X3 of the recorders' slots at the step's start (one element per lane)
        const int q = tid - 32;
        double2 c4[8];
#pragma unroll
        for (int c = 0; c < 8; c++) c4[c] = make_double2(0.0, 0.0);
        if (q < NN) {
#pragma unroll
          for (int r = 0; r < 4; r++)
            if (rec[r]) {
              const int j = q / NT, l = q - j * NT;
              const double2 x = X3[l * NT + j];
              const int sq = J.rec[r].q, sr = J.rec[r].r;
              const double2 z = rho[q * SP + sq * nado + a.ado0];
              c4[2 * r] = make_double2(z.x * x.x - z.y * x.y, z.x * x.y + z.y * x.x);
              if (sr >= 0) {
                const double2 u = rho[q * SP + sr * nado + a.ado0];
                c4[2 * r + 1] = make_double2(u.x * x.x - u.y * x.y, u.x * x.y + u.y * x.x);
              }
            }
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
          if (rec[r]) {
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1)
#pragma unroll
              for (int c = 2 * r; c < 2 * r + 2; c++) {
                c4[c].x += __shfl_xor_sync(0xffffffffu, c4[c].x, o);
                c4[c].y += __shfl_xor_sync(0xffffffffu, c4[c].y, o);
              }
            if (q == 0) {
              s_tr[2 * r] = c4[2 * r];
              s_tr[2 * r + 1] = c4[2 * r + 1];
            }
          }
      }
      if (rebuild) __syncthreads();
      if (tid == 0)
#pragma unroll
        for (int r = 0; r < 4; r++)
          if (rec[r]) {
            const int k = J.rec[r].rec0 + rcn[r];
            if (rcn[r] < J.rec[r].nrec)
              J.rec[r].P[k] = make_double2(s_tr[2 * r].x - s_tr[2 * r + 1].x, s_tr[2 * r].y - s_tr[2 * r + 1].y);
            else
              atomicMax(a.err, 2); // more records than planned: skipped
          }
#pragma unroll
      for (int r = 0; r < 4; r++) rcn[r] += rec[r];
      const bool live = sl >= 0 && i >= my.wake && i < my.stop;
      const int blk = live ? sl * nado + n : 0;
      const unsigned am = live ? s_mask[sl] : 0u;
      // sources whose pulse is on in this slot's field set
      const int f = my.fset;
      const bool son0 = live && my.src[0] >= 0 && on[3 * f + my.srcq[0]];
      const bool son1 = live && my.src[1] >= 0 && on[3 * f + my.srcq[1]];
      const int sb0 = son0 ? my.src[0] : -1, sb1 = son1 ? my.src[1] : -1;
      const unsigned sm0 = son0 ? s_mask[4 + 2 * f + my.srcq[0] - 1] : 0u;
      const unsigned sm1 = son1 ? s_mask[4 + 2 * f + my.srcq[1] - 1] : 0u;
      const T2 *S0 = Aall + (4 + 2 * f + (son0 ? my.srcq[0] - 1 : 0)) * NN;
      const T2 *S1 = Aall + (4 + 2 * f + (son1 ? my.srcq[1] - 1 : 0)) * NN;
      double2 w64[NN];
#pragma unroll
      for (int e = 0; e < NN; e++) w64[e] = live ? rho[e * SP + blk] : make_double2(0.0, 0.0);
      for (int m = 4; m >= 1; m--) {
        const double cm = a.h / m;
        const T2 *W = w32 + (size_t)buf * EP;
        T2 *Wn = w32 + (size_t)(buf ^ 1) * EP;
        if (live)
          sl_stage<T, NT>(gsh, n, blk, am, Aall + sl * NN, sb0, sm0, S0, sb1, sm1, S1, W, Wn, Hdd, rho, links, sl,
                          dmp, cm, m == 1, w64);
        buf ^= 1;
        __syncthreads();
      }
      t += a.dt;
    }
  }
}

// ------------------------------------------------------------------ tail kernel
// The pulse-free tails of a staged scan, after the slot kernel.  Once every pulse is off
// the step map is one fixed matrix T = sum_{j<=4} (hL)^j / j! (L: the pulse-free HEOM
// operator on the reduced positions of the tail table), the same for every point, so
// the tail records of a point with state q at its window end s3 are
//   P(s3 + k) = x3^T T^k q = w_k^T q,   w_k = (T^T)^k x3,
// x3 the readout (Tr X3 . on ADO 0).  The host propagates the dual vectors w_k once per
// sample in FP64.  A point's records use the rows k0, k0 + stride, k0 + 2 stride, ...,
// so points with the same k0 share every row, and their records form one complex FP64
// matrix product P[g][j] = sum_c w_{k0 + j stride}[c] q_g[c] over the reduced cells.
// The host groups the points by k0 into tiles of at most kTailTP points; a CTA makes
// one tile's records j0 .. j0 + kTailTJ - 1 from kTailKC-cell slices of the states and
// of the rows staged in shared memory, each thread a 2 x 2 block (points ty, ty + 16;
// records tx, tx + 16) accumulated over the cells in order.

constexpr int kTailTP = 32, kTailTJ = 32, kTailKC = 16, kTailThreads = 256;
static_assert(kTailTJ == kTailTP && kTailKC * kTailTP % kTailThreads == 0, "one staging loop for both slices");

struct DualPoint {
  const double2 *q;  // the point's state at s3, [NN][n_ado] (Q, or Q - R)
  double2 *P;        // its first tail record
  int k0, count;     // records at k = k0 + j * stride, j < count
};

struct DualArgs {
  int ne, nado, stride, n_pts, NN, W_rows;
  const int *pos;        // the reduced positions (r * N + c)
  const double2 *W;      // w_k, [k][cell], cell = e * nado + n
  const DualPoint *pts;  // grouped by k0
  const int2 *tiles;     // (first point, points) of each tile, one k0 per tile
  int *err;              // set when a check fails (the access is skipped)
};

__global__ void __launch_bounds__(kTailThreads) scan_tail_dual(DualArgs a) {
  __shared__ double2 Qs[kTailKC][kTailTP + 1], Ws[kTailKC][kTailTJ + 1];
  __shared__ DualPoint s_pt[kTailTP];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int2 tile = a.tiles[blockIdx.x];
  const int np = min(tile.y, kTailTP), j0 = (int)blockIdx.y * kTailTJ;
  if (tid < np) s_pt[tid] = a.pts[tile.x + tid];
  __syncthreads();
  int jmax = 0;
  for (int g = 0; g < np; g++) jmax = max(jmax, s_pt[g].count);
  if (j0 >= jmax) return; // the same for every thread of the CTA
  const int k0 = s_pt[0].k0, cells = a.ne * a.nado;
  const double2 zero = make_double2(0.0, 0.0);
  double re[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, im[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int c0 = 0; c0 < cells; c0 += kTailKC) {
    for (int t = tid; t < kTailKC * kTailTP; t += kTailThreads) {
      const int kc = t % kTailKC, g = t / kTailKC, c = c0 + kc; // consecutive threads: consecutive cells
      double2 v = zero;
      if (g < np && c < cells) {
        const int e = c / a.nado, n = c - e * a.nado, ps = a.pos[e];
        if (ps < 0 || ps >= a.NN) atomicMax(a.err, 5);
        else if (s_pt[g].k0 != k0) atomicMax(a.err, 7);
        else v = __ldcg(s_pt[g].q + (size_t)ps * a.nado + n);
      }
      Qs[kc][g] = v;
      const int j = j0 + g; // the same slice of the tile's rows (kTailTJ == kTailTP)
      const long long row = (long long)k0 + (long long)j * a.stride;
      double2 w = zero;
      if (j < jmax && c < cells) {
        if (row >= a.W_rows) atomicMax(a.err, 6);
        else w = __ldg(a.W + row * cells + c);
      }
      Ws[kc][g] = w;
    }
    __syncthreads();
#pragma unroll
    for (int kc = 0; kc < kTailKC; kc++) {
      const double2 x0 = Ws[kc][tx], x1 = Ws[kc][tx + 16], z0 = Qs[kc][ty], z1 = Qs[kc][ty + 16];
      re[0][0] = fma(x0.x, z0.x, fma(-x0.y, z0.y, re[0][0]));
      im[0][0] = fma(x0.x, z0.y, fma(x0.y, z0.x, im[0][0]));
      re[0][1] = fma(x1.x, z0.x, fma(-x1.y, z0.y, re[0][1]));
      im[0][1] = fma(x1.x, z0.y, fma(x1.y, z0.x, im[0][1]));
      re[1][0] = fma(x0.x, z1.x, fma(-x0.y, z1.y, re[1][0]));
      im[1][0] = fma(x0.x, z1.y, fma(x0.y, z1.x, im[1][0]));
      re[1][1] = fma(x1.x, z1.x, fma(-x1.y, z1.y, re[1][1]));
      im[1][1] = fma(x1.x, z1.y, fma(x1.y, z1.x, im[1][1]));
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 2; u++)
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const int g = ty + 16 * u, j = j0 + tx + 16 * v;
      if (g < np && j < s_pt[g].count && s_pt[g].k0 == k0) s_pt[g].P[j] = make_double2(re[u][v], im[u][v]);
    }
}
