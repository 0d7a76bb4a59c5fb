// Position-major scan kernel for a compile-time system size NT (included by scan.cu).
//
// Thread (c, g, n) owns rows [g*RPT, g*RPT + RPT) of the N x N block of ADO n in
// component c (RPT = NT: the whole block).  Shared arrays are position-major: element
// (r, col) of all S = 4 n_ado blocks is contiguous (index pos * S + block), so a warp's
// accesses to one element position of 32 consecutive blocks are bank-conflict free.
// Per stage a thread reads the FP32 copy of its block, gathers the neighbour rows and
// columns it needs, keeps the FP64 Horner accumulator of its rows in registers and
// writes only the FP32 copy of the result (double-buffered: one barrier per stage).
// The FP64 state rho stays in shared memory, touched only by its owner.
#pragma once

template <int NT> __host__ __device__ inline size_t pm_smem_bytes(size_t tsz, int n_ado, int M, int K_m, int E) {
  constexpr int NN = NT * NT;
  const size_t nM = (size_t)n_ado * M;
  size_t b = 0;
  b += 16 * (size_t)E;             // rho (FP64)
  b += 2 * 2 * tsz * (size_t)E;    // w copies, double-buffered
  b += al16(2 * tsz * 6 * NN);     // A[4], S2, S3
  b += al16(16 * (size_t)NN);      // X3
  b += al16(8 * (size_t)NN);       // Hd[r] - Hd[c]
  b += al16(2 * tsz * K_m);        // alpha
  b += al16(tsz * nM) * 2;         // x, y   ([o][n])
  b += al16(2 * nM) * 2;           // up, dn ([o][n])
  return b;
}

struct PmShared {
  int S, nado, M, K, Km;
};

// One Horner stage for the rows R0 .. R0+RPT-1 of the thread's block.
template <typename T, int NT, int RPT, int R0>
__device__ __forceinline__ void pm_stage(const PmShared &g, int cc, int n, int tid, bool src, int on2, int on3,
                                         const typename V2<T>::t *__restrict__ W, typename V2<T>::t *__restrict__ Wn,
                                         const typename V2<T>::t *__restrict__ Aall, const double *__restrict__ Hdd,
                                         double2 *__restrict__ rho, const short *__restrict__ up,
                                         const short *__restrict__ dn, const T *__restrict__ xc,
                                         const T *__restrict__ yc, const typename V2<T>::t *__restrict__ alpha,
                                         double2 dmp, double cm, bool last, double2 (&w64)[RPT * NT]) {
  using T2 = typename V2<T>::t;
  constexpr int NN = NT * NT;
  const int S = g.S, nado = g.nado, K = g.K, Km = g.Km;
  const T2 *Ac = Aall + cc * NN;
  // X = A w - w A  ->  k = -i X, accumulated as kr = X.im, ki = -X.re.  Two streaming
  // passes keep few operands live: A w by rows l of w, then w A by columns c of A.
  T kr[RPT * NT], ki[RPT * NT];
#pragma unroll
  for (int e = 0; e < RPT * NT; e++) { kr[e] = 0; ki[e] = 0; }
#pragma unroll
  for (int l = 0; l < NT; l++) {
    T2 wl[NT];
#pragma unroll
    for (int c = 0; c < NT; c++) wl[c] = W[(l * NT + c) * S + tid];
#pragma unroll
    for (int rr = 0; rr < RPT; rr++) {
      const T2 a = Ac[(R0 + rr) * NT + l];
#pragma unroll
      for (int c = 0; c < NT; c++) { // X += a * w[l][c]
        const int e = rr * NT + c;
        ki[e] = fma(-a.x, wl[c].x, ki[e]);
        ki[e] = fma(a.y, wl[c].y, ki[e]);
        kr[e] = fma(a.x, wl[c].y, kr[e]);
        kr[e] = fma(a.y, wl[c].x, kr[e]);
      }
    }
  }
#pragma unroll
  for (int rr = 0; rr < RPT; rr++) {
    T2 wr[NT];
#pragma unroll
    for (int l = 0; l < NT; l++) wr[l] = W[((R0 + rr) * NT + l) * S + tid];
#pragma unroll
    for (int c = 0; c < NT; c++) {
      const int e = rr * NT + c;
#pragma unroll
      for (int l = 0; l < NT; l++) { // X -= w[r][l] * A[l][c]
        const T2 a = Ac[l * NT + c];
        ki[e] = fma(wr[l].x, a.x, ki[e]);
        ki[e] = fma(-wr[l].y, a.y, ki[e]);
        kr[e] = fma(-wr[l].x, a.y, kr[e]);
        kr[e] = fma(-wr[l].y, a.x, kr[e]);
      }
    }
  }
  if (src) {
    // pulse sources: D2 <- P2 R, D3 <- P3 R, Q <- P2 D3 + P3 D2
#pragma unroll 1
    for (int s2 = 0; s2 < 2; s2++) {
      int from = -1, op = 0;
      if (cc == 1 && s2 == 0 && on2) { from = 0; op = 4; }
      if (cc == 2 && s2 == 0 && on3) { from = 0; op = 5; }
      if (cc == 3 && s2 == 0 && on2) { from = 2; op = 4; }
      if (cc == 3 && s2 == 1 && on3) { from = 1; op = 5; }
      if (from < 0) continue;
      const T2 *Sm = Aall + op * NN;
      const int fbk = from * nado + n;
#pragma unroll
      for (int rr = 0; rr < RPT; rr++) {
        const int r = R0 + rr;
#pragma unroll
        for (int c = 0; c < NT; c++) {
          T sr = 0, si = 0;
#pragma unroll
          for (int l = 0; l < NT; l++) {
            const T2 a1 = Sm[r * NT + l], z1 = W[(l * NT + c) * S + fbk], z2 = W[(r * NT + l) * S + fbk],
                     a2 = Sm[l * NT + c];
            sr = fma(a1.x, z1.x, sr);
            sr = fma(-a1.y, z1.y, sr);
            si = fma(a1.x, z1.y, si);
            si = fma(a1.y, z1.x, si);
            sr = fma(-z2.x, a2.x, sr);
            sr = fma(z2.y, a2.y, sr);
            si = fma(-z2.x, a2.y, si);
            si = fma(-z2.y, a2.x, si);
          }
          kr[rr * NT + c] += si;
          ki[rr * NT + c] -= sr;
        }
      }
    }
  }
  // Bath couplings of site j (level s = j+1): row s and column s of the block
  // (dynamics.cpp:143-179 with the one-hot S_j written out).
#pragma unroll
  for (int s = 1; s < NT; s++) {
    if (s > K) break;
    for (int k = 0; k < Km; k++) {
      const int o = (s - 1) + k * K, to = o * nado + n;
      const int u = up[to], d = dn[to];
      if (u >= 0) {
        const T x = xc[to];
        const int ub = cc * nado + u;
        if (s >= R0 && s < R0 + RPT) { // row s: +i x w_u
#pragma unroll
          for (int c = 0; c < NT; c++) {
            if (c == s) continue;
            const T2 z = W[(s * NT + c) * S + ub];
            kr[(s - R0) * NT + c] = fma(-x, z.y, kr[(s - R0) * NT + c]);
            ki[(s - R0) * NT + c] = fma(x, z.x, ki[(s - R0) * NT + c]);
          }
        }
#pragma unroll
        for (int rr = 0; rr < RPT; rr++) { // column s: -i x w_u
          const int r = R0 + rr;
          if (r == s) continue;
          const T2 z = W[(r * NT + s) * S + ub];
          kr[rr * NT + s] = fma(x, z.y, kr[rr * NT + s]);
          ki[rr * NT + s] = fma(-x, z.x, ki[rr * NT + s]);
        }
      }
      if (d >= 0) {
        const T y = yc[to];
        const T2 al = alpha[k];
        const T by = al.y * y, ay = al.x * y;
        const int db = cc * nado + d;
        if (s >= R0 && s < R0 + RPT) { // row s: (-b y, a y) w_d; diagonal (-2 b y, 0)
#pragma unroll
          for (int c = 0; c < NT; c++) {
            const T2 z = W[(s * NT + c) * S + db];
            const T cr = c == s ? -2 * by : -by, ci = c == s ? (T)0 : ay;
            kr[(s - R0) * NT + c] = fma(cr, z.x, fma(-ci, z.y, kr[(s - R0) * NT + c]));
            ki[(s - R0) * NT + c] = fma(cr, z.y, fma(ci, z.x, ki[(s - R0) * NT + c]));
          }
        }
#pragma unroll
        for (int rr = 0; rr < RPT; rr++) { // column s: (-b y, -a y) w_d
          const int r = R0 + rr;
          if (r == s) continue;
          const T2 z = W[(r * NT + s) * S + db];
          kr[rr * NT + s] = fma(-by, z.x, fma(ay, z.y, kr[rr * NT + s]));
          ki[rr * NT + s] = fma(-by, z.y, fma(-ay, z.x, ki[rr * NT + s]));
        }
      }
    }
  }
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
      const double2 r0v = rho[q * S + tid];
      const double2 wn = make_double2(fma(cm, k_r, r0v.x), fma(cm, k_i, r0v.y));
      w64[e] = wn;
      Wn[q * S + tid] = mk2<T>(wn.x, wn.y);
      if (last) rho[q * S + tid] = wn;
    }
}

template <typename T, int NT, int RPT, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) scan_pm(ScanArgs a) {
  using T2 = typename V2<T>::t;
  constexpr int NN = NT * NT, GPR = NT / RPT;
  static_assert(NT % RPT == 0 && GPR <= 4, "rows per thread must divide N");
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ double2 s_field[3], s_tr[8];
  __shared__ int s_on[3], s_point;
  const int E = a.E, M = a.M, nado = a.n_ado, K = a.K, Km = a.K_m;
  const int S = 4 * nado;
  const int tid = threadIdx.x, bs = blockDim.x;
  const size_t nM = (size_t)nado * M;
  unsigned char *p = sm;
  double2 *rho = (double2 *)p;
  p += 16 * (size_t)E;
  T2 *w32 = (T2 *)p; // [2][NN][S]
  p += 2 * sizeof(T2) * (size_t)E;
  T2 *Aall = (T2 *)p;
  p += al16(sizeof(T2) * 6 * NN);
  double2 *X3 = (double2 *)p;
  p += al16(16 * (size_t)NN);
  double *Hdd = (double *)p;
  p += al16(8 * (size_t)NN);
  T2 *alpha = (T2 *)p;
  p += al16(sizeof(T2) * Km);
  T *xc = (T *)p;
  p += al16(sizeof(T) * nM);
  T *yc = (T *)p;
  p += al16(sizeof(T) * nM);
  short *up = (short *)p;
  p += al16(2 * nM);
  short *dn = (short *)p;
  TableLayout tl(nado, M, Km);
  const short *g_up = (const short *)(a.tables + tl.up), *g_dn = (const short *)(a.tables + tl.dn);
  const double *g_x = (const double *)(a.tables + tl.x), *g_y = (const double *)(a.tables + tl.y);
  const double2 *g_damp = (const double2 *)(a.tables + tl.damp), *g_alpha = (const double2 *)(a.tables + tl.alpha);
  for (size_t q = tid; q < nM; q += bs) { // transpose to [o][n]
    const size_t nn_ = q / M, o = q - nn_ * M, t = o * nado + nn_;
    up[t] = g_up[q];
    dn[t] = g_dn[q];
    xc[t] = (T)g_x[q];
    yc[t] = (T)g_y[q];
  }
  for (int q = tid; q < Km; q += bs) alpha[q] = mk2<T>(g_alpha[q].x, g_alpha[q].y);
  const double *g_Hd = a.sys, *g_Hoff = a.sys + NT, *g_Xs = g_Hoff + 2 * NN, *g_X3 = g_Xs + 6 * NN;
  for (int q = tid; q < NN; q += bs) {
    X3[q] = make_double2(g_X3[2 * q], g_X3[2 * q + 1]);
    Hdd[q] = g_Hd[q / NT] - g_Hd[q % NT];
  }
  const bool active = tid < S * GPR;
  const int blkid = active ? tid % S : 0;      // block = cc * nado + n
  const int grp = active ? tid / S : 0;        // row group
  const int cc = blkid / nado, n = blkid - cc * nado;
  const double2 dmp = active ? g_damp[n] : make_double2(0.0, 0.0);
  const PmShared gsh{S, nado, M, K, Km};

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
    double2 w64[RPT * NT];
#pragma unroll
    for (int e = 0; e < RPT * NT; e++) {
      const int q = grp * RPT * NT + e;
      const double v = (blkid == 0 && q == 0 && active) ? 1.0 : 0.0;
      w64[e] = make_double2(v, 0.0);
      if (active) {
        rho[q * S + blkid] = w64[e];
        w32[q * S + blkid] = mk2<T>(v, 0.0);
      }
    }
    int buf = 0, rec = 0;
    float t = a.t_start;
    for (int i = 0; i < nsteps; i++) {
      if (tid < 3) {
        const int q = tid;
        const double d = (double)t - (q == 0 ? pt.tau1 : q == 1 ? pt.tau2 : pt.tau3);
        const int on = fabs(d) <= a.taup[q] * 2;
        double2 ef = make_double2(0.0, 0.0);
        if (on) {
          const double Eq = a.E0[q] * exp(-2.77 * d * d / a.taup[q] / a.taup[q]);
          double sn, cs;
          sincos(q == 0 ? a.w0[q] * d : -a.w0[q] * d, &sn, &cs);
          ef = make_double2(Eq * cs, Eq * sn);
        }
        s_on[q] = on;
        s_field[q] = ef;
      }
      __syncthreads();
      const int on1 = s_on[0], on2 = s_on[1], on3 = s_on[2];
      for (int q = tid; q < NN; q += bs) {
        double vr[3], vi[3];
        for (int s = 0; s < 3; s++) {
          const double xr = g_Xs[2 * (s * NN + q)], xi = g_Xs[2 * (s * NN + q) + 1];
          const double2 ef = s_field[s];
          vr[s] = -(xr * ef.x - xi * ef.y);
          vi[s] = -(xr * ef.y + xi * ef.x);
        }
        const double br = g_Hoff[2 * q] + (on1 ? vr[0] : 0.0), bi = g_Hoff[2 * q + 1] + (on1 ? vi[0] : 0.0);
        const double r2 = on2 ? vr[1] : 0.0, i2 = on2 ? vi[1] : 0.0, r3 = on3 ? vr[2] : 0.0, i3 = on3 ? vi[2] : 0.0;
        Aall[q] = mk2<T>(br, bi);
        Aall[NN + q] = mk2<T>(br + r2, bi + i2);
        Aall[2 * NN + q] = mk2<T>(br + r3, bi + i3);
        Aall[3 * NN + q] = mk2<T>(br + r2 + r3, bi + i2 + i3);
        Aall[4 * NN + q] = mk2<T>(r2, i2);
        Aall[5 * NN + q] = mk2<T>(r3, i3);
      }
      // P = Tr(X3 (Q - R)) on ADO 0 before the step: each owner of a row group of
      // R_0 or Q_0 traces its rows (FP64); thread 0 combines after the barrier.
      const bool do_rec = t >= pt.tau3 && i % a.stride == 0;
      if (do_rec && active && n == 0 && (cc == 0 || cc == 3)) {
        double sr = 0.0, si = 0.0;
#pragma unroll
        for (int rr = 0; rr < RPT; rr++)
#pragma unroll
          for (int l = 0; l < NT; l++) {
            const int jr = grp * RPT + rr;
            const double2 v = w64[rr * NT + l], x = X3[l * NT + jr];
            sr += v.x * x.x - v.y * x.y;
            si += v.x * x.y + v.y * x.x;
          }
        s_tr[(cc == 0 ? 0 : 4) + grp] = make_double2(sr, si);
      }
      __syncthreads();
      if (do_rec) {
        if (tid == 0) {
          double pr = 0.0, pim = 0.0;
          for (int q = 0; q < GPR; q++) {
            pr += s_tr[4 + q].x - s_tr[q].x;
            pim += s_tr[4 + q].y - s_tr[q].y;
          }
          a.P[off + rec] = make_double2(pr, pim);
        }
        rec++;
      }
      const bool src = (on2 || on3) && cc > 0;
      for (int m = 4; m >= 1; m--) {
        const double cm = a.h / m;
        const T2 *W = w32 + (size_t)buf * E;
        T2 *Wn = w32 + (size_t)(buf ^ 1) * E;
        if (active) {
          // the row group is warp-uniform except where a warp straddles two groups
          if (grp == 0)
            pm_stage<T, NT, RPT, 0>(gsh, cc, n, blkid, src, on2, on3, W, Wn, Aall, Hdd, rho, up, dn, xc, yc, alpha,
                                    dmp, cm, m == 1, w64);
          else if (GPR > 1 && grp == 1)
            pm_stage<T, NT, RPT, (GPR > 1 ? RPT : 0)>(gsh, cc, n, blkid, src, on2, on3, W, Wn, Aall, Hdd, rho, up,
                                                        dn, xc, yc, alpha, dmp, cm, m == 1, w64);
          else if (GPR > 2 && grp == 2)
            pm_stage<T, NT, RPT, (GPR > 2 ? 2 * RPT : 0)>(gsh, cc, n, blkid, src, on2, on3, W, Wn, Aall, Hdd, rho,
                                                            up, dn, xc, yc, alpha, dmp, cm, m == 1, w64);
          else if (GPR > 3)
            pm_stage<T, NT, RPT, (GPR > 3 ? 3 * RPT : 0)>(gsh, cc, n, blkid, src, on2, on3, W, Wn, Aall, Hdd, rho,
                                                            up, dn, xc, yc, alpha, dmp, cm, m == 1, w64);
        }
        buf ^= 1;
        __syncthreads();
      }
      t += a.dt;
    }
  }
}
