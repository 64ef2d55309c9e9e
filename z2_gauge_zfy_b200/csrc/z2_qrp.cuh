// z2_qrp.cuh -- register-resident pivoted Householder QR (DGEQP3 / DLAQP2
// semantics) for the UDV stabilization of one chain.
//
// The n x n work matrix (n <= 16 S) is held in the register file of the CTA:
// thread (tr, tc) = (lane % 16, 2 warp + lane / 16) owns the S x S elements
// A(tr + 16 p, tc + 16 q).  The 16 threads of a column group are the lanes of
// one half-warp, so a column dot product is S x S register FMAs plus a
// four-step shuffle reduction, and the rank-1 update of the trailing columns
// never touches shared memory.  The norm downdate of a column group runs on S
// lanes of its half-warp at once.  A step costs two block barriers: one after
// the reflector of the pivot column is published, one after the per-warp
// pivot candidates are published.  The reflector is on every step's critical
// path (the other warps wait for it), so its warp extracts the pivot column
// with a jump to a static copy, forms |beta| with one square root, and writes
// the finished column straight to its final place in A.
//
// Pivoting follows DGEQP3 without moving data: the logical position of every
// physical column is tracked (pos / lp2c), the arg-max breaks ties by logical
// position as IDAMAX does on the swapped arrays, and the partial norm
// downdate and its recompute threshold are DLAQP2's (its test and update
// multiplied out by vn1^2, so that no division sits on the step).  Each column is written
// to A at the step that factors it, at its logical position, so the result
// has DGEQP3's layout (R above the diagonal, reflectors below, tau, 1-based
// jpvt).
#pragma once
#include "z2_dmma.cuh"

__device__ __forceinline__ double hw_sum(double v) {
  v += __shfl_xor_sync(Z2_FULL, v, 8);
  v += __shfl_xor_sync(Z2_FULL, v, 4);
  v += __shfl_xor_sync(Z2_FULL, v, 2);
  v += __shfl_xor_sync(Z2_FULL, v, 1);
  return v;
}

// Arg-max over the 32 lanes of a warp of (v, p): larger v, then smaller p.
// v is a column norm (>= 0) or negative for "no candidate" (p = INT_MAX).
// Non-negative doubles order like their bit patterns, so the key is the
// 64-bit pattern (0 for v <= 0 or NaN, where the ordering only has to put
// every real candidate ahead of the empty lanes) and the reduction is three
// warp reductions (high word, low word, position) instead of a five-level
// shuffle butterfly over three values.
__device__ __forceinline__ void warp_argmax_vp(double v, int p, double &bv, int &bp) {
  const unsigned long long key = (v > 0.0) ? (unsigned long long)__double_as_longlong(v) : 0ull;
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(Z2_FULL, hi);
  const unsigned mlo = __reduce_max_sync(Z2_FULL, hi == mhi ? lo : 0u);
  const bool cand = hi == mhi && lo == mlo;
  const unsigned mp = __reduce_min_sync(Z2_FULL, cand ? (unsigned)p : 0xffffffffu);
  bp = (int)mp;
  bv = (mp >= 0x7fffffffu) ? -1.0
                           : __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}

// The per-step pivot: every warp reduces the eight warp candidates (lanes
// 0..7) the same way and takes the winner's physical column from widx
// (logical positions are unique, so the winning warp is the one whose wpos
// matches).
__device__ __forceinline__ int block_pivot(const double *wmax, const int *wpos, const int *widx) {
  const int lane = threadIdx.x & 31;
  const double v = lane < Z2_WARPS ? wmax[lane] : -1.0;
  const int p = lane < Z2_WARPS ? wpos[lane] : 0x7fffffff;
  const int c = lane < Z2_WARPS ? widx[lane] : 0;
  double bv; int bp;
  warp_argmax_vp(v, p, bv, bp);
  const unsigned w = __ballot_sync(Z2_FULL, lane < Z2_WARPS && p == bp);
  return __shfl_sync(Z2_FULL, c, w ? __ffs(w) - 1 : 0);
}

// Column sums of the trailing dot products over the 16 lanes of a column
// group, in every lane.  For S >= 5 the first 8 column slots are reduced by
// halving (lanes that differ in bit 8 / 4 / 2 of tr swap halves of what they
// hold, then the last bit is a plain exchange), which leaves each column's
// sum in two lanes after 4 + 2 + 1 + 1 exchanges, and the sums are then
// broadcast (8 more); slot 8 takes the plain butterfly.  Each sum is formed
// by the same pairwise additions as the four-level butterfly over all slots
// (36 exchanges), so the result is the same to the bit.
template <int S>
__device__ __forceinline__ void qrp_colsum8(double (&d)[S], int tr, int hl);
template <int S>
__device__ __forceinline__ void qrp_colsum(double (&d)[S], int tr, int hl) {
  if (S < 5) {
#pragma unroll
    for (int o = 8; o; o >>= 1) {
#pragma unroll
      for (int q = 0; q < S; ++q) d[q] += __shfl_xor_sync(Z2_FULL, d[q], o);
    }
  } else {
    qrp_colsum8<S>(d, tr, hl);
  }
}

template <int S>
__device__ __forceinline__ void qrp_colsum8(double (&d)[S], int tr, int hl) {
  double e[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) e[q] = (q < S) ? d[q < S ? q : 0] : 0.0;
  // bit 8: keep slots [0,4) (bit clear) or [4,8) (bit set)
  const bool b8 = tr & 8, b4 = tr & 4, b2 = tr & 2;
  double f[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double send = b8 ? e[k] : e[4 + k];
    const double keep = b8 ? e[4 + k] : e[k];
    f[k] = keep + __shfl_xor_sync(Z2_FULL, send, 8);
  }
  double g[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double send = b4 ? f[k] : f[2 + k];
    const double keep = b4 ? f[2 + k] : f[k];
    g[k] = keep + __shfl_xor_sync(Z2_FULL, send, 4);
  }
  double h;
  {
    const double send = b2 ? g[0] : g[1];
    const double keep = b2 ? g[1] : g[0];
    h = keep + __shfl_xor_sync(Z2_FULL, send, 2);
  }
  h += __shfl_xor_sync(Z2_FULL, h, 1);
  // lane tr now holds slot 4 (tr>>3 & 1) + 2 (tr>>2 & 1) + (tr>>1 & 1)
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double x = __shfl_sync(Z2_FULL, h, hl | (((q >> 2) & 1) << 3) | (((q >> 1) & 1) << 2) | ((q & 1) << 1));
    if (q < S) d[q < S ? q : 0] = x;
  }
  if (S > 8) {
    double x = d[S > 8 ? 8 : 0];
#pragma unroll
    for (int o = 8; o; o >>= 1) x += __shfl_xor_sync(Z2_FULL, x, o);
    d[S > 8 ? 8 : 0] = x;
  }
}

// Static-index views of the register tile: a[.][q] / a[p][.] for a warp-
// uniform runtime q or p, as a jump into one of S straight copies (a
// predicated select over all S x S registers costs S times more issue).
#define QRP_CASE_COL(Q) \
  case Q:               \
    if (Q < S) {        \
      _Pragma("unroll") for (int p = 0; p < S; ++p) col[p] = a[p][Q < S ? Q : 0]; \
    }                   \
    break;
#define QRP_CASE_ROW(P) \
  case P:               \
    if (P < S) {        \
      _Pragma("unroll") for (int q = 0; q < S; ++q) rowj[q] = a[P < S ? P : 0][q]; \
    }                   \
    break;
// Row blocks above the current step are zero in the reflector: the dot
// products and the rank-1 update enter their unrolled sequences at block pj
// (fall-through switch).
#define QRP_CASE_DOT(P) \
  case P:               \
    if (P < S) {        \
      _Pragma("unroll") for (int q = 0; q < S; ++q) d[q] += vr[P < S ? P : 0] * a[P < S ? P : 0][q]; \
    }
#define QRP_CASE_UPD(P) \
  case P:               \
    if (P < S) {        \
      _Pragma("unroll") for (int q = 0; q < S; ++q) a[P < S ? P : 0][q] -= d[q] * vr[P < S ? P : 0]; \
    }

// work: >= 2 n doubles (reflector + two int maps); red: >= 32 doubles.
template <int S>
__device__ __noinline__ void qrp_reg(double *A, int lda, int n, int *jpvt, double *tau,
                                     double *vn1, double *vn2, double *work, double *red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tr = lane & 15, tc = (warp << 1) | (lane >> 4);
  const int hl = lane & 16;
  const double tol3z = 1.0536712127723509e-08;   // sqrt(dlamch('E'))
  double *vsh = work;                                   // [n] reflector of the step
  int *pos = reinterpret_cast<int *>(work + n);         // physical -> logical
  int *lp2c = pos + n;                                  // logical -> physical
  double *wmax = red + 8;
  int *wpos = reinterpret_cast<int *>(red + 16);
  int *widx = reinterpret_cast<int *>(red + 20);
  double *tsh = red + 24;

  double a[S][S];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const int r = tr + 16 * p, c = tc + 16 * q;
      a[p][q] = (r < n && c < n) ? A[r + (size_t)c * lda] : 0.0;
    }
  unsigned done = 0;   // bit q: column tc + 16 q factored (or outside the matrix)
#pragma unroll
  for (int q = 0; q < S; ++q)
    if (tc + 16 * q >= n) done |= 1u << q;
  {
    // initial column norms (DNRM2 of each column)
    double d[S];
#pragma unroll
    for (int q = 0; q < S; ++q) {
      double t = 0.0;
#pragma unroll
      for (int p = 0; p < S; ++p) t += a[p][q] * a[p][q];
      d[q] = t;
    }
#pragma unroll
    for (int q = 0; q < S; ++q) d[q] = hw_sum(d[q]);
    if (tr == 0) {
#pragma unroll
      for (int q = 0; q < S; ++q) {
        const int c = tc + 16 * q;
        if (c < n) {
          const double nr = sqrt(d[q]);
          vn1[c] = nr; vn2[c] = nr; pos[c] = c; lp2c[c] = c;
        }
      }
    }
  }
  __syncthreads();
  int pc;
  {
    // pivot of step 0 (physical = logical order)
    double bv = -1.0; int bp = 0x7fffffff;
    for (int c = lane; c < n; c += 32) {
      const double v = vn1[c];
      if (v > bv || (v == bv && c < bp)) { bv = v; bp = c; }
    }
    double wv; int wp;
    warp_argmax_vp(bv, bp, wv, wp);
    pc = wp;   // every warp scans all columns: no block step
  }

  for (int j = 0; j < n; ++j) {
    const int qc = pc >> 4, gc = pc & 15;
    const int pj = j >> 4, oj = j & 15;
    // ---- reflector of the pivot column (DLARFG), by the warp holding it.
    // The finished column (R above the diagonal, beta, v below) goes straight
    // to its final place A(:, j); its registers are not used again. ----
    if (warp == (gc >> 1)) {
      const bool mine = (lane >> 4) == (gc & 1);
      double col[S];
#pragma unroll
      for (int p = 0; p < S; ++p) col[p] = 0.0;
      switch (qc) {
        QRP_CASE_COL(0) QRP_CASE_COL(1) QRP_CASE_COL(2) QRP_CASE_COL(3) QRP_CASE_COL(4)
        QRP_CASE_COL(5) QRP_CASE_COL(6) QRP_CASE_COL(7) QRP_CASE_COL(8)
        default: break;
      }
      double s0 = 0.0, s1 = 0.0, aj = 0.0;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int r = tr + 16 * p;
        const double x = (r > j && r < n) ? col[p] : 0.0;
        if (p & 1) s1 += x * x; else s0 += x * x;
        if (p == pj) aj = col[p];
      }
      const double ss = hw_sum(s0 + s1);
      const double alpha = __shfl_sync(Z2_FULL, aj, hl | oj);
      double t = 0.0, beta = alpha, sc = 1.0;
      if (j < n - 1 && ss != 0.0) {
        // |beta| = sqrt(alpha^2 + xnorm^2) (DLAPY2 without its rescaling,
        // which only matters past the overflow threshold: kept as fallback)
        double nb = sqrt(fma(alpha, alpha, ss));
        if (isinf(nb)) nb = dlapy2(alpha, sqrt(ss));
        beta = -copysign(nb, alpha);
        t = (beta - alpha) / beta;
        sc = 1.0 / (alpha - beta);
      }
      if (mine) {
#pragma unroll
        for (int p = 0; p < S; ++p) {
          const int r = tr + 16 * p;
          double vv = 0.0, out = col[p];
          if (r > j) {
            if (t != 0.0) out *= sc;
            vv = out;
          } else if (r == j) {
            out = beta;
            vv = 1.0;
          }
          if (r < n) {
            vsh[r] = vv;
            A[r + (size_t)j * lda] = out;
          }
        }
        if (tr == 0) { *tsh = t; tau[j] = t; }
      }
    }
    if (tid == Z2_NT - 1) {
      // logical interchange of positions j and pos[pc] (DGEQP3's column swap)
      const int lp = pos[pc], cj = lp2c[j];
      lp2c[lp] = cj; pos[cj] = lp;
      lp2c[j] = pc; pos[pc] = j;
    }
    __syncthreads();
    if (tc == gc) done |= 1u << qc;
    // ---- apply H to the trailing columns (DLARF) ----
    const double t = *tsh;
    if (t != 0.0) {
      double vr[S], d[S];
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int r = tr + 16 * p;
        vr[p] = (r < n) ? vsh[r] : 0.0;   // 0 above row j
        d[p] = 0.0;
      }
      switch (pj) {
        QRP_CASE_DOT(0) QRP_CASE_DOT(1) QRP_CASE_DOT(2) QRP_CASE_DOT(3) QRP_CASE_DOT(4)
        QRP_CASE_DOT(5) QRP_CASE_DOT(6) QRP_CASE_DOT(7) QRP_CASE_DOT(8)
        default: break;
      }
      qrp_colsum<S>(d, tr, hl);
#pragma unroll
      for (int q = 0; q < S; ++q) d[q] = ((done >> q) & 1u) ? 0.0 : t * d[q];
      switch (pj) {
        QRP_CASE_UPD(0) QRP_CASE_UPD(1) QRP_CASE_UPD(2) QRP_CASE_UPD(3) QRP_CASE_UPD(4)
        QRP_CASE_UPD(5) QRP_CASE_UPD(6) QRP_CASE_UPD(7) QRP_CASE_UPD(8)
        default: break;
      }
    }
    // ---- partial norm downdate (DLAQP2): lane q of each half-warp takes
    // column slot q; row j of the group comes from its owner lane ----
    double rowj[S];
#pragma unroll
    for (int q = 0; q < S; ++q) rowj[q] = 0.0;
    switch (pj) {
      QRP_CASE_ROW(0) QRP_CASE_ROW(1) QRP_CASE_ROW(2) QRP_CASE_ROW(3) QRP_CASE_ROW(4)
      QRP_CASE_ROW(5) QRP_CASE_ROW(6) QRP_CASE_ROW(7) QRP_CASE_ROW(8)
      default: break;
    }
    double ajc = 0.0;
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const double x = __shfl_sync(Z2_FULL, rowj[q], hl | oj);
      if (q == tr) ajc = x;
    }
    const bool act = tr < S && !((done >> tr) & 1u);
    const int cq = tc + 16 * tr;
    double v1 = -1.0;
    bool need = false;
    if (act) {
      v1 = vn1[cq];
      if (v1 != 0.0) {
        // DLAQP2's test temp (vn1/vn2)^2 <= tol3z with temp = 1 - (|a|/vn1)^2
        // and its update vn1 sqrt(temp), multiplied out: (vn1^2 - a^2) is
        // formed as (vn1 - |a|)(vn1 + |a|), so no division sits on the step
        const double aa = fabs(ajc), w2 = vn2[cq];
        const double r2 = fmax((v1 - aa) * (v1 + aa), 0.0);
        if (r2 <= tol3z * (w2 * w2)) {
          need = true;
        } else {
          v1 = sqrt(r2);
          vn1[cq] = v1;
        }
      }
    }
    const unsigned rec = __ballot_sync(Z2_FULL, need);
    const unsigned recw = (rec | (rec >> 16)) & 0xffffu;   // warp-uniform
    if (recw) {
#pragma unroll
      for (int q = 0; q < S; ++q) {
        if ((recw >> q) & 1u) {
          double s0 = 0.0;
#pragma unroll
          for (int p = 0; p < S; ++p) {
            const int r = tr + 16 * p;
            if (r > j && r < n) s0 += a[p][q] * a[p][q];
          }
          s0 = hw_sum(s0);
          if (tr == q && need) {
            const double nv = (j < n - 1) ? sqrt(s0) : 0.0;
            vn1[cq] = nv; vn2[cq] = nv;
            v1 = nv;
          }
        }
      }
    }
    // ---- pivot candidate of this warp, then of the block ----
    double bv; int bp;
    warp_argmax_vp(act ? v1 : -1.0, act ? pos[cq] : 0x7fffffff, bv, bp);
    if (lane == 0) {
      // lp2c changes next only after the barrier below (the next swap)
      wmax[warp] = bv; wpos[warp] = bp; widx[warp] = (bp < n) ? lp2c[bp] : 0;
    }
    __syncthreads();
    if (j + 1 < n) pc = block_pivot(wmax, wpos, widx);
    // no barrier here: wmax, vsh, tsh and pos are written again only after
    // the next step's first barrier, which every reader passes after its
    // reads
  }
  for (int l = tid; l < n; l += Z2_NT) jpvt[l] = lp2c[l] + 1;
  __syncthreads();
}
// Householder QR WITHOUT pivoting (DGEQR2 semantics) in the same register
// tile, for the pre-pivoted stabilization: the columns are already in
// decreasing norm order, so step j factors column j.  With no norm downdate
// and no arg-max, a step has one block barrier: the reflector of column j
// (its warp publishes v, tau) -> barrier -> every warp applies H_j to its
// trailing columns.  v and tau alternate between two buffers by the parity
// of j: the warp that writes the buffer of step j + 2 has passed the barrier
// of step j + 1, which every reader of step j reaches only after its reads.
// work: >= 2 n doubles; red: >= 32 doubles.  perm (optional, 1-based like
// ZGEQP3's jpvt): factor A P instead of A, column j of A P being column
// perm[j] - 1 of A.  Every column is read into the register tile before the
// first finished column is written back, so the permutation costs nothing.
template <int S>
__device__ __noinline__ void qr_reg(double *A, int lda, int n, double *tau, double *work,
                                    double *red, const int *perm) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tr = lane & 15, tc = (warp << 1) | (lane >> 4);
  const int hl = lane & 16;
  double *tsh = red + 24;                              // [2] tau of the step
  double a[S][S];
  int src[S];
#pragma unroll
  for (int q = 0; q < S; ++q) {
    const int c = tc + 16 * q;
    src[q] = (c < n) ? (perm ? perm[c] - 1 : c) : 0;
  }
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const int r = tr + 16 * p, c = tc + 16 * q;
      a[p][q] = (r < n && c < n) ? A[r + (size_t)src[q] * lda] : 0.0;
    }
  __syncthreads();   // every column read before the first is written back
  unsigned done = 0;   // bit q: column tc + 16 q factored (or outside the matrix)
#pragma unroll
  for (int q = 0; q < S; ++q)
    if (tc + 16 * q >= n) done |= 1u << q;
  for (int j = 0; j < n; ++j) {
    const int qc = j >> 4, gc = j & 15;
    const int pj = j >> 4, oj = j & 15;
    double *vsh = work + (j & 1) * n;
    // ---- reflector of column j (DLARFG), by the warp holding it; the
    // finished column goes straight to A(:, j) ----
    if (warp == (gc >> 1)) {
      const bool mine = (lane >> 4) == (gc & 1);
      double col[S];
#pragma unroll
      for (int p = 0; p < S; ++p) col[p] = 0.0;
      switch (qc) {
        QRP_CASE_COL(0) QRP_CASE_COL(1) QRP_CASE_COL(2) QRP_CASE_COL(3) QRP_CASE_COL(4)
        QRP_CASE_COL(5) QRP_CASE_COL(6) QRP_CASE_COL(7) QRP_CASE_COL(8)
        default: break;
      }
      double s0 = 0.0, s1 = 0.0, aj = 0.0;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int r = tr + 16 * p;
        const double x = (r > j && r < n) ? col[p] : 0.0;
        if (p & 1) s1 += x * x; else s0 += x * x;
        if (p == pj) aj = col[p];
      }
      const double ss = hw_sum(s0 + s1);
      const double alpha = __shfl_sync(Z2_FULL, aj, hl | oj);
      double t = 0.0, beta = alpha, sc = 1.0;
      if (j < n - 1 && ss != 0.0) {
        double nb = sqrt(fma(alpha, alpha, ss));
        if (isinf(nb)) nb = dlapy2(alpha, sqrt(ss));
        beta = -copysign(nb, alpha);
        t = (beta - alpha) / beta;
        sc = 1.0 / (alpha - beta);
      }
      if (mine) {
#pragma unroll
        for (int p = 0; p < S; ++p) {
          const int r = tr + 16 * p;
          double vv = 0.0, out = col[p];
          if (r > j) {
            if (t != 0.0) out *= sc;
            vv = out;
          } else if (r == j) {
            out = beta;
            vv = 1.0;
          }
          if (r < n) {
            vsh[r] = vv;
            A[r + (size_t)j * lda] = out;
          }
        }
        if (tr == 0) { tsh[j & 1] = t; tau[j] = t; }
      }
    }
    __syncthreads();
    if (tc == gc) done |= 1u << qc;
    // ---- apply H_j to the trailing columns (DLARF) ----
    const double t = tsh[j & 1];
    if (t != 0.0) {
      double vr[S], d[S];
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int r = tr + 16 * p;
        vr[p] = (r < n) ? vsh[r] : 0.0;   // 0 above row j
        d[p] = 0.0;
      }
      switch (pj) {
        QRP_CASE_DOT(0) QRP_CASE_DOT(1) QRP_CASE_DOT(2) QRP_CASE_DOT(3) QRP_CASE_DOT(4)
        QRP_CASE_DOT(5) QRP_CASE_DOT(6) QRP_CASE_DOT(7) QRP_CASE_DOT(8)
        default: break;
      }
      qrp_colsum<S>(d, tr, hl);
#pragma unroll
      for (int q = 0; q < S; ++q) d[q] = ((done >> q) & 1u) ? 0.0 : t * d[q];
      switch (pj) {
        QRP_CASE_UPD(0) QRP_CASE_UPD(1) QRP_CASE_UPD(2) QRP_CASE_UPD(3) QRP_CASE_UPD(4)
        QRP_CASE_UPD(5) QRP_CASE_UPD(6) QRP_CASE_UPD(7) QRP_CASE_UPD(8)
        default: break;
      }
    }
  }
  __syncthreads();
}

#undef QRP_CASE_COL
#undef QRP_CASE_ROW
#undef QRP_CASE_DOT
#undef QRP_CASE_UPD

// Pivoted QR of the stabilization: register-resident for n <= 144, the
// thread-per-column kernel above that (or without 2n doubles of work space).
__device__ __forceinline__ void blk_geqp3_fast(double *A, int lda, int n, int *jpvt, double *tau,
                                               double *vn1, double *vn2, double *work, int wd,
                                               double *red) {
  if (work != nullptr && wd >= 2 * n) {
    switch ((n + 15) >> 4) {
      case 1: qrp_reg<1>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 2: qrp_reg<2>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 3: qrp_reg<3>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 4: qrp_reg<4>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 5: qrp_reg<5>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 6: qrp_reg<6>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 7: qrp_reg<7>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 8: qrp_reg<8>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      case 9: qrp_reg<9>(A, lda, n, jpvt, tau, vn1, vn2, work, red); return;
      default: break;
    }
  }
  blk_geqp3_tc(A, lda, n, jpvt, tau, vn1, vn2);
}

// QR without pivoting of the pre-pivoted stabilization, register-resident for
// n <= 144 (false when the size or the work space does not allow it).
__device__ __forceinline__ bool qr_reg_any(double *A, int lda, int n, double *tau, double *work,
                                           int wd, double *red, const int *perm = nullptr) {
  if (work == nullptr || wd < 2 * n) return false;
  switch ((n + 15) >> 4) {
    case 1: qr_reg<1>(A, lda, n, tau, work, red, perm); return true;
    case 2: qr_reg<2>(A, lda, n, tau, work, red, perm); return true;
    case 3: qr_reg<3>(A, lda, n, tau, work, red, perm); return true;
    case 4: qr_reg<4>(A, lda, n, tau, work, red, perm); return true;
    case 5: qr_reg<5>(A, lda, n, tau, work, red, perm); return true;
    case 6: qr_reg<6>(A, lda, n, tau, work, red, perm); return true;
    case 7: qr_reg<7>(A, lda, n, tau, work, red, perm); return true;
    case 8: qr_reg<8>(A, lda, n, tau, work, red, perm); return true;
    case 9: qr_reg<9>(A, lda, n, tau, work, red, perm); return true;
    default: return false;
  }
}
