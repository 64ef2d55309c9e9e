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
// pivot candidates are published.
//
// Pivoting follows DGEQP3 without moving data: the logical position of every
// physical column is tracked (pos / lp2c), the arg-max breaks ties by logical
// position as IDAMAX does on the swapped arrays, and the partial norm
// downdate and its recompute threshold are DLAQP2's.  The factors are written
// back in logical column order at the end, so the result has DGEQP3's layout
// (R above the diagonal, reflectors below, tau, 1-based jpvt).
#pragma once
#include "z2_dmma.cuh"

__device__ __forceinline__ double hw_sum(double v) {
  v += __shfl_xor_sync(Z2_FULL, v, 8);
  v += __shfl_xor_sync(Z2_FULL, v, 4);
  v += __shfl_xor_sync(Z2_FULL, v, 2);
  v += __shfl_xor_sync(Z2_FULL, v, 1);
  return v;
}

// better pivot candidate: larger norm, then smaller logical position
__device__ __forceinline__ bool qrp_better(double v, int p, double bv, int bp) {
  return v > bv || (v == bv && p < bp);
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
    // pivot of step 0
    double bv = -1.0; int bp = 0x7fffffff, bc = -1;
    for (int c = tid; c < n; c += Z2_NT)
      if (qrp_better(vn1[c], c, bv, bp)) { bv = vn1[c]; bp = c; bc = c; }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const double ov = __shfl_xor_sync(Z2_FULL, bv, o);
      const int op = __shfl_xor_sync(Z2_FULL, bp, o), oc = __shfl_xor_sync(Z2_FULL, bc, o);
      if (qrp_better(ov, op, bv, bp)) { bv = ov; bp = op; bc = oc; }
    }
    if (lane == 0) { wmax[warp] = bv; wpos[warp] = bp; widx[warp] = bc; }
    __syncthreads();
    bv = wmax[0]; bp = wpos[0]; bc = widx[0];
#pragma unroll
    for (int w = 1; w < Z2_WARPS; ++w)
      if (qrp_better(wmax[w], wpos[w], bv, bp)) { bv = wmax[w]; bp = wpos[w]; bc = widx[w]; }
    pc = bc;
    __syncthreads();
  }

  for (int j = 0; j < n; ++j) {
    const int qc = pc >> 4, gc = pc & 15;
    const int pj = j >> 4, oj = j & 15;
    // ---- reflector of the pivot column (DLARFG), by the warp holding it ----
    if (warp == (gc >> 1)) {
      const bool mine = (lane >> 4) == (gc & 1);
      double col[S];
#pragma unroll
      for (int p = 0; p < S; ++p) col[p] = 0.0;
#pragma unroll
      for (int q = 0; q < S; ++q)
        if (q == qc) {
#pragma unroll
          for (int p = 0; p < S; ++p) col[p] = a[p][q];
        }
      double ss = 0.0, aj = 0.0;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int r = tr + 16 * p;
        if (r > j && r < n) ss += col[p] * col[p];
        if (p == pj) aj = col[p];
      }
      ss = hw_sum(ss);
      const double alpha = __shfl_sync(Z2_FULL, aj, hl | oj);
      double t = 0.0, beta = alpha, sc = 1.0;
      if (j < n - 1 && ss != 0.0) {
        const double xnorm = sqrt(ss);
        beta = -copysign(dlapy2(alpha, xnorm), alpha);
        t = (beta - alpha) / beta;
        sc = 1.0 / (alpha - beta);
      }
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int r = tr + 16 * p;
        double vv = 0.0;
        if (r > j) {
          if (t != 0.0) col[p] *= sc;
          vv = col[p];
        } else if (r == j) {
          col[p] = beta;
          vv = 1.0;
        }
        if (mine && r < n) vsh[r] = vv;
      }
      if (mine) {
#pragma unroll
        for (int q = 0; q < S; ++q)
          if (q == qc) {
#pragma unroll
            for (int p = 0; p < S; ++p) a[p][q] = col[p];
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
      }
#pragma unroll
      for (int q = 0; q < S; ++q) {
        double s0 = 0.0;
#pragma unroll
        for (int p = 0; p < S; ++p) s0 += vr[p] * a[p][q];
        d[q] = s0;
      }
#pragma unroll
      for (int q = 0; q < S; ++q) d[q] = hw_sum(d[q]);
#pragma unroll
      for (int q = 0; q < S; ++q) d[q] = ((done >> q) & 1u) ? 0.0 : t * d[q];
#pragma unroll
      for (int p = 0; p < S; ++p)
#pragma unroll
        for (int q = 0; q < S; ++q) a[p][q] -= d[q] * vr[p];
    }
    // ---- partial norm downdate (DLAQP2): lane q of each half-warp takes
    // column slot q; row j of the group comes from its owner lane ----
    double rowj[S];
#pragma unroll
    for (int q = 0; q < S; ++q) rowj[q] = 0.0;
#pragma unroll
    for (int p = 0; p < S; ++p)
      if (p == pj) {
#pragma unroll
        for (int q = 0; q < S; ++q) rowj[q] = a[p][q];
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
        double temp = fabs(ajc) / v1;
        temp = 1.0 - temp * temp;
        temp = fmax(temp, 0.0);
        const double qq = v1 / vn2[cq];
        if (temp * qq * qq <= tol3z) {
          need = true;
        } else {
          v1 = v1 * sqrt(temp);
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
    // ---- pivot candidate of this warp ----
    double bv = -1.0; int bp = 0x7fffffff, bc = -1;
    if (act) { bv = v1; bp = pos[cq]; bc = cq; }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const double ov = __shfl_xor_sync(Z2_FULL, bv, o);
      const int op = __shfl_xor_sync(Z2_FULL, bp, o), oc = __shfl_xor_sync(Z2_FULL, bc, o);
      if (qrp_better(ov, op, bv, bp)) { bv = ov; bp = op; bc = oc; }
    }
    if (lane == 0) { wmax[warp] = bv; wpos[warp] = bp; widx[warp] = bc; }
    __syncthreads();
    if (j + 1 < n) {
      bv = wmax[0]; bp = wpos[0]; bc = widx[0];
#pragma unroll
      for (int w = 1; w < Z2_WARPS; ++w)
        if (qrp_better(wmax[w], wpos[w], bv, bp)) { bv = wmax[w]; bp = wpos[w]; bc = widx[w]; }
      pc = bc;
    }
    // no barrier here: wmax, vsh, tsh and pos are written again only after
    // the next step's first barrier, which every reader passes after its reads
  }
  // write back in logical column order
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const int r = tr + 16 * p, c = tc + 16 * q;
      if (r < n && c < n) A[r + (size_t)pos[c] * lda] = a[p][q];
    }
  for (int l = tid; l < n; l += Z2_NT) jpvt[l] = lp2c[l] + 1;
  __syncthreads();
}

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
