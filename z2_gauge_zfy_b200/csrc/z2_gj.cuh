// z2_gj.cuh -- register-resident matrix inverse by Gauss-Jordan elimination
// with partial pivoting, for the middle matrix of the pre-pivoted
// stabilization.
//
// The scale-split middle matrix M' (entries of order one) only has to be
// inverted, not orthogonalised, so elimination with partial pivoting
// (DGETRF's pivot rule, the largest |entry| of the column among the rows not
// yet used, here to within 2^-12 relative) replaces the Householder QR there:
// per column one arg-max, one reciprocal and a rank-1 update, against the
// QR's norm, square root, two divisions, dot products with their reductions
// and update; and the inverse comes out whole, so no triangular solves and no
// orthogonal factor follow.
#pragma once
#include "z2_qrp.cuh"

#define GJ_COL(Q) \
  case Q:         \
    if (Q < S) {  \
      _Pragma("unroll") for (int p = 0; p < S; ++p) col[p] = a[p][Q < S ? Q : 0]; \
    }             \
    break;
#define GJ_ROW(P) \
  case P:         \
    if (P < S) {  \
      _Pragma("unroll") for (int q = 0; q < S; ++q) rowv[q] = a[P < S ? P : 0][q]; \
    }             \
    break;
#define GJ_PICK(P) \
  case P:          \
    if (P < S) cv = col[P < S ? P : 0]; \
    break;
#define GJ_PCOL(Q) \
  case Q:          \
    if (Q < S) {   \
      _Pragma("unroll") for (int p = 0; p < S; ++p) \
        a[p][Q < S ? Q : 0] = (tr + 16 * p == pr) ? 1.0 : -l[p] * rd; \
    }              \
    break;

// Inverse of the n x n matrix A (lda; shared or global memory) in place by
// Gauss-Jordan elimination with partial pivoting (exchange steps on the
// pivots (piv[j], j), rows not swapped), n <= 16 S.  The tile lives in
// registers as in qr_reg: lane tr of column group tc holds rows tr + 16 p of
// columns tc + 16 q.  A step j, with pivot row p, pivot d and
// l_r = A(r, j) (r != p):  A(p, :) /= d, then A(r, c) -= l_r A(p, c) for
// r != p, c != j, A(r, j) = -l_r / d, A(p, j) = 1 / d (one barrier per
// step: the half-warp holding column j picks the pivot with one warp max and
// publishes the column (one buffer of n per step parity), every thread takes
// the pivot row from its own half-warp by shuffles).
// The registers keep each picked row times its pivot d (so the pivot row
// needs no rescaling at its step: its multiplier is 0 and only A(p, j) is
// set, to 1); later steps scale it consistently, and the write-back divides
// by d.  After the n steps the tile T satisfies A^-1(j, k) = T(piv[j], m)
// with piv[m] = k, so on exit row j of A holds rs[j] T(piv[j], :) (rs
// optional, nullptr for 1) and
//   A^-1 = (that matrix) P,   P(m, k) = 1 iff piv[m] = k.
// work: >= 4 n doubles; red: >= 32 doubles.
template <int S>
__device__ __noinline__ void gj_reg(double *A, int lda, int n, int *piv, const double *rs,
                                    double *work, double *red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tr = lane & 15, tc = (warp << 1) | (lane >> 4);
  const int hl = lane & 16;
  double *lbuf = work;                                      // [2][n] column j of the step
  int *rstep = reinterpret_cast<int *>(work + 2 * n);       // [n] step at which row r was picked
  int *pbuf = reinterpret_cast<int *>(red + 24);            // [2] pivot row of the step
  double *dbuf = red + 26;                                  // [2] 1 / pivot of the step
  double *rdk = work + 2 * n + (n + 1) / 2;                 // [n] 1 / pivot of step k
  double a[S][S];
#pragma unroll
  for (int p = 0; p < S; ++p)
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const int r = tr + 16 * p, c = tc + 16 * q;
      a[p][q] = (r < n && c < n) ? A[r + (size_t)c * lda] : 0.0;
    }
  __syncthreads();
  unsigned used = 0;   // bit p: row tr + 16 p was picked at an earlier step (or is outside)
#pragma unroll
  for (int p = 0; p < S; ++p)
    if (tr + 16 * p >= n) used |= 1u << p;
  for (int j = 0; j < n; ++j) {
    const int qj = j >> 4, gj = j & 15;
    double *lb = lbuf + (size_t)(j & 1) * n;
    if (warp == (gj >> 1)) {
      const bool mine = (lane >> 4) == (gj & 1);
      double col[S];
#pragma unroll
      for (int p = 0; p < S; ++p) col[p] = 0.0;
      switch (qj) {
        GJ_COL(0) GJ_COL(1) GJ_COL(2) GJ_COL(3) GJ_COL(4) GJ_COL(5) GJ_COL(6) GJ_COL(7) GJ_COL(8)
        default: break;
      }
      unsigned key = 0;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const unsigned k =
            ((unsigned)__double2hiint(fabs(col[p])) & 0xFFFFFF00u) | (unsigned)(255 - (tr + 16 * p));
        if (mine && !((used >> p) & 1u)) key = max(key, k);
      }
      key = __reduce_max_sync(Z2_FULL, key);
      const int br = 255 - (int)(key & 0xFFu);
      double cv = 0.0;
      switch (br >> 4) {
        GJ_PICK(0) GJ_PICK(1) GJ_PICK(2) GJ_PICK(3) GJ_PICK(4) GJ_PICK(5) GJ_PICK(6) GJ_PICK(7)
        GJ_PICK(8)
        default: break;
      }
      const double pv = __shfl_sync(Z2_FULL, cv, hl | (br & 15));
      if (mine) {
#pragma unroll
        for (int p = 0; p < S; ++p) {
          const int r = tr + 16 * p;
          if (r < n) lb[r] = (r == br) ? 0.0 : col[p];
        }
        if (tr == 0) {
          const double rpv = 1.0 / pv;
          pbuf[j & 1] = br;
          dbuf[j & 1] = rpv;
          rdk[j] = rpv;
          piv[j] = br;
          rstep[br] = j;
        }
      }
    }
    __syncthreads();
    const int pr = pbuf[j & 1];
    const double rd = dbuf[j & 1];
    if ((pr & 15) == tr) used |= 1u << (pr >> 4);
    double rowv[S];
#pragma unroll
    for (int q = 0; q < S; ++q) rowv[q] = 0.0;
    switch (pr >> 4) {
      GJ_ROW(0) GJ_ROW(1) GJ_ROW(2) GJ_ROW(3) GJ_ROW(4) GJ_ROW(5) GJ_ROW(6) GJ_ROW(7) GJ_ROW(8)
      default: break;
    }
    double u[S], l[S];
#pragma unroll
    for (int q = 0; q < S; ++q) u[q] = __shfl_sync(Z2_FULL, rowv[q], hl | (pr & 15)) * rd;
#pragma unroll
    for (int p = 0; p < S; ++p) {
      const int r = tr + 16 * p;
      l[p] = (r < n) ? lb[r] : 0.0;   // 0 for the pivot row
    }
    // column j becomes -l / d, and 1 in the pivot row (the stored pivot row
    // keeps the factor d, see below); set before the rank-1 update, which
    // leaves it as it is (u is 0 in column j)
    if (tc == gj) {
      switch (qj) {
        GJ_PCOL(0) GJ_PCOL(1) GJ_PCOL(2) GJ_PCOL(3) GJ_PCOL(4) GJ_PCOL(5) GJ_PCOL(6) GJ_PCOL(7)
        GJ_PCOL(8)
        default: break;
      }
    }
#pragma unroll
    for (int q = 0; q < S; ++q)
      if (tc == gj && q == qj) u[q] = 0.0;
#pragma unroll
    for (int p = 0; p < S; ++p)
#pragma unroll
      for (int q = 0; q < S; ++q) a[p][q] -= l[p] * u[q];
  }
  __syncthreads();
  // row r of T (picked at step rstep[r]) goes to row rstep[r], scaled
#pragma unroll
  for (int p = 0; p < S; ++p) {
    const int r = tr + 16 * p;
    if (r < n) {
      const int k = rstep[r];
      const double sc = rs ? rs[k] * rdk[k] : rdk[k];
#pragma unroll
      for (int q = 0; q < S; ++q) {
        const int c = tc + 16 * q;
        if (c < n) A[k + (size_t)c * lda] = a[p][q] * sc;
      }
    }
  }
  __syncthreads();
}

#undef GJ_COL
#undef GJ_ROW
#undef GJ_PICK
#undef GJ_PCOL

// gj_reg for n <= 144 with work >= 4 n doubles; false when it does not apply.
__device__ __forceinline__ bool gj_reg_any(double *A, int lda, int n, int *piv, const double *rs,
                                           double *work, int wd, double *red) {
  if (work == nullptr || n < 1 || n > 144 || wd < 4 * n) return false;
  switch ((n + 15) >> 4) {
    case 1: gj_reg<1>(A, lda, n, piv, rs, work, red); return true;
    case 2: gj_reg<2>(A, lda, n, piv, rs, work, red); return true;
    case 3: gj_reg<3>(A, lda, n, piv, rs, work, red); return true;
    case 4: gj_reg<4>(A, lda, n, piv, rs, work, red); return true;
    case 5: gj_reg<5>(A, lda, n, piv, rs, work, red); return true;
    case 6: gj_reg<6>(A, lda, n, piv, rs, work, red); return true;
    case 7: gj_reg<7>(A, lda, n, piv, rs, work, red); return true;
    case 8: gj_reg<8>(A, lda, n, piv, rs, work, red); return true;
    case 9: gj_reg<9>(A, lda, n, piv, rs, work, red); return true;
    default: return false;
  }
}
