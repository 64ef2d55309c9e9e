// z2_qrf.cuh -- Householder QR without pivoting for the UDV stabilization of
// the chain (the pre-pivoted form below), and the application of Q^T.
//
// A panel of PW columns is factored by ONE warp with the panel held in its
// registers (lane l keeps rows j0 + l + 32 t): each column step needs only
// warp shuffles, no block barrier.  The panel's reflectors then reach the
// trailing columns as the compact WY form, C <- C - V (T^T (V^T C)), by DMMA
// GEMMs over the whole block (DGEQRF's structure).  Q^T is applied to a
// right-hand side the same way (DORMQR 'L','T'), with the T of each panel
// kept from the factorization.
#pragma once
#include "z2_dmma.cuh"

// DGEQR2 on the panel A(j0:n, j0:j0+ib), ib <= PW, n - j0 <= 32 T, by the
// calling warp (all 32 lanes).  Reflector j = j0 + k: v(j) = 1 implicit,
// v(j+1:n) stored below the diagonal, beta on the diagonal, tau[j].  The
// panel stays in registers; the column loop is not unrolled (the current
// column is selected out of the register tile), so each instantiation is
// compiled once per (T, PW).
template <int T, int PW>
__device__ __noinline__ void warp_panel_qr(double *A, int lda, int n, int j0, int ib, double *tau) {
  const int lane = threadIdx.x & 31;
  double a[T][PW];
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int r = j0 + lane + 32 * t;
#pragma unroll
    for (int c = 0; c < PW; ++c) a[t][c] = (r < n && c < ib) ? A[r + (size_t)(j0 + c) * lda] : 0.0;
  }
  for (int k = 0; k < ib; ++k) {
    // column k below the diagonal (rows past n hold zeros), and A(j, j) on lane k
    double v[T];
    double akk = 0.0;
#pragma unroll
    for (int c = 0; c < PW; ++c) akk = (c == k) ? a[0][c] : akk;
#pragma unroll
    for (int t = 0; t < T; ++t) {
      double x = 0.0;
#pragma unroll
      for (int c = 0; c < PW; ++c) x = (c == k) ? a[t][c] : x;
      v[t] = (lane + 32 * t > k) ? x : 0.0;
    }
    double ss = 0.0;
#pragma unroll
    for (int t = 0; t < T; ++t) ss = fma(v[t], v[t], ss);
    ss = warp_sum(ss);
    const double alpha = __shfl_sync(Z2_FULL, akk, k);
    double tk = 0.0, beta = alpha, sc = 1.0;
    if (j0 + k < n - 1 && ss != 0.0) {
      beta = -copysign(dlapy2(alpha, sqrt(ss)), alpha);
      tk = (beta - alpha) / beta;
      sc = 1.0 / (alpha - beta);
    }
    if (tk != 0.0) {
#pragma unroll
      for (int t = 0; t < T; ++t) v[t] *= sc;
      // H_k on the panel's later columns: w_c = A(j, c) + v^T A(j+1:, c)
      double w[PW];
#pragma unroll
      for (int c = 0; c < PW; ++c) {
        double d = 0.0;
#pragma unroll
        for (int t = 0; t < T; ++t) d = fma(v[t], a[t][c], d);
        w[c] = d;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int c = 0; c < PW; ++c) w[c] += __shfl_xor_sync(Z2_FULL, w[c], off);
#pragma unroll
      for (int c = 0; c < PW; ++c) {
        if (c > k) {                                   // warp-uniform
          const double akc = __shfl_sync(Z2_FULL, a[0][c], k);
          const double ww = (w[c] + akc) * tk;
          if (lane == k) a[0][c] = akc - ww;
#pragma unroll
          for (int t = 0; t < T; ++t) a[t][c] = fma(-ww, v[t], a[t][c]);
        } else if (c == k) {
#pragma unroll
          for (int t = 0; t < T; ++t)
            if (lane + 32 * t > k) a[t][c] = v[t];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < PW; ++c)
      if (c == k && lane == k) a[0][c] = beta;
    if (lane == 0) tau[j0 + k] = tk;
  }
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int r = j0 + lane + 32 * t;
#pragma unroll
    for (int c = 0; c < PW; ++c)
      if (r < n && c < ib) A[r + (size_t)(j0 + c) * lda] = a[t][c];
  }
  __syncwarp();
}

// T of one block of ib <= 16 reflectors from S = V^T V and the block's tau
// (DLARFT forward / columnwise, as in blk_geqrf): T upper triangular, ld ib;
// threads 0..ib-1 each form one row.  Caller synchronises.
__device__ __forceinline__ void larft_rows(const double *S, double *Tm, int ib, const double *tb) {
  const int r = threadIdx.x;
  if (r >= ib) return;
  double tr[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    double t = 0.0;
    if (c < ib) {
      if (c == r) {
        t = tb[c];
      } else if (c > r) {
        double a0 = 0.0, a1 = 0.0;
#pragma unroll
        for (int q = 0; q < c; ++q) {
          if (q >= r) {
            if (q & 1) a1 += tr[q] * S[q + c * ib];
            else a0 += tr[q] * S[q + c * ib];
          }
        }
        t = -tb[c] * (a0 + a1);
      }
    }
    tr[c] = t;
  }
#pragma unroll
  for (int c = 0; c < 16; ++c)
    if (c < ib) Tm[r + c * ib] = tr[c];
}

// C (mp x nc, ldc) <- (I - V T V^T)^T C = C - V (T^T (V^T C)) with V (mp x ib,
// ldv, unit lower) and T (ib x ib, ld ib), in chunks of ncb columns; W:
// ldw x ncb scratch (ldw >= ib).
__device__ __noinline__ void blk_apply_wy_t(const double *V, int ldv, const double *Tm, int ib,
                                            int mp, double *C, int ldc, int nc, double *W,
                                            int ldw, int ncb) {
  for (int c0 = 0; c0 < nc; c0 += ncb) {
    const int w = (nc - c0) < ncb ? (nc - c0) : ncb;
    double *Cc = C + (size_t)c0 * ldc;
    blk_dmma(ib, w, mp, 1.0, MatRef{V, ldv, 1}, false, MatRef{Cc, 1, ldc}, false, 0.0, W, ldw);
    for (int c = threadIdx.x; c < w; c += Z2_NT) {
      double x[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) x[q] = (q < ib) ? W[q + (size_t)c * ldw] : 0.0;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        if (r < ib) {
          double t = 0.0;
#pragma unroll
          for (int q = 0; q <= r; ++q) t += Tm[q + r * ib] * x[q];   // (T^T x)_r
          W[r + (size_t)c * ldw] = t;
        }
      }
    }
    __syncthreads();
    blk_dmma(mp, w, ib, -1.0, MatRef{V, 1, ldv}, false, MatRef{W, 1, ldw}, false, 1.0, Cc, ldc);
  }
}

// V (mp x ib, ldv) = the unit lower trapezoidal reflectors stored in
// A(j0:n, j0:j0+ib).
__device__ __forceinline__ void blk_load_v(double *V, int ldv, const double *A, int lda, int j0,
                                           int mp, int ib) {
  for (int c = threadIdx.x >> 5; c < ib; c += Z2_WARPS)
    for (int r = threadIdx.x & 31; r < mp; r += 32)
      V[r + (size_t)c * ldv] = (r == c) ? 1.0 : (r > c ? A[(j0 + r) + (size_t)(j0 + c) * lda] : 0.0);
  __syncthreads();
}

// Shared work space (doubles) of blk_geqrf_wp / blk_ormqr_wp for an n x n
// matrix with panels of nb columns, updating ncb columns at a time.
__host__ __device__ __forceinline__ int qrf_ldv(int n) { return ((n + 11) & ~15) + 4; }
__host__ __device__ __forceinline__ int qrf_work(int n, int nb, int ncb) {
  return qrf_ldv(n) * nb + (nb + 1) * ncb + 2 * nb * nb;
}
// Panel width of the pre-pivoted QR for an n x n matrix (the warp holds
// n <= 32 T rows of 16 columns up to n = 160, of 8 columns above).
__host__ __device__ __forceinline__ int qrf_pw(int n) { return n <= 160 ? 16 : 8; }
// Columns updated per chunk within wd doubles of work space (a multiple of 8,
// at most n), 0 when even 8 do not fit.
__host__ __device__ __forceinline__ int qrf_ncb(int n, int wd) {
  const int nb = qrf_pw(n);
  int c = (wd - qrf_ldv(n) * nb - 2 * nb * nb) / (nb + 1);
  c = c < n ? c : n;
  c &= ~7;
  return c >= 8 ? c : 0;
}
// The work space the chain reserves so that the pre-pivoted QR always runs:
// chunks of 64 columns.
__host__ __device__ __forceinline__ int qrf_min_work(int n) {
  return qrf_work(n, qrf_pw(n), n < 64 ? ((n + 7) & ~7) : 64);
}

// Householder QR without pivoting of the square n x n matrix A (DGEQRF):
// panels of PW columns by warp 0 in registers (n <= 32 T), trailing updates
// as DMMA GEMMs on ncb columns at a time.  Tsave (optional, global,
// (n / PW + 1) PW^2 doubles) keeps each panel's T for blk_ormqr_wp.  work:
// qrf_work(n, PW, ncb) doubles.
template <int T, int PW>
__device__ __noinline__ void blk_geqrf_wp(double *A, int lda, int n, double *tau, double *Tsave,
                                          double *work, int ncb) {
  const int ldv = qrf_ldv(n), ldw = PW + 1;
  double *V = work;
  double *W = V + (size_t)ldv * PW;
  double *S = W + (size_t)ldw * ncb;
  double *Tm = S + PW * PW;
  for (int j0 = 0, p = 0; j0 < n; j0 += PW, ++p) {
    const int ib = (n - j0) < PW ? (n - j0) : PW;
    const int mp = n - j0, nc = n - j0 - ib;
    if ((threadIdx.x >> 5) == 0) warp_panel_qr<T, PW>(A, lda, n, j0, ib, tau);
    __syncthreads();
    if (nc <= 0 && !Tsave) break;
    blk_load_v(V, ldv, A, lda, j0, mp, ib);
    blk_dmma(ib, ib, mp, 1.0, MatRef{V, ldv, 1}, false, MatRef{V, 1, ldv}, false, 0.0, S, ib);
    double *Tp = Tsave ? Tsave + (size_t)p * PW * PW : Tm;
    larft_rows(S, Tp, ib, tau + j0);
    __syncthreads();
    if (nc > 0)
      blk_apply_wy_t(V, ldv, Tp, ib, mp, A + j0 + (size_t)(j0 + ib) * lda, lda, nc, W, ldw, ncb);
  }
}

// X (n x nc, ldx) <- Q^T X for Q = H_0 H_1 ... H_{n-1} of blk_geqrf_wp (DORMQR
// 'L','T'): panel by panel from the first, each as the compact WY form with
// the T kept in Tsave, ncb columns at a time.  work: qrf_work(n, PW, ncb).
template <int PW>
__device__ __noinline__ void blk_ormqr_wp(const double *A, int lda, int n, const double *Tsave,
                                          double *X, int ldx, int nc, double *work, int ncb) {
  const int ldv = qrf_ldv(n), ldw = PW + 1;
  double *V = work;
  double *W = V + (size_t)ldv * PW;
  for (int j0 = 0, p = 0; j0 < n; j0 += PW, ++p) {
    const int ib = (n - j0) < PW ? (n - j0) : PW;
    const int mp = n - j0;
    blk_load_v(V, ldv, A, lda, j0, mp, ib);
    blk_apply_wy_t(V, ldv, Tsave + (size_t)p * PW * PW, ib, mp, X + j0, ldx, nc, W, ldw, ncb);
  }
}
