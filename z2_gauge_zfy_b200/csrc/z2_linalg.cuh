// z2_linalg.cuh -- CTA-cooperative dense FP64 linear algebra.
//
// Every routine is called by all Z2_NT threads of a block, operates on
// column-major matrices through generic pointers (shared or global memory)
// and ends with the block synchronised.  The routines restate the LAPACK /
// BLAS operations the reference's stabilization calls (ZGEQP3, ZUNGQR,
// ZUNMQR, ZTRMM, ZTRSM, ZLAPMR, ZLAPMT, ZGEMM; src/stabilization.f90:42-200)
// for real matrices, with the same algorithms (Householder reflectors of
// DLARFG, partial column-norm downdating of DLAQP2, column-oriented
// triangular solves of DTRSM).
#pragma once
#include "z2_common.cuh"

__device__ __forceinline__ double dlapy2(double x, double y) {
  double xa = fabs(x), ya = fabs(y);
  double w = fmax(xa, ya), z = fmin(xa, ya);
  if (z == 0.0) return w;
  double q = z / w;
  return w * sqrt(1.0 + q * q);
}

// Element walk over an m x n column-major block whose operands sit in L2 or
// HBM: the elements are dealt to the threads in column-major order
// (consecutive threads take consecutive rows, so accesses stay coalesced), B
// per thread at a time, and every batch issues its B loads before any use.  ld(i, j) returns
// the element's operands, use(v, i, j) consumes them.
template <int B, class T, class Ld, class Use>
__device__ __forceinline__ void blk_walk(int m, int n, Ld ld, Use use) {
  if (m <= 0 || n <= 0) return;
  const int dj = Z2_NT / m, di = Z2_NT % m;
  int i = threadIdx.x % m, j = threadIdx.x / m;
  const long long total = (long long)m * n;
  for (long long e0 = 0; e0 < total; e0 += (long long)B * Z2_NT) {
    int ii[B], jj[B];
    T v[B];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      ii[b] = i;
      jj[b] = j;
      if (j < n) v[b] = ld(i, j);
      i += di;
      j += dj;
      if (i >= m) { i -= m; ++j; }
    }
#pragma unroll
    for (int b = 0; b < B; ++b)
      if (jj[b] < n) use(v[b], ii[b], jj[b]);
  }
}

// Element copies are issued in batches of 4 loads before 4 stores (dst and
// src may be the same allocation, so the compiler keeps program order).
__device__ __noinline__ void blk_copy(double *dst, int ldd, const double *src, int lds, int m, int n) {
  const int lane = threadIdx.x & 31;
  for (int j = threadIdx.x / 32; j < n; j += Z2_WARPS) {
    const double *s = src + (size_t)j * lds;
    double *d = dst + (size_t)j * ldd;
    int i = lane;
    for (; i + 96 < m; i += 128) {
      const double a0 = s[i], a1 = s[i + 32], a2 = s[i + 64], a3 = s[i + 96];
      d[i] = a0; d[i + 32] = a1; d[i + 64] = a2; d[i + 96] = a3;
    }
    for (; i < m; i += 32) d[i] = s[i];
  }
  __syncthreads();
}
// dst = src^T (src m x n -> dst n x m)
__device__ __noinline__ void blk_transpose(double *dst, int ldd, const double *src, int lds, int m, int n) {
  for (int j = threadIdx.x / 32; j < m; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < n; i += 32) dst[i + (size_t)j * ldd] = src[j + (size_t)i * lds];
  __syncthreads();
}
__device__ __noinline__ void blk_identity(double *A, int lda, int n) {
  for (int j = threadIdx.x / 32; j < n; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < n; i += 32) A[i + (size_t)j * lda] = (i == j) ? 1.0 : 0.0;
  __syncthreads();
}
__device__ __noinline__ void blk_fill(double *v, int n, double x) {
  for (int i = threadIdx.x; i < n; i += Z2_NT) v[i] = x;
  __syncthreads();
}
__device__ __noinline__ void blk_scale(double *A, int lda, int m, int n, double a) {
  for (int j = threadIdx.x / 32; j < n; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < m; i += 32) A[i + (size_t)j * lda] *= a;
  __syncthreads();
}
// A(:, j) *= d(j)
__device__ __noinline__ void blk_scale_cols(double *A, int lda, int m, int n, const double *d) {
  for (int j = threadIdx.x / 32; j < n; j += Z2_WARPS) {
    double dj = d[j];
    for (int i = threadIdx.x & 31; i < m; i += 32) A[i + (size_t)j * lda] *= dj;
  }
  __syncthreads();
}

// max |A - B| (compare_mat, src/stabilization.f90:365-372)
__device__ __noinline__ double blk_maxdiff(const double *A, int lda, const double *B, int ldb, int n, double *red) {
  double m = 0.0;
  for (int j = threadIdx.x / 32; j < n; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < n; i += 32) {
      double d = fabs(A[i + (size_t)j * lda] - B[i + (size_t)j * ldb]);
      m = (d > m || d != d) ? d : m;   // keep NaN visible
    }
  double r = blk_max(m, red);
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------
// Pivoted Householder QR (DGEQP3 -> DLAQP2 semantics, all columns free).
// On exit A holds R and the reflectors, tau the scalar factors, jpvt the
// 1-based pivots (column j of A*P is column jpvt(j) of A).
// ---------------------------------------------------------------------------
__device__ __noinline__ void blk_geqp3(double *A, int lda, int n, int *jpvt, double *tau, double *vn1,
                          double *vn2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double tol3z = 1.0536712127723509e-08;   // sqrt(dlamch('E')) = sqrt(2^-53)
  for (int j = warp; j < n; j += Z2_WARPS) {
    double s = 0.0;
    for (int i = lane; i < n; i += 32) { double a = A[i + (size_t)j * lda]; s += a * a; }
    s = warp_sum(s);
    if (lane == 0) { double nr = sqrt(s); vn1[j] = nr; vn2[j] = nr; jpvt[j] = j + 1; }
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    // IDAMAX over vn1(j:n): first index of the largest value
    double bv = -1.0; int bi = n;
    for (int k = j + lane; k < n; k += 32) { double v = vn1[k]; if (v > bv) { bv = v; bi = k; } }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      double ov = __shfl_xor_sync(Z2_FULL, bv, o);
      int oi = __shfl_xor_sync(Z2_FULL, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    const int pvt = bi;
    __syncthreads();
    if (warp == 0) {
      double *Aj = A + (size_t)j * lda;
      if (pvt != j) {
        double *Ap = A + (size_t)pvt * lda;
        for (int i = lane; i < n; i += 32) { double t = Ap[i]; Ap[i] = Aj[i]; Aj[i] = t; }
        if (lane == 0) {
          int t = jpvt[pvt]; jpvt[pvt] = jpvt[j]; jpvt[j] = t;
          vn1[pvt] = vn1[j]; vn2[pvt] = vn2[j];
        }
      }
      __syncwarp();
      // DLARFG on A(j:n, j)
      double s = 0.0;
      for (int i = j + 1 + lane; i < n; i += 32) { double a = Aj[i]; s += a * a; }
      s = warp_sum(s);
      double alpha = Aj[j];
      double t = 0.0, beta = alpha;
      if (j < n - 1 && s != 0.0) {
        double xnorm = sqrt(s);
        beta = -copysign(dlapy2(alpha, xnorm), alpha);
        t = (beta - alpha) / beta;
        double sc = 1.0 / (alpha - beta);
        for (int i = j + 1 + lane; i < n; i += 32) Aj[i] *= sc;
      }
      __syncwarp();
      if (lane == 0) { tau[j] = t; Aj[j] = beta; }
    }
    __syncthreads();
    // DLARF('Left') on the trailing columns + norm downdate, one warp per column
    const double tj = tau[j];
    const double *v = A + (size_t)j * lda;
    for (int k = j + 1 + warp; k < n; k += Z2_WARPS) {
      double *Ak = A + (size_t)k * lda;
      if (tj != 0.0) {
        double w = 0.0;
        for (int i = j + 1 + lane; i < n; i += 32) w += v[i] * Ak[i];
        w = warp_sum(w) + Ak[j];
        double tw = tj * w;
        __syncwarp();
        if (lane == 0) Ak[j] -= tw;
        for (int i = j + 1 + lane; i < n; i += 32) Ak[i] -= v[i] * tw;
      }
      __syncwarp();
      double v1 = vn1[k];
      if (v1 != 0.0) {
        double r = fabs(Ak[j]) / v1;
        double temp = fmax(1.0 - r * r, 0.0);
        double q = v1 / vn2[k];
        double temp2 = temp * q * q;
        if (temp2 <= tol3z) {
          double nv = 0.0;
          if (j < n - 1) {
            double s2 = 0.0;
            for (int i = j + 1 + lane; i < n; i += 32) { double a = Ak[i]; s2 += a * a; }
            nv = sqrt(warp_sum(s2));
          }
          if (lane == 0) { vn1[k] = nv; vn2[k] = nv; }
        } else if (lane == 0) {
          vn1[k] = v1 * sqrt(temp);
        }
      }
    }
    __syncthreads();
  }
}

// Unpivoted Householder QR (DGEQR2), used for the 2N x 2N UDV of the
// time-displaced Green's function.
__device__ __noinline__ void blk_geqr2(double *A, int lda, int m, int n, double *tau) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kmax = m < n ? m : n;
  for (int j = 0; j < kmax; ++j) {
    if (warp == 0) {
      double *Aj = A + (size_t)j * lda;
      double s = 0.0;
      for (int i = j + 1 + lane; i < m; i += 32) { double a = Aj[i]; s += a * a; }
      s = warp_sum(s);
      double alpha = Aj[j];
      double t = 0.0, beta = alpha;
      if (j < m - 1 && s != 0.0) {
        double xnorm = sqrt(s);
        beta = -copysign(dlapy2(alpha, xnorm), alpha);
        t = (beta - alpha) / beta;
        double sc = 1.0 / (alpha - beta);
        for (int i = j + 1 + lane; i < m; i += 32) Aj[i] *= sc;
      }
      __syncwarp();
      if (lane == 0) { tau[j] = t; Aj[j] = beta; }
    }
    __syncthreads();
    const double tj = tau[j];
    const double *v = A + (size_t)j * lda;
    if (tj != 0.0) {
      for (int k = j + 1 + warp; k < n; k += Z2_WARPS) {
        double *Ak = A + (size_t)k * lda;
        double w = 0.0;
        for (int i = j + 1 + lane; i < m; i += 32) w += v[i] * Ak[i];
        w = warp_sum(w) + Ak[j];
        double tw = tj * w;
        __syncwarp();
        if (lane == 0) Ak[j] -= tw;
        for (int i = j + 1 + lane; i < m; i += 32) Ak[i] -= v[i] * tw;
      }
    }
    __syncthreads();
  }
}

// QDRP_decompose's split (src/stabilization.f90:61-66): D(i) = |R(i,i)|,
// R(i, i:n) /= D(i).
// The rows are scaled by the reciprocal of D (one division per row instead
// of one per element; rd: n doubles of scratch, left holding 1/D).
__device__ __noinline__ void blk_qdrp_scale(double *A, int lda, int n, double *D, double *rd) {
  for (int i = threadIdx.x; i < n; i += Z2_NT) {
    const double d = fabs(A[i + (size_t)i * lda]);
    D[i] = d;
    rd[i] = 1.0 / d;
  }
  __syncthreads();
  for (int j = threadIdx.x / 32; j < n; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i <= j; i += 32) A[i + (size_t)j * lda] = A[i + (size_t)j * lda] * rd[i];
  __syncthreads();
}

// Row / column permutations with 1-based pivots (ZLAPMR, ZLAPMT).
// forward row: dst(i,:) = src(jpvt(i),:) ; backward row: dst(jpvt(i),:) = src(i,:)
__device__ __noinline__ void blk_perm_rows(double *dst, int ldd, const double *src, int lds, int n, int nc,
                              const int *jpvt, bool forward) {
  for (int j = threadIdx.x / 32; j < nc; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < n; i += 32) {
      int p = jpvt[i] - 1;
      if (forward) dst[i + (size_t)j * ldd] = src[p + (size_t)j * lds];
      else dst[p + (size_t)j * ldd] = src[i + (size_t)j * lds];
    }
  __syncthreads();
}
// forward col: dst(:,j) = src(:,jpvt(j)) ; backward col: dst(:,jpvt(j)) = src(:,j)
__device__ __noinline__ void blk_perm_cols(double *dst, int ldd, const double *src, int lds, int nr, int n,
                              const int *jpvt, bool forward) {
  for (int j = threadIdx.x / 32; j < n; j += Z2_WARPS) {
    int p = jpvt[j] - 1;
    for (int i = threadIdx.x & 31; i < nr; i += 32) {
      if (forward) dst[i + (size_t)j * ldd] = src[i + (size_t)p * lds];
      else dst[i + (size_t)p * ldd] = src[i + (size_t)j * lds];
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double ld_op(const double *X, int ld, bool t, bool tri, int r, int c) {
  // element (r, c) of op(X)
  int sr = t ? c : r, sc = t ? r : c;
  if (tri && sr > sc) return 0.0;
  return X[sr + (size_t)sc * ld];
}

// ---------------------------------------------------------------------------
// LU with partial pivoting and explicit inverse (stands in for LINPACK
// ZGEFA/ZGEDI of INV_C, lib/package_of_matrix/Modules/mat_mod.f90:296-336).
// A (n x n) is overwritten by its inverse; W is an n x n workspace.
// ---------------------------------------------------------------------------
__device__ __noinline__ void blk_inverse(double *A, int lda, int n, double *W, int ldw, int *ipiv,
                            double *red, int *flag) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // LU (right-looking, unblocked)
  for (int k = 0; k < n; ++k) {
    double bv = -1.0; int bi = n;
    for (int i = k + threadIdx.x; i < n; i += Z2_NT) {
      double v = fabs(A[i + (size_t)k * lda]);
      if (v > bv) { bv = v; bi = i; }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      double ov = __shfl_xor_sync(Z2_FULL, bv, o);
      int oi = __shfl_xor_sync(Z2_FULL, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    __syncthreads();
    if (lane == 0) { red[warp] = bv; flag[warp] = bi; }
    __syncthreads();
    bv = red[0]; bi = flag[0];
    for (int w = 1; w < Z2_WARPS; ++w)
      if (red[w] > bv || (red[w] == bv && flag[w] < bi)) { bv = red[w]; bi = flag[w]; }
    const int p = bi;
    __syncthreads();
    if (threadIdx.x == 0) ipiv[k] = p;
    if (p != k)
      for (int j = threadIdx.x; j < n; j += Z2_NT) {
        double t = A[k + (size_t)j * lda];
        A[k + (size_t)j * lda] = A[p + (size_t)j * lda];
        A[p + (size_t)j * lda] = t;
      }
    __syncthreads();
    const double piv = A[k + (size_t)k * lda];
    for (int i = k + 1 + threadIdx.x; i < n; i += Z2_NT) A[i + (size_t)k * lda] /= piv;
    __syncthreads();
    for (int j = k + 1 + warp; j < n; j += Z2_WARPS) {
      double akj = A[k + (size_t)j * lda];
      if (akj != 0.0)
        for (int i = k + 1 + lane; i < n; i += 32) A[i + (size_t)j * lda] -= A[i + (size_t)k * lda] * akj;
    }
    __syncthreads();
  }
  // inverse: solve L U X = P^T I column by column into W, then copy back
  blk_identity(W, ldw, n);
  // apply row interchanges to the identity
  for (int c = threadIdx.x; c < n; c += Z2_NT)
    for (int k = 0; k < n; ++k) {
      int p = ipiv[k];
      if (p != k) {
        double t = W[k + (size_t)c * ldw];
        W[k + (size_t)c * ldw] = W[p + (size_t)c * ldw];
        W[p + (size_t)c * ldw] = t;
      }
    }
  __syncthreads();
  for (int c = warp; c < n; c += Z2_WARPS) {
    double *Wc = W + (size_t)c * ldw;
    // forward substitution with unit L
    for (int k = 0; k < n; ++k) {
      __syncwarp();
      double bk = Wc[k];
      if (bk != 0.0)
        for (int i = k + 1 + lane; i < n; i += 32) Wc[i] -= bk * A[i + (size_t)k * lda];
    }
    // back substitution with U
    for (int k = n - 1; k >= 0; --k) {
      __syncwarp();
      double bk = Wc[k];
      if (bk != 0.0) {
        bk = bk / A[k + (size_t)k * lda];
        __syncwarp();
        if (lane == 0) Wc[k] = bk;
        for (int i = lane; i < k; i += 32) Wc[i] -= bk * A[i + (size_t)k * lda];
      }
    }
  }
  __syncthreads();
  blk_copy(A, lda, W, ldw, n, n);
}
