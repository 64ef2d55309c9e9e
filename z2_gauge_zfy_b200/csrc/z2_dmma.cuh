// z2_dmma.cuh -- FP64 tensor-core (DMMA) GEMM and the thread-per-column
// Householder kernels used by the UDV stabilization.
//
// sm_100 has no FP64 kind of tcgen05.mma; its FP64 tensor path is the warp
// level mma.sync m8n8k4 .f64.  Fragment layout (PTX ISA, mma.m8n8k4 .f64):
//   A (8x4, row):  a0 = A[lane/4][lane%4]
//   B (4x8, col):  b0 = B[lane%4][lane/4]
//   C (8x8):       c{0,1} = C[lane/4][2*(lane%4) + {0,1}]
//
// Loops that read and write the same matrix are written in explicit batches
// (all loads of a batch, then the arithmetic, then the stores): the compiler
// cannot prove that a store does not alias the next element's load, so a
// plain loop pays one full shared-memory round trip per element.
#pragma once
#include "z2_linalg.cuh"

__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// A strided matrix view: element (i, j) at p[i * rs + j * cs].
struct MatRef {
  const double *p;
  int rs, cs;
};

// C (m x n, column-major ldc) = alpha * A (m x k) B (k x n) + beta * C.
// a_upper: A(i, l) reads as 0 for i > l; b_lower: B(l, j) reads as 0 for l < j
// (B = R^T of an upper-triangular R).  Operands may live in shared or global
// memory.  Each warp owns 16 x 16 groups of 8 x 8 DMMA tiles; interior groups
// run a pointer-increment loop without bounds checks.  beta == 0 never reads
// C.  Ends with the block synchronised.
__device__ __noinline__ void blk_dmma(int m, int n, int k, double alpha, MatRef A, bool a_upper,
                                     MatRef B, bool b_lower, double beta, double *C, int ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lr = lane >> 2, lc = lane & 3;
  const int gm = (m + 15) >> 4, gn = (n + 15) >> 4;
  const bool plain = !a_upper && !b_lower && (k & 3) == 0;
  for (int g = warp; g < gm * gn; g += Z2_WARPS) {
    const int r0 = (g % gm) << 4, c0 = (g / gm) << 4;
    double acc[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int ra0 = r0 + lr, ra1 = r0 + 8 + lr;
    const int cb0 = c0 + lr, cb1 = c0 + 8 + lr;
    const bool full = plain && (r0 + 16 <= m) && (c0 + 16 <= n);
    if (full) {
      const double *pa0 = A.p + (size_t)ra0 * A.rs + (size_t)lc * A.cs;
      const double *pa1 = pa0 + (size_t)8 * A.rs;
      const double *pb0 = B.p + (size_t)lc * B.rs + (size_t)cb0 * B.cs;
      const double *pb1 = pb0 + (size_t)8 * B.cs;
      const size_t sa = (size_t)4 * A.cs, sb = (size_t)4 * B.rs;
#pragma unroll 4
      for (int l0 = 0; l0 < k; l0 += 4) {
        const double a0 = *pa0, a1 = *pa1, b0 = *pb0, b1 = *pb1;
        pa0 += sa; pa1 += sa; pb0 += sb; pb1 += sb;
        dmma884(acc[0][0][0], acc[0][0][1], a0, b0);
        dmma884(acc[0][1][0], acc[0][1][1], a0, b1);
        dmma884(acc[1][0][0], acc[1][0][1], a1, b0);
        dmma884(acc[1][1][0], acc[1][1][1], a1, b1);
      }
    } else {
#pragma unroll 4
      for (int l0 = 0; l0 < k; l0 += 4) {
        const int l = l0 + lc;
        const bool lk = l < k;
        double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
        if (lk) {
          if (ra0 < m && !(a_upper && ra0 > l)) a0 = A.p[(size_t)ra0 * A.rs + (size_t)l * A.cs];
          if (ra1 < m && !(a_upper && ra1 > l)) a1 = A.p[(size_t)ra1 * A.rs + (size_t)l * A.cs];
          if (cb0 < n && !(b_lower && l < cb0)) b0 = B.p[(size_t)l * B.rs + (size_t)cb0 * B.cs];
          if (cb1 < n && !(b_lower && l < cb1)) b1 = B.p[(size_t)l * B.rs + (size_t)cb1 * B.cs];
        }
        dmma884(acc[0][0][0], acc[0][0][1], a0, b0);
        dmma884(acc[0][1][0], acc[0][1][1], a0, b1);
        dmma884(acc[1][0][0], acc[1][0][1], a1, b0);
        dmma884(acc[1][1][0], acc[1][1][1], a1, b1);
      }
    }
    // epilogue: all loads of C first, then the stores
    double *cp[2][2][2];
    bool ok[2][2][2];
    double old[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int row = r0 + 8 * a + lr, col = c0 + 8 * b + 2 * lc + e;
          ok[a][b][e] = row < m && col < n;
          cp[a][b][e] = C + row + (size_t)col * ldc;
          old[a][b][e] = (beta != 0.0 && ok[a][b][e]) ? *cp[a][b][e] : 0.0;
        }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (ok[a][b][e])
            *cp[a][b][e] = (beta == 0.0) ? alpha * acc[a][b][e]
                                         : alpha * acc[a][b][e] + beta * old[a][b][e];
  }
  __syncthreads();
}

// w = v^T x over rows [i0, n) (x, v column vectors of one matrix).
__device__ __forceinline__ double dot_col(const double *v, const double *x, int i0, int n) {
  double w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int i = i0;
  for (; i + 7 < n; i += 8) {
#pragma unroll
    for (int q = 0; q < 8; ++q) w[q] += v[i + q] * x[i + q];
  }
  for (; i < n; ++i) w[0] += v[i] * x[i];
  return ((w[0] + w[1]) + (w[2] + w[3])) + ((w[4] + w[5]) + (w[6] + w[7]));
}

// x(i0:n) -= t * v(i0:n), batched loads before stores.
__device__ __forceinline__ void axpy_col(double *x, const double *v, double t, int i0, int n) {
  int i = i0;
  for (; i + 7 < n; i += 8) {
    double a[8], b[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { a[q] = x[i + q]; b[q] = v[i + q]; }
#pragma unroll
    for (int q = 0; q < 8; ++q) x[i + q] = a[q] - b[q] * t;
  }
  for (; i < n; ++i) x[i] -= v[i] * t;
}

__device__ __forceinline__ double sumsq_col(const double *x, int i0, int n) {
  return dot_col(x, x, i0, n);
}

// Pivoted Householder QR, DGEQP3/DLAQP2 semantics (all columns free), with the
// trailing update and the norm downdate done one thread per column.
__device__ __noinline__ void blk_geqp3_tc(double *A, int lda, int n, int *jpvt, double *tau,
                                         double *vn1, double *vn2) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double tol3z = 1.0536712127723509e-08;   // sqrt(dlamch('E'))
  for (int j = threadIdx.x; j < n; j += Z2_NT) {
    const double nr = sqrt(sumsq_col(A + (size_t)j * lda, 0, n));
    vn1[j] = nr; vn2[j] = nr; jpvt[j] = j + 1;
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
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
      double s = 0.0;
      for (int i = j + 1 + lane; i < n; i += 32) { double a = Aj[i]; s += a * a; }
      s = warp_sum(s);
      const double alpha = Aj[j];
      double t = 0.0, beta = alpha;
      if (j < n - 1 && s != 0.0) {
        const double xnorm = sqrt(s);
        beta = -copysign(dlapy2(alpha, xnorm), alpha);
        t = (beta - alpha) / beta;
        const double sc = 1.0 / (alpha - beta);
        for (int i = j + 1 + lane; i < n; i += 32) Aj[i] *= sc;
      }
      __syncwarp();
      if (lane == 0) { tau[j] = t; Aj[j] = beta; }
    }
    __syncthreads();
    const double tj = tau[j];
    const double *v = A + (size_t)j * lda;
    for (int k = j + 1 + threadIdx.x; k < n; k += Z2_NT) {
      double *Ak = A + (size_t)k * lda;
      double akj = Ak[j];
      if (tj != 0.0) {
        const double tw = tj * (dot_col(v, Ak, j + 1, n) + akj);
        akj -= tw;
        Ak[j] = akj;
        axpy_col(Ak, v, tw, j + 1, n);
      }
      const double v1 = vn1[k];
      if (v1 != 0.0) {
        const double r = fabs(akj) / v1;
        const double temp = fmax(1.0 - r * r, 0.0);
        const double q = v1 / vn2[k];
        if (temp * q * q <= tol3z) {
          const double nv = (j < n - 1) ? sqrt(sumsq_col(Ak, j + 1, n)) : 0.0;
          vn1[k] = nv; vn2[k] = nv;
        } else {
          vn1[k] = v1 * sqrt(temp);
        }
      }
    }
    __syncthreads();
  }
}

// DORG2R (m x n, n reflectors) with one thread per trailing column.
__device__ __noinline__ void blk_org2r_tc(double *A, int lda, int m, int n, const double *tau) {
  for (int i = n - 1; i >= 0; --i) {
    const double ti = tau[i];
    const double *v = A + (size_t)i * lda;
    if (ti != 0.0) {
      for (int k = i + 1 + threadIdx.x; k < n; k += Z2_NT) {
        double *Ak = A + (size_t)k * lda;
        const double aki = Ak[i];
        const double tw = ti * (dot_col(v, Ak, i + 1, m) + aki);
        Ak[i] = aki - tw;
        axpy_col(Ak, v, tw, i + 1, m);
      }
    }
    __syncthreads();
    double *Ai = A + (size_t)i * lda;
    for (int r = threadIdx.x; r < m; r += Z2_NT) {
      if (r > i) Ai[r] *= -ti;
      else if (r == i) Ai[r] = 1.0 - ti;
      else Ai[r] = 0.0;
    }
    __syncthreads();
  }
}

// Solve R Z = Y in place (DTRSM 'L','U','N','N'), Y n x nc (ldy), R upper
// (ldr).  Blocks of 8 rows from the bottom: the 8 x 8 diagonal block is
// solved one thread per column (block of R held in registers), the rows
// above are updated by DMMA.
__device__ __noinline__ void blk_trsm_lun_blocked(const double *R, int ldr, int n, double *Y,
                                                  int ldy, int nc) {
  const int last = ((n - 1) / 8) * 8;
  for (int k0 = last; k0 >= 0; k0 -= 8) {
    const int kb = (n - k0) < 8 ? (n - k0) : 8;
    double rr[8][8];
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
      for (int q = 0; q < 8; ++q)
        rr[p][q] = (p <= q && q < kb) ? R[(k0 + p) + (size_t)(k0 + q) * ldr] : 0.0;
    for (int j = threadIdx.x; j < nc; j += Z2_NT) {
      double *Yj = Y + (size_t)j * ldy + k0;
      double y[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) y[q] = (q < kb) ? Yj[q] : 0.0;
#pragma unroll
      for (int q = 7; q >= 0; --q) {
        if (q < kb) {
          double z = y[q];
          if (z != 0.0) {
            z = z / rr[q][q];
            y[q] = z;
#pragma unroll
            for (int p = 0; p < 8; ++p)
              if (p < q) y[p] -= z * rr[p][q];
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) if (q < kb) Yj[q] = y[q];
    }
    __syncthreads();
    if (k0 > 0) {
      MatRef Ar{R + (size_t)k0 * ldr, 1, ldr};
      MatRef Br{Y + k0, 1, ldy};
      blk_dmma(k0, nc, kb, -1.0, Ar, false, Br, false, 1.0, Y, ldy);
    }
  }
}
