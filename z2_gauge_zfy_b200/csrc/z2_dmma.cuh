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
// (B = R^T of an upper-triangular R); a group's k loop then starts at its
// first row (a_upper) or column (b_lower), below which every term is zero.
// When an operand's k index is contiguous (B column-major, or A seen
// transposed), interior groups of a plain product take it as 16-byte loads
// covering two k steps (the k order within each group of 8 changes, not the
// terms).  Operands may live in shared or global memory.  Each warp owns 16 x 16
// groups of 8 x 8 DMMA tiles; interior groups run a pointer-increment loop
// without bounds checks.  beta == 0 never reads C.  Ends with the block
// synchronised.
__device__ __noinline__ void blk_dmma(int m, int n, int k, double alpha, MatRef A, bool a_upper,
                                     MatRef B, bool b_lower, double beta, double *C, int ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lr = lane >> 2, lc = lane & 3;
  const int gm = (m + 15) >> 4, gn = (n + 15) >> 4;
  const bool plain = !a_upper && !b_lower && (k & 3) == 0;
  // 16-byte operand loads: k contiguous, the matrix 16-byte aligned and its
  // other stride even (so every lane's pair starts on a 16-byte boundary)
  const bool va = A.cs == 1 && (A.rs & 1) == 0 && ((uintptr_t)A.p & 15) == 0;
  const bool vb = B.rs == 1 && (B.cs & 1) == 0 && ((uintptr_t)B.p & 15) == 0;
  const bool pair = (k & 7) == 0 && (va || vb);
  for (int g = warp; g < gm * gn; g += Z2_WARPS) {
    const int r0 = (g % gm) << 4, c0 = (g / gm) << 4;
    double acc[2][2][2];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    const int ra0 = r0 + lr, ra1 = r0 + 8 + lr;
    const int cb0 = c0 + lr, cb1 = c0 + 8 + lr;
    int lbeg = a_upper ? r0 : 0;   // a multiple of 16
    if (b_lower && c0 > lbeg) lbeg = c0;
    const bool full = (k & 3) == 0 && (r0 + 16 <= m) && (c0 + 16 <= n);
    if (full) {
      const double *pa0 = A.p + (size_t)ra0 * A.rs + (size_t)(lbeg + lc) * A.cs;
      const double *pa1 = pa0 + (size_t)8 * A.rs;
      const double *pb0 = B.p + (size_t)(lbeg + lc) * B.rs + (size_t)cb0 * B.cs;
      const double *pb1 = pb0 + (size_t)8 * B.cs;
      const size_t sa = (size_t)4 * A.cs, sb = (size_t)4 * B.rs;
      if (plain && pair) {
        // two k steps per pass over 8 k values: lane lc takes k = l0 + 2 lc in
        // the first and l0 + 2 lc + 1 in the second, so an operand whose k is
        // contiguous arrives as one 16-byte load for both
        const double *qa0 = A.p + (size_t)ra0 * A.rs + (size_t)(2 * lc) * A.cs;
        const double *qa1 = qa0 + (size_t)8 * A.rs;
        const double *qb0 = B.p + (size_t)(2 * lc) * B.rs + (size_t)cb0 * B.cs;
        const double *qb1 = qb0 + (size_t)8 * B.cs;
        const size_t ta = (size_t)8 * A.cs, tb = (size_t)8 * B.rs;
#pragma unroll 2
        for (int l0 = 0; l0 < k; l0 += 8) {
          double2 x0, x1, y0, y1;
          if (va) {
            x0 = *reinterpret_cast<const double2 *>(qa0);
            x1 = *reinterpret_cast<const double2 *>(qa1);
          } else {
            x0 = make_double2(qa0[0], qa0[A.cs]);
            x1 = make_double2(qa1[0], qa1[A.cs]);
          }
          if (vb) {
            y0 = *reinterpret_cast<const double2 *>(qb0);
            y1 = *reinterpret_cast<const double2 *>(qb1);
          } else {
            y0 = make_double2(qb0[0], qb0[B.rs]);
            y1 = make_double2(qb1[0], qb1[B.rs]);
          }
          qa0 += ta; qa1 += ta; qb0 += tb; qb1 += tb;
          dmma884(acc[0][0][0], acc[0][0][1], x0.x, y0.x);
          dmma884(acc[0][1][0], acc[0][1][1], x0.x, y1.x);
          dmma884(acc[1][0][0], acc[1][0][1], x1.x, y0.x);
          dmma884(acc[1][1][0], acc[1][1][1], x1.x, y1.x);
          dmma884(acc[0][0][0], acc[0][0][1], x0.y, y0.y);
          dmma884(acc[0][1][0], acc[0][1][1], x0.y, y1.y);
          dmma884(acc[1][0][0], acc[1][0][1], x1.y, y0.y);
          dmma884(acc[1][1][0], acc[1][1][1], x1.y, y1.y);
        }
      } else if (plain) {
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
        // triangular operand: the same loop with the masked entries zeroed
        // (no bounds checks inside a full tile)
#pragma unroll 4
        for (int l0 = lbeg; l0 < k; l0 += 4) {
          const int l = l0 + lc;
          double a0 = *pa0, a1 = *pa1, b0 = *pb0, b1 = *pb1;
          pa0 += sa; pa1 += sa; pb0 += sb; pb1 += sb;
          if (a_upper) { if (ra0 > l) a0 = 0.0; if (ra1 > l) a1 = 0.0; }
          if (b_lower) { if (l < cb0) b0 = 0.0; if (l < cb1) b1 = 0.0; }
          dmma884(acc[0][0][0], acc[0][0][1], a0, b0);
          dmma884(acc[0][1][0], acc[0][1][1], a0, b1);
          dmma884(acc[1][0][0], acc[1][0][1], a1, b0);
          dmma884(acc[1][1][0], acc[1][1][1], a1, b1);
        }
      }
    } else {
#pragma unroll 4
      for (int l0 = lbeg; l0 < k; l0 += 4) {
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

// T of one block of reflectors (DLARFT forward / columnwise), by one warp:
// T is the inverse of the upper-triangular matrix with diagonal 1/tau and
// strict upper part S = V^T V (DLARFT's column recurrence is exactly the
// forward substitution of that inverse); diagonal blocks of size b pair up
// as T12 = -T11 S12 T22, four levels of short dot products instead of 16
// dependent columns.  A zero tau zeroes its row and column, as in DLARFT.
// S, T: ib x ib (ld ib); tb: the block's tau; Xs: 4 ib doubles of scratch.
__device__ __forceinline__ void warp_larft_t(const double *S, double *T, int ib, const double *tb,
                                             double *Xs) {
  const int lane = threadIdx.x & 31;
  for (int e = lane; e < ib * ib; e += 32) {
    const int r = e % ib, c = e / ib;
    T[e] = (r == c) ? tb[c] : 0.0;
  }
  __syncwarp();
  for (int b = 1; b < ib; b <<= 1) {
    const int np = (ib + 2 * b - 1) / (2 * b), bb = b * b;
    for (int e = lane; e < np * bb; e += 32) {
      const int p = e / bb, r = (e % bb) % b, c = (e % bb) / b;
      const int k = 2 * b * p, k2 = k + b;
      if (k2 + c < ib) {
        double x0 = 0.0, x1 = 0.0;
        for (int q = 0; q <= c; q += 2) {
          x0 += S[(k + r) + (k2 + q) * ib] * T[(k2 + q) + (k2 + c) * ib];
          if (q + 1 <= c) x1 += S[(k + r) + (k2 + q + 1) * ib] * T[(k2 + q + 1) + (k2 + c) * ib];
        }
        Xs[e] = x0 + x1;
      }
    }
    __syncwarp();
    for (int e = lane; e < np * bb; e += 32) {
      const int p = e / bb, r = (e % bb) % b, c = (e % bb) / b;
      const int k = 2 * b * p, k2 = k + b;
      if (k2 + c < ib) {
        double t0 = 0.0, t1 = 0.0;
        for (int q = r; q < b; q += 2) {
          t0 += T[(k + r) + (k + q) * ib] * Xs[p * bb + q + c * b];
          if (q + 1 < b) t1 += T[(k + r) + (k + q + 1) * ib] * Xs[p * bb + q + 1 + c * b];
        }
        T[(k + r) + (k2 + c) * ib] = -(t0 + t1);
      }
    }
    __syncwarp();
  }
}

// S = V^T V (ib x ib, ld ib, ib <= 16) for the unit lower trapezoidal V of
// the reflectors stored in A(i0:n, i0:i0+ib), by one warp: one 16 x 16 DMMA
// group over k = n - i0, the operand read from A with the unit diagonal and
// zero upper part applied (the same k order and values as blk_dmma on a
// copy of V, so the same bits).
__device__ __forceinline__ void warp_gram_v(const double *A, int lda, int n, int i0, int ib, double *S) {
  const int lane = threadIdx.x & 31, lr = lane >> 2, lc = lane & 3;
  const int mp = n - i0;
  auto vat = [&](int l, int c) -> double {
    if (l >= mp || c >= ib) return 0.0;
    return (l == c) ? 1.0 : (l > c ? A[(i0 + l) + (size_t)(i0 + c) * lda] : 0.0);
  };
  double acc[2][2][2] = {};
  for (int l0 = 0; l0 < mp; l0 += 4) {
    const double f0 = vat(l0 + lc, lr), f1 = vat(l0 + lc, 8 + lr);
    dmma884(acc[0][0][0], acc[0][0][1], f0, f0);
    dmma884(acc[0][1][0], acc[0][1][1], f0, f1);
    dmma884(acc[1][0][0], acc[1][0][1], f1, f0);
    dmma884(acc[1][1][0], acc[1][1][1], f1, f1);
  }
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = 8 * u + lr, c = 8 * v + 2 * lc + e;
        if (r < ib && c < ib) S[r + c * ib] = 1.0 * acc[u][v][e];
      }
}

// DORGQR for a square n x n matrix with n reflectors, blocked: blocks of nb
// reflectors from the last to the first, each applied as the compact WY form
// H_i0 ... H_i0+ib-1 = I - V T V^T (DLARFT forward/columnwise) by DMMA GEMMs:
//   trailing columns  C <- C - V (T (V^T C)),
//   block columns     A(i0:, i0:i0+ib) = E - V (T V1^T),  rows above = 0.
// work (shared memory, wd doubles) holds V (ldv x nb, ldv = 4 mod 16 so both
// DMMA fragment orientations are bank-conflict free) and W (ldw x (n - nb),
// ldw odd for the thread-per-column T W product); T and the Gram matrix
// (nb x nb each) go to small (sd doubles) when it is large enough, else to
// work.  When work is too small the unblocked DORG2R runs instead (same Q up
// to rounding).
__device__ __noinline__ void blk_orgqr(double *A, int lda, int n, const double *tau, double *work,
                                      int wd, double *small, int sd, double *tscr = nullptr) {
  const int ldv = ((n + 11) & ~15) + 4;
  int nb = 16;
  auto need = [n, ldv, sd](int b) {
    return ldv * b + (b + 1) * (n > b ? n - b : 0) + (2 * b * b <= sd ? 0 : 2 * b * b);
  };
  if (need(nb) > wd) nb = 8;
  if (need(nb) > wd) {
    blk_org2r_tc(A, lda, n, n, tau);
    return;
  }
  const int ldw = nb + 1;
  double *V = work;
  double *W = V + (size_t)ldv * nb;
  double *T = (2 * nb * nb <= sd) ? small : W + (size_t)ldw * (n > nb ? n - nb : 0);
  double *S = T + nb * nb;
  const int tid = threadIdx.x;
  // Prologue (tscr: nb^2 ceil(n / nb) doubles of global scratch): the T of
  // every block depends only on that block's reflectors, which the backward
  // loop below does not touch before the block's turn, so all of them are
  // formed first, one warp per block in parallel, instead of one after the
  // other inside the loop.
  if (tscr != nullptr && wd < Z2_WARPS * (2 * nb * nb + 4 * nb)) tscr = nullptr;
  if (tscr != nullptr) {
    const int nblk = (n + nb - 1) / nb, warp = tid >> 5;
    double *Sw = work + (size_t)warp * (2 * nb * nb + 4 * nb);
    double *Tw = Sw + nb * nb, *Xw = Tw + nb * nb;
    for (int bi = warp; bi < nblk; bi += Z2_WARPS) {
      const int i0 = bi * nb, ib = (n - i0) < nb ? (n - i0) : nb;
      warp_gram_v(A, lda, n, i0, ib, Sw);
      __syncwarp();
      warp_larft_t(Sw, Tw, ib, tau + i0, Xw);
      __syncwarp();
      double *td = tscr + (size_t)bi * nb * nb;
      for (int e = tid & 31; e < ib * ib; e += 32) td[e] = Tw[e];
      __syncwarp();
    }
    __syncthreads();
  }
  for (int i0 = ((n - 1) / nb) * nb; i0 >= 0; i0 -= nb) {
    const int ib = (n - i0) < nb ? (n - i0) : nb;
    const int mp = n - i0, nc = n - i0 - ib;
    // V: unit lower trapezoidal, mp x ib
    for (int c = tid >> 5; c < ib; c += Z2_WARPS)
      for (int r = tid & 31; r < mp; r += 32)
        V[r + (size_t)c * ldv] = (r == c) ? 1.0 : (r > c ? A[(i0 + r) + (size_t)(i0 + c) * lda] : 0.0);
    __syncthreads();
    // S = V^T V (the prologue already folded it into T)
    if (tscr == nullptr)
      blk_dmma(ib, ib, mp, 1.0, MatRef{V, ldv, 1}, false, MatRef{V, 1, ldv}, false, 0.0, S, ib);
    // T (DLARFT): from the prologue when it ran, else by one warp here
    if (tscr != nullptr) {
      const double *tsrc = tscr + (size_t)(i0 / nb) * nb * nb;
      for (int e = tid; e < ib * ib; e += Z2_NT) T[e] = tsrc[e];
    } else if (ldw * (n - nb) >= 4 * nb) {
      if (tid < 32) warp_larft_t(S, T, ib, tau + i0, W);
    } else if (tid < ib) {
      const int r = tid;
      double tr[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        double t = 0.0;
        if (c < ib) {
          if (c == r) {
            t = tau[i0 + c];
          } else if (c > r) {
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int q = 0; q < c; ++q) {
              if (q >= r) {
                if (q & 1) a1 += tr[q] * S[q + c * ib];
                else a0 += tr[q] * S[q + c * ib];
              }
            }
            t = -tau[i0 + c] * (a0 + a1);
          }
        }
        tr[c] = t;
      }
#pragma unroll
      for (int c = 0; c < 16; ++c)
        if (c < ib) T[r + c * ib] = tr[c];
    }
    __syncthreads();
    if (nc > 0) {
      double *C = A + i0 + (size_t)(i0 + ib) * lda;
      // W = V^T C  (ib x nc, ld ldw)
      blk_dmma(ib, nc, mp, 1.0, MatRef{V, ldv, 1}, false, MatRef{C, 1, lda}, false, 0.0, W, ldw);
      // W <- T W, one thread per column
      for (int j = tid; j < nc; j += Z2_NT) {
        double w[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) w[q] = (q < ib) ? W[q + j * ldw] : 0.0;
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          if (r < ib) {
            double t = 0.0;
#pragma unroll
            for (int q = r; q < 16; ++q)
              if (q < ib) t += T[r + q * ib] * w[q];
            W[r + j * ldw] = t;
          }
        }
      }
      __syncthreads();
      // C -= V W
      blk_dmma(mp, nc, ib, -1.0, MatRef{V, 1, ldv}, false, MatRef{W, 1, ldw}, false, 1.0, C, lda);
    }
    // S <- T V1^T (ib x ib); block columns <- E - V S, rows above i0 <- 0
    for (int e = tid; e < ib * ib; e += Z2_NT) {
      const int r = e % ib, c = e / ib;
      double t = 0.0;
      for (int q = r; q <= c; ++q) t += T[r + q * ib] * V[c + (size_t)q * ldv];
      S[r + c * ib] = t;
    }
    for (int c = tid >> 5; c < ib; c += Z2_WARPS)
      for (int r = tid & 31; r < n; r += 32) A[r + (size_t)(i0 + c) * lda] = (r == i0 + c) ? 1.0 : 0.0;
    __syncthreads();
    blk_dmma(mp, ib, ib, -1.0, MatRef{V, 1, ldv}, false, MatRef{S, 1, ib}, false, 1.0,
             A + i0 + (size_t)i0 * lda, lda);
  }
}

// Householder QR without pivoting of a square n x n matrix, blocked (DGEQRF
// structure): panels of nb columns are factored column by column (DLARFG on
// the column, the reflector applied to the rest of the panel one warp per
// column), then the panel's reflectors reach the trailing columns as
// C <- (I - V T^T V^T) C = C - V (T^T (V^T C)) by DMMA GEMMs (T by DLARFT's
// recurrence, as in blk_orgqr).  Same R, tau and reflectors as DGEQR2 up to
// rounding.  Workspace as blk_orgqr; falls back to blk_geqr2 when short.
__device__ __noinline__ void blk_geqrf(double *A, int lda, int n, double *tau, double *work, int wd,
                                      double *small, int sd, double *red) {
  const int ldv = ((n + 11) & ~15) + 4;
  int nb = 16;
  auto need = [n, ldv, sd](int b) {
    return ldv * b + (b + 1) * (n > b ? n - b : 0) + (2 * b * b <= sd ? 0 : 2 * b * b);
  };
  if (need(nb) > wd) nb = 8;
  if (need(nb) > wd) {
    blk_geqr2(A, lda, n, n, tau);
    return;
  }
  const int ldw = nb + 1;
  double *V = work;
  double *W = V + (size_t)ldv * nb;
  double *T = (2 * nb * nb <= sd) ? small : W + (size_t)ldw * (n > nb ? n - nb : 0);
  double *S = T + nb * nb;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j0 = 0; j0 < n; j0 += nb) {
    const int ib = (n - j0) < nb ? (n - j0) : nb;
    const int mp = n - j0, nc = n - j0 - ib;
    // ---- panel (DGEQR2 on columns j0 .. j0+ib-1) ----
    for (int k = 0; k < ib; ++k) {
      const int j = j0 + k;
      double *Aj = A + (size_t)j * lda;
      double ss = 0.0;
      for (int r = j + 1 + tid; r < n; r += Z2_NT) { const double a = Aj[r]; ss += a * a; }
      ss = blk_sum(ss, red);
      const double alpha = Aj[j];
      double t = 0.0, beta = alpha, sc = 1.0;
      if (j < n - 1 && ss != 0.0) {
        const double xnorm = sqrt(ss);
        beta = -copysign(dlapy2(alpha, xnorm), alpha);
        t = (beta - alpha) / beta;
        sc = 1.0 / (alpha - beta);
      }
      if (t != 0.0)
        for (int r = j + 1 + tid; r < n; r += Z2_NT) Aj[r] *= sc;
      __syncthreads();
      // H_j on the remaining panel columns, one warp per column (v_j = 1)
      if (t != 0.0) {
        for (int c = j + 1 + warp; c < j0 + ib; c += Z2_WARPS) {
          double *Ac = A + (size_t)c * lda;
          const double acj = Ac[j];
          double w = 0.0;
          for (int r = j + 1 + lane; r < n; r += 32) w += Aj[r] * Ac[r];
          w = (warp_sum(w) + acj) * t;
          __syncwarp();
          if (lane == 0) Ac[j] = acj - w;
          for (int r = j + 1 + lane; r < n; r += 32) Ac[r] -= w * Aj[r];
        }
      }
      __syncthreads();
      if (tid == 0) { tau[j] = t; Aj[j] = beta; }
      __syncthreads();
    }
    if (nc <= 0) continue;
    // ---- V (unit lower), S = V^T V, T (DLARFT) ----
    for (int c = tid >> 5; c < ib; c += Z2_WARPS)
      for (int r = tid & 31; r < mp; r += 32)
        V[r + (size_t)c * ldv] = (r == c) ? 1.0 : (r > c ? A[(j0 + r) + (size_t)(j0 + c) * lda] : 0.0);
    __syncthreads();
    blk_dmma(ib, ib, mp, 1.0, MatRef{V, ldv, 1}, false, MatRef{V, 1, ldv}, false, 0.0, S, ib);
    if (tid < ib) {
      const int r = tid;
      double tr[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        double t = 0.0;
        if (c < ib) {
          if (c == r) {
            t = tau[j0 + c];
          } else if (c > r) {
            double a0 = 0.0, a1 = 0.0;
#pragma unroll
            for (int q = 0; q < c; ++q) {
              if (q >= r) {
                if (q & 1) a1 += tr[q] * S[q + c * ib];
                else a0 += tr[q] * S[q + c * ib];
              }
            }
            t = -tau[j0 + c] * (a0 + a1);
          }
        }
        tr[c] = t;
      }
#pragma unroll
      for (int c = 0; c < 16; ++c)
        if (c < ib) T[r + c * ib] = tr[c];
    }
    __syncthreads();
    // ---- trailing columns: C -= V (T^T (V^T C)) ----
    double *C = A + j0 + (size_t)(j0 + ib) * lda;
    blk_dmma(ib, nc, mp, 1.0, MatRef{V, ldv, 1}, false, MatRef{C, 1, lda}, false, 0.0, W, ldw);
    for (int c = tid; c < nc; c += Z2_NT) {
      double w[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) w[q] = (q < ib) ? W[q + c * ldw] : 0.0;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        if (r < ib) {
          double t = 0.0;
#pragma unroll
          for (int q = 0; q <= r; ++q) t += T[q + r * ib] * w[q];   // (T^T w)_r
          W[r + c * ldw] = t;
        }
      }
    }
    __syncthreads();
    blk_dmma(mp, nc, ib, -1.0, MatRef{V, 1, ldv}, false, MatRef{W, 1, ldw}, false, 1.0, C, lda);
  }
}

// Solve L Z = Y in place, L unit lower triangular (below the diagonal of L),
// Y n x nc: blocks of 8 rows from the top, the 8 x 8 diagonal block solved one
// thread per column in registers, the rows below updated by DMMA.
__device__ __noinline__ void blk_trsm_lln_blocked(const double *L, int ldl, int n, double *Y,
                                                  int ldy, int nc) {
  for (int k0 = 0; k0 < n; k0 += 8) {
    const int kb = (n - k0) < 8 ? (n - k0) : 8;
    double ll[8][8];
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
      for (int q = 0; q < 8; ++q)
        ll[p][q] = (p > q && p < kb) ? L[(k0 + p) + (size_t)(k0 + q) * ldl] : 0.0;
    for (int j = threadIdx.x; j < nc; j += Z2_NT) {
      double *Yj = Y + (size_t)j * ldy + k0;
      double y[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) y[q] = (q < kb) ? Yj[q] : 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double z = y[q];
#pragma unroll
        for (int p = 0; p < 8; ++p)
          if (p > q) y[p] -= z * ll[p][q];
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) if (q < kb) Yj[q] = y[q];
    }
    __syncthreads();
    if (k0 + kb < n) {
      blk_dmma(n - k0 - kb, nc, kb, -1.0, MatRef{L + (k0 + kb) + (size_t)k0 * ldl, 1, ldl}, false,
               MatRef{Y + k0, 1, ldy}, false, 1.0, Y + k0 + kb, ldy);
    }
  }
}

__device__ __noinline__ void blk_trsm_lun_blocked(const double *R, int ldr, int n, double *Y,
                                                  int ldy, int nc);

// Inverse of a general n x n matrix by LU with partial pivoting (the
// ZGEFA/ZGEDI pair of INV_C, lib/package_of_matrix/Modules/mat_mod.f90:296-336),
// blocked: panels of 16 columns (pivot search over the column, full-row
// interchanges, in-panel rank-1 updates one warp per column), U12 = L11^-1 A12
// one thread per column (L11 staged in work), A22 -= L21 U12 by DMMA; then
// A^-1 = U^-1 L^-1 P from the identity by the two blocked triangular solves.
// A is overwritten by its inverse; W (ldw) is an n x n workspace; work holds
// >= 256 doubles of shared memory (else the unblocked blk_inverse runs).
__device__ __noinline__ void blk_inverse_blocked(double *A, int lda, int n, double *W, int ldw,
                                                 int *ipiv, double *red, int *flag, double *work,
                                                 int wd) {
  if (work == nullptr || wd < 256) {
    blk_inverse(A, lda, n, W, ldw, ipiv, red, flag);
    return;
  }
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j0 = 0; j0 < n; j0 += 16) {
    const int jb = (n - j0) < 16 ? (n - j0) : 16;
    for (int k = j0; k < j0 + jb; ++k) {
      double bv = -1.0; int bi = n;
      for (int i = k + tid; i < n; i += Z2_NT) {
        const double v = fabs(A[i + (size_t)k * lda]);
        if (v > bv) { bv = v; bi = i; }
      }
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_xor_sync(Z2_FULL, bv, o);
        const int oi = __shfl_xor_sync(Z2_FULL, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (lane == 0) { red[warp] = bv; flag[warp] = bi; }
      __syncthreads();
      bv = red[0]; bi = flag[0];
      for (int w = 1; w < Z2_WARPS; ++w)
        if (red[w] > bv || (red[w] == bv && flag[w] < bi)) { bv = red[w]; bi = flag[w]; }
      const int p = bi;
      __syncthreads();
      if (tid == 0) ipiv[k] = p;
      if (p != k)
        for (int j = tid; j < n; j += Z2_NT) {
          const double t = A[k + (size_t)j * lda];
          A[k + (size_t)j * lda] = A[p + (size_t)j * lda];
          A[p + (size_t)j * lda] = t;
        }
      __syncthreads();
      const double piv = A[k + (size_t)k * lda];
      for (int i = k + 1 + tid; i < n; i += Z2_NT) A[i + (size_t)k * lda] /= piv;
      __syncthreads();
      for (int j = k + 1 + warp; j < j0 + jb; j += Z2_WARPS) {
        const double akj = A[k + (size_t)j * lda];
        if (akj != 0.0)
          for (int i = k + 1 + lane; i < n; i += 32) A[i + (size_t)j * lda] -= A[i + (size_t)k * lda] * akj;
      }
      __syncthreads();
    }
    const int nc = n - j0 - jb;
    if (nc <= 0) continue;
    // U12 = L11^-1 A12 (L11 unit lower, staged in shared memory)
    for (int e = tid; e < jb * jb; e += Z2_NT) {
      const int p = e % jb, q = e / jb;
      work[p + 16 * q] = (p > q) ? A[(j0 + p) + (size_t)(j0 + q) * lda] : 0.0;
    }
    __syncthreads();
    for (int c = tid; c < nc; c += Z2_NT) {
      double *Ac = A + j0 + (size_t)(j0 + jb + c) * lda;
      double y[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) y[q] = (q < jb) ? Ac[q] : 0.0;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const double z = y[q];
#pragma unroll
        for (int p = 0; p < 16; ++p)
          if (p > q) y[p] -= z * work[p + 16 * q];
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) if (q < jb) Ac[q] = y[q];
    }
    __syncthreads();
    // A22 -= L21 U12
    blk_dmma(n - j0 - jb, nc, jb, -1.0, MatRef{A + (j0 + jb) + (size_t)j0 * lda, 1, lda}, false,
             MatRef{A + j0 + (size_t)(j0 + jb) * lda, 1, lda}, false, 1.0,
             A + (j0 + jb) + (size_t)(j0 + jb) * lda, lda);
  }
  // W = P I (row interchanges of the factorization, in order)
  blk_identity(W, ldw, n);
  for (int c = tid; c < n; c += Z2_NT)
    for (int k = 0; k < n; ++k) {
      const int p = ipiv[k];
      if (p != k) {
        const double t = W[k + (size_t)c * ldw];
        W[k + (size_t)c * ldw] = W[p + (size_t)c * ldw];
        W[p + (size_t)c * ldw] = t;
      }
    }
  __syncthreads();
  blk_trsm_lln_blocked(A, lda, n, W, ldw, n);   // L^-1 P
  blk_trsm_lun_blocked(A, lda, n, W, ldw, n);   // U^-1 L^-1 P
  blk_copy(A, lda, W, ldw, n, n);
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
    // reciprocals of the diagonal: one division per entry instead of one per
    // entry and right-hand side, off the columns' dependent chains
    double rd[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) rd[q] = (q < kb) ? 1.0 / rr[q][q] : 0.0;
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
            z = z * rd[q];
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
