// z2_stab.cuh -- UDV stabilization (src/stabilization.f90:42-200) on the
// DMMA GEMM, the register-resident pivoted QR and the blocked DORGQR.
#pragma once
#include "z2_gj.cuh"
#include "z2_qrf.cuh"
#include "z2_qrp.cuh"

// stab_UR (left = false) / stab_UL (left = true), src/stabilization.f90:70-120.
// On entry A (lda; shared arena or global) holds the propagated U (UR, or
// UL^T).  U, D, V are the factors in global memory (U = UR or UL^T); W0 is an
// N x N global workspace.
__device__ __noinline__ void dev_stab_U(const Smem &s, int N, double *A, int lda, double *U,
                                        double *D, double *V, double *W0, bool left) {
  double *tau = s.vec, *vn1 = s.vec + N, *vn2 = s.vec + 2 * N, *Dn = s.vec + 3 * N;
  int *jpvt = s.ivec;
  blk_scale_cols(A, lda, N, N, D);                 // matUDV(:,i) *= D(i)
  blk_geqp3_fast(A, lda, N, jpvt, tau, vn1, vn2, s.tile, s.tile_doubles, s.red);   // ZGEQP3
  blk_qdrp_scale(A, lda, N, Dn, vn2);              // D = |R_ii|, R rows /= D
  for (int i = threadIdx.x; i < N; i += Z2_NT) D[i] = Dn[i];
  if (!left) {
    // VR <- R (P^T VR)     (ZLAPMR(.true.) + ZTRMM('L','U','N','N'))
    blk_perm_rows(W0, N, V, N, N, N, jpvt, true);
    blk_dmma(N, N, N, 1.0, MatRef{A, 1, lda}, true, MatRef{W0, 1, N}, false, 0.0, V, N);
  } else {
    // VL <- (VL P) R^T     (ZLAPMT(.true.) + ZTRMM('R','U','C','N'))
    blk_perm_cols(W0, N, V, N, N, N, jpvt, true);
    blk_dmma(N, N, N, 1.0, MatRef{W0, 1, N}, false, MatRef{A, lda, 1}, true, 0.0, V, N);
  }
  blk_orgqr(A, lda, N, tau, s.tile, s.tile_doubles, s.vec + 4 * N, 4 * N, W0);   // ZUNGQR (W0 free)
  blk_copy(U, N, A, lda, N, N);                    // UR = Q, or UL^T = Q
}

// stab_green (src/stabilization.f90:122-200): G = (I + UR DR VR VL DL UL)^-1
// into Gout (global, ld N).  The reference applies Q^H with ZUNMQR; here Q is
// formed (ZUNGQR) and applied by a DMMA GEMM, then D^-1, the triangular solve
// (DMMA-blocked) and the permutation follow in the reference's order.
// M (ldm) is the QR work matrix (shared arena when it fits); W1, W2, W3 are
// N x N global workspaces (W3 keeps the scaled R).
__device__ __noinline__ void dev_stab_green(const Smem &s, int N, int nt, int Ltrot,
                                            const double *UR, const double *DR,
                                            const double *VR, const double *ULT,
                                            const double *DL, const double *VL, double *M,
                                            int ldm, double *W1, double *W2, double *W3,
                                            double *Gout) {
  double *tau = s.vec, *vn1 = s.vec + N, *vn2 = s.vec + 2 * N, *Dn = s.vec + 3 * N;
  int *jpvt = s.ivec;
  // invULUR = UR^T UL^T -> M ; VRVL = VR VL -> W1
  blk_dmma(N, N, N, 1.0, MatRef{UR, N, 1}, false, MatRef{ULT, 1, N}, false, 0.0, M, ldm);
  blk_dmma(N, N, N, 1.0, MatRef{VR, 1, N}, false, MatRef{VL, 1, N}, false, 0.0, W1, N);
  // matUDV = invULUR + DR (VRVL DL)   (src/stabilization.f90:138-146)
  for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS) {
    const double dl = DL[j];
    for (int i = threadIdx.x & 31; i < N; i += 32) {
      const double t = W1[i + (size_t)j * N] * dl;
      const double u = DR[i] * t;
      M[i + (size_t)j * ldm] = M[i + (size_t)j * ldm] + u;
    }
  }
  __syncthreads();
  const int half = Ltrot / 2;
  if (nt > half) {   // matUDV = matUDV^dagger
    for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
      for (int i = threadIdx.x & 31; i < j; i += 32) {
        const double a = M[i + (size_t)j * ldm], b = M[j + (size_t)i * ldm];
        M[i + (size_t)j * ldm] = b;
        M[j + (size_t)i * ldm] = a;
      }
    __syncthreads();
  }
  blk_geqp3_fast(M, ldm, N, jpvt, tau, vn1, vn2, s.tile, s.tile_doubles, s.red);
  blk_qdrp_scale(M, ldm, N, Dn, vn2);   // vn2 keeps 1/D for the D^-1 scalings below
  // keep the scaled R (upper triangle) for the triangular solve
  for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i <= j; i += 32) W3[i + (size_t)j * N] = M[i + (size_t)j * ldm];
  __syncthreads();
  blk_orgqr(M, ldm, N, tau, s.tile, s.tile_doubles, s.vec + 4 * N, 4 * N, W1);   // Q in M (W1 free)
  if (nt < half + 1) {
    // G = UL^T P R^-1 D^-1 Q^T UR^T
    blk_dmma(N, N, N, 1.0, MatRef{M, ldm, 1}, false, MatRef{UR, N, 1}, false, 0.0, W2, N);
    // Y = D^-1 (Q^T UR^T) back into the arena (Q is no longer needed)
    for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
      for (int i = threadIdx.x & 31; i < N; i += 32)
        M[i + (size_t)j * ldm] = W2[i + (size_t)j * N] * vn2[i];
    __syncthreads();
    blk_trsm_lun_blocked(W3, N, N, M, ldm, N);     // R_s^-1 Y
    blk_perm_rows(W1, N, M, ldm, N, N, jpvt, false);   // ZLAPMR(.false.)
    blk_dmma(N, N, N, 1.0, MatRef{ULT, 1, N}, false, MatRef{W1, 1, N}, false, 0.0, Gout, N);
  } else {
    // G = UL^T Q D^-1 R^-T P^T UR^T, solved transposed: X^T = R_s^-1 D^-1 (UL^T Q)^T
    blk_dmma(N, N, N, 1.0, MatRef{ULT, 1, N}, false, MatRef{M, 1, ldm}, false, 0.0, W2, N);
    for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
      for (int i = threadIdx.x & 31; i < N; i += 32)
        M[i + (size_t)j * ldm] = W2[j + (size_t)i * N] * vn2[i];
    __syncthreads();
    blk_trsm_lun_blocked(W3, N, N, M, ldm, N);     // X^T
    blk_perm_rows(W1, N, M, ldm, N, N, jpvt, false);   // (X P^T)^T
    blk_dmma(N, N, N, 1.0, MatRef{W1, N, 1}, false, MatRef{UR, N, 1}, false, 0.0, Gout, N);
  }
}

// ---------------------------------------------------------------------------
// Pre-pivoted stabilization (the chain's default).  The reference factors with
// column-pivoted QR (ZGEQP3), a column step of which waits on the norm
// downdate and the arg-max of the previous one.  Here the columns are put in
// decreasing norm order once ("pre-pivoting", Bai, Lee, Li and Xu, Linear
// Algebra Appl. 435 (2011) 659) and factored by the blocked Householder QR
// without pivoting; the Green's function is formed from the scale-split
// middle matrix (Loh and Gubernatis; the same construction as QUEST's
// stabilized G):
//   M  = UR^T UL^T + DR (VR VL) DL
//      = DRb (DRb^-1 UR^T UL^T DLb^-1 + DRs VR VL DLs) DLb = DRb M' DLb,
//   DRb = max(DR, 1), DRs = min(DR, 1) (DLb, DLs likewise),
//   G  = UL^T M^-1 UR^T = UL^T DLb^-1 M'^-1 DRb^-1 UR^T,
// where M' has entries of order one.  M' is only inverted: for N <= 144 in
// registers by Gauss-Jordan elimination with partial pivoting, above that
// through the blocked Householder QR without pivoting (M' = Q' R').  U, D, V and G are the same as the reference's up to
// rounding (the UDV factors of a product are not unique: the column order of
// D may differ).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool qrf_ok(int n, int wd) { return n <= 256 && qrf_ncb(n, wd) > 0; }

__device__ __forceinline__ void geqrf_wp_any(double *A, int lda, int n, double *tau,
                                             double *Tsave, double *work, int wd) {
  const int ncb = qrf_ncb(n, wd);
  if (n <= 64) blk_geqrf_wp<2, 16>(A, lda, n, tau, Tsave, work, ncb);
  else if (n <= 128) blk_geqrf_wp<4, 16>(A, lda, n, tau, Tsave, work, ncb);
  else if (n <= 160) blk_geqrf_wp<5, 16>(A, lda, n, tau, Tsave, work, ncb);
  else blk_geqrf_wp<8, 8>(A, lda, n, tau, Tsave, work, ncb);
}

__device__ __forceinline__ void ormqr_wp_any(const double *A, int lda, int n, const double *Tsave,
                                             double *X, int ldx, int nc, double *work, int wd) {
  const int ncb = qrf_ncb(n, wd);
  if (qrf_pw(n) == 16) blk_ormqr_wp<16>(A, lda, n, Tsave, X, ldx, nc, work, ncb);
  else blk_ormqr_wp<8>(A, lda, n, Tsave, X, ldx, nc, work, ncb);
}

// stab_UR / stab_UL with the pre-pivoted QR; arguments as dev_stab_U.
__device__ __noinline__ void dev_stab_U_fast(const Smem &s, int N, double *A, int lda, double *U,
                                             double *D, double *V, double *W0, bool left) {
  const bool reg = N <= 144 && s.tile_doubles >= 2 * N;   // register-resident QR
  if (!reg && !qrf_ok(N, s.tile_doubles)) {
    dev_stab_U(s, N, A, lda, U, D, V, W0, left);
    return;
  }
  double *tau = s.vec, *nrm = s.vec + N, *Dn = s.vec + 2 * N, *rd = s.vec + 3 * N;
  int *jpvt = s.ivec;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  blk_scale_cols(A, lda, N, N, D);                 // matUDV(:,i) *= D(i)
  for (int j = warp; j < N; j += Z2_WARPS) {
    double ss = 0.0;
    for (int i = lane; i < N; i += 32) { const double a = A[i + (size_t)j * lda]; ss = fma(a, a, ss); }
    ss = warp_sum(ss);
    if (lane == 0) nrm[j] = (ss == ss) ? ss : -1.0;   // a NaN column sorts last
  }
  __syncthreads();
  // decreasing norm, ties in column order: a permutation for any input
  for (int j = threadIdx.x; j < N; j += Z2_NT) {
    const double x = nrm[j];
    int r = 0;
    for (int i = 0; i < N; ++i) {
      const double y = nrm[i];
      r += (y > x || (y == x && i < j)) ? 1 : 0;
    }
    jpvt[r] = j + 1;                               // 1-based, as ZGEQP3's jpvt
  }
  __syncthreads();
  if (reg) {
    qr_reg_any(A, lda, N, tau, s.tile, s.tile_doubles, s.red, jpvt);   // QR of A P
  } else {
    blk_copy(W0, N, A, lda, N, N);                 // A <- A P
    for (int j = warp; j < N; j += Z2_WARPS) {
      const double *src = W0 + (size_t)(jpvt[j] - 1) * N;
      for (int i = lane; i < N; i += 32) A[i + (size_t)j * lda] = src[i];
    }
    __syncthreads();
    geqrf_wp_any(A, lda, N, tau, nullptr, s.tile, s.tile_doubles);
  }
  blk_qdrp_scale(A, lda, N, Dn, rd);               // D = |R_ii|, R rows /= D
  for (int i = threadIdx.x; i < N; i += Z2_NT) D[i] = Dn[i];
  if (!left) {
    blk_perm_rows(W0, N, V, N, N, N, jpvt, true);  // VR <- R (P^T VR)
    blk_dmma(N, N, N, 1.0, MatRef{A, 1, lda}, true, MatRef{W0, 1, N}, false, 0.0, V, N);
  } else {
    blk_perm_cols(W0, N, V, N, N, N, jpvt, true);  // VL <- (VL P) R^T
    blk_dmma(N, N, N, 1.0, MatRef{W0, 1, N}, false, MatRef{A, lda, 1}, true, 0.0, V, N);
  }
  blk_orgqr(A, lda, N, tau, s.tile, s.tile_doubles, s.vec + 4 * N, 4 * N, W0);
  blk_copy(U, N, A, lda, N, N);
}

// stab_green with the scale-split middle matrix; arguments as dev_stab_green
// (W1 and W2 are N x N scratch; above N = 144, W3 keeps the T factors of the
// QR's panels and W2 the right-hand side).
__device__ __noinline__ void dev_stab_green_fast(const Smem &s, int N, int nt, int Ltrot,
                                                 const double *UR, const double *DR,
                                                 const double *VR, const double *ULT,
                                                 const double *DL, const double *VL, double *M,
                                                 int ldm, double *W1, double *W2, double *W3,
                                                 double *Gout) {
  const bool reg = N <= 144 && s.tile_doubles >= 4 * N;   // register-resident inverse
  if (!reg && !qrf_ok(N, s.tile_doubles)) {
    dev_stab_green(s, N, nt, Ltrot, UR, DR, VR, ULT, DL, VL, M, ldm, W1, W2, W3, Gout);
    return;
  }
  double *tau = s.vec, *rRb = s.vec + N, *rLb = s.vec + 2 * N, *Rs = s.vec + 3 * N,
         *Ls = s.vec + 4 * N;
  for (int i = threadIdx.x; i < N; i += Z2_NT) {
    rRb[i] = 1.0 / fmax(DR[i], 1.0);
    rLb[i] = 1.0 / fmax(DL[i], 1.0);
    Rs[i] = fmin(DR[i], 1.0);
    Ls[i] = fmin(DL[i], 1.0);
  }
  blk_dmma(N, N, N, 1.0, MatRef{UR, N, 1}, false, MatRef{ULT, 1, N}, false, 0.0, M, ldm);
  blk_dmma(N, N, N, 1.0, MatRef{VR, 1, N}, false, MatRef{VL, 1, N}, false, 0.0, W1, N);
  // M' = DRb^-1 (UR^T UL^T) DLb^-1 + DRs (VR VL) DLs
  blk_walk<8, double2>(
      N, N, [&](int i, int j) { return make_double2(M[i + (size_t)j * ldm], W1[i + (size_t)j * N]); },
      [&](double2 v, int i, int j) {
        const double a = v.x * rRb[i] * rLb[j];
        M[i + (size_t)j * ldm] = fma(Rs[i] * v.y, Ls[j], a);
      });
  __syncthreads();
  if (reg) {
    // M' is inverted in place in registers (Gauss-Jordan with partial
    // pivoting): on exit row j of M is DLb^-1(j) T(piv j, :) with
    // DLb^-1 M'^-1 = M P, P(m, k) = 1 iff piv[m] = k.  Then
    //   Y = P DRb^-1 UR^T,  Y(m, c) = DRb^-1(piv m) UR(c, piv m)  (in W2,
    //   column-major, so that the GEMM reads its k index contiguously),
    //   W1 = M Y,  G = UL^T W1.
    int *piv = s.ivec;
    gj_reg_any(M, ldm, N, piv, rLb, s.tile, s.tile_doubles, s.red);
    blk_walk<8, double>(
        N, N, [&](int c, int m) { return UR[c + (size_t)piv[m] * N]; },
        [&](double v, int c, int m) { W2[m + (size_t)c * N] = v * rRb[piv[m]]; });
    __syncthreads();
    blk_dmma(N, N, N, 1.0, MatRef{M, 1, ldm}, false, MatRef{W2, 1, N}, false, 0.0, W1, N);
    blk_dmma(N, N, N, 1.0, MatRef{ULT, 1, N}, false, MatRef{W1, 1, N}, false, 0.0, Gout, N);
    return;
  }
  // X = DRb^-1 UR^T
  for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < N; i += 32)
      W2[i + (size_t)j * N] = UR[j + (size_t)i * N] * rRb[i];
  __syncthreads();
  geqrf_wp_any(M, ldm, N, tau, W3, s.tile, s.tile_doubles);        // M' = Q' R'
  ormqr_wp_any(M, ldm, N, W3, W2, N, N, s.tile, s.tile_doubles);   // X <- Q'^T X
  blk_trsm_lun_blocked(M, ldm, N, W2, N, N);                       // X <- R'^-1 X
  for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < N; i += 32) W2[i + (size_t)j * N] *= rLb[i];
  __syncthreads();
  blk_dmma(N, N, N, 1.0, MatRef{ULT, 1, N}, false, MatRef{W2, 1, N}, false, 0.0, Gout, N);
}
