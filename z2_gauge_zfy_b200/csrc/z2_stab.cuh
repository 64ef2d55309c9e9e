// z2_stab.cuh -- UDV stabilization (src/stabilization.f90:42-200) on the
// DMMA GEMM, the register-resident pivoted QR and the blocked DORGQR.
#pragma once
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
