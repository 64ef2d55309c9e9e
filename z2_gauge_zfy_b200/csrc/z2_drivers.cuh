// z2_drivers.cuh -- slice, half-sweep, bin, time-displaced and adjoint
// drivers of one chain (src/local_sweep.f90, src/dynamics.f90).
#pragma once
#include "z2_chain.cuh"

// Wrap_tau (src/stabilization.f90:478-514) on the Dyn copy of the propagator.
__device__ __noinline__ void wrap_tau(const ChainDesc &c, const Smem &s, int nt, Pend &pd) {
  const int N = c.N, NN = N * N, n2 = 2 * N;
  int lda; double *A = qr_matrix(c, s, lda);
  const int st = nt / c.Nwrap;
  blk_copy(c.ULTd, N, c.ULTs + (size_t)st * NN, N, N, N);
  blk_copy(c.VLd, N, c.VLs + (size_t)st * NN, N, N, N);
  copy_vec(c.DLd, c.DLs + (size_t)st * N, N);
  blk_copy(A, lda, c.URd, N, N, N);
  apply_pending_R(c, s, A, lda, pd.lo, pd.hi, c.use_kin != 0);
  pd.lo = 1; pd.hi = 0;
  dev_stab_U(s, N, A, lda, c.URd, c.DRd, c.VRd, c.W0, false);
  dev_stab_green_big(s, N, c.URd, c.DRd, c.VRd, c.ULTd, c.DLd, c.VLd, c.W0, c.W1, c.W2, c.W3,
                     c.B0, c.B1, c.B2, c.B3);
  const double *T = c.B3;
  double d0 = blk_maxdiff(T + (size_t)N * n2, n2, c.G0t, N, N, s.red);
  double d1 = blk_maxdiff(T + N, n2, c.Gt0, N, N, s.red);
  double d2 = blk_maxdiff(T + N + (size_t)N * n2, n2, c.Gtt, N, N, s.red);
  if (threadIdx.x == 0) {
    double d[3] = {d0, d1, d2};
    for (int q = 0; q < 3; ++q) {
      if (d[q] > c.acc[A_TXMAX0 + q] || d[q] != d[q]) c.acc[A_TXMAX0 + q] = d[q];
      c.acc[A_TXMEAN0 + q] += d[q];
      if (!(d[q] == d[q]) || isinf(d[q])) atomicOr(c.status, ST_NONFINITE);
    }
  }
  green_big_extract(N, T, c.G00, c.G0t, c.Gt0, c.Gtt);
}

// Dyn_reset + Dyn_sweep_R (src/dynamics.f90:41-62): the G(tau,0) chain.
// The arena is free here (G is spilled in c.G).
__device__ __noinline__ void dyn_sweep(const ChainDesc &c, const Smem &s) {
  const int N = c.N;
  blk_copy(c.URd, N, c.UR, N, N, N);
  blk_copy(c.VRd, N, c.VR, N, N, N);
  copy_vec(c.DRd, c.DR, N);
  blk_copy(c.ULTd, N, c.ULT, N, N, N);
  blk_copy(c.VLd, N, c.VL, N, N, N);
  copy_vec(c.DLd, c.DL, N);
  // Propgr_reset (src/process_matrix.f90:88-96)
  for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < N; i += 32) {
      double g = c.G[i + (size_t)j * N];
      c.G00[i + (size_t)j * N] = g;
      c.Gtt[i + (size_t)j * N] = g;
      c.Gt0[i + (size_t)j * N] = g;
      c.G0t[i + (size_t)j * N] = -((i == j ? 1.0 : 0.0) - g);
    }
  __syncthreads();
  Pend pd{1, 0};
  for (int nt = 1; nt <= c.Ltrot; ++nt) {
    obs_tau(c, s, nt);
    if (c.use_kin) {      // propgrK_R (src/multiply.f90:43-63)
      build_table(c, s, nt);
      kin_global(c, s, c.Gt0, 1, 0);
      kin_global(c, s, c.G0t, 0, -1);
      kin_global(c, s, c.Gtt, 1, -1);
    }
    if (c.eP != 1.0 || c.eM != 1.0) {   // propgrT_R (src/multiply.f90:110-130)
      blk_scale(c.Gt0, N, N, N, c.eP);
      blk_scale(c.G0t, N, N, N, c.eM);
      blk_scale(c.Gtt, N, N, N, c.eP);
      blk_scale(c.Gtt, N, N, N, c.eM);
    }
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.hi = nt;
    if (nt % c.Nwrap == 0) wrap_tau(c, s, nt, pd);
  }
}

// Local_sweep_pre (src/local_sweep.f90:87-104)
__device__ __noinline__ void chain_pre(const ChainDesc &c, const Smem &s) {
  const int N = c.N;
  blk_identity(c.UR, N, N); blk_identity(c.VR, N, N); blk_fill(c.DR, N, 1.0);
  blk_identity(c.ULT, N, N); blk_identity(c.VL, N, N); blk_fill(c.DL, N, 1.0);
  blk_identity(c.G, N, N);
  Pend pd{1, 0};
  wrap_pre(c, s, 0, pd);
  for (int nt = 1; nt <= c.Ltrot; ++nt) {
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.hi = nt;
    if (nt % c.Nwrap == 0) wrap_pre(c, s, nt, pd);
  }
}

__device__ __noinline__ void scale_G_mu(const ChainDesc &c, const Smem &s) {
  if (c.eP != 1.0 || c.eM != 1.0) {
    blk_scale(s.G, s.ldg, c.N, c.N, c.eP);
    blk_scale(s.G, s.ldg, c.N, c.N, c.eM);
  }
}

// Local_sweep_L (src/local_sweep.f90:106-124)
__device__ __noinline__ void sweep_L(const ChainDesc &c, const Smem &s) {
  const int N = c.N;
  Pend pd{1, 0};
  for (int nt = c.Ltrot; nt >= 1; --nt) {
    if (nt % c.Nwrap == 0) { PhTimer t(c, PH_WRAP); wrap_L(c, s, nt, pd, true); }
    { PhTimer t(c, PH_OBS); obs_equal(c, s, nt); }
    scale_G_mu(c, s);                               // propT_L
    { PhTimer t(c, PH_PROP); propose_slice(c, s, nt, true, 0); }   // bonds 2N..1
    {
      PhTimer t(c, PH_KIN);
      build_table(c, s, nt);
      kin_cols(c, s, s.G, s.ldg, N, 1);             // G B
      kin_rows(c, s, s.G, s.ldg, N, -1);            // B^-1 G
    }
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.lo = nt;
  }
  { PhTimer t(c, PH_WRAP); wrap_L(c, s, 0, pd, true); }
}

// Local_sweep_R (src/local_sweep.f90:126-150)
__device__ __noinline__ void sweep_R(const ChainDesc &c, const Smem &s, bool toggle) {
  const int N = c.N;
  if (toggle) {
    { PhTimer t(c, PH_DYN); dyn_sweep(c, s); }
    if (threadIdx.x == 0) c.acc[A_NOBST] += 1.0;
    __syncthreads();
    load_G(c, s);     // the time-displaced pass used the arena
  }
  Pend pd{1, 0};
  { PhTimer t(c, PH_WRAP); wrap_R(c, s, 0, pd, true); }
  for (int nt = 1; nt <= c.Ltrot; ++nt) {
    {
      PhTimer t(c, PH_KIN);
      build_table(c, s, nt);
      kin_rows(c, s, s.G, s.ldg, N, 1);             // B G
      kin_cols(c, s, s.G, s.ldg, N, -1);            // G B^-1
    }
    { PhTimer t(c, PH_PROP); propose_slice(c, s, nt, false, 1); }  // bonds 1..2N
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.hi = nt;
    scale_G_mu(c, s);                               // propT_R
    if (nt % c.Nwrap == 0) { PhTimer t(c, PH_WRAP); wrap_R(c, s, nt, pd, true); }
    { PhTimer t(c, PH_OBS); obs_equal(c, s, nt); }
  }
}

// Local_sweep (src/local_sweep.f90:152-195): one bin.
__device__ __noinline__ void chain_sweep(const ChainDesc &c, const Smem &s, int nsweep, bool toggle,
                            double h_is_zero) {
  const int N = c.N;
  // Local_sweep_reset (src/local_sweep.f90:56-71)
  if (threadIdx.x == 0) {
    for (int q = A_FLUX_SUM; q <= A_ACC_DEN; ++q) c.acc[q] = 0.0;
  }
  if (toggle) {
    const size_t n = (size_t)7 * c.Ltrot * N;
    for (size_t i = threadIdx.x; i < n; i += Z2_NT) c.obs_tau[i] = 0.0;
  }
  if (h_is_zero != 0.0) {
    for (int b = threadIdx.x; b < c.nb; b += Z2_NT) {
      signed char v = c.sigma[b];
      for (int t = 1; t < c.Ltrot; ++t) c.sigma[(size_t)t * c.nb + b] = v;
    }
  }
  for (int i = threadIdx.x; i < 2 * c.nb; i += Z2_NT) s.bond[i] = c.bonds[i];
  __syncthreads();
  load_G(c, s);
  for (int n = 0; n < nsweep; ++n) {
    sweep_L(c, s);
    sweep_R(c, s, toggle);
  }
  if (threadIdx.x == 0) {
    // Obs_equal_ave (src/obser_equal.f90:50-71)
    const double nobs = c.acc[A_NOBS];
    double *o = c.acc + A_BIN0;
    for (int q = 0; q < 7; ++q) o[q] = 0.0;
    if (nobs > 0.0) {
      const double z = 1.0 / nobs;
      const double fm = c.acc[A_FLUX_SUM] * z, fsq = c.acc[A_FLUX_SQ] * z;
      o[0] = fm;
      o[1] = c.beta * (double)N * fmax(0.0, fsq - fm * fm);
      o[2] = (c.acc[A_PAIR] * z) / (double)N;
      o[3] = (c.acc[A_CDW] * z) / (double)N;
      o[4] = (c.acc[A_CDWS] * z) / (double)N;
      o[5] = (o[3] > 1.0e-12) ? 1.0 - o[4] / o[3] : 0.0;
      o[6] = c.acc[A_DENS] * z;
    }
    // Acc_calc_ratio (src/process_matrix.f90:134-140)
    if (c.acc[A_ACC_DEN] > 0.0) c.acc[A_ACC] += c.acc[A_ACC_NUM] / c.acc[A_ACC_DEN];
  }
  if (toggle) {   // Obs_tau_ave (src/obser_tau.f90:37-47)
    __syncthreads();
    const double z = 1.0 / c.acc[A_NOBST];
    const size_t n = (size_t)7 * c.Ltrot * N;
    for (size_t i = threadIdx.x; i < n; i += Z2_NT) c.obs_tau[i] = z * c.obs_tau[i];
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Adjoint of log|det(1 + B_Ltrot ... B_1)| wrt per-bond hopping and mu.
// d/dt_b = sum over the two occurrences of b in each slice of
//   (dtau/2) sigma_b Tr[(I - G_F) X_b] = -(dtau/2) sigma_b (G_F(p1,p2) + G_F(p2,p1)),
// G_F the Green's function whose product starts at factor F; walking the
// factors one at a time is G <- F G F^-1.  UDV checkpoints every Nwrap slices
// (the L stacks from a backward pass, the R chain recomputed going forward)
// restore G at every stabilization point.  d/dmu = beta Tr(I - G(0)).
// ---------------------------------------------------------------------------
__device__ __noinline__ void chain_logdet_grad(const ChainDesc &c, const Smem &s) {
  const int N = c.N;
  for (int i = threadIdx.x; i < 2 * c.nb; i += Z2_NT) s.bond[i] = c.bonds[i];
  for (int b = threadIdx.x; b < c.nb; b += Z2_NT) c.grad[b] = 0.0;
  __syncthreads();
  chain_pre(c, s);
  // log|det(1 + UR DR VR)| = log|det(UR^T + DR VR)| = sum log D of its QRP
  {
    int lda; double *A = qr_matrix(c, s, lda);
    for (int j = threadIdx.x / 32; j < N; j += Z2_WARPS)
      for (int i = threadIdx.x & 31; i < N; i += 32)
        A[i + (size_t)j * lda] = c.UR[j + (size_t)i * N] + c.DR[i] * c.VR[i + (size_t)j * N];
    __syncthreads();
    blk_geqp3(A, lda, N, s.ivec, s.vec, s.vec + N, s.vec + 2 * N);
    double l = 0.0;
    for (int i = threadIdx.x; i < N; i += Z2_NT) l += log(fabs(A[i + (size_t)i * lda]));
    l = blk_sum(l, s.red);
    if (threadIdx.x == 0) c.acc[A_LOGDET] = l;
    __syncthreads();
  }
  load_G(c, s);
  // backward pass: L stacks
  Pend pd{1, 0};
  for (int nt = c.Ltrot; nt >= 1; --nt) {
    if (nt % c.Nwrap == 0) wrap_L(c, s, nt, pd, false);
    scale_G_mu(c, s);
    build_table(c, s, nt);
    kin_cols(c, s, s.G, s.ldg, N, 1);
    kin_rows(c, s, s.G, s.ldg, N, -1);
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.lo = nt;
  }
  wrap_L(c, s, 0, pd, false);
  {
    double t = 0.0;
    for (int i = threadIdx.x; i < N; i += Z2_NT) t += 1.0 - s.G[i + (size_t)i * s.ldg];
    t = blk_sum(t, s.red);
    if (threadIdx.x == 0) c.acc[A_DMU] = c.beta * t;
    __syncthreads();
  }
  // forward pass with factor-by-factor wraps
  pd.lo = 1; pd.hi = 0;
  wrap_R(c, s, 0, pd, false);
  const double hd = 0.5 * c.dtau;
  for (int nt = 1; nt <= c.Ltrot; ++nt) {
    build_table(c, s, nt);
    for (int p = 0; p < 8; ++p) {
      const int g = c_gorder[p];
      for (int k = threadIdx.x; k < c.half; k += Z2_NT) {
        const int q = g * c.half + k;
        const int b = c.groups[q];
        const int p1 = s.tp[2 * q], p2 = s.tp[2 * q + 1];
        const double sgm = (double)c.sigma[(size_t)(nt - 1) * c.nb + b];
        c.grad[b] += hd * sgm * (-(s.G[p1 + (size_t)p2 * s.ldg] + s.G[p2 + (size_t)p1 * s.ldg]));
      }
      __syncthreads();
      kin_group_rows(c, s, s.G, s.ldg, N, g, 1);
      kin_group_cols(c, s, s.G, s.ldg, N, g, -1);
    }
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.hi = nt;
    scale_G_mu(c, s);
    if (nt % c.Nwrap == 0) wrap_R(c, s, nt, pd, false);
  }
  spill_G(c, s);
}
