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
  chain_stab_U(c, s, A, lda, c.URd, c.DRd, c.VRd, false);
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

// Dyn_reset (src/dynamics.f90:41-48, Propgr_reset src/process_matrix.f90:88-96):
// the Dyn copy of the propagator and G00 = Gtt = Gt0 = G, G0t = -(I - G),
// from the chain's G in global memory.
__device__ __noinline__ void dyn_reset(const ChainDesc &c, const Smem &s) {
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
}

// propgrK_R (src/multiply.f90:43-63) without the U factor, and propgrT_R
// (src/multiply.f90:110-130): Gt0 <- B Gt0, G0t <- G0t B^-1, Gtt <- B Gtt B^-1,
// then the mu factors.
__device__ __noinline__ void propgr_R(const ChainDesc &c, const Smem &s, int nt, bool kin, bool mu) {
  const int N = c.N;
  if (kin && c.use_kin) {
    build_table(c, s, nt);
    kin_global(c, s, c.Gt0, 1, 0);
    kin_global(c, s, c.G0t, 0, -1);
    kin_global(c, s, c.Gtt, 1, -1);
  }
  if (mu && (c.eP != 1.0 || c.eM != 1.0)) {
    blk_scale(c.Gt0, N, N, N, c.eP);
    blk_scale(c.G0t, N, N, N, c.eM);
    blk_scale(c.Gtt, N, N, N, c.eP);
    blk_scale(c.Gtt, N, N, N, c.eM);
  }
}

// Dyn_reset + Dyn_sweep_R (src/dynamics.f90:41-62): the G(tau,0) chain.
// The arena is free here (G is spilled in c.G).
__device__ __noinline__ void dyn_sweep(const ChainDesc &c, const Smem &s) {
  dyn_reset(c, s);
  Pend pd{1, 0};
  for (int nt = 1; nt <= c.Ltrot; ++nt) {
    obs_tau(c, s, nt);
    propgr_R(c, s, nt, true, true);
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.hi = nt;
    if (nt % c.Nwrap == 0) wrap_tau(c, s, nt, pd);
  }
}

// Local_sweep_pre (src/local_sweep.f90:87-104)
__device__ __noinline__ void chain_pre(const ChainDesc &c, const Smem &s) {
  const int N = c.N;
  if (threadIdx.x == 0) c.acc[A_NOTBETA] = 0.0;   // is_beta = .true. (src/main.f90:73)
  if (c.hzero) {   // this%reset (src/local_sweep.f90:63-69): sigma constant in tau
    for (int b = threadIdx.x; b < c.nb; b += Z2_NT) {
      const signed char v = c.sigma[b];
      for (int t = 1; t < c.Ltrot; ++t) c.sigma[(size_t)t * c.nb + b] = v;
    }
    __syncthreads();
  }
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

// Asks L2 for n doubles at p, one 128-byte line per prefetch, the lines
// spread over the block (a hint: nothing waits for it).
__device__ __forceinline__ void l2_prefetch(const double *p, int n) {
  const char *b = reinterpret_cast<const char *>(p);
  const size_t bytes = (size_t)n * sizeof(double);
  for (size_t o = (size_t)threadIdx.x * 128; o < bytes; o += (size_t)Z2_NT * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(b + o));
}

// The matrices a wrap reads from global memory, fetched into L2 about a
// slice ahead of it: the stack entry st of the other sweep direction (kept
// since the previous sweep) and this direction's U, V, D (from the previous
// wrap), which other chains' traffic has usually evicted by then.
__device__ __noinline__ void prefetch_wrap(const ChainDesc &c, int st, bool left) {
  const int N = c.N, NN = N * N;
  if (left) {
    l2_prefetch(c.URs + (size_t)st * NN, NN);
    l2_prefetch(c.VRs + (size_t)st * NN, NN);
    l2_prefetch(c.DRs + (size_t)st * N, N);
    l2_prefetch(c.ULT, NN);
    l2_prefetch(c.VL, NN);
    l2_prefetch(c.DL, N);
  } else {
    l2_prefetch(c.ULTs + (size_t)st * NN, NN);
    l2_prefetch(c.VLs + (size_t)st * NN, NN);
    l2_prefetch(c.DLs + (size_t)st * N, N);
    l2_prefetch(c.UR, NN);
    l2_prefetch(c.VR, NN);
    l2_prefetch(c.DR, N);
  }
}

// Local_sweep_L (src/local_sweep.f90:106-124)
__device__ __noinline__ void sweep_L(const ChainDesc &c, const Smem &s) {
  const int N = c.N;
  Pend pd{1, 0};
  for (int nt = c.Ltrot; nt >= 1; --nt) {
    if (nt % c.Nwrap == 0) { PhTimer t(c, PH_WRAP); wrap_L(c, s, nt, pd, true); }
    if ((nt - 1) % c.Nwrap == 0) prefetch_wrap(c, (nt - 1) / c.Nwrap, true);
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
    if (nt % c.Nwrap == 0) prefetch_wrap(c, nt / c.Nwrap, false);
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

__device__ __noinline__ void bin_average(const ChainDesc &c, bool toggle);

// Local_sweep_reset (src/local_sweep.f90:56-71): the bin's sums and
// acceptance counters, the tau correlators when toggle, and for h = 0 the
// links made constant in tau.
__device__ __noinline__ void sweep_reset(const ChainDesc &c, bool toggle, bool h_is_zero) {
  const int N = c.N;
  if (threadIdx.x == 0) {
    for (int q = A_FLUX_SUM; q <= A_ACC_DEN; ++q) c.acc[q] = 0.0;
  }
  if (toggle) {
    const size_t n = (size_t)7 * c.Ltrot * N;
    for (size_t i = threadIdx.x; i < n; i += Z2_NT) c.obs_tau[i] = 0.0;
  }
  if (h_is_zero) {
    for (int b = threadIdx.x; b < c.nb; b += Z2_NT) {
      signed char v = c.sigma[b];
      for (int t = 1; t < c.Ltrot; ++t) c.sigma[(size_t)t * c.nb + b] = v;
    }
  }
  __syncthreads();
}

// Local_sweep (src/local_sweep.f90:152-195): one bin.
__device__ __noinline__ void chain_sweep(const ChainDesc &c, const Smem &s, int nsweep, bool toggle,
                            double h_is_zero) {
  sweep_reset(c, toggle, h_is_zero != 0.0);
  for (int i = threadIdx.x; i < 2 * c.nb; i += Z2_NT) s.bond[i] = c.bonds[i];
  __syncthreads();
  load_G(c, s);
  for (int n = 0; n < nsweep; ++n) {
    if (c.acc[A_NOTBETA] == 0.0) {   // is_beta: L then R
      sweep_L(c, s);
      sweep_R(c, s, toggle);
    } else {
      sweep_R(c, s, toggle);
      sweep_L(c, s);
    }
  }
  bin_average(c, toggle);
}

// Obs_equal_ave (src/obser_equal.f90:50-71): the bin averages of nobs
// slices into the chain's readback slots.
__device__ __noinline__ void obs_equal_ave(const ChainDesc &c, double nobs) {
  const int N = c.N;
  if (threadIdx.x == 0) {
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
  }
  __syncthreads();
}

// Obs_tau_ave (src/obser_tau.f90:37-47): the tau correlators / nobst.
__device__ __noinline__ void obs_tau_ave(const ChainDesc &c, double nobst) {
  const double z = 1.0 / nobst;
  const size_t n = (size_t)7 * c.Ltrot * c.N;
  for (size_t i = threadIdx.x; i < n; i += Z2_NT) c.obs_tau[i] = z * c.obs_tau[i];
  __syncthreads();
}

// End of a bin: Obs_equal_ave, Acc_calc_ratio (src/process_matrix.f90:134-140)
// and, with toggle, Obs_tau_ave, with the counts the half-sweeps kept.
__device__ __noinline__ void bin_average(const ChainDesc &c, bool toggle) {
  obs_equal_ave(c, c.acc[A_NOBS]);
  if (threadIdx.x == 0 && c.acc[A_ACC_DEN] > 0.0)
    c.acc[A_ACC] += c.acc[A_ACC_NUM] / c.acc[A_ACC_DEN];
  if (toggle) obs_tau_ave(c, c.acc[A_NOBST]);
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Boson-only warm-up: Local_sweep_therm (src/local_sweep.f90:73-85) with
// LocalK_therm (src/localK.f90:400-420), Metropolis on the gauge weight alone.
// The sweep is one ordered pass of ranf draws, so thread 0 runs it, on the
// configuration staged in shared memory when it fits (the arena is free
// before z2_pre).  Acc_Kt%acc accumulates in A_TACC.
// ---------------------------------------------------------------------------
__device__ __noinline__ void chain_therm(const ChainDesc &c, const Smem &s, int nwarm) {
  const int L = c.Ltrot, nb = c.nb;
  const size_t bytes = (size_t)L * nb;
  const size_t arena = 8 * ((c.g_in_smem ? (size_t)c.N * s.ldg : 0) + (size_t)s.tile_doubles);
  const bool staged = bytes <= arena;
  signed char *sig = staged ? reinterpret_cast<signed char *>(s.arena) : c.sigma;
  if (staged) {
    for (size_t i = threadIdx.x; i < bytes; i += Z2_NT) sig[i] = c.sigma[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int st = *c.rng;
    double acc = 0.0;
    for (int w = 0; w < nwarm; ++w) {
      if (c.hzero)   // Local_sweep_reset (src/local_sweep.f90:63-66)
        for (int t = 1; t < L; ++t)
          for (int b = 0; b < nb; ++b) sig[(size_t)t * nb + b] = sig[b];
      int num = 0;
      for (int t = 0; t < L; ++t) {
        signed char *sg = sig + (size_t)t * nb;
        const signed char *sp = sig + (size_t)((t - 1 + L) % L) * nb;
        const signed char *sn = sig + (size_t)((t + 1) % L) * nb;
        for (int b = 0; b < nb; ++b) {
          const int *bb = c.bbonds + 6 * b;
          const double s_old = (double)sg[b];
          const double tmp_old = s_old * sg[bb[0]] * sg[bb[1]] * sg[bb[2]] +
                                 s_old * sg[bb[3]] * sg[bb[4]] * sg[bb[5]];
          const int is = (int)(-2.0 * tmp_old + 4.0) >> 2;
          const double tn = s_old * ((double)sp[b] + (double)sn[b]);
          const int it = (int)(-2.0 * tn + 4.0) >> 2;
          st = ranf_adv(st, 1);
          if (c.rb[is * 3 + it] > (double)st * (1.0 / 2147483648.0)) {
            sg[b] = (signed char)(-sg[b]);
            ++num;
          }
        }
      }
      acc += (double)num / (double)((size_t)nb * L);
    }
    *c.rng = st;
    c.acc[A_TACC] += acc;
  }
  __syncthreads();
  if (staged) {
    for (size_t i = threadIdx.x; i < bytes; i += Z2_NT) c.sigma[i] = sig[i];
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Global Wolff-in-tau move (src/global_update.f90, src/globalK.f90)
// ---------------------------------------------------------------------------
// nranf (src/calc_basic.f90:113-121): nint(ranf*N + 0.5) clamped to 1..N.
__device__ __forceinline__ int dev_nranf(unsigned int &st, int N) {
  st = ranf_adv(st, 1);
  const double x = (double)st * (1.0 / 2147483648.0) * (double)N + 0.5;
  long long n = llround(x);            // nint: half away from zero
  if (n < 1) n = 1;
  if (n > N) n = N;
  return (int)n;
}

// State of the chain that a rejected move restores (Prop_assign and
// Wrlist_assign, src/process_matrix.f90:58-66, 104-112): G, UR, VR, ULT, VL
// (contiguous), DR, DL, the four UDV stacks, their D stacks and Xmaxm.
__device__ __noinline__ void global_backup(const ChainDesc &c, bool save) {
  const size_t NN = (size_t)c.N * c.N, S1 = (size_t)c.Nst + 1;
  const size_t n0 = 5 * NN, n1 = 2 * (size_t)c.N, n2 = 4 * NN * S1, n3 = 2 * (size_t)c.N * S1;
  double *src[4] = {c.G, c.DR, c.URs, c.DRs};
  double *bak[4] = {c.gbak, c.gbak + n0, c.gbak + n0 + n1, c.gbak + n0 + n1 + n2};
  const size_t len[4] = {n0, n1, n2, n3};
  for (int q = 0; q < 4; ++q) {
    const double *from = save ? src[q] : bak[q];
    double *to = save ? bak[q] : src[q];
    for (size_t i = threadIdx.x; i < len[q]; i += Z2_NT) to[i] = from[i];
  }
  if (threadIdx.x == 0) {
    double *x = c.gbak + n0 + n1 + n2 + n3;
    if (save) *x = c.acc[A_XMAX]; else c.acc[A_XMAX] = *x;
  }
  __syncthreads();
}

// One cluster site of a trial half-sweep (ratioK_fermion, src/globalK.f90:15-113):
// the bond flips at slice nt if the cluster holds nt; |det Prod|^2 goes into
// the fermion log ratio (thread 0) and G takes the rank-2 update.
__device__ __noinline__ void global_flip_slice(const ChainDesc &c, const Smem &s, int nt, int b,
                                               double &lrf) {
  if (!c.gmask[nt - 1]) return;
  const int N = c.N, ldg = s.ldg, ldx = s.ldx;
  double *G = s.G, *X = s.X, *Yt = s.Yt;
  signed char *sg = c.sigma + (size_t)(nt - 1) * c.nb;
  const int p1 = s.bond[2 * b], p2 = s.bond[2 * b + 1];
  const double s_old = (double)sg[b], s_new = -s_old;
  const double D11 = c.dlt[2 * b], D12 = s_new * c.dlt[2 * b + 1];
  const double g11 = G[p1 + (size_t)p1 * ldg], g12 = G[p1 + (size_t)p2 * ldg];
  const double g21 = G[p2 + (size_t)p1 * ldg], g22 = G[p2 + (size_t)p2 * ldg];
  const double l11 = __dsub_rn(1.0, g11), l12 = -g12, l21 = -g21, l22 = __dsub_rn(1.0, g22);
  const double m11 = __dadd_rn(__dmul_rn(D11, l11), __dmul_rn(D12, l21));
  const double m12 = __dadd_rn(__dmul_rn(D11, l12), __dmul_rn(D12, l22));
  const double m21 = __dadd_rn(__dmul_rn(D12, l11), __dmul_rn(D11, l21));
  const double m22 = __dadd_rn(__dmul_rn(D12, l12), __dmul_rn(D11, l22));
  const double p11 = __dadd_rn(1.0, m11), p12 = m12, p21 = m21, p22 = __dadd_rn(1.0, m22);
  const double det = __dsub_rn(__dmul_rn(p11, p22), __dmul_rn(p12, p21));
  if (threadIdx.x == 0) lrf += log(fmax(fabs(__dmul_rn(det, det)), 1.0e-300));
  const double q00 = p22 / det, q01 = -p12 / det, q10 = -p21 / det, q11 = p11 / det;
  __syncthreads();   // every thread has read G(P, P)
  for (int i = threadIdx.x; i < N; i += Z2_NT) {
    const double u0 = G[i + (size_t)p1 * ldg], u1 = G[i + (size_t)p2 * ldg];
    const double v0 = G[p1 + (size_t)i * ldg], v1 = G[p2 + (size_t)i * ldg];
    X[2 * i] = u0 * q00 + u1 * q10;       // columns 0, 1 of the paired layout
    X[2 * i + 1] = u0 * q01 + u1 * q11;
    double y0 = -D11 * v0 - D12 * v1;
    double y1 = -D12 * v0 - D11 * v1;
    if (i == p1) { y0 += D11; y1 += D12; }
    if (i == p2) { y0 += D12; y1 += D11; }
    Yt[2 * i] = y0;
    Yt[2 * i + 1] = y1;
  }
  __syncthreads();
  rank_update(G, ldg, X, Yt, N, ldx, 2);
  if (threadIdx.x == 0) sg[b] = (signed char)(-sg[b]);
  __syncthreads();
}

// Global_sweep_L's trial (src/global_update.f90:228-272 with GlobalK_prop_L,
// src/globalK.f90:115-133): the Local_sweep_L structure without observables
// or drift statistics, the cluster's flips forced.
__device__ __noinline__ void sweep_L_trial(const ChainDesc &c, const Smem &s, int b, double &lrf) {
  const int N = c.N;
  Pend pd{1, 0};
  for (int nt = c.Ltrot; nt >= 1; --nt) {
    if (nt % c.Nwrap == 0) { PhTimer t(c, PH_WRAP); wrap_L(c, s, nt, pd, false); }
    scale_G_mu(c, s);                                          // propT_L
    global_flip_slice(c, s, nt, b, lrf);
    {
      PhTimer t(c, PH_KIN);
      build_table(c, s, nt);
      kin_cols(c, s, s.G, s.ldg, N, 1);
      kin_rows(c, s, s.G, s.ldg, N, -1);
    }
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.lo = nt;
  }
  { PhTimer t(c, PH_WRAP); wrap_L(c, s, 0, pd, false); }
}

// Global_sweep_R's trial (src/global_update.f90:274-318, GlobalK_prop_R,
// src/globalK.f90:135-153).
__device__ __noinline__ void sweep_R_trial(const ChainDesc &c, const Smem &s, int b, double &lrf) {
  const int N = c.N;
  Pend pd{1, 0};
  { PhTimer t(c, PH_WRAP); wrap_R(c, s, 0, pd, false); }
  for (int nt = 1; nt <= c.Ltrot; ++nt) {
    {
      PhTimer t(c, PH_KIN);
      build_table(c, s, nt);
      kin_rows(c, s, s.G, s.ldg, N, 1);
      kin_cols(c, s, s.G, s.ldg, N, -1);
    }
    global_flip_slice(c, s, nt, b, lrf);
    if (pd.lo > pd.hi) { pd.lo = nt; pd.hi = nt; } else pd.hi = nt;
    scale_G_mu(c, s);                                          // propT_R
    if (nt % c.Nwrap == 0) { PhTimer t(c, PH_WRAP); wrap_R(c, s, nt, pd, false); }
  }
}

// Global_sweep (src/global_update.f90:320-337): nglobal Wolff moves.
__device__ __noinline__ void chain_global(const ChainDesc &c, const Smem &s, int nglobal) {
  const int L = c.Ltrot, nb = c.nb;
  for (int i = threadIdx.x; i < 2 * nb; i += Z2_NT) s.bond[i] = c.bonds[i];
  __syncthreads();
  double *gs = s.red + 40;   // [0] bond, [1] size, [2] log ratio space, [3] accept
  int num = 0;
  double size_sum = 0.0;
  for (int g = 0; g < nglobal; ++g) {
    const bool left = c.acc[A_NOTBETA] == 0.0;
    if (threadIdx.x == 0) {
      // Wolff_flip (src/global_update.f90:66-86) on the current sigma
      unsigned int st = *c.rng;
      const int b = dev_nranf(st, nb) - 1;
      for (int t = 0; t < L; ++t) c.gmask[t] = 0;
      int head = 0, tail = 0;
      const int q0 = dev_nranf(st, L) - 1;
      c.gqueue[tail++] = q0;
      c.gmask[q0] = 1;
      while (head < tail) {
        const int cur = c.gqueue[head++];
        for (int off = -1; off <= 1; off += 2) {
          const int nbr = (cur + off + L) % L;
          if (c.gmask[nbr]) continue;
          if (c.sigma[(size_t)nbr * nb + b] == c.sigma[(size_t)cur * nb + b]) {
            if (c.ptime > 0.0) {
              st = ranf_adv(st, 1);
              if ((double)st * (1.0 / 2147483648.0) < c.ptime) {
                c.gqueue[tail++] = nbr;
                c.gmask[nbr] = 1;
              }
            }
          }
        }
      }
      // compute_space_log_ratio (src/global_update.f90:133-172), old sigma
      double lrs = 0.0;
      if (c.alphaJ != 0.0) {
        for (int t = 0; t < L; ++t) {
          if (!c.gmask[t]) continue;
          const signed char *sgt = c.sigma + (size_t)t * nb;
          for (int h = 0; h < 2; ++h) {
            double prod = (double)sgt[b];
            for (int k = 0; k < 3; ++k) prod = prod * (double)sgt[c.bbonds[6 * b + 3 * h + k]];
            lrs += -2.0 * c.alphaJ * prod;
          }
        }
      }
      *c.rng = st;
      gs[0] = (double)b; gs[1] = (double)tail; gs[2] = lrs;
    }
    __syncthreads();
    const int b = (int)gs[0];
    const double size = gs[1];
    size_sum += size;
    global_backup(c, true);
    load_G(c, s);
    double lrf = 0.0;
    if (left) sweep_L_trial(c, s, b, lrf);
    else sweep_R_trial(c, s, b, lrf);
    if (threadIdx.x == 0) {
      const double lrt = lrf + gs[2];
      unsigned int st = ranf_adv(*c.rng, 1);
      *c.rng = st;
      const double r = (double)st * (1.0 / 2147483648.0);
      const bool acc = fmin(0.0, lrt) >= log(fmax(r, 1.0e-300));
      gs[3] = acc ? 1.0 : 0.0;
      if (acc) c.acc[A_NOTBETA] = left ? 1.0 : 0.0;
    }
    __syncthreads();
    if (gs[3] != 0.0) {
      ++num;
    } else {
      // restore the state and flip the cluster back
      global_backup(c, false);
      for (int t = threadIdx.x; t < L; t += Z2_NT)
        if (c.gmask[t]) {
          signed char *p = c.sigma + (size_t)t * nb + b;
          *p = (signed char)(-*p);
        }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    // Acc_Kg%ratio and the cluster-size average (src/global_update.f90:330-335)
    c.acc[A_GNUM] = (double)num;
    c.acc[A_GDEN] = (double)nglobal;
    if (nglobal > 0) {
      c.acc[A_GACC] += (double)num / (double)nglobal;
      c.acc[A_GSIZE] += size_sum / (double)nglobal;
    }
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
