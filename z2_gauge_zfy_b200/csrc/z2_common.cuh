// z2_common.cuh -- shared definitions of the B200 DQMC library.
//
// One chain (one Markov chain = one MPI rank of the reference) is run by one
// CTA of Z2_NT threads.  All chain state lives in HBM; the equal-time Green's
// function G and the delayed-update factors X, Y live in shared memory while
// a time slice is processed.  Everything is real FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define Z2_NT 256
#define Z2_WARPS (Z2_NT / 32)
#define Z2_FULL 0xffffffffu
#define Z2_NRED 64              // doubles of block-reduction scratch
#define Z2_MIN_TILE 2080        // doubles of shared work space kept after G and X, Y

// Accumulator layout of ChainDesc::acc (doubles).
enum {
  A_FLUX_SUM = 0, A_FLUX_SQ, A_PAIR, A_CDW, A_CDWS, A_DENS,
  A_NOBS, A_NOBST, A_ACC_NUM, A_ACC_DEN, A_ACC, A_XMAX, A_XMEAN,
  A_TXMAX0, A_TXMAX1, A_TXMAX2, A_TXMEAN0, A_TXMEAN1, A_TXMEAN2,
  A_BIN0,                        // 7 bin results: flux_avg .. density
  A_LOGDET = A_BIN0 + 7, A_DMU, A_DRAWS,
  // global moves (src/global_update.f90): accepted / proposed of the last
  // Global_sweep, Acc_Kg%acc, Wolff%size_cluster, sweep direction (0: the
  // next bin runs L then R, the reference's is_beta = .true.)
  A_GNUM, A_GDEN, A_GACC, A_GSIZE, A_NOTBETA,
  A_TACC,                        // Acc_Kt%acc of the boson-only warm-up
  A_PH0,                         // Z2_NPHASE per-phase SM cycle counters
  A_COUNT = A_PH0 + 12
};

// Phases of a bin timed with clock64() by thread 0 (tracing; no effect on
// results): checkerboard wrap of G, proposals (evaluation + rank-2 bookkeeping),
// rank-2k flushes, equal-time observables, wraps/stabilization, the
// time-displaced chain; inside those: the UDV stabilization, the stabilized
// Green's function, warp-0 flip-ratio rounds, the accepted-flip columns of X
// and Y, the pending slice products of a wrap, and the UDV stack copies.
enum { PH_KIN = 0, PH_PROP, PH_FLUSH, PH_OBS, PH_WRAP, PH_DYN, PH_STABU, PH_STABG,
       PH_EVAL, PH_COLS, PH_PEND, PH_STACK, PH_COUNT = 12 };

// Status flags (ChainDesc::status).
enum { ST_NONFINITE = 1, ST_BADARG = 2 };

// Per-chain descriptor, built on the host and copied to device memory.
struct ChainDesc {
  // sizes
  int N, Lx, Ly, Ltrot, Nwrap, Nst, nb, half;
  int ldg;          // leading dimension of shared-memory matrices (N + 2 when
                    // 4 divides N: 16-byte pairs, conflict-free DMMA
                    // accumulator fragments; else odd)
  int k2;           // 2 * delayed-update rank
  int g_in_smem;    // G (and the QR work matrix) fit in the arena
  int small_bytes;  // bytes of the fixed small region (start of smem)
  // physics
  double beta, dtau, eP, eM, rt_scalar;
  double rb[9];     // boson ratio table [(ds+4)/4 * 3 + (dt+4)/4]
  int use_kin;      // RT > Zero (src/local_sweep.f90:96, dynamics.f90:57)
  int hzero;        // |h| <= Zero (src/local_sweep.f90:64)
  int flush_shape;  // tile shape of the rank-2k flush (FS_*; 0 = by divisibility)
  int stab_exact;   // 1: the reference's column-pivoted QR in the wraps; 0: the
                    // pre-pivoted blocked QR and scale-split G (z2_stab.cuh)
  int kin_fused;    // L when the bond table has the square-lattice layout of
                    // kin_rows_fused / kin_cols_fused (host-checked), else 0
  // lattice tables (device)
  const int *bonds;     // [2N][2] endpoints (0-based sites)
  const int *groups;    // [4][half] bond ids of checkerboard groups 1..4
  const int *bbonds;    // [2N][6] plaquette partner bonds (bond_bonds 1..6)
  const int *plaq;      // [N][4] bonds of the plaquette at each site
  const int *xy;        // [N][2] 1-based coordinates
  const int *nbx;       // [N] +x neighbour (L_bonds(:,1))
  const double *chsh;   // [2N][2] cosh(alpha_b), sinh(alpha_b)
  const double *dlt;    // [2N][2] Delta(1,1), Delta(1,2) for sigma_new = +1
  const double *stag;   // [N] staggered sign
  const double *pshift; // [(2Lx-1)(2Ly-1)] cos(qx dx + pi dy)
  // state (device)
  signed char *sigma;   // [Ltrot][2N]
  double *G, *UR, *VR, *DR, *ULT, *VL, *DL;      // ULT = UL^T
  double *URs, *VRs, *DRs, *ULTs, *VLs, *DLs;    // stacks (Nst+1)
  double *W0, *W1, *W2, *W3;                      // N x N workspaces
  double *W4;       // QR work matrix when the arena cannot hold N x N
  // time-displaced chain
  double *G00, *Gtt, *Gt0, *G0t;
  double *URd, *VRd, *DRd, *ULTd, *VLd, *DLd;
  double *B0, *B1, *B2, *B3;                      // 2N x 2N workspaces
  double *obs_tau;      // [7][Ltrot][N]
  double *grad;         // [2N] adjoint output
  // global moves: state backup (G..VL, DR DL, stacks, Xmaxm), cluster mask
  // and queue, allocated by the first z2_sweep_global
  double *gbak;
  signed char *gmask;   // [Ltrot]
  int *gqueue;          // [Ltrot]
  double alphaJ;        // dtau J (plaquette log ratio)
  double ptime;         // compute_time_bond_prob
  // accumulators
  double *acc;          // [A_COUNT]
  unsigned int *rng;    // ranf state (iseed), always in [0, 2^31)
  const double *replay; // optional replayed uniforms
  long long *replay_pos;
  long long nreplay;
  unsigned char *dec;   // optional decisions [2][Ltrot][2N]
  double *ratios;       // optional ratios, same layout
  int *status;
  int pad1;
};

// Shared-memory layout of one chain (pointers into dynamic smem).
struct Smem {
  double *red;      // [Z2_NRED]
  double *vec;      // [8N]: tau, vn1, vn2, D, dtmp, ...
  int *ivec;        // [2N]: jpvt, ...
  int *tp;          // [2N][2] slice rotation table (p1, p2) in group order
  double *tc;       // [2N] C of the slice table
  double *ts;       // [2N] S of the slice table (for nflag = +1)
  int *bond;        // [2N][2] bond endpoints
  signed char *sig; // [2N] sigma of the current slice
  int *flag;        // [16] scalars
  double *arena;    // big region
  double *G;        // G (smem arena or global)
  int ldg;          // leading dimension of G
  double *X, *Yt;   // delayed-update factors [k2][ldx]
  int ldx;          // leading dimension of X, Yt (4 mod 16: conflict-free DMMA fragments)
  double *Wq;       // QR work matrix (arena or global)
  int ldq;
  double *tile;     // GEMM/panel staging (arena tail)
  int tile_doubles;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(Z2_FULL, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(Z2_FULL, v, o));
  return v;
}

// Block-wide sum; every thread gets the total.  The leading barrier makes
// the scratch reusable back to back.
__device__ __forceinline__ double blk_sum(double v, double *red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < Z2_WARPS; ++w) t += red[w];
  return t;
}
__device__ __forceinline__ double blk_max(double v, double *red) {
  v = warp_max(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = red[0];
#pragma unroll
  for (int w = 1; w < Z2_WARPS; ++w) t = fmax(t, red[w]);
  return t;
}
// Sum of NV values per thread in one pass (NV <= 8).
template <int NV>
__device__ __forceinline__ void blk_sum_n(double *v, double *red) {
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) red[q * Z2_WARPS + (threadIdx.x >> 5)] = v[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < Z2_WARPS; ++w) t += red[q * Z2_WARPS + w];
    v[q] = t;
  }
}

__device__ __forceinline__ long long ph_now() { return clock64(); }

// Leading dimension of the delayed-update factors X, Yt: = 4 (mod 16), so
// each half-warp's 4 rows x 4 columns of a DMMA A/B fragment (row + 4 column
// mod 16) fall on distinct shared-memory bank pairs (two wavefronts per
// fragment load).
__host__ __device__ __forceinline__ int z2_ldx(int N) { return ((N + 15) & ~15) + 4; }

// ranf multiplier powers IP^i mod 2^31, i = 0..32 (filled by the host).
__constant__ unsigned int c_ipow[33];

__device__ __forceinline__ unsigned int ranf_adv(unsigned int s, int n) {
  return (unsigned int)(((unsigned long long)s * c_ipow[n]) & 0x7fffffffull);
}
