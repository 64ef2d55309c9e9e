// z2_chain.cuh -- per-chain DQMC drivers run by one CTA.
//
// Restates the reference's hot path (src/local_sweep.f90, src/localK.f90,
// src/multiply.f90, src/operator_kin.f90, src/stabilization.f90,
// src/dynamics.f90, src/obser_equal.f90, src/obser_tau.f90) for one spin
// sector in real FP64.  Orders of operations follow the reference; the
// implementation is B200-first: G stays in shared memory across a slice,
// accepted flips are queued as rank-2 factors and flushed as one rank-2k
// update, and the U factors of the UDV chains are propagated lazily (all
// Nwrap slices at once, right before the stabilization that needs them).
#pragma once
#include "z2_stab.cuh"

// Checkerboard group order of one B (src/operator_kin.f90:74-85).
__device__ __constant__ int c_gorder[8] = {0, 1, 2, 3, 3, 2, 1, 0};

// ---------------------------------------------------------------------------
// Shared-memory layout
// ---------------------------------------------------------------------------
__device__ __forceinline__ size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

__device__ Smem make_smem(const ChainDesc &c, unsigned char *base, size_t smem_bytes) {
  Smem s;
  const int N = c.N;
  size_t off = 0;
  s.red = (double *)(base + off); off += sizeof(double) * Z2_NRED;
  s.vec = (double *)(base + off); off += sizeof(double) * 8 * N;
  s.tc = (double *)(base + off); off += sizeof(double) * 2 * N;
  s.ts = (double *)(base + off); off += sizeof(double) * 2 * N;
  s.ivec = (int *)(base + off); off += align16(sizeof(int) * 2 * N);
  s.tp = (int *)(base + off); off += align16(sizeof(int) * 4 * N);
  s.bond = (int *)(base + off); off += align16(sizeof(int) * 4 * N);
  s.flag = (int *)(base + off); off += sizeof(int) * 16;
  s.sig = (signed char *)(base + off); off += align16(6 * N);   // slices nt, nt-1, nt+1
  off = align16(off);
  s.arena = (double *)(base + off);
  const size_t arena_doubles = (smem_bytes - off) / sizeof(double);
  const size_t nn = (size_t)N * c.ldg;
  if (c.g_in_smem) {
    s.G = s.arena; s.ldg = c.ldg;
    s.ldx = z2_ldx(N); s.X = s.arena + nn; s.Yt = s.X + (size_t)s.ldx * c.k2;
    s.Wq = s.arena; s.ldq = c.ldg;
    s.tile = s.arena + nn;
    s.tile_doubles = (int)(arena_doubles - nn);
  } else {
    s.G = c.G; s.ldg = N;
    s.ldx = z2_ldx(N); s.X = s.arena; s.Yt = s.X + (size_t)s.ldx * c.k2;
    s.Wq = c.W4;
    s.ldq = N;
    s.tile = s.arena;
    s.tile_doubles = (int)arena_doubles;
  }
  return s;
}

// ---------------------------------------------------------------------------
// Checkerboard kinetic propagator (src/operator_kin.f90:61-179)
// ---------------------------------------------------------------------------
// Slice table in group order: position q = g*half + k holds bond groups[q].
__device__ __noinline__ void build_table(const ChainDesc &c, const Smem &s, int nt) {
  const signed char *sg = c.sigma + (size_t)(nt - 1) * c.nb;
  for (int q = threadIdx.x; q < c.nb; q += Z2_NT) {
    int b = c.groups[q];
    s.tp[2 * q] = c.bonds[2 * b];
    s.tp[2 * q + 1] = c.bonds[2 * b + 1];
    s.tc[q] = c.chsh[2 * b];
    s.ts[q] = (double)sg[b] * c.chsh[2 * b + 1];   // sinh(alpha*sigma) = sigma*sinh(alpha)
  }
  __syncthreads();
}

// One bond of a checkerboard group (process_group): [a, b] <- [[C, S], [S, C]]
// [a, b], with the rounding sequence fixed (one product, one FMA per output)
// so that every kinetic kernel below gives the same bits.
__device__ __forceinline__ void kin_rot(double &a, double &b, double C, double S) {
  const double na = __fma_rn(C, a, __dmul_rn(S, b));
  const double nb = __fma_rn(S, a, __dmul_rn(C, b));
  a = na;
  b = nb;
}

// M <- B^nflag M : rows P1, P2 rotated by [[C,S],[S,C]] (process_group).
// Row rotations never mix columns, so one thread carries its column through
// all eight group passes: no barrier between passes.
// Bonds of one group are disjoint, so a batch of 8 rotations is loaded,
// rotated and stored as a whole (no store-to-load ordering inside a batch).
template <bool ROWS>
__device__ __forceinline__ void kin_group_vec(const Smem &s, double *base, size_t stride, int g0,
                                              int half, double fl) {
  // table pointers in registers (the Smem struct would otherwise be re-read
  // after every store, which may alias it)
  const int2 *__restrict__ tp2 = reinterpret_cast<const int2 *>(s.tp);
  const double *__restrict__ tc = s.tc;
  const double *__restrict__ ts = s.ts;
  int kq = 0;
  for (; kq + 7 < half; kq += 8) {
    int2 pp[8];
    double C[8], S[8], a[8], b[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      pp[q] = tp2[g0 + kq + q];
      C[q] = tc[g0 + kq + q];
      S[q] = fl * ts[g0 + kq + q];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) { a[q] = base[pp[q].x * stride]; b[q] = base[pp[q].y * stride]; }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      kin_rot(a[q], b[q], C[q], S[q]);
      base[pp[q].x * stride] = a[q];
      base[pp[q].y * stride] = b[q];
    }
  }
  for (; kq < half; ++kq) {
    const int2 pp = tp2[g0 + kq];
    const double C = tc[g0 + kq], S = fl * ts[g0 + kq];
    double a = base[pp.x * stride], b = base[pp.y * stride];
    kin_rot(a, b, C, S);
    base[pp.x * stride] = a;
    base[pp.y * stride] = b;
  }
}

// Fused passes on an L x L lattice with periodic boundaries (sites
// y L + x).  The four groups are the x bonds from odd x (group 0) and from
// even x (group 1), and the y bonds from odd y (group 2) and from even y
// (group 3), each listed row by row (HostLattice, src/lattice.f90:72-102):
//   group 0: bond (y L + x, y L + x+1 mod L), x = 2m+1, table slot y L/2 + m
//   group 1: x = 2m, same slots;  group 2: (y L + x, (y+1 mod L) L + x),
//   y = 2m+1, slot m L + x;  group 3: y = 2m, same slots.
// Groups 0 and 1 only mix the sites of one lattice row and groups 2 and 3
// only those of one lattice column, so the pass sequence 0 1 | 2 3 3 2 | 1 0
// runs as three sweeps over lines: a thread loads one line of one matrix
// column (or row) into registers, applies its passes and stores it, instead
// of streaming the whole matrix through shared memory once per pass.  The
// rotations and their order within each bond are those of the pass-by-pass
// kernel, so the results are bitwise equal.
template <int L>
__device__ __forceinline__ void kin_line_odd(double (&v)[L], const double *__restrict__ tc,
                                             const double *__restrict__ ts, double fl, int q0,
                                             int qs) {
#pragma unroll
  for (int m = 0; m < L / 2; ++m) {
    const int q = q0 + m * qs;
    kin_rot(v[2 * m + 1], v[(2 * m + 2) % L], tc[q], fl * ts[q]);
  }
}
template <int L>
__device__ __forceinline__ void kin_line_even(double (&v)[L], const double *__restrict__ tc,
                                              const double *__restrict__ ts, double fl, int q0,
                                              int qs) {
#pragma unroll
  for (int m = 0; m < L / 2; ++m) {
    const int q = q0 + m * qs;
    kin_rot(v[2 * m], v[2 * m + 1], tc[q], fl * ts[q]);
  }
}

// The three sweeps for n independent vectors: vector i's site k sits at
// M[i * vs + k * ks] (kin_rows: vs = ld, ks = 1; kin_cols: vs = 1, ks = ld).
// Threads take (vector, line) pairs, vector fastest, so a warp touches one
// line of 32 consecutive vectors.
template <int L>
__device__ __noinline__ void kin_fused(const Smem &s, double *M, size_t vs, size_t ks, int n,
                                       int nflag) {
  constexpr int H = L * L / 2, HL = L / 2;
  const double fl = (double)nflag;
  const double *__restrict__ tc = s.tc;
  const double *__restrict__ ts = s.ts;
  const int tasks = n * L;
  // a lattice row of one matrix column is contiguous when ks == 1: with an
  // even column stride and an aligned matrix it moves as 16-byte pairs
  const bool pairs = ks == 1 && (vs & 1) == 0 && (reinterpret_cast<size_t>(M) & 15) == 0;
  // groups 0, 1 on lattice rows
  for (int t = threadIdx.x; t < tasks; t += Z2_NT) {
    const int i = t % n, y = t / n;
    double *p = M + (size_t)i * vs + (size_t)(y * L) * ks;
    double v[L];
    if (pairs) {
#pragma unroll
      for (int x = 0; x < L; x += 2) {
        const double2 w = reinterpret_cast<const double2 *>(p)[x >> 1];
        v[x] = w.x; v[x + 1] = w.y;
      }
    } else {
#pragma unroll
      for (int x = 0; x < L; ++x) v[x] = p[(size_t)x * ks];
    }
    kin_line_odd<L>(v, tc, ts, fl, y * HL, 1);
    kin_line_even<L>(v, tc, ts, fl, H + y * HL, 1);
    if (pairs) {
#pragma unroll
      for (int x = 0; x < L; x += 2) reinterpret_cast<double2 *>(p)[x >> 1] = make_double2(v[x], v[x + 1]);
    } else {
#pragma unroll
      for (int x = 0; x < L; ++x) p[(size_t)x * ks] = v[x];
    }
  }
  __syncthreads();
  // groups 2, 3, 3, 2 on lattice columns
  for (int t = threadIdx.x; t < tasks; t += Z2_NT) {
    const int i = t % n, x = t / n;
    double *p = M + (size_t)i * vs + (size_t)x * ks;
    double v[L];
#pragma unroll
    for (int y = 0; y < L; ++y) v[y] = p[(size_t)(y * L) * ks];
    kin_line_odd<L>(v, tc, ts, fl, 2 * H + x, L);
    kin_line_even<L>(v, tc, ts, fl, 3 * H + x, L);
    kin_line_even<L>(v, tc, ts, fl, 3 * H + x, L);
    kin_line_odd<L>(v, tc, ts, fl, 2 * H + x, L);
#pragma unroll
    for (int y = 0; y < L; ++y) p[(size_t)(y * L) * ks] = v[y];
  }
  __syncthreads();
  // groups 1, 0 on lattice rows
  for (int t = threadIdx.x; t < tasks; t += Z2_NT) {
    const int i = t % n, y = t / n;
    double *p = M + (size_t)i * vs + (size_t)(y * L) * ks;
    double v[L];
    if (pairs) {
#pragma unroll
      for (int x = 0; x < L; x += 2) {
        const double2 w = reinterpret_cast<const double2 *>(p)[x >> 1];
        v[x] = w.x; v[x + 1] = w.y;
      }
    } else {
#pragma unroll
      for (int x = 0; x < L; ++x) v[x] = p[(size_t)x * ks];
    }
    kin_line_even<L>(v, tc, ts, fl, H + y * HL, 1);
    kin_line_odd<L>(v, tc, ts, fl, y * HL, 1);
    if (pairs) {
#pragma unroll
      for (int x = 0; x < L; x += 2) reinterpret_cast<double2 *>(p)[x >> 1] = make_double2(v[x], v[x + 1]);
    } else {
#pragma unroll
      for (int x = 0; x < L; ++x) p[(size_t)x * ks] = v[x];
    }
  }
  __syncthreads();
}

// kin_fused for M <- M B (vectors are the rows of M, sites stride ld) when ld
// is even: a thread takes two adjacent rows, so every site moves as one
// 16-byte pair; the rotations and their order are kin_fused's.
template <int L>
__device__ __forceinline__ void kin_pair_odd(double (&v)[L], double (&w)[L], const double *__restrict__ tc,
                                             const double *__restrict__ ts, double fl, int q0, int qs) {
#pragma unroll
  for (int m = 0; m < L / 2; ++m) {
    const int q = q0 + m * qs;
    const double C = tc[q], S = fl * ts[q];
    kin_rot(v[2 * m + 1], v[(2 * m + 2) % L], C, S);
    kin_rot(w[2 * m + 1], w[(2 * m + 2) % L], C, S);
  }
}
template <int L>
__device__ __forceinline__ void kin_pair_even(double (&v)[L], double (&w)[L], const double *__restrict__ tc,
                                              const double *__restrict__ ts, double fl, int q0, int qs) {
#pragma unroll
  for (int m = 0; m < L / 2; ++m) {
    const int q = q0 + m * qs;
    const double C = tc[q], S = fl * ts[q];
    kin_rot(v[2 * m], v[2 * m + 1], C, S);
    kin_rot(w[2 * m], w[2 * m + 1], C, S);
  }
}
template <int L>
__device__ __noinline__ void kin_fused_rowpairs(const Smem &s, double *M, size_t ld, int n, int nflag) {
  constexpr int H = L * L / 2, HL = L / 2;
  const double fl = (double)nflag;
  const double *__restrict__ tc = s.tc;
  const double *__restrict__ ts = s.ts;
  const int n2 = n >> 1, tasks = n2 * L;
  for (int sweep = 0; sweep < 3; ++sweep) {
    for (int t = threadIdx.x; t < tasks; t += Z2_NT) {
      const int i = 2 * (t % n2), line = t / n2;
      double v[L], w[L];
      // sweep 0 and 2: lattice row `line` (sites line L + x); sweep 1:
      // lattice column `line` (sites y L + line)
      const size_t base = (sweep == 1) ? (size_t)line * ld : (size_t)(line * L) * ld;
      const size_t step = (sweep == 1) ? (size_t)L * ld : ld;
      double2 *p = reinterpret_cast<double2 *>(M + i + base);
      const size_t st2 = step >> 1;
#pragma unroll
      for (int x = 0; x < L; ++x) {
        const double2 u = p[(size_t)x * st2];
        v[x] = u.x; w[x] = u.y;
      }
      if (sweep == 0) {
        kin_pair_odd<L>(v, w, tc, ts, fl, line * HL, 1);
        kin_pair_even<L>(v, w, tc, ts, fl, H + line * HL, 1);
      } else if (sweep == 1) {
        kin_pair_odd<L>(v, w, tc, ts, fl, 2 * H + line, L);
        kin_pair_even<L>(v, w, tc, ts, fl, 3 * H + line, L);
        kin_pair_even<L>(v, w, tc, ts, fl, 3 * H + line, L);
        kin_pair_odd<L>(v, w, tc, ts, fl, 2 * H + line, L);
      } else {
        kin_pair_even<L>(v, w, tc, ts, fl, H + line * HL, 1);
        kin_pair_odd<L>(v, w, tc, ts, fl, line * HL, 1);
      }
#pragma unroll
      for (int x = 0; x < L; ++x) p[(size_t)x * st2] = make_double2(v[x], w[x]);
    }
    __syncthreads();
  }
}

// kin_fused for the lattice sizes it is instantiated for; false otherwise.
__device__ __forceinline__ bool kin_fused_any(int L, const Smem &s, double *M, size_t vs, size_t ks,
                                              int n, int nflag) {
  switch (L) {
    case 4: kin_fused<4>(s, M, vs, ks, n, nflag); return true;
    case 6: kin_fused<6>(s, M, vs, ks, n, nflag); return true;
    case 8: kin_fused<8>(s, M, vs, ks, n, nflag); return true;
    case 10: kin_fused<10>(s, M, vs, ks, n, nflag); return true;
    case 12: kin_fused<12>(s, M, vs, ks, n, nflag); return true;
    case 14: kin_fused<14>(s, M, vs, ks, n, nflag); return true;
    case 16: kin_fused<16>(s, M, vs, ks, n, nflag); return true;
    default: return false;
  }
}

__device__ __noinline__ void kin_rows(const ChainDesc &c, const Smem &s, double *M, int ld, int ncols,
                         int nflag) {
  if (kin_fused_any(c.kin_fused, s, M, (size_t)ld, 1, ncols, nflag)) return;
  const int half = c.half;
  const double fl = (double)nflag;
  for (int col = threadIdx.x; col < ncols; col += Z2_NT) {
    double *mc = M + (size_t)col * ld;
    for (int p = 0; p < 8; ++p) kin_group_vec<true>(s, mc, 1, c_gorder[p] * half, half, fl);
  }
  __syncthreads();
}

// M <- M B^nflag : columns P1, P2 rotated (process_group_L); one thread per
// row through all eight passes.
__device__ __noinline__ void kin_cols(const ChainDesc &c, const Smem &s, double *M, int ld, int nrows,
                         int nflag) {
  if ((ld & 1) == 0 && (nrows & 1) == 0 && (reinterpret_cast<size_t>(M) & 15) == 0) {
    switch (c.kin_fused) {
      case 4: kin_fused_rowpairs<4>(s, M, (size_t)ld, nrows, nflag); return;
      case 6: kin_fused_rowpairs<6>(s, M, (size_t)ld, nrows, nflag); return;
      case 8: kin_fused_rowpairs<8>(s, M, (size_t)ld, nrows, nflag); return;
      case 10: kin_fused_rowpairs<10>(s, M, (size_t)ld, nrows, nflag); return;
      case 12: kin_fused_rowpairs<12>(s, M, (size_t)ld, nrows, nflag); return;
      case 14: kin_fused_rowpairs<14>(s, M, (size_t)ld, nrows, nflag); return;
      case 16: kin_fused_rowpairs<16>(s, M, (size_t)ld, nrows, nflag); return;
      default: break;
    }
  }
  if (kin_fused_any(c.kin_fused, s, M, 1, (size_t)ld, nrows, nflag)) return;
  const int half = c.half;
  const double fl = (double)nflag;
  for (int row = threadIdx.x; row < nrows; row += Z2_NT) {
    double *mr = M + row;
    for (int p = 0; p < 8; ++p) kin_group_vec<false>(s, mr, (size_t)ld, c_gorder[p] * half, half, fl);
  }
  __syncthreads();
}

// One group (one factor E_g) of B applied to rows / columns.
__device__ __noinline__ void kin_group_rows(const ChainDesc &c, const Smem &s, double *M, int ld, int ncols,
                               int g, int nflag) {
  const int half = c.half, g0 = g * half;
  const double fl = (double)nflag;
  for (int col = threadIdx.x; col < ncols; col += Z2_NT)
    kin_group_vec<true>(s, M + (size_t)col * ld, 1, g0, half, fl);
  __syncthreads();
}
__device__ __noinline__ void kin_group_cols(const ChainDesc &c, const Smem &s, double *M, int ld, int nrows,
                               int g, int nflag) {
  const int half = c.half, g0 = g * half;
  const double fl = (double)nflag;
  for (int row = threadIdx.x; row < nrows; row += Z2_NT)
    kin_group_vec<false>(s, M + row, (size_t)ld, g0, half, fl);
  __syncthreads();
}

// Apply B-multiplications to a global N x N matrix, staging it through the
// arena when it fits (the arena must be free).
__device__ __noinline__ void kin_global(const ChainDesc &c, const Smem &s, double *M, int row_flag,
                           int col_flag) {
  const int N = c.N;
  if (c.g_in_smem) {
    double *A = s.arena;
    blk_copy(A, c.ldg, M, N, N, N);
    if (row_flag) kin_rows(c, s, A, c.ldg, N, row_flag);
    if (col_flag) kin_cols(c, s, A, c.ldg, N, col_flag);
    blk_copy(M, N, A, c.ldg, N, N);
  } else {
    if (row_flag) kin_rows(c, s, M, N, N, row_flag);
    if (col_flag) kin_cols(c, s, M, N, N, col_flag);
  }
}

// Lazily propagated U factors.  R chain: for nt' = lo..hi, U <- B_nt' U then
// U *= e^{dtau mu} (LocalK_prop_R + propT_R, src/localK.f90:395-396,
// src/multiply.f90:106).  L chain (ULT = UL^T, B symmetric): for nt' = hi
// down to lo, ULT *= e^{dtau mu} then ULT <- B_nt' ULT (propT_L + prop_L,
// src/multiply.f90:91, src/localK.f90:370).
__device__ __noinline__ void apply_pending_R(const ChainDesc &c, const Smem &s, double *A, int lda, int lo,
                                int hi, bool kin) {
  for (int t = lo; t <= hi; ++t) {
    if (kin) {
      build_table(c, s, t);
      kin_rows(c, s, A, lda, c.N, 1);
    }
    if (c.eP != 1.0) blk_scale(A, lda, c.N, c.N, c.eP);
  }
}
__device__ __noinline__ void apply_pending_L(const ChainDesc &c, const Smem &s, double *A, int lda, int lo,
                                int hi) {
  for (int t = hi; t >= lo; --t) {
    if (c.eP != 1.0) blk_scale(A, lda, c.N, c.N, c.eP);
    build_table(c, s, t);
    kin_rows(c, s, A, lda, c.N, 1);
  }
}

// ---------------------------------------------------------------------------
// Stabilization (src/stabilization.f90:42-264)
// ---------------------------------------------------------------------------
// stab_green_big (src/stabilization.f90:202-264): the four blocks of the
// 2N x 2N Green's function.  Inverses of the orthogonal factors (UL UR,
// bigU, UR, UL) are their transposes; VR VL, VR and VL are inverted by LU;
// bigV (triangular) by a triangular solve.  The 2N x 2N QR (UDV_C) is the
// blocked Householder QR, bigU the blocked DORGQR, products DMMA GEMMs.
__device__ __noinline__ void dev_stab_green_big(const Smem &s, int N, const double *UR, const double *DR,
                                   const double *VR, const double *ULT, const double *DL,
                                   const double *VL, double *W0, double *W1, double *W2,
                                   double *W3, double *B0, double *B1, double *B2, double *B3) {
  const int n2 = 2 * N;
  double *tau = s.vec;          // 2N
  double *bigD = s.vec + 2 * N; // 2N
  int *ipiv = s.ivec;
  // invVRVL = (VR VL)^-1  -> W0
  {
    blk_dmma(N, N, N, 1.0, MatRef{VR, 1, N}, false, MatRef{VL, 1, N}, false, 0.0, W0, N);
    blk_inverse_blocked(W0, N, N, W1, N, ipiv, s.red, s.flag, s.tile,
                        s.tile_doubles);
  }
  // invULUR = UR^T UL^T -> W1
  {
    blk_dmma(N, N, N, 1.0, MatRef{UR, N, 1}, false, MatRef{ULT, 1, N}, false, 0.0, W1, N);
  }
  // big matrix
  for (int j = threadIdx.x / 32; j < n2; j += Z2_WARPS)
    for (int i = threadIdx.x & 31; i < n2; i += 32) {
      double v = 0.0;
      if (i < N && j < N) v = W0[i + (size_t)j * N];
      else if (i >= N && j >= N) v = W1[(i - N) + (size_t)(j - N) * N];
      else if (i < N && j == i + N) v = DL[i];
      else if (i >= N && j == i - N) v = -DR[j];
      B0[i + (size_t)j * n2] = v;
    }
  __syncthreads();
  // UDV_C: QR, D = |R_ii|, V = R / D, determinant-sign fix
  blk_geqrf(B0, n2, n2, tau, s.tile, s.tile_doubles, s.vec + 4 * N, 4 * N, s.red);
  blk_copy(B1, n2, B0, n2, n2, n2);
  blk_orgqr(B1, n2, n2, tau, s.tile, s.tile_doubles, s.vec + 4 * N, 4 * N);   // bigU
  {
    // sign of prod R_ii (mat_mod.f90:650-657): count negative diagonals
    int neg = 0;
    for (int i = threadIdx.x; i < n2; i += Z2_NT) neg += (B0[i + (size_t)i * n2] < 0.0);
    double t = blk_sum((double)neg, s.red);
    int flip = ((int)t) & 1;
    for (int i = threadIdx.x; i < n2; i += Z2_NT) bigD[i] = fabs(B0[i + (size_t)i * n2]);
    __syncthreads();
    // bigV = R / D (upper), into B2 ; flip row 0 of V and column 0 of U if needed
    for (int j = threadIdx.x / 32; j < n2; j += Z2_WARPS)
      for (int i = threadIdx.x & 31; i < n2; i += 32) {
        double v = (i <= j) ? B0[i + (size_t)j * n2] : 0.0;
        if (flip && i == 0) v = -v;
        B2[i + (size_t)j * n2] = v / bigD[i];
      }
    if (flip)
      for (int i = threadIdx.x; i < n2; i += Z2_NT) B1[i] = -B1[i];
    __syncthreads();
  }
  // invbigV: solve bigV X = I -> B3
  blk_identity(B3, n2, n2);
  blk_trsm_lun_blocked(B2, n2, n2, B3, n2, n2);
  // invVUR -> W2, invVUL -> W3
  blk_copy(W2, N, VR, N, N, N);
  blk_inverse_blocked(W2, N, N, W0, N, ipiv, s.red, s.flag, s.tile,
                        s.tile_doubles);
  blk_copy(W3, N, VL, N, N, N);
  blk_inverse_blocked(W3, N, N, W0, N, ipiv, s.red, s.flag, s.tile,
                        s.tile_doubles);
  // mat_left = diag(invVUR, invUUL) invbigV -> B0
  {
    blk_dmma(N, n2, N, 1.0, MatRef{W2, 1, N}, false, MatRef{B3, 1, n2}, false, 0.0, B0, n2);
    blk_dmma(N, n2, N, 1.0, MatRef{ULT, 1, N}, false, MatRef{B3 + N, 1, n2}, false, 0.0, B0 + N, n2);
  }
  // mat_right = invbigU diag(invVUL, invUUR) -> B2 ; invbigU = bigU^T
  {
    blk_dmma(n2, N, N, 1.0, MatRef{B1, n2, 1}, false, MatRef{W3, 1, N}, false, 0.0, B2, n2);
    blk_dmma(n2, N, N, 1.0, MatRef{B1 + N, n2, 1}, false, MatRef{UR, N, 1}, false, 0.0,
             B2 + (size_t)N * n2, n2);
  }
  // mat_left(:, nr) /= bigD(nr)
  for (int j = threadIdx.x / 32; j < n2; j += Z2_WARPS) {
    double d = bigD[j];
    for (int i = threadIdx.x & 31; i < n2; i += 32) B0[i + (size_t)j * n2] = B0[i + (size_t)j * n2] / d;
  }
  __syncthreads();
  {
    blk_dmma(n2, n2, n2, 1.0, MatRef{B0, 1, n2}, false, MatRef{B2, 1, n2}, false, 0.0, B3, n2);
  }
}

// Blocks of the 2N x 2N Green's function left in B3 by dev_stab_green_big.
__device__ __noinline__ void green_big_extract(int N, const double *B3, double *G00, double *G0t,
                                  double *Gt0, double *Gtt) {
  const int n2 = 2 * N;
  blk_copy(G00, N, B3, n2, N, N);
  blk_copy(G0t, N, B3 + (size_t)N * n2, n2, N, N);
  blk_copy(Gt0, N, B3 + N, n2, N, N);
  blk_copy(Gtt, N, B3 + N + (size_t)N * n2, n2, N, N);
}

// ---------------------------------------------------------------------------
// Delayed rank-2 updates (LocalK_metro, src/localK.f90:45-173)
// ---------------------------------------------------------------------------
// The delayed-update factors X and Yt (N x k2 each) keep their columns in
// interleaved pairs: element (i, q) sits at (q / 2) 2 ldx + 2 i + q % 2, so
// the two columns an accepted flip adds are one 16-byte word per row (one
// load in the ratio evaluation and in the column phase, one store), and a
// DMMA fragment (rows r + 0..7, columns l + 0..3) still hits 16 distinct
// bank pairs per half-warp for ldx = 4 (mod 16).
__device__ __forceinline__ size_t xy_at(int i, int q, int ldx) {
  return (size_t)(q >> 1) * (2 * ldx) + 2 * i + (q & 1);
}

// G <- G - X Yt^T over the m queued columns (paired layout) when 8 TR and 8 TC
// divide N: each warp owns (8 TR) x (8 TC) blocks of G, loads their old
// values straight into the DMMA accumulators and adds (-X) Yt^T to them in
// chunks of 4 columns, reusing each X fragment TC times and each Yt fragment
// TR times.
template <int TR, int TC>
__device__ __noinline__ void flush_tiles(double *G, int ldg, const double *X, const double *Yt,
                                         int N, int ldx, int m) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lr = lane >> 2, lc = lane & 3;
  const int gr = N / (8 * TR), gcn = N / (8 * TC);
  const int m4 = m & ~3;
  const size_t s4 = (size_t)4 * ldx;
  for (int g = warp; g < gr * gcn; g += Z2_WARPS) {
    const int r0 = (g % gr) * 8 * TR, c0 = (g / gr) * 8 * TC;
    double *cp = G + r0 + lr + (size_t)(c0 + 2 * lc) * ldg;
    double acc[TR][TC][2];
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) acc[a][b][e] = cp[8 * a + (size_t)(8 * b + e) * ldg];
    const double *pa = X + xy_at(r0 + lr, lc, ldx);
    const double *pb = Yt + xy_at(c0 + lr, lc, ldx);
#pragma unroll 2
    for (int l0 = 0; l0 < m4; l0 += 4) {
      double fa[TR], fb[TC];
#pragma unroll
      for (int u = 0; u < TR; ++u) fa[u] = -pa[16 * u];
#pragma unroll
      for (int v = 0; v < TC; ++v) fb[v] = pb[16 * v];
      pa += s4; pb += s4;
#pragma unroll
      for (int u = 0; u < TR; ++u)
#pragma unroll
        for (int v = 0; v < TC; ++v) dmma884(acc[u][v][0], acc[u][v][1], fa[u], fb[v]);
    }
    if (m4 < m) {
      // two trailing columns: lanes lc >= m - m4 feed zeros
      const bool ok = lc < m - m4;
      double fa[TR], fb[TC];
#pragma unroll
      for (int u = 0; u < TR; ++u) fa[u] = ok ? -pa[16 * u] : 0.0;
#pragma unroll
      for (int v = 0; v < TC; ++v) fb[v] = ok ? pb[16 * v] : 0.0;
#pragma unroll
      for (int u = 0; u < TR; ++u)
#pragma unroll
        for (int v = 0; v < TC; ++v) dmma884(acc[u][v][0], acc[u][v][1], fa[u], fb[v]);
    }
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) cp[8 * a + (size_t)(8 * b + e) * ldg] = acc[a][b][e];
  }
  __syncthreads();
}

// The same update for any N: (8 GS) x (8 GS) groups with bounds checks.
template <int GS>
__device__ __noinline__ void flush_generic(double *G, int ldg, const double *X, const double *Yt,
                                           int N, int ldx, int m) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lr = lane >> 2, lc = lane & 3;
  const int gm = (N + 8 * GS - 1) / (8 * GS);
  for (int g = warp; g < gm * gm; g += Z2_WARPS) {
    const int r0 = (g % gm) * 8 * GS, c0 = (g / gm) * 8 * GS;
    double acc[GS][GS][2];
#pragma unroll
    for (int a = 0; a < GS; ++a)
#pragma unroll
      for (int b = 0; b < GS; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int row = r0 + 8 * a + lr, col = c0 + 8 * b + 2 * lc + e;
          acc[a][b][e] = (row < N && col < N) ? G[row + (size_t)col * ldg] : 0.0;
        }
    for (int l0 = 0; l0 < m; l0 += 4) {
      const int l = l0 + lc;
      const bool lk = l < m;
      double fa[GS], fb[GS];
#pragma unroll
      for (int u = 0; u < GS; ++u) {
        const int ra = r0 + 8 * u + lr, cb = c0 + 8 * u + lr;
        fa[u] = (lk && ra < N) ? -X[xy_at(ra, l, ldx)] : 0.0;
        fb[u] = (lk && cb < N) ? Yt[xy_at(cb, l, ldx)] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < GS; ++u)
#pragma unroll
        for (int v = 0; v < GS; ++v) dmma884(acc[u][v][0], acc[u][v][1], fa[u], fb[v]);
    }
#pragma unroll
    for (int a = 0; a < GS; ++a)
#pragma unroll
      for (int b = 0; b < GS; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int row = r0 + 8 * a + lr, col = c0 + 8 * b + 2 * lc + e;
          if (row < N && col < N) G[row + (size_t)col * ldg] = acc[a][b][e];
        }
  }
  __syncthreads();
}

// Tile shapes of the rank-2k flush (z2_options.flush_shape_chain).  Every
// shape forms each element of G from its old value with the same k chunks,
// so they give the same bits; they differ in how the N x N update
// is cut into warp blocks (load balance over the 8 warps against fragment
// reuse).  0 picks by divisibility: 24 x 24 blocks when 24 | N, 16 x 16 when
// 16 | N, else the bounded 16 x 16 groups.
enum {
  FS_DEFAULT = 0, FS_GEN16 = 1, FS_GEN8 = 2, FS_T11 = 3, FS_T22 = 4, FS_T33 = 5, FS_T21 = 6,
  FS_T32 = 7, FS_COUNT = 8
};
__host__ __device__ __forceinline__ bool flush_shape_ok(int shape, int N) {
  switch (shape) {
    case FS_DEFAULT: case FS_GEN16: case FS_GEN8: return true;
    case FS_T11: return N % 8 == 0;
    case FS_T22: case FS_T21: return N % 16 == 0;
    case FS_T33: return N % 24 == 0;
    case FS_T32: return N % 48 == 0;
    default: return false;
  }
}

// G <- G - X Yt^T over the m queued columns: one DMMA rank-m update.
__device__ __forceinline__ void rank_update(double *G, int ldg, const double *X, const double *Yt,
                                            int N, int ldx, int m, int shape = FS_DEFAULT) {
  switch (shape) {
    case FS_GEN16: flush_generic<2>(G, ldg, X, Yt, N, ldx, m); return;
    case FS_GEN8: flush_generic<1>(G, ldg, X, Yt, N, ldx, m); return;
    case FS_T11: flush_tiles<1, 1>(G, ldg, X, Yt, N, ldx, m); return;
    case FS_T22: flush_tiles<2, 2>(G, ldg, X, Yt, N, ldx, m); return;
    case FS_T33: flush_tiles<3, 3>(G, ldg, X, Yt, N, ldx, m); return;
    case FS_T21: flush_tiles<2, 1>(G, ldg, X, Yt, N, ldx, m); return;
    case FS_T32: flush_tiles<3, 2>(G, ldg, X, Yt, N, ldx, m); return;
    default: break;
  }
  if (N % 24 == 0) flush_tiles<3, 3>(G, ldg, X, Yt, N, ldx, m);
  else if (N % 16 == 0) flush_tiles<2, 2>(G, ldg, X, Yt, N, ldx, m);
  else flush_generic<2>(G, ldg, X, Yt, N, ldx, m);
}

// The 2N proposals of one slice (LocalK_prop_L: bonds 2N..1, LocalK_prop_R:
// bonds 1..2N).  Warp 0 evaluates 32 consecutive proposals speculatively
// against the current G = G0 - X Yt^T; all proposals before the first
// accepted one are rejections (G and sigma unchanged), so they are exact.
// One ranf draw per proposal (src/localK.f90:123), advanced in closed form.
// The slice's sigma (and its neighbours in tau), the Delta table and the
// plaquette partners are staged in shared memory; warp 0 keeps the ranf state
// and the acceptance counters in registers for the whole slice.
__device__ __noinline__ void propose_slice(const ChainDesc &c, const Smem &s, int nt,
                                           bool descending, int dir) {
  const int N = c.N, nb = c.nb, k2 = c.k2, Lt = c.Ltrot;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *G = s.G;
  const int ldg = s.ldg;
  double *X = s.X, *Yt = s.Yt;
  const int ldx = s.ldx;
  signed char *sg = c.sigma + (size_t)(nt - 1) * nb;
  const signed char *gprev = c.sigma + (size_t)((nt - 2 + Lt) % Lt) * nb;
  const signed char *gnext = c.sigma + (size_t)(nt % Lt) * nb;
  signed char *sig = s.sig, *sprev = s.sig + nb, *snext = s.sig + 2 * nb;
  double *dl = s.vec;                                 // [2N][2] Delta(1,1), Delta(1,2)
  short *bbs = reinterpret_cast<short *>(s.vec + 2 * nb);   // [2N][6]
  for (int i = threadIdx.x; i < nb; i += Z2_NT) {
    sig[i] = sg[i];
    sprev[i] = gprev[i];
    snext[i] = gnext[i];
    dl[2 * i] = c.dlt[2 * i];
    dl[2 * i + 1] = c.dlt[2 * i + 1];
#pragma unroll
    for (int q = 0; q < 6; ++q) bbs[6 * i + q] = (short)c.bbonds[6 * i + q];
  }
  __syncthreads();
  double *pdat = s.red + 48;      // accepted proposal: Prod(4), D11, D12, det(Prod)
  // column pairs of X and Yt as 16-byte words: pair q / 2 of row i
  const double2 *X2 = reinterpret_cast<const double2 *>(X);
  const double2 *Y2 = reinterpret_cast<const double2 *>(Yt);
  const int *__restrict__ bond = s.bond;
  volatile int *flag = s.flag;
  unsigned int st = 0;
  // 48828125^(lane+1) mod 2^31 in a register: lane L draws the (L+1)-th
  // number of the batch without a divergent constant-memory read
  const unsigned long long ipl = c_ipow[lane + 1];
  long long rpos = 0;
  int den = 0, num = 0;
  if (warp == 0) {
    st = *c.rng;
    if (c.replay) rpos = *c.replay_pos;
  }
  int m = 0, done = 0;
  long long t_eval = 0, t_cols = 0;
  while (done < nb) {
    const long long t0 = ph_now();
    if (warp == 0) {
      const int kk = done + lane;
      const bool valid = kk < nb;
      const int b = valid ? (descending ? nb - 1 - kk : kk) : 0;
      const int p1 = bond[2 * b], p2 = bond[2 * b + 1];
      double g11 = G[p1 + (size_t)p1 * ldg], g12 = G[p1 + (size_t)p2 * ldg];
      double g21 = G[p2 + (size_t)p1 * ldg], g22 = G[p2 + (size_t)p2 * ldg];
      {
        // m is even (two columns per accept): two independent FMA chains
        double h11 = 0.0, h12 = 0.0, h21 = 0.0, h22 = 0.0;
#pragma unroll 2
        for (int q = 0; q < m; q += 2) {
          const size_t o = (size_t)(q >> 1) * ldx;
          const double2 xa = X2[o + p1], xb = X2[o + p2], ya = Y2[o + p1], yb = Y2[o + p2];
          g11 -= xa.x * ya.x; g12 -= xa.x * yb.x; g21 -= xb.x * ya.x; g22 -= xb.x * yb.x;
          h11 += xa.y * ya.y; h12 += xa.y * yb.y; h21 += xb.y * ya.y; h22 += xb.y * yb.y;
        }
        g11 -= h11; g12 -= h12; g21 -= h21; g22 -= h22;
      }
      const double s_old = (double)sig[b];
      const double s_new = -s_old;
      const double D11 = dl[2 * b], D12 = s_new * dl[2 * b + 1];
      // (I - G)_PP, Prod = I + Delta (I - G)_PP, determinant (no FMA
      // contraction: same rounding sequence as the reference)
      const double l11 = __dsub_rn(1.0, g11), l12 = -g12, l21 = -g21, l22 = __dsub_rn(1.0, g22);
      const double m11 = __dadd_rn(__dmul_rn(D11, l11), __dmul_rn(D12, l21));
      const double m12 = __dadd_rn(__dmul_rn(D11, l12), __dmul_rn(D12, l22));
      const double m21 = __dadd_rn(__dmul_rn(D12, l11), __dmul_rn(D11, l21));
      const double m22 = __dadd_rn(__dmul_rn(D12, l12), __dmul_rn(D11, l22));
      const double p11 = __dadd_rn(1.0, m11), p12 = m12, p21 = m21, p22 = __dadd_rn(1.0, m22);
      const double det = __dsub_rn(__dmul_rn(p11, p22), __dmul_rn(p12, p21));
      // boson ratio (src/fields.f90:40-119) from the host table
      const short *bb = bbs + 6 * b;
      const double tmp_old = s_old * sig[bb[0]] * sig[bb[1]] * sig[bb[2]] +
                             s_old * sig[bb[3]] * sig[bb[4]] * sig[bb[5]];
      const int is = (int)(-2.0 * tmp_old + 4.0) >> 2;
      const double tn = s_old * ((double)sprev[b] + (double)snext[b]);
      const int it = (int)(-2.0 * tn + 4.0) >> 2;
      const double ratio = __dmul_rn(__dmul_rn(det, det), c.rb[is * 3 + it]);
      double r;
      if (c.replay && rpos + lane < c.nreplay) r = c.replay[rpos + lane];
      else r = (double)(unsigned int)(((unsigned long long)st * ipl) & 0x7fffffffull) *
               (1.0 / 2147483648.0);
      const bool acc = valid && (fabs(ratio) > r);
      const unsigned ball = __ballot_sync(Z2_FULL, acc);
      const int first = ball ? (__ffs(ball) - 1) : 32;
      const int rem = nb - done;
      const int cnt = (first < 32) ? first + 1 : (rem < 32 ? rem : 32);
      if (lane < cnt && c.dec) {
        const size_t li = ((size_t)dir * Lt + (nt - 1)) * nb + b;
        c.dec[li] = (lane == first) ? 1 : 0;
        if (c.ratios) c.ratios[li] = ratio;
      }
      if (lane == first) {
        // Prod and its determinant; the inverse is formed by the column
        // phase, where the division overlaps the loads of G, X and Yt
        pdat[0] = p11; pdat[1] = p12; pdat[2] = p21; pdat[3] = p22;
        pdat[4] = D11; pdat[5] = D12; pdat[6] = det;
        flag[1] = b;
      }

      st = ranf_adv(st, cnt);
      rpos += cnt;
      den += cnt;
      num += (first < 32) ? 1 : 0;
      __syncwarp();
      if (lane == 0) {
        flag[0] = done + cnt;
        if (first == 32) flag[1] = -1;
      }
    }
    __syncthreads();
    const long long t1 = ph_now();
    t_eval += t1 - t0;
    done = flag[0];
    const int b = flag[1];
    if (b >= 0) {
      const int p1 = bond[2 * b], p2 = bond[2 * b + 1];
      const double idet = 1.0 / pdat[6];
      const double q00 = pdat[3] * idet, q01 = -pdat[1] * idet, q10 = -pdat[2] * idet,
                   q11 = pdat[0] * idet;
      const double D11 = pdat[4], D12 = pdat[5];
      for (int i = threadIdx.x; i < N; i += Z2_NT) {
        double u0 = G[i + (size_t)p1 * ldg], u1 = G[i + (size_t)p2 * ldg];
        double v0 = G[p1 + (size_t)i * ldg], v1 = G[p2 + (size_t)i * ldg];
        {
          // m is even: two independent FMA chains per output
          double w0 = 0.0, w1 = 0.0, z0 = 0.0, z1 = 0.0;
#pragma unroll 2
          for (int q = 0; q < m; q += 2) {
            const size_t o = (size_t)(q >> 1) * ldx;
            const double2 xr = X2[o + i], yr = Y2[o + i];
            const double2 y1 = Y2[o + p1], y2 = Y2[o + p2], x1 = X2[o + p1], x2 = X2[o + p2];
            u0 -= xr.x * y1.x; u1 -= xr.x * y2.x; v0 -= x1.x * yr.x; v1 -= x2.x * yr.x;
            w0 += xr.y * y1.y; w1 += xr.y * y2.y; z0 += x1.y * yr.y; z1 += x2.y * yr.y;
          }
          u0 -= w0; u1 -= w1; v0 -= z0; v1 -= z1;
        }
        // temp = Uhlp * Prodinv ; Vhlp = Delta (I - G)(P, :)
        const size_t om = (size_t)(m >> 1) * ldx + i;
        reinterpret_cast<double2 *>(X)[om] = make_double2(u0 * q00 + u1 * q10, u0 * q01 + u1 * q11);
        double y0 = -D11 * v0 - D12 * v1;
        double y1 = -D12 * v0 - D11 * v1;
        if (i == p1) { y0 += D11; y1 += D12; }
        if (i == p2) { y0 += D12; y1 += D11; }
        reinterpret_cast<double2 *>(Yt)[om] = make_double2(y0, y1);
      }
      if (threadIdx.x == 0) {
        const signed char sn = (signed char)(-sig[b]);
        sig[b] = sn;
        sg[b] = sn;
      }
      __syncthreads();
      t_cols += ph_now() - t1;
      m += 2;
      if (m >= k2) {
        const long long tf = ph_now();
        rank_update(G, ldg, X, Yt, N, ldx, m, c.flush_shape);
        m = 0;
        if (threadIdx.x == 0) c.acc[A_PH0 + PH_FLUSH] += (double)(ph_now() - tf);
      }
    }
  }
  if (m > 0) {
    const long long tf = ph_now();
    rank_update(G, ldg, X, Yt, N, ldx, m, c.flush_shape);
    if (threadIdx.x == 0) c.acc[A_PH0 + PH_FLUSH] += (double)(ph_now() - tf);
  }
  if (threadIdx.x == 0) {
    *c.rng = st;
    if (c.replay) *c.replay_pos = rpos;
    c.acc[A_ACC_DEN] += (double)den;
    c.acc[A_DRAWS] += (double)den;
    c.acc[A_ACC_NUM] += (double)num;
    c.acc[A_PH0 + PH_EVAL] += (double)t_eval;
    c.acc[A_PH0 + PH_COLS] += (double)t_cols;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Equal-time observables (Obs_equal_calc, src/obser_equal.f90:73-149)
// ---------------------------------------------------------------------------
__device__ __noinline__ void obs_equal(const ChainDesc &c, const Smem &s, int nt) {
  const int N = c.N;
  const double *G = s.G; const int ldg = s.ldg;
  const signed char *sg = c.sigma + (size_t)(nt - 1) * c.nb;
  double v[5] = {0, 0, 0, 0, 0};   // flux, pair, cdw, cdw_shift, density
  for (int i = threadIdx.x; i < N; i += Z2_NT) {
    const int *pl = c.plaq + 4 * i;
    v[0] += (double)sg[pl[0]] * (double)sg[pl[1]] * (double)sg[pl[2]] * (double)sg[pl[3]];
    double n = 1.0 - G[i + (size_t)i * ldg];
    v[4] += n + n;
  }
  const int W = 2 * c.Lx - 1;
  // task = (row i, one third of the columns j): the row's density, phase
  // and coordinates stay in registers, the warp's lanes take consecutive
  // rows (G(i, j) contiguous, G(j, i) at the stride ldg, column values
  // broadcast), and no element needs an index division
  const int J3 = (N + 2) / 3;
  for (int t = threadIdx.x; t < 3 * N; t += Z2_NT) {
    const int i = t % N, j0 = (t / N) * J3;
    const int j1 = (j0 + J3 < N) ? j0 + J3 : N;
    const double ni = 1.0 - G[i + (size_t)i * ldg];
    const double sti = c.stag[i];
    const int xi = c.xy[2 * i] + c.Lx - 1, yi = c.xy[2 * i + 1] + c.Ly - 1;
    const double *gi = G + i, *gj = G + (size_t)i * ldg;
#pragma unroll 4
    for (int j = j0; j < j1; ++j) {
      const double gij = gi[(size_t)j * ldg], gji = gj[j];
      const double nj = 1.0 - G[j + (size_t)j * ldg];
      const double dl = (i == j) ? 1.0 : 0.0;
      const double pq = dl - gij;
      v[1] += pq * pq;
      const double a = ni * nj;
      const double ex = (dl - gji) * gij;
      double dc = a - ex;
      dc = (dc + a) - ex;
      dc = (dc + a) + a;
      const double ph = sti * c.stag[j];
      const int dx = xi - c.xy[2 * j], dy = yi - c.xy[2 * j + 1];
      const double ps = c.pshift[dx + dy * W];
      v[2] += ph * dc;
      v[3] += ps * dc;
    }
  }
  blk_sum_n<5>(v, s.red);
  if (threadIdx.x == 0) {
    const double flux = v[0] / (double)N;
    c.acc[A_FLUX_SUM] += flux;
    c.acc[A_FLUX_SQ] += flux * flux;
    c.acc[A_PAIR] += v[1];
    c.acc[A_CDW] += v[2];
    c.acc[A_CDWS] += v[3];
    c.acc[A_DENS] += v[4] / (double)N;
    c.acc[A_NOBS] += 1.0;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Time-displaced observables (Obs_tau_calc, src/obser_tau.f90:56-133), real
// parts, both identical spin sectors summed; binned by imj deterministically
// (one thread per displacement).
// ---------------------------------------------------------------------------
__device__ __noinline__ void obs_tau(const ChainDesc &c, const Smem &s, int nt) {
  const int N = c.N, Lx = c.Lx, Ly = c.Ly;
  const double *G00 = c.G00, *Gtt = c.Gtt, *Gt0 = c.Gt0, *G0t = c.G0t;
  const signed char *sgt = c.sigma + (size_t)(nt - 1) * c.nb;
  const signed char *sg1 = c.sigma;
  const double rt2 = c.rt_scalar * c.rt_scalar;
  for (int r = threadIdx.x; r < N; r += Z2_NT) {
    const int rx = c.xy[2 * r], ry = c.xy[2 * r + 1];
    double o[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int ii = 0; ii < N; ++ii) {
      const int ix = c.xy[2 * ii], iy = c.xy[2 * ii + 1];
      int jx = ix - rx; if (jx < 1) jx += Lx;
      int jy = iy - ry; if (jy < 1) jy += Ly;
      const int jj = (jy - 1) * Lx + (jx - 1);
      const int ip = c.nbx[ii], jp = c.nbx[jj];
      // spin: sigma(ii, ntau) * sigma(jj, 1)
      o[0] += (double)sgt[ii] * (double)sg1[jj];
      const double g0t_ji = G0t[jj + (size_t)ii * N];
      const double gt0_ij = Gt0[ii + (size_t)jj * N];
      // single: term = Grt0u + Grt0d ; += term + conj(term)
      const double term = gt0_ij + gt0_ij;
      o[1] += term + term;
      // pair_d / pair_s: (diag1 + diag2) * 4
      const double d1 = g0t_ji * g0t_ji;
      const double pr = (d1 + d1) * 4.0;
      o[2] += pr;
      o[3] += pr;
      // charge: -Gr0t(jj,ii) Grt0(ii,jj) - conj(...) for both spins
      const double y = g0t_ji * gt0_ij;
      const double tt = 2.0 * (1.0 - Gtt[ii + (size_t)ii * N]);
      const double t0 = 2.0 * (1.0 - G00[jj + (size_t)jj * N]);
      const double chc = ((-y - y) - y) - y;
      o[4] += chc + (tt - tt) * (t0 - t0);
      o[5] += chc + (tt + tt) * (t0 + t0);
      // curxx with NB_field = 0
      const double tc = -G0t[jj + (size_t)ip * N] * Gt0[ii + (size_t)jp * N]
                        - G0t[jp + (size_t)ii * N] * Gt0[ip + (size_t)jj * N]
                        + G0t[jj + (size_t)ii * N] * Gt0[ip + (size_t)jp * N]
                        + G0t[jp + (size_t)ip * N] * Gt0[ii + (size_t)jj * N];
      const double cu = -rt2 * tc - rt2 * tc;
      o[6] += cu + cu;
    }
    double *ot = c.obs_tau + (size_t)(nt - 1) * N + r;
#pragma unroll
    for (int q = 0; q < 7; ++q) ot[(size_t)q * c.Ltrot * N] += o[q];
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Wraps (src/stabilization.f90:374-514)
// ---------------------------------------------------------------------------
struct Pend { int lo, hi; };   // lazily propagated slices, lo > hi = none

// Phase timer: accumulates SM cycles of a phase into the chain's counters.
struct PhTimer {
  const ChainDesc &c;
  int ph;
  long long t0;
  __device__ PhTimer(const ChainDesc &cc, int p) : c(cc), ph(p), t0(ph_now()) {}
  __device__ ~PhTimer() {
    if (threadIdx.x == 0) c.acc[A_PH0 + ph] += (double)(ph_now() - t0);
  }
};

__device__ __forceinline__ double *qr_matrix(const ChainDesc &c, const Smem &s, int &ld) {
  ld = s.ldq;
  return s.Wq;
}

__device__ __noinline__ void spill_G(const ChainDesc &c, const Smem &s) {
  if (c.g_in_smem) blk_copy(c.G, c.N, s.G, s.ldg, c.N, c.N);
}
__device__ __noinline__ void load_G(const ChainDesc &c, const Smem &s) {
  if (c.g_in_smem) blk_copy(s.G, s.ldg, c.G, c.N, c.N, c.N);
}

// The stabilized Green's function Gn replaces the propagated one in one pass
// over both: returns the drift max |Gn - G| (compare_mat,
// src/stabilization.f90:365-372) and leaves G = Gn in global memory and, for
// a chain whose G lives in shared memory, there too.
__device__ __noinline__ double take_green(const ChainDesc &c, const Smem &s, const double *Gn) {
  const int N = c.N, ldg = s.ldg;
  double *Gg = c.G, *Gs = s.G;
  const bool sm = c.g_in_smem != 0;
  double m = 0.0;
  blk_walk<8, double2>(
      N, N, [&](int i, int j) { return make_double2(Gn[i + (size_t)j * N], Gg[i + (size_t)j * N]); },
      [&](double2 v, int i, int j) {
        const double d = fabs(v.x - v.y);
        m = (d > m || d != d) ? d : m;   // keep NaN visible
        Gg[i + (size_t)j * N] = v.x;
        if (sm) Gs[i + (size_t)j * ldg] = v.x;
      });
  const double r = blk_max(m, s.red);
  __syncthreads();
  return r;
}

__device__ __noinline__ void copy_vec(double *dst, const double *src, int n) {
  for (int i = threadIdx.x; i < n; i += Z2_NT) dst[i] = src[i];
  __syncthreads();
}

__device__ __noinline__ void record_drift(const ChainDesc &c, double dif, bool stats) {
  if (threadIdx.x == 0) {
    if (dif > c.acc[A_XMAX] || dif != dif) c.acc[A_XMAX] = dif;
    if (stats) c.acc[A_XMEAN] += dif;
    if (!(dif == dif) || isinf(dif)) atomicOr(c.status, ST_NONFINITE);
  }
}

// The chain's stabilization: the reference's pivoted QR, or the pre-pivoted
// blocked QR (dev_stab_U_fast / dev_stab_green_fast).
__device__ __forceinline__ void chain_stab_U(const ChainDesc &c, const Smem &s, double *A, int lda,
                                             double *U, double *D, double *V, bool left) {
  if (c.stab_exact) dev_stab_U(s, c.N, A, lda, U, D, V, c.W0, left);
  else dev_stab_U_fast(s, c.N, A, lda, U, D, V, c.W0, left);
}
__device__ __forceinline__ void chain_stab_green(const ChainDesc &c, const Smem &s, int nt, double *A,
                                                 int lda, double *Gout) {
  if (c.stab_exact)
    dev_stab_green(s, c.N, nt, c.Ltrot, c.UR, c.DR, c.VR, c.ULT, c.DL, c.VL, A, lda, c.W1, c.W2,
                   c.W0, Gout);
  else
    dev_stab_green_fast(s, c.N, nt, c.Ltrot, c.UR, c.DR, c.VR, c.ULT, c.DL, c.VL, A, lda, c.W1,
                        c.W2, c.W0, Gout);
}

// Wrap_pre (src/stabilization.f90:374-398)
__device__ __noinline__ void wrap_pre(const ChainDesc &c, const Smem &s, int nt, Pend &pd) {
  const int N = c.N, NN = N * N;
  int lda; double *A = qr_matrix(c, s, lda);
  const int st = nt / c.Nwrap;
  if (nt != 0) {
    blk_copy(A, lda, c.UR, N, N, N);
    { PhTimer t(c, PH_PEND); apply_pending_R(c, s, A, lda, pd.lo, pd.hi, c.use_kin != 0); }
    chain_stab_U(c, s, A, lda, c.UR, c.DR, c.VR, false);
  }
  pd.lo = 1; pd.hi = 0;
  { PhTimer t(c, PH_STACK);
    blk_copy(c.URs + (size_t)st * NN, N, c.UR, N, N, N);
    blk_copy(c.VRs + (size_t)st * NN, N, c.VR, N, N, N);
    copy_vec(c.DRs + (size_t)st * N, c.DR, N); }
  if (nt == c.Ltrot) {
    chain_stab_green(c, s, nt, A, lda, c.G);
  }
}

// Wrap_L (src/stabilization.f90:400-437)
__device__ __noinline__ void wrap_L(const ChainDesc &c, const Smem &s, int nt, Pend &pd, bool stats) {
  const int N = c.N, NN = N * N;
  spill_G(c, s);
  int lda; double *A = qr_matrix(c, s, lda);
  const int st = nt / c.Nwrap;
  { PhTimer t(c, PH_STACK);
    blk_copy(c.UR, N, c.URs + (size_t)st * NN, N, N, N);
    blk_copy(c.VR, N, c.VRs + (size_t)st * NN, N, N, N);
    copy_vec(c.DR, c.DRs + (size_t)st * N, N); }
  if (pd.lo <= pd.hi) {
    blk_copy(A, lda, c.ULT, N, N, N);
    { PhTimer t(c, PH_PEND); apply_pending_L(c, s, A, lda, pd.lo, pd.hi); }
    if (nt == c.Ltrot) blk_copy(c.ULT, N, A, lda, N, N);
  } else if (nt != c.Ltrot) {
    blk_copy(A, lda, c.ULT, N, N, N);
  }
  pd.lo = 1; pd.hi = 0;
  if (nt != c.Ltrot) {
    { PhTimer t(c, PH_STABU); chain_stab_U(c, s, A, lda, c.ULT, c.DL, c.VL, true); }
    { PhTimer t(c, PH_STABG); chain_stab_green(c, s, nt, A, lda, c.W3); }
    record_drift(c, take_green(c, s, c.W3), stats);
  }
  { PhTimer t(c, PH_STACK);
    blk_copy(c.ULTs + (size_t)st * NN, N, c.ULT, N, N, N);
    blk_copy(c.VLs + (size_t)st * NN, N, c.VL, N, N, N);
    copy_vec(c.DLs + (size_t)st * N, c.DL, N); }
  if (nt == c.Ltrot) load_G(c, s);   // otherwise take_green reloaded it
}

// Wrap_R (src/stabilization.f90:439-476)
__device__ __noinline__ void wrap_R(const ChainDesc &c, const Smem &s, int nt, Pend &pd, bool stats) {
  const int N = c.N, NN = N * N;
  spill_G(c, s);
  int lda; double *A = qr_matrix(c, s, lda);
  const int st = nt / c.Nwrap;
  { PhTimer t(c, PH_STACK);
    blk_copy(c.ULT, N, c.ULTs + (size_t)st * NN, N, N, N);
    blk_copy(c.VL, N, c.VLs + (size_t)st * NN, N, N, N);
    copy_vec(c.DL, c.DLs + (size_t)st * N, N); }
  if (pd.lo <= pd.hi) {
    blk_copy(A, lda, c.UR, N, N, N);
    { PhTimer t(c, PH_PEND); apply_pending_R(c, s, A, lda, pd.lo, pd.hi, true); }
    if (nt == 0) blk_copy(c.UR, N, A, lda, N, N);
  } else if (nt != 0) {
    blk_copy(A, lda, c.UR, N, N, N);
  }
  pd.lo = 1; pd.hi = 0;
  if (nt != 0) {
    { PhTimer t(c, PH_STABU); chain_stab_U(c, s, A, lda, c.UR, c.DR, c.VR, false); }
    { PhTimer t(c, PH_STABG); chain_stab_green(c, s, nt, A, lda, c.W3); }
    record_drift(c, take_green(c, s, c.W3), stats);
  }
  { PhTimer t(c, PH_STACK);
    blk_copy(c.URs + (size_t)st * NN, N, c.UR, N, N, N);
    blk_copy(c.VRs + (size_t)st * NN, N, c.VR, N, N, N);
    copy_vec(c.DRs + (size_t)st * N, c.DR, N); }
  if (nt == 0) load_G(c, s);   // otherwise take_green reloaded it
}

