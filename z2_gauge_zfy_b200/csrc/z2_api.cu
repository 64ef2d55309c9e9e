// z2_api.cu -- kernels and the C ABI (include/z2dqmc.h) of the B200 DQMC
// library.  Build: nvcc -gencode arch=compute_100a,code=sm_100a -O3 -shared.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <string>
#include <vector>

#include "../../include/z2dqmc.h"
#include "z2_drivers.cuh"

static_assert(PH_COUNT == Z2_NPHASE, "phase counters and the C ABI disagree");

enum { OP_PRE = 1, OP_SWEEP = 2, OP_LOGDET = 3, OP_GLOBAL = 4, OP_THERM = 5 };
enum { U_MMULT_R = 1, U_MMULT_L, U_STAB_UR, U_STAB_UL, U_STAB_GREEN, U_STAB_GREEN_BIG };

struct UnitArgs {
  double *M;                      // mmult: in/out
  double *U, *D, *V;              // stab_U: in/out (U = UR or UL^T)
  const double *UR, *DR, *VR, *ULT, *DL, *VL;
  double *G, *G0t, *Gt0, *Gtt;    // outputs
  int nt, nflag;
};

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_desc(ChainDesc &sc, const ChainDesc *g) {
  const long long *src = (const long long *)g;
  long long *dst = (long long *)&sc;
  for (int i = threadIdx.x; i < (int)(sizeof(ChainDesc) / 8); i += Z2_NT) dst[i] = src[i];
  __syncthreads();
}

// Persistent launch: every CTA pulls chains from a work queue (ordered by
// decreasing cost) and runs the whole operation of that chain.
__global__ void __launch_bounds__(Z2_NT, 1)
z2_chain_kernel(const ChainDesc *descs, const int *order, int nchains, int *queue, int op,
                int nsweep, int toggle, unsigned smem_bytes) {
  extern __shared__ __align__(16) unsigned char z2_smem[];
  __shared__ ChainDesc sc;
  __shared__ Smem s;     // pointer table in shared memory, not on the local stack
  __shared__ int s_idx;
  for (;;) {
    if (threadIdx.x == 0) s_idx = atomicAdd(queue, 1);
    __syncthreads();
    const int idx = s_idx;
    if (idx >= nchains) break;
    load_desc(sc, descs + order[idx]);
    if (threadIdx.x == 0) s = make_smem(sc, z2_smem, smem_bytes);
    __syncthreads();
    if (op == OP_PRE) {
      for (int i = threadIdx.x; i < 2 * sc.nb; i += Z2_NT) s.bond[i] = sc.bonds[i];
      __syncthreads();
      chain_pre(sc, s);
    } else if (op == OP_SWEEP) {
      chain_sweep(sc, s, nsweep, toggle != 0, sc.hzero ? 1.0 : 0.0);
    } else if (op == OP_LOGDET) {
      chain_logdet_grad(sc, s);
    } else if (op == OP_GLOBAL) {
      chain_global(sc, s, nsweep);
    } else if (op == OP_THERM) {
      chain_therm(sc, s, nsweep);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(Z2_NT, 1)
z2_state_kernel(const ChainDesc *desc, int op, int nt, int flag, double x, unsigned smem_bytes);

// Module-level mirrors on single matrices, one CTA.
__global__ void __launch_bounds__(Z2_NT, 1)
z2_unit_kernel(const ChainDesc *desc, int op, UnitArgs a, unsigned smem_bytes) {
  extern __shared__ __align__(16) unsigned char z2_smem[];
  __shared__ ChainDesc sc;
  __shared__ Smem s;
  load_desc(sc, desc);
  if (threadIdx.x == 0) s = make_smem(sc, z2_smem, smem_bytes);
  __syncthreads();
  const int N = sc.N;
  if (op == U_MMULT_R || op == U_MMULT_L) {
    build_table(sc, s, a.nt);
    if (op == U_MMULT_R) kin_global(sc, s, a.M, a.nflag, 0);
    else kin_global(sc, s, a.M, 0, a.nflag);
  } else if (op == U_STAB_UR || op == U_STAB_UL) {
    int lda; double *A = qr_matrix(sc, s, lda);
    blk_copy(A, lda, a.U, N, N, N);
    dev_stab_U(s, N, A, lda, a.U, a.D, a.V, sc.W0, op == U_STAB_UL);
  } else if (op == U_STAB_GREEN) {
    int lda; double *A = qr_matrix(sc, s, lda);
    dev_stab_green(s, N, a.nt, sc.Ltrot, a.UR, a.DR, a.VR, a.ULT, a.DL, a.VL, A, lda, sc.W1,
                   sc.W2, sc.W0, a.G);
  } else if (op == U_STAB_GREEN_BIG) {
    dev_stab_green_big(s, N, a.UR, a.DR, a.VR, a.ULT, a.DL, a.VL, sc.W0, sc.W1, sc.W2, sc.W3,
                       sc.B0, sc.B1, sc.B2, sc.B3);
    green_big_extract(N, sc.B3, a.G, a.G0t, a.Gt0, a.Gtt);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace {

const double kZero = 1.0e-10;      // src/calc_basic.f90:5
const double kUpbound = 1.0e200;   // src/calc_basic.f90:7
const int kSmemMax = 227 * 1024 - 2048;
const int kGemmTile = Z2_MIN_TILE;

int npbc(int nr, int L) { return nr < 1 ? nr + L : (nr > L ? nr - L : nr); }

// ranf (lib/package_of_matrix/Ran/ran_imada.f:55-68): iq*IP mod 2^31.
double ranf_host(uint32_t &iq) {
  iq = (uint32_t)(((uint64_t)iq * 48828125ull) & 0x7fffffffull);
  return (double)iq / 2147483648.0;
}
uint32_t fold_seed(int32_t seed) {
  // a negative Fortran seed behaves like seed mod 2^31 after the first draw;
  // keep the 32-bit pattern and let ranf_host reduce it.
  return (uint32_t)seed;
}

struct HostLattice {
  int Lx, Ly, N;
  std::vector<int> bonds, groups, bbonds, plaq, xy, nbx;
  std::vector<int> inv_n, inv_bond;
  bool ok = true;
  HostLattice(int lx, int ly) : Lx(lx), Ly(ly), N(lx * ly) {
    // n_list / bond_list (src/lattice.f90:31-60)
    inv_n.assign((Lx + 1) * (Ly + 1), 0);
    xy.assign(2 * N, 0);
    for (int ny = 1, nc = 0; ny <= Ly; ++ny)
      for (int nx = 1; nx <= Lx; ++nx, ++nc) { xy[2 * nc] = nx; xy[2 * nc + 1] = ny; inv_n[nx + ny * (Lx + 1)] = nc; }
    auto site = [&](int x, int y) { return inv_n[x + y * (Lx + 1)]; };
    bonds.assign(4 * N, 0);
    inv_bond.assign(N * N, -1);
    for (int ny = 1, nc = 0; ny <= Ly; ++ny)
      for (int nx = 1; nx <= Lx; ++nx) {
        int ii = site(nx, ny);
        int ix = site(npbc(nx + 1, Lx), ny);
        bonds[2 * nc] = ii; bonds[2 * nc + 1] = ix; inv_bond[ii * N + ix] = nc; ++nc;
        int iy = site(nx, npbc(ny + 1, Ly));
        bonds[2 * nc] = ii; bonds[2 * nc + 1] = iy; inv_bond[ii * N + iy] = nc; ++nc;
      }
    // checkerboard groups (src/lattice.f90:72-102)
    std::vector<int> g[4];
    for (int nc = 0; nc < 2 * N; ++nc) {
      int ii = bonds[2 * nc], jj = bonds[2 * nc + 1];
      int ixc = xy[2 * ii], iyc = xy[2 * ii + 1], jxc = xy[2 * jj], jyc = xy[2 * jj + 1];
      if (npbc(ixc + 1, Lx) == jxc) g[(ixc % 2 == 0) ? 0 : 1].push_back(nc);
      else if (npbc(iyc + 1, Ly) == jyc) g[(iyc % 2 == 0) ? 2 : 3].push_back(nc);
    }
    for (int q = 0; q < 4; ++q) {
      if ((int)g[q].size() != N / 2) ok = false;
      groups.insert(groups.end(), g[q].begin(), g[q].end());
    }
    // plaquette partners (src/lattice.f90:104-141)
    bbonds.assign(6 * 2 * N, 0);
    auto ib = [&](int a, int b) { return inv_bond[a * N + b]; };
    for (int nc = 0; nc < 2 * N; ++nc) {
      int ii = bonds[2 * nc], jj = bonds[2 * nc + 1];
      int ixc = xy[2 * ii], iyc = xy[2 * ii + 1], jxc = xy[2 * jj], jyc = xy[2 * jj + 1];
      int *o = &bbonds[6 * nc];
      if (npbc(ixc + 1, Lx) == jxc) {
        int nx = site(ixc, npbc(iyc + 1, Ly)); o[0] = ib(ii, nx);
        int ny = site(jxc, npbc(jyc + 1, Ly)); o[1] = ib(nx, ny); o[2] = ib(jj, ny);
        nx = site(ixc, npbc(iyc - 1, Ly)); o[3] = ib(nx, ii);
        ny = site(jxc, npbc(jyc - 1, Ly)); o[4] = ib(nx, ny); o[5] = ib(ny, jj);
      } else {
        int nx = site(npbc(jxc - 1, Lx), jyc); o[0] = ib(nx, jj);
        int ny = site(npbc(ixc - 1, Lx), iyc); o[1] = ib(ny, nx); o[2] = ib(ny, ii);
        nx = site(npbc(jxc + 1, Lx), jyc); o[3] = ib(jj, nx);
        ny = site(npbc(ixc + 1, Lx), iyc); o[4] = ib(ny, nx); o[5] = ib(ii, ny);
      }
    }
    // plaquettes of Obs_equal_calc (src/obser_equal.f90:84-96), +x neighbours
    plaq.assign(4 * N, 0);
    nbx.assign(N, 0);
    for (int s = 0; s < N; ++s) {
      int x = xy[2 * s], y = xy[2 * s + 1];
      int right = site(npbc(x + 1, Lx), y), up = site(x, npbc(y + 1, Ly));
      int diag = site(npbc(xy[2 * up] + 1, Lx), xy[2 * up + 1]);
      int rup = site(xy[2 * right], npbc(xy[2 * right + 1] + 1, Ly));
      plaq[4 * s] = ib(s, right); plaq[4 * s + 1] = ib(right, rup);
      plaq[4 * s + 2] = ib(up, diag); plaq[4 * s + 3] = ib(s, up);
      nbx[s] = right;
    }
  }
};

// L when the checkerboard table of an L x L lattice has the layout the fused
// kinetic kernels assume (group 0/1: x bonds from odd/even x, slot
// y L/2 + m; group 2/3: y bonds from odd/even y, slot m L + x; bond
// orientation (site, next site)), else 0.
int kin_fused_size(const HostLattice &lat) {
  const int L = lat.Lx;
  if (lat.Ly != L || L % 2 != 0 || L < 4 || L > 16 || !lat.ok) return 0;
  const int H = L * L / 2, HL = L / 2;
  auto check = [&](int g, int slot, int a, int b) {
    const int bd = lat.groups[g * H + slot];
    return lat.bonds[2 * bd] == a && lat.bonds[2 * bd + 1] == b;
  };
  for (int y = 0; y < L; ++y)
    for (int m = 0; m < HL; ++m) {
      const int xo = 2 * m + 1, xe = 2 * m;
      if (!check(0, y * HL + m, y * L + xo, y * L + (xo + 1) % L)) return 0;
      if (!check(1, y * HL + m, y * L + xe, y * L + xe + 1)) return 0;
    }
  for (int m = 0; m < HL; ++m)
    for (int x = 0; x < L; ++x) {
      const int yo = 2 * m + 1, ye = 2 * m;
      if (!check(2, m * L + x, yo * L + x, ((yo + 1) % L) * L + x)) return 0;
      if (!check(3, m * L + x, ye * L + x, (ye + 1) * L + x)) return 0;
    }
  return L;
}

struct ChainHost {
  z2_chain_params p;
  int N, Ltrot, Nst, nb;
  double dtau;
  std::vector<double> rt;
  std::vector<signed char> sigma0;   // initial configuration
  uint32_t iseed0;
  ChainDesc d;                       // with device pointers
  size_t bytes = 0;
  char *base = nullptr;              // device allocation of this chain
  double *replay = nullptr;
  double *ktab = nullptr;            // [2][N][N] cos, sin of k.r (tau chains only)
  double *kout = nullptr;            // [2][7][Ltrot][N] k-space correlators
  char *gbase = nullptr;             // global-move backup block
};

}  // namespace

struct z2_handle {
  std::string err;
  int device = 0;
  int nchains = 0;
  z2_options opt{};
  std::vector<ChainHost> ch;
  ChainDesc *d_desc = nullptr;
  int *d_order = nullptr;
  int *d_queue = nullptr;
  unsigned smem = 0;
  int grid = 1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool pre_done = false;
  // unit-op scratch
  double *u_buf = nullptr;
  // per-chain status flags in one array (one readback per launch)
  int *d_status = nullptr;
  std::vector<int> h_status;
  double *d_obs_all = nullptr;   // [nchains][7] gathered bin observables
  // CUDA graphs of the bin launch, keyed by (nsweep, toggle)
  struct GraphEntry { int nsweep, toggle; cudaGraphExec_t exec; };
  std::vector<GraphEntry> graphs;
  size_t u_n = 0;
};

static int set_err(z2_handle *h, int code, const char *fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->err = buf;
  }
  return code;
}
#define CUDA_TRY(h, x)                                                               \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess)                                                           \
      return set_err(h, Z2_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_));   \
  } while (0)

// conf_set + conf_transfer for a fresh start (src/fields.f90:311-427, 429-507)
// with the thermalisation lattice equal to the run lattice.
static void conf_set_host(const z2_chain_params &p, int N, int Ltrot, std::vector<signed char> &sig,
                          uint32_t &iq) {
  const int nb = 2 * N;
  sig.assign((size_t)nb * Ltrot, 1);
  iq = fold_seed(p.seed);
  if (p.absolute == 1) {
    for (int nt = 0; nt < Ltrot; ++nt)
      for (int b = 0; b < nb; ++b) sig[(size_t)nt * nb + b] = ranf_host(iq) >= 0.5 ? 1 : -1;
  } else if (p.absolute == 2) {
    for (int nt = 0; nt < Ltrot; ++nt)
      for (int b = 0; b < nb; ++b) {
        double x1 = ranf_host(iq), x2 = ranf_host(iq);
        double x = std::sqrt(-2.0 * std::log(x1)) * std::cos(2.0 * M_PI * x2);
        sig[(size_t)nt * nb + b] = x >= 0.0 ? 1 : -1;
      }
  } else if (p.absolute == 3) {
    // all +1
  } else if (p.absolute == 4) {
    for (int nt = 0; nt < Ltrot; ++nt)
      for (int b = 0; b < nb; ++b) {
        int s = b / 2, nx = s % p.Nlx + 1, ny = s / p.Nlx + 1;
        sig[(size_t)nt * nb + b] = ((nx + ny) % 2 == 0) ? 1 : -1;
      }
  } else if (p.absolute == 5) {
    for (int b = 0; b < nb; ++b) {
      signed char v = ranf_host(iq) >= 0.5 ? 1 : -1;
      for (int nt = 0; nt < Ltrot; ++nt) sig[(size_t)nt * nb + b] = v;
    }
  }
  // lambda_random_fill: N draws (the lambda field is not on the hot path)
  for (int i = 0; i < N; ++i) ranf_host(iq);
}

static size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

static int smem_small_bytes(int N) {
  size_t off = 0;
  auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
  off += 8 * Z2_NRED; off += 8 * 8 * N; off += 8 * 2 * N; off += 8 * 2 * N;
  off += a16(4 * 2 * N); off += a16(4 * 4 * N); off += a16(4 * 4 * N); off += 4 * 16;
  off += a16(6 * N);
  return (int)a16(off);
}

// Shared work space (doubles) a chain keeps after G and the delayed-update
// factors: the GEMM staging minimum, the pre-pivoted QR's 64-column chunks,
// and the blocked DORGQR with its parallel T prologue.
static size_t tile_min(int N) {
  const int ldv = qrf_ldv(N);
  size_t t = kGemmTile;
  t = std::max<size_t>(t, qrf_min_work(N));
  t = std::max<size_t>(t, (size_t)ldv * 16 + 17 * (size_t)std::max(N - 16, 0));
  t = std::max<size_t>(t, (size_t)Z2_WARPS * (2 * 16 * 16 + 4 * 16));
  return t;
}

static int default_k(int N) {
  if (N <= 36) return 16;
  if (N <= 64) return 16;
  if (N <= 100) return 12;
  return 8;
}

extern "C" int z2_create(z2_handle **out, const z2_chain_params *params, int32_t nchains,
                         const z2_options *opt) {
  if (!out || !params || nchains <= 0) return Z2_ERR_ARG;
  z2_handle *h = new z2_handle();
  *out = h;
  h->nchains = nchains;
  if (opt) h->opt = *opt;
  h->device = h->opt.device;
  // argument checks first (the reference stops on these, src/calc_basic.f90:96-100,
  // src/fields.f90:422-424), before any CUDA call
  for (int c = 0; c < nchains; ++c) {
    const z2_chain_params &p = params[c];
    if (p.Nlx < 2 || p.Nly < 2 || (p.Nlx % 2) || (p.Nly % 2))
      return set_err(h, Z2_ERR_ARG, "chain %d: Nlx, Nly must be even and >= 2", c);
    if (p.Ltrot < 1 || p.Nwrap < 1 || p.Ltrot % p.Nwrap)
      return set_err(h, Z2_ERR_ARG, "chain %d: Ltrot must be a multiple of Nwrap", c);
    if (p.absolute < 1 || p.absolute > 5)
      return set_err(h, Z2_ERR_ARG, "chain %d: incorrect absolute input %d", c, p.absolute);
    if (!(p.beta > 0.0)) return set_err(h, Z2_ERR_ARG, "chain %d: beta must be positive", c);
    if (p.Nlx * p.Nly > 1024)
      return set_err(h, Z2_ERR_ARG, "chain %d: N = %d exceeds 1024", c, p.Nlx * p.Nly);
    if (h->opt.flush_shape_chain && !flush_shape_ok(h->opt.flush_shape_chain[c], p.Nlx * p.Nly))
      return set_err(h, Z2_ERR_ARG, "chain %d: flush shape %d does not fit N = %d", c,
                     h->opt.flush_shape_chain[c], p.Nlx * p.Nly);
  }
  CUDA_TRY(h, cudaSetDevice(h->device));
  // ranf multiplier powers
  {
    unsigned int pw[33];
    uint64_t v = 1;
    for (int i = 0; i <= 32; ++i) { pw[i] = (unsigned)v; v = (v * 48828125ull) & 0x7fffffffull; }
    CUDA_TRY(h, cudaMemcpyToSymbol(c_ipow, pw, sizeof(pw)));
  }
  h->ch.resize(nchains);
  int smem_needed = 0;
  for (int c = 0; c < nchains; ++c) {
    ChainHost &C = h->ch[c];
    C.p = params[c];
    const z2_chain_params &p = C.p;
    if (p.Nlx < 2 || p.Nly < 2 || (p.Nlx % 2) || (p.Nly % 2))
      return set_err(h, Z2_ERR_ARG, "chain %d: Nlx, Nly must be even and >= 2", c);
    if (p.Ltrot < 1 || p.Nwrap < 1 || p.Ltrot % p.Nwrap)
      return set_err(h, Z2_ERR_ARG, "chain %d: Ltrot must be a multiple of Nwrap", c);
    if (p.absolute < 1 || p.absolute > 5)
      return set_err(h, Z2_ERR_ARG, "chain %d: incorrect absolute input %d", c, p.absolute);
    C.N = p.Nlx * p.Nly;
    if (C.N > 1024) return set_err(h, Z2_ERR_ARG, "chain %d: N = %d exceeds 1024", c, C.N);
    C.Ltrot = p.Ltrot;
    C.Nst = p.Ltrot / p.Nwrap;
    C.nb = 2 * C.N;
    C.dtau = p.beta / (double)p.Ltrot;
    C.rt.assign(C.nb, p.RT);
    if (p.rt_bond) for (int b = 0; b < C.nb; ++b) C.rt[b] = p.rt_bond[b];
    conf_set_host(p, C.N, C.Ltrot, C.sigma0, C.iseed0);
    // shared-memory plan
    const int N = C.N;
    // leading dimension of G and the QR work matrix in shared memory: N + 2
    // (= 2 mod 4) when 4 divides N, so the flush's accumulator fragments hit
    // distinct banks and the checkerboard sweeps move 16-byte pairs; odd
    // otherwise (conflict-free strided rows)
    const int ldg = (N % 4 == 0) ? N + 2 : ((N % 2) ? N : N + 1);
    int small = smem_small_bytes(N);
    int k = h->opt.delay_k > 0 ? h->opt.delay_k : default_k(N);
    if (h->opt.delay_k_chain && h->opt.delay_k_chain[c] > 0) k = h->opt.delay_k_chain[c];
    if (k > 64) k = 64;
    size_t arena = (size_t)(kSmemMax - small) / 8;
    size_t nn = (size_t)N * ldg;
    int g_in = 0;
    int k2 = 2 * k;
    const size_t tmin = tile_min(N);
    if (nn + std::max<size_t>(2 * (size_t)z2_ldx(N) * k2, tmin) <= arena) g_in = 1;
    else if (nn + std::max<size_t>(2 * (size_t)z2_ldx(N) * 4, tmin) <= arena) {
      g_in = 1;
      while (k2 > 4 && nn + 2 * (size_t)z2_ldx(N) * k2 > arena) k2 -= 2;
    }
    if (!g_in) {
      while (k2 > 2 && 2 * (size_t)z2_ldx(N) * k2 > arena) k2 -= 2;
    }
    size_t need = small + 8 * (g_in ? nn + std::max<size_t>(2 * (size_t)z2_ldx(N) * k2, tmin)
                                    : std::max<size_t>(2 * (size_t)z2_ldx(N) * k2, tmin));
    smem_needed = std::max(smem_needed, (int)need);
    C.d = ChainDesc{};
    C.d.N = N; C.d.Lx = p.Nlx; C.d.Ly = p.Nly; C.d.Ltrot = p.Ltrot; C.d.Nwrap = p.Nwrap;
    C.d.Nst = C.Nst; C.d.nb = C.nb; C.d.half = N / 2; C.d.ldg = ldg; C.d.k2 = k2;
    C.d.g_in_smem = g_in;
  }
  // the launch uses one dynamic smem size; chains planned for a larger
  // arena still fit because the plan used the maximum.
  h->smem = (unsigned)std::max(smem_needed, 4096);
  if ((int)h->smem > kSmemMax) h->smem = kSmemMax;
  // re-plan with the final arena: G in smem only if it fits h->smem
  for (auto &C : h->ch) {
    const int N = C.N;
    size_t arena = (h->smem - smem_small_bytes(N)) / 8;
    size_t nn = (size_t)N * C.d.ldg;
    if (C.d.g_in_smem && nn + std::max<size_t>(2 * (size_t)z2_ldx(N) * C.d.k2, tile_min(N)) > arena)
      C.d.g_in_smem = 0;
  }
  CUDA_TRY(h, cudaFuncSetAttribute(z2_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)h->smem));
  CUDA_TRY(h, cudaFuncSetAttribute(z2_unit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)h->smem));
  CUDA_TRY(h, cudaFuncSetAttribute(z2_state_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)h->smem));
  CUDA_TRY(h, cudaMalloc(&h->d_status, sizeof(int) * nchains));
  CUDA_TRY(h, cudaMemset(h->d_status, 0, sizeof(int) * nchains));
  h->h_status.assign(nchains, 0);
  // device memory and tables
  for (int c = 0; c < nchains; ++c) {
    ChainHost &C = h->ch[c];
    const z2_chain_params &p = C.p;
    const int N = C.N, nb = C.nb, Lt = C.Ltrot, Nst = C.Nst;
    HostLattice lat(p.Nlx, p.Nly);
    if (!lat.ok) return set_err(h, Z2_ERR_ARG, "chain %d: checkerboard groups not of size N/2", c);
    const size_t NN = (size_t)N * N;
    std::vector<double> chsh(2 * nb), dlt(2 * nb), stag(N);
    for (int b = 0; b < nb; ++b) {
      double alpha = 0.5 * C.dtau * C.rt[b];      // opK_set (src/operator_kin.f90:26)
      chsh[2 * b] = std::cosh(alpha);
      chsh[2 * b + 1] = std::sinh(alpha);
      double a2 = C.dtau * C.rt[b];               // opK_get_delta (src/operator_kin.f90:40-59)
      double c_new = std::cosh(a2 * 1.0), c_old = std::cosh(a2 * -1.0);
      double s_new = std::sinh(a2 * 1.0), s_old = std::sinh(a2 * -1.0);
      dlt[2 * b] = c_new * c_old - s_new * s_old - 1.0;
      dlt[2 * b + 1] = s_new * c_old - c_new * s_old;
    }
    for (int s = 0; s < N; ++s) stag[s] = ((lat.xy[2 * s] + lat.xy[2 * s + 1]) % 2 == 0) ? 1.0 : -1.0;
    const int W = 2 * p.Nlx - 1, H = 2 * p.Nly - 1;
    std::vector<double> psh((size_t)W * H);
    const double PI = std::acos(-1.0);
    const double qx = PI - 2.0 * PI / (double)p.Nlx;
    for (int dy = -(p.Nly - 1); dy <= p.Nly - 1; ++dy)
      for (int dx = -(p.Nlx - 1); dx <= p.Nlx - 1; ++dx)
        psh[(dx + p.Nlx - 1) + (size_t)(dy + p.Nly - 1) * W] = std::cos(qx * (double)dx + PI * (double)dy);
    // boson ratio table (src/fields.f90:52-117)
    double rb[9];
    {
      const double alpha = C.dtau * p.J;
      double gamma = 0.0; bool temporal = false;
      if (std::fabs(p.h) > kZero) {
        double ta = std::tanh(C.dtau * p.h);
        if (ta < 1.0e-300) ta = 1.0e-300;
        gamma = -0.5 * std::log(ta);
        temporal = true;
      }
      const double lub = std::log(kUpbound);
      for (int is = 0; is < 3; ++is)
        for (int it = 0; it < 3; ++it) {
          double ds = 4.0 * is - 4.0, dt = 4.0 * it - 4.0;
          double e = alpha * ds;
          e = std::min(std::max(e, -lub), lub);
          double r = std::exp(e);
          if (temporal) {
            double e2 = gamma * dt;
            e2 = std::min(std::max(e2, -lub), lub);
            r = r * std::exp(e2);
          }
          rb[is * 3 + it] = r;
        }
    }
    // layout of this chain's device block
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += al256(bytes); return o; };
    size_t o_bonds = take(4 * lat.bonds.size()), o_groups = take(4 * lat.groups.size());
    size_t o_bb = take(4 * lat.bbonds.size()), o_plaq = take(4 * lat.plaq.size());
    size_t o_xy = take(4 * lat.xy.size()), o_nbx = take(4 * lat.nbx.size());
    size_t o_chsh = take(8 * chsh.size()), o_dlt = take(8 * dlt.size());
    size_t o_stag = take(8 * stag.size()), o_psh = take(8 * psh.size());
    size_t o_sigma = take((size_t)nb * Lt);
    size_t o_mat = take(8 * NN * 10);             // G, UR, VR, ULT, VL, W0..W4
    size_t o_vec = take(8 * (size_t)N * 2);       // DR, DL
    size_t o_stk = take(8 * NN * 4 * (Nst + 1));  // URs, VRs, ULTs, VLs
    size_t o_stv = take(8 * (size_t)N * 2 * (Nst + 1));
    size_t o_tau = take(8 * NN * 8);              // G00, Gtt, Gt0, G0t, URd, VRd, ULTd, VLd
    size_t o_tauv = take(8 * (size_t)N * 2);      // DRd, DLd
    size_t o_big = take(8 * NN * 16);             // B0..B3 (2N x 2N)
    size_t o_otau = take(8 * (size_t)7 * Lt * N);
    size_t o_grad = take(8 * (size_t)nb);
    size_t o_acc = take(8 * A_COUNT);
    size_t o_misc = take(64);                     // rng, replay_pos, status
    size_t o_ktab = 0, o_kout = 0;
    if (h->opt.tau) { o_ktab = take(8 * NN * 2); o_kout = take(8 * (size_t)14 * Lt * N); }
    size_t o_dec = 0, o_rat = 0;
    if (h->opt.record) { o_dec = take((size_t)2 * Lt * nb); o_rat = take(8 * (size_t)2 * Lt * nb); }
    C.bytes = off;
    char *base = nullptr;
    if (cudaMalloc(&base, C.bytes) != cudaSuccess)
      return set_err(h, Z2_ERR_NOMEM, "chain %d: cudaMalloc of %zu bytes failed", c, C.bytes);
    C.base = base;
    CUDA_TRY(h, cudaMemset(base, 0, C.bytes));
    auto up = [&](size_t o, const void *src, size_t bytes) {
      return cudaMemcpy(base + o, src, bytes, cudaMemcpyHostToDevice);
    };
    CUDA_TRY(h, up(o_bonds, lat.bonds.data(), 4 * lat.bonds.size()));
    CUDA_TRY(h, up(o_groups, lat.groups.data(), 4 * lat.groups.size()));
    CUDA_TRY(h, up(o_bb, lat.bbonds.data(), 4 * lat.bbonds.size()));
    CUDA_TRY(h, up(o_plaq, lat.plaq.data(), 4 * lat.plaq.size()));
    CUDA_TRY(h, up(o_xy, lat.xy.data(), 4 * lat.xy.size()));
    CUDA_TRY(h, up(o_nbx, lat.nbx.data(), 4 * lat.nbx.size()));
    CUDA_TRY(h, up(o_chsh, chsh.data(), 8 * chsh.size()));
    CUDA_TRY(h, up(o_dlt, dlt.data(), 8 * dlt.size()));
    CUDA_TRY(h, up(o_stag, stag.data(), 8 * stag.size()));
    CUDA_TRY(h, up(o_psh, psh.data(), 8 * psh.size()));
    CUDA_TRY(h, up(o_sigma, C.sigma0.data(), C.sigma0.size()));
    if (h->opt.tau) {
      // exp(i k.r) of Fourier_R_to_K (src/lattice.f90:159-173, 263-281):
      // k = ((ix-1) 2pi/Nlx, (iy-1) 2pi/Nly), r = (ix, iy) 1-based
      std::vector<double> kt(2 * NN);
      const double PI2 = 2.0 * std::acos(-1.0);
      for (int r = 0; r < N; ++r)
        for (int k = 0; k < N; ++k) {
          const double kx = (double)(lat.xy[2 * k] - 1) * PI2 / (double)p.Nlx;
          const double ky = (double)(lat.xy[2 * k + 1] - 1) * PI2 / (double)p.Nly;
          const double kr = kx * (double)lat.xy[2 * r] + ky * (double)lat.xy[2 * r + 1];
          kt[k + (size_t)r * N] = std::cos(kr);
          kt[NN + k + (size_t)r * N] = std::sin(kr);
        }
      CUDA_TRY(h, up(o_ktab, kt.data(), 8 * kt.size()));
      C.ktab = (double *)(base + o_ktab);
      C.kout = (double *)(base + o_kout);
    }
    ChainDesc &d = C.d;
    d.beta = p.beta; d.dtau = C.dtau;
    d.eP = std::exp(C.dtau * p.mu); d.eM = std::exp(-C.dtau * p.mu);
    d.rt_scalar = p.RT;
    for (int q = 0; q < 9; ++q) d.rb[q] = rb[q];
    d.use_kin = p.RT > kZero ? 1 : 0;
    // global moves: dtau J of the plaquette ratio and the time-bond
    // probability of compute_time_bond_prob (src/global_update.f90:88-101)
    d.alphaJ = C.dtau * p.J;
    {
      double pt = 0.0;
      if (std::fabs(p.h) > kZero) {
        const double ta = std::max(std::tanh(C.dtau * std::fabs(p.h)), 1.0e-300);
        pt = 1.0 - std::exp(-2.0 * (-0.5 * std::log(ta)));
      }
      d.ptime = std::max(0.0, std::min(1.0, pt));
    }
    d.hzero = std::fabs(p.h) <= kZero ? 1 : 0;
    d.stab_exact = h->opt.stab_exact ? 1 : 0;
    d.flush_shape = h->opt.flush_shape_chain ? h->opt.flush_shape_chain[c] : 0;
    d.kin_fused = kin_fused_size(lat);
    d.bonds = (const int *)(base + o_bonds); d.groups = (const int *)(base + o_groups);
    d.bbonds = (const int *)(base + o_bb); d.plaq = (const int *)(base + o_plaq);
    d.xy = (const int *)(base + o_xy); d.nbx = (const int *)(base + o_nbx);
    d.chsh = (const double *)(base + o_chsh); d.dlt = (const double *)(base + o_dlt);
    d.stag = (const double *)(base + o_stag); d.pshift = (const double *)(base + o_psh);
    d.sigma = (signed char *)(base + o_sigma);
    double *m = (double *)(base + o_mat);
    d.G = m; d.UR = m + NN; d.VR = m + 2 * NN; d.ULT = m + 3 * NN; d.VL = m + 4 * NN;
    d.W0 = m + 5 * NN; d.W1 = m + 6 * NN; d.W2 = m + 7 * NN; d.W3 = m + 8 * NN; d.W4 = m + 9 * NN;
    double *v = (double *)(base + o_vec);
    d.DR = v; d.DL = v + N;
    double *st = (double *)(base + o_stk);
    d.URs = st; d.VRs = st + NN * (Nst + 1); d.ULTs = st + 2 * NN * (Nst + 1); d.VLs = st + 3 * NN * (Nst + 1);
    double *sv = (double *)(base + o_stv);
    d.DRs = sv; d.DLs = sv + (size_t)N * (Nst + 1);
    double *tm = (double *)(base + o_tau);
    d.G00 = tm; d.Gtt = tm + NN; d.Gt0 = tm + 2 * NN; d.G0t = tm + 3 * NN;
    d.URd = tm + 4 * NN; d.VRd = tm + 5 * NN; d.ULTd = tm + 6 * NN; d.VLd = tm + 7 * NN;
    double *tv = (double *)(base + o_tauv);
    d.DRd = tv; d.DLd = tv + N;
    double *bg = (double *)(base + o_big);
    d.B0 = bg; d.B1 = bg + 4 * NN; d.B2 = bg + 8 * NN; d.B3 = bg + 12 * NN;
    d.obs_tau = (double *)(base + o_otau);
    d.grad = (double *)(base + o_grad);
    d.acc = (double *)(base + o_acc);
    char *misc = base + o_misc;
    d.rng = (unsigned int *)misc;
    d.replay_pos = (long long *)(misc + 8);
    d.status = h->d_status + c;
    d.replay = nullptr; d.nreplay = 0;
    d.dec = h->opt.record ? (unsigned char *)(base + o_dec) : nullptr;
    d.ratios = h->opt.record ? (double *)(base + o_rat) : nullptr;
    uint32_t s0 = C.iseed0;
    CUDA_TRY(h, cudaMemcpy(d.rng, &s0, 4, cudaMemcpyHostToDevice));
  }
  // descriptors, LPT order
  CUDA_TRY(h, cudaMalloc(&h->d_desc, sizeof(ChainDesc) * nchains));
  CUDA_TRY(h, cudaMalloc(&h->d_order, sizeof(int) * nchains));
  CUDA_TRY(h, cudaMalloc(&h->d_queue, sizeof(int)));
  {
    std::vector<ChainDesc> dd(nchains);
    for (int c = 0; c < nchains; ++c) dd[c] = h->ch[c].d;
    CUDA_TRY(h, cudaMemcpy(h->d_desc, dd.data(), sizeof(ChainDesc) * nchains, cudaMemcpyHostToDevice));
    std::vector<int> order(nchains);
    for (int c = 0; c < nchains; ++c) order[c] = c;
    auto cost = [&](int c) {
      const ChainHost &C = h->ch[c];
      double n = C.N;
      return (double)C.Ltrot * n * n * (n / C.p.Nwrap * 14.0 + 80.0);
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    CUDA_TRY(h, cudaMemcpy(h->d_order, order.data(), sizeof(int) * nchains, cudaMemcpyHostToDevice));
  }
  int nsm = 0, occ = 0;
  CUDA_TRY(h, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
  CUDA_TRY(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, z2_chain_kernel, Z2_NT, h->smem));
  if (occ < 1) occ = 1;
  h->grid = std::min(nchains, nsm * occ);
  CUDA_TRY(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  CUDA_TRY(h, cudaEventCreate(&h->ev0));
  CUDA_TRY(h, cudaEventCreate(&h->ev1));
  return Z2_OK;
}

extern "C" int z2_destroy(z2_handle *h) {
  if (!h) return Z2_OK;
  cudaSetDevice(h->device);
  for (auto &C : h->ch) {
    if (C.base) cudaFree(C.base);
    if (C.replay) cudaFree(C.replay);
    if (C.gbase) cudaFree(C.gbase);
  }
  if (h->d_desc) cudaFree(h->d_desc);
  if (h->d_order) cudaFree(h->d_order);
  if (h->d_queue) cudaFree(h->d_queue);
  if (h->u_buf) cudaFree(h->u_buf);
  if (h->d_status) cudaFree(h->d_status);
  if (h->d_obs_all) cudaFree(h->d_obs_all);
  for (auto &g : h->graphs) cudaGraphExecDestroy(g.exec);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return Z2_OK;
}

extern "C" const char *z2_last_error(const z2_handle *h) { return h ? h->err.c_str() : "null handle"; }

static int check_chain(const z2_handle *h, int chain) {
  if (!h) return Z2_ERR_ARG;
  if (chain < 0 || chain >= h->nchains)
    return set_err(const_cast<z2_handle *>(h), Z2_ERR_ARG, "chain %d out of range", chain);
  return Z2_OK;
}

// Host buffers an entry point reads or writes must be present; a null one is
// an argument error, reported before any copy.
static int check_ptrs(const z2_handle *h, const char *fn, std::initializer_list<const void *> ps) {
  for (const void *p : ps)
    if (!p) return set_err(const_cast<z2_handle *>(h), Z2_ERR_ARG, "%s: null buffer", fn);
  return Z2_OK;
}

extern "C" int z2_chain_dims(const z2_handle *h, int32_t chain, int32_t *N, int32_t *Ltrot,
                             int32_t *Nst) {
  int r = check_chain(h, chain);
  if (r) return r;
  const ChainHost &C = h->ch[chain];
  if (N) *N = C.N;
  if (Ltrot) *Ltrot = C.Ltrot;
  if (Nst) *Nst = C.Nst;
  return Z2_OK;
}

extern "C" int z2_set_config(z2_handle *h, int32_t chain, const double *sigma, int32_t iseed) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_set_config", {sigma}))) return r;
  ChainHost &C = h->ch[chain];
  std::vector<signed char> s((size_t)C.nb * C.Ltrot);
  for (size_t i = 0; i < s.size(); ++i) {
    if (sigma[i] != 1.0 && sigma[i] != -1.0)
      return set_err(h, Z2_ERR_ARG, "sigma[%zu] = %g is not +-1", i, sigma[i]);
    s[i] = sigma[i] > 0 ? 1 : -1;
  }
  CUDA_TRY(h, cudaSetDevice(h->device));
  CUDA_TRY(h, cudaMemcpy(C.d.sigma, s.data(), s.size(), cudaMemcpyHostToDevice));
  uint32_t st = (uint32_t)iseed;
  CUDA_TRY(h, cudaMemcpy(C.d.rng, &st, 4, cudaMemcpyHostToDevice));
  h->pre_done = false;
  return Z2_OK;
}

extern "C" int z2_get_config(const z2_handle *h, int32_t chain, double *sigma, int32_t *iseed) {
  int r = check_chain(h, chain);
  if (r) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  const ChainHost &C = h->ch[chain];
  std::vector<signed char> s((size_t)C.nb * C.Ltrot);
  CUDA_TRY(hh, cudaSetDevice(h->device));
  CUDA_TRY(hh, cudaMemcpy(s.data(), C.d.sigma, s.size(), cudaMemcpyDeviceToHost));
  if (sigma) for (size_t i = 0; i < s.size(); ++i) sigma[i] = (double)s[i];
  if (iseed) {
    uint32_t st;
    CUDA_TRY(hh, cudaMemcpy(&st, C.d.rng, 4, cudaMemcpyDeviceToHost));
    *iseed = (int32_t)st;
  }
  return Z2_OK;
}

static int enqueue_chains(z2_handle *h, int op, int nsweep, int toggle) {
  CUDA_TRY(h, cudaMemsetAsync(h->d_queue, 0, sizeof(int), h->stream));
  z2_chain_kernel<<<h->grid, Z2_NT, h->smem, h->stream>>>(h->d_desc, h->d_order, h->nchains,
                                                          h->d_queue, op, nsweep, toggle, h->smem);
  CUDA_TRY(h, cudaGetLastError());
  return Z2_OK;
}

static int launch_chains(z2_handle *h, int op, int nsweep, int toggle, float *ms) {
  CUDA_TRY(h, cudaSetDevice(h->device));
  cudaGraphExec_t exec = nullptr;
  if (h->opt.graph && op == OP_SWEEP) {
    for (auto &g : h->graphs)
      if (g.nsweep == nsweep && g.toggle == toggle) exec = g.exec;
    if (!exec) {
      // capture the bin (queue reset + persistent launch) once, replay after
      cudaGraph_t graph = nullptr;
      CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      int r = enqueue_chains(h, op, nsweep, toggle);
      cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
      if (r) {
        if (graph) cudaGraphDestroy(graph);
        return r;
      }
      if (e != cudaSuccess) return set_err(h, Z2_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return set_err(h, Z2_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
      h->graphs.push_back({nsweep, toggle, exec});
    }
  }
  if (ms) CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
  if (exec) {
    CUDA_TRY(h, cudaGraphLaunch(exec, h->stream));
  } else {
    int r = enqueue_chains(h, op, nsweep, toggle);
    if (r) return r;
  }
  if (ms) CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (ms) CUDA_TRY(h, cudaEventElapsedTime(ms, h->ev0, h->ev1));
  // status flags of every chain, one readback
  CUDA_TRY(h, cudaMemcpy(h->h_status.data(), h->d_status, sizeof(int) * h->nchains,
                         cudaMemcpyDeviceToHost));
  for (int c = 0; c < h->nchains; ++c)
    if (h->h_status[c] & ST_NONFINITE)
      return set_err(h, Z2_ERR_NONFINITE, "chain %d: non-finite Green's function", c);
  return Z2_OK;
}

extern "C" int z2_pre(z2_handle *h) {
  if (!h) return Z2_ERR_ARG;
  int r = launch_chains(h, OP_PRE, 0, 0, nullptr);
  if (r == Z2_OK) h->pre_done = true;
  return r;
}

extern "C" int z2_sweep_timed(z2_handle *h, int32_t nsweep, int32_t toggle, float *ms) {
  if (!h) return Z2_ERR_ARG;
  if (!h->pre_done) return set_err(h, Z2_ERR_STATE, "z2_pre must run before z2_sweep");
  if (nsweep < 1) return set_err(h, Z2_ERR_ARG, "nsweep must be >= 1");
  return launch_chains(h, OP_SWEEP, nsweep, toggle, ms);
}

extern "C" int z2_sweep(z2_handle *h, int32_t nsweep, int32_t toggle) {
  return z2_sweep_timed(h, nsweep, toggle, nullptr);
}

extern "C" int z2_get_green(const z2_handle *h, int32_t chain, double *G) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_get_green", {G}))) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  const ChainHost &C = h->ch[chain];
  CUDA_TRY(hh, cudaSetDevice(h->device));
  CUDA_TRY(hh, cudaMemcpy(G, C.d.G, sizeof(double) * C.N * C.N, cudaMemcpyDeviceToHost));
  return Z2_OK;
}

extern "C" int z2_get_obs_equal(const z2_handle *h, int32_t chain, double out[Z2_NOBS_EQ]) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_get_obs_equal", {out}))) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  CUDA_TRY(hh, cudaSetDevice(h->device));
  CUDA_TRY(hh, cudaMemcpy(out, h->ch[chain].d.acc + A_BIN0, sizeof(double) * Z2_NOBS_EQ,
                          cudaMemcpyDeviceToHost));
  return Z2_OK;
}

// The bin observables of every chain gathered into one buffer, so that a
// driver reads all of them with one copy after each bin.
__global__ void z2_gather_obs_kernel(const ChainDesc *descs, int nchains, double *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nchains * Z2_NOBS_EQ;
       i += gridDim.x * blockDim.x) {
    const int c = i / Z2_NOBS_EQ, q = i % Z2_NOBS_EQ;
    out[i] = descs[c].acc[A_BIN0 + q];
  }
}

extern "C" int z2_get_obs_equal_all(z2_handle *h, double *out) {
  if (!h) return Z2_ERR_ARG;
  if (!out) return set_err(h, Z2_ERR_ARG, "z2_get_obs_equal_all: null buffer");
  CUDA_TRY(h, cudaSetDevice(h->device));
  const size_t n = (size_t)h->nchains * Z2_NOBS_EQ;
  if (!h->d_obs_all) CUDA_TRY(h, cudaMalloc(&h->d_obs_all, n * sizeof(double)));
  z2_gather_obs_kernel<<<(int)((n + 255) / 256), 256, 0, h->stream>>>(h->d_desc, h->nchains,
                                                                       h->d_obs_all);
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaMemcpyAsync(out, h->d_obs_all, n * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return Z2_OK;
}

extern "C" int z2_get_obs_tau(const z2_handle *h, int32_t chain, double *out) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_get_obs_tau", {out}))) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  const ChainHost &C = h->ch[chain];
  CUDA_TRY(hh, cudaSetDevice(h->device));
  CUDA_TRY(hh, cudaMemcpy(out, C.d.obs_tau, sizeof(double) * 7 * C.Ltrot * C.N,
                          cudaMemcpyDeviceToHost));
  return Z2_OK;
}

// Fourier_R_to_K of the seven time-displaced correlators of one chain
// (FFT_RtoK_2, src/lattice.f90:263-281, as called by m_write_obs_tau,
// src/fourier_trans.f90:306-440): out = exp(i k.r) [N x N] times the
// correlators [N x 7 Ltrot] / N, as two DMMA GEMMs (cos and sin parts; the
// correlators are real).  One CTA per slab of 64 columns.
__global__ void __launch_bounds__(Z2_NT, 1)
z2_kspace_kernel(int N, int ncol, const double *tab, const double *obs, double *out) {
  const int c0 = blockIdx.x * 64;
  const int nc = (ncol - c0) < 64 ? (ncol - c0) : 64;
  if (nc <= 0) return;
  const double sc = 1.0 / (double)N;
  for (int part = 0; part < 2; ++part)
    blk_dmma(N, nc, N, sc, MatRef{tab + (size_t)part * N * N, 1, N}, false,
             MatRef{obs + (size_t)c0 * N, 1, N}, false, 0.0,
             out + (size_t)part * N * ncol + (size_t)c0 * N, N);
}

extern "C" int z2_get_obs_tau_k(const z2_handle *h, int32_t chain, double *re, double *im) {
  int r = check_chain(h, chain);
  if (r) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  if (!re || !im) return set_err(hh, Z2_ERR_ARG, "z2_get_obs_tau_k: null output");
  const ChainHost &C = h->ch[chain];
  if (!C.ktab)
    return set_err(hh, Z2_ERR_STATE, "z2_get_obs_tau_k: handle created without tau (z2_options.tau)");
  CUDA_TRY(hh, cudaSetDevice(h->device));
  const int ncol = 7 * C.Ltrot;
  z2_kspace_kernel<<<(ncol + 63) / 64, Z2_NT, 0, h->stream>>>(C.N, ncol, C.ktab, C.d.obs_tau, C.kout);
  CUDA_TRY(hh, cudaGetLastError());
  const size_t n = (size_t)ncol * C.N;
  CUDA_TRY(hh, cudaMemcpyAsync(re, C.kout, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(hh, cudaMemcpyAsync(im, C.kout + n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(hh, cudaStreamSynchronize(h->stream));
  return Z2_OK;
}

static int upload_desc(z2_handle *h, int chain);

// Boson-only warm-up of every chain (Local_sweep_therm, src/main.f90:38-67):
// nwarm sweeps of LocalK_therm; acc (optional, [nchains]) receives each
// chain's Acc_Kt%acc / nwarm.  Changes sigma, so z2_pre must follow.
extern "C" int z2_therm(z2_handle *h, int32_t nwarm, double *acc) {
  if (!h) return Z2_ERR_ARG;
  if (nwarm < 0) return set_err(h, Z2_ERR_ARG, "z2_therm: nwarm = %d", nwarm);
  if (nwarm > 0) {
    int r = launch_chains(h, OP_THERM, nwarm, 0, nullptr);
    if (r) return r;
  }
  h->pre_done = false;
  if (acc) {
    CUDA_TRY(h, cudaSetDevice(h->device));
    for (int c = 0; c < h->nchains; ++c) {
      double a = 0.0;
      CUDA_TRY(h, cudaMemcpy(&a, h->ch[c].d.acc + A_TACC, sizeof(double), cudaMemcpyDeviceToHost));
      acc[c] = nwarm > 0 ? a / nwarm : 0.0;
    }
  }
  return Z2_OK;
}

// Global_sweep for every chain (src/global_update.f90:320-337).  The backup
// of the chain state that a rejected move restores is allocated on the first
// call.
extern "C" int z2_sweep_global(z2_handle *h, int32_t nglobal) {
  if (!h) return Z2_ERR_ARG;
  if (nglobal < 0) return set_err(h, Z2_ERR_ARG, "z2_sweep_global: nglobal = %d", nglobal);
  if (!h->pre_done) return set_err(h, Z2_ERR_STATE, "z2_sweep_global before z2_pre");
  CUDA_TRY(h, cudaSetDevice(h->device));
  for (int c = 0; c < h->nchains; ++c) {
    ChainHost &C = h->ch[c];
    if (C.gbase) continue;
    const size_t NN = (size_t)C.N * C.N, S1 = (size_t)C.Nst + 1;
    const size_t nd = 5 * NN + 2 * (size_t)C.N + 4 * NN * S1 + 2 * (size_t)C.N * S1 + 1;
    const size_t bytes = al256(8 * nd) + al256((size_t)C.Ltrot) + al256(4 * (size_t)C.Ltrot);
    char *b = nullptr;
    if (cudaMalloc(&b, bytes) != cudaSuccess)
      return set_err(h, Z2_ERR_NOMEM, "chain %d: cudaMalloc of %zu bytes failed", c, bytes);
    C.gbase = b;
    C.d.gbak = (double *)b;
    C.d.gmask = (signed char *)(b + al256(8 * nd));
    C.d.gqueue = (int *)(b + al256(8 * nd) + al256((size_t)C.Ltrot));
    int r = upload_desc(h, c);
    if (r) return r;
  }
  if (nglobal == 0) return Z2_OK;
  return launch_chains(h, OP_GLOBAL, nglobal, 0, nullptr);
}

extern "C" int z2_get_global_stats(const z2_handle *h, int32_t chain, double out[5]) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_get_global_stats", {out}))) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  double a[A_COUNT];
  CUDA_TRY(hh, cudaSetDevice(h->device));
  CUDA_TRY(hh, cudaMemcpy(a, h->ch[chain].d.acc, sizeof(a), cudaMemcpyDeviceToHost));
  out[0] = a[A_GACC]; out[1] = a[A_GSIZE]; out[2] = a[A_GNUM]; out[3] = a[A_GDEN];
  out[4] = a[A_NOTBETA] == 0.0 ? 1.0 : 0.0;
  return Z2_OK;
}

extern "C" int z2_get_stats(const z2_handle *h, int32_t chain, double out[Z2_NSTATS]) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_get_stats", {out}))) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  double a[A_COUNT];
  CUDA_TRY(hh, cudaSetDevice(h->device));
  CUDA_TRY(hh, cudaMemcpy(a, h->ch[chain].d.acc, sizeof(a), cudaMemcpyDeviceToHost));
  out[0] = a[A_ACC]; out[1] = a[A_XMAX]; out[2] = a[A_XMEAN];
  out[3] = a[A_TXMAX0]; out[4] = a[A_TXMAX1]; out[5] = a[A_TXMAX2];
  out[6] = a[A_TXMEAN0]; out[7] = a[A_TXMEAN1]; out[8] = a[A_TXMEAN2];
  out[9] = a[A_ACC_NUM]; out[10] = a[A_ACC_DEN]; out[11] = a[A_DRAWS];
  out[12] = a[A_NOBS]; out[13] = a[A_NOBST];
  return Z2_OK;
}

extern "C" int z2_get_phase_cycles(const z2_handle *h, int32_t chain, double out[Z2_NPHASE]) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_get_phase_cycles", {out}))) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  CUDA_TRY(hh, cudaSetDevice(h->device));
  CUDA_TRY(hh, cudaMemcpy(out, h->ch[chain].d.acc + A_PH0, sizeof(double) * Z2_NPHASE,
                          cudaMemcpyDeviceToHost));
  return Z2_OK;
}

// ---------------------------------------------------------------------------
// Autotuner of the delay rank and the flush tile shape.  The reference applies
// every accepted flip to G at once (src/localK.f90:141-165); here flips are
// queued and flushed as one rank-2k GEMM, and the best k trades the flush
// GEMM's efficiency (grows with k) against the per-proposal corrections and
// the column build (grow with k); the tile shape of the flush trades the load
// balance of its N x N blocks over the 8 warps against fragment reuse.  Every
// (k, shape) gives the same decisions, so the choice is a matter of time only.
// ---------------------------------------------------------------------------
static const int kTuneCand[] = {4, 6, 8, 12, 16, 24, 32, 48, 64};
static const int kTuneShapes[] = {FS_DEFAULT, FS_GEN16, FS_GEN8, FS_T11, FS_T22, FS_T33, FS_T21,
                                  FS_T32};

// SM cycles of one bin of every probe chain (after a warm-up bin), the
// chain kernel's phases summed (flushes are nested in the proposals).
static int probe_cycles(const std::vector<z2_chain_params> &probe, const z2_options &o,
                        std::vector<double> &cyc) {
  z2_handle *h = nullptr;
  const int n = (int)probe.size();
  int rc = z2_create(&h, probe.data(), n, &o);
  if (rc == Z2_OK) rc = z2_pre(h);
  if (rc == Z2_OK) rc = z2_sweep(h, 1, 0);
  std::vector<double> c0((size_t)n * Z2_NPHASE), c1((size_t)n * Z2_NPHASE);
  for (int c = 0; rc == Z2_OK && c < n; ++c) rc = z2_get_phase_cycles(h, c, &c0[(size_t)c * Z2_NPHASE]);
  if (rc == Z2_OK) rc = z2_sweep(h, 1, 0);
  for (int c = 0; rc == Z2_OK && c < n; ++c) rc = z2_get_phase_cycles(h, c, &c1[(size_t)c * Z2_NPHASE]);
  cyc.assign(n, 0.0);
  for (int c = 0; rc == Z2_OK && c < n; ++c)
    for (int ph : {PH_KIN, PH_PROP, PH_OBS, PH_WRAP, PH_DYN})
      cyc[c] += c1[(size_t)c * Z2_NPHASE + ph] - c0[(size_t)c * Z2_NPHASE + ph];
  z2_destroy(h);
  return rc;
}

// The delay rank (and, with shapes, the flush tile shape) per distinct
// lattice size: three probe chains per size (the chain's couplings and time
// step, Ltrot cut to 2 Nwrap), every size side by side in one launch per
// candidate, the median SM cycles of the three, and the first candidate in
// preference order (default shape, then smaller rank) within 3 % of the
// fastest.
static int tune_core(const z2_chain_params *params, int nchains, const z2_options *opt,
                     bool shapes, int32_t *k_out, int32_t *shape_out) {
  if (!params || nchains <= 0 || !k_out) return Z2_ERR_ARG;
  const int reps = 3;
  std::vector<int> sizes, rep;
  for (int c = 0; c < nchains; ++c) {
    const int N = params[c].Nlx * params[c].Nly;
    if (std::find(sizes.begin(), sizes.end(), N) == sizes.end()) {
      sizes.push_back(N);
      rep.push_back(c);
    }
  }
  const int ns = (int)sizes.size();
  std::vector<z2_chain_params> probe;
  for (int i = 0; i < ns; ++i) {
    z2_chain_params p = params[rep[i]];
    const double dtau = p.beta / (double)p.Ltrot;
    const int Lt = std::min(p.Ltrot, 2 * p.Nwrap);
    p.beta = dtau * Lt;
    p.Ltrot = Lt;
    for (int r = 0; r < reps; ++r) {
      z2_chain_params q = p;
      q.seed = p.seed + 7919 * r;
      probe.push_back(q);
    }
  }
  z2_options base{};
  base.device = opt ? opt->device : 0;
  base.stab_exact = opt ? opt->stab_exact : 0;
  // the ranks shared memory allows for each size (no launch: the plan only)
  std::vector<std::vector<int>> ks(ns);
  for (int k : kTuneCand) {
    z2_options o = base;
    o.delay_k = k;
    z2_handle *h = nullptr;
    int rc = z2_create(&h, probe.data(), (int)probe.size(), &o);
    if (rc != Z2_OK) { z2_destroy(h); return rc; }
    for (int i = 0; i < ns; ++i) {
      const int keff = h->ch[(size_t)i * reps].d.k2 / 2;
      if (std::find(ks[i].begin(), ks[i].end(), keff) == ks[i].end()) ks[i].push_back(keff);
    }
    z2_destroy(h);
  }
  struct Cand { int k, shape; };
  std::vector<std::vector<Cand>> cands(ns);
  size_t ncmax = 0;
  for (int i = 0; i < ns; ++i) {
    for (int sh : kTuneShapes) {
      if (!shapes && sh != FS_DEFAULT) continue;
      if (!flush_shape_ok(sh, sizes[i])) continue;
      for (int k : ks[i]) cands[i].push_back({k, sh});
    }
    ncmax = std::max(ncmax, cands[i].size());
  }
  std::vector<std::vector<double>> cost(ns);
  std::vector<int32_t> kc(probe.size()), sc(probe.size());
  std::vector<double> cyc;
  for (size_t ci = 0; ci < ncmax; ++ci) {
    for (int i = 0; i < ns; ++i) {
      const Cand &cd = cands[i][std::min(ci, cands[i].size() - 1)];
      for (int r = 0; r < reps; ++r) { kc[(size_t)i * reps + r] = cd.k; sc[(size_t)i * reps + r] = cd.shape; }
    }
    z2_options o = base;
    o.delay_k_chain = kc.data();
    o.flush_shape_chain = sc.data();
    const int rc = probe_cycles(probe, o, cyc);
    if (rc != Z2_OK) return rc;
    for (int i = 0; i < ns; ++i) {
      if (ci >= cands[i].size()) continue;
      double v[reps];
      for (int r = 0; r < reps; ++r) v[r] = cyc[(size_t)i * reps + r];
      std::sort(v, v + reps);
      cost[i].push_back(v[reps / 2]);
    }
  }
  std::vector<Cand> pick(ns);
  for (int i = 0; i < ns; ++i) {
    const double best = *std::min_element(cost[i].begin(), cost[i].end());
    for (size_t ci = 0; ci < cands[i].size(); ++ci)
      if (cost[i][ci] <= 1.03 * best) { pick[i] = cands[i][ci]; break; }
  }
  for (int c = 0; c < nchains; ++c) {
    const int N = params[c].Nlx * params[c].Nly;
    const int i = (int)(std::find(sizes.begin(), sizes.end(), N) - sizes.begin());
    k_out[c] = pick[i].k;
    if (shape_out) shape_out[c] = pick[i].shape;
  }
  return Z2_OK;
}

extern "C" int z2_tune_delay(const z2_chain_params *params, int32_t nchains,
                             const z2_options *opt, int32_t *k_out) {
  return tune_core(params, nchains, opt, false, k_out, nullptr);
}

extern "C" int z2_tune(const z2_chain_params *params, int32_t nchains, const z2_options *opt,
                       int32_t *k_out, int32_t *shape_out) {
  if (!shape_out) return Z2_ERR_ARG;
  return tune_core(params, nchains, opt, true, k_out, shape_out);
}

static int upload_desc(z2_handle *h, int chain) {
  CUDA_TRY(h, cudaMemcpy(h->d_desc + chain, &h->ch[chain].d, sizeof(ChainDesc),
                         cudaMemcpyHostToDevice));
  return Z2_OK;
}

extern "C" int z2_set_replay(z2_handle *h, int32_t chain, const double *rr, size_t n) {
  int r = check_chain(h, chain);
  if (r) return r;
  if (n > 0 && !rr) return set_err(h, Z2_ERR_ARG, "z2_set_replay: null buffer with n = %zu", n);
  ChainHost &C = h->ch[chain];
  CUDA_TRY(h, cudaSetDevice(h->device));
  if (C.replay) { cudaFree(C.replay); C.replay = nullptr; }
  C.d.replay = nullptr; C.d.nreplay = 0;
  if (n > 0) {
    CUDA_TRY(h, cudaMalloc(&C.replay, n * sizeof(double)));
    CUDA_TRY(h, cudaMemcpy(C.replay, rr, n * sizeof(double), cudaMemcpyHostToDevice));
    C.d.replay = C.replay; C.d.nreplay = (long long)n;
  }
  long long z = 0;
  CUDA_TRY(h, cudaMemcpy(C.d.replay_pos, &z, sizeof(z), cudaMemcpyHostToDevice));
  return upload_desc(h, chain);
}

extern "C" int z2_get_decisions(const z2_handle *h, int32_t chain, uint8_t *dec, double *ratios,
                                size_t n) {
  int r = check_chain(h, chain);
  if (r) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  const ChainHost &C = h->ch[chain];
  if (!C.d.dec) return set_err(hh, Z2_ERR_STATE, "decisions are recorded only with options.record = 1");
  size_t tot = (size_t)2 * C.Ltrot * C.nb;
  if (n > tot) n = tot;
  CUDA_TRY(hh, cudaSetDevice(h->device));
  if (dec) CUDA_TRY(hh, cudaMemcpy(dec, C.d.dec, n, cudaMemcpyDeviceToHost));
  if (ratios) CUDA_TRY(hh, cudaMemcpy(ratios, C.d.ratios, n * sizeof(double), cudaMemcpyDeviceToHost));
  return Z2_OK;
}

extern "C" int z2_logdet_grad(z2_handle *h, int32_t chain, double *logdet, double *dlogdet_dt,
                              double *dlogdet_dmu) {
  int r = check_chain(h, chain);
  if (r) return r;
  ChainHost &C = h->ch[chain];
  CUDA_TRY(h, cudaSetDevice(h->device));
  // run only this chain: a one-entry order list pointing at it
  int *d_one = nullptr;
  CUDA_TRY(h, cudaMalloc(&d_one, sizeof(int)));
  CUDA_TRY(h, cudaMemcpy(d_one, &chain, sizeof(int), cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemsetAsync(h->d_queue, 0, sizeof(int), h->stream));
  z2_chain_kernel<<<1, Z2_NT, h->smem, h->stream>>>(h->d_desc, d_one, 1, h->d_queue, OP_LOGDET, 0,
                                                     0, h->smem);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_one);
  if (e != cudaSuccess) return set_err(h, Z2_ERR_CUDA, "logdet kernel: %s", cudaGetErrorString(e));
  double a[A_COUNT];
  CUDA_TRY(h, cudaMemcpy(a, C.d.acc, sizeof(a), cudaMemcpyDeviceToHost));
  if (logdet) *logdet = a[A_LOGDET];
  if (dlogdet_dmu) *dlogdet_dmu = a[A_DMU];
  if (dlogdet_dt) CUDA_TRY(h, cudaMemcpy(dlogdet_dt, C.d.grad, sizeof(double) * C.nb, cudaMemcpyDeviceToHost));
  h->pre_done = true;
  return Z2_OK;
}

// ---- module-level mirrors ----
static int unit_scratch(z2_handle *h, size_t doubles) {
  if (h->u_n >= doubles) return Z2_OK;
  if (h->u_buf) cudaFree(h->u_buf);
  h->u_buf = nullptr; h->u_n = 0;
  CUDA_TRY(h, cudaMalloc(&h->u_buf, doubles * sizeof(double)));
  h->u_n = doubles;
  return Z2_OK;
}

static int run_unit(z2_handle *h, int chain, int op, const UnitArgs &a) {
  z2_unit_kernel<<<1, Z2_NT, h->smem, h->stream>>>(h->d_desc + chain, op, a, h->smem);
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return Z2_OK;
}

static int mmult(z2_handle *h, int chain, double *M, int nt, int nflag, int op) {
  int r = check_chain(h, chain);
  if (r) return r;
  if ((r = check_ptrs(h, "z2_opk_mmult", {M}))) return r;
  ChainHost &C = h->ch[chain];
  if (nt < 1 || nt > C.Ltrot) return set_err(h, Z2_ERR_ARG, "nt = %d out of 1..Ltrot", nt);
  if (nflag != 1 && nflag != -1) return set_err(h, Z2_ERR_ARG, "incorrect nflag %d", nflag);
  const size_t NN = (size_t)C.N * C.N;
  CUDA_TRY(h, cudaSetDevice(h->device));
  if ((r = unit_scratch(h, NN))) return r;
  CUDA_TRY(h, cudaMemcpy(h->u_buf, M, NN * 8, cudaMemcpyHostToDevice));
  UnitArgs a{};
  a.M = h->u_buf; a.nt = nt; a.nflag = nflag;
  if ((r = run_unit(h, chain, op, a))) return r;
  CUDA_TRY(h, cudaMemcpy(M, h->u_buf, NN * 8, cudaMemcpyDeviceToHost));
  return Z2_OK;
}

extern "C" int z2_opk_mmult_R(z2_handle *h, int32_t chain, double *M, int32_t nt, int32_t nflag) {
  return mmult(h, chain, M, nt, nflag, U_MMULT_R);
}
extern "C" int z2_opk_mmult_L(z2_handle *h, int32_t chain, double *M, int32_t nt, int32_t nflag) {
  return mmult(h, chain, M, nt, nflag, U_MMULT_L);
}

static void transpose_host(const double *src, double *dst, int N) {
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) dst[j + (size_t)i * N] = src[i + (size_t)j * N];
}

static int stab_u(z2_handle *h, int chain, double *U, double *D, double *V, bool left) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, left ? "z2_stab_UL" : "z2_stab_UR", {U, D, V}))) return r;
  ChainHost &C = h->ch[chain];
  const int N = C.N;
  const size_t NN = (size_t)N * N;
  CUDA_TRY(h, cudaSetDevice(h->device));
  if ((r = unit_scratch(h, 2 * NN + N))) return r;
  std::vector<double> tmp(NN);
  const double *Usrc = U;
  if (left) { transpose_host(U, tmp.data(), N); Usrc = tmp.data(); }
  CUDA_TRY(h, cudaMemcpy(h->u_buf, Usrc, NN * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(h->u_buf + NN, V, NN * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(h->u_buf + 2 * NN, D, N * 8, cudaMemcpyHostToDevice));
  UnitArgs a{};
  a.U = h->u_buf; a.V = h->u_buf + NN; a.D = h->u_buf + 2 * NN;
  if ((r = run_unit(h, chain, left ? U_STAB_UL : U_STAB_UR, a))) return r;
  CUDA_TRY(h, cudaMemcpy(tmp.data(), h->u_buf, NN * 8, cudaMemcpyDeviceToHost));
  if (left) transpose_host(tmp.data(), U, N);
  else memcpy(U, tmp.data(), NN * 8);
  CUDA_TRY(h, cudaMemcpy(V, h->u_buf + NN, NN * 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(h, cudaMemcpy(D, h->u_buf + 2 * NN, N * 8, cudaMemcpyDeviceToHost));
  return Z2_OK;
}

extern "C" int z2_stab_UR(z2_handle *h, int32_t chain, double *U, double *D, double *V) {
  return stab_u(h, chain, U, D, V, false);
}
extern "C" int z2_stab_UL(z2_handle *h, int32_t chain, double *U, double *D, double *V) {
  return stab_u(h, chain, U, D, V, true);
}

static int upload_udv(z2_handle *h, int N, const double *UR, const double *DR, const double *VR,
                      const double *UL, const double *DL, const double *VL, size_t extra,
                      UnitArgs &a) {
  const size_t NN = (size_t)N * N;
  int r = unit_scratch(h, 4 * NN + 2 * N + extra);
  if (r) return r;
  std::vector<double> ult(NN);
  transpose_host(UL, ult.data(), N);
  double *b = h->u_buf;
  CUDA_TRY(h, cudaMemcpy(b, UR, NN * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(b + NN, VR, NN * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(b + 2 * NN, ult.data(), NN * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(b + 3 * NN, VL, NN * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(b + 4 * NN, DR, N * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(b + 4 * NN + N, DL, N * 8, cudaMemcpyHostToDevice));
  a.UR = b; a.VR = b + NN; a.ULT = b + 2 * NN; a.VL = b + 3 * NN;
  a.DR = b + 4 * NN; a.DL = b + 4 * NN + N;
  return Z2_OK;
}

extern "C" int z2_stab_green(z2_handle *h, int32_t chain, const double *UR, const double *DR,
                             const double *VR, const double *UL, const double *DL,
                             const double *VL, int32_t nt, double *G) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_stab_green", {UR, DR, VR, UL, DL, VL, G}))) return r;
  ChainHost &C = h->ch[chain];
  const int N = C.N;
  const size_t NN = (size_t)N * N;
  if (nt < 0 || nt > C.Ltrot) return set_err(h, Z2_ERR_ARG, "illegal nt = %d in stab_green", nt);
  CUDA_TRY(h, cudaSetDevice(h->device));
  UnitArgs a{};
  if ((r = upload_udv(h, N, UR, DR, VR, UL, DL, VL, NN, a))) return r;
  a.G = h->u_buf + 4 * NN + 2 * N;
  a.nt = nt;
  if ((r = run_unit(h, chain, U_STAB_GREEN, a))) return r;
  CUDA_TRY(h, cudaMemcpy(G, a.G, NN * 8, cudaMemcpyDeviceToHost));
  return Z2_OK;
}

extern "C" int z2_stab_green_big(z2_handle *h, int32_t chain, const double *UR, const double *DR,
                                 const double *VR, const double *UL, const double *DL,
                                 const double *VL, double *G00, double *G0t, double *Gt0,
                                 double *Gtt) {
  int r = check_chain(h, chain);
  if (r || (r = check_ptrs(h, "z2_stab_green_big",
                           {UR, DR, VR, UL, DL, VL, G00, G0t, Gt0, Gtt})))
    return r;
  ChainHost &C = h->ch[chain];
  const int N = C.N;
  const size_t NN = (size_t)N * N;
  CUDA_TRY(h, cudaSetDevice(h->device));
  UnitArgs a{};
  if ((r = upload_udv(h, N, UR, DR, VR, UL, DL, VL, 4 * NN, a))) return r;
  double *o = h->u_buf + 4 * NN + 2 * N;
  a.G = o; a.G0t = o + NN; a.Gt0 = o + 2 * NN; a.Gtt = o + 3 * NN;
  if ((r = run_unit(h, chain, U_STAB_GREEN_BIG, a))) return r;
  CUDA_TRY(h, cudaMemcpy(G00, a.G, NN * 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(h, cudaMemcpy(G0t, a.G0t, NN * 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(h, cudaMemcpy(Gt0, a.Gt0, NN * 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(h, cudaMemcpy(Gtt, a.Gtt, NN * 8, cudaMemcpyDeviceToHost));
  return Z2_OK;
}

// ---------------------------------------------------------------------------
// Module-level mirrors on a chain's resident state.  Each entry point runs one
// procedure of the reference's multiply / stabilization / dynamics /
// obser_equal / obser_tau / localK modules on one chain of the handle, on the
// state the handle keeps in global memory between calls (the Propagator G,
// UR DR VR, UL DL VL, the UDV stacks, the Dyn copy and PropGreen, sigma, the
// ranf state and the observable sums), so that a driver can replace the
// reference's modules one at a time.  The U factors are propagated at every
// call (the whole-bin path propagates them lazily, with the same operations in
// the same order).  One CTA, the chain kernel's shared-memory plan.
// ---------------------------------------------------------------------------
enum {
  SO_PROPK_PRE = 1, SO_PROPT_PRE, SO_PROPK_L, SO_PROPK_R, SO_PROPT_L, SO_PROPT_R,
  SO_PROPGRK_R, SO_PROPGRT_R, SO_WRAP_PRE, SO_WRAP_L, SO_WRAP_R, SO_WRAP_TAU,
  SO_DYN_RESET, SO_SWEEP_RESET, SO_OBS_EQ_CALC, SO_OBS_EQ_AVE, SO_OBS_TAU_CALC,
  SO_OBS_TAU_AVE, SO_SLICE_L, SO_SLICE_R
};

__global__ void __launch_bounds__(Z2_NT, 1)
z2_state_kernel(const ChainDesc *desc, int op, int nt, int flag, double x, unsigned smem_bytes) {
  extern __shared__ __align__(16) unsigned char z2_smem[];
  __shared__ ChainDesc sc;
  __shared__ Smem s;
  load_desc(sc, desc);
  if (threadIdx.x == 0) s = make_smem(sc, z2_smem, smem_bytes);
  __syncthreads();
  const ChainDesc &c = sc;
  const int N = c.N;
  Pend pd{1, 0};
  switch (op) {
    case SO_PROPK_PRE:      // propK_pre (src/multiply.f90:8-15) as Local_sweep_pre calls it
      if (c.use_kin) { build_table(c, s, nt); kin_global(c, s, c.UR, 1, 0); }
      break;
    case SO_PROPT_PRE:      // propT_pre (src/multiply.f90:65-77)
      blk_scale(c.UR, N, N, N, c.eP);
      break;
    case SO_PROPK_L:        // propK_L (src/multiply.f90:17-28): G B, B^-1 G, UL B
      load_G(c, s);
      build_table(c, s, nt);
      kin_cols(c, s, s.G, s.ldg, N, 1);
      kin_rows(c, s, s.G, s.ldg, N, -1);
      spill_G(c, s);
      kin_global(c, s, c.ULT, 1, 0);      // UL^T <- B UL^T (B symmetric)
      break;
    case SO_PROPK_R:        // propK_R (src/multiply.f90:30-41): B G, G B^-1, B UR
      load_G(c, s);
      build_table(c, s, nt);
      kin_rows(c, s, s.G, s.ldg, N, 1);
      kin_cols(c, s, s.G, s.ldg, N, -1);
      spill_G(c, s);
      kin_global(c, s, c.UR, 1, 0);
      break;
    case SO_PROPT_L:        // propT_L (src/multiply.f90:79-93)
      blk_scale(c.G, N, N, N, c.eP);
      blk_scale(c.G, N, N, N, c.eM);
      blk_scale(c.ULT, N, N, N, c.eP);
      break;
    case SO_PROPT_R:        // propT_R (src/multiply.f90:95-108)
      blk_scale(c.G, N, N, N, c.eP);
      blk_scale(c.G, N, N, N, c.eM);
      blk_scale(c.UR, N, N, N, c.eP);
      break;
    case SO_PROPGRK_R:      // propgrK_R (src/multiply.f90:43-63) on the Dyn copy
      if (c.use_kin) {
        propgr_R(c, s, nt, true, false);
        kin_global(c, s, c.URd, 1, 0);
      }
      break;
    case SO_PROPGRT_R:      // propgrT_R (src/multiply.f90:110-130)
      propgr_R(c, s, nt, false, true);
      blk_scale(c.URd, N, N, N, c.eP);
      break;
    case SO_WRAP_PRE:       // Wrap_pre (src/stabilization.f90:374-398)
      wrap_pre(c, s, nt, pd);
      break;
    case SO_WRAP_L:         // Wrap_L (src/stabilization.f90:400-437)
      load_G(c, s);
      wrap_L(c, s, nt, pd, flag != 0);
      spill_G(c, s);
      break;
    case SO_WRAP_R:         // Wrap_R (src/stabilization.f90:439-476)
      load_G(c, s);
      wrap_R(c, s, nt, pd, flag != 0);
      spill_G(c, s);
      break;
    case SO_WRAP_TAU:       // Wrap_tau (src/stabilization.f90:478-514)
      wrap_tau(c, s, nt, pd);
      break;
    case SO_DYN_RESET:      // Dyn_reset (src/dynamics.f90:41-48)
      dyn_reset(c, s);
      break;
    case SO_SWEEP_RESET:    // Local_sweep_reset (src/local_sweep.f90:56-71)
      sweep_reset(c, flag != 0, c.hzero != 0);
      break;
    case SO_OBS_EQ_CALC:    // Obs_equal%calc (src/obser_equal.f90:73-149)
      load_G(c, s);
      obs_equal(c, s, nt);
      break;
    case SO_OBS_EQ_AVE:     // Obs_equal%ave (src/obser_equal.f90:50-71)
      obs_equal_ave(c, x);
      break;
    case SO_OBS_TAU_CALC:   // Obs_tau%calc (src/obser_tau.f90:56-133)
      obs_tau(c, s, nt);
      break;
    case SO_OBS_TAU_AVE:    // Obs_tau%ave (src/obser_tau.f90:37-47)
      obs_tau_ave(c, x);
      break;
    case SO_SLICE_L:        // LocalK_prop_L (src/localK.f90:347-373)
    case SO_SLICE_R:        // LocalK_prop_R (src/localK.f90:375-398)
      for (int i = threadIdx.x; i < 2 * c.nb; i += Z2_NT) s.bond[i] = c.bonds[i];
      __syncthreads();
      load_G(c, s);
      if (op == SO_SLICE_L) {
        propose_slice(c, s, nt, true, 0);            // bonds 2N..1
        build_table(c, s, nt);
        kin_cols(c, s, s.G, s.ldg, N, 1);
        kin_rows(c, s, s.G, s.ldg, N, -1);
        spill_G(c, s);
        kin_global(c, s, c.ULT, 1, 0);
      } else {
        build_table(c, s, nt);
        kin_rows(c, s, s.G, s.ldg, N, 1);
        kin_cols(c, s, s.G, s.ldg, N, -1);
        propose_slice(c, s, nt, false, 1);           // bonds 1..2N
        spill_G(c, s);
        build_table(c, s, nt);                       // B_nt with the flipped links
        kin_global(c, s, c.UR, 1, 0);
      }
      break;
    default:
      break;
  }
}

// Launch one state procedure on one chain, synchronously; a non-finite drift
// or Green's function found by it is Z2_ERR_NONFINITE.
static int run_state(z2_handle *h, int chain, int op, int nt, int flag, double x) {
  CUDA_TRY(h, cudaSetDevice(h->device));
  z2_state_kernel<<<1, Z2_NT, h->smem, h->stream>>>(h->d_desc + chain, op, nt, flag, x, h->smem);
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  int st = 0;
  CUDA_TRY(h, cudaMemcpy(&st, h->d_status + chain, sizeof(int), cudaMemcpyDeviceToHost));
  if (st & ST_NONFINITE) return set_err(h, Z2_ERR_NONFINITE, "chain %d: non-finite Green's function", chain);
  return Z2_OK;
}

// nt of a per-slice procedure: 1..Ltrot.
static int slice_op(z2_handle *h, int chain, int nt, int op, const char *fn) {
  int r = check_chain(h, chain);
  if (r) return r;
  if (nt < 1 || nt > h->ch[chain].Ltrot)
    return set_err(h, Z2_ERR_ARG, "%s: nt = %d out of 1..Ltrot", fn, nt);
  return run_state(h, chain, op, nt, 0, 0.0);
}

// nt of a wrap: a stabilization point 0..Ltrot (a multiple of Nwrap).
static int wrap_op(z2_handle *h, int chain, int nt, int flag, int op, const char *fn, int lo) {
  int r = check_chain(h, chain);
  if (r) return r;
  const ChainHost &C = h->ch[chain];
  if (nt < lo || nt > C.Ltrot || nt % C.p.Nwrap != 0)
    return set_err(h, Z2_ERR_ARG, "%s: nt = %d is not a stabilization point (%d..Ltrot, a multiple "
                   "of Nwrap)", fn, nt, lo);
  r = run_state(h, chain, op, nt, flag, 0.0);
  if (r == Z2_OK && op == SO_WRAP_PRE && nt == C.Ltrot) h->pre_done = true;
  return r;
}

static int chain_op(z2_handle *h, int chain, int op, int flag, double x) {
  int r = check_chain(h, chain);
  if (r) return r;
  return run_state(h, chain, op, 0, flag, x);
}

extern "C" int z2_propK_pre(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_PROPK_PRE, "z2_propK_pre");
}
extern "C" int z2_propK_L(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_PROPK_L, "z2_propK_L");
}
extern "C" int z2_propK_R(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_PROPK_R, "z2_propK_R");
}
extern "C" int z2_propgrK_R(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_PROPGRK_R, "z2_propgrK_R");
}
extern "C" int z2_propT_pre(z2_handle *h, int32_t chain) { return chain_op(h, chain, SO_PROPT_PRE, 0, 0.0); }
extern "C" int z2_propT_L(z2_handle *h, int32_t chain) { return chain_op(h, chain, SO_PROPT_L, 0, 0.0); }
extern "C" int z2_propT_R(z2_handle *h, int32_t chain) { return chain_op(h, chain, SO_PROPT_R, 0, 0.0); }
extern "C" int z2_propgrT_R(z2_handle *h, int32_t chain) {
  return chain_op(h, chain, SO_PROPGRT_R, 0, 0.0);
}
extern "C" int z2_wrap_pre(z2_handle *h, int32_t chain, int32_t nt) {
  return wrap_op(h, chain, nt, 0, SO_WRAP_PRE, "z2_wrap_pre", 0);
}
extern "C" int z2_wrap_L(z2_handle *h, int32_t chain, int32_t nt, int32_t flag) {
  return wrap_op(h, chain, nt, flag, SO_WRAP_L, "z2_wrap_L", 0);
}
extern "C" int z2_wrap_R(z2_handle *h, int32_t chain, int32_t nt, int32_t flag) {
  return wrap_op(h, chain, nt, flag, SO_WRAP_R, "z2_wrap_R", 0);
}
extern "C" int z2_wrap_tau(z2_handle *h, int32_t chain, int32_t nt) {
  return wrap_op(h, chain, nt, 0, SO_WRAP_TAU, "z2_wrap_tau", 1);
}
extern "C" int z2_dyn_reset(z2_handle *h, int32_t chain) { return chain_op(h, chain, SO_DYN_RESET, 0, 0.0); }
extern "C" int z2_sweep_reset(z2_handle *h, int32_t chain, int32_t toggle) {
  return chain_op(h, chain, SO_SWEEP_RESET, toggle != 0, 0.0);
}
extern "C" int z2_obs_equal_calc(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_OBS_EQ_CALC, "z2_obs_equal_calc");
}
extern "C" int z2_obs_equal_ave(z2_handle *h, int32_t chain, int32_t nobs) {
  if (nobs < 0) return set_err(h, Z2_ERR_ARG, "z2_obs_equal_ave: nobs = %d", nobs);
  return chain_op(h, chain, SO_OBS_EQ_AVE, 0, (double)nobs);
}
extern "C" int z2_obs_tau_calc(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_OBS_TAU_CALC, "z2_obs_tau_calc");
}
extern "C" int z2_obs_tau_ave(z2_handle *h, int32_t chain, int32_t nobst) {
  if (nobst < 1) return set_err(h, Z2_ERR_ARG, "z2_obs_tau_ave: nobst = %d", nobst);
  return chain_op(h, chain, SO_OBS_TAU_AVE, 0, (double)nobst);
}
extern "C" int z2_prop_slice_L(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_SLICE_L, "z2_prop_slice_L");
}
extern "C" int z2_prop_slice_R(z2_handle *h, int32_t chain, int32_t nt) {
  return slice_op(h, chain, nt, SO_SLICE_R, "z2_prop_slice_R");
}

// Propagator readback / upload: G, UR DR VR, UL DL VL (UL in the reference's
// orientation; the handle keeps UL^T).  Each buffer is optional.
extern "C" int z2_get_prop(const z2_handle *h, int32_t chain, double *G, double *UR, double *DR,
                           double *VR, double *UL, double *DL, double *VL) {
  int r = check_chain(h, chain);
  if (r) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  const ChainHost &C = h->ch[chain];
  const int N = C.N;
  const size_t NN = (size_t)N * N;
  CUDA_TRY(hh, cudaSetDevice(h->device));
  auto get = [&](double *dst, const double *src, size_t n) {
    return dst ? cudaMemcpy(dst, src, n * 8, cudaMemcpyDeviceToHost) : cudaSuccess;
  };
  CUDA_TRY(hh, get(G, C.d.G, NN));
  CUDA_TRY(hh, get(UR, C.d.UR, NN));
  CUDA_TRY(hh, get(DR, C.d.DR, N));
  CUDA_TRY(hh, get(VR, C.d.VR, NN));
  CUDA_TRY(hh, get(DL, C.d.DL, N));
  CUDA_TRY(hh, get(VL, C.d.VL, NN));
  if (UL) {
    std::vector<double> t(NN);
    CUDA_TRY(hh, cudaMemcpy(t.data(), C.d.ULT, NN * 8, cudaMemcpyDeviceToHost));
    transpose_host(t.data(), UL, N);
  }
  return Z2_OK;
}

extern "C" int z2_set_prop(z2_handle *h, int32_t chain, const double *G, const double *UR,
                           const double *DR, const double *VR, const double *UL, const double *DL,
                           const double *VL) {
  int r = check_chain(h, chain);
  if (r) return r;
  const ChainHost &C = h->ch[chain];
  const int N = C.N;
  const size_t NN = (size_t)N * N;
  CUDA_TRY(h, cudaSetDevice(h->device));
  auto put = [&](double *dst, const double *src, size_t n) {
    return src ? cudaMemcpy(dst, src, n * 8, cudaMemcpyHostToDevice) : cudaSuccess;
  };
  CUDA_TRY(h, put(C.d.G, G, NN));
  CUDA_TRY(h, put(C.d.UR, UR, NN));
  CUDA_TRY(h, put(C.d.DR, DR, N));
  CUDA_TRY(h, put(C.d.VR, VR, NN));
  CUDA_TRY(h, put(C.d.DL, DL, N));
  CUDA_TRY(h, put(C.d.VL, VL, NN));
  if (UL) {
    std::vector<double> t(NN);
    transpose_host(UL, t.data(), N);
    CUDA_TRY(h, cudaMemcpy(C.d.ULT, t.data(), NN * 8, cudaMemcpyHostToDevice));
  }
  return Z2_OK;
}

// PropGreen readback (src/process_matrix.f90:14-20): Gr00, Gr0t, Grt0, Grtt
// of the time-displaced chain; each buffer optional.
extern "C" int z2_get_propgr(const z2_handle *h, int32_t chain, double *G00, double *G0t,
                             double *Gt0, double *Gtt) {
  int r = check_chain(h, chain);
  if (r) return r;
  z2_handle *hh = const_cast<z2_handle *>(h);
  const ChainHost &C = h->ch[chain];
  const size_t NN = (size_t)C.N * C.N;
  CUDA_TRY(hh, cudaSetDevice(h->device));
  const double *src[4] = {C.d.G00, C.d.G0t, C.d.Gt0, C.d.Gtt};
  double *dst[4] = {G00, G0t, Gt0, Gtt};
  for (int q = 0; q < 4; ++q)
    if (dst[q]) CUDA_TRY(hh, cudaMemcpy(dst[q], src[q], NN * 8, cudaMemcpyDeviceToHost));
  return Z2_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free stab_green.
//
// Some callers cannot call cudaMalloc: for instance a host program whose
// device memory is owned by another allocator (a framework's caching
// allocator, or a Fortran driver that reserves one pool at start-up and
// forbids further driver allocations inside its time-stepping loop).  For
// them this entry point computes the same Green's function as z2_stab_green,
// with caller-owned device buffers for inputs and outputs and its scratch in
// the file-scope array below, which every GPU that loads this library keeps
// until the process exits: 5 * Z2_NOALLOC_NMAX^2 doubles (829,440 bytes).
// ---------------------------------------------------------------------------
#include <cuda.h>   // CUcontext / CUresult types of the two driver entry points below

#include <mutex>

static __device__ __align__(256) double z2_noalloc_scratch[5 * Z2_NOALLOC_NMAX * Z2_NOALLOC_NMAX];

// Shared work space of the two QR steps, enough for every N <= 144 so that
// this kernel runs the same QR code as z2_stab_green: the register-resident
// pivoted QR needs 2N doubles, the blocked DORGQR (16-column blocks) its V and
// W panels (4544 doubles at N = 144) and, for the T prologue, 8 warps x
// (2 * 16^2 + 4 * 16) = 4608 doubles.
constexpr int kNoallocTile = Z2_WARPS * (2 * 16 * 16 + 4 * 16);

__global__ void __launch_bounds__(Z2_NT, 1)
z2_stab_green_noalloc_kernel(int N, int nt, int Ltrot, const double *UR, const double *DR,
                             const double *VR, const double *UL, const double *DL,
                             const double *VL, double *G, double *scratch) {
  extern __shared__ __align__(16) unsigned char z2_smem[];
  Smem s{};
  size_t off = 0;
  s.red = (double *)(z2_smem + off); off += sizeof(double) * Z2_NRED;
  s.vec = (double *)(z2_smem + off); off += sizeof(double) * 8 * N;
  s.ivec = (int *)(z2_smem + off); off += align16(sizeof(int) * 2 * N);
  s.flag = (int *)(z2_smem + off); off += sizeof(int) * 16;
  off = align16(off);
  s.tile = (double *)(z2_smem + off);
  s.tile_doubles = kNoallocTile;
  // scratch: M (QR work matrix), W1, W2, W3, UL^T; every entry read is
  // written first by this call, so nothing has to start at zero.
  const size_t NN = (size_t)N * N;
  double *M = scratch, *W1 = M + NN, *W2 = W1 + NN, *W3 = W2 + NN, *ULT = W3 + NN;
  blk_transpose(ULT, N, UL, N, N, N);
  dev_stab_green(s, N, nt, Ltrot, UR, DR, VR, ULT, DL, VL, M, N, W1, W2, W3, G);
}

static constexpr size_t noalloc_smem_bytes(int N) {
  return ((((sizeof(double) * Z2_NRED + sizeof(double) * 8 * (size_t)N) +
            (((sizeof(int) * 2 * (size_t)N) + 15) & ~size_t(15)) + sizeof(int) * 16) + 15) &
          ~size_t(15)) + sizeof(double) * kNoallocTile;
}
// within the 48 KB a launch gets without opting in to more
static_assert(noalloc_smem_bytes(Z2_NOALLOC_NMAX) <= 48 * 1024, "no-alloc shared memory");

// Identity of the calling thread's current CUDA context: a 64-bit id that the
// driver never reuses within a process (cuCtxGetId), or 0 when no context is
// current or the driver does not offer the call.  The driver entry points
// come through the runtime, so the library needs no link to libcuda.
static unsigned long long current_ctx_id() {
  typedef CUresult (*get_current_t)(CUcontext *);
  typedef CUresult (*get_id_t)(CUcontext, unsigned long long *);
  static get_current_t get_current = nullptr;
  static get_id_t get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (get_current_t)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (get_id_t)f;
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

extern "C" int z2_stab_green_noalloc(int32_t N, int32_t nt, int32_t Ltrot, const double *UR,
                                     const double *DR, const double *VR, const double *UL,
                                     const double *DL, const double *VL, double *G,
                                     void *stream) {
  if (N < 1 || N > Z2_NOALLOC_NMAX) return Z2_ERR_ARG;
  if (Ltrot < 1 || nt < 0 || nt > Ltrot) return Z2_ERR_ARG;
  if (!UR || !DR || !VR || !UL || !DL || !VL || !G) return Z2_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return Z2_ERR_CUDA;
  // Set-up, once per device with that device current: the device address of
  // the scratch array (host code must not use the symbol itself).  The
  // address belongs to the context the array was loaded into, so it is looked
  // up again when the device's current context changes (a new context after
  // cudaDeviceReset, or a caller's own driver-API context).
  struct Slot { unsigned long long ctx; double *ptr; };
  static std::mutex mu;
  static Slot scratch_of[64] = {};
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long id = current_ctx_id();
    Slot &sl = scratch_of[dev];
    if (!sl.ptr || id == 0 || sl.ctx != id) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, z2_noalloc_scratch) != cudaSuccess || !p) return Z2_ERR_CUDA;
      sl.ptr = (double *)p;
      // the lookup makes the runtime's context current when none was
      sl.ctx = id ? id : current_ctx_id();
    }
    scratch = sl.ptr;
  }
  z2_stab_green_noalloc_kernel<<<1, Z2_NT, noalloc_smem_bytes(N), (cudaStream_t)stream>>>(
      N, nt, Ltrot, UR, DR, VR, UL, DL, VL, G, scratch);
  if (cudaGetLastError() != cudaSuccess) return Z2_ERR_CUDA;
  return Z2_OK;
}
