// z2_main.cpp -- host driver over the C ABI, restating the flow of the
// reference program (src/main.f90) for the local-sweep path:
//
//   paramC_sets.txt  (read_input, src/calc_basic.f90:50-89)
//   confin.txt / seeds.txt -> sigma (conf_therm_in + conf_set + conf_transfer,
//                                    src/fields.f90:214-507)
//   optional boson-only warm-up (LocalK_therm, src/localK.f90:400-420) on the GPU
//   Sweep_local%pre, then Nbin bins of Sweep_local%sweep (src/main.f90:72-103)
//   per bin: flux_avg, chi_flux, pair_sc_q0, cdw_pi, cdw_ratio, density
//            appended, averaged over chains (Fourier%preq, src/fourier_trans.f90:251-315)
//   info.txt summary and confout.txt (src/main.f90:104-134, src/fields.f90:509-557)
//
// One chain per "rank": --chains N runs N independent chains in one batch on
// one GPU (the reference runs one per MPI rank; seeds.txt gives one seed per
// chain).  is_global runs Nglobal Wolff-in-tau moves before every bin
// (Sweep_global%sweep, src/main.f90:76) on the GPU.
//
//   z2_gauge_b200 [--chains N] [--device D] [--dir PATH]
#include <chrono>
#include <cmath>
#include <cstdint>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/z2dqmc.h"

namespace {

struct Params {
  double RT = 1, J = 0.5, h = 0.5, mu = 0, Q = 1;
  int Nlx = 4, Nly = 4, Ltrot = 40;
  double beta = 4;
  int NlxT = 4, NlyT = 4, LtrotT = 40;
  int Nwrap = 10, Nbin = 1, Nsweep = 1;
  bool is_tau = false; int Nthermal = 0;
  bool is_warm = false; int Nwarm = 0;
  bool is_global = false; int Nglobal = 0;
  int absolute = 1;
};

bool logical(const std::string &t) {
  std::string s;
  for (char c : t) if (c != '.') s += (char)std::tolower(c);
  return s == "true" || s == "t";
}

bool read_params(const std::string &path, Params &p) {
  std::ifstream f(path);
  if (!f) return false;
  std::vector<std::vector<std::string>> lines;
  std::string ln;
  while (lines.size() < 8 && std::getline(f, ln)) {
    std::istringstream is(ln);
    std::vector<std::string> tok;
    std::string t;
    while (is >> t) tok.push_back(t);
    if (!tok.empty()) lines.push_back(tok);
  }
  if (lines.size() < 8) return false;
  auto D = [&](int l, int k) { return std::atof(lines[l].at(k).c_str()); };
  auto I = [&](int l, int k) { return std::atoi(lines[l].at(k).c_str()); };
  try {   // a line with too few fields is a file that cannot be read
    p.RT = D(0, 0); p.J = D(0, 1); p.h = D(0, 2); p.mu = D(0, 3); p.Q = D(0, 4);
    p.Nlx = I(1, 0); p.Nly = I(1, 1); p.Ltrot = I(1, 2); p.beta = D(1, 3);
    p.NlxT = I(2, 0); p.NlyT = I(2, 1); p.LtrotT = I(2, 2);
    p.Nwrap = I(3, 0); p.Nbin = I(3, 1); p.Nsweep = I(3, 2);
    p.is_tau = logical(lines[4][0]); p.Nthermal = I(4, 1);
    p.is_warm = logical(lines[5][0]); p.Nwarm = I(5, 1);
    p.is_global = logical(lines[6][0]); p.Nglobal = I(6, 1);
    p.absolute = I(7, 0);
  } catch (const std::out_of_range &) {
    return false;
  }
  return true;
}

// ranf (lib/package_of_matrix/Ran/ran_imada.f:55-68)
double ranf(uint32_t &iq) {
  iq = (uint32_t)(((uint64_t)iq * 48828125ull) & 0x7fffffffull);
  return (double)iq / 2147483648.0;
}

int npbc(int nr, int L) { return nr < 1 ? nr + L : (nr > L ? nr - L : nr); }

// conf_set on the thermalisation lattice (src/fields.f90:311-427);
// sigma[(nt) * 2*LqT + b], lambda is drawn (and discarded: not on this path).
void conf_set(const Params &p, std::vector<double> &s, uint32_t &iq) {
  const int nb = 2 * p.NlxT * p.NlyT, lt = p.LtrotT;
  s.assign((size_t)nb * lt, 1.0);
  if (p.absolute == 1) {
    for (int nt = 0; nt < lt; ++nt)
      for (int b = 0; b < nb; ++b) s[(size_t)nt * nb + b] = ranf(iq) >= 0.5 ? 1.0 : -1.0;
  } else if (p.absolute == 2) {
    for (int nt = 0; nt < lt; ++nt)
      for (int b = 0; b < nb; ++b) {
        double x1 = ranf(iq), x2 = ranf(iq);
        double x = std::sqrt(-2.0 * std::log(x1)) * std::cos(2.0 * M_PI * x2);
        s[(size_t)nt * nb + b] = x >= 0.0 ? 1.0 : -1.0;
      }
  } else if (p.absolute == 4) {
    for (int nt = 0; nt < lt; ++nt)
      for (int b = 0; b < nb; ++b) {
        int site = b / 2, nx = site % p.NlxT + 1, ny = site / p.NlxT + 1;
        s[(size_t)nt * nb + b] = ((nx + ny) % 2 == 0) ? 1.0 : -1.0;
      }
  } else if (p.absolute == 5) {
    for (int b = 0; b < nb; ++b) {
      double v = ranf(iq) >= 0.5 ? 1.0 : -1.0;
      for (int nt = 0; nt < lt; ++nt) s[(size_t)nt * nb + b] = v;
    }
  }
  for (int i = 0; i < p.NlxT * p.NlyT; ++i) ranf(iq);   // lambda_random_fill
}

// conf_transfer (src/fields.f90:429-507): tile the thermalisation lattice and
// time extent up to the run size.
std::vector<double> conf_transfer(const Params &p, const std::vector<double> &st) {
  const int nb = 2 * p.Nlx * p.Nly, nbT = 2 * p.NlxT * p.NlyT;
  std::vector<double> s((size_t)nb * p.Ltrot, 1.0);
  for (int nt = 0; nt < std::min(p.LtrotT, p.Ltrot); ++nt)
    for (int b = 0; b < nb; ++b) {
      int site = b / 2, nx = site % p.Nlx + 1, ny = site / p.Nlx + 1;
      int nxt = (nx - 1) % p.NlxT + 1, nyt = (ny - 1) % p.NlyT + 1;
      int bt = (nyt - 1) * p.NlxT * 2 + (nxt - 1) * 2 + (b % 2);   // +x: 1, +y: 2 (0-based)
      s[(size_t)nt * nb + b] = st[(size_t)nt * nbT + bt];
    }
  for (int nt = p.LtrotT; nt < p.Ltrot; ++nt)
    for (int b = 0; b < nb; ++b) s[(size_t)nt * nb + b] = s[(size_t)(nt - p.LtrotT) * nb + b];
  return s;
}

void append(const std::string &dir, const char *name, double v) {
  FILE *f = std::fopen((dir + "/" + name).c_str(), "a");
  if (!f) return;
  std::fprintf(f, " %25.17E\n", v);
  std::fclose(f);
}

// ---------------------------------------------------------------------------
// Momentum-space output of the time-displaced correlators, one record per bin
// in the files of m_write_obs_tau (src/fourier_trans.f90:306-440).  The DFT
// (Fourier_R_to_K) runs on the GPU (z2_get_obs_tau_k, averaged over chains);
// the tau integration and the Matsubara transform of curxx are O(N Ltrot) and
// O(Ltrot^2) host loops.  Numbers are written with %.17g (the reference uses
// Fortran list-directed output: same values, different spacing).
// ---------------------------------------------------------------------------
struct KOut {
  const std::string &dir;
  int N, Lt, Nlx, Nly;
  double dtau, beta;
  void k_line(FILE *f, int k) const {   // Latt%xk_v(k, 1:2)
    const double PI2 = 2.0 * std::acos(-1.0);
    std::fprintf(f, " %.17g %.17g\n", (double)(k % Nlx) * PI2 / Nlx, (double)(k / Nlx) * PI2 / Nly);
  }
  FILE *open(const char *name) const { return std::fopen((dir + "/" + name).c_str(), "a"); }
  // write_reciprocal_1: per k the momentum, then gk
  void reciprocal(const char *name, const std::vector<std::complex<double>> &g) const {
    FILE *f = open(name); if (!f) return;
    for (int k = 0; k < N; ++k) { k_line(f, k); std::fprintf(f, " (%.17g,%.17g)\n", g[k].real(), g[k].imag()); }
    std::fclose(f);
  }
  // write_k_1: one momentum
  void at_k(const char *name, const std::vector<std::complex<double>> &g, int k) const {
    FILE *f = open(name); if (!f) return;
    std::fprintf(f, " %.17g %.17g\n", g[k].real(), g[k].imag());
    std::fclose(f);
  }
  // write_k_tau_2: momentum, then gk(k, tau) for every tau
  void k_tau(const char *name, const double *re, const double *im, int k) const {
    FILE *f = open(name); if (!f) return;
    k_line(f, k);
    for (int t = 0; t < Lt; ++t) std::fprintf(f, " %.17g %.17g\n", re[(size_t)t * N + k], im[(size_t)t * N + k]);
    std::fclose(f);
  }
  // integrate_susc: dtau * sum_tau gk(k, tau)
  std::vector<std::complex<double>> susc(const double *re, const double *im) const {
    std::vector<std::complex<double>> g(N, 0.0);
    for (int t = 0; t < Lt; ++t)
      for (int k = 0; k < N; ++k) g[k] += std::complex<double>(re[(size_t)t * N + k], im[(size_t)t * N + k]);
    for (auto &x : g) x *= dtau;
    return g;
  }
};

static int write_obs_tau_k(z2_handle *h, const std::string &dir, const Params &p, int nch,
                           const std::vector<double> &tau_real) {
  const int N = p.Nlx * p.Nly, Lt = p.Ltrot;
  const size_t n = (size_t)7 * Lt * N;
  std::vector<double> re(n), im(n), sr(n, 0.0), si(n, 0.0);
  for (int c = 0; c < nch; ++c) {
    if (int r = z2_get_obs_tau_k(h, c, re.data(), im.data())) return r;
    for (size_t i = 0; i < n; ++i) { sr[i] += re[i] / nch; si[i] += im[i] / nch; }
  }
  const KOut o{dir, N, Lt, p.Nlx, p.Nly, p.beta / Lt, p.beta};
  const bool has_pi = (p.Nlx % 2 == 0) && (p.Nly % 2 == 0);
  const int kzero = 0, kpi = (p.Nly / 2) * p.Nlx + p.Nlx / 2;
  const int kqx = p.Nlx > 1 ? 1 : kzero, kqy = p.Nly > 1 ? p.Nlx : kzero;
  auto R = [&](int q) { return sr.data() + (size_t)q * Lt * N; };
  auto I = [&](int q) { return si.data() + (size_t)q * Lt * N; };
  // correlator order: spin, single, pair_d, pair_s, charge_d, charge_s, curxx
  {
    auto g = o.susc(R(0), I(0));
    o.reciprocal("sdw_susc", g);
    if (has_pi) o.at_k("sdw_pipi_susc", g, kpi);
    o.at_k("sdw_zero_susc", g, kzero);
  }
  const char *cd[2][5] = {{"cdw_d_pipi_tau", "cdw_d_susc", "cdw_d_pipi_susc", "cdw_d_zero_susc", ""},
                          {"cdw_s_pipi_tau", "cdw_s_susc", "cdw_s_pipi_susc", "cdw_s_zero_susc", ""}};
  for (int w = 0; w < 2; ++w) {
    const int q = 4 + w;
    if (has_pi) o.k_tau(cd[w][0], R(q), I(q), kpi);
    auto g = o.susc(R(q), I(q));
    o.reciprocal(cd[w][1], g);
    if (has_pi) o.at_k(cd[w][2], g, kpi);
    o.at_k(cd[w][3], g, kzero);
  }
  {
    // g_r0_tau: real-space single-particle correlator at imj = Lq, / Lq
    FILE *f = o.open("g_r0_tau");
    if (f) {
      std::fprintf(f, " %d %d\n", p.Nlx, p.Nly);   // Latt%aimj_v(Lq, 1:2)
      const double *g1 = tau_real.data() + (size_t)1 * Lt * N;
      for (int t = 0; t < Lt; ++t) std::fprintf(f, " %.17g %.17g\n", g1[(size_t)t * N + N - 1] / N, 0.0);
      std::fclose(f);
    }
    auto g = o.susc(R(1), I(1));
    o.reciprocal("g_susc", g);
    if (has_pi) o.at_k("g_pipi_susc", g, kpi);
    o.at_k("g_zero_susc", g, kzero);
  }
  {
    const int q = 6;
    if (p.Nlx > 1) o.k_tau("curxx_L_tau", R(q), I(q), kqx);
    if (p.Nly > 1) o.k_tau("curxx_T_tau", R(q), I(q), kqy);
    o.k_tau("curxx_zero_tau", R(q), I(q), kzero);
    auto g = o.susc(R(q), I(q));
    // Matsubara transform of the k = 0 row (integrate_susc_freq)
    FILE *f = o.open("curxx_freq");
    if (f) {
      const double PI2 = 2.0 * std::acos(-1.0);
      for (int w = 0; w < Lt; ++w) {
        std::complex<double> s(0.0, 0.0);
        for (int t = 0; t < Lt; ++t)
          s += std::exp(std::complex<double>(0.0, PI2 * (double)t * (double)w / Lt)) *
               std::complex<double>(R(q)[(size_t)t * N], I(q)[(size_t)t * N]);
        s *= o.dtau;
        std::fprintf(f, " %.17g\n %.17g %.17g\n", PI2 * w / p.beta, s.real(), s.imag());
      }
      std::fclose(f);
    }
    o.reciprocal("curxx_susc", g);
    if (p.Nlx > 1) o.at_k("curxx_L_susc", g, kqx);
    if (p.Nly > 1) o.at_k("curxx_T_susc", g, kqy);
    o.at_k("curxx_zero_susc", g, kzero);
  }
  const char *pr[2][3] = {{"pair_s_zero_tau", "pair_s_susc", "pair_s_zero_susc"},
                          {"pair_d_zero_tau", "pair_d_susc", "pair_d_zero_susc"}};
  for (int w = 0; w < 2; ++w) {
    const int q = w == 0 ? 3 : 2;
    o.k_tau(pr[w][0], R(q), I(q), kzero);
    auto g = o.susc(R(q), I(q));
    o.reciprocal(pr[w][1], g);
    o.at_k(pr[w][2], g, kzero);
  }
  return Z2_OK;
}

int fail(z2_handle *h, const char *what, int code) {
  std::fprintf(stderr, "%s failed (%d): %s\n", what, code, h ? z2_last_error(h) : "");
  return 1;
}

}  // namespace

int main(int argc, char **argv) {
  int nch = 1, device = 0;
  std::string dir = ".";
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--chains") && i + 1 < argc) nch = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--dir") && i + 1 < argc) dir = argv[++i];
  }
  auto t0 = std::chrono::steady_clock::now();
  Params p;
  if (!read_params(dir + "/paramC_sets.txt", p)) {
    std::fprintf(stderr, "cannot read %s/paramC_sets.txt\n", dir.c_str());
    return 1;
  }
  // the sizes that conf_transfer's tiling and the stabilization divide by
  if (p.Nlx < 1 || p.Nly < 1 || p.Ltrot < 1 || p.NlxT < 1 || p.NlyT < 1 || p.LtrotT < 1 ||
      p.Nwrap < 1 || p.Nsweep < 1 || p.Nbin < 0) {
    std::fprintf(stderr, "paramC_sets.txt: lattice sizes, Ltrot, Nwrap and Nsweep must be >= 1\n");
    return 1;
  }
  if (nch < 1) { std::fprintf(stderr, "--chains must be >= 1\n"); return 1; }
  if (p.Ltrot % p.Nwrap) { std::fprintf(stderr, "Ltrot must be a multiple of Nwrap\n"); return 1; }
  const int N = p.Nlx * p.Nly, nb = 2 * N;
  // initial configurations (conf_therm_in, src/fields.f90:227-309)
  std::vector<std::vector<double>> sig(nch);
  std::vector<uint32_t> iseed(nch, 0);
  {
    std::ifstream cin_(dir + "/confin.txt");
    long long first = 0;
    if (!(cin_ >> first)) first = 0;
    if (first == 0) {
      std::ifstream sf(dir + "/seeds.txt");
      for (int c = 0; c < nch; ++c) {
        long long s = 0;
        if (!(sf >> s)) { std::fprintf(stderr, "seeds.txt has fewer than %d seeds\n", nch); return 1; }
        uint32_t iq = (uint32_t)(int32_t)s;
        std::vector<double> st;
        conf_set(p, st, iq);
        sig[c] = conf_transfer(p, st);
        iseed[c] = iq;
      }
    } else {
      // rank blocks: iseed, sigma(2*LqT, LtrotT), lambda(LqT)
      const int nbT = 2 * p.NlxT * p.NlyT;
      for (int c = 0; c < nch; ++c) {
        long long s = (c == 0) ? first : 0;
        if (c > 0 && !(cin_ >> s)) { std::fprintf(stderr, "confin.txt: missing rank %d\n", c); return 1; }
        std::vector<double> st((size_t)nbT * p.LtrotT);
        for (auto &x : st) if (!(cin_ >> x)) { std::fprintf(stderr, "confin.txt truncated\n"); return 1; }
        for (int i = 0; i < p.NlxT * p.NlyT; ++i) { double l; cin_ >> l; }
        sig[c] = conf_transfer(p, st);
        iseed[c] = (uint32_t)(int32_t)s;
      }
    }
  }
  // every output file goes to dir: one that cannot be written is an error
  // here, not lost output later
  FILE *info = std::fopen((dir + "/info.txt").c_str(), "w");
  if (!info) {
    std::fprintf(stderr, "cannot write %s/info.txt\n", dir.c_str());
    return 1;
  }
  std::fprintf(info, " ==============================================\n");
  std::fprintf(info, " Lx %d Ly %d RT %.17g J %.17g h %.17g mu %.17g Q %.17g absolute %d\n", p.Nlx,
               p.Nly, p.RT, p.J, p.h, p.mu, p.Q, p.absolute);
  std::fprintf(info, " Beta %.17g Ltrot %d Dtau %.17g Nwrap %d Nbin %d Nsweep %d chains %d\n",
               p.beta, p.Ltrot, p.beta / p.Ltrot, p.Nwrap, p.Nbin, p.Nsweep, nch);
  std::fprintf(info, " ==============================================\n");
  std::vector<z2_chain_params> cp(nch);
  for (int c = 0; c < nch; ++c)
    cp[c] = z2_chain_params{p.RT, p.J, p.h, p.mu, p.Q, p.Nlx, p.Nly, p.Ltrot, p.beta,
                            p.Nwrap, 1, 1, nullptr};
  z2_options opt{0, 0, device, p.is_tau ? 1 : 0, 1, nullptr};
  // delayed-update rank and flush tile shape from the library's autotuner
  std::vector<int32_t> kdelay(nch, 0), kshape(nch, 0);
  int r = z2_tune(cp.data(), nch, &opt, kdelay.data(), kshape.data());
  if (r) return fail(nullptr, "z2_tune", r);
  opt.delay_k_chain = kdelay.data();
  opt.flush_shape_chain = kshape.data();
  z2_handle *h = nullptr;
  r = z2_create(&h, cp.data(), nch, &opt);
  if (r) return fail(h, "z2_create", r);
  for (int c = 0; c < nch; ++c)
    if ((r = z2_set_config(h, c, sig[c].data(), (int32_t)iseed[c]))) return fail(h, "z2_set_config", r);
  // boson-only warm-up on the GPU (src/main.f90:38-67)
  if (p.is_warm && p.Nwarm > 0) {
    std::vector<double> wacc(nch, 0.0);
    if ((r = z2_therm(h, p.Nwarm, wacc.data()))) return fail(h, "z2_therm", r);
    double acc = 0.0;
    for (double a : wacc) acc += a / nch;
    std::fprintf(info, " Thermalize Accept Ratio : %.17g\n", acc);
  }
  if ((r = z2_pre(h))) return fail(h, "z2_pre", r);
  const char *names[7] = {"flux_avg", "chi_flux", "pair_sc_q0", "cdw_pi", "cdw_shift", "cdw_ratio", "density"};
  std::vector<double> tau((size_t)7 * N * p.Ltrot), tau_sum;
  for (int nbc = 1; nbc <= p.Nbin; ++nbc) {
    const bool istau = p.is_tau && nbc > p.Nthermal;
    if (p.is_global && (r = z2_sweep_global(h, p.Nglobal))) return fail(h, "z2_sweep_global", r);
    if ((r = z2_sweep(h, p.Nsweep, istau ? 1 : 0))) return fail(h, "z2_sweep", r);
    double mean[7] = {0};
    for (int c = 0; c < nch; ++c) {
      double o[Z2_NOBS_EQ];
      if ((r = z2_get_obs_equal(h, c, o))) return fail(h, "z2_get_obs_equal", r);
      for (int q = 0; q < 7; ++q) mean[q] += o[q] / nch;
    }
    for (int q = 0; q < 7; ++q) if (q != 4) append(dir, names[q], mean[q]);
    if (istau) {   // raw time-displaced correlators, averaged over chains
      tau_sum.assign(tau.size(), 0.0);
      for (int c = 0; c < nch; ++c) {
        if ((r = z2_get_obs_tau(h, c, tau.data()))) return fail(h, "z2_get_obs_tau", r);
        for (size_t i = 0; i < tau.size(); ++i) tau_sum[i] += tau[i] / nch;
      }
      FILE *f = std::fopen((dir + "/obs_tau_raw").c_str(), "a");
      if (f) { for (double v : tau_sum) std::fprintf(f, " %25.17E\n", v); std::fclose(f); }
      if ((r = write_obs_tau_k(h, dir, p, nch, tau_sum))) return fail(h, "z2_get_obs_tau_k", r);
    }
    if (nbc % 20 == 0) {
      double acc = 0;
      for (int c = 0; c < nch; ++c) {
        double st[Z2_NSTATS];
        if ((r = z2_get_stats(h, c, st))) return fail(h, "z2_get_stats", r);
        acc += st[0];
      }
      std::fprintf(info, " Progress %d : Accept_Klocal_shift: %.17g\n", nbc, acc / (nch * nbc));
      if (p.is_global) {
        double ga = 0;
        for (int c = 0; c < nch; ++c) {
          double g[5];
          if ((r = z2_get_global_stats(h, c, g))) return fail(h, "z2_get_global_stats", r);
          ga += g[0];
        }
        std::fprintf(info, " Progress %d : Accept_Kglobal: %.17g\n", nbc, ga / (nch * nbc));
      }
    }
  }
  double acc = 0, xmax = 0, xmean = 0;
  for (int c = 0; c < nch; ++c) {
    double st[Z2_NSTATS];
    if ((r = z2_get_stats(h, c, st))) return fail(h, "z2_get_stats", r);
    acc += st[0]; xmax = std::max(xmax, st[1]); xmean += st[2];
  }
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (p.is_global) {   // Global_control_print (src/global_update.f90:339-354)
    double ga = 0, gs = 0;
    for (int c = 0; c < nch; ++c) {
      double g[5];
      if ((r = z2_get_global_stats(h, c, g))) return fail(h, "z2_get_global_stats", r);
      ga += g[0];
      gs += g[1];
    }
    std::fprintf(info, " Average size of Wolff cluster : %.17g\n", gs / (nch * p.Nbin));
    std::fprintf(info, " Accept_Kglobal                : %.17g\n", ga / (nch * p.Nbin));
  }
  std::fprintf(info, " Accept_Klocal_shift : %.17g\n", acc / (nch * p.Nbin));
  std::fprintf(info, " Max diff Matrix     : %.17g\n", xmax);
  std::fprintf(info, " Mean diff Matrix    : %.17g\n",
               xmean / (2.0 * nch * p.Nbin * (p.Ltrot / p.Nwrap) * p.Nsweep));
  std::fprintf(info, " Tot CPU time        : %.10g\n", secs);
  std::fclose(info);
  // conf_out (src/fields.f90:509-557)
  FILE *co = std::fopen((dir + "/confout.txt").c_str(), "w");
  if (!co) {
    std::fprintf(stderr, "cannot write %s/confout.txt\n", dir.c_str());
    return 1;
  }
  for (int c = 0; c < nch; ++c) {
    std::vector<double> s((size_t)nb * p.Ltrot);
    int32_t is = 0;
    if ((r = z2_get_config(h, c, s.data(), &is))) return fail(h, "z2_get_config", r);
    std::fprintf(co, " %d\n", is);
    for (double v : s) std::fprintf(co, " %.1f\n", v);
    for (int i = 0; i < N; ++i) std::fprintf(co, " 1.0\n");
  }
  std::fclose(co);
  z2_destroy(h);
  return 0;
}
