/*
 * z2dqmc.h -- C ABI of the B200 (sm_100a) DQMC library for spinful fermions
 * coupled to a Z2 lattice gauge field.
 *
 * The library replaces the hot path of the Fortran program z2_gauge.out
 * (SONY932/z2_gauge_zfy).  Each entry point names the reference module
 * procedure it stands in for (file:line relative to the reference root).
 * The reference keeps its state in module globals (src/model.f90:10-13,
 * src/local_sweep.f90:27-29, src/stabilization.f90:10-17); here that state
 * lives in an opaque handle that owns the device memory of a batch of
 * independent Markov chains (one chain = one MPI rank of the reference).
 *
 * Conventions
 *  - Every call returns an int status (z2_status); z2_last_error() gives text.
 *    A null handle, a chain index out of range or a null buffer that the call
 *    must read or write returns Z2_ERR_ARG before any device work; outputs
 *    documented as optional may be null.  z2_destroy(NULL) does nothing.
 *  - All matrices are real float64, column-major N x N, N = Nlx*Nly (the
 *    reference stores complex(kind=8) but every entry is real).
 *  - sigma is float64 (+1/-1) laid out as the Fortran array sigma(2*N, Ltrot).
 *  - Time-slice numbers nt follow the reference (1..Ltrot, 0 for the
 *    boundary), bond numbers are 0-based (reference bond ii -> ii-1).
 *  - Calls are synchronous on the handle's stream; the library copies into
 *    and out of caller-owned host buffers.  A handle is not thread-safe.
 */
#ifndef Z2DQMC_H
#define Z2DQMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum z2_status {
  Z2_OK = 0,
  Z2_ERR_ARG = 1,        /* invalid argument (the reference would `stop`) */
  Z2_ERR_CUDA = 2,       /* a CUDA runtime call failed */
  Z2_ERR_NONFINITE = 3,  /* NaN/Inf in a Green's function or a D factor */
  Z2_ERR_STATE = 4,      /* call out of order (e.g. sweep before pre) */
  Z2_ERR_NOMEM = 5,      /* device allocation failed */
  Z2_ERR_TIMEOUT = 6     /* a bounded device-side wait gave up */
};

/* Number of doubles returned by z2_get_obs_equal: flux_avg, chi_flux,
 * pair_sc_q0, cdw_pi, cdw_shift, cdw_ratio, density (the fields written by
 * Obs_equal_ave, src/obser_equal.f90:50-71). */
#define Z2_NOBS_EQ 7
/* Number of time-displaced correlators (src/obser_tau.f90:9-10), in the
 * order spin, single, pair_d, pair_s, charge_d, charge_s, curxx. */
#define Z2_NOBS_TAU 7
/* Number of doubles returned by z2_get_stats: acc (sum over bins of the
 * accepted fraction, AccCounter%acc), Xmaxm, Xmeanm (Propagator drift,
 * src/process_matrix.f90:10), Xmaxm(1:3), Xmeanm(1:3) of the time-displaced
 * chain (src/process_matrix.f90:20), accepted, proposed (this bin),
 * rng draws so far, nobs, nobst. */
#define Z2_NSTATS 14

/* One chain's parameters: the lines of paramC_sets.txt that the hot path
 * reads (src/calc_basic.f90:52-62) plus this chain's seed (seeds.txt). */
typedef struct z2_chain_params {
  double RT, J, h, mu, Q;       /* line 1 */
  int32_t Nlx, Nly, Ltrot;      /* line 2 */
  double beta;                  /* line 2 */
  int32_t Nwrap;                /* line 4 */
  int32_t absolute;             /* line 8: initial sigma mode 1..5 */
  int32_t seed;                 /* seeds.txt row of this chain */
  const double *rt_bond;        /* optional [2N] per-bond hopping, NULL = RT */
} z2_chain_params;

typedef struct z2_options {
  int32_t delay_k;   /* accepted flips queued before a rank-2k flush; 0 = tuned */
  int32_t record;    /* 1: keep decisions and ratios of each half-sweep */
  int32_t device;    /* CUDA device ordinal */
  int32_t tau;       /* 1: allocate the time-displaced chain (is_tau) */
  int32_t graph;     /* 1: capture each bin's launch as a CUDA graph, replayed */
  const int32_t *delay_k_chain;  /* optional [nchains] per-chain delay rank (autotuner) */
  const int32_t *flush_shape_chain;  /* optional [nchains] tile shape of each chain's
                          rank-2k flush (z2_tune picks it; 0 = by divisibility):
                          1 bounded 16x16 groups, 2 bounded 8x8 groups, 3 8x8
                          blocks (8 | N), 4 16x16 (16 | N), 5 24x24 (24 | N),
                          6 16x8 (16 | N), 7 24x16 (48 | N).  All shapes give
                          the same bits. */
  int32_t stab_exact;  /* 1: stabilize with the reference's column-pivoted QR
                          (ZGEQP3) and its stab_green branches; 0: pre-pivoted
                          blocked QR and the scale-split Green's function (the
                          same U D V products and G up to rounding, faster on
                          the GPU).  The module-level z2_stab_* mirrors always
                          use the reference's pivoted QR. */
} z2_options;

typedef struct z2_handle z2_handle;

/* ---- life cycle: Model_init + Prop/WrapList make + Stabilize_init
 *      (src/model.f90:16-36, src/process_matrix.f90:46-112,
 *       src/stabilization.f90:20-32); the initial sigma follows conf_set +
 *      conf_transfer (src/fields.f90:311-507) from each chain's seed.
 *      Unless out or params is NULL or nchains < 1, *out receives a handle
 *      even when the call fails: z2_last_error() on it says why, and
 *      z2_destroy() releases it. ---- */
int z2_create(z2_handle **out, const z2_chain_params *params, int32_t nchains,
              const z2_options *opt);
int z2_destroy(z2_handle *h);
const char *z2_last_error(const z2_handle *h);
/* N, Ltrot and Nst (= Ltrot / Nwrap) of one chain; each output is optional. */
int z2_chain_dims(const z2_handle *h, int32_t chain, int32_t *N, int32_t *Ltrot,
                  int32_t *Nst);

/* ---- configuration I/O: conf_in / conf_out (src/fields.f90:214-309,
 *      509-557).  iseed is the ranf state that continues the chain. ---- */
int z2_set_config(z2_handle *h, int32_t chain, const double *sigma, int32_t iseed);
/* sigma and iseed are each optional outputs. */
int z2_get_config(const z2_handle *h, int32_t chain, double *sigma, int32_t *iseed);

/* ---- Local_sweep%pre (src/local_sweep.f90:87-104) on every chain ---- */
int z2_pre(z2_handle *h);
/* ---- Local_sweep%sweep (src/local_sweep.f90:152-195): one bin of nsweep
 *      (sweep_L, sweep_R) pairs on every chain; toggle = is_tau for this
 *      bin (runs Dyn%reset/sweep_R, src/dynamics.f90:41-62).  The whole bin
 *      of every chain runs in one persistent launch. ---- */
int z2_sweep(z2_handle *h, int32_t nsweep, int32_t toggle);
/* Same as z2_sweep, also returning the device time of the launch (ms; optional). */
int z2_sweep_timed(z2_handle *h, int32_t nsweep, int32_t toggle, float *ms);

/* ---- readback ---- */
int z2_get_green(const z2_handle *h, int32_t chain, double *G);
int z2_get_obs_equal(const z2_handle *h, int32_t chain, double out[Z2_NOBS_EQ]);
/* The bin observables of every chain, out[nchains][Z2_NOBS_EQ] (chain-major),
 * gathered on the device and read back with one copy (what z2_get_obs_equal
 * gives chain by chain; Obs_equal%ave of every rank, src/obser_equal.f90:50-71,
 * before the driver's MPI reduction).  The first call allocates the gather
 * buffer. */
int z2_get_obs_equal_all(z2_handle *h, double *out);
/* out: Z2_NOBS_TAU arrays of (N, Ltrot) column-major, real parts (the
 * imaginary parts of ObserTau are identically zero for real G). */
int z2_get_obs_tau(const z2_handle *h, int32_t chain, double *out);
/* The same correlators in momentum space: Fourier_R_to_K (FFT_RtoK_2,
 * src/lattice.f90:263-281) as applied by the reference's output layer
 * (m_write_obs_tau, src/fourier_trans.f90:306-440),
 *   gk(k, tau) = (1/N) sum_r exp(i k.r) g(r, tau),
 * k = ((ix-1) 2pi/Nlx, (iy-1) 2pi/Nly) and r = (ix, iy) in the site order
 * (x fastest), computed on the GPU.  re, im: [7][Ltrot][N] each, momentum
 * index in place of the distance index of z2_get_obs_tau.  Needs a handle
 * created with z2_options.tau = 1 (else Z2_ERR_STATE). */
int z2_get_obs_tau_k(const z2_handle *h, int32_t chain, double *re, double *im);
int z2_get_stats(const z2_handle *h, int32_t chain, double out[Z2_NSTATS]);
/* Replay: use r[0..n) instead of ranf for the next n proposals (n = 0
 * restores ranf).  Decisions/ratios of the last half-sweeps, in the order
 * (half-sweep L then R, slice nt = 1..Ltrot, bond 0..2N-1). */
int z2_set_replay(z2_handle *h, int32_t chain, const double *r, size_t n);
/* Tracing: SM clock cycles spent by the chain's CTA in each phase since
 * z2_create, accumulated over all z2_sweep calls (no reference counterpart;
 * the reference only records total wall time, src/main.f90:27-28,114-122).
 * out[Z2_NPHASE]: checkerboard wrap of G, proposals, rank-2k flushes,
 * equal-time observables, wraps + stabilization, time-displaced chain, and
 * nested in those: UDV stabilization, stabilized G, flip-ratio rounds,
 * accepted-flip X/Y columns, pending slice products, UDV stack copies. */
#define Z2_NPHASE 12
int z2_get_phase_cycles(const z2_handle *h, int32_t chain, double out[Z2_NPHASE]);
/* Global Wolff-in-tau moves: Global_sweep (src/global_update.f90:320-337)
 * for every chain, nglobal moves each.  A move picks a bond and grows a
 * cluster of its links along tau (build_time_cluster, :103-131, flip
 * probability 1 - tanh(dtau h)), adds the plaquette log ratio (:133-172),
 * runs a trial half-sweep in the chain's current direction with the
 * cluster's links flipped (GlobalK_prop_L/R, src/globalK.f90:115-153) and
 * accepts with min(1, ratio); an accepted move reverses the direction of the
 * next bin (is_beta, src/main.f90:73-77; z2_sweep honours it).  The first
 * call allocates a backup of each chain's state that a rejected move
 * restores.  Call after z2_pre. */
int z2_sweep_global(z2_handle *h, int32_t nglobal);
/* Boson-only warm-up (Local_sweep_therm, src/local_sweep.f90:73-85, and
 * LocalK_therm, src/localK.f90:400-420; src/main.f90:38-67): nwarm sweeps of
 * single-link Metropolis on the gauge weight alone for every chain, on the
 * GPU.  acc (optional, [nchains]) receives each chain's mean accepted
 * fraction (Acc_Kt%acc / nwarm).  Changes sigma: call before z2_pre. */
int z2_therm(z2_handle *h, int32_t nwarm, double *acc);
/* out[5]: Acc_Kg%acc (sum over calls of the accepted fraction), Wolff
 * size_cluster (sum over calls of the mean cluster size), accepted and
 * proposed moves of the last call, is_beta (1 or 0). */
int z2_get_global_stats(const z2_handle *h, int32_t chain, double out[5]);
/* Delay-rank autotuner (no reference counterpart: the reference applies each
 * accepted flip to G at once, src/localK.f90:141-165).  For every distinct
 * lattice size among params[0..nchains) it times one bin of short probe
 * chains (the chain's couplings and time step, Ltrot cut to 2*Nwrap) at the
 * ranks 4, 6, 8, 12, 16, 24, 32, 48, 64 (capped by shared memory) and writes
 * the fastest rank of each chain's size to k_out[nchains], ready to pass as
 * z2_options.delay_k_chain.  Uses opt->device (opt may be NULL: device 0);
 * allocates and frees its own probe handles. */
int z2_tune_delay(const z2_chain_params *params, int32_t nchains, const z2_options *opt,
                  int32_t *k_out);
/* Joint autotuner of the delayed-update rank and the flush tile shape (no
 * reference counterpart).  For every distinct lattice size it times one bin of
 * three short probe chains per candidate (the chain's couplings and time step,
 * Ltrot cut to 2*Nwrap; ranks 4..64 as z2_tune_delay, capped by shared memory,
 * times every flush shape valid for N) by the SM cycles of the chain kernel,
 * takes the median over the three probes, and picks, in the order (default
 * shape first, then smaller rank), the first candidate within 3 % of the
 * fastest, so that repeated runs pick the same configuration.  k_out and
 * shape_out [nchains] are ready to pass as z2_options.delay_k_chain and
 * flush_shape_chain. */
int z2_tune(const z2_chain_params *params, int32_t nchains, const z2_options *opt,
            int32_t *k_out, int32_t *shape_out);
/* The first n recorded decisions and ratios of one chain; dec and ratios are
 * each optional. */
int z2_get_decisions(const z2_handle *h, int32_t chain, uint8_t *dec,
                     double *ratios, size_t n);

/* ---- adjoint (no reference routine): log|det(1 + B_Ltrot...B_1)| of one
 *      spin sector and its gradient wrt the 2N per-bond hopping amplitudes
 *      and mu, at the chain's current sigma; each output is optional. ---- */
int z2_logdet_grad(z2_handle *h, int32_t chain, double *logdet,
                   double *dlogdet_dt, double *dlogdet_dmu);

/* ---- module-level mirrors on single matrices (host buffers) ----
 * OperatorKin%mmult_R / mmult_L (src/operator_kin.f90:61-86, 122-145):
 *   M <- B_nt^nflag M   /   M <- M B_nt^nflag, with the chain's sigma. */
int z2_opk_mmult_R(z2_handle *h, int32_t chain, double *M, int32_t nt, int32_t nflag);
int z2_opk_mmult_L(z2_handle *h, int32_t chain, double *M, int32_t nt, int32_t nflag);
/* stab_UR / stab_UL (src/stabilization.f90:70-120): in-place U, D, V. */
int z2_stab_UR(z2_handle *h, int32_t chain, double *U, double *D, double *V);
int z2_stab_UL(z2_handle *h, int32_t chain, double *U, double *D, double *V);
/* stab_green (src/stabilization.f90:122-200). */
int z2_stab_green(z2_handle *h, int32_t chain, const double *UR, const double *DR,
                  const double *VR, const double *UL, const double *DL,
                  const double *VL, int32_t nt, double *G);
/* stab_green_big (src/stabilization.f90:202-264). */
int z2_stab_green_big(z2_handle *h, int32_t chain, const double *UR,
                      const double *DR, const double *VR, const double *UL,
                      const double *DL, const double *VL, double *G00,
                      double *G0t, double *Gt0, double *Gtt);

/* ---- module-level mirrors on a chain's resident state ----
 * Each call runs one procedure of the reference's modules on one chain of the
 * handle, on the state the handle keeps on the device between calls, so that
 * a driver can replace the modules one at a time:
 *   Propagator   G, UR DR VR, UL DL VL (src/process_matrix.f90:7-12)
 *   WrapList     the UDV stacks of both chains (src/process_matrix.f90:26-31)
 *   Dyn copy     the propagator copy and PropGreen G00, G0t, Gt0, Gtt of the
 *                time-displaced chain (src/dynamics.f90:8-12)
 *   sigma, the ranf state, the observable sums of the bin.
 * nt is a slice 1..Ltrot for per-slice procedures and a stabilization point
 * (a multiple of Nwrap, 0..Ltrot) for the wraps; anything else is Z2_ERR_ARG.
 * The Fortran module procedures take both spin sectors (PropU, PropD); the
 * sectors are identical, so one call covers both.
 * multiply (src/multiply.f90:8-130): */
int z2_propK_pre(z2_handle *h, int32_t chain, int32_t nt);  /* UR <- B_nt UR (RT > Zero)    */
int z2_propK_L(z2_handle *h, int32_t chain, int32_t nt);    /* G <- B^-1 G B, UL <- UL B    */
int z2_propK_R(z2_handle *h, int32_t chain, int32_t nt);    /* G <- B G B^-1, UR <- B UR    */
int z2_propgrK_R(z2_handle *h, int32_t chain, int32_t nt);  /* Gt0 <- B Gt0, G0t <- G0t B^-1,
                                                               Gtt <- B Gtt B^-1, Dyn UR <- B UR */
int z2_propT_pre(z2_handle *h, int32_t chain);  /* UR *= e^{dtau mu}                          */
int z2_propT_L(z2_handle *h, int32_t chain);    /* G *= e^{dtau mu} e^{-dtau mu}, UL *= e^{..} */
int z2_propT_R(z2_handle *h, int32_t chain);    /* G likewise, UR *= e^{dtau mu}              */
int z2_propgrT_R(z2_handle *h, int32_t chain);  /* the mu factors of propgrT_R               */
/* stabilization (src/stabilization.f90:374-514); flag = Xmeanm is accumulated
 * (the reference's `flag` argument of Wrap_L / Wrap_R). */
int z2_wrap_pre(z2_handle *h, int32_t chain, int32_t nt);
int z2_wrap_L(z2_handle *h, int32_t chain, int32_t nt, int32_t flag);
int z2_wrap_R(z2_handle *h, int32_t chain, int32_t nt, int32_t flag);
int z2_wrap_tau(z2_handle *h, int32_t chain, int32_t nt);    /* nt >= Nwrap, on the Dyn copy */
/* dynamics: Dyn_reset (src/dynamics.f90:41-48) */
int z2_dyn_reset(z2_handle *h, int32_t chain);
/* localK: LocalK_prop_L / LocalK_prop_R (src/localK.f90:347-398), the slice's
 * 2N flip proposals with its propagation (decisions recorded as by z2_sweep
 * when the handle records them). */
int z2_prop_slice_L(z2_handle *h, int32_t chain, int32_t nt);
int z2_prop_slice_R(z2_handle *h, int32_t chain, int32_t nt);
/* local_sweep: Local_sweep_reset (src/local_sweep.f90:56-71) */
int z2_sweep_reset(z2_handle *h, int32_t chain, int32_t toggle);
/* obser_equal / obser_tau: calc adds slice nt to the bin's sums
 * (src/obser_equal.f90:73-149, src/obser_tau.f90:56-133); ave divides them by
 * the count (src/obser_equal.f90:50-71, src/obser_tau.f90:37-47) into what
 * z2_get_obs_equal / z2_get_obs_tau read. */
int z2_obs_equal_calc(z2_handle *h, int32_t chain, int32_t nt);
int z2_obs_equal_ave(z2_handle *h, int32_t chain, int32_t nobs);
int z2_obs_tau_calc(z2_handle *h, int32_t chain, int32_t nt);
int z2_obs_tau_ave(z2_handle *h, int32_t chain, int32_t nobst);
/* State transfer: the Propagator (each buffer optional; N x N column-major,
 * D vectors of length N) and the PropGreen of the Dyn copy. */
int z2_get_prop(const z2_handle *h, int32_t chain, double *G, double *UR, double *DR,
                double *VR, double *UL, double *DL, double *VL);
int z2_set_prop(z2_handle *h, int32_t chain, const double *G, const double *UR,
                const double *DR, const double *VR, const double *UL, const double *DL,
                const double *VL);
int z2_get_propgr(const z2_handle *h, int32_t chain, double *G00, double *G0t, double *Gt0,
                  double *Gtt);

/* ---- allocation-free stab_green.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc (their device memory is owned by
 * another allocator, e.g. a framework's caching allocator or a driver that
 * reserves one pool at start-up): same result as z2_stab_green, but UR, DR,
 * VR, UL, DL, VL (inputs) and G (output) are caller-owned DEVICE pointers,
 * column-major N x N (DR, DL of length N), and no memory is allocated.  The
 * scratch is a file-scope device array of 5 * Z2_NOALLOC_NMAX^2 doubles
 * (829,440 bytes) that every GPU loading this library holds until exit.
 * N > Z2_NOALLOC_NMAX (or N < 1, nt outside 0..Ltrot, a null pointer) is
 * rejected with Z2_ERR_ARG.  The work is enqueued on `stream` (a
 * cudaStream_t, NULL = default stream); the call returns after the launch.
 * The first call on a device looks up the device address of the scratch
 * array (cudaGetSymbolAddress) with that device current, and so does the
 * first call after the device's context changes (e.g. after
 * cudaDeviceReset); make such a call before any stream capture.  Every call
 * shares the one scratch array,
 * so calls that overlap on the GPU (other streams, other host threads) race;
 * no part of the scratch needs to start at zero. ---- */
#define Z2_NOALLOC_NMAX 144
int z2_stab_green_noalloc(int32_t N, int32_t nt, int32_t Ltrot, const double *UR,
                          const double *DR, const double *VR, const double *UL,
                          const double *DL, const double *VL, double *G, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* Z2DQMC_H */
