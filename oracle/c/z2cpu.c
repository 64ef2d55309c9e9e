/*
 * z2cpu.c -- CPU restatement of the reference DQMC local sweep, in C
 * (TEST INFRASTRUCTURE and the timed CPU baseline; never the product).
 *
 * Same algorithm and order of operations as oracle/z2_oracle.py, which
 * restates src/local_sweep.f90, src/localK.f90, src/multiply.f90,
 * src/operator_kin.f90, src/stabilization.f90, src/obser_equal.f90 and
 * src/fields.f90 of the reference.  LAPACK/BLAS calls go to the reference
 * LAPACK routines of SciPy's bundled OpenBLAS (dgeqp3, dorgqr, dormqr, dtrmm,
 * dtrsm, dgemm), single-threaded, one chain per process (the reference runs
 * one chain per MPI rank).
 *
 * As a baseline it is a lower bound on the reference's cost: it keeps one of
 * the two bit-identical spin sectors and real arithmetic (the reference
 * repeats every step for PropU and PropD in complex(kind=8)).
 *
 * Parity status: cross-checked against the NumPy oracle
 * (tests/test_cpu_port.py), which replays the reference's own recorded run
 * (tests/test_oracle_testrun.py); the reference itself cannot be built here.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

extern void scipy_dgeqp3_(const int *, const int *, double *, const int *, int *, double *,
                          double *, const int *, int *);
extern void scipy_dorgqr_(const int *, const int *, const int *, double *, const int *,
                          const double *, double *, const int *, int *);
extern void scipy_dormqr_(const char *, const char *, const int *, const int *, const int *,
                          const double *, const int *, const double *, double *, const int *,
                          double *, const int *, int *, size_t, size_t);
extern void scipy_dtrmm_(const char *, const char *, const char *, const char *, const int *,
                         const int *, const double *, const double *, const int *, double *,
                         const int *, size_t, size_t, size_t, size_t);
extern void scipy_dtrsm_(const char *, const char *, const char *, const char *, const int *,
                         const int *, const double *, const double *, const int *, double *,
                         const int *, size_t, size_t, size_t, size_t);
extern void scipy_dgemm_(const char *, const char *, const int *, const int *, const int *,
                         const double *, const double *, const int *, const double *,
                         const int *, const double *, double *, const int *, size_t, size_t);
extern void scipy_openblas_set_num_threads(int);

#define IX(i, j) ((size_t)(i) + (size_t)(j) * (size_t)N)

typedef struct {
  /* parameters */
  double RT, J, h, mu, beta, dtau, alpha, alpha2, eP, eM;
  int Lx, Ly, N, nb, Ltrot, Nwrap, Nst;
  /* lattice */
  int *bond;      /* [nb][2] */
  int *grp;       /* [4][N/2] */
  int gsz[4];
  int *bb;        /* [nb][7] */
  int *xy;        /* [N][2] */
  int *plaq;      /* [N][4] */
  /* state */
  double *sigma;  /* [Ltrot][nb] */
  uint32_t iq;
  double *G, *UR, *VR, *DR, *UL, *VL, *DL;
  double *URs, *VRs, *DRs, *ULs, *VLs, *DLs;
  double *T1, *T2, *T3, *work;
  int lwork, *jpvt;
  double *tau, *Dn;
  /* accumulators */
  double flux_sum, flux_sq, pair, cdw, cdws, dens, nobs;
  double acc_num, acc_den, Xmaxm, Xmeanm, acc_sum;
  unsigned char *dec;   /* optional [2][Ltrot][nb] */
} Chain;

static double ranf(uint32_t *iq) {   /* lib/package_of_matrix/Ran/ran_imada.f:55-68 */
  *iq = (uint32_t)(((uint64_t)*iq * 48828125ull) & 0x7fffffffull);
  return (double)*iq / 2147483648.0;
}

static int npbc(int nr, int L) { return nr < 1 ? nr + L : (nr > L ? nr - L : nr); }

static void lattice(Chain *c) {   /* src/lattice.f90:25-141 */
  int Lx = c->Lx, Ly = c->Ly, N = c->N;
  int *inv = malloc(sizeof(int) * (Lx + 1) * (Ly + 1));
  int *ib = malloc(sizeof(int) * N * N);
  c->xy = malloc(sizeof(int) * 2 * N);
  int nc = 0;
  for (int ny = 1; ny <= Ly; ++ny)
    for (int nx = 1; nx <= Lx; ++nx, ++nc) { c->xy[2 * nc] = nx; c->xy[2 * nc + 1] = ny; inv[nx + ny * (Lx + 1)] = nc; }
#define SITE(x, y) inv[(x) + (y) * (Lx + 1)]
  c->bond = malloc(sizeof(int) * 2 * c->nb);
  for (int i = 0; i < N * N; ++i) ib[i] = -1;
  nc = 0;
  for (int ny = 1; ny <= Ly; ++ny)
    for (int nx = 1; nx <= Lx; ++nx) {
      int ii = SITE(nx, ny), ix = SITE(npbc(nx + 1, Lx), ny), iy = SITE(nx, npbc(ny + 1, Ly));
      c->bond[2 * nc] = ii; c->bond[2 * nc + 1] = ix; ib[ii * N + ix] = nc; ++nc;
      c->bond[2 * nc] = ii; c->bond[2 * nc + 1] = iy; ib[ii * N + iy] = nc; ++nc;
    }
  c->grp = malloc(sizeof(int) * c->nb);
  int cnt[4] = {0, 0, 0, 0};
  int *g[4];
  for (int q = 0; q < 4; ++q) g[q] = malloc(sizeof(int) * c->nb);
  for (nc = 0; nc < c->nb; ++nc) {
    int ii = c->bond[2 * nc], jj = c->bond[2 * nc + 1];
    int ixc = c->xy[2 * ii], iyc = c->xy[2 * ii + 1], jxc = c->xy[2 * jj], jyc = c->xy[2 * jj + 1];
    int q = -1;
    if (npbc(ixc + 1, Lx) == jxc) q = (ixc % 2 == 0) ? 0 : 1;
    else if (npbc(iyc + 1, Ly) == jyc) q = (iyc % 2 == 0) ? 2 : 3;
    if (q >= 0) g[q][cnt[q]++] = nc;
  }
  int off = 0;
  for (int q = 0; q < 4; ++q) { memcpy(c->grp + off, g[q], sizeof(int) * cnt[q]); c->gsz[q] = cnt[q]; off += cnt[q]; free(g[q]); }
  c->bb = malloc(sizeof(int) * 7 * c->nb);
  for (nc = 0; nc < c->nb; ++nc) {
    int ii = c->bond[2 * nc], jj = c->bond[2 * nc + 1];
    int ixc = c->xy[2 * ii], iyc = c->xy[2 * ii + 1], jxc = c->xy[2 * jj], jyc = c->xy[2 * jj + 1];
    int *o = c->bb + 7 * nc;
    o[0] = nc;
    if (npbc(ixc + 1, Lx) == jxc) {
      int nx = SITE(ixc, npbc(iyc + 1, Ly)); o[1] = ib[ii * N + nx];
      int ny = SITE(jxc, npbc(jyc + 1, Ly)); o[2] = ib[nx * N + ny]; o[3] = ib[jj * N + ny];
      nx = SITE(ixc, npbc(iyc - 1, Ly)); o[4] = ib[nx * N + ii];
      ny = SITE(jxc, npbc(jyc - 1, Ly)); o[5] = ib[nx * N + ny]; o[6] = ib[ny * N + jj];
    } else {
      int nx = SITE(npbc(jxc - 1, Lx), jyc); o[1] = ib[nx * N + jj];
      int ny = SITE(npbc(ixc - 1, Lx), iyc); o[2] = ib[ny * N + nx]; o[3] = ib[ny * N + ii];
      nx = SITE(npbc(jxc + 1, Lx), jyc); o[4] = ib[jj * N + nx];
      ny = SITE(npbc(ixc + 1, Lx), iyc); o[5] = ib[ny * N + nx]; o[6] = ib[ii * N + ny];
    }
  }
  c->plaq = malloc(sizeof(int) * 4 * N);   /* src/obser_equal.f90:84-96 */
  for (int s = 0; s < N; ++s) {
    int x = c->xy[2 * s], y = c->xy[2 * s + 1];
    int right = SITE(npbc(x + 1, Lx), y), up = SITE(x, npbc(y + 1, Ly));
    int diag = SITE(npbc(c->xy[2 * up] + 1, Lx), c->xy[2 * up + 1]);
    int rup = SITE(c->xy[2 * right], npbc(c->xy[2 * right + 1] + 1, Ly));
    c->plaq[4 * s] = ib[s * N + right]; c->plaq[4 * s + 1] = ib[right * N + rup];
    c->plaq[4 * s + 2] = ib[up * N + diag]; c->plaq[4 * s + 3] = ib[s * N + up];
  }
#undef SITE
  free(inv);
  free(ib);
}

/* ---- checkerboard (src/operator_kin.f90:61-179) ---- */
static const int GORDER[8] = {0, 1, 2, 3, 3, 2, 1, 0};

static void mmult_R(Chain *c, double *M, int nt, int nflag) {   /* M <- B^nflag M */
  const int N = c->N;
  const double *sg = c->sigma + (size_t)nt * c->nb;
  for (int p = 0; p < 8; ++p) {
    int g = GORDER[p], off = 0;
    for (int q = 0; q < g; ++q) off += c->gsz[q];
    for (int k = 0; k < c->gsz[g]; ++k) {
      int b = c->grp[off + k];
      double x = nflag * c->alpha * sg[b];
      double C = cosh(x), S = sinh(x);
      int p1 = c->bond[2 * b], p2 = c->bond[2 * b + 1];
      for (int j = 0; j < N; ++j) {
        double a = M[IX(p1, j)], bb = M[IX(p2, j)];
        M[IX(p1, j)] = C * a + S * bb;
        M[IX(p2, j)] = S * a + C * bb;
      }
    }
  }
}

static void mmult_L(Chain *c, double *M, int nt, int nflag) {   /* M <- M B^nflag */
  const int N = c->N;
  const double *sg = c->sigma + (size_t)nt * c->nb;
  for (int p = 0; p < 8; ++p) {
    int g = GORDER[p], off = 0;
    for (int q = 0; q < g; ++q) off += c->gsz[q];
    for (int k = 0; k < c->gsz[g]; ++k) {
      int b = c->grp[off + k];
      double x = nflag * c->alpha * sg[b];
      double C = cosh(x), S = sinh(x);
      int p1 = c->bond[2 * b], p2 = c->bond[2 * b + 1];
      for (int i = 0; i < N; ++i) {
        double a = M[IX(i, p1)], bb = M[IX(i, p2)];
        M[IX(i, p1)] = a * C + bb * S;
        M[IX(i, p2)] = a * S + bb * C;
      }
    }
  }
}

static void scale(double *M, size_t n, double f) { for (size_t i = 0; i < n; ++i) M[i] = M[i] * f; }

/* ---- boson ratio (src/fields.f90:40-119) ---- */
static double boson_ratio(Chain *c, int ii, int nt, double s_new) {
  const double alpha = c->dtau * c->J, lub = log(1.0e200);
  double gamma = 0.0;
  int temporal = 0;
  if (fabs(c->h) > 1.0e-10) {
    double ta = tanh(c->dtau * c->h);
    if (ta < 1.0e-300) ta = 1.0e-300;
    gamma = -0.5 * log(ta);
    temporal = 1;
  }
  const double *sg = c->sigma + (size_t)nt * c->nb;
  const int *o = c->bb + 7 * ii;
  double s_old = sg[ii];
  double t = s_new * sg[o[1]] * sg[o[2]] * sg[o[3]];
  double tn = 0.0 + t;
  t = s_new * sg[o[4]] * sg[o[5]] * sg[o[6]];
  tn = tn + t;
  t = s_old * sg[o[1]] * sg[o[2]] * sg[o[3]];
  double to = 0.0 + t;
  t = s_old * sg[o[4]] * sg[o[5]] * sg[o[6]];
  to = to + t;
  double e = alpha * (tn - to);
  if (e > lub) e = lub;
  if (e < -lub) e = -lub;
  double r = exp(e);
  if (temporal) {
    double a = 0.0, b = 0.0;
    for (int nf = -1; nf <= 1; nf += 2) {
      int ntn = (nt + nf + c->Ltrot) % c->Ltrot;
      double sn = c->sigma[(size_t)ntn * c->nb + ii];
      a = a + s_new * sn;
      b = b + s_old * sn;
    }
    e = gamma * (a - b);
    if (e > lub) e = lub;
    if (e < -lub) e = -lub;
    r = r * exp(e);
  }
  return r;
}

/* ---- LocalK_metro (src/localK.f90:45-173) ---- */
static int metro(Chain *c, int ii, int nt, size_t rec) {
  const int N = c->N;
  double *G = c->G;
  double *sg = c->sigma + (size_t)nt * c->nb;
  double s_old = sg[ii], s_new = -s_old;
  int P[2] = {c->bond[2 * ii], c->bond[2 * ii + 1]};
  double a2 = c->alpha2;
  double cn = cosh(a2 * s_new), co = cosh(a2 * s_old), sn = sinh(a2 * s_new), so = sinh(a2 * s_old);
  double D[2][2];
  D[0][0] = cn * co - sn * so - 1.0;
  D[0][1] = sn * co - cn * so;
  D[1][0] = sn * co - cn * so;
  D[1][1] = cn * co - sn * so - 1.0;
  double Gl[2][2], prod[2][2];
  for (int r = 0; r < 2; ++r)
    for (int l = 0; l < 2; ++l) Gl[l][r] = (l == r ? 1.0 : 0.0) - G[IX(P[l], P[r])];
  for (int r = 0; r < 2; ++r)
    for (int l = 0; l < 2; ++l) prod[l][r] = (l == r ? 1.0 : 0.0) + (D[l][0] * Gl[0][r] + D[l][1] * Gl[1][r]);
  double det = prod[0][0] * prod[1][1] - prod[0][1] * prod[1][0];
  double ratio = det * det * boson_ratio(c, ii, nt, s_new);
  double r = ranf(&c->iq);
  int acc = fabs(ratio) > r;
  c->acc_den += 1.0;
  if (c->dec) c->dec[rec] = (unsigned char)acc;
  if (acc) {
    c->acc_num += 1.0;
    double pi[2][2] = {{prod[1][1] / det, -prod[0][1] / det}, {-prod[1][0] / det, prod[0][0] / det}};
    double *t0 = c->T1, *t1 = c->T1 + N, *v0 = c->T1 + 2 * N, *v1 = c->T1 + 3 * N;
    for (int j = 0; j < N; ++j) {
      double u0 = G[IX(j, P[0])], u1 = G[IX(j, P[1])];
      t0[j] = u0 * pi[0][0] + u1 * pi[1][0];
      t1[j] = u0 * pi[0][1] + u1 * pi[1][1];
      v0[j] = -D[0][0] * G[IX(P[0], j)] - D[0][1] * G[IX(P[1], j)];
      v1[j] = -D[1][0] * G[IX(P[0], j)] - D[1][1] * G[IX(P[1], j)];
    }
    v0[P[0]] += D[0][0]; v0[P[1]] += D[0][1];
    v1[P[0]] += D[1][0]; v1[P[1]] += D[1][1];
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) G[IX(i, j)] = G[IX(i, j)] - (t0[i] * v0[j] + t1[i] * v1[j]);
    sg[ii] = s_new;
  }
  return acc;
}

/* ---- stabilization (src/stabilization.f90:42-200) ---- */
static void qdrp(Chain *c, double *A, double *D) {
  const int N = c->N;
  int info;
  for (int i = 0; i < N; ++i) c->jpvt[i] = 0;
  scipy_dgeqp3_(&N, &N, A, &N, c->jpvt, c->tau, c->work, &c->lwork, &info);
  for (int i = 0; i < N; ++i) {
    double x = fabs(A[IX(i, i)]);
    D[i] = x;
    for (int j = i; j < N; ++j) A[IX(i, j)] = A[IX(i, j)] / x;
  }
}

static void stab_UR(Chain *c) {
  const int N = c->N;
  double one = 1.0;
  int info;
  double *A = c->T2;
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) A[IX(i, j)] = c->UR[IX(i, j)] * c->DR[j];
  qdrp(c, A, c->DR);
  for (int j = 0; j < N; ++j)                       /* ZLAPMR(.true.) */
    for (int i = 0; i < N; ++i) c->T3[IX(i, j)] = c->VR[IX(c->jpvt[i] - 1, j)];
  memcpy(c->VR, c->T3, sizeof(double) * N * N);
  scipy_dtrmm_("L", "U", "N", "N", &N, &N, &one, A, &N, c->VR, &N, 1, 1, 1, 1);
  scipy_dorgqr_(&N, &N, &N, A, &N, c->tau, c->work, &c->lwork, &info);
  memcpy(c->UR, A, sizeof(double) * N * N);
}

static void stab_UL(Chain *c) {
  const int N = c->N;
  double one = 1.0;
  int info;
  double *A = c->T2;
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) A[IX(i, j)] = c->UL[IX(j, i)] * c->DL[j];
  qdrp(c, A, c->DL);
  for (int j = 0; j < N; ++j)                       /* ZLAPMT(.true.) */
    for (int i = 0; i < N; ++i) c->T3[IX(i, j)] = c->VL[IX(i, c->jpvt[j] - 1)];
  memcpy(c->VL, c->T3, sizeof(double) * N * N);
  scipy_dtrmm_("R", "U", "T", "N", &N, &N, &one, A, &N, c->VL, &N, 1, 1, 1, 1);
  scipy_dorgqr_(&N, &N, &N, A, &N, c->tau, c->work, &c->lwork, &info);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) c->UL[IX(i, j)] = A[IX(j, i)];
}

static void stab_green(Chain *c, int nt, double *Gout) {
  const int N = c->N;
  double one = 1.0, zero = 0.0;
  int info;
  double *M = c->T2, *tmp = c->T1, *vv = c->T3;
  scipy_dgemm_("N", "N", &N, &N, &N, &one, c->VR, &N, c->VL, &N, &zero, vv, &N, 1, 1);
  scipy_dgemm_("T", "T", &N, &N, &N, &one, c->UR, &N, c->UL, &N, &zero, M, &N, 1, 1);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) {
      double t = vv[IX(i, j)] * c->DL[j];
      M[IX(i, j)] = M[IX(i, j)] + c->DR[i] * t;
    }
  const int half = c->Ltrot / 2;
  if (nt > half)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < j; ++i) { double a = M[IX(i, j)]; M[IX(i, j)] = M[IX(j, i)]; M[IX(j, i)] = a; }
  qdrp(c, M, c->Dn);
  if (nt < half + 1) {
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) tmp[IX(i, j)] = c->UR[IX(j, i)];
    scipy_dormqr_("L", "T", &N, &N, &N, M, &N, c->tau, tmp, &N, c->work, &c->lwork, &info, 1, 1);
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) tmp[IX(i, j)] = tmp[IX(i, j)] / c->Dn[i];
    scipy_dtrsm_("L", "U", "N", "N", &N, &N, &one, M, &N, tmp, &N, 1, 1, 1, 1);
    for (int j = 0; j < N; ++j)                     /* ZLAPMR(.false.) */
      for (int i = 0; i < N; ++i) vv[IX(c->jpvt[i] - 1, j)] = tmp[IX(i, j)];
    scipy_dgemm_("T", "N", &N, &N, &N, &one, c->UL, &N, vv, &N, &zero, Gout, &N, 1, 1);
  } else {
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) tmp[IX(i, j)] = c->UL[IX(j, i)];
    scipy_dormqr_("R", "N", &N, &N, &N, M, &N, c->tau, tmp, &N, c->work, &c->lwork, &info, 1, 1);
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) tmp[IX(i, j)] = tmp[IX(i, j)] / c->Dn[j];
    scipy_dtrsm_("R", "U", "T", "N", &N, &N, &one, M, &N, tmp, &N, 1, 1, 1, 1);
    for (int j = 0; j < N; ++j)                     /* ZLAPMT(.false.) */
      for (int i = 0; i < N; ++i) vv[IX(i, c->jpvt[j] - 1)] = tmp[IX(i, j)];
    scipy_dgemm_("N", "T", &N, &N, &N, &one, vv, &N, c->UR, &N, &zero, Gout, &N, 1, 1);
  }
}

static double maxdiff(const double *A, const double *B, size_t n) {
  double m = 0.0;
  for (size_t i = 0; i < n; ++i) { double d = fabs(A[i] - B[i]); if (d > m) m = d; }
  return m;
}

/* ---- wraps (src/stabilization.f90:374-476) ---- */
static void push(double *dst, const double *src, size_t n) { memcpy(dst, src, sizeof(double) * n); }

static void wrap_pre(Chain *c, int nt) {
  const int N = c->N;
  const size_t NN = (size_t)N * N;
  int st = nt / c->Nwrap;
  if (nt != 0) stab_UR(c);
  push(c->URs + st * NN, c->UR, NN); push(c->VRs + st * NN, c->VR, NN); push(c->DRs + st * N, c->DR, N);
  if (nt == c->Ltrot) stab_green(c, nt, c->G);
}

static void wrap_L(Chain *c, int nt) {
  const int N = c->N;
  const size_t NN = (size_t)N * N;
  int st = nt / c->Nwrap;
  push(c->UR, c->URs + st * NN, NN); push(c->VR, c->VRs + st * NN, NN); push(c->DR, c->DRs + st * N, N);
  if (nt != c->Ltrot) {
    stab_UL(c);
    double *Gn = malloc(sizeof(double) * NN);
    stab_green(c, nt, Gn);
    double d = maxdiff(Gn, c->G, NN);
    if (d > c->Xmaxm) c->Xmaxm = d;
    c->Xmeanm += d;
    memcpy(c->G, Gn, sizeof(double) * NN);
    free(Gn);
  }
  push(c->ULs + st * NN, c->UL, NN); push(c->VLs + st * NN, c->VL, NN); push(c->DLs + st * N, c->DL, N);
}

static void wrap_R(Chain *c, int nt) {
  const int N = c->N;
  const size_t NN = (size_t)N * N;
  int st = nt / c->Nwrap;
  push(c->UL, c->ULs + st * NN, NN); push(c->VL, c->VLs + st * NN, NN); push(c->DL, c->DLs + st * N, N);
  if (nt != 0) {
    stab_UR(c);
    double *Gn = malloc(sizeof(double) * NN);
    stab_green(c, nt, Gn);
    double d = maxdiff(Gn, c->G, NN);
    if (d > c->Xmaxm) c->Xmaxm = d;
    c->Xmeanm += d;
    memcpy(c->G, Gn, sizeof(double) * NN);
    free(Gn);
  }
  push(c->URs + st * NN, c->UR, NN); push(c->VRs + st * NN, c->VR, NN); push(c->DRs + st * N, c->DR, N);
}

/* ---- Obs_equal_calc (src/obser_equal.f90:73-149) ---- */
static void obs_equal(Chain *c, int nt) {
  const int N = c->N;
  const double *sg = c->sigma + (size_t)nt * c->nb, *G = c->G;
  const double PI = acos(-1.0), qx = PI - 2.0 * PI / (double)c->Lx;
  double flux = 0.0;
  for (int s = 0; s < N; ++s) {
    const int *p = c->plaq + 4 * s;
    flux = flux + sg[p[0]] * sg[p[1]] * sg[p[2]] * sg[p[3]];
  }
  flux = flux / (double)N;
  c->flux_sum += flux;
  c->flux_sq += flux * flux;
  double pair = 0.0, cdw = 0.0, cdws = 0.0, dens = 0.0;
  for (int i = 0; i < N; ++i) {
    double ni = 1.0 - G[IX(i, i)];
    dens = dens + ni + ni;
    for (int j = 0; j < N; ++j) {
      double nj = 1.0 - G[IX(j, j)];
      double dl = (i == j) ? 1.0 : 0.0;
      double gij = G[IX(i, j)], gji = G[IX(j, i)];
      pair = pair + (dl - gij) * (dl - gij);
      double a = ni * nj, ex = (dl - gji) * gij;
      double dc = a - ex;
      dc = dc + a - ex;
      dc = dc + a + a;
      double si = ((c->xy[2 * i] + c->xy[2 * i + 1]) % 2 == 0) ? 1.0 : -1.0;
      double sj = ((c->xy[2 * j] + c->xy[2 * j + 1]) % 2 == 0) ? 1.0 : -1.0;
      double dx = (double)(c->xy[2 * i] - c->xy[2 * j]), dy = (double)(c->xy[2 * i + 1] - c->xy[2 * j + 1]);
      double ps = cos(qx * dx + PI * dy);
      cdw = cdw + si * sj * dc;
      cdws = cdws + ps * dc;
    }
  }
  c->pair += pair; c->cdw += cdw; c->cdws += cdws; c->dens += dens / (double)N;
  c->nobs += 1.0;
}

/* ---- sweeps (src/local_sweep.f90:87-195) ---- */
/* Local_sweep_reset (src/local_sweep.f90:63-69): for |h| <= Zero the links
 * are made constant in tau (the value of slice 1). */
static void reset_h0(Chain *c) {
  if (fabs(c->h) > 1.0e-10) return;
  for (int t = 1; t < c->Ltrot; ++t)
    for (int b = 0; b < c->nb; ++b) c->sigma[(size_t)t * c->nb + b] = c->sigma[b];
}

static void pre(Chain *c) {
  reset_h0(c);
  const int N = c->N;
  const size_t NN = (size_t)N * N;
  memset(c->UR, 0, NN * 8); memset(c->VR, 0, NN * 8); memset(c->UL, 0, NN * 8);
  memset(c->VL, 0, NN * 8); memset(c->G, 0, NN * 8);
  for (int i = 0; i < N; ++i) {
    c->UR[IX(i, i)] = 1; c->VR[IX(i, i)] = 1; c->UL[IX(i, i)] = 1; c->VL[IX(i, i)] = 1;
    c->G[IX(i, i)] = 1; c->DR[i] = 1; c->DL[i] = 1;
  }
  wrap_pre(c, 0);
  for (int nt = 1; nt <= c->Ltrot; ++nt) {
    if (c->RT > 1.0e-10) mmult_R(c, c->UR, nt - 1, 1);
    scale(c->UR, NN, c->eP);
    if (nt % c->Nwrap == 0) wrap_pre(c, nt);
  }
}

static void sweep_L(Chain *c) {
  const int N = c->N, nb = c->nb;
  const size_t NN = (size_t)N * N;
  for (int nt = c->Ltrot; nt >= 1; --nt) {
    if (nt % c->Nwrap == 0) wrap_L(c, nt);
    obs_equal(c, nt - 1);
    scale(c->G, NN, c->eP); scale(c->G, NN, c->eM); scale(c->UL, NN, c->eP);
    for (int ii = nb - 1; ii >= 0; --ii) metro(c, ii, nt - 1, ((size_t)0 * c->Ltrot + nt - 1) * nb + ii);
    mmult_L(c, c->G, nt - 1, 1);
    mmult_R(c, c->G, nt - 1, -1);
    mmult_L(c, c->UL, nt - 1, 1);
  }
  wrap_L(c, 0);
}

static void sweep_R(Chain *c) {
  const int N = c->N, nb = c->nb;
  const size_t NN = (size_t)N * N;
  wrap_R(c, 0);
  for (int nt = 1; nt <= c->Ltrot; ++nt) {
    mmult_R(c, c->G, nt - 1, 1);
    mmult_L(c, c->G, nt - 1, -1);
    for (int ii = 0; ii < nb; ++ii) metro(c, ii, nt - 1, ((size_t)1 * c->Ltrot + nt - 1) * nb + ii);
    mmult_R(c, c->UR, nt - 1, 1);
    scale(c->G, NN, c->eP); scale(c->G, NN, c->eM); scale(c->UR, NN, c->eP);
    if (nt % c->Nwrap == 0) wrap_R(c, nt);
    obs_equal(c, nt - 1);
  }
}

static double now(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

/*
 * Persistent chains (the reference keeps one chain's state in its process
 * between bins, src/main.f90:70-110):
 *   z2cpu_new   seeded start, conf_set absolute = 1 / 3 / 5 on the run
 *               lattice (src/fields.f90:311-427) + the lambda_random_fill
 *               draws; dparams = {RT, J, h, mu, beta}, iparams = {Nlx, Nly,
 *               Ltrot, Nwrap, absolute, seed}.
 *   z2cpu_pre   Local_sweep_pre (src/local_sweep.f90:87-104).
 *   z2cpu_bin   one bin of nsweep (sweep_L, sweep_R) pairs
 *               (src/local_sweep.f90:152-195); obs[7] = flux_avg, chi_flux,
 *               pair_sc_q0, cdw_pi, cdw_shift, cdw_ratio, density; dec
 *               (optional) receives the decisions of the last half-sweeps
 *               [2][Ltrot][2N]; returns the seconds spent.
 *   z2cpu_state G (column-major), sigma [Ltrot][2N] as +-1 doubles, stats
 *               {acc (sum over bins), Xmaxm, Xmeanm, iseed}; each optional.
 *   z2cpu_free  releases the chain.
 */
void *z2cpu_new(const double *dparams, const int *iparams) {
  scipy_openblas_set_num_threads(1);
  Chain *c = calloc(1, sizeof(Chain));
  if (!c) return NULL;
  c->RT = dparams[0]; c->J = dparams[1]; c->h = dparams[2]; c->mu = dparams[3]; c->beta = dparams[4];
  c->Lx = iparams[0]; c->Ly = iparams[1]; c->Ltrot = iparams[2]; c->Nwrap = iparams[3];
  int absolute = iparams[4], seed = iparams[5];
  c->N = c->Lx * c->Ly; c->nb = 2 * c->N; c->Nst = c->Ltrot / c->Nwrap;
  c->dtau = c->beta / (double)c->Ltrot;
  c->alpha = 0.5 * c->dtau * c->RT; c->alpha2 = c->dtau * c->RT;
  c->eP = exp(c->dtau * c->mu); c->eM = exp(-c->dtau * c->mu);
  const int N = c->N, nb = c->nb;
  const size_t NN = (size_t)N * N;
  lattice(c);
  /* conf_set (src/fields.f90:311-427) + lambda_random_fill draws */
  c->sigma = malloc(sizeof(double) * nb * c->Ltrot);
  c->iq = (uint32_t)seed;
  for (int nt = 0; nt < c->Ltrot; ++nt)
    for (int b = 0; b < nb; ++b) c->sigma[(size_t)nt * nb + b] = 1.0;
  if (absolute == 1)
    for (int nt = 0; nt < c->Ltrot; ++nt)
      for (int b = 0; b < nb; ++b) c->sigma[(size_t)nt * nb + b] = ranf(&c->iq) >= 0.5 ? 1.0 : -1.0;
  else if (absolute == 5)
    for (int b = 0; b < nb; ++b) {
      double v = ranf(&c->iq) >= 0.5 ? 1.0 : -1.0;
      for (int nt = 0; nt < c->Ltrot; ++nt) c->sigma[(size_t)nt * nb + b] = v;
    }
  for (int i = 0; i < N; ++i) ranf(&c->iq);
  double *m = malloc(sizeof(double) * NN * 10);
  c->G = m; c->UR = m + NN; c->VR = m + 2 * NN; c->UL = m + 3 * NN; c->VL = m + 4 * NN;
  c->T1 = m + 5 * NN; c->T2 = m + 6 * NN; c->T3 = m + 7 * NN;
  c->DR = malloc(sizeof(double) * 4 * N); c->DL = c->DR + N; c->tau = c->DR + 2 * N; c->Dn = c->DR + 3 * N;
  c->URs = malloc(sizeof(double) * NN * 4 * (c->Nst + 1));
  c->VRs = c->URs + NN * (c->Nst + 1); c->ULs = c->URs + 2 * NN * (c->Nst + 1); c->VLs = c->URs + 3 * NN * (c->Nst + 1);
  c->DRs = malloc(sizeof(double) * 2 * N * (c->Nst + 1)); c->DLs = c->DRs + N * (c->Nst + 1);
  c->jpvt = malloc(sizeof(int) * N);
  c->lwork = 64 * N + 64;
  c->work = malloc(sizeof(double) * c->lwork);
  c->acc_sum = 0.0;
  return c;
}

void z2cpu_pre(void *h) {
  scipy_openblas_set_num_threads(1);
  pre((Chain *)h);
}

double z2cpu_bin(void *h, int nsweep, double *obs, unsigned char *dec) {
  scipy_openblas_set_num_threads(1);
  Chain *c = (Chain *)h;
  const int N = c->N;
  c->dec = dec;
  double t0 = now();
  c->flux_sum = c->flux_sq = c->pair = c->cdw = c->cdws = c->dens = c->nobs = 0.0;
  c->acc_num = c->acc_den = 0.0;
  reset_h0(c);
  for (int s = 0; s < nsweep; ++s) { sweep_L(c); sweep_R(c); }
  double z = 1.0 / c->nobs, fm = c->flux_sum * z, fsq = c->flux_sq * z;
  double o[7];
  o[0] = fm;
  o[1] = c->beta * (double)N * fmax(0.0, fsq - fm * fm);
  o[2] = (c->pair * z) / (double)N;
  o[3] = (c->cdw * z) / (double)N;
  o[4] = (c->cdws * z) / (double)N;
  o[5] = (o[3] > 1.0e-12) ? 1.0 - o[4] / o[3] : 0.0;
  o[6] = c->dens * z;
  if (c->acc_den > 0.0) c->acc_sum += c->acc_num / c->acc_den;
  double sec = now() - t0;
  if (obs) memcpy(obs, o, sizeof(o));
  c->dec = NULL;
  return sec;
}

void z2cpu_state(void *h, double *Gout, double *sigma, double *stats) {
  Chain *c = (Chain *)h;
  if (Gout) memcpy(Gout, c->G, sizeof(double) * c->N * c->N);
  if (sigma) memcpy(sigma, c->sigma, sizeof(double) * c->nb * c->Ltrot);
  if (stats) {
    stats[0] = c->acc_sum; stats[1] = c->Xmaxm; stats[2] = c->Xmeanm; stats[3] = (double)c->iq;
  }
}

void z2cpu_free(void *h) {
  Chain *c = (Chain *)h;
  if (!c) return;
  free(c->G); free(c->DR); free(c->URs); free(c->DRs); free(c->jpvt); free(c->work);
  free(c->sigma); free(c->bond); free(c->grp); free(c->bb); free(c->xy); free(c->plaq);
  free(c);
}

/*
 * One chain from a seeded start to nbins bins (z2cpu_new, z2cpu_pre, then
 * z2cpu_bin per bin).  iparams = {Nlx, Nly, Ltrot, Nwrap, absolute, seed,
 * nbins, nsweep}.  Outputs: obs [nbins][7], the final G (column-major), the
 * decisions of the last half-sweeps [2][Ltrot][2N] (optional), stats {acc,
 * Xmaxm, Xmeanm, iseed}, and the seconds spent in the bins (pre excluded).
 * Returns 0, or 1 when the chain cannot be allocated.
 */
int z2cpu_run(const double *dparams, const int *iparams, double *obs, double *Gout,
              unsigned char *dec, double *stats, double *seconds) {
  void *c = z2cpu_new(dparams, iparams);
  if (!c) return 1;
  const int nbins = iparams[6], nsweep = iparams[7];
  z2cpu_pre(c);
  double sec = 0.0;
  for (int b = 0; b < nbins; ++b) sec += z2cpu_bin(c, nsweep, obs + 7 * b, dec);
  *seconds = sec;
  z2cpu_state(c, Gout, NULL, stats);
  z2cpu_free(c);
  return 0;
}
