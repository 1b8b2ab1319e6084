/*
 * ibfs_oracle.c -- CPU FP64 restatement of the IBFS per-timestep advance.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; never shipped on
 * the product path). Parity with the Fortran+FFTW binary is UNPINNED: the
 * reference cannot be compiled in this environment. See ibfs_oracle.h.
 *
 * Index helpers mirror the Fortran 1-based declarations so every loop below
 * reads like the line of the reference Fortran source it cites:
 *   OM(a,i,j)  element (i,j) of an array declared DIMENSION(2:m,2:n)
 *   R1(a,i,j)  element (i,j) of an assumed-shape DIMENSION(:,:) dummy
 *              (lower bound 1) -- used by get_bc / apply_bc, which receive
 *              omega(:,:,k) sections (operators.f90:342, 376)
 *   UI(i,j), VI(i,j)  1-based face indices u(i,j), v(i,j) (grid.f90:119-134)
 *   X1(a,idx)  1-based element of a vector
 * Compile with -ffp-contract=off so a*b+c is not fused (the reference's
 * x86-64 build has no FMA).
 */
#include "ibfs_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

/* ------------------------------------------------------------------------ */
/* Mixed-radix complex FFT (decimation in time, recursive).                  */
/* ------------------------------------------------------------------------ */
typedef struct {
  int n;
  int nfac;
  int fac[40];
  cplx* tw; /* tw[j] = exp(-2 pi i j / n) */
  cplx* zin;
  cplx* zout;
} fftplan;

static void fft_plan_init(fftplan* P, int n) {
  P->n = n;
  P->nfac = 0;
  int r = n;
  while (r % 4 == 0) { P->fac[P->nfac++] = 4; r /= 4; }
  while (r % 2 == 0) { P->fac[P->nfac++] = 2; r /= 2; }
  for (int p = 3; r > 1; p += 2) {
    while (r % p == 0) { P->fac[P->nfac++] = p; r /= p; }
  }
  P->tw = (cplx*)malloc(sizeof(cplx) * n);
  for (int j = 0; j < n; j++) {
    double a = -2.0 * M_PI * (double)j / (double)n;
    P->tw[j] = cos(a) + I * sin(a);
  }
  P->zin = (cplx*)malloc(sizeof(cplx) * n);
  P->zout = (cplx*)malloc(sizeof(cplx) * n);
}

static void fft_plan_free(fftplan* P) {
  free(P->tw);
  free(P->zin);
  free(P->zout);
}

static void fft_rec(const fftplan* P, cplx* out, const cplx* in, int n, int is,
                    int fi, int twstep) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = P->fac[fi], q = n / p;
  for (int r = 0; r < p; r++)
    fft_rec(P, out + r * q, in + r * is, q, is * p, fi + 1, twstep * p);
  cplx t[p];
  int np = P->n / p;
  for (int k = 0; k < q; k++) {
    for (int s = 0; s < p; s++) t[s] = out[s * q + k] * P->tw[s * k * twstep];
    if (p == 2) {
      out[k] = t[0] + t[1];
      out[q + k] = t[0] - t[1];
    } else if (p == 4) {
      cplx a0 = t[0] + t[2], a1 = t[0] - t[2];
      cplx b0 = t[1] + t[3], b1 = (t[1] - t[3]) * (-I);
      out[k] = a0 + b0;
      out[q + k] = a1 + b1;
      out[2 * q + k] = a0 - b0;
      out[3 * q + k] = a1 - b1;
    } else {
      for (int s2 = 0; s2 < p; s2++) {
        cplx acc = 0;
        for (int s = 0; s < p; s++) acc += t[s] * P->tw[((s * s2) % p) * np];
        out[s2 * q + k] = acc;
      }
    }
  }
}

static void fft_exec(const fftplan* P) { fft_rec(P, P->zout, P->zin, P->n, 1, 0, 1); }

/* DST-I (FFTW RODFT00, Y_k = 2 sum_j X_j sin(pi j k / N+1)) of two real
 * vectors a, b of length N = len-1 at once: the odd extension of a + i b has
 * DFT  -i Y_a + Y_b. */
static void dst1_pair(const fftplan* P, const double* a, int sa, const double* b,
                      int sb, double* ya, int sya, double* yb, int syb, int N) {
  int L = P->n; /* = 2(N+1) */
  int h = L / 2;
  cplx* z = P->zin;
  z[0] = 0;
  z[h] = 0;
  for (int t = 1; t <= N; t++) {
    cplx v = a[(t - 1) * sa] + I * (b ? b[(t - 1) * sb] : 0.0);
    z[t] = v;
    z[L - t] = -v;
  }
  fft_exec(P);
  for (int k = 1; k <= N; k++) {
    cplx Z = P->zout[k];
    ya[(k - 1) * sya] = -cimag(Z);
    if (yb) yb[(k - 1) * syb] = creal(Z);
  }
}

/* ------------------------------------------------------------------------ */
/* Case                                                                      */
/* ------------------------------------------------------------------------ */
struct or_case {
  or_params p;
  int m, n, L;
  int nq, nb, nf, ns;
  int nsmear;
  double delta;
  int left, right, bottom, top;
  double *xb, *yb;
  int* bdyno;
  int* ismear;   /* Nq x nsmear, 1-based force index */
  double* smear; /* Nq x nsmear */
  /* myfft tables */
  double *lam, *laminv, *lam1, *lam1i, *con1, *con2, *vfac;
  double normalize;
  fftplan px, py;
  double* dwork;
  /* state */
  double *omega, *fb, *rhs_old, *q, *q0;
  double *cholmat, *cholvec;
  int cg_rel;
};

#define OMs(m_) ((m_)-1)
#define OM(a, i, j) ((a)[((i)-2) + ((j)-2) * (m - 1)])
#define R1(a, i, j) ((a)[((i)-1) + ((j)-1) * (m - 1)])
#define UI(i, j) ((i) + ((j)-1) * (m + 1))
#define VI(i, j) ((m + 1) * n + (i) + ((j)-1) * m)
#define X1(a, idx) ((a)[(idx)-1])

/* grid.f90:79 -- FLOOR(LOG(REAL(MIN(m,n)/2))/LOG(2.d0)) - 1, with the
 * single-precision LOG of a single-precision REAL. */
int or_nlevmax(int m, int n) {
  int mn = (m < n ? m : n) / 2;
  float lf = logf((float)mn);
  return (int)floor((double)lf / log(2.0)) - 1;
}

/* grid.f90:233-249 (Roma, Peskin & Berger 3-point kernel). */
double or_deltafnc(double r, double r0, double dr) {
  double d = fabs(r - r0);
  if (d <= 0.5 * dr) {
    double t = (r - r0) / dr;
    return (1.0 + sqrt(-3.0 * t * t + 1.0)) / (3.0 * dr);
  } else if (d <= 1.5 * dr) {
    double a = fabs((r - r0) / dr);
    double u = 1.0 - a;
    return (5.0 - 3.0 * a - sqrt(-3.0 * u * u + 1.0)) / (6.0 * dr);
  }
  return 0.0;
}

/* grid.f90:142-230. */
static void setup_reg(or_case* c) {
  int m = c->m, n = c->n;
  double delta = c->delta;
  double d2 = 0.5 * delta;
  double sup = 3.0 * d2; /* support = 3.0 (grid.f90:11) */
  double ox = c->p.offsetx, oy = c->p.offsety;
  int nb = c->nb;
  free(c->ismear);
  free(c->smear);
  int nsm = 0;
  for (int i = 1; i <= m + 1; i++)
    for (int j = 1; j <= n; j++) {
      double x = delta * (double)(i - 1) - ox;
      double y = delta * (double)(j - 1) - oy + d2;
      int cnt = 0;
      for (int k = 0; k < nb; k++)
        if (fabs(x - c->xb[k]) < sup && fabs(y - c->yb[k]) < sup) cnt++;
      if (cnt > nsm) nsm = cnt;
    }
  for (int i = 1; i <= m; i++)
    for (int j = 1; j <= n + 1; j++) {
      double x = delta * (double)(i - 1) - ox + d2;
      double y = delta * (double)(j - 1) - oy;
      int cnt = 0;
      for (int k = 0; k < nb; k++)
        if (fabs(x - c->xb[k]) < sup && fabs(y - c->yb[k]) < sup) cnt++;
      if (cnt > nsm) nsm = cnt;
    }
  c->nsmear = nsm;
  size_t tot = (size_t)c->nq * (nsm > 0 ? nsm : 1);
  c->ismear = (int*)malloc(sizeof(int) * tot);
  c->smear = (double*)malloc(sizeof(double) * tot);
  for (size_t t = 0; t < tot; t++) {
    c->ismear[t] = 1;
    c->smear[t] = 0.0;
  }
  int nq = c->nq;
  for (int i = 1; i <= m + 1; i++)
    for (int j = 1; j <= n; j++) {
      double x = delta * (double)(i - 1) - ox;
      double y = delta * (double)(j - 1) - oy + d2;
      int cnt = 0;
      for (int k = 0; k < nb; k++)
        if (fabs(x - c->xb[k]) < sup && fabs(y - c->yb[k]) < sup) {
          cnt++;
          size_t at = (size_t)(UI(i, j) - 1) + (size_t)(cnt - 1) * nq;
          c->ismear[at] = k + 1; /* f(k,1) */
          c->smear[at] = (delta * delta) * or_deltafnc(x, c->xb[k], delta) *
                         or_deltafnc(y, c->yb[k], delta);
        }
    }
  for (int i = 1; i <= m; i++)
    for (int j = 1; j <= n + 1; j++) {
      double x = delta * (double)(i - 1) - ox + d2;
      double y = delta * (double)(j - 1) - oy;
      int cnt = 0;
      for (int k = 0; k < nb; k++)
        if (fabs(x - c->xb[k]) < sup && fabs(y - c->yb[k]) < sup) {
          cnt++;
          size_t at = (size_t)(VI(i, j) - 1) + (size_t)(cnt - 1) * nq;
          c->ismear[at] = nb + k + 1; /* f(k,2) */
          c->smear[at] = (delta * delta) * or_deltafnc(x, c->xb[k], delta) *
                         or_deltafnc(y, c->yb[k], delta);
        }
    }
}

/* myfft.f90:21-70. */
static void setup_fft(or_case* c) {
  int m = c->m, n = c->n, L = c->L;
  double dt = c->p.dt, Re = c->p.re;
  double pi = 3.1415926535897932384;
  size_t ns = (size_t)(m - 1) * (n - 1);
  c->normalize = 4.0 * (double)((float)((long long)m * n));
  c->con1 = (double*)malloc(sizeof(double) * L);
  c->con2 = (double*)malloc(sizeof(double) * L);
  c->vfac = (double*)malloc(sizeof(double) * L);
  c->lam = (double*)malloc(sizeof(double) * ns);
  c->laminv = (double*)malloc(sizeof(double) * ns);
  c->lam1 = (double*)malloc(sizeof(double) * ns * L);
  c->lam1i = (double*)malloc(sizeof(double) * ns * L);
  double del2 = c->delta * c->delta;
  double normalize = c->normalize;
  for (int k = 1; k <= L; k++) {
    double del22 = del2 * pow(4.0, k - 1);
    c->vfac[k - 1] = 0.5 * dt / Re / del22 / normalize;
    c->con1[k - 1] = 1.5 * dt / del22 / normalize;
    c->con2[k - 1] = -0.5 * dt / del22 / normalize;
  }
  for (int j = 1; j <= n - 1; j++)
    for (int i = 1; i <= m - 1; i++) {
      size_t at = (size_t)(i - 1) + (size_t)(j - 1) * (m - 1);
      double lam = -2.0 * (cos(pi * (double)i / (double)m) +
                           cos(pi * (double)j / (double)n) - 2.0);
      c->lam[at] = lam;
      c->laminv[at] = 1.0 / lam / normalize;
      for (int k = 1; k <= L; k++) {
        double del22 = del2 * pow(4.0, k - 1);
        c->lam1[at + (k - 1) * ns] = (1.0 - 0.5 * dt * lam / del22 / Re) / normalize;
        c->lam1i[at + (k - 1) * ns] = 1.0 / (1.0 + 0.5 * dt * lam / del22 / Re);
      }
    }
  fft_plan_init(&c->px, 2 * m);
  fft_plan_init(&c->py, 2 * n);
  c->dwork = (double*)malloc(sizeof(double) * ns);
}

int or_create(const or_params* p, int nb, const double* xb, const double* yb,
              const int* bdyno, or_case** out) {
  *out = NULL;
  if (p->m % 4 != 0 || p->n % 4 != 0) return 1; /* grid.f90:67-69 */
  or_case* c = (or_case*)calloc(1, sizeof(or_case));
  c->p = *p;
  int m = p->m, n = p->n;
  c->m = m;
  c->n = n;
  c->delta = p->len / (double)m; /* grid.f90:64 */
  c->left = 0;
  c->right = n + 1;
  c->bottom = 2 * (n + 1);
  c->top = 2 * (n + 1) + m + 1;
  int nlevmax = or_nlevmax(m, n);
  c->L = p->mgridlev < nlevmax ? p->mgridlev : nlevmax; /* grid.f90:81 */
  c->p.mgridlev = c->L;
  c->nb = nb;
  c->nf = 2 * nb;
  c->ns = (m - 1) * (n - 1);
  c->nq = (m + 1) * n + (n + 1) * m;
  c->xb = (double*)malloc(sizeof(double) * (nb > 0 ? nb : 1));
  c->yb = (double*)malloc(sizeof(double) * (nb > 0 ? nb : 1));
  c->bdyno = (int*)malloc(sizeof(int) * (nb > 0 ? nb : 1));
  for (int k = 0; k < nb; k++) {
    c->xb[k] = xb[k];
    c->yb[k] = yb[k];
    c->bdyno[k] = bdyno ? bdyno[k] : 0;
  }
  setup_reg(c);
  setup_fft(c);
  size_t ns = c->ns, nq = c->nq;
  int L = c->L;
  c->omega = (double*)calloc(ns * L, sizeof(double));
  c->rhs_old = (double*)calloc(ns * L, sizeof(double));
  c->q = (double*)calloc(nq * L, sizeof(double));
  c->q0 = (double*)calloc(nq * L, sizeof(double));
  c->fb = (double*)calloc(c->nf > 0 ? c->nf : 1, sizeof(double));
  if (p->unif_flow) { /* variables.f90:60-64 */
    for (int k = 1; k <= L; k++)
      for (size_t t = 0; t < (size_t)(m + 1) * n; t++)
        c->q0[t + (k - 1) * nq] = c->delta * pow(2.0, k - 1);
  }
  size_t nf = c->nf > 0 ? c->nf : 1;
  c->cholmat = (double*)calloc(nf * nf, sizeof(double));
  c->cholvec = (double*)calloc(nf, sizeof(double));
  *out = c;
  return 0;
}

void or_destroy(or_case* c) {
  if (!c) return;
  free(c->xb); free(c->yb); free(c->bdyno); free(c->ismear); free(c->smear);
  free(c->lam); free(c->laminv); free(c->lam1); free(c->lam1i);
  free(c->con1); free(c->con2); free(c->vfac);
  fft_plan_free(&c->px); fft_plan_free(&c->py);
  free(c->dwork);
  free(c->omega); free(c->fb); free(c->rhs_old); free(c->q); free(c->q0);
  free(c->cholmat); free(c->cholvec);
  free(c);
}

void or_sizes(const or_case* c, int* m, int* n, int* nlev, int* nq, int* nb,
              int* nsmear, double* delta) {
  if (m) *m = c->m;
  if (n) *n = c->n;
  if (nlev) *nlev = c->L;
  if (nq) *nq = c->nq;
  if (nb) *nb = c->nb;
  if (nsmear) *nsmear = c->nsmear;
  if (delta) *delta = c->delta;
}

void or_get_state(const or_case* c, double* omega, double* fb, double* rhs_old,
                  double* q, double* q0) {
  size_t ns = (size_t)c->ns * c->L, nq = (size_t)c->nq * c->L;
  if (omega) memcpy(omega, c->omega, ns * sizeof(double));
  if (fb) memcpy(fb, c->fb, c->nf * sizeof(double));
  if (rhs_old) memcpy(rhs_old, c->rhs_old, ns * sizeof(double));
  if (q) memcpy(q, c->q, nq * sizeof(double));
  if (q0) memcpy(q0, c->q0, nq * sizeof(double));
}

void or_set_state(or_case* c, const double* omega, const double* fb,
                  const double* rhs_old, const double* q, const double* q0) {
  size_t ns = (size_t)c->ns * c->L, nq = (size_t)c->nq * c->L;
  if (omega) memcpy(c->omega, omega, ns * sizeof(double));
  if (fb) memcpy(c->fb, fb, c->nf * sizeof(double));
  if (rhs_old) memcpy(c->rhs_old, rhs_old, ns * sizeof(double));
  if (q) memcpy(c->q, q, nq * sizeof(double));
  if (q0) memcpy(c->q0, q0, nq * sizeof(double));
}

void or_get_cholesky(const or_case* c, double* cholmat, double* cholvec) {
  size_t nf = c->nf;
  if (cholmat) memcpy(cholmat, c->cholmat, nf * nf * sizeof(double));
  if (cholvec) memcpy(cholvec, c->cholvec, nf * sizeof(double));
}

void or_set_cholesky(or_case* c, const double* cholmat, const double* cholvec) {
  size_t nf = c->nf;
  if (cholmat) memcpy(c->cholmat, cholmat, nf * nf * sizeof(double));
  if (cholvec) memcpy(c->cholvec, cholvec, nf * sizeof(double));
}

void or_set_body(or_case* c, const double* xb, const double* yb) {
  for (int k = 0; k < c->nb; k++) {
    c->xb[k] = xb[k];
    c->yb[k] = yb[k];
  }
  setup_reg(c);
}

void or_set_cg_relative(or_case* c, int cg_rel) { c->cg_rel = cg_rel; }

void or_tables(const or_case* c, double* lam, double* laminv, double* lam1,
               double* lam1i, double* con1, double* con2, double* vfac) {
  size_t ns = c->ns;
  int L = c->L;
  if (lam) memcpy(lam, c->lam, ns * sizeof(double));
  if (laminv) memcpy(laminv, c->laminv, ns * sizeof(double));
  if (lam1) memcpy(lam1, c->lam1, ns * L * sizeof(double));
  if (lam1i) memcpy(lam1i, c->lam1i, ns * L * sizeof(double));
  if (con1) memcpy(con1, c->con1, L * sizeof(double));
  if (con2) memcpy(con2, c->con2, L * sizeof(double));
  if (vfac) memcpy(vfac, c->vfac, L * sizeof(double));
}

/* ------------------------------------------------------------------------ */
/* Spectral operators (myfft.f90:83-124)                                     */
/* ------------------------------------------------------------------------ */
/* dst (myfft.f90:83-94): 2-D RODFT00, in may alias out. */
void or_dst(or_case* c, const double* in, double* out) {
  int m = c->m, n = c->n;
  int N1 = m - 1, N2 = n - 1;
  double* w = c->dwork;
  /* along x (contiguous columns), two columns per complex FFT */
  for (int j = 0; j < N2; j += 2) {
    const double* a = in + (size_t)j * N1;
    const double* b = (j + 1 < N2) ? in + (size_t)(j + 1) * N1 : NULL;
    dst1_pair(&c->px, a, 1, b, 1, w + (size_t)j * N1, 1,
              b ? w + (size_t)(j + 1) * N1 : NULL, 1, N1);
  }
  /* along y (stride N1), two rows per complex FFT */
  for (int i = 0; i < N1; i += 2) {
    const double* a = w + i;
    const double* b = (i + 1 < N1) ? w + i + 1 : NULL;
    dst1_pair(&c->py, a, N1, b, N1, out + i, N1, b ? out + i + 1 : NULL, N1, N2);
  }
}

/* ctci (myfft.f90:97-109). */
void or_ctci(or_case* c, const double* in, double* out) {
  size_t ns = c->ns;
  double* t = (double*)malloc(sizeof(double) * ns);
  or_dst(c, in, t);
  for (size_t a = 0; a < ns; a++) t[a] = c->laminv[a] * t[a];
  or_dst(c, t, out);
  free(t);
}

/* ainv (myfft.f90:112-124): lam1i of level 1 only. */
void or_ainv(or_case* c, const double* in, double* out) {
  size_t ns = c->ns;
  double* t = (double*)malloc(sizeof(double) * ns);
  or_dst(c, in, t);
  for (size_t a = 0; a < ns; a++) t[a] = c->lam1i[a] * t[a] / c->normalize;
  or_dst(c, t, out);
  free(t);
}

/* ------------------------------------------------------------------------ */
/* Stencils (operators.f90)                                                  */
/* ------------------------------------------------------------------------ */
/* curl (operators.f90:243-288). */
void or_curl(const or_case* c, const double* x, const double* xbc, double* out) {
  int m = c->m, n = c->n;
  int left = c->left, right = c->right, bottom = c->bottom, top = c->top;
  for (int i = 2; i <= m; i++) {
    for (int j = 2; j <= n - 1; j++) X1(out, UI(i, j)) = OM(x, i, j + 1) - OM(x, i, j);
    int j = 1;
    X1(out, UI(i, j)) = OM(x, i, j + 1) - X1(xbc, bottom + i);
    j = n;
    X1(out, UI(i, j)) = X1(xbc, top + i) - OM(x, i, j);
  }
  {
    int i = 1;
    for (int j = 1; j <= n; j++) X1(out, UI(i, j)) = X1(xbc, left + j + 1) - X1(xbc, left + j);
    i = m + 1;
    for (int j = 1; j <= n; j++) X1(out, UI(i, j)) = X1(xbc, right + j + 1) - X1(xbc, right + j);
  }
  for (int j = 2; j <= n; j++) {
    for (int i = 2; i <= m - 1; i++) X1(out, VI(i, j)) = OM(x, i, j) - OM(x, i + 1, j);
    int i = 1;
    X1(out, VI(i, j)) = -OM(x, i + 1, j) + X1(xbc, left + j);
    i = m;
    X1(out, VI(i, j)) = -X1(xbc, right + j) + OM(x, i, j);
  }
  {
    int j = 1;
    for (int i = 1; i <= m; i++) X1(out, VI(i, j)) = X1(xbc, bottom + i) - X1(xbc, bottom + i + 1);
    j = n + 1;
    for (int i = 1; i <= m; i++) X1(out, VI(i, j)) = X1(xbc, top + i) - X1(xbc, top + i + 1);
  }
}

/* rot (operators.f90:291-304). */
void or_rot(const or_case* c, const double* x, double* out) {
  int m = c->m, n = c->n;
  for (int i = 2; i <= m; i++)
    for (int j = 2; j <= n; j++)
      OM(out, i, j) = X1(x, VI(i, j)) - X1(x, VI(i - 1, j)) - X1(x, UI(i, j)) + X1(x, UI(i, j - 1));
}

/* nonlinear (operators.f90:465-510). Entries of fq not written by the
 * reference (u at i=1,m+1; v at j=1,n+1) are set to zero here. */
void or_nonlinear(const or_case* c, const double* omega, const double* q,
                  const double* q0, const double* bc, double* fq) {
  int m = c->m, n = c->n;
  int left = c->left, right = c->right, bottom = c->bottom, top = c->top;
  double* uavg = (double*)malloc(sizeof(double) * (m + 1) * (n - 1)); /* (1:m+1,2:n) */
  double* vavg = (double*)malloc(sizeof(double) * (m - 1) * (n + 1)); /* (2:m,1:n+1) */
#define UAVG(i, j) uavg[((i)-1) + ((j)-2) * (m + 1)]
#define VAVG(i, j) vavg[((i)-2) + ((j)-1) * (m - 1)]
  for (int j = 2; j <= n; j++)
    for (int i = 1; i <= m + 1; i++)
      UAVG(i, j) = 0.5 * (X1(q, UI(i, j)) + X1(q, UI(i, j - 1)) + X1(q0, UI(i, j)) + X1(q0, UI(i, j - 1)));
  for (int j = 1; j <= n + 1; j++)
    for (int i = 2; i <= m; i++)
      VAVG(i, j) = 0.5 * (X1(q, VI(i, j)) + X1(q, VI(i - 1, j)) + X1(q0, VI(i, j)) + X1(q0, VI(i - 1, j)));
  memset(fq, 0, sizeof(double) * c->nq);
  for (int i = 2; i <= m; i++) {
    for (int j = 2; j <= n - 1; j++)
      X1(fq, UI(i, j)) = 0.5 * (VAVG(i, j + 1) * OM(omega, i, j + 1) + VAVG(i, j) * OM(omega, i, j));
    int j = 1;
    X1(fq, UI(i, j)) = 0.5 * (VAVG(i, j + 1) * OM(omega, i, j + 1) + VAVG(i, j) * X1(bc, bottom + i));
    j = n;
    X1(fq, UI(i, j)) = 0.5 * (VAVG(i, j + 1) * X1(bc, top + i) + VAVG(i, j) * OM(omega, i, j));
  }
  for (int j = 2; j <= n; j++) {
    for (int i = 2; i <= m - 1; i++)
      X1(fq, VI(i, j)) = -0.5 * (UAVG(i + 1, j) * OM(omega, i + 1, j) + UAVG(i, j) * OM(omega, i, j));
    int i = 1;
    X1(fq, VI(i, j)) = -0.5 * (UAVG(i + 1, j) * OM(omega, i + 1, j) + UAVG(i, j) * X1(bc, left + j));
    i = m;
    X1(fq, VI(i, j)) = -0.5 * (UAVG(i + 1, j) * X1(bc, right + j) + UAVG(i, j) * OM(omega, i, j));
  }
#undef UAVG
#undef VAVG
  free(uavg);
  free(vavg);
}

/* coarsify (operators.f90:307-333): out may alias crhs. */
void or_coarsify(const or_case* c, const double* crhs, const double* rhs, double* out) {
  int m = c->m, n = c->n;
  if (out != crhs) memcpy(out, crhs, sizeof(double) * c->ns);
  for (int i = m / 4 + 2; i <= 3 * m / 4; i++) {
    int ii = 2 * i - m / 2 - 1;
    for (int j = n / 4 + 2; j <= 3 * n / 4; j++) {
      int jj = 2 * j - n / 2 - 1;
      OM(out, i, j) = OM(rhs, ii, jj) +
                      0.50 * (OM(rhs, ii - 1, jj) + OM(rhs, ii + 1, jj) + OM(rhs, ii, jj - 1) + OM(rhs, ii, jj + 1)) +
                      0.25 * (OM(rhs, ii - 1, jj - 1) + OM(rhs, ii - 1, jj + 1) + OM(rhs, ii + 1, jj - 1) + OM(rhs, ii + 1, jj + 1));
    }
  }
}

/* get_bc (operators.f90:336-367); r is an assumed-shape (1-based) section. */
void or_get_bc(const or_case* c, const double* r, double* rbc, double fac) {
  int m = c->m, n = c->n;
  int left = c->left, right = c->right, bottom = c->bottom, top = c->top;
  for (int i = 0; i <= m; i += 2) {
    X1(rbc, bottom + i + 1) = R1(r, m / 4 + i / 2, n / 4);
    X1(rbc, top + i + 1) = R1(r, m / 4 + i / 2, 3 * n / 4);
  }
  for (int i = 1; i <= m - 1; i += 2) {
    X1(rbc, bottom + i + 1) = 0.5 * (R1(r, m / 4 + (i + 1) / 2, n / 4) + R1(r, m / 4 - 1 + (i + 1) / 2, n / 4));
    X1(rbc, top + i + 1) = 0.5 * (R1(r, m / 4 + (i + 1) / 2, 3 * n / 4) + R1(r, m / 4 - 1 + (i + 1) / 2, 3 * n / 4));
  }
  for (int j = 0; j <= n; j += 2) {
    X1(rbc, left + j + 1) = R1(r, m / 4, n / 4 + j / 2);
    X1(rbc, right + j + 1) = R1(r, 3 * m / 4, n / 4 + j / 2);
  }
  for (int j = 1; j <= n - 1; j += 2) {
    X1(rbc, left + j + 1) = 0.5 * (R1(r, m / 4, n / 4 + (j + 1) / 2) + R1(r, m / 4, n / 4 - 1 + (j + 1) / 2));
    X1(rbc, right + j + 1) = 0.5 * (R1(r, 3 * m / 4, n / 4 + (j + 1) / 2) + R1(r, 3 * m / 4, n / 4 - 1 + (j + 1) / 2));
  }
  int nr = 2 * (m + 1) + 2 * (n + 1);
  for (int t = 0; t < nr; t++) rbc[t] = rbc[t] * fac;
}

/* apply_bc (operators.f90:370-390); r is an assumed-shape (1-based) array. */
void or_apply_bc(const or_case* c, double* r, const double* rbc, double fac) {
  int m = c->m, n = c->n;
  int left = c->left, right = c->right, bottom = c->bottom, top = c->top;
  for (int i = 1; i <= m - 1; i++) {
    R1(r, i, 1) = R1(r, i, 1) + fac * X1(rbc, bottom + i + 1);
    R1(r, i, n - 1) = R1(r, i, n - 1) + fac * X1(rbc, top + i + 1);
  }
  for (int j = 1; j <= n - 1; j++) {
    R1(r, 1, j) = R1(r, 1, j) + fac * X1(rbc, left + j + 1);
    R1(r, m - 1, j) = R1(r, m - 1, j) + fac * X1(rbc, right + j + 1);
  }
}

/* reg (operators.f90:513-528). */
void or_reg(const or_case* c, const double* h0, double* h) {
  size_t nq = c->nq;
  for (size_t i = 0; i < nq; i++) {
    double s = 0.0;
    for (int k = 0; k < c->nsmear; k++)
      s = s + c->smear[i + k * nq] * X1(h0, c->ismear[i + k * nq]);
    h[i] = s;
  }
}

/* regT (operators.f90:531-546). */
void or_regT(const or_case* c, const double* h, double* h0) {
  size_t nq = c->nq;
  memset(h0, 0, sizeof(double) * c->nf);
  for (size_t i = 0; i < nq; i++)
    for (int k = 0; k < c->nsmear; k++)
      X1(h0, c->ismear[i + k * nq]) = X1(h0, c->ismear[i + k * nq]) + c->smear[i + k * nq] * h[i];
}

/* vort2flux (operators.f90:191-240): modifies omega levels 2..L in place. */
void or_vort2flux(or_case* c, double* vel, double* omega, int nlev) {
  int m = c->m, n = c->n, L = c->L;
  size_t ns = c->ns, nq = c->nq;
  int nr = 2 * (m + 1) + 2 * (n + 1);
  double* s = (double*)malloc(sizeof(double) * ns);
  double* vort = (double*)malloc(sizeof(double) * ns);
  double* sbc = (double*)calloc(nr, sizeof(double));
  (void)m; (void)n;
  for (int k = 2; k <= L; k++)
    or_coarsify(c, omega + (k - 1) * ns, omega + (k - 2) * ns, omega + (k - 1) * ns);
  memcpy(vort, omega + (L - 1) * ns, sizeof(double) * ns);
  or_ctci(c, vort, s);
  if (nlev >= L) or_curl(c, s, sbc, vel + (L - 1) * nq);
  for (int k = L - 1; k >= 1; k--) {
    or_get_bc(c, s, sbc, 1.0);
    memcpy(vort, omega + (k - 1) * ns, sizeof(double) * ns);
    or_apply_bc(c, vort, sbc, 1.0);
    or_ctci(c, vort, s);
    if (nlev >= k) or_curl(c, s, sbc, vel + (k - 1) * nq);
  }
  free(s);
  free(vort);
  free(sbc);
}

/* a_times (operators.f90:444-462). */
void or_a_times(or_case* c, const double* x, double* out) {
  size_t ns = c->ns, nq = c->nq;
  int L = c->L;
  double* vort = (double*)calloc(ns * L, sizeof(double));
  double* h = (double*)malloc(sizeof(double) * nq);
  double* r = (double*)malloc(sizeof(double) * ns);
  double* vel = (double*)malloc(sizeof(double) * nq);
  or_reg(c, x, h);
  or_rot(c, h, r);
  or_ainv(c, r, vort);
  or_vort2flux(c, vel, vort, 1);
  or_regT(c, vel, out);
  free(vort);
  free(h);
  free(r);
  free(vel);
}

/* choldc (operators.f90:766-791). */
static int choldc(or_case* c) {
  int nf = c->nf;
  double* A = c->cholmat;
#define CM(i, j) A[((i)-1) + (size_t)((j)-1) * nf]
  for (int i = 1; i <= nf; i++)
    for (int j = i; j <= nf; j++) {
      double sum = CM(i, j);
      for (int k = i - 1; k >= 1; k--) sum = sum - CM(i, k) * CM(j, k);
      if (i == j) {
        if (sum <= 0.0) return 2;
        c->cholvec[i - 1] = sqrt(sum);
      } else {
        CM(j, i) = sum / c->cholvec[i - 1];
      }
    }
  return 0;
}

/* cholsl (operators.f90:794-819). */
void or_cholsl(const or_case* c, const double* b, double* x) {
  int nf = c->nf;
  const double* A = c->cholmat;
  for (int i = 1; i <= nf; i++) {
    double sum = b[i - 1];
    for (int k = i - 1; k >= 1; k--) sum = sum - CM(i, k) * x[k - 1];
    x[i - 1] = sum / c->cholvec[i - 1];
  }
  for (int i = nf; i >= 1; i--) {
    double sum = x[i - 1];
    for (int k = i + 1; k <= nf; k++) sum = sum - CM(k, i) * x[k - 1];
    x[i - 1] = sum / c->cholvec[i - 1];
  }
#undef CM
}

/* preprocess (operators.f90:29-59), without the ibfs.chd cache. */
int or_preprocess(or_case* c) {
  int nf = c->nf;
  double* z = (double*)calloc(nf, sizeof(double));
  for (int i = 0; i < nf; i++) {
    memset(z, 0, sizeof(double) * nf);
    z[i] = 1.0;
    or_a_times(c, z, c->cholmat + (size_t)i * nf);
  }
  free(z);
  return choldc(c);
}

static double dot(const double* a, const double* b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s = s + a[i] * b[i];
  return s;
}

/* cjgr (operators.f90:393-441): x holds the initial guess on entry. */
static int cjgr(or_case* c, double* x, const double* b, int* iters) {
  int nf = c->nf;
  if (iters) *iters = 0;
  if (nf <= 0) return 0;  /* no body points: nothing to solve */
  double* r = (double*)malloc(sizeof(double) * nf);
  double* d = (double*)malloc(sizeof(double) * nf);
  double* q = (double*)malloc(sizeof(double) * nf);
  double* s = (double*)malloc(sizeof(double) * nf);
  int iter = 0;
  or_a_times(c, x, q);
  for (int i = 0; i < nf; i++) r[i] = b[i] - q[i];
  memcpy(d, r, sizeof(double) * nf);
  double delta_new = dot(r, d, nf);
  double eps = c->p.cgtol * c->p.cgtol;
  if (c->cg_rel) eps = eps * dot(b, b, nf);
  while (iter < c->p.cg_max_iter && delta_new > eps) {
    iter++;
    or_a_times(c, d, q);
    double alpha = delta_new / dot(d, q, nf);
    for (int i = 0; i < nf; i++) x[i] = x[i] + alpha * d[i];
    if (iter % 50 == 0) {
      or_a_times(c, x, s);
      for (int i = 0; i < nf; i++) r[i] = b[i] - s[i];
    } else {
      for (int i = 0; i < nf; i++) r[i] = r[i] - alpha * q[i];
    }
    memcpy(s, r, sizeof(double) * nf);
    double delta_old = delta_new;
    delta_new = dot(r, s, nf);
    double beta = delta_new / delta_old;
    for (int i = 0; i < nf; i++) d[i] = s[i] + beta * d[i];
  }
  free(r); free(d); free(q); free(s);
  if (iters) *iters = iter;
  return iter == c->p.cg_max_iter ? 3 : 0;
}

/* advance (operators.f90:62-188). */
int or_advance(or_case* c, int* itime, const double* body_vel, double* fx,
               double* fy, double* circ, double* slip_out, int* cg_iters) {
  int m = c->m, n = c->n, L = c->L, nf = c->nf, nb = c->nb;
  size_t ns = c->ns, nq = c->nq;
  int nr = 2 * (m + 1) + 2 * (n + 1);
  int rc = 0;
  *itime = *itime + 1;
  int it = *itime;
  if (it == 1 && c->p.stationary) {
    rc = or_preprocess(c);
    if (rc) return rc;
  }
  double* rhs = (double*)malloc(sizeof(double) * ns);
  double* rhsbc = (double*)malloc(sizeof(double) * ns);
  double* t1 = (double*)malloc(sizeof(double) * ns);
  double* t2 = (double*)malloc(sizeof(double) * ns);
  double* fq = (double*)malloc(sizeof(double) * nq);
  double* omega_bc = (double*)malloc(sizeof(double) * nr);
  double* lastbc = (double*)malloc(sizeof(double) * nr * L);
  double* motion = (double*)calloc(nf > 0 ? nf : 1, sizeof(double));
  double* rhsf = (double*)malloc(sizeof(double) * (nf > 0 ? nf : 1));
  double* tmpf = (double*)malloc(sizeof(double) * (nf > 0 ? nf : 1));
  double* h = (double*)malloc(sizeof(double) * nq);

  /* STEP 1 (operators.f90:97-134) */
  for (int k = 1; k <= L - 1; k++) or_get_bc(c, c->omega + k * ns, lastbc + (k - 1) * nr, 0.25);
  memset(lastbc + (L - 1) * nr, 0, sizeof(double) * nr);
  for (int k = L; k >= 1; k--) {
    double* om = c->omega + (k - 1) * ns;
    double* ro = c->rhs_old + (k - 1) * ns;
    if (k < L) or_get_bc(c, c->omega + k * ns, omega_bc, 0.25);
    else memset(omega_bc, 0, sizeof(double) * nr);
    or_nonlinear(c, om, c->q + (k - 1) * nq, c->q0 + (k - 1) * nq, lastbc + (k - 1) * nr, fq);
    or_rot(c, fq, rhs);
    if (it == 1) memcpy(ro, rhs, sizeof(double) * ns);
    memset(rhsbc, 0, sizeof(double) * ns);
    or_apply_bc(c, rhsbc, lastbc + (k - 1) * nr, c->vfac[k - 1]);
    or_apply_bc(c, rhsbc, omega_bc, c->vfac[k - 1]);
    const double* l1 = c->lam1 + (k - 1) * ns;
    const double* l1i = c->lam1i + (k - 1) * ns;
    for (size_t a = 0; a < ns; a++)
      t1[a] = c->con1[k - 1] * rhs[a] + c->con2[k - 1] * ro[a] + rhsbc[a];
    or_dst(c, t1, t1);
    or_dst(c, om, t2);
    for (size_t a = 0; a < ns; a++) t1[a] = l1i[a] * (t1[a] + l1[a] * t2[a]);
    or_dst(c, t1, om);
    memcpy(ro, rhs, sizeof(double) * ns);
  }

  /* STEP 2 (operators.f90:142-171) */
  int anymove = 0;
  for (int k = 0; k < nb; k++) if (c->bdyno[k] > 0) anymove = 1;
  if (body_vel) {
    for (int i = 0; i < nf; i++) motion[i] = body_vel[i] * c->delta; /* grid.f90:573-574 */
  } else if (anymove) {
    for (int i = 0; i < nf; i++) motion[i] = 0.0; /* move_body with no example enabled */
  }
  or_regT(c, c->q0, tmpf); /* regT(q0(:,1)) */
  for (int i = 0; i < nf; i++) motion[i] = motion[i] - tmpf[i];
  or_vort2flux(c, c->q, c->omega, 1);
  or_regT(c, c->q, rhsf);
  for (int i = 0; i < nf; i++) rhsf[i] = rhsf[i] - motion[i];
  int iters = 0;
  if (c->p.stationary) {
    or_cholsl(c, rhsf, c->fb);
  } else {
    rc = cjgr(c, c->fb, rhsf, &iters);
  }
  if (cg_iters) *cg_iters = iters;

  /* STEP 3 (operators.f90:174) */
  or_reg(c, c->fb, h);
  or_rot(c, h, t1);
  or_ainv(c, t1, t2);
  for (size_t a = 0; a < ns; a++) c->omega[a] = c->omega[a] - t2[a];

  /* STEP 4 (operators.f90:177) */
  or_vort2flux(c, c->q, c->omega, L);

  /* write_force (operators.f90:583-659) with xg = fb/dt */
  if (fx || fy) {
    int bmin = 0, bmax = 0;
    for (int k = 0; k < nb; k++) {
      if (k == 0 || c->bdyno[k] < bmin) bmin = c->bdyno[k];
      if (k == 0 || c->bdyno[k] > bmax) bmax = c->bdyno[k];
    }
    double* gtemp = tmpf;
    for (int b = bmin; b <= bmax; b++) {
      for (int i = 0; i < nf; i++) gtemp[i] = 0.0;
      for (int i = 0; i < nb; i++)
        if (c->bdyno[i] == b) {
          gtemp[i] = c->fb[i] / c->p.dt;
          gtemp[i + nb] = c->fb[i + nb] / c->p.dt;
        }
      or_reg(c, gtemp, h);
      double sx = 0.0, sy = 0.0;
      for (int i = 1; i <= m + 1; i++)
        for (int j = 1; j <= n; j++) sx = sx + X1(h, UI(i, j));
      for (int j = 1; j <= n + 1; j++)
        for (int i = 1; i <= m; i++) sy = sy + X1(h, VI(i, j));
      if (fx) fx[b - bmin] = sx * 2.0 * c->delta;
      if (fy) fy[b - bmin] = sy * 2.0 * c->delta;
    }
  }
  /* write_circ (operators.f90:662-699) */
  if (circ) {
    for (int k = 1; k <= L; k++) {
      double s = 0.0;
      const double* om = c->omega + (k - 1) * ns;
      for (int i = 2; i <= m; i++)
        for (int j = 2; j <= n; j++) s = s + OM(om, i, j);
      circ[k - 1] = s;
    }
  }
  /* write_slip (operators.f90:549-580) */
  if (slip_out) {
    or_regT(c, c->q, tmpf);
    double s = 0.0;
    for (int i = 0; i < nf; i++) {
      double d = fabs(tmpf[i] - motion[i]);
      if (d > s) s = d;
    }
    *slip_out = s;
  }
  free(rhs); free(rhsbc); free(t1); free(t2); free(fq); free(omega_bc);
  free(lastbc); free(motion); free(rhsf); free(tmpf); free(h);
  return rc;
}
