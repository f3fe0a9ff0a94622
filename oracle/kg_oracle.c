/*
 * kg_oracle.c -- CPU FP64 restatement of the KG method-of-lines path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle: it is
 * compiled into oracle/_build/libkg_oracle.so and may be loaded only by
 * tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline /
 * --impl reference leg.  The product (kg_b200/, libkg_b200.so) never links,
 * loads or calls it.
 *
 * What it restates (reference paths are relative to the FlavioRosales/KG tree):
 *   grid            MoL/mesh_refinement_lib.f90:100-147
 *   metric tables   MoL/geometry.f90:92-406 (Kerr_Schild, Schw_EF)
 *   metric check    MoL/geometry.f90:409-492
 *   dt rule         MoL/diagnostic_lib.f90:101-107
 *   stencils        tools/finite_differences.f90:17-44, 193-239, 310-338, 767-801
 *   RHS             MoL/lines_method_lib.f90:671-753
 *   steppers        MoL/lines_method_lib.f90:211-474
 *   boundaries      MoL/lines_method_lib.f90:507-597
 *   diagnostics     MoL/diagnostic_lib.f90:185-289, tools/integral.f90:220-362,646-704
 *   projection      tools/FFT_sph.f90:247-336, 525-651
 *
 * Semantics follow the Fortran whole-array statements one by one: each
 * operator returns a full temporary, expressions are evaluated left to right
 * in the same order as the Fortran source, complex-by-real products and
 * quotients are taken component-wise (what gfortran emits for a real operand),
 * and the file is compiled with -ffp-contract=off so no multiply-add is fused.
 *
 * Parity pinning: the reference cannot be built here (no Fortran compiler,
 * MPI, HDF5 or GSL in the image).  The restatement is pinned against the
 * reference's own self-checks (inverse-metric identity to 1e-10, Y_lm
 * orthonormality to 1e-5, the analytic l<=2 forms of tools/harmonics.f90)
 * and against an independent whole-array numpy restatement
 * (oracle/kg_numpy.py); bit-for-bit agreement with the Fortran binary itself
 * is therefore unpinned.
 *
 * The one third-party routine on the path, GSL's gsl_sf_legendre_Plm
 * (version not pinned by the reference Makefile), is restated as the standard
 * upward recurrence in l from P_m^m = (-1)^m (2m-1)!! (1-x^2)^{m/2}, which
 * carries the Condon-Shortley phase like GSL's.
 *
 * Array layout: the state is the reference's u(1:5, -g:Nx+g, -g:Ny+g, 0:Nz)
 * complex(8) array in Fortran order (variable fastest).  Internally each
 * variable is a separate 3-D complex array with r fastest.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

enum { KGO_KERR_SCHILD = 0, KGO_SCHW_EF = 1 };
enum { KGO_OUTFLOW = 0, KGO_INFLOW = 1 };

typedef struct kgo_params {
  int Nx, Ny, Nz, g_pts;     /* reference namelist integers */
  double xmin, xmax, tmin, tmax, CFL;
  double a, M_bh, m;         /* spin, BH mass, field mass */
  int metric;                /* KGO_KERR_SCHILD / KGO_SCHW_EF */
  int bc_rmax;               /* KGO_OUTFLOW / KGO_INFLOW */
  int n_det;                 /* number of detectors (>= 2) */
  int l_max;                 /* Y_lm table size used by the projection */
  double dt_override;        /* > 0 replaces the reference dt rule */
} kgo_params;

typedef struct kgo {
  kgo_params p;
  int Nx, Ny, Nz, g;
  int iL, iR, jL, jR, kL, kR;   /* -g..Nx+g, -g..Ny+g, 0..Nz */
  int NI, NJ, NK;
  size_t npts;
  double xmin, xmax, dx, dy, dz, dt, t;
  int Nt;
  /* 2-D (r, theta) metric tables, index (i-iL) + NI*(j-jL) */
  double *x1d, *y1d;
  double *g_dn[4][4], *g_up[4][4];
  double *alpha, *sqrtg, *beta[3], *gamma_up[3][3], *dx_beta;
  /* state arrays, each 5 x 3-D complex */
  cplx *u[5], *u_p[5], *u_stage[5], *u_stage_2[5];
  cplx *k1[5], *k2[5], *k3[5], *k4[5], *rhs_u[5];
  cplx *tmp[6];
  /* detectors */
  double *r_det; int *index_det;
  /* scheme: 0 = the reference's second-order method, 1 = configured method */
  int scheme; double ko_eps;
  double *dx_beta4;          /* d_r beta^r by the fourth-order stencil (scheme 1) */
} kgo;

/* ------------------------------------------------------------------ */
static inline size_t P3(const kgo *s, int i, int j, int k) {
  return (size_t)(i - s->iL) + (size_t)s->NI * ((size_t)(j - s->jL) + (size_t)s->NJ * (size_t)(k - s->kL));
}
static inline size_t P2(const kgo *s, int i, int j) {
  return (size_t)(i - s->iL) + (size_t)s->NI * (size_t)(j - s->jL);
}
static inline cplx cadd(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cplx csub(cplx a, cplx b) { cplx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cplx cneg(cplx a) { cplx r = {-a.re, -a.im}; return r; }
static inline cplx rmul(double s, cplx a) { cplx r = {s * a.re, s * a.im}; return r; }
static inline cplx cmulr(cplx a, double s) { cplx r = {a.re * s, a.im * s}; return r; }
static inline cplx cdivr(cplx a, double s) { cplx r = {a.re / s, a.im / s}; return r; }

#define FOR_ALL(s) for (int k = (s)->kL; k <= (s)->kR; ++k) for (int j = (s)->jL; j <= (s)->jR; ++j) for (int i = (s)->iL; i <= (s)->iR; ++i)
#define OMP_K _Pragma("omp parallel for schedule(static)")

static void *xcalloc(size_t n, size_t sz) { void *p = calloc(n, sz); if (!p) abort(); return p; }

/* ------------------------------------------------------------------ */
/* finite differences (tools/finite_differences.f90)                   */

/* first_derivative_x_2_uniform, finite_differences.f90:17-44 */
static void op_dx1(const kgo *s, const cplx *f, cplx *df, double h) {
  const double res = 0.50 / h;
  const int a = s->iL, b = s->iR;
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k)
    for (int j = s->jL; j <= s->jR; ++j) {
      const cplx *F = f + P3(s, a, j, k); cplx *D = df + P3(s, a, j, k);
      D[0] = cmulr(csub(cadd(cneg(rmul(3.0, F[0])), rmul(4.0, F[1])), F[2]), res);
      for (int i = a + 1; i <= b - 1; ++i) {
        int o = i - a;
        D[o] = cmulr(cadd(cneg(F[o - 1]), F[o + 1]), res);
      }
      int n = b - a;
      D[n] = cmulr(cadd(csub(rmul(3.0, F[n]), rmul(4.0, F[n - 1])), F[n - 2]), res);
    }
}

/* first_derivative_y_2, finite_differences.f90:193-239 (row bounds(2,1)
 * is overwritten by the pole formula for every k; inpar selects it). */
static void op_dx2(const kgo *s, const cplx *f, cplx *df, double h, int inpar) {
  const double res = 0.50 / h;
  const int jl = s->jL, jr = s->jR;
  const int dis = s->kR / 2;
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) {
    const int kt = (k + dis) % (s->kR - 1);
    for (int i = s->iL; i <= s->iR; ++i) {
      if (inpar)
        df[P3(s, i, jl, k)] = cmulr(cadd(f[P3(s, i, jl + 2, kt)], f[P3(s, i, jl + 1, k)]), res);
      else
        df[P3(s, i, jl, k)] = cmulr(cadd(cneg(f[P3(s, i, jl + 1, k)]), f[P3(s, i, jl + 2, kt)]), res);
    }
    for (int j = jl + 1; j <= jr - 1; ++j)
      for (int i = s->iL; i <= s->iR; ++i)
        df[P3(s, i, j, k)] = cmulr(cadd(cneg(f[P3(s, i, j - 1, k)]), f[P3(s, i, j + 1, k)]), res);
    for (int i = s->iL; i <= s->iR; ++i)
      df[P3(s, i, jr, k)] = cmulr(cadd(csub(rmul(3.0, f[P3(s, i, jr, k)]), rmul(4.0, f[P3(s, i, jr - 1, k)])),
                                       f[P3(s, i, jr - 2, k)]), res);
  }
}

/* first_derivative_z_2, finite_differences.f90:310-338 (seam rows use the
 * duplicated points; the k = Nz row carries the reference's sign). */
static void op_dx3(const kgo *s, const cplx *f, cplx *df, double h) {
  const double res = 0.50 / h;
  const int kl = s->kL, kr = s->kR;
  OMP_K
  for (int k = kl; k <= kr; ++k)
    for (int j = s->jL; j <= s->jR; ++j)
      for (int i = s->iL; i <= s->iR; ++i) {
        cplx v;
        if (k == kl) v = cadd(cneg(f[P3(s, i, j, kr - 2)]), f[P3(s, i, j, kl + 1)]);
        else if (k == kr) v = cadd(cneg(f[P3(s, i, j, kl + 2)]), f[P3(s, i, j, kr - 1)]);
        else v = cadd(cneg(f[P3(s, i, j, k - 1)]), f[P3(s, i, j, k + 1)]);
        df[P3(s, i, j, k)] = cmulr(v, res);
      }
}

/* advec_x_uniform, finite_differences.f90:767-801 */
static void op_ad1(const kgo *s, const cplx *f, const double *beta2d, cplx *df, double dxh) {
  const double res = 0.5 / dxh;
  const int a = s->iL, b = s->iR;
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k)
    for (int j = s->jL; j <= s->jR; ++j) {
      const cplx *F = f + P3(s, a, j, k); cplx *D = df + P3(s, a, j, k);
      const double *B = beta2d + P2(s, a, j);
      D[0] = cmulr(csub(cadd(cneg(rmul(3.0, F[0])), rmul(4.0, F[1])), F[2]), res);
      D[1] = cmulr(csub(cadd(cneg(rmul(3.0, F[1])), rmul(4.0, F[2])), F[3]), res);
      for (int i = a + 2; i <= b - 2; ++i) {
        int o = i - a;
        if (B[o] > 0.0) D[o] = cmulr(csub(cadd(cneg(rmul(3.0, F[o])), rmul(4.0, F[o + 1])), F[o + 2]), res);
        else if (B[o] < 0.0) D[o] = cmulr(cadd(csub(rmul(3.0, F[o]), rmul(4.0, F[o - 1])), F[o - 2]), res);
        else D[o] = cmulr(csub(F[o + 1], F[o - 1]), res);
      }
      int n = b - a;
      D[n - 1] = cmulr(csub(F[n], F[n - 2]), res);
      D[n] = cmulr(cadd(csub(rmul(3.0, F[n]), rmul(4.0, F[n - 1])), F[n - 2]), res);
    }
}

/* ------------------------------------------------------------------ */
/* grid and metric                                                     */

/* mesh_refinement_boundary / _create with nproc = 1
 * (MoL/mesh_refinement_lib.f90:100-147) and the dt rule
 * (MoL/diagnostic_lib.f90:101-107). */
static void build_grid(kgo *s) {
  const double pi = acos(-1.0);
  double dxr = (s->p.xmax - s->p.xmin) / 1.0;
  s->xmin = s->p.xmin + 0.0 * dxr;
  s->xmax = s->p.xmin + 1.0 * dxr;
  s->dx = (s->xmax - s->xmin) / (double)s->Nx;
  s->dy = pi / (double)(s->Ny - 1);
  s->dz = 2.0 * pi / (double)(s->Nz - 1);
  s->x1d = xcalloc(s->NI, sizeof(double));
  s->y1d = xcalloc(s->NJ, sizeof(double));
  for (int i = s->iL; i <= s->iR; ++i) s->x1d[i - s->iL] = s->xmin + (double)(i + s->g) * s->dx;
  for (int j = s->jL; j <= s->jR; ++j) s->y1d[j - s->jL] = -s->dy / 2.0 + (double)j * s->dy;
  double dxx = s->x1d[1] - s->x1d[0];
  double c1 = dxx, c2 = exp(s->p.xmin) * s->dy, c3 = exp(s->p.xmin) * sin(s->dy / 2.0) * s->dz;
  double mn = c1 < c2 ? c1 : c2; mn = mn < c3 ? mn : c3;
  s->dt = s->p.CFL * mn;
  if (s->p.dt_override > 0.0) s->dt = s->p.dt_override;
  s->Nt = (int)((s->p.tmax - s->p.tmin) / s->dt);
  if (s->Nt % 2 != 0) s->Nt += 1;
  s->t = s->p.tmin;
}

/* geometry_load_metric / geometry_load_inverse / boundary_theta_dn/up
 * (MoL/geometry.f90:92-406).  All tables are phi-independent, so the 2-D
 * (r, theta) slice carries them exactly. */
static void build_metric(kgo *s) {
  const size_t n2 = (size_t)s->NI * s->NJ;
  for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) {
    s->g_dn[a][b] = xcalloc(n2, sizeof(double));
    s->g_up[a][b] = xcalloc(n2, sizeof(double));
  }
  s->alpha = xcalloc(n2, sizeof(double)); s->sqrtg = xcalloc(n2, sizeof(double));
  s->dx_beta = xcalloc(n2, sizeof(double));
  for (int a = 0; a < 3; ++a) { s->beta[a] = xcalloc(n2, sizeof(double));
    for (int b = 0; b < 3; ++b) s->gamma_up[a][b] = xcalloc(n2, sizeof(double)); }
  const double M = s->p.M_bh, A = s->p.a;
  double **gd = &s->g_dn[0][0];
#define GD(a, b) s->g_dn[a][b][q]
#define GU(a, b) s->g_up[a][b][q]
  (void)gd;
  for (int j = s->jL; j <= s->jR; ++j)
    for (int i = s->iL; i <= s->iR; ++i) {
      size_t q = P2(s, i, j);
      double x = s->x1d[i - s->iL], y = s->y1d[j - s->jL];
      if (s->p.metric == KGO_KERR_SCHILD) {
        double cy = cos(y), sy = sin(y);
        double c2 = cy * cy, s2 = sy * sy;
        double rho2 = x * x + (A * A) * c2;
        GD(0, 0) = -1.0 + 2.0 * M * x / rho2;
        GD(0, 1) = (2.0 * M * x / rho2);
        GD(0, 2) = 0.0;
        GD(0, 3) = -(2.0 * A * M * x * s2 / rho2);
        GD(1, 0) = GD(0, 1);
        GD(1, 1) = (1.0 + 2.0 * M * x / rho2);
        GD(1, 2) = 0.0;
        GD(1, 3) = (-(A * (1.0 + 2.0 * M * x / rho2) * s2));
        GD(2, 0) = 0.0; GD(2, 1) = 0.0;
        GD(2, 2) = (x * x + (A * A) * c2);
        GD(2, 3) = 0.0;
        GD(3, 0) = GD(0, 3); GD(3, 1) = GD(1, 3); GD(3, 2) = 0.0;
        double ax = (A * A + x * x);
        GD(3, 3) = ((ax * ax) - (A * A) * (-(2.0 * M * x) + A * A + x * x) * s2) * s2 / rho2;
      } else {
        double sy = sin(y);
        GD(0, 0) = -(1.0 - 2.0 * M / x);
        GD(0, 1) = 2.0 * M / x;
        GD(0, 2) = 0.0; GD(0, 3) = 0.0;
        GD(1, 0) = GD(0, 1);
        GD(1, 1) = 1.0 + 2.0 * M / x;
        GD(1, 2) = 0.0; GD(1, 3) = 0.0;
        GD(2, 0) = GD(0, 2); GD(2, 1) = GD(1, 2);
        GD(2, 2) = x * x;
        GD(2, 3) = 0.0;
        GD(3, 0) = GD(0, 3); GD(3, 1) = GD(1, 3); GD(3, 2) = GD(2, 3);
        GD(3, 3) = x * x * (sy * sy);
      }
    }
  /* boundary_theta_dn: row jR+g <- row jR+g-1 (phi-independent values) */
  {
    int jt = s->jR, js = s->jR - 1;
    for (int i = s->iL; i <= s->iR; ++i) {
      size_t qt = P2(s, i, jt), qs = P2(s, i, js);
      for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) s->g_dn[a][b][qt] = s->g_dn[a][b][qs];
      s->g_dn[0][2][qt] = -s->g_dn[0][2][qs];
      s->g_dn[1][2][qt] = -s->g_dn[1][2][qs];
    }
  }
  for (size_t q = 0; q < n2; ++q) {
    GD(1, 0) = GD(0, 1); GD(2, 0) = GD(0, 2); GD(3, 0) = GD(0, 3);
    GD(2, 1) = GD(1, 2); GD(3, 1) = GD(1, 3); GD(3, 2) = GD(2, 3);
    s->sqrtg[q] = sqrt(GD(2, 2) * (GD(1, 1) * GD(3, 3) - GD(1, 3) * GD(1, 3)));
  }
  for (size_t q = 0; q < n2; ++q) {
    double g00 = GD(0, 0), g01 = GD(0, 1), g03 = GD(0, 3), g11 = GD(1, 1), g13 = GD(1, 3),
           g22 = GD(2, 2), g33 = GD(3, 3);
    double det = ((g33 * g11 - g13 * g13) * g00 - g33 * (g01 * g01) + 2.0 * g13 * g03 * g01 - g11 * (g03 * g03)) * g22;
    double idetg = 1.0 / det;
    GU(0, 0) = g22 * (g11 * g33 - g13 * g13) * idetg;
    GU(0, 1) = g22 * (g13 * g03 - g01 * g33) * idetg;
    GU(0, 2) = 0.0;
    GU(0, 3) = g22 * (g13 * g01 - g11 * g03) * idetg;
    GU(1, 1) = g22 * (g33 * g00 - g03 * g03) * idetg;
    GU(1, 2) = 0.0;
    GU(1, 3) = g22 * (-(g13 * g00) + g03 * g01) * idetg;
    GU(2, 2) = ((g33 * g11 - g13 * g13) * g00 - g33 * (g01 * g01) + 2.0 * g13 * g03 * g01 - g11 * (g03 * g03)) * idetg;
    GU(2, 3) = 0.0;
    GU(3, 3) = g22 * (g11 * g00 - g01 * g01) * idetg;
  }
  {
    int jt = s->jR, js = s->jR - 1;
    for (int i = s->iL; i <= s->iR; ++i) {
      size_t qt = P2(s, i, jt), qs = P2(s, i, js);
      for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) s->g_up[a][b][qt] = s->g_up[a][b][qs];
      s->g_up[0][2][qt] = -s->g_up[0][2][qs];
      s->g_up[1][2][qt] = -s->g_up[1][2][qs];
    }
  }
  for (size_t q = 0; q < n2; ++q) {
    GU(1, 0) = GU(0, 1); GU(2, 0) = GU(0, 2); GU(3, 0) = GU(0, 3);
    GU(2, 1) = GU(1, 2); GU(3, 1) = GU(1, 3); GU(3, 2) = GU(2, 3);
    double al = sqrt(-1.0 / GU(0, 0));
    s->alpha[q] = al;
    double a2 = al * al;
    s->beta[0][q] = a2 * GU(0, 1);
    s->beta[1][q] = a2 * GU(0, 2);
    s->beta[2][q] = a2 * GU(0, 3);
  }
  for (size_t q = 0; q < n2; ++q) {
    double a2 = s->alpha[q] * s->alpha[q];
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b)
      s->gamma_up[a][b][q] = s->g_up[a + 1][b + 1][q] + s->beta[a][q] * s->beta[b][q] / a2;
  }
  /* dx_beta = dx1(dcmplx(beta(1))) (real part), geometry.f90:344 */
  {
    const double res = 0.50 / s->dx;
    for (int j = s->jL; j <= s->jR; ++j) {
      const double *F = s->beta[0] + P2(s, s->iL, j); double *D = s->dx_beta + P2(s, s->iL, j);
      int n = s->iR - s->iL;
      D[0] = (-(3.0 * F[0]) + 4.0 * F[1] - F[2]) * res;
      for (int o = 1; o <= n - 1; ++o) D[o] = (-F[o - 1] + F[o + 1]) * res;
      D[n] = (3.0 * F[n] - 4.0 * F[n - 1] + F[n - 2]) * res;
    }
  }
#undef GD
#undef GU
}

/* validate_inverse_metric, MoL/geometry.f90:409-492: count entries of
 * g_dn.g_up - delta and g_dn(ij).gamma_up - delta above 1e-10. */
int kgo_validate_inverse_metric(const kgo *s, int *errors_4d, int *errors_3d) {
  const double tol = 1.0e-10;
  int e4 = 0, e3 = 0;
  for (int j = s->jL; j <= s->jR; ++j)
    for (int i = s->iL; i <= s->iR; ++i) {
      size_t q = P2(s, i, j);
      for (int mu = 0; mu < 4; ++mu) for (int la = 0; la < 4; ++la) {
        double d = 0.0;
        for (int nu = 0; nu < 4; ++nu) d = d + s->g_dn[mu][nu][q] * s->g_up[nu][la][q];
        if (mu == la ? fabs(d - 1.0) > tol : fabs(d) > tol) e4++;
      }
      for (int mu = 1; mu < 4; ++mu) for (int la = 1; la < 4; ++la) {
        double d = 0.0;
        for (int nu = 1; nu < 4; ++nu) d = d + s->g_dn[mu][nu][q] * s->gamma_up[nu - 1][la - 1][q];
        if (mu == la ? fabs(d - 1.0) > tol : fabs(d) > tol) e3++;
      }
    }
  /* the reference loops over every k as well; tables are k-independent */
  if (errors_4d) *errors_4d = e4 * s->NK;
  if (errors_3d) *errors_3d = e3 * s->NK;
  return e4 + e3;
}

/* ------------------------------------------------------------------ */
/* RHS (MoL/lines_method_lib.f90:671-753)                              */

static double met(const double *t, const kgo *s, int i, int j) { return t[P2(s, i, j)]; }

void kgo_rhs_phi(kgo *s, cplx *rhs, cplx *const *v) {
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k);
    rhs[p] = cadd(rmul(met(s->alpha, s, i, j), v[4][p]), rmul(met(s->beta[0], s, i, j), v[1][p]));
  }
}

void kgo_rhs_psi1(kgo *s, cplx *rhs, cplx *const *v) {
  cplx *t0 = s->tmp[0], *d0 = s->tmp[1], *a0 = s->tmp[2];
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k);
    t0[p] = rmul(met(s->alpha, s, i, j), v[4][p]);
  }
  op_dx1(s, t0, d0, s->dx);
  op_ad1(s, v[1], s->beta[0], a0, s->dx);
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k);
    rhs[p] = cadd(cadd(d0[p], rmul(met(s->beta[0], s, i, j), a0[p])), rmul(met(s->dx_beta, s, i, j), v[1][p]));
  }
}

static void lin_comb_w(kgo *s, cplx *w, cplx *const *v) {
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k);
    w[p] = cadd(rmul(met(s->alpha, s, i, j), v[4][p]), rmul(met(s->beta[0], s, i, j), v[1][p]));
  }
}

void kgo_rhs_psi2(kgo *s, cplx *rhs, cplx *const *v) {
  lin_comb_w(s, s->tmp[0], v);
  op_dx2(s, s->tmp[0], rhs, s->dy, 0);
}

void kgo_rhs_psi3(kgo *s, cplx *rhs, cplx *const *v) {
  lin_comb_w(s, s->tmp[0], v);
  op_dx3(s, s->tmp[0], rhs, s->dz);
}

void kgo_rhs_pi(kgo *s, cplx *rhs, cplx *const *v) {
  cplx *t0 = s->tmp[0], *t1 = s->tmp[1], *t2 = s->tmp[2], *t3 = s->tmp[3], *d = s->tmp[4], *e = s->tmp[5];
  const int ks = (s->p.metric == KGO_KERR_SCHILD);
  const double m2 = s->p.m * s->p.m;
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k), q = P2(s, i, j);
    double al = s->alpha[q], sg = s->sqrtg[q];
    double grr = s->gamma_up[0][0][q], grp = s->gamma_up[0][2][q], gtt = s->gamma_up[1][1][q], gpp = s->gamma_up[2][2][q];
    if (ks) {
      t0[p] = rmul(al * sg, cadd(rmul(grr, v[1][p]), rmul(grp, v[3][p])));
      t1[p] = rmul(al * sg * gtt, v[2][p]);
      t2[p] = rmul(al * sg, cadd(rmul(grp, v[1][p]), rmul(gpp, v[3][p])));
    } else {
      t0[p] = rmul(al * sg * grr, v[1][p]);
      t1[p] = rmul(al * sg * gtt, v[2][p]);
      t2[p] = rmul(al * gpp, v[3][p]);
    }
    t3[p] = cmulr(v[4][p], sg);
  }
  /* dx1(t0) -> d, ad1(t3) -> e, then reuse t0 for dx2(t1) and t3 for dx3(t2) */
  op_dx1(s, t0, d, s->dx);
  op_ad1(s, t3, s->beta[0], e, s->dx);
  op_dx2(s, t1, t0, s->dy, 0);
  op_dx3(s, t2, t3, s->dz);
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k), q = P2(s, i, j);
    double al = s->alpha[q], sg = s->sqrtg[q], b1 = s->beta[0][q], dxb = s->dx_beta[q];
    cplx r1 = cdivr(d[p], sg);
    cplx r2 = cdivr(t0[p], sg);
    cplx r3 = ks ? cdivr(t3[p], sg) : t3[p];
    cplx r4 = cmulr(v[4][p], dxb);
    cplx r5 = cdivr(rmul(b1, e[p]), sg);
    cplx r6 = rmul(al * m2, v[0][p]);
    rhs[p] = csub(cadd(cadd(cadd(cadd(r1, r2), r3), r4), r5), r6);
  }
}

static void rhs_all(kgo *s, cplx *const *v) {
  kgo_rhs_phi(s, s->rhs_u[0], v);
  kgo_rhs_psi1(s, s->rhs_u[1], v);
  kgo_rhs_psi2(s, s->rhs_u[2], v);
  kgo_rhs_psi3(s, s->rhs_u[3], v);
  kgo_rhs_pi(s, s->rhs_u[4], v);
}

/* ------------------------------------------------------------------ */
/* boundaries (MoL/lines_method_lib.f90:507-597), all act on u          */

void kgo_boundary_xL(kgo *s) {
  int i0 = s->iL;
  for (int v = 0; v < 5; ++v) { cplx *u = s->u[v];
    for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j)
      u[P3(s, i0, j, k)] = cadd(csub(rmul(3.0, u[P3(s, i0 + 1, j, k)]), rmul(3.0, u[P3(s, i0 + 2, j, k)])), u[P3(s, i0 + 3, j, k)]);
  }
}
void kgo_boundary_xR(kgo *s) {
  int i0 = s->iR;
  for (int v = 0; v < 5; ++v) { cplx *u = s->u[v], *up = s->u_p[v];
    for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j)
      u[P3(s, i0, j, k)] = (s->p.bc_rmax == KGO_OUTFLOW) ? u[P3(s, i0 - 1, j, k)] : up[P3(s, i0, j, k)];
  }
}
void kgo_boundary_yL(kgo *s) {
  int dis = s->Nz / 2;
  for (int k = s->kL; k <= s->kR; ++k) {
    int kt = (k + dis) % (s->Nz - 1);
    for (int g = s->g; g >= 0; --g)
      for (int v = 0; v < 5; ++v) { cplx *u = s->u[v];
        for (int i = s->iL; i <= s->iR; ++i) u[P3(s, i, 0 - g, k)] = u[P3(s, i, 0 + g + 1, kt)]; }
  }
}
void kgo_boundary_yR(kgo *s) {
  int dis = s->Nz / 2;
  for (int k = s->kL; k <= s->kR; ++k) {
    int kt = (k + dis) % (s->Nz - 1);
    for (int g = s->g; g >= 0; --g)
      for (int v = 0; v < 5; ++v) { cplx *u = s->u[v];
        for (int i = s->iL; i <= s->iR; ++i) u[P3(s, i, s->Ny + g, k)] = u[P3(s, i, s->Ny - g - 1, kt)]; }
  }
}
void kgo_boundary_zL(kgo *s) {
  for (int v = 0; v < 5; ++v) { cplx *u = s->u[v];
    for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i)
      u[P3(s, i, j, s->kL)] = u[P3(s, i, j, s->kR - 1)]; }
}
void kgo_boundary_zR(kgo *s) {
  for (int v = 0; v < 5; ++v) { cplx *u = s->u[v];
    for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i)
      u[P3(s, i, j, s->kR)] = u[P3(s, i, j, s->kL + 1)]; }
}
/* the steppers' internal `boundary` with nproc = 1 */
void kgo_boundary(kgo *s) {
  kgo_boundary_xL(s); kgo_boundary_xR(s);
  kgo_boundary_yL(s); kgo_boundary_yR(s);
  kgo_boundary_zL(s); kgo_boundary_zR(s);
}

/* ------------------------------------------------------------------ */
/* steppers (MoL/lines_method_lib.f90:211-474)                         */

static void copy_state(kgo *s, cplx **dst, cplx *const *src) {
  for (int v = 0; v < 5; ++v) memcpy(dst[v], src[v], s->npts * sizeof(cplx));
}

void kgo_pirk2(kgo *s, int nsteps) {
  const double dt = s->dt;
  for (int step = 0; step < nsteps; ++step) {
    copy_state(s, s->u_p, s->u);
    kgo_rhs_phi(s, s->rhs_u[0], s->u);
    kgo_rhs_psi1(s, s->rhs_u[1], s->u);
    kgo_rhs_psi2(s, s->rhs_u[2], s->u);
    kgo_rhs_psi3(s, s->rhs_u[3], s->u);
    for (int v = 0; v < 4; ++v) { cplx *us = s->u_stage[v], *u = s->u[v], *r = s->rhs_u[v];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) us[p] = cadd(u[p], rmul(dt, r[p])); }
    kgo_rhs_pi(s, s->rhs_u[4], s->u_stage);
    { cplx *us = s->u_stage[4], *u = s->u[4], *r = s->rhs_u[4];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) us[p] = cadd(u[p], rmul(dt, r[p])); }
    kgo_boundary(s);
    rhs_all(s, s->u_stage);
    for (int v = 0; v < 5; ++v) { cplx *u = s->u[v], *up = s->u_p[v], *us = s->u_stage[v], *r = s->rhs_u[v];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) u[p] = rmul(0.5, cadd(cadd(up[p], us[p]), rmul(dt, r[p]))); }
    kgo_boundary(s);
    s->t = s->t + dt;
  }
}

void kgo_pirk3(kgo *s, int nsteps) {
  const double dt = s->dt;
  const double third = 1.0 / 3.0, twothird = 2.0 / 3.0;
  for (int step = 0; step < nsteps; ++step) {
    copy_state(s, s->u_p, s->u);
    kgo_rhs_phi(s, s->rhs_u[0], s->u);
    kgo_rhs_psi1(s, s->rhs_u[1], s->u);
    kgo_rhs_psi2(s, s->rhs_u[2], s->u);
    kgo_rhs_psi3(s, s->rhs_u[3], s->u);
    for (int v = 0; v < 4; ++v) { cplx *us = s->u_stage[v], *u = s->u[v], *r = s->rhs_u[v];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) us[p] = cadd(u[p], rmul(dt, r[p])); }
    kgo_rhs_pi(s, s->rhs_u[4], s->u_stage);
    { cplx *us = s->u_stage[4], *u = s->u[4], *r = s->rhs_u[4];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) us[p] = cadd(u[p], rmul(dt, r[p])); }
    kgo_boundary(s);
    kgo_rhs_phi(s, s->rhs_u[0], s->u_stage);
    kgo_rhs_psi1(s, s->rhs_u[1], s->u_stage);
    kgo_rhs_psi2(s, s->rhs_u[2], s->u_stage);
    kgo_rhs_psi3(s, s->rhs_u[3], s->u_stage);
    for (int v = 0; v < 4; ++v) { cplx *u2 = s->u_stage_2[v], *up = s->u_p[v], *us = s->u_stage[v], *r = s->rhs_u[v];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) u2[p] = cadd(rmul(0.75, up[p]), rmul(0.25, cadd(us[p], rmul(dt, r[p])))); }
    kgo_rhs_pi(s, s->rhs_u[4], s->u_stage_2);
    { cplx *u2 = s->u_stage_2[4], *up = s->u_p[4], *us = s->u_stage[4], *r = s->rhs_u[4];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) u2[p] = cadd(rmul(0.75, up[p]), rmul(0.25, cadd(us[p], rmul(dt, r[p])))); }
    kgo_boundary(s);
    rhs_all(s, s->u_stage_2);
    for (int v = 0; v < 5; ++v) { cplx *u = s->u[v], *up = s->u_p[v], *u2 = s->u_stage_2[v], *r = s->rhs_u[v];
      OMP_K for (long p = 0; p < (long)s->npts; ++p) u[p] = cadd(rmul(third, up[p]), rmul(twothird, cadd(u2[p], rmul(dt, r[p])))); }
    kgo_boundary(s);
    s->t = s->t + dt;
  }
}

/* rk3 with the type-bound rhs_* applied to u as the rhs(1) callback */
void kgo_rk3(kgo *s, int nsteps) {
  const double dt = s->dt;
  for (int step = 0; step < nsteps; ++step) {
    copy_state(s, s->u_p, s->u);
    for (int rk = 1; rk <= 3; ++rk) {
      rhs_all(s, s->u);
      for (int v = 0; v < 5; ++v) { cplx *u = s->u[v], *up = s->u_p[v], *r = s->rhs_u[v];
        OMP_K for (long p = 0; p < (long)s->npts; ++p) {
          if (rk == 1) u[p] = cadd(up[p], cmulr(r[p], dt));
          else if (rk == 2) u[p] = cadd(rmul(0.750, up[p]), rmul(0.250, cadd(u[p], cmulr(r[p], dt))));
          else u[p] = cadd(cdivr(up[p], 3.0), cdivr(rmul(2.0, cadd(u[p], cmulr(r[p], dt))), 3.0));
        } }
      kgo_boundary(s);
    }
    s->t = s->t + dt;
  }
}

static void rk4_cfg(kgo *s, int nsteps);
void kgo_rk4(kgo *s, int nsteps) {
  if (s->scheme == 1) { rk4_cfg(s, nsteps); return; }
  const double dt = s->dt;
  for (int step = 0; step < nsteps; ++step) {
    copy_state(s, s->u_p, s->u);
    for (int rk = 1; rk <= 4; ++rk) {
      rhs_all(s, s->u);
      for (int v = 0; v < 5; ++v) {
        cplx *u = s->u[v], *up = s->u_p[v], *r = s->rhs_u[v];
        cplx *k1 = s->k1[v], *k2 = s->k2[v], *k3 = s->k3[v], *k4 = s->k4[v];
        OMP_K for (long p = 0; p < (long)s->npts; ++p) {
          if (rk == 1) { k1[p] = cmulr(r[p], dt); u[p] = cadd(up[p], rmul(0.50, k1[p])); }
          else if (rk == 2) { k2[p] = cmulr(r[p], dt); u[p] = cadd(up[p], rmul(0.50, k2[p])); }
          else if (rk == 3) { k3[p] = cmulr(r[p], dt); u[p] = cadd(up[p], k3[p]); }
          else { k4[p] = cmulr(r[p], dt);
            u[p] = cadd(up[p], cdivr(cadd(cadd(cadd(k1[p], rmul(2.0, k2[p])), rmul(2.0, k3[p])), k4[p]), 6.0)); }
        }
      }
      kgo_boundary(s);
    }
    s->t = s->t + dt;
  }
}

/* ------------------------------------------------------------------ */
/* configured method (scheme 1): not in the reference, which wires only
 * second-order operators (its fourth-order x stencil, first_derivative_x_4 in
 * tools/finite_differences.f90:124-154, is real-only and never called).
 *   - first derivatives: the centred fourth-order stencil of
 *     first_derivative_x_4, (f(i-2) - 8 f(i-1) + 8 f(i+1) - f(i+2)) / (12 h), on
 *     complex data; in r its one-sided closures at the two first and two last
 *     stored planes; in theta on the interior rows, whose +-2 neighbours are
 *     ghost rows; in phi periodic over the Nz-1 distinct planes.  The shift
 *     advection term uses the same centred operator.
 *   - sixth-order Kreiss-Oliger dissipation on all five variables,
 *     + eps / (64 h) (f(-3) - 6 f(-2) + 15 f(-1) - 20 f(0) + 15 f(1) - 6 f(2) + f(3))
 *     per direction, in r where the stencil fits (planes 3..N-3).
 *   - Sommerfeld condition at the outermost r plane: d_t u = -(d_r u + u / r).
 *   - the innermost r planes (inside the horizon) evolve with the one-sided
 *     closures; no extrapolation.
 *   - ghost fills: the duplicated phi planes, then the theta ghost rows from
 *     the interior rows at phi + pi with the parity of a smooth function on the
 *     sphere (psi_2 = d_theta phi changes sign, the others do not); the theta
 *     flux alpha sqrt(gamma) gamma^thth psi_2 takes the sign of sin(theta) on
 *     the ghost rows.
 * RK4 only; Kerr-Schild metric form only.  Operation order is fixed so the GPU
 * restatement can match it bit for bit. */
static inline cplx d4_r(const kgo *s, cplx (*F)(const kgo *, cplx *const *, int, int, int, int), cplx *const *v,
                        int w, int i, int j, int k, double res) {
  const int a = s->iL, n = s->iR;
  cplx r;
  if (i == a)
    r = csub(cadd(csub(cadd(rmul(-25.0, F(s, v, w, a, j, k)), rmul(48.0, F(s, v, w, a + 1, j, k))),
                       rmul(36.0, F(s, v, w, a + 2, j, k))), rmul(16.0, F(s, v, w, a + 3, j, k))),
             rmul(3.0, F(s, v, w, a + 4, j, k)));
  else if (i == a + 1)
    r = cadd(csub(cadd(csub(rmul(-3.0, F(s, v, w, a, j, k)), rmul(10.0, F(s, v, w, a + 1, j, k))),
                       rmul(18.0, F(s, v, w, a + 2, j, k))), rmul(6.0, F(s, v, w, a + 3, j, k))),
             rmul(1.0, F(s, v, w, a + 4, j, k)));
  else if (i == n - 1)
    r = csub(cadd(csub(cadd(rmul(3.0, F(s, v, w, n, j, k)), rmul(10.0, F(s, v, w, n - 1, j, k))),
                       rmul(18.0, F(s, v, w, n - 2, j, k))), rmul(6.0, F(s, v, w, n - 3, j, k))),
             rmul(1.0, F(s, v, w, n - 4, j, k)));
  else if (i == n)
    r = cadd(csub(cadd(csub(rmul(25.0, F(s, v, w, n, j, k)), rmul(48.0, F(s, v, w, n - 1, j, k))),
                       rmul(36.0, F(s, v, w, n - 2, j, k))), rmul(16.0, F(s, v, w, n - 3, j, k))),
             rmul(3.0, F(s, v, w, n - 4, j, k)));
  else
    r = csub(cadd(csub(F(s, v, w, i - 2, j, k), rmul(8.0, F(s, v, w, i - 1, j, k))), rmul(8.0, F(s, v, w, i + 1, j, k))),
             F(s, v, w, i + 2, j, k));
  return cmulr(r, res);
}
static inline int kper(const kgo *s, int k, int d) {
  const int M = s->kR - 1; /* Nz - 1 distinct planes 1..Nz-1 */
  int kk = (k - 1 + d) % M;
  if (kk < 0) kk += M;
  return kk + 1;
}
static inline cplx d4_c(cplx fm2, cplx fm1, cplx fp1, cplx fp2, double res) {
  return cmulr(csub(cadd(csub(fm2, rmul(8.0, fm1)), rmul(8.0, fp1)), fp2), res);
}
static inline cplx ko6(cplx m3, cplx m2, cplx m1, cplx c0, cplx p1, cplx p2, cplx p3) {
  return cadd(csub(cadd(csub(cadd(csub(m3, rmul(6.0, m2)), rmul(15.0, m1)), rmul(20.0, c0)), rmul(15.0, p1)),
                   rmul(6.0, p2)), p3);
}
/* point functions of the configured RHS */
static cplx cf_A(const kgo *s, cplx *const *v, int w, int i, int j, int k) {
  (void)w;
  return rmul(s->alpha[P2(s, i, j)], v[4][P3(s, i, j, k)]);
}
static cplx cf_E(const kgo *s, cplx *const *v, int w, int i, int j, int k) {
  (void)w;
  size_t q = P2(s, i, j), p = P3(s, i, j, k);
  return cadd(rmul(s->alpha[q], v[4][p]), rmul(s->beta[0][q], v[1][p]));
}
static cplx cf_G1(const kgo *s, cplx *const *v, int w, int i, int j, int k) {
  (void)w;
  size_t q = P2(s, i, j), p = P3(s, i, j, k);
  return rmul(s->alpha[q] * s->sqrtg[q], cadd(rmul(s->gamma_up[0][0][q], v[1][p]), rmul(s->gamma_up[0][2][q], v[3][p])));
}
/* alpha sqrt(gamma) gamma^thth psi_2: sqrt(gamma) ~ r^2 sin(theta) continues
 * through the pole with the sign of sin(theta), so on the ghost rows (theta < 0
 * or > pi, where the table holds |sqrt(gamma)|) the product is negated; with
 * psi_2 odd the flux is then even and smooth across the pole */
static cplx cf_H(const kgo *s, cplx *const *v, int w, int i, int j, int k) {
  (void)w;
  size_t q = P2(s, i, j);
  cplx h = rmul(s->alpha[q] * s->sqrtg[q] * s->gamma_up[1][1][q], v[2][P3(s, i, j, k)]);
  return (j <= 0 || j >= s->Ny) ? cneg(h) : h;
}
static cplx cf_Fp(const kgo *s, cplx *const *v, int w, int i, int j, int k) {
  (void)w;
  size_t q = P2(s, i, j), p = P3(s, i, j, k);
  return rmul(s->alpha[q] * s->sqrtg[q], cadd(rmul(s->gamma_up[0][2][q], v[1][p]), rmul(s->gamma_up[2][2][q], v[3][p])));
}
static cplx cf_Q(const kgo *s, cplx *const *v, int w, int i, int j, int k) {
  (void)w;
  return cmulr(v[4][P3(s, i, j, k)], s->sqrtg[P2(s, i, j)]);
}
static cplx cf_P1(const kgo *s, cplx *const *v, int w, int i, int j, int k) {
  (void)w; return v[1][P3(s, i, j, k)]; }
static cplx cf_V(const kgo *s, cplx *const *v, int w, int i, int j, int k) { return v[w][P3(s, i, j, k)]; }

/* the configured RHS of all five variables at every stored point */
static void rhs_cfg(kgo *s, cplx *const *v) {
  const double rr = 1.0 / (12.0 * s->dx), rt = 1.0 / (12.0 * s->dy), rp = 1.0 / (12.0 * s->dz);
  const double kr = s->ko_eps / (64.0 * s->dx), kt = s->ko_eps / (64.0 * s->dy), kp = s->ko_eps / (64.0 * s->dz);
  const double m2 = s->p.m * s->p.m;
  const int n = s->iR;
  const double rN = s->x1d[s->iR - s->iL];
  const cplx z0 = {0.0, 0.0};
  OMP_K
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k), q = P2(s, i, j);
    if (j <= 0 || j >= s->Ny || k == s->kL || k == s->kR) {
      for (int w = 0; w < 5; ++w) s->rhs_u[w][p] = z0;
      continue;
    }
    if (i == n) { /* Sommerfeld */
      for (int w = 0; w < 5; ++w)
        s->rhs_u[w][p] = cneg(cadd(d4_r(s, cf_V, v, w, i, j, k, rr), cdivr(v[w][p], rN)));
      continue;
    }
    const double al = s->alpha[q], b1 = s->beta[0][q], sg = s->sqrtg[q], dxb = s->dx_beta4[q];
    const int km2 = kper(s, k, -2), km1 = kper(s, k, -1), kp1 = kper(s, k, 1), kp2 = kper(s, k, 2);
    cplx r[5];
    r[0] = cadd(rmul(al, v[4][p]), rmul(b1, v[1][p]));
    r[1] = cadd(cadd(d4_r(s, cf_A, v, 0, i, j, k, rr), rmul(b1, d4_r(s, cf_P1, v, 0, i, j, k, rr))), rmul(dxb, v[1][p]));
    r[2] = d4_c(cf_E(s, v, 0, i, j - 2, k), cf_E(s, v, 0, i, j - 1, k), cf_E(s, v, 0, i, j + 1, k), cf_E(s, v, 0, i, j + 2, k), rt);
    r[3] = d4_c(cf_E(s, v, 0, i, j, km2), cf_E(s, v, 0, i, j, km1), cf_E(s, v, 0, i, j, kp1), cf_E(s, v, 0, i, j, kp2), rp);
    {
      cplx t1 = cdivr(d4_r(s, cf_G1, v, 0, i, j, k, rr), sg);
      cplx t2 = cdivr(d4_c(cf_H(s, v, 0, i, j - 2, k), cf_H(s, v, 0, i, j - 1, k), cf_H(s, v, 0, i, j + 1, k),
                           cf_H(s, v, 0, i, j + 2, k), rt), sg);
      cplx t3 = cdivr(d4_c(cf_Fp(s, v, 0, i, j, km2), cf_Fp(s, v, 0, i, j, km1), cf_Fp(s, v, 0, i, j, kp1),
                           cf_Fp(s, v, 0, i, j, kp2), rp), sg);
      cplx t4 = cmulr(v[4][p], dxb);
      cplx t5 = cdivr(rmul(b1, d4_r(s, cf_Q, v, 0, i, j, k, rr)), sg);
      cplx t6 = rmul(al * m2, v[0][p]);
      r[4] = csub(cadd(cadd(cadd(cadd(t1, t2), t3), t4), t5), t6);
    }
    const int km3 = kper(s, k, -3), kp3 = kper(s, k, 3);
    for (int w = 0; w < 5; ++w) {
      cplx *u = v[w];
      cplx a = r[w];
      if (i >= s->iL + 3 && i <= n - 3)
        a = cadd(a, rmul(kr, ko6(u[P3(s, i - 3, j, k)], u[P3(s, i - 2, j, k)], u[P3(s, i - 1, j, k)], u[p],
                                 u[P3(s, i + 1, j, k)], u[P3(s, i + 2, j, k)], u[P3(s, i + 3, j, k)])));
      a = cadd(a, rmul(kt, ko6(u[P3(s, i, j - 3, k)], u[P3(s, i, j - 2, k)], u[P3(s, i, j - 1, k)], u[p],
                               u[P3(s, i, j + 1, k)], u[P3(s, i, j + 2, k)], u[P3(s, i, j + 3, k)])));
      a = cadd(a, rmul(kp, ko6(u[P3(s, i, j, km3)], u[P3(s, i, j, km2)], u[P3(s, i, j, km1)], u[p],
                               u[P3(s, i, j, kp1)], u[P3(s, i, j, kp2)], u[P3(s, i, j, kp3)])));
      s->rhs_u[w][p] = a;
    }
  }
}

/* ghost fills of the configured method: duplicated phi planes, then the theta
 * ghost rows (three per pole) from interior rows at phi + pi, psi_2 negated */
static void boundary_cfg(kgo *s) {
  const int NZ = s->kR;
  for (int w = 0; w < 5; ++w)
    for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
      s->u[w][P3(s, i, j, 0)] = s->u[w][P3(s, i, j, NZ - 1)];
      s->u[w][P3(s, i, j, NZ)] = s->u[w][P3(s, i, j, 1)];
    }
  const int dis = NZ / 2;
  for (int k = s->kL; k <= s->kR; ++k) {
    const int kt = (k + dis) % (NZ - 1);
    for (int g = s->g; g >= 0; --g)
      for (int w = 0; w < 5; ++w) {
        const double sgn = (w == 2) ? -1.0 : 1.0;
        for (int i = s->iL; i <= s->iR; ++i) {
          s->u[w][P3(s, i, 0 - g, k)] = rmul(sgn, s->u[w][P3(s, i, 0 + g + 1, kt)]);
          s->u[w][P3(s, i, s->Ny + g, k)] = rmul(sgn, s->u[w][P3(s, i, s->Ny - g - 1, kt)]);
        }
      }
  }
}

static void rk4_cfg(kgo *s, int nsteps) {
  const double dt = s->dt;
  for (int step = 0; step < nsteps; ++step) {
    copy_state(s, s->u_p, s->u);
    for (int rk = 1; rk <= 4; ++rk) {
      rhs_cfg(s, s->u);
      for (int v = 0; v < 5; ++v) {
        cplx *u = s->u[v], *up = s->u_p[v], *r = s->rhs_u[v];
        cplx *k1 = s->k1[v], *k2 = s->k2[v], *k3 = s->k3[v], *k4 = s->k4[v];
        for (long p = 0; p < (long)s->npts; ++p) {
          if (rk == 1) { k1[p] = cmulr(r[p], dt); u[p] = cadd(up[p], rmul(0.50, k1[p])); }
          else if (rk == 2) { k2[p] = cmulr(r[p], dt); u[p] = cadd(up[p], rmul(0.50, k2[p])); }
          else if (rk == 3) { k3[p] = cmulr(r[p], dt); u[p] = cadd(up[p], k3[p]); }
          else { k4[p] = cmulr(r[p], dt);
            u[p] = cadd(up[p], cdivr(cadd(cadd(cadd(k1[p], rmul(2.0, k2[p])), rmul(2.0, k3[p])), k4[p]), 6.0)); }
        }
      }
      boundary_cfg(s);
    }
    s->t = s->t + dt;
  }
}

/* 0: the reference's second-order method; 1: the configured method above
 * (RK4 only, Kerr-Schild form); returns 0 or -1 */
int kgo_set_scheme(kgo *s, int scheme, double ko_eps) {
  if (scheme < 0 || scheme > 1) return -1;
  if (scheme == 1 && s->p.metric != KGO_KERR_SCHILD) return -1;
  if (scheme == 1 && !s->dx_beta4) {
    /* first_derivative_x_4 (tools/finite_differences.f90:124-154) of beta^r; the
     * second-order dx_beta of the reference would cap the method at second order */
    s->dx_beta4 = xcalloc((size_t)s->NI * s->NJ, sizeof(double));
    const double res = 1.0 / (12.0 * s->dx);
    const int n = s->iR - s->iL;
    for (int j = s->jL; j <= s->jR; ++j) {
      const double *F = s->beta[0] + P2(s, s->iL, j);
      double *D = s->dx_beta4 + P2(s, s->iL, j);
      D[0] = (-25.0 * F[0] + 48.0 * F[1] - 36.0 * F[2] + 16.0 * F[3] - 3.0 * F[4]) * res;
      D[1] = (-3.0 * F[0] - 10.0 * F[1] + 18.0 * F[2] - 6.0 * F[3] + 1.0 * F[4]) * res;
      for (int o = 2; o <= n - 2; ++o) D[o] = (F[o - 2] - 8.0 * F[o - 1] + 8.0 * F[o + 1] - F[o + 2]) * res;
      D[n - 1] = (3.0 * F[n] + 10.0 * F[n - 1] - 18.0 * F[n - 2] + 6.0 * F[n - 3] - 1.0 * F[n - 4]) * res;
      D[n] = (25.0 * F[n] - 48.0 * F[n - 1] + 36.0 * F[n - 2] - 16.0 * F[n - 3] + 3.0 * F[n - 4]) * res;
    }
  }
  s->scheme = scheme;
  s->ko_eps = ko_eps;
  return 0;
}

/* the configured ghost fills on the current state (initial data) */
void kgo_boundary_cfg(kgo *s) { boundary_cfg(s); }

/* ------------------------------------------------------------------ */
/* diagnostics                                                         */

/* density, MoL/diagnostic_lib.f90:277-289 (result is the real part) */
void kgo_density(const kgo *s, double *rho) {
  const double m2 = s->p.m * s->p.m;
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k), q = P2(s, i, j);
    cplx u1 = s->u[0][p], u2 = s->u[1][p], u3 = s->u[2][p], u4 = s->u[3][p], u5 = s->u[4][p];
    double a5 = hypot(u5.re, u5.im), a2 = hypot(u2.re, u2.im), a3 = hypot(u3.re, u3.im),
           a4 = hypot(u4.re, u4.im), a1 = hypot(u1.re, u1.im);
    double t1 = s->gamma_up[0][0][q] * (a2 * a2);
    cplx t2 = rmul(2.0 * s->gamma_up[0][2][q] * a2, u4);
    double t3 = s->gamma_up[1][1][q] * (a3 * a3);
    double t4 = s->gamma_up[2][2][q] * (a4 * a4);
    double t5 = m2 * a1;
    /* ((((a5 + t1) + t2) + t3) + t4) + t5, complex from t2 on */
    double re = a5 + t1;
    re = re + t2.re;
    re = re + t3; re = re + t4; re = re + t5;
    rho[p] = 0.5 * re;
  }
}

/* trapezium_real over the integrate() slice (tools/integral.f90:220-255,646-674):
 * i in 0..Nx, j in 0..Ny, k in 0..Nz. */
double kgo_integrate_real(const kgo *s, const double *f) {
  int ni = s->Nx + 1, nj = s->Ny + 1, nk = s->Nz + 1;
  double *f2 = xcalloc((size_t)ni * nj, sizeof(double)), *f1 = xcalloc(ni, sizeof(double));
  for (int kk = 0; kk < nk - 1; ++kk)
    for (int jj = 0; jj < nj; ++jj) for (int ii = 0; ii < ni; ++ii) {
      size_t q = (size_t)ii + (size_t)ni * jj;
      f2[q] = f2[q] + f[P3(s, ii, jj, kk)] + f[P3(s, ii, jj, kk + 1)];
    }
  for (size_t q = 0; q < (size_t)ni * nj; ++q) f2[q] = 0.50 * f2[q] * s->dz;
  for (int jj = 0; jj < nj - 1; ++jj)
    for (int ii = 0; ii < ni; ++ii) f1[ii] = f1[ii] + f2[ii + (size_t)ni * jj] + f2[ii + (size_t)ni * (jj + 1)];
  for (int ii = 0; ii < ni; ++ii) f1[ii] = 0.50 * f1[ii] * s->dy;
  double f0 = 0.0;
  for (int ii = 0; ii < ni - 1; ++ii) f0 = f0 + f1[ii] + f1[ii + 1];
  f0 = 0.50 * f0 * s->dx;
  free(f2); free(f1);
  return f0;
}

/* Mass_scalar = integrate(rho*sqrtg) with rho from density() */
double kgo_mass(const kgo *s) {
  double *rho = xcalloc(s->npts, sizeof(double));
  kgo_density(s, rho);
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i)
    rho[P3(s, i, j, k)] = rho[P3(s, i, j, k)] * s->sqrtg[P2(s, i, j)];
  double r = kgo_integrate_real(s, rho);
  free(rho);
  return r;
}

/* currents_ADM, MoL/diagnostic_lib.f90:219-229; out: 3 x npts complex */
void kgo_currents_adm(const kgo *s, double *j_out) {
  cplx *J = (cplx *)j_out;
  for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
    size_t p = P3(s, i, j, k), q = P2(s, i, j);
    cplx u2 = s->u[1][p], u3 = s->u[2][p], u4 = s->u[3][p], u5n = cneg(s->u[4][p]);
    cplx a = cadd(rmul(s->gamma_up[0][0][q], u2), rmul(s->gamma_up[0][2][q], u4));
    cplx b = rmul(s->gamma_up[1][1][q], u3);
    cplx c = cadd(rmul(s->gamma_up[0][2][q], u2), rmul(s->gamma_up[2][2][q], u4));
    /* -u5 * (...) : complex product */
    J[p] = (cplx){u5n.re * a.re - u5n.im * a.im, u5n.re * a.im + u5n.im * a.re};
    J[s->npts + p] = (cplx){u5n.re * b.re - u5n.im * b.im, u5n.re * b.im + u5n.im * b.re};
    J[2 * s->npts + p] = (cplx){u5n.re * c.re - u5n.im * c.im, u5n.re * c.im + u5n.im * c.re};
  }
}

/* domain_to_sph restricted to one vertex r index (1-based iv), tools/FFT_sph.f90:525-651.
 * f_d: 3-D complex on the evolution grid; out: Ny x Nz complex (theta fastest). */
void kgo_domain_to_sph_shell(const kgo *s, const cplx *f_d, int iv, cplx *out) {
  const int b1l = s->iL, b1r = s->iR, b2l = s->jL, b2r = s->jR, b3l = s->kL, b3r = s->kR;
  const double *X = s->x1d, *Y = s->y1d;
#define RD(i) X[(i) - b1l]
#define TD(j) Y[(j) - b2l]
#define PD(k) ((double)(k) * s->dz)
  double rmin = RD(b1l), dr = RD(b1l + 1) - RD(b1l);
  double thetamin = TD(b2l), dth = fabs(TD(b2l + 1) - TD(b2l));
  double phimin = PD(b3l), dph = fabs(PD(b3l + 1) - PD(b3l));
  for (int kv = 1; kv <= s->Nz; ++kv)
    for (int jv = 1; jv <= s->Ny; ++jv) {
      double rr = s->xmin + (double)(iv - 1) * s->dx;
      double tt = (double)(jv - 1) * s->dy;
      double pp = (double)(kv - 1) * s->dz;
      int i_r = (int)((rr - rmin) / dr) + b1l;
      int i_th = (int)((tt - thetamin) / dth) + b2l;
      int i_ph = (int)((pp - phimin) / dph) + b3l;
      if (i_r < b1l) i_r = b1l; if (i_r > b1r - 1) i_r = b1r - 1;
      if (i_th < b2l) i_th = b2l; if (i_th > b2r - 1) i_th = b2r - 1;
      if (i_ph < b3l) i_ph = b3l; if (i_ph > b3r - 1) i_ph = b3r - 1;
      while (i_r < b1r - 1 && rr >= RD(i_r + 1)) i_r++;
      while (i_r > b1l && rr < RD(i_r)) i_r--;
      while (i_th < b2r - 1 && tt >= TD(i_th + 1)) i_th++;
      while (i_th > b2l && tt < TD(i_th)) i_th--;
      while (i_ph < b3r - 1 && pp >= PD(i_ph + 1)) i_ph++;
      while (i_ph > b3l && pp < PD(i_ph)) i_ph--;
      cplx *o = out + (size_t)(jv - 1) + (size_t)s->Ny * (kv - 1);
      if (tt <= thetamin) { *o = f_d[P3(s, i_r, b2l, i_ph)]; continue; }
      if (tt >= thetamin + dth * (double)(b2r - b2l)) { *o = f_d[P3(s, i_r, b2r, i_ph)]; continue; }
      int i_ph_p1 = i_ph + 1;
      if (i_ph_p1 > b3r) continue;
      cplx f000 = f_d[P3(s, i_r, i_th, i_ph)], f001 = f_d[P3(s, i_r, i_th, i_ph_p1)];
      cplx f010 = f_d[P3(s, i_r, i_th + 1, i_ph)], f011 = f_d[P3(s, i_r, i_th + 1, i_ph_p1)];
      cplx f100 = f_d[P3(s, i_r + 1, i_th, i_ph)], f101 = f_d[P3(s, i_r + 1, i_th, i_ph_p1)];
      cplx f110 = f_d[P3(s, i_r + 1, i_th + 1, i_ph)], f111 = f_d[P3(s, i_r + 1, i_th + 1, i_ph_p1)];
      double w_r = (rr - RD(i_r)) / dr, w_th = (tt - TD(i_th)) / dth, w_ph = (pp - PD(i_ph)) / dph;
      cplx f00 = cadd(rmul(1.0 - w_ph, f000), rmul(w_ph, f001));
      cplx f01 = cadd(rmul(1.0 - w_ph, f010), rmul(w_ph, f011));
      cplx f10 = cadd(rmul(1.0 - w_ph, f100), rmul(w_ph, f101));
      cplx f11 = cadd(rmul(1.0 - w_ph, f110), rmul(w_ph, f111));
      cplx f0 = cadd(rmul(1.0 - w_th, f00), rmul(w_th, f01));
      cplx f1 = cadd(rmul(1.0 - w_th, f10), rmul(w_th, f11));
      *o = cadd(rmul(1.0 - w_r, f0), rmul(w_r, f1));
    }
#undef RD
#undef TD
#undef PD
}

/* associated Legendre P_l^m(x) with Condon-Shortley phase (GSL convention) */
static double plm(int l, int m, double x) {
  double pmm = 1.0;
  if (m > 0) {
    double somx2 = sqrt((1.0 - x) * (1.0 + x)), fact = 1.0;
    for (int i = 1; i <= m; ++i) { pmm *= -fact * somx2; fact += 2.0; }
  }
  if (l == m) return pmm;
  double pmmp1 = x * (2.0 * m + 1.0) * pmm;
  if (l == m + 1) return pmmp1;
  double pll = 0.0;
  for (int ll = m + 2; ll <= l; ++ll) {
    pll = (x * (2.0 * ll - 1.0) * pmmp1 - (ll + m - 1.0) * pmm) / (double)(ll - m);
    pmm = pmmp1; pmmp1 = pll;
  }
  return pll;
}

/* sph_harmonics, tools/FFT_sph.f90:282-336.  Ylm(0:L, -L:L, Ny, Nz) complex,
 * index l + (L+1)*((m+L) + (2L+1)*((j-1) + Ny*(k-1))) on the vertex grid. */
void kgo_sph_harmonics(const kgo *s, int L, double *ylm_out) {
  cplx *Y = (cplx *)ylm_out;
  const double pi = acos(-1.0);
  const int NL = L + 1, NM = 2 * L + 1;
  memset(Y, 0, sizeof(cplx) * (size_t)NL * NM * s->Ny * s->Nz);
  for (int l = 0; l <= L; ++l) {
    double fact = sqrt((2.0 * l + 1.0) / (4.0 * pi));
    for (int m = 0; m <= l; ++m) {
      double norm = fact;
      if (m > 0) for (int i = 1; i <= 2 * m; ++i) norm = norm / sqrt((double)(l - m + i));
      for (int jv = 1; jv <= s->Ny; ++jv) {
        double th = (double)(jv - 1) * s->dy;
        double x = cos(th), P;
        if (fabs(x) > 0.9999) P = (m == 0) ? fact : 0.0;
        else P = plm(l, m, x);
        for (int kv = 1; kv <= s->Nz; ++kv) {
          double ph = (double)(kv - 1) * s->dz;
          cplx phase = {cos(m * ph), sin(m * ph)};
          cplx y = rmul(norm * P, phase);
          Y[l + NL * ((m + L) + NM * ((size_t)(jv - 1) + (size_t)s->Ny * (kv - 1)))] = y;
          if (m > 0) {
            double sg = (m % 2) ? -1.0 : 1.0;
            Y[l + NL * ((-m + L) + NM * ((size_t)(jv - 1) + (size_t)s->Ny * (kv - 1)))] = (cplx){sg * y.re, sg * -y.im};
          }
        }
      }
    }
  }
}

/* project_sh, tools/FFT_sph.f90:247-279, with trapezium_2D_complex
 * (tools/integral.f90:330-362).  f: Ny x Nz (theta fastest); out (0:L,-L:L). */
void kgo_project_sh(const kgo *s, const cplx *f, const double *ylm, int L, double *flm_out) {
  const cplx *Y = (const cplx *)ylm;
  cplx *F = (cplx *)flm_out;
  const int NL = L + 1, NM = 2 * L + 1, Nth = s->Ny, Nph = s->Nz;
  memset(F, 0, sizeof(cplx) * NL * NM);
  for (int l = 0; l <= L; ++l)
    for (int m = -l; m <= l; ++m) {
      cplx integ = {0.0, 0.0};
      for (int j = 1; j <= Nth; ++j) {
        double st = sin((double)(j - 1) * s->dy);
        for (int k = 1; k <= Nph; ++k) {
          cplx a = f[(j - 1) + (size_t)Nth * (k - 1)];
          cplx y = Y[l + NL * ((m + L) + NM * ((size_t)(j - 1) + (size_t)Nth * (k - 1)))];
          cplx c = {y.re, -y.im};
          cplx fy = {a.re * c.re - a.im * c.im, a.re * c.im + a.im * c.re};
          cplx fun = {fy.re * st, fy.im * st};
          int sel = ((j == 1 || j == Nth) ? 1 : 0) + 2 * ((k == 1 || k == Nph) ? 1 : 0);
          if (sel == 0) integ = cadd(integ, fun);
          else if (sel == 3) integ = cadd(integ, rmul(0.25, fun));
          else integ = cadd(integ, rmul(0.5, fun));
        }
      }
      double w = s->dy * s->dz;
      F[l + NL * (m + L)] = rmul(w, integ);
    }
}

/* complex trapezium_2D over an Ny x Nz vertex slice (tools/integral.f90:330-362) */
static cplx trap2d(const kgo *s, const cplx *f) {
  cplx integ = {0.0, 0.0};
  for (int j = 1; j <= s->Ny; ++j)
    for (int k = 1; k <= s->Nz; ++k) {
      cplx v = f[(j - 1) + (size_t)s->Ny * (k - 1)];
      int sel = ((j == 1 || j == s->Ny) ? 1 : 0) + 2 * ((k == 1 || k == s->Nz) ? 1 : 0);
      if (sel == 0) integ = cadd(integ, v);
      else if (sel == 3) integ = cadd(integ, rmul(0.25, v));
      else integ = cadd(integ, rmul(0.5, v));
    }
  return rmul(s->dy * s->dz, integ);
}

/* detector radii and indices (MoL/diagnostic_lib.f90:124-134,
 * main/global_numbers.f90:152-164).  Returns number of detectors found. */
static void build_detectors(kgo *s) {
  int n = s->p.n_det;
  if (n < 2) n = 2;
  s->p.n_det = n;
  s->r_det = xcalloc(n, sizeof(double));
  s->index_det = xcalloc(n, sizeof(int));
  s->r_det[0] = (1.0 + sqrt(1.0 - s->p.a * s->p.a));
  s->r_det[n - 1] = s->p.xmax * 0.99;
  for (int d = 2; d <= n - 1; ++d)
    s->r_det[d - 1] = s->r_det[0] + (s->r_det[n - 1] - s->r_det[0]) / (double)n * (double)(d - 1);
  for (int d = 0; d < n; ++d) {
    s->index_det[d] = 0;
    for (int i = 1; i <= s->Nx - 1; ++i) {
      double ri = s->xmin + (double)(i - 1) * s->dx, ri1 = s->xmin + (double)i * s->dx;
      if (ri <= s->r_det[d] && s->r_det[d] <= ri1) { s->index_det[d] = i; break; }
    }
  }
}

/* currents_detectors, MoL/diagnostic_lib.f90:252-274: momentum(3, n_det) */
void kgo_currents_detectors(const kgo *s, double *momentum) {
  double *J = xcalloc(6 * s->npts, sizeof(double));
  kgo_currents_adm(s, J);
  cplx *Jc = (cplx *)J;
  cplx *g = xcalloc(s->npts, sizeof(cplx));
  cplx *sl = xcalloc((size_t)s->Ny * s->Nz, sizeof(cplx));
  double rfirst = s->xmin, rlast = s->xmin + (double)(s->Nx - 1) * s->dx;
  for (int c = 0; c < 3; ++c) {
    for (int k = s->kL; k <= s->kR; ++k) for (int j = s->jL; j <= s->jR; ++j) for (int i = s->iL; i <= s->iR; ++i) {
      size_t p = P3(s, i, j, k);
      g[p] = cmulr(Jc[c * s->npts + p], s->sqrtg[P2(s, i, j)]);
    }
    for (int d = 0; d < s->p.n_det; ++d) {
      if (rfirst <= s->r_det[d] && rlast > s->r_det[d] && s->index_det[d] > 0) {
        kgo_domain_to_sph_shell(s, g, s->index_det[d], sl);
        momentum[c + 3 * d] = trap2d(s, sl).re;
      }
    }
  }
  free(sl); free(g); free(J);
}

/* proyector_detectors, MoL/diagnostic_lib.f90:231-250: alm(n_det, 0:L, -L:L) */
void kgo_proyector_detectors(const kgo *s, int L, double *alm) {
  size_t ny = s->Ny, nz = s->Nz;
  double *ylm = xcalloc(2 * (size_t)(L + 1) * (2 * L + 1) * ny * nz, sizeof(double));
  kgo_sph_harmonics(s, L, ylm);
  cplx *sl = xcalloc(ny * nz, sizeof(cplx));
  double rfirst = s->xmin, rlast = s->xmin + (double)(s->Nx - 1) * s->dx;
  int NL = L + 1, NM = 2 * L + 1;
  for (int d = 0; d < s->p.n_det; ++d) {
    if (rfirst <= s->r_det[d] && rlast > s->r_det[d] && s->index_det[d] > 0) {
      kgo_domain_to_sph_shell(s, s->u[0], s->index_det[d], sl);
      kgo_project_sh(s, sl, ylm, L, alm + 2 * (size_t)d * NL * NM);
    }
  }
  free(sl); free(ylm);
}

/* project_sh at every vertex shell iv = 1..Nx (tools/FFT_sph.f90:247-279 with
 * domain_to_sph at r = rv(iv), tools/FFT_sph.f90:525-651): alm(l, m, shell). */
void kgo_project_all_shells(const kgo *s, int L, double *alm) {
  size_t ny = s->Ny, nz = s->Nz;
  double *ylm = xcalloc(2 * (size_t)(L + 1) * (2 * L + 1) * ny * nz, sizeof(double));
  kgo_sph_harmonics(s, L, ylm);
  cplx *sl = xcalloc(ny * nz, sizeof(cplx));
  const size_t per = (size_t)(L + 1) * (2 * L + 1);
  for (int iv = 1; iv <= s->Nx; ++iv) {
    kgo_domain_to_sph_shell(s, s->u[0], iv, sl);
    kgo_project_sh(s, sl, ylm, L, alm + 2 * per * (size_t)(iv - 1));
  }
  free(sl); free(ylm);
}

/* project_all_shells restricted to the vertex shells listed in iv[0..n-1]
 * (1-based), for spheres where the full Y_lm table does not fit: the same
 * Y_lm values (sph_harmonics' formulas) and the same trapezium order as
 * kgo_project_sh, so every coefficient equals kgo_project_all_shells' bit for
 * bit; Y_lm is formed per (l, m) on the fly instead of from a stored table.
 * out: n x (2L+1) x (L+1) complex, l fastest.  Threads over (l, m). */
void kgo_project_shells(const kgo *s, int L, int n, const int *iv, double *alm) {
  const int NL = L + 1, NM = 2 * L + 1, Nth = s->Ny, Nph = s->Nz;
  const size_t per = (size_t)NL * NM, sz = (size_t)Nth * Nph;
  const double pi = acos(-1.0);
  cplx *F = (cplx *)alm;
  memset(F, 0, sizeof(cplx) * per * (size_t)n);
  cplx *sl = xcalloc(sz * (size_t)n, sizeof(cplx));
  for (int q = 0; q < n; ++q) kgo_domain_to_sph_shell(s, s->u[0], iv[q], sl + sz * (size_t)q);
  double *st = xcalloc(Nth, sizeof(double));
  for (int j = 1; j <= Nth; ++j) st[j - 1] = sin((double)(j - 1) * s->dy);
  #pragma omp parallel for schedule(dynamic, 1)
  for (int lm = 0; lm < NL * NL; ++lm) {
    const int l = lm / NL, m = lm % NL;
    if (m > l) continue;
    double fact = sqrt((2.0 * l + 1.0) / (4.0 * pi));
    double norm = fact;
    if (m > 0) for (int i = 1; i <= 2 * m; ++i) norm = norm / sqrt((double)(l - m + i));
    cplx *Y = malloc(sizeof(cplx) * sz);
    if (!Y) abort();
    for (int jv = 1; jv <= Nth; ++jv) {
      double x = cos((double)(jv - 1) * s->dy), P;
      if (fabs(x) > 0.9999) P = (m == 0) ? fact : 0.0;
      else P = plm(l, m, x);
      for (int kv = 1; kv <= Nph; ++kv) {
        double ph = (double)(kv - 1) * s->dz;
        cplx phase = {cos(m * ph), sin(m * ph)};
        Y[(jv - 1) + (size_t)Nth * (kv - 1)] = rmul(norm * P, phase);
      }
    }
    for (int sgn = 0; sgn < (m > 0 ? 2 : 1); ++sgn) {
      const int mm = sgn ? -m : m;
      const double sg = (m % 2) ? -1.0 : 1.0;
      for (int q = 0; q < n; ++q) {
        const cplx *f = sl + sz * (size_t)q;
        cplx integ = {0.0, 0.0};
        for (int j = 1; j <= Nth; ++j)
          for (int k = 1; k <= Nph; ++k) {
            cplx a = f[(j - 1) + (size_t)Nth * (k - 1)];
            cplx y = Y[(j - 1) + (size_t)Nth * (k - 1)];
            if (sgn) y = (cplx){sg * y.re, sg * -y.im};
            cplx c = {y.re, -y.im};
            cplx fy = {a.re * c.re - a.im * c.im, a.re * c.im + a.im * c.re};
            cplx fun = {fy.re * st[j - 1], fy.im * st[j - 1]};
            int sel = ((j == 1 || j == Nth) ? 1 : 0) + 2 * ((k == 1 || k == Nph) ? 1 : 0);
            if (sel == 0) integ = cadd(integ, fun);
            else if (sel == 3) integ = cadd(integ, rmul(0.25, fun));
            else integ = cadd(integ, rmul(0.5, fun));
          }
        F[per * (size_t)q + l + NL * (mm + L)] = rmul(s->dy * s->dz, integ);
      }
    }
    free(Y);
  }
  free(st); free(sl);
}

/* spherical Bessel j_l(x) (GSL's gsl_sf_bessel_jl in the reference,
 * tools/FFT_sph.f90:29-34; GSL is not available here): Miller's downward
 * recurrence j_{k-1} = (2k+1)/x j_k - j_{k+1} from an order above both l and
 * x, normalised by the closed forms of j_0 or j_1. */
double kgo_sph_jl(int l, double x) {
  if (x == 0.0) return l == 0 ? 1.0 : 0.0;
  double ax = fabs(x), sg = (x < 0.0 && (l & 1)) ? -1.0 : 1.0;
  double j0 = sin(ax) / ax, j1 = sin(ax) / (ax * ax) - cos(ax) / ax;
  if (l == 0) return j0;
  if (l == 1 && ax > 1.0) return sg * j1; /* closed form cancels for small x */
  double big = (double)l > ax ? (double)l : ax;
  int top = (int)big + 30 + (int)sqrt(40.0 * big);
  double jp = 0.0, jc = 1e-30, keep = 0.0;
  for (int k = top; k >= 1; --k) {
    double jm = (2.0 * k + 1.0) / ax * jc - jp;
    jp = jc; jc = jm;
    if (k - 1 == l) keep = jc;
    if (fabs(jc) > 1e250) { jc *= 1e-250; jp *= 1e-250; keep *= 1e-250; }
  }
  double scale = fabs(j0) >= fabs(j1) ? j0 / jc : j1 / jp;
  return sg * keep * scale;
}

/* n-th positive zero of j_l for l = 0..L, n = 1..Nk (gsl_sf_bessel_zero_Jnu(l+1/2, n),
 * tools/FFT_sph.f90:22-27): zeros of j_0 are n pi, and the zeros of J_nu and
 * J_{nu+1} interlace, so each zero of j_{l+1} is bisected between two
 * consecutive zeros of j_l.  z[l*Nk + n-1]. */
void kgo_sph_jl_zeros(int L, int Nk, double *z) {
  const double pi = acos(-1.0);
  int cnt0 = Nk + L;
  double *prev = xcalloc(cnt0 + 1, sizeof(double)), *cur = xcalloc(cnt0 + 1, sizeof(double));
  for (int n = 1; n <= cnt0; ++n) prev[n - 1] = n * pi;
  for (int n = 0; n < Nk; ++n) z[n] = prev[n];
  for (int l = 1; l <= L; ++l) {
    int cnt = Nk + L - l;
    for (int n = 0; n < cnt; ++n) {
      double lo = prev[n], hi = prev[n + 1], flo = kgo_sph_jl(l, lo);
      for (int it = 0; it < 200; ++it) {
        double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        double fm = kgo_sph_jl(l, mid);
        if (fm == 0.0) { lo = hi = mid; break; }
        if ((fm > 0.0) == (flo > 0.0)) { lo = mid; flo = fm; } else hi = mid;
      }
      cur[n] = 0.5 * (lo + hi);
    }
    for (int n = 0; n < Nk; ++n) z[(size_t)l * Nk + n] = cur[n];
    double *t = prev; prev = cur; cur = t;
  }
  free(prev); free(cur);
}

/* generate_full_bessel_basis (tools/FFT_sph.f90:13-95) on the vertex radii
 * r(i) = xmin + (i-1) dx: k_values(0:L, Nk), j_basis(0:L, Nk, Nx), Fortran
 * order (l fastest); normalised by sqrt(trapezium_1D(j^2 r^2, dr)). */
void kgo_bessel_basis(const kgo *s, int L, int Nk, double *k_values, double *j_basis) {
  const int NL = L + 1, Nx = s->Nx;
  double *z = xcalloc((size_t)NL * Nk, sizeof(double));
  kgo_sph_jl_zeros(L, Nk, z);
  double *r = xcalloc(Nx, sizeof(double)), *jb = xcalloc(Nx, sizeof(double)), *f = xcalloc(Nx, sizeof(double));
  for (int i = 1; i <= Nx; ++i) r[i - 1] = s->xmin + (double)(i - 1) * s->dx;
  double dr = fabs(r[1] - r[0]);
  /* r_max: the outermost point of the evolution grid, x(Nx + g) (MoL/diagnostic_lib.f90:90-92) */
  const double r_max = s->x1d[s->iR - s->iL];
  for (int l = 0; l <= L; ++l)
    for (int n = 1; n <= Nk; ++n) {
      double kv = z[(size_t)l * Nk + n - 1] / r_max;
      k_values[l + (size_t)NL * (n - 1)] = kv;
      for (int i = 0; i < Nx; ++i) jb[i] = kgo_sph_jl(l, kv * r[i]);
      for (int i = 0; i < Nx; ++i) f[i] = (jb[i] * jb[i]) * (r[i] * r[i]);
      double sum = 0.0;
      for (int i = 1; i < Nx - 1; ++i) sum += f[i];
      double nrm = sqrt(dr * (0.5 * f[0] + sum + 0.5 * f[Nx - 1]));
      for (int i = 0; i < Nx; ++i)
        j_basis[l + (size_t)NL * ((n - 1) + (size_t)Nk * i)] = nrm > 0.0 ? jb[i] / nrm : jb[i];
    }
  free(z); free(r); free(jb); free(f);
}

/* SphFT_discrete_radial (tools/FFT_sph.f90:213-244) of phi: ft(1:Nk, 0:L, -L:L),
 * n fastest; flm from project_sh on every vertex shell, then
 * trapezium_1D_complex (tools/integral.f90:197-217) of flm j_basis r^2 over r
 * for n = 1..Nk (the reference's own loop runs n = 0..Nk over a dummy declared
 * with the wrong shape; this is the contraction of the basis as built). */
void kgo_sph_ft_radial(const kgo *s, int L, int Nk, double *ft_out) {
  const int NL = L + 1, NM = 2 * L + 1, Nx = s->Nx;
  double *k = xcalloc((size_t)NL * Nk, sizeof(double));
  double *jb = xcalloc((size_t)NL * Nk * Nx, sizeof(double));
  kgo_bessel_basis(s, L, Nk, k, jb);
  cplx *flm = xcalloc((size_t)NL * NM * Nx, sizeof(cplx));
  kgo_project_all_shells(s, L, (double *)flm);
  cplx *ft = (cplx *)ft_out;
  double dr = fabs((s->xmin + s->dx) - s->xmin);
  memset(ft, 0, sizeof(cplx) * (size_t)Nk * NL * NM);
  for (int l = 0; l <= L; ++l)
    for (int m = -l; m <= l; ++m)
      for (int n = 0; n < Nk; ++n) {
        /* first and last terms with weight 1/2, interior terms in order */
        cplx sum;
        {
          int i0 = 0, i1 = Nx - 1;
          double r0 = s->xmin, r1 = s->xmin + (double)i1 * s->dx;
          double w0 = jb[l + (size_t)NL * (n + (size_t)Nk * i0)] * (r0 * r0);
          double w1 = jb[l + (size_t)NL * (n + (size_t)Nk * i1)] * (r1 * r1);
          cplx f0 = flm[l + (size_t)NL * ((m + L) + (size_t)NM * i0)];
          cplx f1 = flm[l + (size_t)NL * ((m + L) + (size_t)NM * i1)];
          cplx t0 = {w0 * f0.re, w0 * f0.im}, t1 = {w1 * f1.re, w1 * f1.im};
          sum = rmul(0.5, cadd(t0, t1));
        }
        for (int i = 1; i < Nx - 1; ++i) {
          double r = s->xmin + (double)i * s->dx;
          double w = jb[l + (size_t)NL * (n + (size_t)Nk * i)] * (r * r);
          cplx f = flm[l + (size_t)NL * ((m + L) + (size_t)NM * i)];
          cplx t = {w * f.re, w * f.im};
          sum = cadd(sum, t);
        }
        ft[n + (size_t)Nk * (l + (size_t)NL * (m + L))] = rmul(dr, sum);
      }
  free(k); free(jb); free(flm);
}

/* ------------------------------------------------------------------ */
/* construction and state access                                       */

kgo *kgo_create(const kgo_params *p) {
  if (p->Nx < 4 || p->Ny < 5 || p->Nz < 5 || p->g_pts != 2) return NULL;
  kgo *s = xcalloc(1, sizeof(kgo));
  s->p = *p;
  s->Nx = p->Nx; s->Ny = p->Ny; s->Nz = p->Nz; s->g = p->g_pts;
  s->iL = -s->g; s->iR = s->Nx + s->g;
  s->jL = -s->g; s->jR = s->Ny + s->g;
  s->kL = 0; s->kR = s->Nz;
  s->NI = s->iR - s->iL + 1; s->NJ = s->jR - s->jL + 1; s->NK = s->kR - s->kL + 1;
  s->npts = (size_t)s->NI * s->NJ * s->NK;
  build_grid(s);
  build_metric(s);
  for (int v = 0; v < 5; ++v) {
    s->u[v] = xcalloc(s->npts, sizeof(cplx)); s->u_p[v] = xcalloc(s->npts, sizeof(cplx));
    s->u_stage[v] = xcalloc(s->npts, sizeof(cplx)); s->u_stage_2[v] = xcalloc(s->npts, sizeof(cplx));
    s->k1[v] = xcalloc(s->npts, sizeof(cplx)); s->k2[v] = xcalloc(s->npts, sizeof(cplx));
    s->k3[v] = xcalloc(s->npts, sizeof(cplx)); s->k4[v] = xcalloc(s->npts, sizeof(cplx));
    s->rhs_u[v] = xcalloc(s->npts, sizeof(cplx));
  }
  for (int t = 0; t < 6; ++t) s->tmp[t] = xcalloc(s->npts, sizeof(cplx));
  build_detectors(s);
  return s;
}

void kgo_destroy(kgo *s) {
  if (!s) return;
  for (int v = 0; v < 5; ++v) {
    free(s->u[v]); free(s->u_p[v]); free(s->u_stage[v]); free(s->u_stage_2[v]);
    free(s->k1[v]); free(s->k2[v]); free(s->k3[v]); free(s->k4[v]); free(s->rhs_u[v]);
  }
  for (int t = 0; t < 6; ++t) free(s->tmp[t]);
  for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) { free(s->g_dn[a][b]); free(s->g_up[a][b]); }
  free(s->alpha); free(s->sqrtg); free(s->dx_beta); free(s->dx_beta4);
  for (int a = 0; a < 3; ++a) { free(s->beta[a]); for (int b = 0; b < 3; ++b) free(s->gamma_up[a][b]); }
  free(s->x1d); free(s->y1d); free(s->r_det); free(s->index_det);
  free(s);
}

/* Fortran-order state u(5, NI, NJ, NK) complex <-> internal arrays */
static void unpack(kgo *s, cplx **dst, const double *src) {
  const cplx *S = (const cplx *)src;
  for (size_t p = 0; p < s->npts; ++p) for (int v = 0; v < 5; ++v) dst[v][p] = S[5 * p + v];
}
static void pack(const kgo *s, cplx *const *src, double *dst) {
  cplx *D = (cplx *)dst;
  for (size_t p = 0; p < s->npts; ++p) for (int v = 0; v < 5; ++v) D[5 * p + v] = src[v][p];
}
void kgo_set_state(kgo *s, const double *u) { unpack(s, s->u, u); }
void kgo_get_state(const kgo *s, double *u) { pack(s, s->u, u); }
void kgo_set_stage(kgo *s, const double *u) { unpack(s, s->u_stage, u); }
void kgo_get_stage(const kgo *s, double *u) { pack(s, s->u_stage, u); }
void kgo_set_stage2(kgo *s, const double *u) { unpack(s, s->u_stage_2, u); }
void kgo_get_stage2(const kgo *s, double *u) { pack(s, s->u_stage_2, u); }

/* rhs of the selected variables (bit v of mask) for an arbitrary state
 * vars (Fortran order); unselected outputs are left untouched. */
void kgo_rhs(kgo *s, const double *vars, double *rhs_out, unsigned mask) {
  cplx *V[5];
  for (int v = 0; v < 5; ++v) V[v] = xcalloc(s->npts, sizeof(cplx));
  unpack(s, V, vars);
  cplx *R[5];
  for (int v = 0; v < 5; ++v) R[v] = xcalloc(s->npts, sizeof(cplx));
  unpack(s, R, rhs_out);
  if (mask & 1u) kgo_rhs_phi(s, R[0], V);
  if (mask & 2u) kgo_rhs_psi1(s, R[1], V);
  if (mask & 4u) kgo_rhs_psi2(s, R[2], V);
  if (mask & 8u) kgo_rhs_psi3(s, R[3], V);
  if (mask & 16u) kgo_rhs_pi(s, R[4], V);
  pack(s, R, rhs_out);
  for (int v = 0; v < 5; ++v) { free(V[v]); free(R[v]); }
}

/* the individual face fills on u; bit order xL,xR,yL,yR,zL,zR */
void kgo_boundary_faces(kgo *s, unsigned mask) {
  if (mask & 1u) kgo_boundary_xL(s);
  if (mask & 2u) kgo_boundary_xR(s);
  if (mask & 4u) kgo_boundary_yL(s);
  if (mask & 8u) kgo_boundary_yR(s);
  if (mask & 16u) kgo_boundary_zL(s);
  if (mask & 32u) kgo_boundary_zR(s);
}
void kgo_set_u_p(kgo *s, const double *u) { unpack(s, s->u_p, u); }

/* scalars: dx, dy, dz, dt, t, xmin, xmax, Nt */
void kgo_get_scalars(const kgo *s, double *out) {
  out[0] = s->dx; out[1] = s->dy; out[2] = s->dz; out[3] = s->dt; out[4] = s->t;
  out[5] = s->xmin; out[6] = s->xmax; out[7] = (double)s->Nt;
}
void kgo_set_time(kgo *s, double t) { s->t = t; }
void kgo_set_dt(kgo *s, double dt) { s->dt = dt; }

/* metric tables, 2-D (NI x NJ) each, in the order
 * alpha, beta_r, dx_beta, sqrtg, gamma_rr, gamma_rphi, gamma_thth, gamma_phph */
void kgo_get_metric(const kgo *s, double *out) {
  size_t n2 = (size_t)s->NI * s->NJ;
  memcpy(out + 0 * n2, s->alpha, n2 * sizeof(double));
  memcpy(out + 1 * n2, s->beta[0], n2 * sizeof(double));
  memcpy(out + 2 * n2, s->dx_beta, n2 * sizeof(double));
  memcpy(out + 3 * n2, s->sqrtg, n2 * sizeof(double));
  memcpy(out + 4 * n2, s->gamma_up[0][0], n2 * sizeof(double));
  memcpy(out + 5 * n2, s->gamma_up[0][2], n2 * sizeof(double));
  memcpy(out + 6 * n2, s->gamma_up[1][1], n2 * sizeof(double));
  memcpy(out + 7 * n2, s->gamma_up[2][2], n2 * sizeof(double));
}
/* g_dn and g_up, 16 tables each (mu-major) */
void kgo_get_4metric(const kgo *s, double *gdn, double *gup) {
  size_t n2 = (size_t)s->NI * s->NJ;
  for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) {
    memcpy(gdn + (a * 4 + b) * n2, s->g_dn[a][b], n2 * sizeof(double));
    memcpy(gup + (a * 4 + b) * n2, s->g_up[a][b], n2 * sizeof(double));
  }
}
void kgo_get_detectors(const kgo *s, double *r_det, int *index_det) {
  for (int d = 0; d < s->p.n_det; ++d) { r_det[d] = s->r_det[d]; index_det[d] = s->index_det[d]; }
}
void kgo_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}
int kgo_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
size_t kgo_npts(const kgo *s) { return s->npts; }
