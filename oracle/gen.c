/*
 * gen.c -- CPU FP64 restatement of the real-space Green kernel build of
 * GilaElectromagnetics.jl (src/glaGen.jl, src/glaInt.jl, src/glaIntSup.jl).
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the GPU kernel build is checked
 * against (oracle/__init__.py).  It is never linked into libgila_b200.
 *
 * Third-party algorithms the reference calls and that are not in its tree:
 *  - Cubature.jl 1.5.1 / Cubature_jll 1.0.5 `hcubature` (src/glaGen.jl:574):
 *    restated from the published method -- the Genz-Malik degree-7 rule with
 *    embedded degree-5 error estimate on a hyper-rectangle (Genz & Malik,
 *    J. Comput. Appl. Math. 6 (1980) 295-302), global adaptive bisection of
 *    the region with the largest error along the axis of largest fourth
 *    difference, and the per-component ("INDIVIDUAL") stopping rule
 *    err_j <= max(abstol, reltol*|val_j|) on the running sums.
 *  - FastGaussQuadrature 1.0.2 `gausslegendre` (src/glaGen.jl:683-687):
 *    Legendre nodes by Newton iteration on P_n, weights 2/((1-x^2) P_n'(x)^2).
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;
static const double PI = 3.14159265358979323846264338327950288;
static const double S3 = 1.7320508075688772935274463415058723669;  /* sqrt(3) */

/* ------------------------------------------------------------------ rationals */
typedef struct { int64_t n, d; } rat;
static int64_t gcd64(int64_t a, int64_t b) {
  if (a < 0) a = -a;
  if (b < 0) b = -b;
  while (b) { int64_t t = a % b; a = b; b = t; }
  return a;
}
static rat mkr(int64_t n, int64_t d) {
  if (d < 0) { n = -n; d = -d; }
  int64_t g = gcd64(n, d);
  if (g == 0) g = 1;
  rat r = {n / g, d / g};
  return r;
}
static rat radd(rat a, rat b) { return mkr(a.n * b.d + b.n * a.d, a.d * b.d); }
static rat rsub(rat a, rat b) { return mkr(a.n * b.d - b.n * a.d, a.d * b.d); }
static rat rmul(rat a, rat b) { return mkr(a.n * b.n, a.d * b.d); }
static rat rdiv(rat a, rat b) { return mkr(a.n * b.d, a.d * b.n); }
static rat rint_(int64_t k) { rat r = {k, 1}; return r; }
static double rdbl(rat a) { return (double)a.n / (double)a.d; }
static int rlt(rat a, rat b) { return (__int128)a.n * b.d < (__int128)b.n * a.d; }
static int rle(rat a, rat b) { return (__int128)a.n * b.d <= (__int128)b.n * a.d; }

/* GlaVol (src/glaMem.jl:12-19,136-148): grid centres start + k*grd */
typedef struct {
  int64_t cel[3];
  rat scl[3], org[3], grd[3];
  rat start[3], stop[3];
} vol;

static vol mkvol(const int64_t cel[3], const int64_t scl_n[3], const int64_t scl_d[3], const int64_t org_n[3],
                 const int64_t org_d[3], const int64_t grd_n[3], const int64_t grd_d[3]) {
  vol v;
  for (int k = 0; k < 3; ++k) {
    v.cel[k] = cel[k];
    v.scl[k] = mkr(scl_n[k], scl_d[k]);
    v.org[k] = mkr(org_n[k], org_d[k]);
    v.grd[k] = (grd_d && grd_d[k]) ? mkr(grd_n[k], grd_d[k]) : v.scl[k];
    /* brd = grd*(floor(cel/2) - iseven(cel)/2) */
    rat half = mkr((cel[k] / 2) * 2 - ((cel[k] % 2 == 0) ? 1 : 0), 2);
    rat brd = rmul(v.grd[k], half);
    v.start[k] = rsub(v.org[k], brd);
    v.stop[k] = radd(v.org[k], brd);
  }
  return v;
}

/* ----------------------------------------------------------- scalar kernels */
/* sclEgo (src/glaInt.jl:41-44): exp(2 pi i d f) / (4 pi d f^2) */
static inline cplx scl_ego(double d, cplx f) {
  cplx z = (2.0 * PI) * d * f;
  return cexp(I * z) / ((4.0 * PI) * d * (f * f));
}
/* sclEgoN (src/glaInt.jl:51-59): singularity removed */
static inline cplx scl_ego_n(double d, cplx f) {
  if (d > 1e-7) {
    cplx z = (2.0 * PI) * d * f;
    return (cexp(I * z) - 1.0) / ((4.0 * PI) * d * (f * f));
  }
  return ((I / f) - PI * d) / 2.0;
}
static inline double dst_mag(double a, double b, double c) { return sqrt(a * a + b * b + c * c); }

/* ------------------------------------------------------------ Gauss-Legendre */
/* nodes ascending on [-1,1] (gauQud, src/glaGen.jl:683-687) */
int gila_ref_gauleg(int n, double* x, double* w) {
  for (int i = 0; i < n; ++i) {
    /* i-th root counted from +1 downward; stored ascending */
    double z = cos(PI * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int k = 1; k <= n; ++k) {
        double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p2) / k;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      double dz = p0 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) {
        /* one more polish step */
        p0 = 1.0; p1 = 0.0;
        for (int k = 1; k <= n; ++k) {
          double p2 = p1;
          p1 = p0;
          p0 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p2) / k;
        }
        dp = n * (z * p0 - p1) / (z * z - 1.0);
        break;
      }
    }
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
  return 0;
}

/* ------------------------------------------------- DIRECTFN weak integrals */
/* src/glaIntSup.jl: triangle-pair integrals of the scalar kernel, reduced to
 * nested 1-D Gauss-Legendre sums.  rPts columns are stored r[col][dim]. */
typedef struct {
  int n;
  const double* x;
  const double* w;
  cplx f;
} quad;

static inline double thf(double a, double b, double p) { return 0.5 * ((b - a) * p + a + b); }

static inline void spx(double xp[3][2], double e1, double e2, double x1, double x2) {
  xp[0][0] = (S3 * (1.0 - e1) - x1) / (2.0 * S3);
  xp[1][0] = (S3 * (1.0 + e1) - x1) / (2.0 * S3);
  xp[2][0] = x1 / S3;
  xp[0][1] = (S3 * (1.0 - e2) - x2) / (2.0 * S3);
  xp[1][1] = (S3 * (1.0 + e2) - x2) / (2.0 * S3);
  xp[2][1] = x2 / S3;
}

/* kerEV / kerEVN (src/glaIntSup.jl:427-455): points on triangles (r0,r1,r2), (r3,r4,r5) */
static inline double ker_dist6(const double r[6][3], const double xp[3][2]) {
  double v[3];
  for (int d = 0; d < 3; ++d)
    v[d] = xp[0][0] * r[0][d] + xp[1][0] * r[1][d] + xp[2][0] * r[2][d] -
           (xp[0][1] * r[3][d] + xp[1][1] * r[4][d] + xp[2][1] * r[5][d]);
  return dst_mag(v[0], v[1], v[2]);
}
/* kerSN (src/glaIntSup.jl:457-469): both points on the same triangle */
static inline double ker_dist3(const double r[6][3], const double xp[3][2]) {
  double v[3];
  for (int d = 0; d < 3; ++d)
    v[d] = xp[0][0] * r[0][d] + xp[1][0] * r[1][d] + xp[2][0] * r[2][d] -
           (xp[0][1] * r[0][d] + xp[1][1] * r[1][d] + xp[2][1] * r[2][d]);
  return dst_mag(v[0], v[1], v[2]);
}

static double cross_norm(const double a[3], const double b[3], const double c[3]) {
  double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
  return sqrt(x * x + y * y + z * z);
}
/* eqvJacEV / eqvJacS (src/glaIntSup.jl:381-395) */
static double jac_ev(const double r[6][3]) { return cross_norm(r[0], r[1], r[2]) * cross_norm(r[3], r[4], r[5]) / 12.0; }
static double jac_s(const double r[6][3]) {
  double u[3] = {r[0][0] - r[1][0], r[0][1] - r[1][1], r[0][2] - r[1][2]};
  double v[3] = {r[2][0] - r[0][0], r[2][1] - r[0][1], r[2][2] - r[0][2]};
  double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
  return (x * x + y * y + z * z) / 12.0;
}

/* subTri (src/glaIntSup.jl:365-379) */
static inline void sub_tri(double l1, double l2, int dir, double* e, double* x) {
  if (dir == 1) { *e = l1; *x = l2; }
  else if (dir == 2) { *e = 0.5 * (1.0 - l1 - l2 * S3); *x = 0.5 * (S3 + l1 * S3 - l2); }
  else { *e = 0.5 * (-1.0 - l1 + l2 * S3); *x = 0.5 * (S3 - l1 * S3 - l2); }
}

/* aS (src/glaIntSup.jl:313-332) */
static cplx a_s(const double r[6][3], double th1, double thB, double th, int dir, const quad* q) {
  double xp[3][2];
  cplx acc = 0;
  double s1 = sin(th1), c1 = cos(th1);
  for (int n = 0; n < q->n; ++n) {
    double e1, x1, e2, x2;
    sub_tri(thB, th * s1, dir, &e1, &x1);
    double t = thf(0.0, th, q->x[n]);
    sub_tri(t * c1 + thB, (th - t) * s1, dir, &e2, &x2);
    spx(xp, e1, e2, x1, x2);
    acc += q->w[n] * t * scl_ego_n(ker_dist3(r, xp), q->f);
  }
  return 0.5 * th * acc;
}

/* nS (src/glaIntSup.jl:201-237) */
static cplx n_s(int dir, int idf, double th1, double thB, const double r[6][3], const quad* q) {
  cplx acc = 0;
  if (idf == 1 || idf == 5) {
    double L = (1.0 - thB) / cos(th1);
    for (int n = 0; n < q->n; ++n) acc += q->w[n] * a_s(r, th1, thB, thf(0.0, L, q->x[n]), dir, q);
    return (1.0 - thB) / (2.0 * cos(th1)) * acc;
  } else if (idf == 2 || idf == 3) {
    double L = S3 * (1.0 - thB) / sin(th1);
    for (int n = 0; n < q->n; ++n) acc += q->w[n] * a_s(r, th1, thB, thf(0.0, L, q->x[n]), dir, q);
    return S3 * (1.0 - thB) / (2.0 * sin(th1)) * acc;
  } else if (idf == 6 || idf == 7) {
    double L = S3 * (1.0 + thB) / sin(th1);
    for (int n = 0; n < q->n; ++n) acc += q->w[n] * a_s(r, th1, thB, thf(0.0, L, q->x[n]), dir, q);
    return S3 * (1.0 + thB) / (2.0 * sin(th1)) * acc;
  } else {
    double L = -(1.0 + thB) / cos(th1);
    for (int n = 0; n < q->n; ++n) acc += q->w[n] * a_s(r, th1, thB, thf(0.0, L, q->x[n]), dir, q);
    return -(1.0 + thB) / (2.0 * cos(th1)) * acc;
  }
}

static void psi_lim_s(int idf, double* a, double* b) {
  if (idf == 1 || idf == 5 || idf == 6) { *a = 0.0; *b = PI / 3.0; }
  else if (idf == 2 || idf == 7) { *a = PI / 3.0; *b = 2.0 * PI / 3.0; }
  else { *a = 2.0 * PI / 3.0; *b = PI; }
}
static void eta_lim_s(int idf, double th, double* a, double* b) {
  if (idf == 1 || idf == 2) { *a = 0.0; *b = 1.0; }
  else if (idf == 3) { *a = (S3 - tan(PI - th)) / (S3 + tan(PI - th)); *b = 1.0; }
  else if (idf == 4) { *a = 0.0; *b = (S3 - tan(PI - th)) / (S3 + tan(PI - th)); }
  else if (idf == 5) { *a = (tan(th) - S3) / (S3 + tan(th)); *b = 0.0; }
  else if (idf == 6) { *a = -1.0; *b = (tan(th) - S3) / (S3 + tan(th)); }
  else { *a = -1.0; *b = 0.0; }
}

/* wekSInt (src/glaIntSup.jl:13-41): sum over (dir 1:3, idf 1:8, k 1:ord) */
static cplx wek_s_int(const double r[6][3], const quad* q) {
  const int n = q->n;
  cplx* part = (cplx*)calloc((size_t)n, sizeof(cplx));
#pragma omp parallel for schedule(dynamic)
  for (int k = 0; k < n; ++k) {
    cplx acc = 0;
    for (int idf = 1; idf <= 8; ++idf)
      for (int dir = 1; dir <= 3; ++dir) {
        double pa, pb, ea, eb;
        psi_lim_s(idf, &pa, &pb);
        double th = thf(pa, pb, q->x[k]);
        eta_lim_s(idf, th, &ea, &eb);
        cplx iv = 0;
        for (int it = 0; it < n; ++it) iv += q->w[it] * n_s(dir, idf, th, thf(ea, eb, q->x[it]), r, q);
        acc += 0.25 * iv * q->w[k] * (pb - pa) * (eb - ea) * sin(th);
      }
    part[k] = acc;
  }
  cplx s = 0;
  for (int k = 0; k < n; ++k) s += part[k];
  free(part);
  return jac_s(r) * s;
}

/* spxE! (src/glaIntSup.jl:395-411) */
static inline void spx_e(double xp[3][2], double lam, double eta, double thB, double th1, int idf) {
  double sB = sin(thB), cB = cos(thB), s1 = sin(th1), c1 = cos(th1);
  if (idf == 1) spx(xp, eta, lam * cB * c1 - eta, lam * sB, lam * cB * s1);
  else spx(xp, -eta, -(lam * cB * c1 - eta), lam * sB, lam * cB * s1);
}
/* aE (src/glaIntSup.jl:334-348) */
static cplx a_e(const double r[6][3], double lam, double eta, double thB, double th1, int idf, const quad* q) {
  double xp[3][2];
  cplx acc = 0;
  for (int n = 0; n < q->n; ++n) {
    double z = thf(0.0, lam, q->x[n]);
    spx_e(xp, z, eta, thB, th1, idf);
    acc += q->w[n] * z * z * scl_ego_n(ker_dist6(r, xp), q->f);
  }
  return 0.5 * lam * acc;
}
/* intNE (src/glaIntSup.jl:283-311) */
static cplx int_ne(int n, int idf1, double gam, double thB, double th1, const double r[6][3], int idf2, const quad* q) {
  double eta, lam;
  double s1 = sin(th1), c1 = cos(th1);
  if (idf1 == 1) {
    eta = thf(0.0, gam, q->x[n]);
    lam = S3 * (1 + eta) / (cos(thB) * (s1 + S3 * c1));
  } else if (idf1 == 2) {
    eta = thf(gam, 1.0, q->x[n]);
    lam = S3 * (1.0 - fabs(eta)) / sin(thB);
  } else if (idf1 == 3) {
    eta = thf(gam, 1.0, q->x[n]);
    lam = S3 * (1.0 - fabs(eta)) / (cos(thB) * (s1 - S3 * c1));
  } else if (idf1 == 4) {
    eta = thf(0.0, 1.0, q->x[n]);
    lam = S3 * (1.0 - fabs(eta)) / (cos(thB) * (s1 - S3 * c1));
  } else {
    eta = thf(0.0, 1.0, q->x[n]);
    lam = S3 * (1.0 - eta) / sin(thB);
  }
  return a_e(r, lam, eta, thB, th1, idf2, q);
}
/* nE (src/glaIntSup.jl:239-281); note the argument order (thB, th1) */
static cplx n_e(int idf1, int idf2, double thB, double th1, const double r[6][3], const quad* q) {
  cplx v1 = 0, v2 = 0;
  if (idf1 == 1 || idf1 == 2) {
    double s1 = sin(th1), c1 = cos(th1);
    double gam = (s1 + S3 * c1 - tan(thB)) / (s1 + S3 * c1 + tan(thB));
    for (int n = 0; n < q->n; ++n) {
      v1 += q->w[n] * int_ne(n, 1, gam, thB, th1, r, idf2, q);
      v2 += q->w[n] * int_ne(n, 2, gam, thB, th1, r, idf2, q);
    }
    return 0.5 * v2 + gam * 0.5 * (v1 - v2);
  } else if (idf1 == 3) {
    double gam = S3 / tan(th1);
    for (int n = 0; n < q->n; ++n) {
      v1 += q->w[n] * int_ne(n, 1, gam, thB, th1, r, idf2, q);
      v2 += q->w[n] * int_ne(n, 3, gam, thB, th1, r, idf2, q);
    }
    return 0.5 * v2 + 0.5 * gam * (v1 - v2);
  } else if (idf1 == 4) {
    for (int n = 0; n < q->n; ++n) v1 += q->w[n] * int_ne(n, 4, 1.0, thB, th1, r, idf2, q);
    return 0.5 * v1;
  } else {
    for (int n = 0; n < q->n; ++n) v1 += q->w[n] * int_ne(n, 5, 1.0, thB, th1, r, idf2, q);
    return 0.5 * v1;
  }
}
static void psi_lim_e(int idf, double* a, double* b) {
  if (idf == 1) { *a = 0.0; *b = PI / 3.0; }
  else if (idf == 2 || idf == 3) { *a = PI / 3.0; *b = PI / 2.0; }
  else if (idf == 4 || idf == 6) { *a = PI / 2.0; *b = PI; }
  else { *a = 0.0; *b = PI / 2.0; }
}
static void eta_lim_e(int idf, double th, double* a, double* b) {
  double s = sin(th), c = cos(th);
  if (idf == 1) { *a = 0.0; *b = atan(s + S3 * c); }
  else if (idf == 2) { *a = atan(s - S3 * c); *b = atan(s + S3 * c); }
  else if (idf == 3 || idf == 4) { *a = 0.0; *b = atan(s - S3 * c); }
  else if (idf == 5) { *a = atan(s + S3 * c); *b = 0.5 * PI; }
  else { *a = atan(s - S3 * c); *b = 0.5 * PI; }
}
/* wekEInt (src/glaIntSup.jl:43-74): sum over (idf 1:6, k 1:ord) */
static cplx wek_e_int(const double r[6][3], const quad* q) {
  const int n = q->n;
  cplx* part = (cplx*)calloc((size_t)(6 * n), sizeof(cplx));
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int k = 0; k < n; ++k)
    for (int idf = 1; idf <= 6; ++idf) {
      double pa, pb, ea, eb;
      psi_lim_e(idf, &pa, &pb);
      double thB = thf(pa, pb, q->x[k]);
      eta_lim_e(idf, thB, &ea, &eb);
      cplx iv = 0;
      for (int it = 0; it < n; ++it) {
        double thA = thf(ea, eb, q->x[it]);
        iv += q->w[it] * cos(thA) * (n_e(idf, 1, thA, thB, r, q) + n_e(idf, -1, thA, thB, r, q));
      }
      part[k * 6 + idf - 1] = 0.25 * iv * q->w[k] * (pb - pa) * (eb - ea);
    }
  cplx s = 0;
  for (int k = 0; k < 6 * n; ++k) s += part[k];
  free(part);
  return jac_ev(r) * s;
}

/* spxV! (src/glaIntSup.jl:384-393) */
static inline void spx_v(double xp[3][2], double t4, double t3, double tB, double t1) {
  double sB = sin(tB), cB = cos(tB), s1 = sin(t1), c1 = cos(t1), s3 = sin(t3), c3 = cos(t3);
  spx(xp, t4 * c3 * c1 - 1.0, t4 * s3 * cB - 1.0, t4 * c3 * s1, t4 * s3 * sB);
}
/* wekVInt (src/glaIntSup.jl:76-140): sum over (i1, i2, i3) in ord^3 */
static cplx wek_v_int(int sng, const double r[6][3], const quad* q) {
  const int n = q->n;
  cplx* part = (cplx*)calloc((size_t)(n * n), sizeof(cplx));
#pragma omp parallel for schedule(dynamic) collapse(2)
  for (int i3 = 0; i3 < n; ++i3)
    for (int i2 = 0; i2 < n; ++i2) {
      cplx acc = 0;
      for (int i1 = 0; i1 < n; ++i1) {
        double xp[3][2];
        double tA = thf(0.0, PI / 3.0, q->x[i1]);
        double LA = 2.0 * S3 / (sin(tA) + S3 * cos(tA));
        double tB = thf(0.0, PI / 3.0, q->x[i2]);
        double LB = 2.0 * S3 / (sin(tB) + S3 * cos(tB));
        double at = atan(LB / LA);
        double tC = thf(0.0, at, q->x[i3]);
        double sC = sin(tC), cC = cos(tC);
        double tD = thf(at, PI / 2.0, q->x[i3]);
        double sD = sin(tD), cD = cos(tD);
        cplx vc = 0, vd = 0;
        for (int a = 0; a < n; ++a) {
          double tx = thf(0.0, LA / cC, q->x[a]);
          spx_v(xp, tx, tC, tB, tA);
          double d = ker_dist6(r, xp);
          vc += q->w[a] * (tx * tx * tx) * (sng ? scl_ego_n(d, q->f) : scl_ego(d, q->f));
        }
        for (int a = 0; a < n; ++a) {
          double tx = thf(0.0, LB / sD, q->x[a]);
          spx_v(xp, tx, tD, tB, tA);
          double d = ker_dist6(r, xp);
          vd += q->w[a] * (tx * tx * tx) * (sng ? scl_ego_n(d, q->f) : scl_ego(d, q->f));
        }
        acc += q->w[i1] * q->w[i2] * q->w[i3] * (at * (LA * sC * vc - LB * cD * vd) + 0.5 * PI * LB * cD * vd);
      }
      part[i3 * n + i2] = acc;
    }
  cplx s = 0;
  for (int k = 0; k < n * n; ++k) s += part[k];
  free(part);
  return jac_ev(r) * PI * PI * s / 144.0;
}

/* wekGrdPts! (src/glaInt.jl:354-389): 18 lattice points, 1-based P1..P18 */
static void grd_pts(int dir, const double scl[3], double P[19][3]) {
  double gx, gy, gz;
  if (dir == 1) { gx = scl[0]; gy = scl[1]; gz = scl[2]; }
  else if (dir == 2) { gx = scl[2]; gy = scl[0]; gz = scl[1]; }
  else { gx = scl[1]; gy = scl[2]; gz = scl[0]; }
  int k = 1;
  for (int zz = 0; zz < 2; ++zz)
    for (int yy = 0; yy < 3; ++yy)
      for (int xx = 0; xx < 3; ++xx, ++k) {
        P[k][0] = xx * gx;
        P[k][1] = yy * gy;
        P[k][2] = zz * gz;
      }
}
static void tri6(double r[6][3], double P[19][3], int a, int b, int c, int d, int e, int f) {
  int id[6] = {a, b, c, d, e, f};
  for (int k = 0; k < 6; ++k) memcpy(r[k], P[id[k]], sizeof(double) * 3);
}
#define WS(a, b, c) (tri6(r, P, a, b, c, a, b, c), wek_s_int(r, q))
#define WE(a, b, c, d, e, f) (tri6(r, P, a, b, c, d, e, f), wek_e_int(r, q))
#define WV(s, a, b, c, d, e, f) (tri6(r, P, a, b, c, d, e, f), wek_v_int(s, r, q))

/* wekSDir (src/glaInt.jl:88-114) */
static cplx wek_s_dir(int dir, const double scl[3], const quad* q) {
  double P[19][3], r[6][3];
  grd_pts(dir, scl, P);
  cplx a = WS(1, 2, 5);
  a += WS(1, 5, 4);
  a += WE(1, 2, 5, 1, 5, 4);
  a += WE(1, 5, 4, 1, 2, 5);
  cplx b = WS(4, 1, 2);
  b += WS(4, 2, 5);
  b += WE(4, 1, 2, 4, 2, 5);
  b += WE(4, 2, 5, 4, 1, 2);
  return (a + b) / 2.0;
}
/* wekEDir (src/glaInt.jl:165-206) */
static void wek_e_dir(int dir, const double scl[3], const quad* q, cplx v[4]) {
  double P[19][3], r[6][3];
  grd_pts(dir, scl, P);
  v[0] = WE(1, 2, 5, 2, 3, 5);
  v[0] += WV(1, 1, 2, 5, 3, 6, 5);
  v[0] += WV(1, 1, 5, 4, 2, 3, 5);
  v[0] += WV(1, 1, 5, 4, 3, 6, 5);
  v[1] = WE(1, 2, 5, 2, 11, 5);
  v[1] += WV(1, 1, 2, 5, 11, 14, 5);
  v[1] += WV(1, 1, 5, 4, 2, 11, 5);
  v[1] += WV(1, 1, 5, 4, 11, 14, 5);
  v[2] = WV(1, 1, 2, 5, 4, 5, 7);
  v[2] += WV(1, 1, 2, 5, 5, 8, 7);
  v[2] += WE(1, 5, 4, 4, 5, 7);
  v[2] += WV(1, 1, 5, 4, 5, 8, 7);
  v[3] = WV(1, 1, 2, 5, 4, 5, 13);
  v[3] += WV(1, 1, 2, 5, 5, 14, 13);
  v[3] += WE(1, 5, 4, 4, 5, 13);
  v[3] += WV(1, 1, 5, 4, 5, 14, 13);
}
/* wekVDir (src/glaInt.jl:236-262) */
static void wek_v_dir(int dir, const double scl[3], const quad* q, cplx v[3]) {
  double P[19][3], r[6][3];
  grd_pts(dir, scl, P);
  v[0] = WV(0, 1, 2, 5, 5, 6, 9);
  v[0] += WV(0, 1, 2, 5, 5, 9, 8);
  v[0] += WV(0, 1, 5, 4, 5, 6, 9);
  v[0] += WV(0, 1, 5, 4, 5, 9, 8);
  v[1] = WV(0, 1, 2, 5, 5, 17, 14);
  v[1] += WV(0, 1, 2, 5, 5, 8, 17);
  v[1] += WV(0, 1, 5, 4, 5, 17, 14);
  v[1] += WV(0, 1, 5, 4, 5, 8, 17);
  v[2] = WV(0, 1, 2, 5, 5, 15, 14);
  v[2] += WV(0, 1, 2, 5, 5, 6, 15);
  v[2] += WV(0, 1, 5, 4, 5, 15, 14);
  v[2] += WV(0, 1, 5, 4, 5, 6, 15);
}

/* ---------------------------------------------- closed-form static parts */
/* rSrfSlf (src/glaInt.jl:410-432) */
static cplx r_srf_slf(double la, double lb, cplx f) {
  double s1 = sqrt(la * la + lb * lb), s4 = sqrt(la * la + 4 * lb * lb);
  double t = 8 * la * la * la + 8 * lb * lb * lb - 8 * la * la * s1 - 8 * lb * lb * s1 -
             3 * la * la * lb *
                 (2 * log(la) + 2 * log(la + lb - s1) + log(s1 - lb) - 5 * log(lb + s1) - 2 * log(lb - la + s1) -
                  2 * log(la + 2 * lb - s4) + log(s4 - 2 * lb) + 2 * log(la - 2 * lb + s4) + log(2 * lb + s4) +
                  2 * log(2 * lb - la + s4) - 2 * log(la + 2 * lb + s4)) +
             6 * la * lb * lb *
                 (log(64.0) + 4 * log(lb) + 2 * log(s1 - la) + 3 * log(la + s1) - 3 * log(s4 - la) -
                  3 * log(sqrt(la * la * la * la + 5 * la * la * lb * lb + 4 * lb * lb * lb * lb) +
                          la * (s1 - la - s4)));
  return (1.0 / ((48.0 * PI) * (f * f))) * t;
}
/* rSrfEdgCrn (src/glaInt.jl:434-462) */
static cplx r_srf_edg_crn(double la, double lb, double lc, cplx f) {
  double sab = sqrt(la * la + lb * lb + lc * lc), sbc = sqrt(lb * lb + lc * lc);
  double t = 8 * lb * lc * sbc - 8 * lb * lc * sab -
             12 * la * la * la * atan(1.0 / (la * lc / (la * la + lb * lb - lb * sab))) + 12 * la * la * la * atan(la / lc) -
             12 * la * lc * lc * atan(la * lb / (lc * sab)) - 12 * la * lb * lb * atan(la * lc / (lb * sab)) -
             16 * la * la * la * atan(lb * lc / (la * sab)) + 6 * lc * lc * lc * atanh(lb / sbc) -
             6 * lc * (la * la + lc * lc) * atanh(lb / sab) - 15 * la * la * lc * log(la * la + lc * lc) -
             lc * lc * lc * log(la * la + lc * lc) + 2 * lc * lc * lc * log(lc / (lb + sbc)) +
             6 * la * la * lc * log(sab - lb) + 24 * la * la * lc * log(sab + lb) + 2 * lc * lc * lc * log(sab + lb) +
             6 * la * lb *
                 (-2 * la * log(la * la + lb * lb) - lc * log((lb * lb + lc * lc) * (sab - la)) +
                  3 * lc * log(la + sab) + la * log(sab - lc) + 3 * la * log(sab + lc)) +
             2 * lb * lb * lb * (log((sab - lc) / (lc + sab)) + log(1 + (2 * lc * (lc + sbc)) / (lb * lb)));
  return (1.0 / ((48.0 * PI) * (f * f))) * t;
}
/* rSrfEdgFlt (src/glaInt.jl:464-488) */
static cplx r_srf_edg_flt(double la, double lb, cplx f) {
  double s1 = sqrt(la * la + lb * lb), s4 = sqrt(la * la + 4 * lb * lb);
  double p1 = -la * la * la + 2 * lb * lb * (3 * lb + s1 - 2 * s4) + la * la * (2 * s1 - s4);
  double p2 =
      la * lb *
      (lb * (-62 * log(2.0) - 5 * log(-la + s1) + 4 * log(8 * lb * lb * (-la + s1)) - 33 * log(la + s1) +
             17 * log(-la + s4) - 24 * log(lb * (-la + s4)) + 57 * log(la + s4)) +
       4 * la *
           (-8 * asinh(lb / la) + 6 * asinh(2 * lb / la) + 6 * atanh(lb / s1) + 12 * log(la) - 13 * log(-lb + s1) +
            log((-lb + s1) / la) + log(la / (lb + s1)) - 7 * log(lb + s1) - 2 * log((lb + s1) / la) -
            3 * log(-(((lb + s1) * (2 * lb - s4)) / (la * la))) - 3 * log((-lb + s1) / (-2 * lb + s4)) +
            11 * log(-2 * lb + s4) - 3 * log((lb + s1) / (2 * lb + s4)) + log(2 * lb + s4) +
            9 * log((2 * lb + s4) / (lb + s1)) - 2 * log(la * la + 2 * lb * (lb - s1))));
  return (1.0 / ((12.0 * PI) * (f * f))) * p1 + (1.0 / (64.0 * PI)) * p2;
}

/* wekS / wekE / wekV (src/glaInt.jl:75-86,123-163,210-234), unscaled */
static void weak_all(const double scl[3], const quad* q, cplx wS[3], cplx wE[9], cplx wV[6]) {
  wS[0] = wek_s_dir(3, scl, q) + r_srf_slf(scl[1], scl[2], q->f);
  wS[1] = wek_s_dir(2, scl, q) + r_srf_slf(scl[0], scl[2], q->f);
  wS[2] = wek_s_dir(1, scl, q) + r_srf_slf(scl[0], scl[1], q->f);
  cplx v[4];
  wek_e_dir(3, scl, q, v);
  cplx xxY = v[0] + r_srf_edg_flt(scl[2], scl[1], q->f);
  cplx xxZ = v[2] + r_srf_edg_flt(scl[1], scl[2], q->f);
  cplx xyA = v[1] + r_srf_edg_crn(scl[2], scl[1], scl[0], q->f);
  cplx xzA = v[3] + r_srf_edg_crn(scl[1], scl[2], scl[0], q->f);
  wek_e_dir(2, scl, q, v);
  cplx yyZ = v[0] + r_srf_edg_flt(scl[0], scl[2], q->f);
  cplx yyX = v[2] + r_srf_edg_flt(scl[2], scl[0], q->f);
  cplx yzA = v[1] + r_srf_edg_crn(scl[0], scl[2], scl[1], q->f);
  cplx xyB = v[3] + r_srf_edg_crn(scl[2], scl[1], scl[0], q->f);
  wek_e_dir(1, scl, q, v);
  cplx zzX = v[0] + r_srf_edg_flt(scl[1], scl[0], q->f);
  cplx zzY = v[2] + r_srf_edg_flt(scl[0], scl[1], q->f);
  cplx xzB = v[1] + r_srf_edg_crn(scl[1], scl[2], scl[0], q->f);
  cplx yzB = v[3] + r_srf_edg_crn(scl[0], scl[2], scl[1], q->f);
  wE[0] = xxY; wE[1] = xxZ; wE[2] = yyX; wE[3] = yyZ; wE[4] = zzX; wE[5] = zzY;
  wE[6] = (xyA + xyB) / 2.0; wE[7] = (xzA + xzB) / 2.0; wE[8] = (yzA + yzB) / 2.0;
  cplx u[3];
  wek_v_dir(3, scl, q, u);
  cplx xxO = u[0], xyA2 = u[1], xzA2 = u[2];
  wek_v_dir(2, scl, q, u);
  cplx yyO = u[0], yzA2 = u[1], xyB2 = u[2];
  wek_v_dir(1, scl, q, u);
  cplx zzO = u[0], xzB2 = u[1], yzB2 = u[2];
  wV[0] = xxO; wV[1] = yyO; wV[2] = zzO;
  wV[3] = (xyA2 + xyB2) / 2.0; wV[4] = (xzA2 + xzB2) / 2.0; wV[5] = (yzA2 + yzB2) / 2.0;
}

/* -------------------------------------------------------- face geometry */
/* cubFac (src/glaInt.jl:296-311): fac[face][vertex][dim], faces yzL yzU xzL xzU xyL xyU */
static void cub_fac(const rat scl[3], double fac[6][4][3]) {
  static const int sg[6][4][3] = {
      {{-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, {-1, -1, 1}},
      {{1, -1, -1}, {1, -1, 1}, {1, 1, 1}, {1, 1, -1}},
      {{-1, -1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, -1, -1}},
      {{-1, 1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, 1, 1}},
      {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}},
      {{-1, -1, 1}, {-1, 1, 1}, {1, 1, 1}, {1, -1, 1}}};
  for (int f = 0; f < 6; ++f)
    for (int v = 0; v < 4; ++v)
      for (int d = 0; d < 3; ++d) fac[f][v][d] = rdbl(mkr(sg[f][v][d] * scl[d].n, 2 * scl[d].d));
}
/* srfScl (src/glaInt.jl:271-294) */
static void srf_scl(const rat sT[3], const rat sS[3], double out[36]) {
  for (int a = 0; a < 6; ++a) {
    rat src = (a < 2) ? rmul(sS[1], sS[2]) : (a < 4) ? rmul(sS[0], sS[2]) : rmul(sS[0], sS[1]);
    for (int b = 0; b < 6; ++b) {
      rat trg = (b < 2) ? sT[0] : (b < 4) ? sT[1] : sT[2];
      out[a * 6 + b] = rdbl(rdiv(src, trg));
    }
  }
}

/* -------------------------------------------------------- hcubature */
typedef struct {
  double c[4], h[4];
  double val[2], err[2], errmax;
  int split;
} region;

typedef struct {
  double sep[3];
  const double (*tf)[4][3];
  const double (*sf)[4][3];
  int ft, fs;  /* target face, source face (0-based) */
  cplx f;
} face_pair;

/* srfKer (src/glaGen.jl:586-598) with cubVecAltAdp (src/glaInt.jl:313-333) */
static inline void face_kernel(const face_pair* fp, const double u[4], double out[2]) {
  double v[3];
  for (int d = 0; d < 3; ++d) {
    const double* t0 = fp->tf[fp->ft][0];
    const double* t1 = fp->tf[fp->ft][1];
    const double* t3 = fp->tf[fp->ft][3];
    const double* s0 = fp->sf[fp->fs][0];
    const double* s1 = fp->sf[fp->fs][1];
    const double* s3 = fp->sf[fp->fs][3];
    double tv = t0[d] + u[2] * (t1[d] - t0[d]) + u[3] * (t3[d] - t0[d]);
    double sv = s0[d] + u[0] * (s1[d] - s0[d]) + u[1] * (s3[d] - s0[d]);
    v[d] = (tv - sv) + fp->sep[d];
  }
  cplx z = scl_ego(dst_mag(v[0], v[1], v[2]), fp->f);
  out[0] = creal(z);
  out[1] = cimag(z);
}

static const double L2 = 0.35856858280031809199064515390793749545;  /* sqrt(9/70) */
static const double L4 = 0.94868329805051379959966806332981556011;  /* sqrt(9/10) */
static const double L5 = 0.68824720161168529772162873429362352512;  /* sqrt(9/19) */

/* Genz-Malik degree 7/5 pair on one 4-D region (57 points) */
static void gm_rule(const face_pair* fp, region* R) {
  const int n = 4;
  const double w1 = (12824.0 - 9120.0 * n + 400.0 * n * n) / 19683.0, w2 = 980.0 / 6561.0,
               w3 = (1820.0 - 400.0 * n) / 19683.0, w4 = 200.0 / 19683.0, w5 = 6859.0 / 19683.0 / 16.0;
  const double e1 = (729.0 - 950.0 * n + 50.0 * n * n) / 729.0, e2 = 245.0 / 486.0, e3 = (265.0 - 100.0 * n) / 1458.0,
               e4 = 25.0 / 729.0;
  const double ratio = (L2 * L2) / (L4 * L4);
  double p[4], f0[2], fa[2], fb[2], fc[2], fd[2];
  double s2[2] = {0, 0}, s3[2] = {0, 0}, s4[2] = {0, 0}, s5[2] = {0, 0};
  double diff[4] = {0, 0, 0, 0};
  face_kernel(fp, R->c, f0);
  for (int i = 0; i < n; ++i) {
    memcpy(p, R->c, sizeof(p));
    p[i] = R->c[i] - L2 * R->h[i];
    face_kernel(fp, p, fa);
    p[i] = R->c[i] + L2 * R->h[i];
    face_kernel(fp, p, fb);
    p[i] = R->c[i] - L4 * R->h[i];
    face_kernel(fp, p, fc);
    p[i] = R->c[i] + L4 * R->h[i];
    face_kernel(fp, p, fd);
    for (int j = 0; j < 2; ++j) {
      s2[j] += fa[j] + fb[j];
      s3[j] += fc[j] + fd[j];
      diff[i] += fabs(fa[j] + fb[j] - 2 * f0[j] - ratio * (fc[j] + fd[j] - 2 * f0[j]));
    }
  }
  for (int i = 0; i < n; ++i)
    for (int k = i + 1; k < n; ++k)
      for (int si = -1; si <= 1; si += 2)
        for (int sk = -1; sk <= 1; sk += 2) {
          memcpy(p, R->c, sizeof(p));
          p[i] += si * L4 * R->h[i];
          p[k] += sk * L4 * R->h[k];
          face_kernel(fp, p, fa);
          s4[0] += fa[0];
          s4[1] += fa[1];
        }
  for (int m = 0; m < 16; ++m) {
    for (int i = 0; i < n; ++i) p[i] = R->c[i] + (((m >> i) & 1) ? L5 : -L5) * R->h[i];
    face_kernel(fp, p, fa);
    s5[0] += fa[0];
    s5[1] += fa[1];
  }
  double vol = 1.0;
  for (int i = 0; i < n; ++i) vol *= 2.0 * R->h[i];
  R->errmax = 0;
  for (int j = 0; j < 2; ++j) {
    double r7 = vol * (w1 * f0[j] + w2 * s2[j] + w3 * s3[j] + w4 * s4[j] + w5 * s5[j]);
    double r5 = vol * (e1 * f0[j] + e2 * s2[j] + e3 * s3[j] + e4 * s4[j]);
    R->val[j] = r7;
    R->err[j] = fabs(r5 - r7);
    if (R->err[j] > R->errmax) R->errmax = R->err[j];
  }
  int sd = 0;
  double md = 0;
  for (int i = 0; i < n; ++i)
    if (diff[i] > md) { md = diff[i]; sd = i; }
  R->split = sd;
}

/* max-heap on errmax */
static void heap_push(region* H, int* nh, region r) {
  int i = (*nh)++;
  H[i] = r;
  while (i > 0) {
    int p = (i - 1) / 2;
    if (H[p].errmax >= H[i].errmax) break;
    region t = H[p]; H[p] = H[i]; H[i] = t;
    i = p;
  }
}
static region heap_pop(region* H, int* nh) {
  region top = H[0];
  H[0] = H[--(*nh)];
  int i = 0;
  for (;;) {
    int l = 2 * i + 1, r = l + 1, m = i;
    if (l < *nh && H[l].errmax > H[m].errmax) m = l;
    if (r < *nh && H[r].errmax > H[m].errmax) m = r;
    if (m == i) break;
    region t = H[m]; H[m] = H[i]; H[i] = t;
    i = m;
  }
  return top;
}

static long g_max_regions = 0;  /* statistic: largest heap seen */

/* hcubature(2, f, [0,0,0,0], [1,1,1,1]; reltol, abstol, maxevals=0, INDIVIDUAL) */
static int hcub(const face_pair* fp, double reltol, double abstol, double out[2], int* nregions) {
  int cap = 1024, nh = 0;
  region* H = (region*)malloc(sizeof(region) * cap);
  region R0;
  for (int i = 0; i < 4; ++i) { R0.c[i] = 0.5; R0.h[i] = 0.5; }
  gm_rule(fp, &R0);
  double tv[2] = {R0.val[0], R0.val[1]}, te[2] = {R0.err[0], R0.err[1]};
  heap_push(H, &nh, R0);
  int it = 0;
  for (;;) {
    int conv = 1;
    for (int j = 0; j < 2; ++j)
      if (te[j] > abstol && te[j] > fabs(tv[j]) * reltol) conv = 0;
    if (conv) break;
    if (++it > 2000000) { free(H); return -1; }
    if (nh + 2 > cap) {
      cap *= 2;
      H = (region*)realloc(H, sizeof(region) * cap);
    }
    region R = heap_pop(H, &nh);
    for (int j = 0; j < 2; ++j) { tv[j] -= R.val[j]; te[j] -= R.err[j]; }
    region A = R, B = R;
    int d = R.split;
    A.h[d] = B.h[d] = R.h[d] * 0.5;
    A.c[d] = R.c[d] - A.h[d];
    B.c[d] = R.c[d] + A.h[d];
    gm_rule(fp, &A);
    gm_rule(fp, &B);
    for (int j = 0; j < 2; ++j) { tv[j] += A.val[j] + B.val[j]; te[j] += A.err[j] + B.err[j]; }
    heap_push(H, &nh, A);
    heap_push(H, &nh, B);
  }
  out[0] = out[1] = 0;
  for (int i = 0; i < nh; ++i) { out[0] += H[i].val[0]; out[1] += H[i].val[1]; }
  if (nregions) *nregions = nh;
  free(H);
  return 0;
}

static const double CUB_RELTOL = 1e-6, CUB_ABSTOL = 1e-9, CNT_TOL = 1e-8;  /* src/glaGen.jl:3-8 */

/* egoSrfAdp! (src/glaGen.jl:559-584) for the listed face pairs (0-based) */
static int srf_adp(const double sep[3], cplx srf[36], const double tf[6][4][3], const double sf[6][4][3],
                   const int* list, int nlist, const double scales[36], cplx f) {
  for (int k = 0; k < nlist; ++k) {
    int fp = list[k];
    face_pair P;
    memcpy(P.sep, sep, sizeof(P.sep));
    P.tf = tf;
    P.sf = sf;
    P.ft = fp / 6;
    P.fs = fp % 6;
    P.f = f;
    double v[2];
    int nr = 0;
    if (hcub(&P, CUB_RELTOL, CUB_ABSTOL, v, &nr)) return -1;
    if (nr > g_max_regions) g_max_regions = nr;
    srf[fp] = (v[0] + I * v[1]) * scales[fp];
  }
  return 0;
}

/* srfSum! (src/glaGen.jl:531-555); out[r][c] 0-based, s 1-based offsets */
static void srf_sum(const cplx s_[36], cplx out[3][3]) {
  const cplx* s = s_ - 1;
  out[0][0] = s[15] - s[16] - s[21] + s[22] + s[29] - s[30] - s[35] + s[36];
  out[1][0] = -s[13] + s[14] + s[19] - s[20];
  out[2][0] = -s[25] + s[26] + s[31] - s[32];
  out[0][1] = -s[3] + s[4] + s[9] - s[10];
  out[1][1] = s[1] - s[2] - s[7] + s[8] + s[29] - s[30] - s[35] + s[36];
  out[2][1] = -s[27] + s[28] + s[33] - s[34];
  out[0][2] = -s[5] + s[6] + s[11] - s[12];
  out[1][2] = -s[17] + s[18] + s[23] - s[24];
  out[2][2] = s[1] - s[2] - s[7] + s[8] + s[15] - s[16] - s[21] + s[22];
}

/* egoFunSng! correction tables (src/glaGen.jl:370-509): code 0 = none,
 * 1..3 = wS[k], 11..19 = wE[k], 21..26 = wV[k] (1-based k) */
static const signed char SNG_COR[8][6][6] = {
    /* (1,1,1) */ {{1, 0, 17, 17, 18, 18}, {0, 1, 17, 17, 18, 18}, {17, 17, 2, 0, 19, 19},
                   {17, 17, 0, 2, 19, 19}, {18, 18, 19, 19, 3, 0}, {18, 18, 19, 19, 0, 3}},
    /* (2,1,1) */ {{0, 1, 17, 17, 18, 18}, {0, 0, 0, 0, 0, 0}, {0, 17, 13, 0, 26, 26},
                   {0, 17, 0, 13, 26, 26}, {0, 18, 26, 26, 15, 0}, {0, 18, 26, 26, 0, 15}},
    /* (2,1,2) */ {{0, 12, 24, 24, 0, 18}, {0, 0, 0, 0, 0, 0}, {0, 24, 22, 0, 0, 26},
                   {0, 24, 0, 22, 0, 26}, {0, 18, 26, 26, 0, 15}, {0, 0, 0, 0, 0, 0}},
    /* (1,1,2) */ {{12, 0, 24, 24, 0, 18}, {0, 12, 24, 24, 0, 18}, {24, 24, 14, 0, 0, 19},
                   {24, 24, 0, 14, 0, 19}, {18, 18, 19, 19, 0, 3}, {0, 0, 0, 0, 0, 0}},
    /* (1,2,1) */ {{11, 0, 0, 17, 25, 25}, {0, 11, 0, 17, 25, 25}, {17, 17, 0, 2, 19, 19},
                   {0, 0, 0, 0, 0, 0}, {25, 25, 0, 19, 16, 0}, {25, 25, 0, 19, 0, 16}},
    /* (2,2,1) */ {{0, 11, 0, 17, 25, 25}, {0, 0, 0, 0, 0, 0}, {0, 17, 0, 13, 26, 26},
                   {0, 0, 0, 0, 0, 0}, {0, 25, 0, 26, 23, 0}, {0, 25, 0, 26, 0, 23}},
    /* (1,2,2) */ {{21, 0, 0, 24, 0, 25}, {0, 21, 0, 24, 0, 25}, {24, 24, 0, 14, 0, 19},
                   {0, 0, 0, 0, 0, 0}, {25, 25, 0, 19, 0, 16}, {0, 0, 0, 0, 0, 0}},
    /* (2,2,2) */ {{0, 21, 0, 24, 0, 25}, {0, 0, 0, 0, 0, 0}, {0, 24, 0, 22, 0, 26},
                   {0, 0, 0, 0, 0, 0}, {0, 25, 0, 26, 0, 23}, {0, 0, 0, 0, 0, 0}}};
static const signed char SNG_MASK[8][6][6] = {
    {{1, 0, 1, 1, 1, 1}, {0, 1, 1, 1, 1, 1}, {1, 1, 1, 0, 1, 1}, {1, 1, 0, 1, 1, 1}, {1, 1, 1, 1, 1, 0}, {1, 1, 1, 1, 0, 1}},
    {{0, 1, 1, 1, 1, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 1, 0, 1, 1}, {0, 1, 0, 1, 1, 1}, {0, 1, 1, 1, 1, 0}, {0, 1, 1, 1, 0, 1}},
    {{0, 1, 1, 1, 0, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 1, 0, 0, 1}, {0, 1, 0, 1, 0, 1}, {0, 1, 1, 1, 0, 1}, {0, 0, 0, 0, 0, 0}},
    {{1, 0, 1, 1, 0, 1}, {0, 1, 1, 1, 0, 1}, {1, 1, 1, 0, 0, 1}, {1, 1, 0, 1, 0, 1}, {1, 1, 1, 1, 0, 1}, {0, 0, 0, 0, 0, 0}},
    {{1, 0, 0, 1, 1, 1}, {0, 1, 0, 1, 1, 1}, {1, 1, 0, 1, 1, 1}, {0, 0, 0, 0, 0, 0}, {1, 1, 0, 1, 1, 0}, {1, 1, 0, 1, 0, 1}},
    {{0, 1, 0, 1, 1, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 1, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 1, 0}, {0, 1, 0, 1, 0, 1}},
    {{1, 0, 0, 1, 0, 1}, {0, 1, 0, 1, 0, 1}, {1, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}, {1, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}},
    {{0, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}, {0, 1, 0, 1, 0, 1}, {0, 0, 0, 0, 0, 0}}};

static int sng_case(int px, int py, int pz, const vol* v) {
  int tx = rlt(v->scl[0], v->grd[0]) ? 0 : 1; /* scl == step (contact) */
  int ty = rlt(v->scl[1], v->grd[1]) ? 0 : 1;
  int tz = rlt(v->scl[2], v->grd[2]) ? 0 : 1;
  if (px == 1 && py == 1 && pz == 1) return 0;
  if (px == 2 && py == 1 && pz == 1 && tx) return 1;
  if (px == 2 && py == 1 && pz == 2 && tx && tz) return 2;
  if (px == 1 && py == 1 && pz == 2 && tz) return 3;
  if (px == 1 && py == 2 && pz == 1 && ty) return 4;
  if (px == 2 && py == 2 && pz == 1 && tx && ty) return 5;
  if (px == 1 && py == 2 && pz == 2 && ty && tz) return 6;
  if (px == 2 && py == 2 && pz == 2 && tx && ty && tz) return 7;
  return -1; /* "empty case selected": every pair by cubature */
}

/* ----------------------------------------------------------- self build */
/* genEgoCrcSlf! (src/glaGen.jl:102-136): Toeplitz toe[iz][iy][ix][3][3] */
static int self_toeplitz(const vol* v, cplx f, int int_ord, cplx* toe, const cplx* wpre) {
  const int64_t nx = v->cel[0], ny = v->cel[1], nz = v->cel[2];
  double tf[6][4][3], sc[36];
  cub_fac(v->scl, tf);
  srf_scl(v->scl, v->scl, sc);
  int all[36];
  for (int k = 0; k < 36; ++k) all[k] = k;
  int fail = 0;
  /* far offsets: some 1-based index > 2 (src/glaGen.jl:322-335) */
#pragma omp parallel for schedule(dynamic) collapse(3)
  for (int64_t iz = 0; iz < nz; ++iz)
    for (int64_t iy = 0; iy < ny; ++iy)
      for (int64_t ix = 0; ix < nx; ++ix) {
        cplx* t = toe + ((iz * ny + iy) * nx + ix) * 9;
        if (!(ix > 1 || iy > 1 || iz > 1)) continue;
        double sep[3] = {rdbl(rmul(rint_(ix), v->grd[0])), rdbl(rmul(rint_(iy), v->grd[1])),
                         rdbl(rmul(rint_(iz), v->grd[2]))};
        cplx srf[36];
        memset(srf, 0, sizeof(srf));
        if (srf_adp(sep, srf, tf, tf, all, 36, sc, f)) fail = 1;
        cplx o[3][3];
        srf_sum(srf, o);
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) t[r * 3 + c] = o[r][c];
      }
  if (fail) return -1;
  /* weak integrals, scaled by 1/prod(scl) (src/glaGen.jl:115-121) */
  cplx wS[3], wE[9], wV[6];
  if (wpre) {
    memcpy(wS, wpre, sizeof(wS));
    memcpy(wE, wpre + 3, sizeof(wE));
    memcpy(wV, wpre + 12, sizeof(wV));
  } else {
    double x[128], w[128];
    gila_ref_gauleg(int_ord, x, w);
    quad q = {int_ord, x, w, f};
    double scl[3] = {rdbl(v->scl[0]), rdbl(v->scl[1]), rdbl(v->scl[2])};
    weak_all(scl, &q, wS, wE, wV);
  }
  double inv = rdbl(rdiv(rint_(1), rmul(rmul(v->scl[0], v->scl[1]), v->scl[2])));
  for (int k = 0; k < 3; ++k) wS[k] *= inv;
  for (int k = 0; k < 9; ++k) wE[k] *= inv;
  for (int k = 0; k < 6; ++k) wV[k] *= inv;
  /* near offsets (src/glaGen.jl:122-126, egoFunSng! :350-528) */
  for (int pz = 1; pz <= (nz < 2 ? nz : 2); ++pz)
    for (int py = 1; py <= (ny < 2 ? ny : 2); ++py)
      for (int px = 1; px <= (nx < 2 ? nx : 2); ++px) {
        int cs = sng_case(px, py, pz, v);
        int mask[6][6];
        cplx cor[6][6];
        for (int a = 0; a < 6; ++a)
          for (int b = 0; b < 6; ++b) {
            mask[a][b] = cs < 0 ? 0 : SNG_MASK[cs][a][b];
            int code = cs < 0 ? 0 : SNG_COR[cs][a][b];
            cor[a][b] = code == 0 ? 0 : code < 10 ? wS[code - 1] : code < 20 ? wE[code - 11] : wV[code - 21];
          }
        if (cs < 0) fprintf(stderr, "empty case selected.\n");
        int list[36], nl = 0;
        for (int fp = 0; fp < 36; ++fp)
          if (!mask[fp / 6][fp % 6]) list[nl++] = fp;
        double sep[3] = {rdbl(rmul(rint_(px - 1), v->grd[0])), rdbl(rmul(rint_(py - 1), v->grd[1])),
                         rdbl(rmul(rint_(pz - 1), v->grd[2]))};
        cplx srf[36];
        memset(srf, 0, sizeof(srf));
        if (srf_adp(sep, srf, tf, tf, list, nl, sc, f)) return -1;
        for (int fp = 0; fp < 36; ++fp)
          if (mask[fp / 6][fp % 6]) srf[fp] = cor[fp / 6][fp % 6];
        cplx o[3][3];
        srf_sum(srf, o);
        cplx* t = toe + (((int64_t)(pz - 1) * ny + (py - 1)) * nx + (px - 1)) * 9;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) t[r * 3 + c] = o[r][c];
      }
  /* identity (src/glaGen.jl:128-130) */
  cplx id = 1.0 / (f * f);
  toe[0] -= id;
  toe[4] -= id;
  toe[8] -= id;
  return 0;
}

/* egoToeCrc! (src/glaGen.jl:143-163): circulant crc[z][y][x][3][3] of 2N */
static void toe_to_crc(const int64_t n[3], const cplx* toe, cplx* crc) {
  const int64_t P[3] = {2 * n[0], 2 * n[1], 2 * n[2]};
  for (int64_t z = 0; z < P[2]; ++z)
    for (int64_t y = 0; y < P[1]; ++y)
      for (int64_t x = 0; x < P[0]; ++x) {
        cplx* o = crc + ((z * P[1] + y) * P[0] + x) * 9;
        int64_t p[3] = {x, y, z};
        int zero = 0;
        int64_t s[3];
        double fl[3];
        for (int d = 0; d < 3; ++d) {
          if (p[d] == n[d]) zero = 1;
          s[d] = p[d] < n[d] ? p[d] : 2 * n[d] - p[d];
          fl[d] = p[d] < n[d] ? 1.0 : -1.0;
        }
        if (zero) {
          for (int k = 0; k < 9; ++k) o[k] = 0;
          continue;
        }
        const cplx* t = toe + ((s[2] * n[1] + s[1]) * n[0] + s[0]) * 9;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) o[r * 3 + c] = t[r * 3 + c] * (r == c ? 1.0 : fl[r] * fl[c]);
      }
}

static int self_circulant(const vol* v, cplx f, int int_ord, cplx* crc, const cplx* wpre) {
  const int64_t V = v->cel[0] * v->cel[1] * v->cel[2];
  cplx* toe = (cplx*)calloc((size_t)V * 9, sizeof(cplx));
  if (!toe) return -2;
  int e = self_toeplitz(v, f, int_ord, toe, wpre);
  if (!e) toe_to_crc(v->cel, toe, crc);
  free(toe);
  return e;
}

/* ------------------------------------------------------- external build */
/* sepGrd (src/glaGen.jl:603-630): value at 0-based k */
typedef struct { rat str, step; } sgrid;
static sgrid sep_grd(const vol* t, const vol* s, int flip, int d) {
  sgrid g;
  rat sep, str, stp;
  if (flip) {
    sep = s->grd[d];
    str = rsub(t->start[d], s->stop[d]);
    stp = rsub(t->start[d], s->start[d]);
  } else {
    sep = t->grd[d];
    str = rsub(t->start[d], s->start[d]);
    stp = rsub(t->stop[d], s->start[d]);
  }
  if (rlt(stp, str)) sep = rmul(sep, rint_(-1));
  g.str = str;
  g.step = sep;
  return g;
}
/* grdSel (src/glaGen.jl:632-645), ind 1-based */
static double grd_sel(int64_t ind, int64_t spt, sgrid tg, sgrid sg) {
  if (ind <= spt) return rdbl(radd(tg.str, rmul(rint_(ind - 1), tg.step)));
  if (ind > 1 + spt) ind -= 1;
  return rdbl(radd(sg.str, rmul(rint_(ind - spt - 1), sg.step)));
}

/* crcIndClc (src/glaGen.jl:665-672) -> 0-based circulant index */
static void crc_ind(const int64_t cel[3], const int64_t t[3], const int64_t s[3], int64_t out[3]) {
  for (int d = 0; d < 3; ++d) {
    int64_t c = t[d] - s[d];
    out[d] = c + (c < 0 ? 2 * cel[d] : 0);
  }
}

/* genEgoCrcExt! (src/glaGen.jl:55-100) with egoFunExt!, egoFunExtCnt!, egoCntOut! */
static int ext_circulant(const vol* t, const vol* s, cplx f, int int_ord, cplx* crc) {
  const int64_t P[3] = {t->cel[0] + s->cel[0], t->cel[1] + s->cel[1], t->cel[2] + s->cel[2]};
  double tf[6][4][3], sf[6][4][3], sc[36];
  cub_fac(t->scl, tf);
  cub_fac(s->scl, sf);
  srf_scl(t->scl, s->scl, sc);
  sgrid gt[3], gs[3];
  for (int d = 0; d < 3; ++d) {
    gt[d] = sep_grd(t, s, 0, d);
    gs[d] = sep_grd(t, s, 1, d);
  }
  /* edges */
  rat sl[3], su[3], tl[3], tu[3];
  for (int d = 0; d < 3; ++d) {
    rat hs = rdiv(s->scl[d], rint_(2)), ht = rdiv(t->scl[d], rint_(2));
    sl[d] = rsub(s->start[d], hs);
    su[d] = radd(s->stop[d], hs);
    tl[d] = rsub(t->start[d], ht);
    tu[d] = radd(t->stop[d], ht);
  }
  int c1 = 1, c2 = 1, ovr = 0;
  for (int d = 0; d < 3; ++d) {
    c1 &= rle(sl[d], tl[d]) && rle(tl[d], su[d]);
    c2 &= rle(sl[d], tu[d]) && rle(tu[d], su[d]);
    ovr += rlt(sl[d], tl[d]) && rlt(tl[d], su[d]);
    ovr += rlt(sl[d], tu[d]) && rlt(tu[d], su[d]);
  }
  int contact = c1 || c2;
  if (contact && ovr > 0) return -3; /* "Source and target volumes are overlapping." */
  vol cv;
  cplx* ccnt = NULL;
  if (contact) {
    /* genCntVol (src/glaGen.jl:308-318) */
    int64_t cel[3], sn[3], sd[3], on[3] = {0, 0, 0}, od[3] = {1, 1, 1};
    for (int d = 0; d < 3; ++d) {
      rat m = rlt(t->scl[d], s->scl[d]) ? t->scl[d] : s->scl[d];
      rat a = rdiv(t->scl[d], m), b = rdiv(s->scl[d], m);
      cel[d] = a.n / a.d + b.n / b.d;
      sn[d] = m.n;
      sd[d] = m.d;
    }
    cv = mkvol(cel, sn, sd, on, od, NULL, NULL);
    ccnt = (cplx*)calloc((size_t)(8 * cel[0] * cel[1] * cel[2]) * 9, sizeof(cplx));
    int e = self_circulant(&cv, f, int_ord, ccnt, NULL);
    if (e) { free(ccnt); return e; }
  }
  int all[36];
  for (int k = 0; k < 36; ++k) all[k] = k;
  int fail = 0;
#pragma omp parallel for schedule(dynamic) collapse(3)
  for (int64_t z = 0; z < P[2]; ++z)
    for (int64_t y = 0; y < P[1]; ++y)
      for (int64_t x = 0; x < P[0]; ++x) {
        cplx* o = crc + ((z * P[1] + y) * P[0] + x) * 9;
        int64_t pi[3] = {x + 1, y + 1, z + 1};
        int split = 0;
        double sep[3];
        for (int d = 0; d < 3; ++d) {
          if (pi[d] == t->cel[d] + 1) split = 1;
          sep[d] = grd_sel(pi[d], t->cel[d], gt[d], gs[d]);
        }
        for (int k = 0; k < 9; ++k) o[k] = 0;
        if (split) continue;
        int touch = contact;
        if (contact)
          for (int d = 0; d < 3; ++d)
            touch &= fabs(sep[d]) < CNT_TOL + (rdbl(t->scl[d]) + rdbl(s->scl[d])) / 2.0;
        if (touch) {
          /* egoCntOut! (src/glaGen.jl:250-306) */
          int64_t sL[3], sU[3], tL[3], tU[3];
          for (int d = 0; d < 3; ++d) {
            rat ss = rdiv(s->scl[d], cv.scl[d]), ts = rdiv(t->scl[d], cv.scl[d]);
            int64_t sspan = ss.n / ss.d, tspan = ts.n / ts.d;
            double span = sep[d] / rdbl(cv.scl[d]);
            sL[d] = 1;
            sU[d] = sspan;
            tL[d] = (int64_t)nearbyint(span + sspan / 2.0 - tspan / 2.0) + 1;
            tU[d] = (int64_t)nearbyint(span + sspan / 2.0 + tspan / 2.0);
            if (tL[d] < 1) {
              int64_t sh = (tL[d] < 0 ? -tL[d] : tL[d]) + 1;
              sL[d] += sh;
              sU[d] += sh;
              tU[d] += sh;
              tL[d] += sh;
            }
          }
          cplx acc[9] = {0};
          for (int64_t a = sL[2]; a <= sU[2]; ++a)
            for (int64_t b = sL[1]; b <= sU[1]; ++b)
              for (int64_t c = sL[0]; c <= sU[0]; ++c)
                for (int64_t aa = tL[2]; aa <= tU[2]; ++aa)
                  for (int64_t bb = tL[1]; bb <= tU[1]; ++bb)
                    for (int64_t cc = tL[0]; cc <= tU[0]; ++cc) {
                      int64_t ti[3] = {cc, bb, aa}, si[3] = {c, b, a}, ci[3];
                      crc_ind(cv.cel, ti, si, ci);
                      const int64_t Pc[3] = {2 * cv.cel[0], 2 * cv.cel[1], 2 * cv.cel[2]};
                      const cplx* src = ccnt + ((ci[2] * Pc[1] + ci[1]) * Pc[0] + ci[0]) * 9;
                      for (int k = 0; k < 9; ++k) acc[k] += src[k];
                    }
          double tot = (double)((tU[2] - tL[2] + 1) * (tU[1] - tL[1] + 1) * (tU[0] - tL[0] + 1));
          for (int k = 0; k < 9; ++k) o[k] = acc[k] / tot;
        } else {
          cplx srf[36];
          memset(srf, 0, sizeof(srf));
          if (srf_adp(sep, srf, tf, sf, all, 36, sc, f)) fail = 1;
          cplx m[3][3];
          srf_sum(srf, m);
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) o[r * 3 + c] = m[r][c];
        }
      }
  free(ccnt);
  return fail ? -1 : 0;
}

/* ============================================================ exported API */
/* All complex outputs are interleaved doubles; circulants are stored
 * crc[z][y][x][3][3] (row r, column c of the 3x3 block at [r*3+c]). */

int gila_ref_weak(const int64_t scl_n[3], const int64_t scl_d[3], double frq_re, double frq_im, int int_ord,
                  double* out /* 18 complex: wS[3], wE[9], wV[6] (unscaled) */) {
  double x[128], w[128];
  if (int_ord < 1 || int_ord > 128) return -4;
  gila_ref_gauleg(int_ord, x, w);
  quad q = {int_ord, x, w, frq_re + I * frq_im};
  double scl[3];
  for (int k = 0; k < 3; ++k) scl[k] = rdbl(mkr(scl_n[k], scl_d[k]));
  cplx wS[3], wE[9], wV[6];
  weak_all(scl, &q, wS, wE, wV);
  cplx* o = (cplx*)out;
  memcpy(o, wS, sizeof(wS));
  memcpy(o + 3, wE, sizeof(wE));
  memcpy(o + 12, wV, sizeof(wV));
  return 0;
}

/* weak: optional 18 precomputed unscaled weak values (NULL = compute) */
int gila_ref_self_circulant(const int64_t cel[3], const int64_t scl_n[3], const int64_t scl_d[3],
                            const int64_t grd_n[3], const int64_t grd_d[3], double frq_re, double frq_im, int int_ord,
                            const double* weak, double* crc_out) {
  int64_t on[3] = {0, 0, 0}, od[3] = {1, 1, 1};
  vol v = mkvol(cel, scl_n, scl_d, on, od, grd_n, grd_d);
  if (int_ord < 1 || int_ord > 128) return -4;
  return self_circulant(&v, frq_re + I * frq_im, int_ord, (cplx*)crc_out, (const cplx*)weak);
}

int gila_ref_ext_circulant(const int64_t tcel[3], const int64_t tscl_n[3], const int64_t tscl_d[3],
                           const int64_t torg_n[3], const int64_t torg_d[3], const int64_t tgrd_n[3],
                           const int64_t tgrd_d[3], const int64_t scel[3], const int64_t sscl_n[3],
                           const int64_t sscl_d[3], const int64_t sorg_n[3], const int64_t sorg_d[3],
                           const int64_t sgrd_n[3], const int64_t sgrd_d[3], double frq_re, double frq_im,
                           int int_ord, double* crc_out) {
  vol t = mkvol(tcel, tscl_n, tscl_d, torg_n, torg_d, tgrd_n, tgrd_d);
  vol s = mkvol(scel, sscl_n, sscl_d, sorg_n, sorg_d, sgrd_n, sgrd_d);
  return ext_circulant(&t, &s, frq_re + I * frq_im, int_ord, (cplx*)crc_out);
}

/* one face-pair integral (tests / GPU parity): faces 0-based, sep in wavelengths */
int gila_ref_face_pair(const int64_t tscl_n[3], const int64_t tscl_d[3], const int64_t sscl_n[3],
                       const int64_t sscl_d[3], const double sep[3], int ft, int fs, double frq_re, double frq_im,
                       double* out2, int* nregions) {
  rat ts[3], ss[3];
  for (int k = 0; k < 3; ++k) {
    ts[k] = mkr(tscl_n[k], tscl_d[k]);
    ss[k] = mkr(sscl_n[k], sscl_d[k]);
  }
  double tf[6][4][3], sf[6][4][3];
  cub_fac(ts, tf);
  cub_fac(ss, sf);
  face_pair P;
  memcpy(P.sep, sep, sizeof(P.sep));
  P.tf = tf;
  P.sf = sf;
  P.ft = ft;
  P.fs = fs;
  P.f = frq_re + I * frq_im;
  return hcub(&P, CUB_RELTOL, CUB_ABSTOL, out2, nregions);
}

long gila_ref_max_regions(void) { return g_max_regions; }
