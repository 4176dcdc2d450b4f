// kerbuild.cu -- the FP64 Green-kernel build on the GPU.
//
// Replaces GlaOprMem's kernel section (src/glaMemSup.jl:44-156) and the
// real-space element generation it calls (src/glaGen.jl, src/glaInt.jl,
// src/glaIntSup.jl), which the reference runs on host threads (hours at
// 256x256x128, hence its JLD2 cache).  Everything stays in FP64:
//
//   1. weak (singular) face-pair integrals wekS / wekE / wekV: the DIRECTFN
//      nested Gauss-Legendre sums (src/glaIntSup.jl) as block reductions,
//      partials reduced in a fixed order (deterministic);
//   2. the 8 near offsets (egoFunSng!, src/glaGen.jl:350-528): corrected
//      pairs from the weak values, the rest by cubature;
//   3. far offsets (egoFunInn! / egoFunOut!, src/glaGen.jl:233-248,322-335):
//      one warp per offset runs the adaptive Genz-Malik degree-7/5 cubature
//      (the algorithm of Cubature.jl's hcubature, src/glaGen.jl:574-576) for
//      the 24 face pairs that feed the six stored components, the region heap
//      of each warp in global scratch;
//   4. external operators: circulant separations by grdSel/sepGrd
//      (src/glaGen.jl:603-645), touching offsets averaged from the contact
//      self circulant (egoCntOut!, src/glaGen.jl:250-306);
//   5. Toeplitz -> circulant embedding (egoToeCrc!, src/glaGen.jl:143-163),
//      FP64 3-D FFT of the six components, parity-branch extraction and
//      symmetric truncation (src/glaMemSup.jl:96-156), cast to the operator
//      dtype, NaN/Inf check.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

namespace gila {
namespace kb {

constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double S3 = 1.7320508075688772935274463415058723669;
constexpr double CUB_RELTOL = 1e-6, CUB_ABSTOL = 1e-9, CNT_TOL = 1e-8;  // src/glaGen.jl:3-8
constexpr int kMaxOrd = 64;

// ------------------------------------------------------------ complex FP64
struct Z {
  double x, y;
};
__host__ __device__ inline Z zmk(double a, double b) { return Z{a, b}; }
__host__ __device__ inline Z zadd(Z a, Z b) { return Z{a.x + b.x, a.y + b.y}; }
__host__ __device__ inline Z zsub(Z a, Z b) { return Z{a.x - b.x, a.y - b.y}; }
__host__ __device__ inline Z zmul(Z a, Z b) { return Z{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__host__ __device__ inline Z zsc(Z a, double s) { return Z{a.x * s, a.y * s}; }
__host__ __device__ inline Z zdiv(Z a, Z b) {
  const double d = b.x * b.x + b.y * b.y;
  return Z{(a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d};
}

struct Consts {
  int ord;
  double x[kMaxOrd], w[kMaxOrd];  // Gauss-Legendre nodes / weights on [-1,1]
  Z f;                            // frqPhz
};

// sclEgo (src/glaInt.jl:41-44): exp(2 pi i d f) / (4 pi d f^2)
__device__ inline Z scl_ego(double d, Z f) {
  const Z z = zsc(f, (2.0 * PI) * d);
  const double e = exp(-z.y);
  double s, c;
  sincos(z.x, &s, &c);
  return zdiv(Z{e * c, e * s}, zsc(zmul(f, f), (4.0 * PI) * d));
}
// sclEgoN (src/glaInt.jl:51-59)
__device__ inline Z scl_ego_n(double d, Z f) {
  if (d > 1e-7) {
    const Z z = zsc(f, (2.0 * PI) * d);
    const double e = exp(-z.y);
    double s, c;
    sincos(z.x, &s, &c);
    return zdiv(Z{e * c - 1.0, e * s}, zsc(zmul(f, f), (4.0 * PI) * d));
  }
  const Z a = zdiv(Z{0.0, 1.0}, f);
  return Z{(a.x - PI * d) / 2.0, a.y / 2.0};
}

__device__ inline double thf(double a, double b, double p) { return 0.5 * ((b - a) * p + a + b); }

struct Tri6 {
  double r[6][3];
};

__device__ inline void spx(double xp[3][2], double e1, double e2, double x1, double x2) {
  xp[0][0] = (S3 * (1.0 - e1) - x1) / (2.0 * S3);
  xp[1][0] = (S3 * (1.0 + e1) - x1) / (2.0 * S3);
  xp[2][0] = x1 / S3;
  xp[0][1] = (S3 * (1.0 - e2) - x2) / (2.0 * S3);
  xp[1][1] = (S3 * (1.0 + e2) - x2) / (2.0 * S3);
  xp[2][1] = x2 / S3;
}
__device__ inline double dist6(const Tri6& t, const double xp[3][2]) {
  double v[3];
  for (int d = 0; d < 3; ++d)
    v[d] = xp[0][0] * t.r[0][d] + xp[1][0] * t.r[1][d] + xp[2][0] * t.r[2][d] -
           (xp[0][1] * t.r[3][d] + xp[1][1] * t.r[4][d] + xp[2][1] * t.r[5][d]);
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}
__device__ inline double dist3(const Tri6& t, const double xp[3][2]) {
  double v[3];
  for (int d = 0; d < 3; ++d)
    v[d] = xp[0][0] * t.r[0][d] + xp[1][0] * t.r[1][d] + xp[2][0] * t.r[2][d] -
           (xp[0][1] * t.r[0][d] + xp[1][1] * t.r[1][d] + xp[2][1] * t.r[2][d]);
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

// subTri (src/glaIntSup.jl:365-379)
__device__ inline void sub_tri(double l1, double l2, int dir, double& e, double& x) {
  if (dir == 1) {
    e = l1;
    x = l2;
  } else if (dir == 2) {
    e = 0.5 * (1.0 - l1 - l2 * S3);
    x = 0.5 * (S3 + l1 * S3 - l2);
  } else {
    e = 0.5 * (-1.0 - l1 + l2 * S3);
    x = 0.5 * (S3 - l1 * S3 - l2);
  }
}
// aS (src/glaIntSup.jl:313-332)
__device__ Z a_s(const Tri6& t, double th1, double thB, double th, int dir, const Consts& q) {
  double xp[3][2];
  Z acc{0, 0};
  double s1, c1;
  sincos(th1, &s1, &c1);
  for (int n = 0; n < q.ord; ++n) {
    double e1, x1, e2, x2;
    sub_tri(thB, th * s1, dir, e1, x1);
    const double u = thf(0.0, th, q.x[n]);
    sub_tri(u * c1 + thB, (th - u) * s1, dir, e2, x2);
    spx(xp, e1, e2, x1, x2);
    acc = zadd(acc, zsc(scl_ego_n(dist3(t, xp), q.f), q.w[n] * u));
  }
  return zsc(acc, 0.5 * th);
}
__device__ inline void psi_lim_s(int idf, double& a, double& b) {
  if (idf == 1 || idf == 5 || idf == 6) {
    a = 0.0;
    b = PI / 3.0;
  } else if (idf == 2 || idf == 7) {
    a = PI / 3.0;
    b = 2.0 * PI / 3.0;
  } else {
    a = 2.0 * PI / 3.0;
    b = PI;
  }
}
__device__ inline void eta_lim_s(int idf, double th, double& a, double& b) {
  if (idf == 1 || idf == 2) {
    a = 0.0;
    b = 1.0;
  } else if (idf == 3) {
    a = (S3 - tan(PI - th)) / (S3 + tan(PI - th));
    b = 1.0;
  } else if (idf == 4) {
    a = 0.0;
    b = (S3 - tan(PI - th)) / (S3 + tan(PI - th));
  } else if (idf == 5) {
    a = (tan(th) - S3) / (S3 + tan(th));
    b = 0.0;
  } else if (idf == 6) {
    a = -1.0;
    b = (tan(th) - S3) / (S3 + tan(th));
  } else {
    a = -1.0;
    b = 0.0;
  }
}
// nS (src/glaIntSup.jl:201-237): the n-th term (weight included) and its factor
__device__ inline Z n_s_term(int dir, int idf, double th1, double thB, int n, const Tri6& t, const Consts& q) {
  double L, fac;
  if (idf == 1 || idf == 5) {
    L = (1.0 - thB) / cos(th1);
    fac = (1.0 - thB) / (2.0 * cos(th1));
  } else if (idf == 2 || idf == 3) {
    L = S3 * (1.0 - thB) / sin(th1);
    fac = S3 * (1.0 - thB) / (2.0 * sin(th1));
  } else if (idf == 6 || idf == 7) {
    L = S3 * (1.0 + thB) / sin(th1);
    fac = S3 * (1.0 + thB) / (2.0 * sin(th1));
  } else {
    L = -(1.0 + thB) / cos(th1);
    fac = -(1.0 + thB) / (2.0 * cos(th1));
  }
  return zsc(a_s(t, th1, thB, thf(0.0, L, q.x[n]), dir, q), fac * q.w[n]);
}

// spxE! / aE / intNE (src/glaIntSup.jl:283-348,395-411)
__device__ inline void spx_e(double xp[3][2], double lam, double eta, double thB, double th1, int idf) {
  double sB, cB, s1, c1;
  sincos(thB, &sB, &cB);
  sincos(th1, &s1, &c1);
  if (idf == 1)
    spx(xp, eta, lam * cB * c1 - eta, lam * sB, lam * cB * s1);
  else
    spx(xp, -eta, -(lam * cB * c1 - eta), lam * sB, lam * cB * s1);
}
__device__ Z a_e(const Tri6& t, double lam, double eta, double thB, double th1, int idf, const Consts& q) {
  double xp[3][2];
  Z acc{0, 0};
  for (int n = 0; n < q.ord; ++n) {
    const double z = thf(0.0, lam, q.x[n]);
    spx_e(xp, z, eta, thB, th1, idf);
    acc = zadd(acc, zsc(scl_ego_n(dist6(t, xp), q.f), q.w[n] * z * z));
  }
  return zsc(acc, 0.5 * lam);
}
__device__ Z int_ne(int n, int idf1, double gam, double thB, double th1, const Tri6& t, int idf2, const Consts& q) {
  double eta, lam, s1, c1;
  sincos(th1, &s1, &c1);
  if (idf1 == 1) {
    eta = thf(0.0, gam, q.x[n]);
    lam = S3 * (1 + eta) / (cos(thB) * (s1 + S3 * c1));
  } else if (idf1 == 2) {
    eta = thf(gam, 1.0, q.x[n]);
    lam = S3 * (1.0 - fabs(eta)) / sin(thB);
  } else if (idf1 == 3) {
    eta = thf(gam, 1.0, q.x[n]);
    lam = S3 * (1.0 - fabs(eta)) / (cos(thB) * (s1 - S3 * c1));
  } else if (idf1 == 4) {
    eta = thf(0.0, 1.0, q.x[n]);
    lam = S3 * (1.0 - fabs(eta)) / (cos(thB) * (s1 - S3 * c1));
  } else {
    eta = thf(0.0, 1.0, q.x[n]);
    lam = S3 * (1.0 - eta) / sin(thB);
  }
  return a_e(t, lam, eta, thB, th1, idf2, q);
}
// n-th term of nE(idf1, idf2, thB, th1) (src/glaIntSup.jl:239-281), weight included
__device__ Z n_e_term(int idf1, int idf2, double thB, double th1, int n, const Tri6& t, const Consts& q) {
  if (idf1 == 1 || idf1 == 2) {
    double s1, c1;
    sincos(th1, &s1, &c1);
    const double gam = (s1 + S3 * c1 - tan(thB)) / (s1 + S3 * c1 + tan(thB));
    const Z a = int_ne(n, 1, gam, thB, th1, t, idf2, q), b = int_ne(n, 2, gam, thB, th1, t, idf2, q);
    return zsc(zadd(zsc(b, 0.5), zsc(zsub(a, b), gam * 0.5)), q.w[n]);
  } else if (idf1 == 3) {
    const double gam = S3 / tan(th1);
    const Z a = int_ne(n, 1, gam, thB, th1, t, idf2, q), b = int_ne(n, 3, gam, thB, th1, t, idf2, q);
    return zsc(zadd(zsc(b, 0.5), zsc(zsub(a, b), 0.5 * gam)), q.w[n]);
  } else if (idf1 == 4) {
    return zsc(int_ne(n, 4, 1.0, thB, th1, t, idf2, q), 0.5 * q.w[n]);
  }
  return zsc(int_ne(n, 5, 1.0, thB, th1, t, idf2, q), 0.5 * q.w[n]);
}
__device__ inline void psi_lim_e(int idf, double& a, double& b) {
  if (idf == 1) {
    a = 0.0;
    b = PI / 3.0;
  } else if (idf == 2 || idf == 3) {
    a = PI / 3.0;
    b = PI / 2.0;
  } else if (idf == 4 || idf == 6) {
    a = PI / 2.0;
    b = PI;
  } else {
    a = 0.0;
    b = PI / 2.0;
  }
}
__device__ inline void eta_lim_e(int idf, double th, double& a, double& b) {
  double s, c;
  sincos(th, &s, &c);
  if (idf == 1) {
    a = 0.0;
    b = atan(s + S3 * c);
  } else if (idf == 2) {
    a = atan(s - S3 * c);
    b = atan(s + S3 * c);
  } else if (idf == 3 || idf == 4) {
    a = 0.0;
    b = atan(s - S3 * c);
  } else if (idf == 5) {
    a = atan(s + S3 * c);
    b = 0.5 * PI;
  } else {
    a = atan(s - S3 * c);
    b = 0.5 * PI;
  }
}
__device__ inline void spx_v(double xp[3][2], double t4, double t3, double tB, double t1) {
  double sB, cB, s1, c1, s3, c3;
  sincos(tB, &sB, &cB);
  sincos(t1, &s1, &c1);
  sincos(t3, &s3, &c3);
  spx(xp, t4 * c3 * c1 - 1.0, t4 * s3 * cB - 1.0, t4 * c3 * s1, t4 * s3 * sB);
}

// One weak item: a triangle pair and its integral type.
enum { W_S = 0, W_E = 1, W_VS = 2, W_VR = 3 };
struct WItem {
  int type;
  Tri6 t;
};

__device__ inline Z block_sum(Z v, Z* sh) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  const int wid = threadIdx.x / 32, lane = threadIdx.x % 32, nw = blockDim.x / 32;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  Z s{0, 0};
  if (threadIdx.x == 0)
    for (int k = 0; k < nw; ++k) s = zadd(s, sh[k]);  // fixed order
  return s;
}

// grid: blockIdx.x = outer index of the item's sum; partial[item][outer]
__global__ void __launch_bounds__(256) k_weak(const WItem* __restrict__ items, int item0, int n_outer,
                                              const Consts* __restrict__ qp, Z* __restrict__ partial) {
  __shared__ Consts q;
  __shared__ Z sh[8];
  __shared__ Tri6 t;
  __shared__ int type;
  const int item = item0 + blockIdx.y;
  if (threadIdx.x == 0) {
    q = *qp;
    t = items[item].t;
    type = items[item].type;
  }
  __syncthreads();
  const int n = q.ord;
  const int outer = blockIdx.x;
  Z acc{0, 0};
  double scale = 1.0;
  if (type == W_S) {
    // outer = (k*8 + idf-1)*3 + dir-1 ; inner (it, nn)
    const int dir = outer % 3 + 1, idf = (outer / 3) % 8 + 1, k = outer / 24;
    double pa, pb, ea, eb;
    psi_lim_s(idf, pa, pb);
    const double th = thf(pa, pb, q.x[k]);
    eta_lim_s(idf, th, ea, eb);
    for (int p = threadIdx.x; p < n * n; p += blockDim.x) {
      const int it = p / n, nn = p % n;
      const double thB = thf(ea, eb, q.x[it]);
      acc = zadd(acc, zsc(n_s_term(dir, idf, th, thB, nn, t, q), q.w[it]));
    }
    scale = 0.25 * q.w[k] * (pb - pa) * (eb - ea) * sin(th);
  } else if (type == W_E) {
    const int idf = outer % 6 + 1, k = outer / 6;
    double pa, pb, ea, eb;
    psi_lim_e(idf, pa, pb);
    const double thB = thf(pa, pb, q.x[k]);
    eta_lim_e(idf, thB, ea, eb);
    for (int p = threadIdx.x; p < n * n; p += blockDim.x) {
      const int it = p / n, nn = p % n;
      const double thA = thf(ea, eb, q.x[it]);
      const Z v = zadd(n_e_term(idf, 1, thA, thB, nn, t, q), n_e_term(idf, -1, thA, thB, nn, t, q));
      acc = zadd(acc, zsc(v, q.w[it] * cos(thA)));
    }
    scale = 0.25 * q.w[k] * (pb - pa) * (eb - ea);
  } else {
    const bool sng = type == W_VS;
    const int i3 = outer;
    for (int p = threadIdx.x; p < n * n; p += blockDim.x) {
      const int i2 = p / n, i1 = p % n;
      double xp[3][2];
      const double tA = thf(0.0, PI / 3.0, q.x[i1]);
      const double LA = 2.0 * S3 / (sin(tA) + S3 * cos(tA));
      const double tB = thf(0.0, PI / 3.0, q.x[i2]);
      const double LB = 2.0 * S3 / (sin(tB) + S3 * cos(tB));
      const double at = atan(LB / LA);
      const double tC = thf(0.0, at, q.x[i3]);
      double sC, cC, sD, cD;
      sincos(tC, &sC, &cC);
      const double tD = thf(at, PI / 2.0, q.x[i3]);
      sincos(tD, &sD, &cD);
      Z vc{0, 0}, vd{0, 0};
      for (int a = 0; a < n; ++a) {
        const double tx = thf(0.0, LA / cC, q.x[a]);
        spx_v(xp, tx, tC, tB, tA);
        const double d = dist6(t, xp);
        vc = zadd(vc, zsc(sng ? scl_ego_n(d, q.f) : scl_ego(d, q.f), q.w[a] * (tx * tx * tx)));
      }
      for (int a = 0; a < n; ++a) {
        const double tx = thf(0.0, LB / sD, q.x[a]);
        spx_v(xp, tx, tD, tB, tA);
        const double d = dist6(t, xp);
        vd = zadd(vd, zsc(sng ? scl_ego_n(d, q.f) : scl_ego(d, q.f), q.w[a] * (tx * tx * tx)));
      }
      const Z term = zadd(zsc(zsub(zsc(vc, LA * sC), zsc(vd, LB * cD)), at), zsc(vd, 0.5 * PI * LB * cD));
      acc = zadd(acc, zsc(term, q.w[i1] * q.w[i2] * q.w[i3]));
    }
  }
  const Z s = block_sum(acc, sh);
  if (threadIdx.x == 0) partial[(size_t)item * n_outer + outer] = zsc(s, scale);
}

__device__ inline double cross_norm(const double a[3], const double b[3], const double c[3]) {
  const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
  return sqrt(x * x + y * y + z * z);
}

// per item: fixed-order sum of its partials times the Jacobian factor
__global__ void k_weak_reduce(const WItem* __restrict__ items, int nitems, const int* __restrict__ nout,
                              const Z* __restrict__ partial, int stride, Z* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitems) return;
  Z s{0, 0};
  for (int k = 0; k < nout[i]; ++k) s = zadd(s, partial[(size_t)i * stride + k]);
  const Tri6& t = items[i].t;
  double jac;
  if (items[i].type == W_S) {
    const double u[3] = {t.r[0][0] - t.r[1][0], t.r[0][1] - t.r[1][1], t.r[0][2] - t.r[1][2]};
    const double v[3] = {t.r[2][0] - t.r[0][0], t.r[2][1] - t.r[0][1], t.r[2][2] - t.r[0][2]};
    const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
    jac = (x * x + y * y + z * z) / 12.0;
  } else {
    jac = cross_norm(t.r[0], t.r[1], t.r[2]) * cross_norm(t.r[3], t.r[4], t.r[5]) / 12.0;
    if (items[i].type != W_E) jac *= PI * PI / 144.0;
  }
  out[i] = zsc(s, jac);
}

// closed-form static parts (src/glaInt.jl:410-488)
__device__ Z r_srf_slf(double la, double lb, Z f) {
  const double s1 = sqrt(la * la + lb * lb), s4 = sqrt(la * la + 4 * lb * lb);
  const double t =
      8 * la * la * la + 8 * lb * lb * lb - 8 * la * la * s1 - 8 * lb * lb * s1 -
      3 * la * la * lb *
          (2 * log(la) + 2 * log(la + lb - s1) + log(s1 - lb) - 5 * log(lb + s1) - 2 * log(lb - la + s1) -
           2 * log(la + 2 * lb - s4) + log(s4 - 2 * lb) + 2 * log(la - 2 * lb + s4) + log(2 * lb + s4) +
           2 * log(2 * lb - la + s4) - 2 * log(la + 2 * lb + s4)) +
      6 * la * lb * lb *
          (log(64.0) + 4 * log(lb) + 2 * log(s1 - la) + 3 * log(la + s1) - 3 * log(s4 - la) -
           3 * log(sqrt(la * la * la * la + 5 * la * la * lb * lb + 4 * lb * lb * lb * lb) + la * (s1 - la - s4)));
  return zsc(zdiv(Z{1.0, 0.0}, zsc(zmul(f, f), 48.0 * PI)), t);
}
__device__ Z r_srf_edg_crn(double la, double lb, double lc, Z f) {
  const double sab = sqrt(la * la + lb * lb + lc * lc), sbc = sqrt(lb * lb + lc * lc);
  const double t =
      8 * lb * lc * sbc - 8 * lb * lc * sab - 12 * la * la * la * atan(1.0 / (la * lc / (la * la + lb * lb - lb * sab))) +
      12 * la * la * la * atan(la / lc) - 12 * la * lc * lc * atan(la * lb / (lc * sab)) -
      12 * la * lb * lb * atan(la * lc / (lb * sab)) - 16 * la * la * la * atan(lb * lc / (la * sab)) +
      6 * lc * lc * lc * atanh(lb / sbc) - 6 * lc * (la * la + lc * lc) * atanh(lb / sab) -
      15 * la * la * lc * log(la * la + lc * lc) - lc * lc * lc * log(la * la + lc * lc) +
      2 * lc * lc * lc * log(lc / (lb + sbc)) + 6 * la * la * lc * log(sab - lb) + 24 * la * la * lc * log(sab + lb) +
      2 * lc * lc * lc * log(sab + lb) +
      6 * la * lb *
          (-2 * la * log(la * la + lb * lb) - lc * log((lb * lb + lc * lc) * (sab - la)) + 3 * lc * log(la + sab) +
           la * log(sab - lc) + 3 * la * log(sab + lc)) +
      2 * lb * lb * lb * (log((sab - lc) / (lc + sab)) + log(1 + (2 * lc * (lc + sbc)) / (lb * lb)));
  return zsc(zdiv(Z{1.0, 0.0}, zsc(zmul(f, f), 48.0 * PI)), t);
}
__device__ Z r_srf_edg_flt(double la, double lb, Z f) {
  const double s1 = sqrt(la * la + lb * lb), s4 = sqrt(la * la + 4 * lb * lb);
  const double p1 = -la * la * la + 2 * lb * lb * (3 * lb + s1 - 2 * s4) + la * la * (2 * s1 - s4);
  const double p2 =
      la * lb *
      (lb * (-62 * log(2.0) - 5 * log(-la + s1) + 4 * log(8 * lb * lb * (-la + s1)) - 33 * log(la + s1) +
             17 * log(-la + s4) - 24 * log(lb * (-la + s4)) + 57 * log(la + s4)) +
       4 * la *
           (-8 * asinh(lb / la) + 6 * asinh(2 * lb / la) + 6 * atanh(lb / s1) + 12 * log(la) - 13 * log(-lb + s1) +
            log((-lb + s1) / la) + log(la / (lb + s1)) - 7 * log(lb + s1) - 2 * log((lb + s1) / la) -
            3 * log(-(((lb + s1) * (2 * lb - s4)) / (la * la))) - 3 * log((-lb + s1) / (-2 * lb + s4)) +
            11 * log(-2 * lb + s4) - 3 * log((lb + s1) / (2 * lb + s4)) + log(2 * lb + s4) +
            9 * log((2 * lb + s4) / (lb + s1)) - 2 * log(la * la + 2 * lb * (lb - s1))));
  return zadd(zsc(zdiv(Z{1.0, 0.0}, zsc(zmul(f, f), 12.0 * PI)), p1), Z{p2 / (64.0 * PI), 0.0});
}

// wS[3], wE[9], wV[6] from the item sums (layout fixed by weak_items) and the
// closed forms, scaled by inv = 1/prod(scl) (src/glaInt.jl:75-262, glaGen.jl:115-121)
__global__ void k_weak_combine(const Z* __restrict__ it, const double* __restrict__ scl, double inv, Z f,
                               Z* __restrict__ w /* 18 scaled */, Z* __restrict__ wraw /* 18 unscaled */) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double s1 = scl[0], s2 = scl[1], s3 = scl[2];
  // items: per dir d (0: dir 3, 1: dir 2, 2: dir 1) -> S block 8 items, E block 16, V block 12
  auto sdir = [&](int b) {  // wekSDir
    const Z* p = it + b * 36;
    Z a = zadd(zadd(zadd(p[0], p[1]), p[2]), p[3]);
    Z c = zadd(zadd(zadd(p[4], p[5]), p[6]), p[7]);
    return zsc(zadd(a, c), 0.5);
  };
  auto edir = [&](int b, int k) {  // wekEDir value k
    const Z* p = it + b * 36 + 8 + 4 * k;
    return zadd(zadd(zadd(p[0], p[1]), p[2]), p[3]);
  };
  auto vdir = [&](int b, int k) {  // wekVDir value k
    const Z* p = it + b * 36 + 24 + 4 * k;
    return zadd(zadd(zadd(p[0], p[1]), p[2]), p[3]);
  };
  Z r[18];
  r[0] = zadd(sdir(0), r_srf_slf(s2, s3, f));
  r[1] = zadd(sdir(1), r_srf_slf(s1, s3, f));
  r[2] = zadd(sdir(2), r_srf_slf(s1, s2, f));
  const Z xxY = zadd(edir(0, 0), r_srf_edg_flt(s3, s2, f)), xxZ = zadd(edir(0, 2), r_srf_edg_flt(s2, s3, f));
  const Z xyA = zadd(edir(0, 1), r_srf_edg_crn(s3, s2, s1, f)), xzA = zadd(edir(0, 3), r_srf_edg_crn(s2, s3, s1, f));
  const Z yyZ = zadd(edir(1, 0), r_srf_edg_flt(s1, s3, f)), yyX = zadd(edir(1, 2), r_srf_edg_flt(s3, s1, f));
  const Z yzA = zadd(edir(1, 1), r_srf_edg_crn(s1, s3, s2, f)), xyB = zadd(edir(1, 3), r_srf_edg_crn(s3, s2, s1, f));
  const Z zzX = zadd(edir(2, 0), r_srf_edg_flt(s2, s1, f)), zzY = zadd(edir(2, 2), r_srf_edg_flt(s1, s2, f));
  const Z xzB = zadd(edir(2, 1), r_srf_edg_crn(s2, s3, s1, f)), yzB = zadd(edir(2, 3), r_srf_edg_crn(s1, s3, s2, f));
  r[3] = xxY;
  r[4] = xxZ;
  r[5] = yyX;
  r[6] = yyZ;
  r[7] = zzX;
  r[8] = zzY;
  r[9] = zsc(zadd(xyA, xyB), 0.5);
  r[10] = zsc(zadd(xzA, xzB), 0.5);
  r[11] = zsc(zadd(yzA, yzB), 0.5);
  r[12] = vdir(0, 0);
  r[13] = vdir(1, 0);
  r[14] = vdir(2, 0);
  r[15] = zsc(zadd(vdir(0, 1), vdir(1, 2)), 0.5);
  r[16] = zsc(zadd(vdir(0, 2), vdir(2, 1)), 0.5);
  r[17] = zsc(zadd(vdir(1, 1), vdir(2, 2)), 0.5);
  for (int k = 0; k < 18; ++k) {
    wraw[k] = r[k];
    w[k] = zsc(r[k], inv);
  }
}

// ------------------------------------------------------- face-pair cubature
// Faces yzL yzU xzL xzU xyL xyU (cubFac, src/glaInt.jl:296-311); vertex 0,
// and the two edge vectors (v1 - v0, v3 - v0) used by cubVecAltAdp.
struct Faces {
  double o[6][3], a[6][3], b[6][3];
};
struct PairGeo {
  Faces tf, sf;
  double scale[36];  // srfScl (src/glaInt.jl:271-294)
  Z f;
};

// the 24 face pairs (0-based fp = 6*ft + fs) that feed the six stored
// components (xx, yy, zz, xy, xz, yz) of srfSum! (src/glaGen.jl:531-555)
__constant__ int c_pairs[24] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 14, 15, 16, 17, 20, 21, 22, 23, 28, 29, 34, 35};

__device__ inline void face_val(const PairGeo& G, int ft, int fs, const double sep[3], const double u[4],
                                double out[2]) {
  double v[3];
  for (int d = 0; d < 3; ++d) {
    const double tv = G.tf.o[ft][d] + u[2] * G.tf.a[ft][d] + u[3] * G.tf.b[ft][d];
    const double sv = G.sf.o[fs][d] + u[0] * G.sf.a[fs][d] + u[1] * G.sf.b[fs][d];
    v[d] = (tv - sv) + sep[d];
  }
  const Z z = scl_ego(sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), G.f);
  out[0] = z.x;
  out[1] = z.y;
}

struct Region {
  double c[4], h[4], val[2], err[2], errmax;
  int split;
};

constexpr double GL2 = 0.35856858280031809199064515390793749545;  // sqrt(9/70)
constexpr double GL4 = 0.94868329805051379959966806332981556011;  // sqrt(9/10)
constexpr double GL5 = 0.68824720161168529772162873429362352512;  // sqrt(9/19)

// point p of the 57-point Genz-Malik rule: offsets in units of the half-widths
__device__ inline void gm_point(int p, double off[4]) {
  off[0] = off[1] = off[2] = off[3] = 0.0;
  if (p == 0) return;
  if (p <= 16) {  // 1 + 4*i + k, k: -l2, +l2, -l4, +l4
    const int q = p - 1, i = q / 4, k = q % 4;
    off[i] = (k < 2 ? GL2 : GL4) * ((k & 1) ? 1.0 : -1.0);
    return;
  }
  if (p <= 40) {
    const int q = p - 17, pr = q / 4;
    const int pi[6] = {0, 0, 0, 1, 1, 2}, pk[6] = {1, 2, 3, 2, 3, 3};
    off[pi[pr]] = GL4 * ((q & 1) ? 1.0 : -1.0);
    off[pk[pr]] = GL4 * ((q & 2) ? 1.0 : -1.0);
    return;
  }
  const int m = p - 41;
  for (int i = 0; i < 4; ++i) off[i] = GL5 * (((m >> i) & 1) ? 1.0 : -1.0);
}
__device__ inline double gm_w7(int p) {
  const double n = 4.0;
  if (p == 0) return (12824.0 - 9120.0 * n + 400.0 * n * n) / 19683.0;
  if (p <= 16) return ((p - 1) % 4 < 2) ? 980.0 / 6561.0 : (1820.0 - 400.0 * n) / 19683.0;
  if (p <= 40) return 200.0 / 19683.0;
  return 6859.0 / 19683.0 / 16.0;
}
__device__ inline double gm_w5(int p) {
  const double n = 4.0;
  if (p == 0) return (729.0 - 950.0 * n + 50.0 * n * n) / 729.0;
  if (p <= 16) return ((p - 1) % 4 < 2) ? 245.0 / 486.0 : (265.0 - 100.0 * n) / 1458.0;
  if (p <= 40) return 25.0 / 729.0;
  return 0.0;
}

// Evaluate the rule on nreg (1 or 2) regions with the whole warp.
__device__ void gm_eval(const PairGeo& G, int ft, int fs, const double sep[3], Region* R, int nreg,
                        double (*fv)[57][2]) {
  const int lane = threadIdx.x & 31;
  for (int p = lane; p < 57 * nreg; p += 32) {
    const int r = p / 57, pp = p - r * 57;
    double off[4], u[4];
    gm_point(pp, off);
    for (int i = 0; i < 4; ++i) u[i] = R[r].c[i] + off[i] * R[r].h[i];
    face_val(G, ft, fs, sep, u, fv[r][pp]);
  }
  __syncwarp();
  if (lane < nreg) {
    Region& Q = R[lane];
    const double ratio = (GL2 * GL2) / (GL4 * GL4);
    double s7[2] = {0, 0}, s5[2] = {0, 0};
    for (int p = 0; p < 57; ++p) {
      const double a = gm_w7(p), b = gm_w5(p);
      s7[0] += a * fv[lane][p][0];
      s7[1] += a * fv[lane][p][1];
      s5[0] += b * fv[lane][p][0];
      s5[1] += b * fv[lane][p][1];
    }
    double vol = 1.0;
    for (int i = 0; i < 4; ++i) vol *= 2.0 * Q.h[i];
    Q.errmax = 0;
    for (int j = 0; j < 2; ++j) {
      Q.val[j] = vol * s7[j];
      Q.err[j] = fabs(vol * s5[j] - vol * s7[j]);
      if (Q.err[j] > Q.errmax) Q.errmax = Q.err[j];
    }
    int sd = 0;
    double md = 0;
    for (int i = 0; i < 4; ++i) {
      double d = 0;
      const double* f0 = fv[lane][0];
      for (int j = 0; j < 2; ++j) {
        const double fa = fv[lane][1 + 4 * i][j], fb = fv[lane][2 + 4 * i][j];
        const double fc = fv[lane][3 + 4 * i][j], fd = fv[lane][4 + 4 * i][j];
        d += fabs(fa + fb - 2 * f0[j] - ratio * (fc + fd - 2 * f0[j]));
      }
      if (d > md) {
        md = d;
        sd = i;
      }
    }
    Q.split = sd;
  }
  __syncwarp();
}

// heap in global memory (lane 0 only)
__device__ void hp_push(Region* H, int& nh, const Region& r) {
  int i = nh++;
  H[i] = r;
  while (i > 0) {
    const int p = (i - 1) / 2;
    if (H[p].errmax >= H[i].errmax) break;
    const Region t = H[p];
    H[p] = H[i];
    H[i] = t;
    i = p;
  }
}
__device__ Region hp_pop(Region* H, int& nh) {
  const Region top = H[0];
  H[0] = H[--nh];
  int i = 0;
  for (;;) {
    const int l = 2 * i + 1, r = l + 1;
    int m = i;
    if (l < nh && H[l].errmax > H[m].errmax) m = l;
    if (r < nh && H[r].errmax > H[m].errmax) m = r;
    if (m == i) break;
    const Region t = H[m];
    H[m] = H[i];
    H[i] = t;
    i = m;
  }
  return top;
}

// hcubature(2, f, 0, 1; reltol, abstol, INDIVIDUAL) with the warp; returns
// false (and sets *err) when the heap capacity or iteration cap is exceeded.
__device__ bool cubature(const PairGeo& G, int ft, int fs, const double sep[3], Region* heap, int cap,
                         Region* reg2, double (*fv)[57][2], double out[2], int* errflag) {
  const int lane = threadIdx.x & 31;
  if (lane == 0) {
    for (int i = 0; i < 4; ++i) {
      reg2[0].c[i] = 0.5;
      reg2[0].h[i] = 0.5;
    }
  }
  __syncwarp();
  gm_eval(G, ft, fs, sep, reg2, 1, fv);
  __shared__ int s_done[8];
  const int wid = threadIdx.x >> 5;
  double tv[2] = {reg2[0].val[0], reg2[0].val[1]}, te[2] = {reg2[0].err[0], reg2[0].err[1]};
  int nh = 0;
  if (lane == 0) hp_push(heap, nh, reg2[0]);
  bool ok = true;
  for (int it = 0;; ++it) {
    if (lane == 0) {
      int conv = 1;
      for (int j = 0; j < 2; ++j)
        if (te[j] > CUB_ABSTOL && te[j] > fabs(tv[j]) * CUB_RELTOL) conv = 0;
      int stop = conv;
      if (!conv && (nh + 2 > cap || it > 4000000)) {
        if (errflag) atomicOr(errflag, 1);  // else the caller defers the item
        stop = 2;
      }
      if (!stop) {
        const Region R = hp_pop(heap, nh);
        for (int j = 0; j < 2; ++j) {
          tv[j] -= R.val[j];
          te[j] -= R.err[j];
        }
        reg2[0] = R;
        reg2[1] = R;
        const int d = R.split;
        reg2[0].h[d] = reg2[1].h[d] = R.h[d] * 0.5;
        reg2[0].c[d] = R.c[d] - reg2[0].h[d];
        reg2[1].c[d] = R.c[d] + reg2[0].h[d];
      }
      s_done[wid] = stop;
    }
    __syncwarp();
    const int stop = s_done[wid];
    __syncwarp();
    if (stop) {
      ok = stop == 1;
      break;
    }
    gm_eval(G, ft, fs, sep, reg2, 2, fv);
    if (lane == 0) {
      for (int j = 0; j < 2; ++j) {
        tv[j] += reg2[0].val[j] + reg2[1].val[j];
        te[j] += reg2[0].err[j] + reg2[1].err[j];
      }
      hp_push(heap, nh, reg2[0]);
      hp_push(heap, nh, reg2[1]);
    }
    __syncwarp();
  }
  if (lane == 0) {
    out[0] = out[1] = 0;
    for (int i = 0; i < nh; ++i) {
      out[0] += heap[i].val[0];
      out[1] += heap[i].val[1];
    }
  }
  __syncwarp();
  return ok;
}

// srfSum! restricted to the six stored components, accumulated in the
// reference's order; s = the 36 srfMat values (unused entries zero)
__device__ inline void srf_sum6(const Z* s_, Z out[6]) {
  const Z* s = s_ - 1;  // 1-based like srfMat
  // xx = s15 - s16 - s21 + s22 + s29 - s30 - s35 + s36
  out[0] = zadd(zsub(zsub(zadd(zadd(zsub(zsub(s[15], s[16]), s[21]), s[22]), s[29]), s[30]), s[35]), s[36]);
  // yy = s1 - s2 - s7 + s8 + s29 - s30 - s35 + s36
  out[1] = zadd(zsub(zsub(zadd(zadd(zsub(zsub(s[1], s[2]), s[7]), s[8]), s[29]), s[30]), s[35]), s[36]);
  // zz = s1 - s2 - s7 + s8 + s15 - s16 - s21 + s22
  out[2] = zadd(zsub(zsub(zadd(zadd(zsub(zsub(s[1], s[2]), s[7]), s[8]), s[15]), s[16]), s[21]), s[22]);
  // xy = -s3 + s4 + s9 - s10
  out[3] = zsub(zadd(zadd(Z{-s[3].x, -s[3].y}, s[4]), s[9]), s[10]);
  // xz = -s5 + s6 + s11 - s12
  out[4] = zsub(zadd(zadd(Z{-s[5].x, -s[5].y}, s[6]), s[11]), s[12]);
  // yz = -s17 + s18 + s23 - s24
  out[5] = zsub(zadd(zadd(Z{-s[17].x, -s[17].y}, s[18]), s[23]), s[24]);
}

// Far offsets: warp per offset, persistent over a work counter.
//   mode 0 (self):  offset (ix,iy,iz) of the Toeplitz field, skipped when all
//                   indices <= 1 (near); sep = index * pitch;
//   mode 1 (ext):   circulant index; split indices zero; touching offsets are
//                   left to the contact kernel; sep from the grdSel tables.
struct FarParams {
  int mode;
  int n[3];                 // extents of the output field
  int64_t nitems;
  const double* sep[3];     // per-axis separation tables
  int split[3];             // ext: 0-based split index (trg cel), self: -1
  double touch[3];          // ext contact threshold per axis (cntTol + (sT+sS)/2), or -1
  Z* out;                   // [6][n2][n1][n0]
  Region* heap;             // per-warp heaps
  int cap;
  unsigned long long* counter;
  int* errflag;
  // overflow handling: the first pass (list == nullptr) appends items whose
  // region heap overflowed to ovf_list and leaves them to a second pass over
  // that list with larger heaps (list != nullptr, *list_count items)
  const int64_t* list;
  const unsigned long long* list_count;
  int64_t* ovf_list;
  unsigned long long* ovf_count;
};

__global__ void __launch_bounds__(128) k_far(const FarParams p, const PairGeo* __restrict__ gp) {
  __shared__ PairGeo G;
  __shared__ Region reg2s[4][2];
  __shared__ double fvs[4][2][57][2];
  __shared__ Z srf[4][36];
  __shared__ unsigned long long s_item[4];
  for (int i = threadIdx.x; i < (int)(sizeof(PairGeo) / sizeof(double)); i += blockDim.x)
    reinterpret_cast<double*>(&G)[i] = reinterpret_cast<const double*>(gp)[i];
  __syncthreads();
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + wid;
  Region* heap = p.heap + gw * p.cap;
  const int64_t plane = (int64_t)p.n[0] * p.n[1], vol = plane * p.n[2];
  const int64_t nitems = p.list ? (int64_t)*p.list_count : p.nitems;
  for (;;) {
    if (lane == 0) s_item[wid] = atomicAdd(p.counter, 1ull);
    __syncwarp();
    const unsigned long long ticket = s_item[wid];
    __syncwarp();
    if ((int64_t)ticket >= nitems) break;
    const unsigned long long item = p.list ? (unsigned long long)p.list[ticket] : ticket;
    const int ix = (int)(item % p.n[0]), iy = (int)((item / p.n[0]) % p.n[1]), iz = (int)(item / plane);
    const int id[3] = {ix, iy, iz};
    bool skip = false, zero = false;
    double sep[3];
    for (int d = 0; d < 3; ++d) sep[d] = p.sep[d][id[d]];
    if (p.mode == 0) {
      skip = !(ix > 1 || iy > 1 || iz > 1);
    } else {
      for (int d = 0; d < 3; ++d) zero |= id[d] == p.split[d];
      if (!zero && p.touch[0] > 0) {
        bool t = true;
        for (int d = 0; d < 3; ++d) t &= fabs(sep[d]) < p.touch[d];
        skip = t;
      }
    }
    if (skip) continue;
    const int64_t o = ((int64_t)iz * p.n[1] + iy) * p.n[0] + ix;
    if (zero) {
      if (lane < 6) p.out[lane * vol + o] = Z{0, 0};
      continue;
    }
    for (int k = lane; k < 36; k += 32) srf[wid][k] = Z{0, 0};
    __syncwarp();
    bool ok = true;
    for (int k = 0; k < 24 && ok; ++k) {
      const int fp = c_pairs[k];
      double v[2];
      ok = cubature(G, fp / 6, fp % 6, sep, heap, p.cap, reg2s[wid], fvs[wid], v, p.ovf_list ? nullptr : p.errflag);
      if (lane == 0) srf[wid][fp] = zsc(Z{v[0], v[1]}, G.scale[fp]);
      __syncwarp();
    }
    if (!ok) {
      if (lane == 0 && p.ovf_list) p.ovf_list[atomicAdd(p.ovf_count, 1ull)] = (int64_t)item;
      __syncwarp();
      continue;
    }
    if (lane == 0) {
      Z c6[6];
      srf_sum6(srf[wid], c6);
      for (int c = 0; c < 6; ++c) p.out[c * vol + o] = c6[c];
    }
    __syncwarp();
  }
}

// Near offsets of a self operator (egoFunSng!, src/glaGen.jl:350-528): one
// warp per offset (px, py, pz) in {0,1}^3 within the volume; corrected pairs
// from the weak values, the others by cubature.
__constant__ signed char c_sng_cor[8][6][6];
__constant__ signed char c_sng_mask[8][6][6];

struct NearParams {
  int n[3];
  int cases[8];  // egoFunSng! case per offset (x fastest), -1 = every pair by cubature
  const double* sep[3];
  const Z* weak;  // 18 scaled weak values
  Z* out;         // toe [6][...]
  Region* heap;
  int cap;
  int* errflag;
};

__global__ void __launch_bounds__(32) k_near(const NearParams p, const PairGeo* __restrict__ gp) {
  __shared__ PairGeo G;
  __shared__ Region reg2[2];
  __shared__ double fv[2][57][2];
  __shared__ Z srf[36];
  for (int i = threadIdx.x; i < (int)(sizeof(PairGeo) / sizeof(double)); i += blockDim.x)
    reinterpret_cast<double*>(&G)[i] = reinterpret_cast<const double*>(gp)[i];
  __syncthreads();
  const int b = blockIdx.x;
  const int px = b & 1, py = (b >> 1) & 1, pz = (b >> 2) & 1;
  if (px >= p.n[0] || py >= p.n[1] || pz >= p.n[2]) return;
  const int cs = p.cases[b];
  const int lane = threadIdx.x;
  Region* heap = p.heap + (int64_t)b * p.cap;
  const double sep[3] = {p.sep[0][px], p.sep[1][py], p.sep[2][pz]};
  for (int k = lane; k < 36; k += 32) srf[k] = Z{0, 0};
  __syncwarp();
  for (int fp = 0; fp < 36; ++fp) {
    const int a = fp / 6, c = fp % 6;
    const int m = cs < 0 ? 0 : c_sng_mask[cs][a][c];
    if (m) {
      if (lane == 0) {
        const int code = c_sng_cor[cs][a][c];
        srf[fp] = code == 0 ? Z{0, 0} : code < 10 ? p.weak[code - 1] : code < 20 ? p.weak[3 + code - 11]
                                                                                  : p.weak[12 + code - 21];
      }
    } else {
      double v[2];
      cubature(G, a, c, sep, heap, p.cap, reg2, fv, v, p.errflag);
      if (lane == 0) srf[fp] = zsc(Z{v[0], v[1]}, G.scale[fp]);
    }
    __syncwarp();
  }
  if (lane == 0) {
    Z c6[6];
    srf_sum6(srf, c6);
    const int64_t vol = (int64_t)p.n[0] * p.n[1] * p.n[2];
    const int64_t o = ((int64_t)pz * p.n[1] + py) * p.n[0] + px;
    for (int c = 0; c < 6; ++c) p.out[c * vol + o] = c6[c];
  }
}

// identity (src/glaGen.jl:128-130) and egoToeCrc! (src/glaGen.jl:143-163):
// toe [6][N] -> circulant crc [6][2N]; off-diagonal signs flip on mirrored axes
__global__ void k_embed(const Z* __restrict__ toe, int nx, int ny, int nz, Z idsub, Z* __restrict__ crc) {
  const int64_t Px = 2 * nx, Py = 2 * ny, Pz = 2 * nz, vol = Px * Py * Pz, tv = (int64_t)nx * ny * nz;
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < vol; o += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(o % Px), y = (int)((o / Px) % Py), z = (int)(o / (Px * Py));
    const bool zero = x == nx || y == ny || z == nz;
    const int sx = x < nx ? x : 2 * nx - x, sy = y < ny ? y : 2 * ny - y, sz = z < nz ? z : 2 * nz - z;
    const double fx = x < nx ? 1.0 : -1.0, fy = y < ny ? 1.0 : -1.0, fz = z < nz ? 1.0 : -1.0;
    const int64_t ti = ((int64_t)sz * ny + sy) * nx + sx;
    // components xx, yy, zz, xy, xz, yz
    const double sg[6] = {1.0, 1.0, 1.0, fx * fy, fx * fz, fy * fz};
    for (int c = 0; c < 6; ++c) {
      Z v = zero ? Z{0, 0} : zsc(toe[c * tv + ti], sg[c]);
      if (!zero && ti == 0 && c < 3) v = zsub(v, idsub);
      crc[c * vol + o] = v;
    }
  }
}

// egoCntOut! (src/glaGen.jl:250-306) for the touching offsets of an external
// circulant, from the contact self circulant ccnt [6][2*cc] of the contact
// volume (genCntVol, src/glaGen.jl:308-318)
struct CntParams {
  int n[3];       // circulant extents
  int split[3];
  const double* sep[3];
  double touch[3];
  double cscl[3];  // contact cell size
  int sspan[3], tspan[3];
  int cc[3];       // contact volume cells
  const Z* ccnt;
  Z* out;
};
__global__ void k_contact(const CntParams p) {
  const int64_t vol = (int64_t)p.n[0] * p.n[1] * p.n[2];
  const int64_t Pc[3] = {2LL * p.cc[0], 2LL * p.cc[1], 2LL * p.cc[2]};
  const int64_t cvol = Pc[0] * Pc[1] * Pc[2];
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < vol; o += (int64_t)gridDim.x * blockDim.x) {
    const int id[3] = {(int)(o % p.n[0]), (int)((o / p.n[0]) % p.n[1]), (int)(o / ((int64_t)p.n[0] * p.n[1]))};
    bool split = false, touch = true;
    double sep[3];
    for (int d = 0; d < 3; ++d) {
      split |= id[d] == p.split[d];
      sep[d] = p.sep[d][id[d]];
      touch &= fabs(sep[d]) < p.touch[d];
    }
    if (split || !touch) continue;
    int64_t sL[3], sU[3], tL[3], tU[3];
    for (int d = 0; d < 3; ++d) {
      const double span = sep[d] / p.cscl[d];
      sL[d] = 1;
      sU[d] = p.sspan[d];
      tL[d] = (int64_t)nearbyint(span + p.sspan[d] / 2.0 - p.tspan[d] / 2.0) + 1;
      tU[d] = (int64_t)nearbyint(span + p.sspan[d] / 2.0 + p.tspan[d] / 2.0);
      if (tL[d] < 1) {
        const int64_t sh = (tL[d] < 0 ? -tL[d] : tL[d]) + 1;
        sL[d] += sh;
        sU[d] += sh;
        tU[d] += sh;
        tL[d] += sh;
      }
    }
    Z acc[6] = {};
    for (int64_t a = sL[2]; a <= sU[2]; ++a)
      for (int64_t b = sL[1]; b <= sU[1]; ++b)
        for (int64_t c = sL[0]; c <= sU[0]; ++c)
          for (int64_t aa = tL[2]; aa <= tU[2]; ++aa)
            for (int64_t bb = tL[1]; bb <= tU[1]; ++bb)
              for (int64_t cc = tL[0]; cc <= tU[0]; ++cc) {
                const int64_t t3[3] = {cc, bb, aa}, s3[3] = {c, b, a};
                int64_t ci[3];
                bool inb = true;
                for (int d = 0; d < 3; ++d) {
                  const int64_t v = t3[d] - s3[d];
                  ci[d] = v + (v < 0 ? 2LL * p.cc[d] : 0);
                  inb = inb && ci[d] >= 0 && ci[d] < Pc[d];
                }
                if (!inb) continue;
                const int64_t q = (ci[2] * Pc[1] + ci[1]) * Pc[0] + ci[0];
                for (int k = 0; k < 6; ++k) acc[k] = zadd(acc[k], p.ccnt[k * cvol + q]);
              }
    const double tot = (double)((tU[2] - tL[2] + 1) * (tU[1] - tL[1] + 1) * (tU[0] - tL[0] + 1));
    for (int k = 0; k < 6; ++k) p.out[k * vol + o] = Z{acc[k].x / tot, acc[k].y / tot};
  }
}

// ----------------------------------------------- FP64 3-D FFT of the circulant
// In-place forward FFT of `lines` lines of length P along one axis: element
// stride es, lines in tiles of TX contiguous (es > 1) or rows (es == 1).
__global__ void __launch_bounds__(512) k_fft_axis(double2* __restrict__ data, const AxisPlan* __restrict__ pl, int P,
                                                   const double2* __restrict__ tw, int64_t es, int64_t group_stride,
                                                   int TX, int64_t nlines_in_group, FDiv md) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* sm = reinterpret_cast<double2*>(smem_raw);
  // block -> (group g, tile t): lines l = t*TX + u, u < TX, of group g.  Line
  // l holds element i at base[l + i*es] (es > 1: lines contiguous) or at
  // base[l*P + i] (es == 1: rows).  Shared memory is [i][u].
  const int64_t ntiles = (nlines_in_group + TX - 1) / TX;
  const int64_t g = blockIdx.x / ntiles, t = blockIdx.x % ntiles;
  const int64_t l0 = t * TX;
  const int tmax = (int)((nlines_in_group - l0) < TX ? (nlines_in_group - l0) : TX);
  double2* base = data + g * group_stride;
  for (int q = threadIdx.x; q < TX * P; q += blockDim.x) {
    int i, u;
    if (es == 1) {  // coalesced along the row
      u = q / P;
      i = q - u * P;
    } else {
      i = (int)md.div((uint32_t)q);
      u = q - i * TX;
    }
    if (u < tmax) sm[i * TX + u] = es == 1 ? base[(l0 + u) * P + i] : base[l0 + u + (int64_t)i * es];
  }
  __syncthreads();
  auto lds = [=](int u, int i) -> double2 { return sm[i * TX + u]; };
  auto sts = [=](int u, int i, double2 v) { sm[i * TX + u] = v; };
  fft_run<double2, 4, false, true, true>(pl, TX, md, tw, lds, lds, sts, sts, true, true);
  for (int q = threadIdx.x; q < TX * P; q += blockDim.x) {
    int i, u;
    if (es == 1) {
      u = q / P;
      i = q - u * P;
    } else {
      i = (int)md.div((uint32_t)q);
      u = q - i * TX;
    }
    if (u < tmax) {
      const double2 v = sm[i * TX + u];
      if (es == 1)
        base[(l0 + u) * P + i] = v;
      else
        base[l0 + u + (int64_t)i * es] = v;
    }
  }
}

// parity-branch extraction + symmetric truncation + cast (src/glaMemSup.jl:138-156)
template <typename C>
__global__ void k_extract(const Z* __restrict__ crc, int Px, int Py, int Pz, int tx, int ty, int tz,
                          C* __restrict__ ker, int* __restrict__ nanflag) {
  const int64_t vol = (int64_t)Px * Py * Pz;
  const int64_t n = (int64_t)8 * tz * ty * tx * 6;
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
    int64_t q = o;  // o = ker_index(eo, iz, iy, c, ix, ...) = ((((py,pz) tz + iz) ty + iy) 6 + c) tx + ix) 2 + px
    const int px = (int)(q & 1);
    q >>= 1;
    const int ix = (int)(q % tx);
    q /= tx;
    const int c = (int)(q % 6);
    q /= 6;
    const int iy = (int)(q % ty);
    q /= ty;
    const int iz = (int)(q % tz);
    const int e = (int)(q / tz);
    const int py = (e >> 1) & 1, pz = e & 1;
    // the reference broadcasts a one-element branch slice over two entries
    const int hx = Px / 2 > 1 ? Px / 2 : 1, hy = Py / 2 > 1 ? Py / 2 : 1, hz = Pz / 2 > 1 ? Pz / 2 : 1;
    const int fx = 2 * (ix < hx ? ix : hx - 1) + px, fy = 2 * (iy < hy ? iy : hy - 1) + py,
              fz = 2 * (iz < hz ? iz : hz - 1) + pz;
    const Z v = crc[c * vol + ((int64_t)fz * Py + fy) * Px + fx];
    if (!isfinite(v.x) || !isfinite(v.y)) atomicOr(nanflag, 1);
    C r;
    r.x = (decltype(r.x))v.x;
    r.y = (decltype(r.y))v.y;
    ker[o] = r;
  }
}

}  // namespace kb
}  // namespace gila

// ======================================================================= host
namespace gila {
namespace kb {

// small rational helpers on top of Rat (exact grid arithmetic, converted to
// FP64 only at the end, as the reference's Rational -> Float64)
static Rat R(int64_t n, int64_t d = 1) { return rat(n, d); }
static Rat radd(Rat a, Rat b) { return rat(a.n * b.d + b.n * a.d, a.d * b.d); }
static Rat rsub(Rat a, Rat b) { return rat(a.n * b.d - b.n * a.d, a.d * b.d); }
static Rat rmul(Rat a, Rat b) { return rat(a.n * b.n, a.d * b.d); }
static Rat rdv(Rat a, Rat b) { return rat(a.n * b.d, a.d * b.n); }
static bool rlt(Rat a, Rat b) { return (__int128)a.n * b.d < (__int128)b.n * a.d; }
static bool rle(Rat a, Rat b) { return (__int128)a.n * b.d <= (__int128)b.n * a.d; }
static double rd(Rat a) { return (double)a.n / (double)a.d; }

struct HVol {  // GlaVol with start / stop of the grid (src/glaMem.jl:136-148)
  int64_t cel[3];
  Rat scl[3], org[3], grd[3], start[3], stop[3];
};
static HVol hvol(const Vol& v) {
  HVol h;
  for (int k = 0; k < 3; ++k) {
    h.cel[k] = v.cel[k];
    h.scl[k] = v.scl[k];
    h.org[k] = v.org[k];
    h.grd[k] = v.grd[k];
    const Rat half = R((v.cel[k] / 2) * 2 - (v.cel[k] % 2 == 0 ? 1 : 0), 2);
    const Rat brd = rmul(v.grd[k], half);
    h.start[k] = rsub(v.org[k], brd);
    h.stop[k] = radd(v.org[k], brd);
  }
  return h;
}

// Gauss-Legendre nodes (ascending) and weights by Newton iteration on P_n
static void gauss_legendre(int n, double* x, double* w) {
  for (int i = 0; i < n; ++i) {
    double z = cos(PI * (i + 0.75) / (n + 0.5)), dp = 0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = 0.0;
      for (int k = 1; k <= n; ++k) {
        const double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p2) / k;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      const double dz = p0 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = 0.0;
    for (int k = 1; k <= n; ++k) {
      const double p2 = p1;
      p1 = p0;
      p0 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p2) / k;
    }
    dp = n * (z * p0 - p1) / (z * z - 1.0);
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// faces of a cuboid (cubFac, src/glaInt.jl:296-311) as origin + two edges
static void faces(const Rat scl[3], Faces& F) {
  static const int sg[6][4][3] = {
      {{-1, -1, -1}, {-1, 1, -1}, {-1, 1, 1}, {-1, -1, 1}}, {{1, -1, -1}, {1, -1, 1}, {1, 1, 1}, {1, 1, -1}},
      {{-1, -1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, -1, -1}}, {{-1, 1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, 1, 1}},
      {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}}, {{-1, -1, 1}, {-1, 1, 1}, {1, 1, 1}, {1, -1, 1}}};
  for (int f = 0; f < 6; ++f)
    for (int d = 0; d < 3; ++d) {
      double v[4];
      for (int k = 0; k < 4; ++k) v[k] = rd(R(sg[f][k][d] * scl[d].n, 2 * scl[d].d));
      F.o[f][d] = v[0];
      F.a[f][d] = v[1] - v[0];
      F.b[f][d] = v[3] - v[0];
    }
}
// srfScl (src/glaInt.jl:271-294)
static void srf_scales(const Rat sT[3], const Rat sS[3], double out[36]) {
  for (int a = 0; a < 6; ++a) {
    const Rat src = a < 2 ? rmul(sS[1], sS[2]) : a < 4 ? rmul(sS[0], sS[2]) : rmul(sS[0], sS[1]);
    for (int b = 0; b < 6; ++b) out[a * 6 + b] = rd(rdv(src, b < 2 ? sT[0] : b < 4 ? sT[1] : sT[2]));
  }
}

// The weak-integral items of wekS / wekE / wekV in the order k_weak_combine
// expects: per direction (3, 2, 1): 8 wekSDir items, 16 wekEDir, 12 wekVDir.
static std::vector<WItem> weak_items(const double scl[3]) {
  std::vector<WItem> v;
  for (int b = 0; b < 3; ++b) {
    const int dir = 3 - b;
    double gx, gy, gz;
    if (dir == 1) {
      gx = scl[0];
      gy = scl[1];
      gz = scl[2];
    } else if (dir == 2) {
      gx = scl[2];
      gy = scl[0];
      gz = scl[1];
    } else {
      gx = scl[1];
      gy = scl[2];
      gz = scl[0];
    }
    double P[19][3];
    int k = 1;
    for (int zz = 0; zz < 2; ++zz)
      for (int yy = 0; yy < 3; ++yy)
        for (int xx = 0; xx < 3; ++xx, ++k) {
          P[k][0] = xx * gx;
          P[k][1] = yy * gy;
          P[k][2] = zz * gz;
        }
    auto add = [&](int type, int a, int bb, int c, int d, int e, int f) {
      WItem it;
      it.type = type;
      const int id[6] = {a, bb, c, d, e, f};
      for (int q = 0; q < 6; ++q)
        for (int r = 0; r < 3; ++r) it.t.r[q][r] = P[id[q]][r];
      v.push_back(it);
    };
    // wekSDir (src/glaInt.jl:88-114)
    add(W_S, 1, 2, 5, 1, 2, 5);
    add(W_S, 1, 5, 4, 1, 5, 4);
    add(W_E, 1, 2, 5, 1, 5, 4);
    add(W_E, 1, 5, 4, 1, 2, 5);
    add(W_S, 4, 1, 2, 4, 1, 2);
    add(W_S, 4, 2, 5, 4, 2, 5);
    add(W_E, 4, 1, 2, 4, 2, 5);
    add(W_E, 4, 2, 5, 4, 1, 2);
    // wekEDir (src/glaInt.jl:165-206)
    add(W_E, 1, 2, 5, 2, 3, 5);
    add(W_VS, 1, 2, 5, 3, 6, 5);
    add(W_VS, 1, 5, 4, 2, 3, 5);
    add(W_VS, 1, 5, 4, 3, 6, 5);
    add(W_E, 1, 2, 5, 2, 11, 5);
    add(W_VS, 1, 2, 5, 11, 14, 5);
    add(W_VS, 1, 5, 4, 2, 11, 5);
    add(W_VS, 1, 5, 4, 11, 14, 5);
    add(W_VS, 1, 2, 5, 4, 5, 7);
    add(W_VS, 1, 2, 5, 5, 8, 7);
    add(W_E, 1, 5, 4, 4, 5, 7);
    add(W_VS, 1, 5, 4, 5, 8, 7);
    add(W_VS, 1, 2, 5, 4, 5, 13);
    add(W_VS, 1, 2, 5, 5, 14, 13);
    add(W_E, 1, 5, 4, 4, 5, 13);
    add(W_VS, 1, 5, 4, 5, 14, 13);
    // wekVDir (src/glaInt.jl:236-262)
    add(W_VR, 1, 2, 5, 5, 6, 9);
    add(W_VR, 1, 2, 5, 5, 9, 8);
    add(W_VR, 1, 5, 4, 5, 6, 9);
    add(W_VR, 1, 5, 4, 5, 9, 8);
    add(W_VR, 1, 2, 5, 5, 17, 14);
    add(W_VR, 1, 2, 5, 5, 8, 17);
    add(W_VR, 1, 5, 4, 5, 17, 14);
    add(W_VR, 1, 5, 4, 5, 8, 17);
    add(W_VR, 1, 2, 5, 5, 15, 14);
    add(W_VR, 1, 2, 5, 5, 6, 15);
    add(W_VR, 1, 5, 4, 5, 15, 14);
    add(W_VR, 1, 5, 4, 5, 6, 15);
  }
  return v;
}

// egoFunSng! tables (src/glaGen.jl:370-509): 0 none, 1..3 wS, 11..19 wE, 21..26 wV
static const signed char SNG_COR[8][6][6] = {
    {{1, 0, 17, 17, 18, 18}, {0, 1, 17, 17, 18, 18}, {17, 17, 2, 0, 19, 19},
     {17, 17, 0, 2, 19, 19}, {18, 18, 19, 19, 3, 0}, {18, 18, 19, 19, 0, 3}},
    {{0, 1, 17, 17, 18, 18}, {0, 0, 0, 0, 0, 0}, {0, 17, 13, 0, 26, 26},
     {0, 17, 0, 13, 26, 26}, {0, 18, 26, 26, 15, 0}, {0, 18, 26, 26, 0, 15}},
    {{0, 12, 24, 24, 0, 18}, {0, 0, 0, 0, 0, 0}, {0, 24, 22, 0, 0, 26},
     {0, 24, 0, 22, 0, 26}, {0, 18, 26, 26, 0, 15}, {0, 0, 0, 0, 0, 0}},
    {{12, 0, 24, 24, 0, 18}, {0, 12, 24, 24, 0, 18}, {24, 24, 14, 0, 0, 19},
     {24, 24, 0, 14, 0, 19}, {18, 18, 19, 19, 0, 3}, {0, 0, 0, 0, 0, 0}},
    {{11, 0, 0, 17, 25, 25}, {0, 11, 0, 17, 25, 25}, {17, 17, 0, 2, 19, 19},
     {0, 0, 0, 0, 0, 0}, {25, 25, 0, 19, 16, 0}, {25, 25, 0, 19, 0, 16}},
    {{0, 11, 0, 17, 25, 25}, {0, 0, 0, 0, 0, 0}, {0, 17, 0, 13, 26, 26},
     {0, 0, 0, 0, 0, 0}, {0, 25, 0, 26, 23, 0}, {0, 25, 0, 26, 0, 23}},
    {{21, 0, 0, 24, 0, 25}, {0, 21, 0, 24, 0, 25}, {24, 24, 0, 14, 0, 19},
     {0, 0, 0, 0, 0, 0}, {25, 25, 0, 19, 0, 16}, {0, 0, 0, 0, 0, 0}},
    {{0, 21, 0, 24, 0, 25}, {0, 0, 0, 0, 0, 0}, {0, 24, 0, 22, 0, 26},
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

// egoFunSng! case of near offset (px, py, pz) in 1-based {1,2}^3, or -1
static int sng_case(int px, int py, int pz, const HVol& v) {
  const bool tx = !rlt(v.scl[0], v.grd[0]), ty = !rlt(v.scl[1], v.grd[1]), tz = !rlt(v.scl[2], v.grd[2]);
  if (px == 1 && py == 1 && pz == 1) return 0;
  if (px == 2 && py == 1 && pz == 1 && tx) return 1;
  if (px == 2 && py == 1 && pz == 2 && tx && tz) return 2;
  if (px == 1 && py == 1 && pz == 2 && tz) return 3;
  if (px == 1 && py == 2 && pz == 1 && ty) return 4;
  if (px == 2 && py == 2 && pz == 1 && tx && ty) return 5;
  if (px == 1 && py == 2 && pz == 2 && ty && tz) return 6;
  if (px == 2 && py == 2 && pz == 2 && tx && ty && tz) return 7;
  return -1;
}

// RAII for build scratch
struct DBuf {
  void* p = nullptr;
  ~DBuf() { cudaFree(p); }
};
#define KB_TRY(expr)                                              \
  do {                                                            \
    cudaError_t e__ = (expr);                                     \
    if (e__ != cudaSuccess) return ::gila::cuda_fail(e__, #expr); \
  } while (0)

struct Build {
  Ctx* ctx;
  cudaStream_t st;
  Z f;
  int ord;
  Consts* q_d = nullptr;  // in `keep`
  std::vector<DBuf*> keep;
  ~Build() {
    for (auto* b : keep) delete b;
  }
  // frees the buffers allocated after `mark` (the stream is synchronised
  // first: kernels in flight may still use them)
  void release_from(size_t mark) {
    if (keep.size() <= mark) return;
    cudaStreamSynchronize(st);
    while (keep.size() > mark) {
      delete keep.back();
      keep.pop_back();
    }
  }
  template <typename T>
  gila_status alloc(T** out, size_t n) {
    DBuf* b = new DBuf;
    keep.push_back(b);
    KB_TRY(dev_malloc(&b->p, n * sizeof(T) + 16));
    *out = static_cast<T*>(b->p);
    return GILA_OK;
  }
};

// weak values (18, scaled by 1/prod(scl)) for a cell of size scl; the
// unscaled values go to raw_out when given
static gila_status weak_values(Build& B, const Rat sclr[3], Z* w_d, Z* raw_out = nullptr) {
  const double scl[3] = {rd(sclr[0]), rd(sclr[1]), rd(sclr[2])};
  std::vector<WItem> items = weak_items(scl);
  const int n = (int)items.size(), ord = B.ord;
  WItem* it_d;
  gila_status s;
  if ((s = B.alloc(&it_d, items.size())) != GILA_OK) return s;
  KB_TRY(cudaMemcpyAsync(it_d, items.data(), items.size() * sizeof(WItem), cudaMemcpyHostToDevice, B.st));
  const int max_outer = 24 * ord;
  Z *part_d, *sums_d, *raw_d;
  int* nout_d;
  if ((s = B.alloc(&part_d, (size_t)n * max_outer)) != GILA_OK) return s;
  if ((s = B.alloc(&sums_d, n)) != GILA_OK) return s;
  if (raw_out)
    raw_d = raw_out;
  else if ((s = B.alloc(&raw_d, 18)) != GILA_OK)
    return s;
  if ((s = B.alloc(&nout_d, n)) != GILA_OK) return s;
  std::vector<int> nout(n);
  for (int i = 0; i < n; ++i) {
    const int t = items[i].type;
    nout[i] = t == W_S ? 24 * ord : t == W_E ? 6 * ord : ord;
  }
  KB_TRY(cudaMemcpyAsync(nout_d, nout.data(), n * sizeof(int), cudaMemcpyHostToDevice, B.st));
  // one launch per item (grid = the item's outer sum); items are independent
  for (int i = 0; i < n; ++i) {
    k_weak<<<dim3(nout[i], 1), 256, 0, B.st>>>(it_d, i, max_outer, B.q_d, part_d);
    KB_TRY(cudaGetLastError());
  }
  k_weak_reduce<<<(n + 127) / 128, 128, 0, B.st>>>(it_d, n, nout_d, part_d, max_outer, sums_d);
  KB_TRY(cudaGetLastError());
  double* scl_d;
  if ((s = B.alloc(&scl_d, 3)) != GILA_OK) return s;
  KB_TRY(cudaMemcpyAsync(scl_d, scl, sizeof(scl), cudaMemcpyHostToDevice, B.st));
  const double inv = rd(rdv(R(1), rmul(rmul(sclr[0], sclr[1]), sclr[2])));
  k_weak_combine<<<1, 32, 0, B.st>>>(sums_d, scl_d, inv, B.f, w_d, raw_d);
  KB_TRY(cudaGetLastError());
  return GILA_OK;
}

// Far pass over nitems with 512-region heaps, then the deferred items with
// 16384-region heaps on 128 warps.
static gila_status run_far(Build& B, FarParams fp, const PairGeo* g_d) {
  gila_status s;
  int nsm = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int64_t blocks = (int64_t)nsm * 4;
  const int64_t need = (fp.nitems + 3) / 4;
  if (blocks > need) blocks = need < 1 ? 1 : need;
  const int cap1 = 512, cap2 = 16384;
  Region* heap;
  if ((s = B.alloc(&heap, (size_t)blocks * 4 * cap1)) != GILA_OK) return s;
  unsigned long long* cnt;
  if ((s = B.alloc(&cnt, 3)) != GILA_OK) return s;
  KB_TRY(cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned long long), B.st));
  int64_t* ovf;
  if ((s = B.alloc(&ovf, (size_t)(fp.nitems > 0 ? fp.nitems : 1))) != GILA_OK) return s;
  fp.heap = heap;
  fp.cap = cap1;
  fp.counter = cnt;
  fp.list = nullptr;
  fp.list_count = nullptr;
  fp.ovf_list = ovf;
  fp.ovf_count = cnt + 1;
  k_far<<<(unsigned)blocks, 128, 0, B.st>>>(fp, g_d);
  KB_TRY(cudaGetLastError());
  Region* heap2;
  if ((s = B.alloc(&heap2, (size_t)32 * 4 * cap2)) != GILA_OK) return s;
  fp.heap = heap2;
  fp.cap = cap2;
  fp.counter = cnt + 2;
  fp.list = ovf;
  fp.list_count = cnt + 1;
  fp.ovf_list = nullptr;
  fp.ovf_count = nullptr;
  k_far<<<32, 128, 0, B.st>>>(fp, g_d);
  KB_TRY(cudaGetLastError());
  return GILA_OK;
}

// Self circulant crc [6][2N] of a volume (genEgoSlf!, src/glaGen.jl:38-53)
static gila_status self_circulant(Build& B, const HVol& v, Z* crc_d, int* err_d) {
  gila_status s;
  const int64_t nx = v.cel[0], ny = v.cel[1], nz = v.cel[2], V = nx * ny * nz;
  Z *toe_d, *w_d;
  if ((s = B.alloc(&toe_d, 6 * V)) != GILA_OK) return s;
  if ((s = B.alloc(&w_d, 18)) != GILA_OK) return s;
  if ((s = weak_values(B, v.scl, w_d)) != GILA_OK) return s;
  PairGeo G;
  faces(v.scl, G.tf);
  faces(v.scl, G.sf);
  srf_scales(v.scl, v.scl, G.scale);
  G.f = B.f;
  PairGeo* g_d;
  if ((s = B.alloc(&g_d, 1)) != GILA_OK) return s;
  KB_TRY(cudaMemcpyAsync(g_d, &G, sizeof(G), cudaMemcpyHostToDevice, B.st));
  double* sep_d[3];
  for (int d = 0; d < 3; ++d) {
    std::vector<double> sp(v.cel[d]);
    for (int64_t i = 0; i < v.cel[d]; ++i) sp[i] = rd(rmul(R(i), v.grd[d]));
    if ((s = B.alloc(&sep_d[d], sp.size())) != GILA_OK) return s;
    KB_TRY(cudaMemcpyAsync(sep_d[d], sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice, B.st));
  }
  // near offsets
  NearParams np;
  for (int d = 0; d < 3; ++d) {
    np.n[d] = (int)v.cel[d];
    np.sep[d] = sep_d[d];
  }
  for (int b = 0; b < 8; ++b) np.cases[b] = sng_case((b & 1) + 1, ((b >> 1) & 1) + 1, ((b >> 2) & 1) + 1, v);
  np.weak = w_d;
  np.out = toe_d;
  np.cap = 16384;
  np.errflag = err_d;
  Region* nheap;
  if ((s = B.alloc(&nheap, (size_t)8 * np.cap)) != GILA_OK) return s;
  np.heap = nheap;
  k_near<<<8, 32, 0, B.st>>>(np, g_d);
  KB_TRY(cudaGetLastError());
  // far offsets
  FarParams fp{};
  fp.mode = 0;
  for (int d = 0; d < 3; ++d) {
    fp.n[d] = (int)v.cel[d];
    fp.sep[d] = sep_d[d];
    fp.split[d] = -1;
    fp.touch[d] = -1;
  }
  fp.nitems = V;
  fp.out = toe_d;
  fp.errflag = err_d;
  if ((s = run_far(B, fp, g_d)) != GILA_OK) return s;
  // identity + circulant embedding
  const Z id = zdiv(Z{1.0, 0.0}, zmul(B.f, B.f));
  k_embed<<<1184, 256, 0, B.st>>>(toe_d, (int)nx, (int)ny, (int)nz, id, crc_d);
  KB_TRY(cudaGetLastError());
  return GILA_OK;
}

// FP64 forward 3-D FFT of the 6-component circulant, in place
static gila_status fft3(Build& B, Z* crc_d, const int P[3]) {
  gila_status s;
  const int64_t vol = (int64_t)P[0] * P[1] * P[2];
  for (int ax = 0; ax < 3; ++ax) {
    AxisPlan pl;
    if ((s = plan_axis(P[ax], &pl)) != GILA_OK) return s;
    AxisPlan* pl_d;
    if ((s = B.alloc(&pl_d, 1)) != GILA_OK) return s;
    KB_TRY(cudaMemcpyAsync(pl_d, &pl, sizeof(pl), cudaMemcpyHostToDevice, B.st));
    const void* tw;
    if ((s = twiddle_table(B.ctx, P[ax], GILA_C128, &tw)) != GILA_OK) return s;
    int TX = 2048 / P[ax];
    if (TX > 8) TX = 8;
    if (TX < 1) TX = 1;
    int T = ((TX * P[ax] + 3) / 4 + 31) / 32 * 32;
    while (T > 512 && TX > 1) {
      TX /= 2;
      T = ((TX * P[ax] + 3) / 4 + 31) / 32 * 32;
    }
    if (T > 512) return fail(GILA_ERR_ARG, "circulant axis too long for the kernel build FFT");
    int64_t es, gstride, lines, groups;
    if (ax == 0) {  // rows
      es = 1;
      lines = 6 * vol / P[0];
      groups = 1;
      gstride = 0;
    } else if (ax == 1) {
      es = P[0];
      lines = P[0];
      groups = 6LL * P[2];
      gstride = (int64_t)P[0] * P[1];
    } else {
      es = (int64_t)P[0] * P[1];
      lines = (int64_t)P[0] * P[1];
      groups = 6;
      gstride = vol;
    }
    const size_t sm = (size_t)TX * P[ax] * sizeof(double2);
    if (sm > 48 * 1024) KB_TRY(cudaFuncSetAttribute(k_fft_axis, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int64_t blocks = groups * ((lines + TX - 1) / TX);
    k_fft_axis<<<(unsigned)blocks, T, sm, B.st>>>(reinterpret_cast<double2*>(crc_d), pl_d, P[ax],
                                                  static_cast<const double2*>(tw), es, gstride, TX, lines,
                                                  make_fdiv((uint32_t)TX));
    KB_TRY(cudaGetLastError());
  }
  return GILA_OK;
}

}  // namespace kb

namespace kb {

// The external circulant of one target / source volume pair
// (genEgoCrcExt!, src/glaGen.jl:55-100) into crc_d [6][P...].
static gila_status ext_circulant(Build& B, const HVol& t, const HVol& sv, const int P[3], Z* crc_d, int* err_d) {
  gila_status s;
  const int64_t vol = (int64_t)P[0] * P[1] * P[2];
  Rat sl[3], su[3], tl[3], tu[3];
  bool c1 = true, c2 = true;
  int ovr = 0;
  for (int d = 0; d < 3; ++d) {
    const Rat hs = rdv(sv.scl[d], R(2)), ht = rdv(t.scl[d], R(2));
    sl[d] = rsub(sv.start[d], hs);
    su[d] = radd(sv.stop[d], hs);
    tl[d] = rsub(t.start[d], ht);
    tu[d] = radd(t.stop[d], ht);
    c1 = c1 && rle(sl[d], tl[d]) && rle(tl[d], su[d]);
    c2 = c2 && rle(sl[d], tu[d]) && rle(tu[d], su[d]);
    ovr += (rlt(sl[d], tl[d]) && rlt(tl[d], su[d])) + (rlt(sl[d], tu[d]) && rlt(tu[d], su[d]));
  }
  const bool contact = c1 || c2;
  if (contact && ovr > 0) return fail(GILA_ERR_OVERLAP, "Source and target volumes are overlapping.");
  // grdSel tables over sepGrd(trg, src, 0) / sepGrd(trg, src, 1)
  double* sep_d[3];
  for (int d = 0; d < 3; ++d) {
    Rat tstr = rsub(t.start[d], sv.start[d]), tstp = rsub(t.stop[d], sv.start[d]), tstep = t.grd[d];
    if (rlt(tstp, tstr)) tstep = rmul(tstep, R(-1));
    Rat sstr = rsub(t.start[d], sv.stop[d]), sstp = rsub(t.start[d], sv.start[d]), sstep = sv.grd[d];
    if (rlt(sstp, sstr)) sstep = rmul(sstep, R(-1));
    std::vector<double> sp(P[d], 0.0);
    for (int64_t ind = 1; ind <= P[d]; ++ind) {
      if (ind <= t.cel[d]) {
        sp[ind - 1] = rd(radd(tstr, rmul(R(ind - 1), tstep)));
      } else if (ind > t.cel[d] + 1) {
        sp[ind - 1] = rd(radd(sstr, rmul(R(ind - 2 - t.cel[d]), sstep)));
      }
    }
    if ((s = B.alloc(&sep_d[d], sp.size())) != GILA_OK) return s;
    KB_TRY(cudaMemcpyAsync(sep_d[d], sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice, B.st));
  }
  PairGeo G;
  faces(t.scl, G.tf);
  faces(sv.scl, G.sf);
  srf_scales(t.scl, sv.scl, G.scale);
  G.f = B.f;
  PairGeo* g_d;
  if ((s = B.alloc(&g_d, 1)) != GILA_OK) return s;
  KB_TRY(cudaMemcpyAsync(g_d, &G, sizeof(G), cudaMemcpyHostToDevice, B.st));
  FarParams fp{};
  fp.mode = 1;
  for (int d = 0; d < 3; ++d) {
    fp.n[d] = P[d];
    fp.sep[d] = sep_d[d];
    fp.split[d] = (int)t.cel[d];
    fp.touch[d] = contact ? CNT_TOL + (rd(t.scl[d]) + rd(sv.scl[d])) / 2.0 : -1.0;
  }
  fp.nitems = vol;
  fp.out = crc_d;
  fp.errflag = err_d;
  if ((s = run_far(B, fp, g_d)) != GILA_OK) return s;
  if (contact) {
    // genCntVol (src/glaGen.jl:308-318) and its self circulant
    int64_t cel[3];
    Rat cs[3];
    for (int d = 0; d < 3; ++d) {
      cs[d] = rlt(t.scl[d], sv.scl[d]) ? t.scl[d] : sv.scl[d];
      const Rat a = rdv(t.scl[d], cs[d]), b = rdv(sv.scl[d], cs[d]);
      cel[d] = a.n / a.d + b.n / b.d;
    }
    Vol cv0;
    for (int d = 0; d < 3; ++d) {
      cv0.cel[d] = cel[d];
      cv0.scl[d] = cs[d];
      cv0.org[d] = R(0);
      cv0.grd[d] = cs[d];
    }
    const HVol cv = hvol(cv0);
    Z* ccnt;
    if ((s = B.alloc(&ccnt, 6 * 8 * cel[0] * cel[1] * cel[2])) != GILA_OK) return s;
    if ((s = self_circulant(B, cv, ccnt, err_d)) != GILA_OK) return s;
    CntParams cp;
    for (int d = 0; d < 3; ++d) {
      cp.n[d] = P[d];
      cp.split[d] = (int)t.cel[d];
      cp.sep[d] = sep_d[d];
      cp.touch[d] = fp.touch[d];
      cp.cscl[d] = rd(cs[d]);
      const Rat ss = rdv(sv.scl[d], cs[d]), ts = rdv(t.scl[d], cs[d]);
      cp.sspan[d] = (int)(ss.n / ss.d);
      cp.tspan[d] = (int)(ts.n / ts.d);
      cp.cc[d] = (int)cel[d];
    }
    cp.ccnt = ccnt;
    cp.out = crc_d;
    k_contact<<<64, 128, 0, B.st>>>(cp);
    KB_TRY(cudaGetLastError());
  }
  return GILA_OK;
}

// Partition `tp` (x fastest) of a volume whose cells sit on a grid `div`
// times coarser than the pair's common grid (src/glaMemSup.jl:60-87): centre
// (off - (div - 1) / 2) * scl + org, cell scale scl, grid step div * scl,
// par_cel cells per axis.
static HVol partition_vol(const Vol& v, const int div[3], const int par_cel[3], const int off[3]) {
  Vol p;
  for (int d = 0; d < 3; ++d) {
    p.cel[d] = par_cel[d];
    p.scl[d] = v.scl[d];
    p.org[d] = radd(rmul(rsub(R(off[d]), R(div[d] - 1, 2)), v.scl[d]), v.org[d]);
    p.grd[d] = rmul(R(div[d]), v.scl[d]);
  }
  return hvol(p);
}

}  // namespace kb

// Build the operator's Fourier kernel on the GPU (GlaOprMem with
// egoFur == nothing).  Volume pairs of different cell scales are built per
// target partition (src/glaMemSup.jl:60-88), each partition's circulant
// transformed and extracted into its slice of the kernel.  Source
// partitions (a source grid finer than the target) are refused: egoOpr!
// cannot apply such an operator (src/glaAct.jl:37-49).
gila_status build_kernel(Core& c) {
  using namespace kb;
  if (c.parS != 1)
    return fail(GILA_ERR_ARG, "the GPU kernel build does not handle source partitions (a source grid finer than "
                              "the target), which egoOpr! cannot apply; pass egoFur instead");
  Build B;
  B.ctx = c.ctx;
  B.st = c.stream;
  B.f = Z{c.opt.frq_re, c.opt.frq_im};
  B.ord = c.opt.int_ord > 0 ? c.opt.int_ord : 32;
  if (B.ord > kMaxOrd) return fail(GILA_ERR_ARG, "intOrd above 64 is not supported");
  gila_status s;
  {
    Consts q;
    q.ord = B.ord;
    gauss_legendre(B.ord, q.x, q.w);
    q.f = B.f;
    if ((s = B.alloc(&B.q_d, 1)) != GILA_OK) return s;
    KB_TRY(cudaMemcpyAsync(B.q_d, &q, sizeof(q), cudaMemcpyHostToDevice, B.st));
  }
  KB_TRY(cudaMemcpyToSymbolAsync(c_sng_cor, SNG_COR, sizeof(SNG_COR), 0, cudaMemcpyHostToDevice, B.st));
  KB_TRY(cudaMemcpyToSymbolAsync(c_sng_mask, SNG_MASK, sizeof(SNG_MASK), 0, cudaMemcpyHostToDevice, B.st));
  int* err_d;
  if ((s = B.alloc(&err_d, 2)) != GILA_OK) return s;
  KB_TRY(cudaMemsetAsync(err_d, 0, 2 * sizeof(int), B.st));
  const HVol t = hvol(c.trg), sv = hvol(c.src);
  const int P[3] = {c.geom.P[0], c.geom.P[1], c.geom.P[2]};
  const int64_t vol = (int64_t)P[0] * P[1] * P[2];
  Z* crc_d;
  if ((s = B.alloc(&crc_d, 6 * vol)) != GILA_OK) return s;
  const Geom& g = c.geom;
  const int parT = g.parT;
  const size_t cs = csize(c.dtype);
  const size_t per = (size_t)g.tru[0] * g.tru[1] * g.tru[2] * 6 * 8;  // elements per target partition
  KB_TRY(dev_malloc(&c.ker, per * parT * cs));
  c.ker_bytes = per * parT * cs;
  const size_t mark = B.keep.size();
  for (int tp = 0; tp < parT; ++tp) {
    if (c.self) {
      if ((s = self_circulant(B, t, crc_d, err_d)) != GILA_OK) return s;
    } else {
      KB_TRY(cudaMemsetAsync(crc_d, 0, (size_t)6 * vol * sizeof(Z), B.st));
      const HVol tv = parT == 1 ? t : partition_vol(c.trg, c.mix.tdiv, c.mix.tc, g.toff[tp]);
      if ((s = ext_circulant(B, tv, sv, P, crc_d, err_d)) != GILA_OK) return s;
    }
    if ((s = fft3(B, crc_d, P)) != GILA_OK) return s;
    // extract into partition tp of the operator's kernel layout
    if (c.dtype == GILA_C128)
      k_extract<double2><<<1184, 256, 0, B.st>>>(crc_d, P[0], P[1], P[2], g.tru[0], g.tru[1], g.tru[2],
                                                static_cast<double2*>(c.ker) + per * tp, err_d + 1);
    else
      k_extract<float2><<<1184, 256, 0, B.st>>>(crc_d, P[0], P[1], P[2], g.tru[0], g.tru[1], g.tru[2],
                                               static_cast<float2*>(c.ker) + per * tp, err_d + 1);
    KB_TRY(cudaGetLastError());
    B.release_from(mark);  // this partition's cubature scratch
  }
  int flags[2];
  KB_TRY(cudaMemcpyAsync(flags, err_d, sizeof(flags), cudaMemcpyDeviceToHost, B.st));
  KB_TRY(cudaStreamSynchronize(B.st));
  if (flags[0]) return fail(GILA_ERR_INTERNAL, "kernel build: cubature region capacity or iteration cap exceeded");
  if (flags[1]) return fail(GILA_ERR_NAN, "Fourier information contains non-numeric values.");
  return GILA_OK;
}

// wekS / wekE / wekV (src/glaInt.jl:75-262) for one cell scale at
// Gauss-Legendre order `ord`, unscaled, evaluated on the GPU by the same
// kernels the operator build uses (out: 18 complex values as re/im pairs,
// wS[3], wE[9], wV[6]).
gila_status weak_integrals(Ctx* ctx, const Rat scl[3], kb::Z f, int ord, double out[36]) {
  using namespace kb;
  if (ord < 1 || ord > kMaxOrd) return fail(GILA_ERR_ARG, "intOrd must be in 1..64");
  for (int d = 0; d < 3; ++d)
    if (scl[d].n <= 0 || scl[d].d <= 0) return fail(GILA_ERR_ARG, "cell scales must be positive");
  cudaStream_t st = nullptr;
  KB_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  gila_status s = GILA_OK;
  {
    Build B;
    B.ctx = ctx;
    B.st = st;
    B.f = f;
    B.ord = ord;
    Consts q;
    q.ord = ord;
    gauss_legendre(ord, q.x, q.w);
    q.f = f;
    Z* w_d = nullptr;
    Z raw[18];
    if ((s = B.alloc(&B.q_d, 1)) == GILA_OK) {
      cudaError_t e = cudaMemcpyAsync(B.q_d, &q, sizeof(q), cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) s = cuda_fail(e, "cudaMemcpyAsync(weak consts)");
    }
    if (s == GILA_OK) s = B.alloc(&w_d, 36);
    if (s == GILA_OK) s = weak_values(B, scl, w_d, w_d + 18);
    if (s == GILA_OK) {
      cudaError_t e = cudaMemcpyAsync(raw, w_d + 18, sizeof(raw), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) s = cuda_fail(e, "weak integrals");
    }
    cudaStreamSynchronize(st);
    if (s == GILA_OK)
      for (int k = 0; k < 18; ++k) {
        out[2 * k] = raw[k].x;
        out[2 * k + 1] = raw[k].y;
      }
  }
  cudaStreamDestroy(st);
  return s;
}

}  // namespace gila

extern "C" gila_status gila_weak_integrals(gila_ctx* ctx, const int64_t scl_num[3], const int64_t scl_den[3],
                                           double frq_re, double frq_im, int32_t int_ord, double out[36]) {
  using namespace gila;
  if (!ctx || !scl_num || !scl_den || !out) return fail(GILA_ERR_ARG, "null argument");
  GILA_CUDA_TRY(cudaSetDevice(ctx->impl->device));
  Rat scl[3];
  for (int d = 0; d < 3; ++d) {
    if (scl_den[d] == 0) return fail(GILA_ERR_ARG, "zero denominator in a cell scale");
    scl[d] = rat(scl_num[d], scl_den[d]);
  }
  return weak_integrals(ctx->impl, scl, kb::Z{frq_re, frq_im}, int_ord, out);
}
