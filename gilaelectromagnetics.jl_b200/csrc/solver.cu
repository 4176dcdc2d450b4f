// solver.cu -- the scattering solve (I - chi G) x = b on the GPU.
//
// The reference's solve is user-side code: LippmannSchwinger
// (examples/GilaOperators.jl:57-96) applies x - chi .* (G x), chi per cell
// broadcast over the three components (:71, :94), and `solve`
// (examples/scattering_film.jl:58-61) hands it to IterativeSolvers.bicgstabl,
// i.e. BiCGStab(l) of Sleijpen & Fokkema (1993) with l = 2, a zero initial
// guess, a random shadow residual and a stop on the recursively updated
// residual.  IterativeSolvers is neither vendored nor pinned by the
// reference; this file restates that published method for many right-hand
// sides at once:
//
//  * every Krylov vector of a batch is [nrhs][n] in HBM, every scalar of the
//    recurrence (rho, sigma, omega, gamma, the Gram matrix of the MR step) is
//    per right-hand side in device memory, so one iteration is a fixed
//    sequence of kernels and is replayed from a CUDA graph;
//  * dot products accumulate in FP64 with a fixed reduction order, so each
//    right-hand side's arithmetic does not depend on what else is batched;
//  * an FP64 iterative-refinement loop wraps the Krylov solve: the residual
//    b - (x - chi G x) is formed from the FP64 matvec, the correction equation
//    is solved by the same BiCGStab(l) either in FP64 (plain) or on the
//    ComplexF32 operator (mixed), and the correction is accumulated in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.h"
#include "solver.h"

namespace gila {
namespace {

constexpr int kMaxEll = 4;
constexpr int kGram = (kMaxEll + 1) * (kMaxEll + 2) / 2;  // upper triangle of the (l+1)^2 Gram matrix
constexpr int kT = 256;                                    // threads of the vector kernels
// per right-hand side scalar slots (complex double)
enum : int { S_RHO = 0, S_SIG = 1, S_OMG = 2, S_GAM = 3, S_GRAM = S_GAM + kMaxEll, kSlots = S_GRAM + kGram };

struct Stat {
  double nrm2;  // squared norm of the recursively updated residual
  int act;      // still iterating
  int broke;    // the recurrence broke down (zero or non-finite scalar)
};

// Krylov vectors of one inner solve, each [nrhs][n]; the shadow residual is
// one [n] vector shared by all right-hand sides.
template <typename C>
struct KVec {
  C* x;
  C* r[kMaxEll + 1];
  C* u[kMaxEll + 1];
  const C* shadow;
};

__device__ __forceinline__ double2 to_d(double2 v) { return v; }
__device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }
template <typename C>
__device__ __forceinline__ C from_d(double2 v);
template <>
__device__ __forceinline__ double2 from_d<double2>(double2 v) {
  return v;
}
template <>
__device__ __forceinline__ float2 from_d<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__device__ __forceinline__ double2 cjmul(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ bool cfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// index of the Gram entry (a, b), a <= b <= kMaxEll
__host__ __device__ constexpr int gidx(int a, int b) { return a * (2 * (kMaxEll + 1) - a + 1) / 2 + (b - a); }

// Sums `k` per-thread accumulators over the block in a fixed order and stores
// sum i at out[i * stride] (one partial of a two-stage reduction).
template <int KM>
__device__ __forceinline__ void block_sum_store(const double2 (&acc)[KM], int k, double2* out, int64_t stride) {
  __shared__ double2 sh[KM][kT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < KM; ++i) {
    if (i < k) {
      double2 v = acc[i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
      }
      if (lane == 0) sh[i][w] = v;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < k) {
    double2 s = make_double2(0.0, 0.0);
    for (int ww = 0; ww < kT / 32; ++ww) s = cadd(s, sh[threadIdx.x][ww]);
    out[threadIdx.x * stride] = s;
  }
}

// ------------------------------------------------------------ reductions
// W complex values per 16-byte transaction: FP32 vectors move two values
// (float4) per load / store, FP64 one; W = 2 needs an even n (host-checked).
template <typename C, int W>
struct VIO;
template <>
struct VIO<float2, 2> {
  __device__ __forceinline__ static void ld(const float2* p, int64_t u, double2 (&v)[2]) {
    const float4 q = reinterpret_cast<const float4*>(p)[u];
    v[0] = make_double2(q.x, q.y);
    v[1] = make_double2(q.z, q.w);
  }
  __device__ __forceinline__ static void st(float2* p, int64_t u, const double2 (&v)[2]) {
    reinterpret_cast<float4*>(p)[u] = make_float4((float)v[0].x, (float)v[0].y, (float)v[1].x, (float)v[1].y);
  }
};
template <typename C>
struct VIO<C, 1> {
  __device__ __forceinline__ static void ld(const C* p, int64_t u, double2 (&v)[1]) { v[0] = to_d(p[u]); }
  __device__ __forceinline__ static void st(C* p, int64_t u, const double2 (&v)[1]) { p[u] = from_d<C>(v[0]); }
};
// the value a store of v leaves in memory (rounded to C)
template <typename C>
__device__ __forceinline__ double2 rounded(double2 v) {
  return to_d(from_d<C>(v));
}

// part[r][0][blk] = sum_i conj(shadow[i]) b_r[i] over W-value units
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_sdot(const C* __restrict__ a, const C* __restrict__ b, int64_t n,
                                             double2* __restrict__ part, const int* __restrict__ act = nullptr) {
  const int r = act ? act[blockIdx.y] : blockIdx.y, nb = gridDim.x;
  b += n * r;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  const int64_t nu = n / W;
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)nb * kT) {
    double2 x[W], y[W];
    VIO<C, W>::ld(a, u, x);
    VIO<C, W>::ld(b, u, y);
#pragma unroll
    for (int w = 0; w < W; ++w) acc[0] = cadd(acc[0], cjmul(x[w], y[w]));
  }
  block_sum_store<1>(acc, 1, part + (int64_t)r * nb + blockIdx.x, nb);
}

// Gram matrix r_a^H r_b, a <= b <= ell, of the MR step (all kGram slots).
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_gram(KVec<C> v, int ell, int64_t n, double2* __restrict__ part,
                                             const int* __restrict__ act = nullptr) {
  const int r = act ? act[blockIdx.y] : blockIdx.y, nb = gridDim.x;
  const int64_t off = (int64_t)r * n / W;
  double2 acc[kGram];
#pragma unroll
  for (int k = 0; k < kGram; ++k) acc[k] = make_double2(0.0, 0.0);
  const int64_t nu = n / W;
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)nb * kT) {
    double2 e[kMaxEll + 1][W];
#pragma unroll
    for (int a = 0; a <= kMaxEll; ++a) {
      if (a <= ell) {
        VIO<C, W>::ld(v.r[a], off + u, e[a]);
      } else {
#pragma unroll
        for (int w = 0; w < W; ++w) e[a][w] = make_double2(0.0, 0.0);
      }
    }
#pragma unroll
    for (int a = 0; a <= kMaxEll; ++a)
#pragma unroll
      for (int b = a; b <= kMaxEll; ++b)
        if (b <= ell)
#pragma unroll
          for (int w = 0; w < W; ++w) acc[gidx(a, b)] = cadd(acc[gidx(a, b)], cjmul(e[a][w], e[b][w]));
  }
  block_sum_store<kGram>(acc, kGram, part + (int64_t)r * kGram * nb + blockIdx.x, nb);
}

enum FinMode : int { FIN_STORE = 0, FIN_CHECK = 1, FIN_RESID = 2, FIN_NORM = 3 };

// Second stage: sums the nb partials of K values per right-hand side in a
// fixed order.  FIN_STORE / FIN_CHECK write scalar slots (FIN_CHECK retires a
// right-hand side whose value is zero or not finite: a breakdown);
// FIN_RESID stores the residual norm and retires converged (nrm2 <= tol2) or
// broken right-hand sides; FIN_NORM stores the squared norm in nrm_out.
__global__ void __launch_bounds__(kT) k_fin(const double2* __restrict__ part, int K, int nb, double2* sc, int slot,
                                            Stat* st, const double* __restrict__ tol2, int mode,
                                            double* __restrict__ nrm_out = nullptr,
                                            const int* __restrict__ act = nullptr) {
  const int r = act ? act[blockIdx.x] : blockIdx.x;
  if (mode == FIN_RESID && !st[r].act) return;
  __shared__ double2 sh[kT / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = 0; k < K; ++k) {
    const double2* p = part + ((int64_t)r * K + k) * nb;
    double2 s = make_double2(0.0, 0.0);
    for (int i = threadIdx.x; i < nb; i += kT) s = cadd(s, p[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s.x += __shfl_down_sync(0xffffffffu, s.x, o);
      s.y += __shfl_down_sync(0xffffffffu, s.y, o);
    }
    if (lane == 0) sh[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double2 t = make_double2(0.0, 0.0);
      for (int ww = 0; ww < kT / 32; ++ww) t = cadd(t, sh[ww]);
      if (mode == FIN_STORE || mode == FIN_CHECK) {
        sc[(int64_t)r * kSlots + slot + k] = t;
        if (mode == FIN_CHECK && st[r].act && (!cfinite(t) || (t.x == 0.0 && t.y == 0.0))) {
          st[r].act = 0;
          st[r].broke = 1;
        }
      } else if (mode == FIN_NORM) {
        nrm_out[r] = t.x;
      } else {
        st[r].nrm2 = t.x;
        {
          if (st[r].broke || !isfinite(t.x)) {
            st[r].act = 0;
            st[r].broke = 1;
          } else if (t.x <= tol2[r]) {
            st[r].act = 0;
          }
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------- scalar steps
// sigma = omega = 1 for the right-hand sides whose Krylov process (re)starts
__global__ void k_scal_init(double2* sc, const int* __restrict__ mask, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs || !mask[r]) return;
  sc[(int64_t)r * kSlots + S_SIG] = make_double2(1.0, 0.0);
  sc[(int64_t)r * kSlots + S_OMG] = make_double2(1.0, 0.0);
}

// sigma = -omega * sigma at the start of an iteration
__global__ void k_iter_start(double2* sc, const Stat* st, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs || !st[r].act) return;
  double2* s = sc + (int64_t)r * kSlots;
  const double2 t = cmul(s[S_OMG], s[S_SIG]);
  s[S_SIG] = make_double2(-t.x, -t.y);
}

// MR step: gamma = M[1:l,1:l] \ M[1:l,0] with M = R^H R (Gaussian elimination
// with partial pivoting per right-hand side); omega = gamma[l-1].
__global__ void k_mr_solve(double2* sc, Stat* st, int ell, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs || !st[r].act) return;
  double2* s = sc + (int64_t)r * kSlots;
  const double2* G = s + S_GRAM;
  auto M = [&](int a, int b) {
    if (a <= b) return G[gidx(a, b)];
    const double2 t = G[gidx(b, a)];
    return make_double2(t.x, -t.y);
  };
  double2 A[kMaxEll][kMaxEll + 1];
  for (int i = 0; i < ell; ++i) {
    for (int k = 0; k < ell; ++k) A[i][k] = M(i + 1, k + 1);
    A[i][ell] = M(i + 1, 0);
  }
  bool ok = true;
  for (int c = 0; c < ell && ok; ++c) {
    int p = c;
    for (int i = c + 1; i < ell; ++i)
      if (cabs2(A[i][c]) > cabs2(A[p][c])) p = i;
    if (!(cabs2(A[p][c]) > 0.0)) {
      ok = false;
      break;
    }
    if (p != c)
      for (int k = 0; k <= ell; ++k) {
        const double2 t = A[c][k];
        A[c][k] = A[p][k];
        A[p][k] = t;
      }
    for (int i = c + 1; i < ell; ++i) {
      const double2 f = cdiv(A[i][c], A[c][c]);
      for (int k = c; k <= ell; ++k) A[i][k] = csub(A[i][k], cmul(f, A[c][k]));
    }
  }
  double2 g[kMaxEll];
  for (int i = ell - 1; i >= 0 && ok; --i) {
    double2 t = A[i][ell];
    for (int k = i + 1; k < ell; ++k) t = csub(t, cmul(A[i][k], g[k]));
    g[i] = cdiv(t, A[i][i]);
    ok = cfinite(g[i]);
  }
  if (!ok) {
    st[r].act = 0;
    st[r].broke = 1;
    return;
  }
  for (int i = 0; i < ell; ++i) s[S_GAM + i] = g[i];
  s[S_OMG] = g[ell - 1];
  // omega = 0 breaks the next iteration; this one's update still holds
  if (g[ell - 1].x == 0.0 && g[ell - 1].y == 0.0) st[r].broke = 1;
}

// ------------------------------------------------------- vector updates
// (all over W-value units; off = the slot's offset in units)
// BiCG part, step j (1-based): u_q = r_q - beta u_q, q < j, beta = rho / sigma
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_bicg_u(KVec<C> v, int j, int64_t n, const double2* __restrict__ sc,
                                               const Stat* __restrict__ st, const int* __restrict__ act = nullptr) {
  const int r = act ? act[blockIdx.y] : blockIdx.y;
  if (!st[r].act) return;
  const double2 beta = cdiv(sc[(int64_t)r * kSlots + S_RHO], sc[(int64_t)r * kSlots + S_SIG]);
  const int64_t off = (int64_t)r * n / W, nu = n / W;
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)gridDim.x * kT)
#pragma unroll
    for (int q = 0; q < kMaxEll; ++q)
      if (q < j) {
        double2 a[W], b[W];
        VIO<C, W>::ld(v.r[q], off + u, a);
        VIO<C, W>::ld(v.u[q], off + u, b);
#pragma unroll
        for (int w = 0; w < W; ++w) b[w] = csub(a[w], cmul(beta, b[w]));
        VIO<C, W>::st(v.u[q], off + u, b);
      }
}

// BiCG part, step j: r_q -= alpha u_{q+1}, q < j; x += alpha u_0; alpha =
// rho / sigma; and the partial of |r_0|^2.  A residual that a BiCG step
// already brought to tolerance ends the solve there: continuing the cycle
// would divide rounding noise by rounding noise (sigma of the next step is
// rho - beta * rho_prev; with chi = 0 the first step converges exactly).
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_bicg_r(KVec<C> v, int j, int64_t n, const double2* __restrict__ sc,
                                               const Stat* __restrict__ st, double2* __restrict__ part,
                                               const int* __restrict__ act = nullptr) {
  const int r = act ? act[blockIdx.y] : blockIdx.y, nb = gridDim.x;
  if (!st[r].act) return;
  const double2 alpha = cdiv(sc[(int64_t)r * kSlots + S_RHO], sc[(int64_t)r * kSlots + S_SIG]);
  const int64_t off = (int64_t)r * n / W, nu = n / W;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)nb * kT) {
#pragma unroll
    for (int q = 0; q < kMaxEll; ++q)
      if (q < j) {
        double2 a[W], b[W];
        VIO<C, W>::ld(v.r[q], off + u, a);
        VIO<C, W>::ld(v.u[q + 1], off + u, b);
#pragma unroll
        for (int w = 0; w < W; ++w) {
          a[w] = csub(a[w], cmul(alpha, b[w]));
          if (q == 0) acc[0].x += cabs2(rounded<C>(a[w]));
        }
        VIO<C, W>::st(v.r[q], off + u, a);
      }
    double2 x[W], u0[W];
    VIO<C, W>::ld(v.x, off + u, x);
    VIO<C, W>::ld(v.u[0], off + u, u0);
#pragma unroll
    for (int w = 0; w < W; ++w) x[w] = cadd(x[w], cmul(alpha, u0[w]));
    VIO<C, W>::st(v.x, off + u, x);
  }
  block_sum_store<1>(acc, 1, part + (int64_t)r * nb + blockIdx.x, nb);
}

// MR part: u_0 -= sum_k gamma_k u_k, x += sum_k gamma_k r_{k-1},
// r_0 -= sum_k gamma_k r_k (k = 1..l), and the partial of |r_0|^2.
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_mr_update(KVec<C> v, int ell, int64_t n, const double2* __restrict__ sc,
                                                  const Stat* __restrict__ st, double2* __restrict__ part,
                                                  const int* __restrict__ act = nullptr) {
  const int r = act ? act[blockIdx.y] : blockIdx.y, nb = gridDim.x;
  if (!st[r].act) return;
  double2 g[kMaxEll];
#pragma unroll
  for (int k = 0; k < kMaxEll; ++k)
    g[k] = k < ell ? sc[(int64_t)r * kSlots + S_GAM + k] : make_double2(0.0, 0.0);
  const int64_t off = (int64_t)r * n / W, nu = n / W;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)nb * kT) {
    double2 u0[W], r0[W], x[W];
    VIO<C, W>::ld(v.u[0], off + u, u0);
    VIO<C, W>::ld(v.r[0], off + u, r0);
    VIO<C, W>::ld(v.x, off + u, x);
#pragma unroll
    for (int w = 0; w < W; ++w) x[w] = cadd(x[w], cmul(g[0], r0[w]));
#pragma unroll
    for (int k = 1; k <= kMaxEll; ++k)
      if (k <= ell) {
        double2 rk[W], uk[W];
        VIO<C, W>::ld(v.r[k], off + u, rk);
        VIO<C, W>::ld(v.u[k], off + u, uk);
#pragma unroll
        for (int w = 0; w < W; ++w) {
          u0[w] = csub(u0[w], cmul(g[k - 1], uk[w]));
          r0[w] = csub(r0[w], cmul(g[k - 1], rk[w]));
          if (k < ell) x[w] = cadd(x[w], cmul(g[k], rk[w]));
        }
      }
    VIO<C, W>::st(v.u[0], off + u, u0);
    VIO<C, W>::st(v.r[0], off + u, r0);
    VIO<C, W>::st(v.x, off + u, x);
#pragma unroll
    for (int w = 0; w < W; ++w) acc[0].x += cabs2(rounded<C>(r0[w]));
  }
  block_sum_store<1>(acc, 1, part + (int64_t)r * nb + blockIdx.x, nb);
}

// ------------------------------------------------- refinement (FP64) steps
// r = b - (x - chi .* t) with t = G x held in r on entry; partial |r|^2
// (masked right-hand sides only when mask is set).
__global__ void __launch_bounds__(kT) k_resid(const double2* __restrict__ b, const double2* __restrict__ x,
                                              double2* __restrict__ r, const double2* __restrict__ chi,
                                              int64_t chi_rs, int64_t V, const int* __restrict__ mask,
                                              double2* __restrict__ part) {
  const int q = blockIdx.y, nb = gridDim.x;
  if (mask && !mask[q]) return;
  chi += chi_rs * q;
  const int64_t off = 3 * V * q;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < V; i += (int64_t)nb * kT) {
    const double2 c = chi[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int64_t j = off + k * V + i;
      const double2 v = cadd(csub(b[j], x[j]), cmul(c, r[j]));
      r[j] = v;
      acc[0].x += cabs2(v);
    }
  }
  block_sum_store<1>(acc, 1, part + (int64_t)q * nb + blockIdx.x, nb);
}

// (Re)start of the Krylov process on the scaled correction equation
// A d = r / s for the masked right-hand sides: r_0 = r64 * inv (inv = 1/s,
// rounded to C), d = 0, u_0 = 0.
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_inner_start(const double2* __restrict__ r64, KVec<C> v,
                                                    const double* __restrict__ inv, const int* __restrict__ mask,
                                                    int64_t n) {
  const int r = blockIdx.y;
  if (!mask[r]) return;
  const double s = inv[r];
  const int64_t off = (int64_t)r * n / W, nu = n / W;
  double2 z[W];
#pragma unroll
  for (int w = 0; w < W; ++w) z[w] = make_double2(0.0, 0.0);
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)gridDim.x * kT) {
    double2 a[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const double2 q = r64[(off + u) * W + w];
      a[w] = make_double2(q.x * s, q.y * s);
    }
    VIO<C, W>::st(v.r[0], off + u, a);
    VIO<C, W>::st(v.u[0], off + u, z);
    VIO<C, W>::st(v.x, off + u, z);
  }
}

// Reliable update, first half: x64 += s * d and d = 0 for the masked
// right-hand sides (the correction leaves the low-precision iterate).
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_accum(double2* __restrict__ x, C* __restrict__ d,
                                              const double* __restrict__ scale, const int* __restrict__ mask,
                                              int64_t n) {
  const int r = blockIdx.y;
  if (!mask[r]) return;
  const double s = scale[r];
  const int64_t off = (int64_t)r * n / W, nu = n / W;
  double2 z[W];
#pragma unroll
  for (int w = 0; w < W; ++w) z[w] = make_double2(0.0, 0.0);
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)gridDim.x * kT) {
    double2 a[W];
    VIO<C, W>::ld(d, off + u, a);
#pragma unroll
    for (int w = 0; w < W; ++w) {
      double2& xv = x[(off + u) * W + w];
      xv = make_double2(xv.x + s * a[w].x, xv.y + s * a[w].y);
    }
    VIO<C, W>::st(d, off + u, z);
  }
}

// Reliable update, second half: the recursive residual of the masked
// right-hand sides is replaced by the FP64 one, r_0 = (b - A64 x) * inv.
template <typename C, int W>
__global__ void __launch_bounds__(kT) k_replace(const double2* __restrict__ r64, C* __restrict__ r0,
                                                const double* __restrict__ inv, const int* __restrict__ mask,
                                                int64_t n) {
  const int r = blockIdx.y;
  if (!mask[r]) return;
  const double s = inv[r];
  const int64_t off = (int64_t)r * n / W, nu = n / W;
  for (int64_t u = (int64_t)blockIdx.x * kT + threadIdx.x; u < nu; u += (int64_t)gridDim.x * kT) {
    double2 a[W];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const double2 q = r64[(off + u) * W + w];
      a[w] = make_double2(q.x * s, q.y * s);
    }
    VIO<C, W>::st(r0, off + u, a);
  }
}

// Shadow residual: uniform [0,1) real and imaginary parts from a counter hash
// (splitmix64), the distribution of IterativeSolvers' rand(T, n).
template <typename C>
__global__ void k_shadow(C* s, int64_t n, uint64_t seed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(2 * i + 1);
    double u[2];
    for (int k = 0; k < 2; ++k) {
      z += 0x9E3779B97F4A7C15ull;
      uint64_t t = z;
      t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
      t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
      t ^= t >> 31;
      u[k] = (double)(t >> 11) * (1.0 / 9007199254740992.0);
    }
    s[i] = from_d<C>(make_double2(u[0], u[1]));
  }
}

template <typename C>
__global__ void k_cast(const double2* __restrict__ a, C* __restrict__ b, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = from_d<C>(a[i]);
}

// ------------------------------------------------------------- host side
struct DevArena {  // frees what it allocated when the solve returns
  std::vector<void*> d;
  std::vector<void*> h;
  ~DevArena() {
    for (void* p : d) cudaFree(p);
    for (void* p : h) cudaFreeHost(p);
  }
  cudaError_t alloc(void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = dev_malloc(p, bytes < 256 ? 256 : bytes);
    if (e == cudaSuccess) d.push_back(*p);
    return e;
  }
  cudaError_t alloc_host(void** p, size_t bytes) {
    *p = nullptr;
    cudaError_t e = cudaMallocHost(p, bytes);
    if (e == cudaSuccess) h.push_back(*p);
    return e;
  }
};

// blocks per right-hand side of the vector kernels: a function of n only, so
// that the reduction order never depends on the batch
int vec_blocks(int64_t n) {
  int64_t b = (n + kT * 4 - 1) / (kT * 4);
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 1024));
}

// partial of |a_r|^2 for the masked right-hand sides
__global__ void __launch_bounds__(kT) k_norm2(const double2* __restrict__ a, int64_t n, const int* __restrict__ mask,
                                              double2* __restrict__ part) {
  const int r = blockIdx.y, nb = gridDim.x;
  if (!mask[r]) return;
  a += n * r;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)nb * kT) acc[0].x += cabs2(a[i]);
  block_sum_store<1>(acc, 1, part + (int64_t)r * nb + blockIdx.x, nb);
}

// maximal runs [r0, r1) of set entries of m
std::vector<std::pair<int, int>> runs_of(const std::vector<char>& m, int cap) {
  std::vector<std::pair<int, int>> out;
  const int S = (int)m.size();
  for (int r0 = 0; r0 < S;) {
    if (!m[r0]) {
      ++r0;
      continue;
    }
    int r1 = r0 + 1;
    while (r1 < S && m[r1] && r1 - r0 < cap) ++r1;
    out.emplace_back(r0, r1);
    r0 = r1;
  }
  return out;
}

template <typename C>
struct OpRef {  // an operator with workspaces owned by a batch
  Core* core;
  Geom geom;    // max_rhs = the workspace capacity
  C* A;
  C* B;
  int cap;      // right-hand sides per matvec launch sequence
  Launch launch;  // launch shapes for cap right-hand sides
};

// right-hand sides the FP64 workspace of a mixed batch holds: reliable
// updates are rare, so their matvecs run in chunks
constexpr int kUpdateCap = 4;

// the Krylov-vector kernels in W-value units: FP32 vectors of even length
// move two values per 16-byte access
#define GILA_VW(KERNEL, GRID, ...)                                        \
  do {                                                                    \
    if (w2_)                                                              \
      KERNEL<CI, kW2><<<GRID, kT, 0, s_>>>(__VA_ARGS__);                  \
    else                                                                  \
      KERNEL<CI, 1><<<GRID, kT, 0, s_>>>(__VA_ARGS__);                    \
  } while (0)

template <typename CI>
class LsBatchT final : public LsBatch {
  static constexpr int kW2 = sizeof(CI) == 8 ? 2 : 1;

 public:
  LsBatchT(Core& a, Core& i, int S, const BatchCfg& c)
      : g64_(a), gi_(i), S_(S), n_(in_elems(a)), V_(in_elems(a) / 3), cfg_(c), sl_(S) {
    nb_ = vec_blocks(n_);
    w2_ = kW2 == 2 && n_ % 2 == 0;
  }
  ~LsBatchT() override {
    if (s_) cudaStreamSynchronize(s_);
    if (graph_) cudaGraphExecDestroy(graph_);
    if (ev_) cudaEventDestroy(ev_);
    mem_.release();
    if (s_) cudaStreamDestroy(s_);
  }

  static size_t bytes(const Core& a, const Core& i, int S, const BatchCfg& c) {
    const int64_t n = in_elems(a), V = n / 3;
    const bool mixed = c.mixed != 0;
    size_t t = 0;
    t += 3ull * S * n * sizeof(double2);                                 // b, x, r (FP64)
    t += (c.chi_shared ? 1ull : (size_t)S) * V * sizeof(double2);        // chi
    if (mixed) t += (c.chi_shared ? 1ull : (size_t)S) * V * sizeof(CI);  // chi, inner precision
    t += (size_t)(2 * c.ell + 3) * S * n * sizeof(CI) + n * sizeof(CI);  // Krylov vectors, shadow
    t += (size_t)S * (kGram * vec_blocks(n) + kSlots) * sizeof(double2) + (size_t)S * (sizeof(Stat) + 64);
    Geom g = a.geom;
    g.max_rhs = mixed ? std::min(S, kUpdateCap) : S;
    Work w = work_sizes(g);
    t += (size_t)(w.a_elems + w.b_rhs * g.max_rhs) * sizeof(double2);
    if (mixed) {
      Geom gi = i.geom;
      gi.max_rhs = S;
      gi.csize = sizeof(CI);
      w = work_sizes(gi);
      t += (size_t)(w.a_elems + w.b_rhs * S) * sizeof(CI);
    }
    return t;
  }

  gila_status init() {
    GILA_CUDA_TRY(cudaStreamCreateWithPriority(&s_, cudaStreamNonBlocking, cfg_.priority));
    GILA_CUDA_TRY(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming));
    const size_t vb = (size_t)S_ * n_;
    const bool mixed = cfg_.mixed != 0;
    const int nchi = cfg_.chi_shared ? 1 : S_;
    GILA_CUDA_TRY(mem_.alloc((void**)&b64_, vb * sizeof(double2)));
    GILA_CUDA_TRY(mem_.alloc((void**)&x64_, vb * sizeof(double2)));
    GILA_CUDA_TRY(mem_.alloc((void**)&r64_, vb * sizeof(double2)));
    GILA_CUDA_TRY(mem_.alloc((void**)&chi64_, (size_t)nchi * V_ * sizeof(double2)));
    if (mixed)
      GILA_CUDA_TRY(mem_.alloc((void**)&chii_, (size_t)nchi * V_ * sizeof(CI)));
    else
      chii_ = reinterpret_cast<CI*>(chi64_);
    GILA_CUDA_TRY(mem_.alloc((void**)&part_, (size_t)S_ * kGram * nb_ * sizeof(double2)));
    GILA_CUDA_TRY(mem_.alloc((void**)&sc_, (size_t)S_ * kSlots * sizeof(double2)));
    GILA_CUDA_TRY(mem_.alloc((void**)&st_d_, (size_t)S_ * sizeof(Stat)));
    GILA_CUDA_TRY(mem_.alloc((void**)&pb_d_, pb_bytes()));
    GILA_CUDA_TRY(mem_.alloc_host((void**)&st_h_, (size_t)S_ * sizeof(Stat)));
    GILA_CUDA_TRY(mem_.alloc_host((void**)&pb_h_, pb_bytes()));
    GILA_CUDA_TRY(mem_.alloc((void**)&act_d_, (size_t)S_ * sizeof(int)));
    GILA_CUDA_TRY(mem_.alloc_host((void**)&act_h_, (size_t)S_ * sizeof(int)));
    memset(st_h_, 0, (size_t)S_ * sizeof(Stat));
    memset(pb_h_, 0, pb_bytes());
    const int nvec = 2 * cfg_.ell + 3;
    CI* base = nullptr;
    GILA_CUDA_TRY(mem_.alloc((void**)&base, (size_t)nvec * vb * sizeof(CI)));
    GILA_CUDA_TRY(mem_.alloc((void**)&shadow_, (size_t)n_ * sizeof(CI)));
    kv_.x = base;
    for (int k = 0; k <= cfg_.ell; ++k) {
      kv_.r[k] = base + (size_t)(1 + k) * vb;
      kv_.u[k] = base + (size_t)(2 + cfg_.ell + k) * vb;
    }
    for (int k = cfg_.ell + 1; k <= kMaxEll; ++k) kv_.r[k] = kv_.u[k] = nullptr;
    kv_.shadow = shadow_;
    // workspaces of the two operators (owned here: batches run concurrently)
    op64_.core = &g64_;
    op64_.geom = g64_.geom;
    op64_.cap = mixed ? std::min(S_, kUpdateCap) : S_;
    op64_.geom.max_rhs = op64_.cap;
    {
      const Work w = work_sizes(op64_.geom);
      GILA_CUDA_TRY(mem_.alloc((void**)&op64_.A, (size_t)w.a_elems * sizeof(double2)));
      GILA_CUDA_TRY(mem_.alloc((void**)&op64_.B, (size_t)w.b_rhs * op64_.cap * sizeof(double2)));
    }
    if (mixed) {
      opi_.core = &gi_;
      opi_.geom = gi_.geom;
      opi_.cap = S_;
      opi_.geom.max_rhs = S_;
      const Work w = work_sizes(opi_.geom);
      GILA_CUDA_TRY(mem_.alloc((void**)&opi_.A, (size_t)w.a_elems * sizeof(CI)));
      GILA_CUDA_TRY(mem_.alloc((void**)&opi_.B, (size_t)w.b_rhs * S_ * sizeof(CI)));
    } else {
      opi_.core = &gi_;
      opi_.geom = op64_.geom;
      opi_.cap = op64_.cap;
      opi_.A = reinterpret_cast<CI*>(op64_.A);
      opi_.B = reinterpret_cast<CI*>(op64_.B);
    }
    // every Krylov vector starts finite
    GILA_CUDA_TRY(cudaMemsetAsync(base, 0, (size_t)nvec * vb * sizeof(CI), s_));
    // launch shapes for the batch's own right-hand-side counts: the tile
    // widths and radix orders that win for one vector need not win for a
    // chunk of several.  Timed on zero vectors (G 0 = 0 leaves every
    // buffer finite), or the operators' own single-vector choice.
    {  // another thread's apply may be re-picking an operator's shapes
      std::lock_guard<std::mutex> lk(g64_.mu);
      op64_.launch = g64_.launch;
    }
    if (&gi_ == &g64_) {
      opi_.launch = op64_.launch;
    } else {
      std::lock_guard<std::mutex> lk(gi_.mu);
      opi_.launch = gi_.launch;
    }
    if (cfg_.tune) {
      gila_status st;
      GILA_CUDA_TRY(cudaMemsetAsync(x64_, 0, vb * sizeof(double2), s_));
      if ((st = tuned_launch<double2>(g64_, op64_.geom, op64_.cap, x64_, r64_, op64_.A, op64_.B, s_,
                                      op64_.launch)) != GILA_OK)
        return st;
      if (!mixed)
        opi_.launch = op64_.launch;
      else if ((st = tuned_launch<CI>(gi_, opi_.geom, opi_.cap, base, kv_.r[0], opi_.A, opi_.B, s_,
                                      opi_.launch)) != GILA_OK)
        return st;
    }
    GILA_CUDA_TRY(cudaMemcpyAsync(st_d_, st_h_, (size_t)S_ * sizeof(Stat), cudaMemcpyHostToDevice, s_));
    k_shadow<CI><<<nb_, kT, 0, s_>>>(shadow_, n_, 0x5EEDull);
    GILA_CUDA_TRY(cudaGetLastError());
    GILA_CUDA_TRY(cudaStreamSynchronize(s_));
    return GILA_OK;
  }

  int slots() const override { return S_; }
  int free_slot() const override {
    for (int r = 0; r < S_; ++r)
      if (sl_[r].state == 0) return r;
    return -1;
  }
  int busy_slots() const override {
    int k = 0;
    for (const auto& q : sl_) k += q.state != 0;
    return k;
  }
  bool in_flight() const override { return in_flight_; }
  bool ready() override {
    if (!in_flight_) return true;
    const cudaError_t e = cudaEventQuery(ev_);
    if (e == cudaErrorNotReady) return false;
    if (e != cudaSuccess) cudaGetLastError();
    in_flight_ = false;
    return true;
  }
  gila_status wait() override {
    if (!in_flight_) return GILA_OK;
    GILA_CUDA_TRY(cudaEventSynchronize(ev_));
    in_flight_ = false;
    return GILA_OK;
  }
  std::vector<SlotResult> take_finished() override {
    std::vector<SlotResult> o;
    o.swap(finished_);
    return o;
  }
  const gila_solve_info& info() const override { return inf_; }
  void reset_info() override { inf_ = gila_solve_info{}; }
  cudaStream_t stream() const override { return s_; }

  gila_status set_shared_chi(const void* chi) override {
    if (!cfg_.chi_shared) return fail(GILA_ERR_ARG, "the batch has one medium per slot");
    if (in_flight_) return fail(GILA_ERR_INTERNAL, "batch busy");
    return load_chi(0, chi);
  }

  gila_status assign(int r, const void* chi, const void* b, void* x_out, const SlotOpts& o, uint64_t tag) override {
    if (r < 0 || r >= S_ || sl_[r].state != 0) return fail(GILA_ERR_ARG, "slot is not free");
    if (in_flight_) return fail(GILA_ERR_INTERNAL, "batch busy");
    if (!b || !x_out || (!cfg_.chi_shared && !chi)) return fail(GILA_ERR_ARG, "null argument");
    gila_status st;
    if (!cfg_.chi_shared && (st = load_chi(r, chi)) != GILA_OK) return st;
    GILA_CUDA_TRY(cudaMemcpyAsync(b64_ + (size_t)r * n_, b, n_ * sizeof(double2), cudaMemcpyDefault, s_));
    if (o.x0)
      GILA_CUDA_TRY(cudaMemcpyAsync(x64_ + (size_t)r * n_, x_out, n_ * sizeof(double2), cudaMemcpyDefault, s_));
    else
      GILA_CUDA_TRY(cudaMemsetAsync(x64_ + (size_t)r * n_, 0, n_ * sizeof(double2), s_));
    Slot& q = sl_[r];
    q = Slot{};
    q.state = 1;
    q.fresh = true;
    q.o = o;
    q.x_out = x_out;
    q.tag = tag;
    st_h_[r] = Stat{0.0, 0, 0};
    return GILA_OK;
  }

  gila_status advance(bool* enq) override {
    *enq = false;
    if (in_flight_) return fail(GILA_ERR_INTERNAL, "advance with a step in flight");
    gila_status st = GILA_OK;
    // slots whose solution copy has completed are released
    for (int r = 0; r < S_; ++r)
      if (sl_[r].state == 2) {
        sl_[r].state = 0;
        finished_.push_back(sl_[r].res);
      }
    switch (ph_) {
      case Ph::Init:
        digest_init();
        break;
      case Ph::Cycle: {
        bool upd = false;
        if ((st = digest_cycle(&upd)) != GILA_OK) return st;
        if (upd) return record(enq, Ph::Update);
        break;
      }
      case Ph::Update:
        if ((st = digest_update()) != GILA_OK) return st;
        break;
      default:
        break;
    }
    bool any_fresh = false, any_iter = false, any_copy = false;
    for (const auto& q : sl_) {
      any_fresh |= q.state == 1 && q.fresh;
      any_copy |= q.state == 2;
    }
    if (any_fresh) {
      if ((st = enqueue_init()) != GILA_OK) return st;
      return record(enq, Ph::Init);
    }
    if ((st = enqueue_starts()) != GILA_OK) return st;
    for (const auto& q : sl_) any_iter |= q.state == 1 && q.iter;
    if (any_iter) {
      if ((st = enqueue_cycle()) != GILA_OK) return st;
      return record(enq, Ph::Cycle);
    }
    for (const auto& q : sl_) any_copy |= q.state == 2;
    if (any_copy) return record(enq, Ph::Idle);
    ph_ = Ph::Idle;
    return GILA_OK;
  }

 private:
  enum class Ph { Idle, Init, Cycle, Update };
  struct Slot {
    int state = 0;  // 0 free, 1 assigned, 2 solution copy in flight
    bool fresh = false;       // norms of b not yet known
    bool need_start = false;  // (re)start the Krylov process from r64
    bool iter = false;        // Krylov process running
    bool pending = false;     // the Krylov iterate holds a correction not yet in x64
    bool broke = false;
    bool in_upd = false;      // part of the reliable update in flight
    double bn = 0, rn = 0, scale = 0, maxr = 0;
    int restarts = 0, cycles = 0, updates = 0, mv = 0;
    int since_upd = 0;  // cycles since the last reliable update or (re)start
    SlotOpts o;
    void* x_out = nullptr;
    uint64_t tag = 0;
    SlotResult res{};
  };

  size_t pb_bytes() const { return (5 * sizeof(double) + sizeof(int)) * (size_t)S_; }
  double* pd(int k) const { return reinterpret_cast<double*>(pb_d_) + (size_t)k * S_; }
  double* ph(int k) const { return reinterpret_cast<double*>(pb_h_) + (size_t)k * S_; }
  int* mask_d() const { return reinterpret_cast<int*>(pb_d_ + 5 * sizeof(double) * S_); }
  int* mask_h() const { return reinterpret_cast<int*>(pb_h_ + 5 * sizeof(double) * S_); }
  int64_t chi_rs() const { return cfg_.chi_shared ? 0 : V_; }
  bool done(const Slot& q) const { return q.bn == 0.0 || q.rn <= q.o.tol * q.bn; }

  gila_status record(bool* enq, Ph p) {
    GILA_CUDA_TRY(cudaEventRecord(ev_, s_));
    in_flight_ = true;
    ph_ = p;
    *enq = true;
    return GILA_OK;
  }

  gila_status load_chi(int r, const void* chi) {
    double2* c64 = chi64_ + (size_t)r * V_;
    GILA_CUDA_TRY(cudaMemcpyAsync(c64, chi, V_ * sizeof(double2), cudaMemcpyDefault, s_));
    if (cfg_.mixed) {
      k_cast<CI><<<vec_blocks(V_), kT, 0, s_>>>(c64, chii_ + (size_t)r * V_, V_);
      GILA_CUDA_TRY(cudaGetLastError());
    }
    return GILA_OK;
  }

  gila_status upload_params() {
    GILA_CUDA_TRY(cudaMemcpyAsync(pb_d_, pb_h_, pb_bytes(), cudaMemcpyHostToDevice, s_));
    return GILA_OK;
  }
  gila_status upload_status() {
    GILA_CUDA_TRY(cudaMemcpyAsync(st_d_, st_h_, (size_t)S_ * sizeof(Stat), cudaMemcpyHostToDevice, s_));
    return GILA_OK;
  }

  // squared norms (partials in part_) -> pd(k) -> ph(k) after the step
  gila_status fin_norms(int k) {
    k_fin<<<S_, kT, 0, s_>>>(part_, 1, nb_, sc_, 0, st_d_, pd(0), FIN_NORM, pd(k));
    GILA_CUDA_TRY(cudaGetLastError());
    GILA_CUDA_TRY(cudaMemcpyAsync(ph(k), pd(k), S_ * sizeof(double), cudaMemcpyDeviceToHost, s_));
    return GILA_OK;
  }

  // out = G in over runs of the slots in m; with chi, the Lippmann-Schwinger
  // epilogue out = in - chi .* (G in) runs in the matvec's last pass
  template <typename C>
  gila_status apply_runs(const OpRef<C>& op, const C* in, C* out, const std::vector<char>& m,
                         const C* chi = nullptr) {
    C one, zero;  // host side: no device helpers here
    one.x = 1;
    one.y = 0;
    zero.x = 0;
    zero.y = 0;
    for (auto [r0, r1] : runs_of(m, op.cap)) {
      LsEpi<C> ep{in + (size_t)r0 * n_, chi ? chi + (size_t)r0 * chi_rs() : nullptr, chi_rs()};
      GILA_CUDA_TRY(launch_matvec<C>(op.geom, devop<C>(*op.core), op.launch, in + (size_t)r0 * n_,
                                     out + (size_t)r0 * n_, op.A, op.B, r1 - r0, false, one, zero, s_,
                                     chi ? &ep : nullptr));
    }
    return GILA_OK;
  }

  // r64 = b - A64 x64 for the slots in m, squared norms into pd(3) -> ph(3)
  gila_status true_residual(const std::vector<char>& m) {
    gila_status st;
    if ((st = apply_runs<double2>(op64_, x64_, r64_, m)) != GILA_OK) return st;
    k_resid<<<dim3(nb_, S_), kT, 0, s_>>>(b64_, x64_, r64_, chi64_, chi_rs(), V_, mask_d(), part_);
    GILA_CUDA_TRY(cudaGetLastError());
    ++inf_.matvecs_f64;
    return fin_norms(3);
  }

  void finish(int r, bool converged) {
    Slot& q = sl_[r];
    q.iter = false;
    q.need_start = false;
    st_h_[r].act = 0;
    q.res = SlotResult{r, q.tag, q.bn == 0.0 ? 0.0 : q.rn / q.bn, converged ? 1 : 0, q.cycles, q.updates,
                       q.broke ? 1 : 0};
    cudaMemcpyAsync(q.x_out, x64_ + (size_t)r * n_, n_ * sizeof(double2), cudaMemcpyDefault, s_);
    q.state = 2;
  }

  // fresh slots: |b|^2 (pd(4)), and for an initial guess r = b - A x (pd(3))
  gila_status enqueue_init() {
    int* mh = mask_h();
    std::vector<char> mx(S_, 0);
    bool any_x0 = false;
    for (int r = 0; r < S_; ++r) {
      const Slot& q = sl_[r];
      mh[r] = q.state == 1 && q.fresh;
      mx[r] = mh[r] && q.o.x0;
      any_x0 |= mx[r] != 0;
      if (mh[r] && !q.o.x0)
        GILA_CUDA_TRY(cudaMemcpyAsync(r64_ + (size_t)r * n_, b64_ + (size_t)r * n_, n_ * sizeof(double2),
                                      cudaMemcpyDeviceToDevice, s_));
    }
    gila_status st;
    if ((st = upload_params()) != GILA_OK) return st;
    k_norm2<<<dim3(nb_, S_), kT, 0, s_>>>(b64_, n_, mask_d(), part_);
    GILA_CUDA_TRY(cudaGetLastError());
    if ((st = fin_norms(4)) != GILA_OK) return st;
    if (any_x0) {
      // the residual of the initial guesses, for those slots only
      for (int r = 0; r < S_; ++r) mh[r] = mx[r];
      if ((st = upload_params()) != GILA_OK) return st;
      if ((st = true_residual(mx)) != GILA_OK) return st;
    }
    return GILA_OK;
  }

  void digest_init() {
    for (int r = 0; r < S_; ++r) {
      Slot& q = sl_[r];
      if (!(q.state == 1 && q.fresh)) continue;
      q.fresh = false;
      q.bn = std::sqrt(ph(4)[r]);
      q.rn = q.o.x0 ? std::sqrt(ph(3)[r]) : q.bn;
      if (done(q))
        finish(r, true);
      else if (!std::isfinite(q.rn))
        finish(r, false);
      else
        q.need_start = true;
    }
  }

  gila_status enqueue_starts() {
    int* mh = mask_h();
    int nstart = 0;
    for (int r = 0; r < S_; ++r) {
      Slot& q = sl_[r];
      mh[r] = 0;
      if (q.state != 1 || !q.need_start) continue;
      q.need_start = false;
      ++q.restarts;
      q.iter = true;
      q.scale = q.rn;
      q.maxr = 1.0;
      st_h_[r] = Stat{1.0, 1, 0};
      mh[r] = 1;
      ++nstart;
    }
    if (!nstart) return GILA_OK;
    for (int r = 0; r < S_; ++r) {
      const Slot& q = sl_[r];
      const bool live = q.state == 1 && q.iter;
      const double t = live ? 0.9 * q.o.tol * q.bn / q.scale : 0.0;
      ph(0)[r] = t * t;
      ph(1)[r] = live ? q.scale : 0.0;
      ph(2)[r] = live ? 1.0 / q.scale : 0.0;
    }
    gila_status st;
    if ((st = upload_params()) != GILA_OK) return st;
    if ((st = upload_status()) != GILA_OK) return st;
    GILA_VW(k_inner_start, dim3(nb_, S_), r64_, kv_, pd(2), mask_d(), n_);
    k_scal_init<<<(S_ + 127) / 128, 128, 0, s_>>>(sc_, mask_d(), S_);
    GILA_CUDA_TRY(cudaGetLastError());
    return GILA_OK;
  }

  // One BiCGStab(l) cycle for the slots in `m` (matvecs over their runs; the
  // vector kernels over the iterating slots only, and skip slots retired
  // during the cycle), ending with the copy of the per-slot status to the
  // host.
  gila_status body(const std::vector<char>& m) {
    // the vector kernels run one block row per iterating slot (act_d_ maps
    // row -> slot, written by enqueue_cycle for this pattern of slots): a
    // batch with few of its slots iterating launches no blocks for the rest
    int na = 0;
    for (char c : m) na += c != 0;
    if (na == 0) return GILA_OK;
    const dim3 gv(nb_, na);
    const int* act = act_d_;
    const int sb = (S_ + 127) / 128;
    double* tol2 = pd(0);
    gila_status st;
    const int ell = cfg_.ell;
    auto lsa = [&](const CI* in, CI* out) -> gila_status { return apply_runs<CI>(opi_, in, out, m, chii_); };
    k_iter_start<<<sb, 128, 0, s_>>>(sc_, st_d_, S_);
    for (int j = 1; j <= ell; ++j) {
      GILA_VW(k_sdot, gv, shadow_, kv_.r[j - 1], n_, part_, act);
      k_fin<<<na, kT, 0, s_>>>(part_, 1, nb_, sc_, S_RHO, st_d_, tol2, FIN_CHECK, nullptr, act);
      GILA_VW(k_bicg_u, gv, kv_, j, n_, sc_, st_d_, act);
      GILA_CUDA_TRY(cudaGetLastError());
      if ((st = lsa(kv_.u[j - 1], kv_.u[j])) != GILA_OK) return st;
      GILA_VW(k_sdot, gv, shadow_, kv_.u[j], n_, part_, act);
      k_fin<<<na, kT, 0, s_>>>(part_, 1, nb_, sc_, S_SIG, st_d_, tol2, FIN_CHECK, nullptr, act);
      GILA_VW(k_bicg_r, gv, kv_, j, n_, sc_, st_d_, part_, act);
      k_fin<<<na, kT, 0, s_>>>(part_, 1, nb_, sc_, 0, st_d_, tol2, FIN_RESID, nullptr, act);
      GILA_CUDA_TRY(cudaGetLastError());
      if ((st = lsa(kv_.r[j - 1], kv_.r[j])) != GILA_OK) return st;
    }
    GILA_VW(k_gram, gv, kv_, ell, n_, part_, act);
    k_fin<<<na, kT, 0, s_>>>(part_, kGram, nb_, sc_, S_GRAM, st_d_, tol2, FIN_STORE, nullptr, act);
    k_mr_solve<<<sb, 128, 0, s_>>>(sc_, st_d_, ell, S_);
    GILA_VW(k_mr_update, gv, kv_, ell, n_, sc_, st_d_, part_, act);
    k_fin<<<na, kT, 0, s_>>>(part_, 1, nb_, sc_, 0, st_d_, tol2, FIN_RESID, nullptr, act);
    GILA_CUDA_TRY(cudaGetLastError());
    GILA_CUDA_TRY(cudaMemcpyAsync(st_h_, st_d_, (size_t)S_ * sizeof(Stat), cudaMemcpyDeviceToHost, s_));
    return GILA_OK;
  }

  gila_status enqueue_cycle() {
    std::vector<char> m(S_, 0);
    for (int r = 0; r < S_; ++r) m[r] = sl_[r].state == 1 && sl_[r].iter;
    int na = 0;
    for (int r = 0; r < S_; ++r)
      if (m[r]) act_h_[na++] = r;
    if (na > 0) GILA_CUDA_TRY(cudaMemcpyAsync(act_d_, act_h_, (size_t)na * sizeof(int), cudaMemcpyHostToDevice, s_));
    std::vector<int> key;
    for (auto [r0, r1] : runs_of(m, S_)) {
      key.push_back(r0);
      key.push_back(r1);
    }
    // a pattern of iterating slots seen twice in a row is captured once and
    // replayed; the first cycle of a pattern runs directly (it also sets the
    // kernels' function attributes outside any capture)
    if (cfg_.graph && graph_ok_ && key != graph_key_ && key == last_key_) {
      if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
      }
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        const gila_status sb = body(m);
        e = cudaStreamEndCapture(s_, &g);
        if (sb == GILA_OK && e == cudaSuccess && g) e = cudaGraphInstantiate(&graph_, g, 0);
        if (g) cudaGraphDestroy(g);
        if (sb != GILA_OK || e != cudaSuccess) {
          graph_ = nullptr;
          graph_ok_ = false;
        } else {
          graph_key_ = key;
        }
      } else {
        graph_ok_ = false;
      }
      cudaGetLastError();
    }
    last_key_ = key;
    ++inf_.iters;
    if (cfg_.mixed)
      inf_.matvecs_f32 += 2 * cfg_.ell;
    else
      inf_.matvecs_f64 += 2 * cfg_.ell;
    if (graph_ && key == graph_key_) {
      GILA_CUDA_TRY(cudaGraphLaunch(graph_, s_));
      return GILA_OK;
    }
    return body(m);
  }

  // after a cycle: per slot, a reliable update on breakdown, claimed
  // convergence, an exhausted matvec budget or (mixed) a recursive residual
  // below delta times its largest value since the last update
  gila_status digest_cycle(bool* upd) {
    *upd = false;
    const bool mixed = cfg_.mixed != 0;
    int* mh = mask_h();
    std::vector<char> m(S_, 0);
    const int mvc = 2 * cfg_.ell;
    for (int r = 0; r < S_; ++r) {
      Slot& q = sl_[r];
      mh[r] = 0;
      q.in_upd = false;
      if (!(q.state == 1 && q.iter)) continue;
      ++q.cycles;
      ++q.since_upd;
      q.mv += mvc;
      q.pending = true;
      const Stat& s = st_h_[r];
      const double nr = std::sqrt(s.nrm2);
      const bool budget = q.mv + mvc > q.o.max_mv;
      // a residual drop of delta triggers an update only kReliableGap cycles
      // after the last one: a system that converges by 10x per cycle would
      // otherwise pay one FP64 matvec per cycle of 2l ComplexF32 ones
      const bool drop = mixed && nr < q.o.delta * q.maxr && q.since_upd >= kReliableGap;
      if (s.broke || !s.act || budget || drop) {
        m[r] = 1;
        mh[r] = 1;
        q.in_upd = true;
      } else if (nr > q.maxr) {
        q.maxr = nr;
      }
    }
    bool any = false;
    for (char c : m) any |= c != 0;
    if (!any) return GILA_OK;
    gila_status st;
    if ((st = upload_params()) != GILA_OK) return st;
    GILA_VW(k_accum, dim3(nb_, S_), x64_, kv_.x, pd(1), mask_d(), n_);
    GILA_CUDA_TRY(cudaGetLastError());
    if ((st = true_residual(m)) != GILA_OK) return st;
    GILA_VW(k_replace, dim3(nb_, S_), r64_, kv_.r[0], pd(2), mask_d(), n_);
    GILA_CUDA_TRY(cudaGetLastError());
    ++inf_.outer;
    *upd = true;
    return GILA_OK;
  }

  gila_status digest_update() {
    const int mvc = 2 * cfg_.ell;
    for (int r = 0; r < S_; ++r) {
      Slot& q = sl_[r];
      if (!q.in_upd) continue;
      q.in_upd = false;
      q.pending = false;
      q.since_upd = 0;
      ++q.updates;
      q.rn = std::sqrt(ph(3)[r]);
      Stat& s = st_h_[r];
      q.broke |= s.broke != 0;
      if (done(q)) {
        finish(r, true);
      } else if (q.mv + mvc > q.o.max_mv || !std::isfinite(q.rn)) {
        finish(r, false);
      } else if (s.broke || !s.act) {
        // breakdown, or convergence the FP64 residual does not confirm:
        // restart from the FP64 residual
        q.iter = false;
        s.act = 0;
        if (q.restarts >= q.o.max_restarts)
          finish(r, false);
        else
          q.need_start = true;
      } else {
        q.maxr = q.rn / q.scale;
        s.nrm2 = q.maxr * q.maxr;
      }
    }
    return upload_status();
  }

  Core& g64_;
  Core& gi_;
  int S_;
  int64_t n_, V_;
  BatchCfg cfg_;
  int nb_ = 1;
  bool w2_ = false;
  cudaStream_t s_ = nullptr;
  cudaEvent_t ev_ = nullptr;
  struct Arena : DevArena {
    void release() {
      for (void* p : d) cudaFree(p);
      for (void* p : h) cudaFreeHost(p);
      d.clear();
      h.clear();
    }
  } mem_;
  OpRef<double2> op64_{};
  OpRef<CI> opi_{};
  double2 *b64_ = nullptr, *x64_ = nullptr, *r64_ = nullptr, *chi64_ = nullptr;
  CI* chii_ = nullptr;
  double2 *part_ = nullptr, *sc_ = nullptr;
  Stat *st_d_ = nullptr, *st_h_ = nullptr;
  char *pb_d_ = nullptr, *pb_h_ = nullptr;
  // iterating slots of the cycle in flight, in slot order (row -> slot map
  // of the cycle's vector kernels); the host copy is rewritten only after the
  // previous cycle has completed
  int *act_d_ = nullptr, *act_h_ = nullptr;
  KVec<CI> kv_{};
  CI* shadow_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  std::vector<int> graph_key_, last_key_;
  bool graph_ok_ = true;
  std::vector<Slot> sl_;
  Ph ph_ = Ph::Idle;
  bool in_flight_ = false;
  gila_solve_info inf_{};
  std::vector<SlotResult> finished_;
};

}  // namespace

bool same_volume(const Core& a, const Core& b) {
  for (int k = 0; k < 3; ++k)
    if (a.geom.sc[k] != b.geom.sc[k] || a.geom.tc[k] != b.geom.tc[k]) return false;
  return a.geom.parT == b.geom.parT && a.parS == b.parS;
}

gila_status check_ls_operator(const Core& a) {
  if (a.dtype != GILA_C128) return fail(GILA_ERR_TYPE, "the residual operator must be ComplexF64");
  if (!a.self || a.geom.parT != 1 || a.parS != 1 || in_elems(a) != out_elems(a))
    return fail(GILA_ERR_SIZE, "Green's operator and medium must have the same size (a self operator).");
  return GILA_OK;
}

size_t ls_batch_bytes(const Core& g64, const Core* g32, int slots, const BatchCfg& cfg) {
  if (cfg.mixed && g32) return LsBatchT<float2>::bytes(g64, *g32, slots, cfg);
  return LsBatchT<double2>::bytes(g64, g64, slots, cfg);
}

gila_status make_ls_batch(Core& g64, Core* g32, int slots, const BatchCfg& cfg, std::unique_ptr<LsBatch>& out) {
  gila_status s = check_ls_operator(g64);
  if (s != GILA_OK) return s;
  if (slots < 1 || slots > 65535) return fail(GILA_ERR_ARG, "slots must be in 1..65535");
  if (cfg.ell < 1 || cfg.ell > kMaxEll) return fail(GILA_ERR_ARG, "BiCGStab(l) degree must be 1..4");
  // launch shapes of the operators for one vector (timed once per geometry,
  // cached): the batch's own choice when it does not time its chunks
  for (Core* c : {&g64, g32}) {
    if (!c || c->tuned || cfg.tune) continue;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((s = ensure_tuned(*c, 1)) != GILA_OK) return s;
  }
  if (cfg.mixed) {
    if (!g32) return fail(GILA_ERR_ARG, "the mixed solve needs the ComplexF32 operator");
    if (g32->dtype != GILA_C64) return fail(GILA_ERR_TYPE, "the inner operator must be ComplexF32");
    if (!same_volume(g64, *g32) || g32->device != g64.device)
      return fail(GILA_ERR_SIZE, "the two operators describe different volumes");
    auto b = std::make_unique<LsBatchT<float2>>(g64, *g32, slots, cfg);
    if ((s = b->init()) != GILA_OK) return s;
    out = std::move(b);
  } else {
    auto b = std::make_unique<LsBatchT<double2>>(g64, g64, slots, cfg);
    if ((s = b->init()) != GILA_OK) return s;
    out = std::move(b);
  }
  return GILA_OK;
}

namespace {
template <typename C>
__global__ void k_cast_any(const void* __restrict__ a, int a_f64, C* __restrict__ b, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double2 v;
    if (a_f64) {
      v = static_cast<const double2*>(a)[i];
    } else {
      const float2 f = static_cast<const float2*>(a)[i];
      v = make_double2(f.x, f.y);
    }
    b[i] = from_d<C>(v);
  }
}

}  // namespace

gila_status cast_core(gila_ctx* ctx, Core& c, gila_dtype dtype, std::shared_ptr<Core>& core) {
  if (dtype != GILA_C64 && dtype != GILA_C128) return fail(GILA_ERR_TYPE, "setTyp must be ComplexF32 or ComplexF64");
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  const gila_vol trg = vol_to_abi(c.trg), src = vol_to_abi(c.src);
  gila_status s = init_core(ctx, &trg, c.self ? nullptr : &src, &c.opt, dtype, core);
  if (s != GILA_OK) return s;
  const int64_t elems = (int64_t)(c.ker_bytes / csize(c.dtype));
  core->ker_bytes = (size_t)elems * csize(dtype);
  GILA_CUDA_TRY(dev_malloc(&core->ker, core->ker_bytes));
  const int blocks = (int)std::min<int64_t>((elems + 255) / 256, 148 * 16);
  if (dtype == GILA_C128)
    k_cast_any<double2><<<blocks, 256, 0, c.stream>>>(c.ker, c.dtype == GILA_C128, static_cast<double2*>(core->ker),
                                                       elems);
  else
    k_cast_any<float2><<<blocks, 256, 0, c.stream>>>(c.ker, c.dtype == GILA_C128, static_cast<float2*>(core->ker),
                                                      elems);
  GILA_CUDA_TRY(cudaGetLastError());
  GILA_CUDA_TRY(cudaStreamSynchronize(c.stream));
  return GILA_OK;
}

// NaN / Inf in a solve's inputs.  A non-finite medium or incident field
// would otherwise surface only as breakdowns and restarts until the matvec
// budget runs out; the reference's LippmannSchwinger has no check of its own,
// the kernel build checks its output (src/glaMemSup.jl:93-95) and this check
// extends that rule to the solve's inputs.
__global__ void k_nonfinite(const double* __restrict__ p, int64_t n, int* __restrict__ flag) {
  int bad = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    bad |= !isfinite(p[i]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

gila_status check_finite(const void* p, int64_t n_complex, const char* what) {
  const double* d = static_cast<const double*>(p);
  const int64_t n = 2 * n_complex;
  bool bad = false;
  if (!is_device_ptr(p)) {
    for (int64_t i = 0; i < n; ++i)
      if (!std::isfinite(d[i])) {
        bad = true;
        break;
      }
  } else {
    int* flag = nullptr;
    GILA_CUDA_TRY(dev_malloc(&flag, sizeof(int)));
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    int h = 0;
    if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(int), st);
    if (e == cudaSuccess) {
      k_nonfinite<<<1184, 256, 0, st>>>(d, n, flag);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (st) cudaStreamDestroy(st);
    cudaFree(flag);
    if (e != cudaSuccess) return cuda_fail(e, "finiteness check of solve inputs");
    bad = h != 0;
  }
  if (bad) return fail(GILA_ERR_NAN, std::string(what) + " contains non-numeric values.");
  return GILA_OK;
}

}  // namespace gila

using namespace gila;

extern "C" {

gila_status gila_opr_cast(gila_opr* opr, gila_dtype dtype, gila_opr** out) {
  if (!opr || !opr->core || !out) return fail(GILA_ERR_ARG, "null argument");
  std::shared_ptr<Core> core;
  gila_status s;
  {
    std::lock_guard<std::mutex> lk(opr->core->mu);
    if ((s = cast_core(opr->ctx, *opr->core, dtype, core)) != GILA_OK) return s;
  }
  auto* o = new gila_opr;
  o->ctx = opr->ctx;
  o->core = core;
  o->trg = opr->trg;
  o->src = opr->src;
  o->adj = opr->adj;
  *out = o;
  return GILA_OK;
}

gila_status gila_ls_solve(gila_opr* g64, gila_opr* g32, const void* chi, const void* b, void* x, int64_t nrhs,
                          const gila_solve_opts* opts, gila_solve_info* info, double* rhs_res, void* stream) {
  if (!g64 || !g64->core || !chi || !b || !x) return fail(GILA_ERR_ARG, "null argument");
  if (nrhs < 1 || nrhs > 65535) return fail(GILA_ERR_ARG, "nrhs must be in 1..65535");
  Core& a = *g64->core;
  gila_status s = check_ls_operator(a);
  if (s != GILA_OK) return s;
  BatchCfg cfg;
  SlotOpts so;
  cfg.ell = opts && opts->ell > 0 ? opts->ell : 2;
  cfg.mixed = opts ? (opts->mixed != 0) : 0;
  cfg.graph = opts ? (opts->no_graph == 0) : 1;
  cfg.chi_shared = 1;
  cfg.tune = 1;
  if (const char* ev = getenv("GILA_SOLVE_GRAPH"))
    if (ev[0] == '0') cfg.graph = 0;
  so.tol = opts && opts->tol > 0 ? opts->tol : 1e-6;
  so.max_mv = opts && opts->max_matvecs > 0 ? opts->max_matvecs : 4000;
  so.max_restarts = opts && opts->max_restarts > 0 ? opts->max_restarts : 20;
  so.delta = opts && opts->delta > 0 ? opts->delta : 0.1;
  so.x0 = opts ? (opts->x0 != 0) : 0;
  if (cfg.ell > 4) return fail(GILA_ERR_ARG, "BiCGStab(l) degree must be 1..4");
  Core* inner = nullptr;
  if (cfg.mixed) {
    if (!g32 || !g32->core) return fail(GILA_ERR_ARG, "the mixed solve needs the ComplexF32 operator");
    inner = g32->core.get();
  }
  GILA_CUDA_TRY(cudaSetDevice(a.device));
  if ((s = check_finite(chi, in_elems(a) / 3, "The medium (chi)")) != GILA_OK) return s;
  if ((s = check_finite(b, in_elems(a) * nrhs, "The incident field (b)")) != GILA_OK) return s;
  const bool keep = opts && opts->keep;
  char key[160];
  snprintf(key, sizeof key, "%p|%d|%d|%d|%d|%lld", (void*)inner, cfg.ell, cfg.mixed, cfg.graph, cfg.chi_shared,
           (long long)nrhs);
  std::shared_ptr<LsBatch> bt;
  std::shared_ptr<Core> innerp = cfg.mixed ? g32->core : nullptr;
  {
    std::lock_guard<std::mutex> lk(a.mu);
    if (a.ls_keep && a.ls_keep_key == key && a.ls_keep_inner.lock() == innerp) bt = a.ls_keep;
    a.ls_keep.reset();  // taken (or stale); put back below when kept
  }
  if (!bt) {
    std::unique_ptr<LsBatch> nb;
    if ((s = make_ls_batch(a, inner, (int)nrhs, cfg, nb)) != GILA_OK) return s;
    bt = std::move(nb);
  }
  bt->reset_info();
  cudaStream_t st = bt->stream();
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  cudaEvent_t ev = nullptr;
  // the ordering event is destroyed on every exit
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      if (*e) cudaEventDestroy(*e);
    }
  } ev_guard{&ev};
  if (user) {
    GILA_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    GILA_CUDA_TRY(cudaEventRecord(ev, user));
    GILA_CUDA_TRY(cudaStreamWaitEvent(st, ev, 0));
  }
  const int64_t n = in_elems(a);
  if ((s = bt->set_shared_chi(chi)) != GILA_OK) return s;
  for (int64_t r = 0; r < nrhs; ++r) {
    const void* br = static_cast<const double2*>(b) + r * n;
    void* xr = static_cast<double2*>(x) + r * n;
    if ((s = bt->assign((int)r, nullptr, br, xr, so, (uint64_t)r)) != GILA_OK) return s;
  }
  for (;;) {
    bool enq = false;
    if ((s = bt->advance(&enq)) != GILA_OK) break;
    if (!enq) break;
    if ((s = bt->wait()) != GILA_OK) break;
  }
  cudaStreamSynchronize(st);
  if (s != GILA_OK) return s;
  std::vector<SlotResult> fin = bt->take_finished();
  gila_solve_info inf = bt->info();
  inf.converged = 0;
  inf.breakdowns = 0;
  inf.rel_res = 0.0;
  std::vector<double> res(nrhs, 0.0);
  for (const SlotResult& q : fin) {
    res[q.slot] = q.rel_res;
    inf.converged += q.converged;
    inf.breakdowns += q.broke;
    inf.rel_res = std::isfinite(inf.rel_res) ? std::max(inf.rel_res, q.rel_res) : inf.rel_res;
    if (!std::isfinite(q.rel_res)) inf.rel_res = q.rel_res;
  }
  if ((int64_t)fin.size() != nrhs) return fail(GILA_ERR_INTERNAL, "a right-hand side was not reported");
  if (ev) {
    cudaEventRecord(ev, st);
    cudaStreamWaitEvent(user, ev, 0);
  }
  if (keep) {
    std::lock_guard<std::mutex> lk(a.mu);
    a.ls_keep = bt;
    a.ls_keep_key = key;
    a.ls_keep_inner = innerp;
  }
  if (info) *info = inf;
  if (rhs_res)
    for (int64_t r = 0; r < nrhs; ++r) rhs_res[r] = res[r];
  if (inf.converged < nrhs)
    return fail(GILA_ERR_NOTCONV, "the solve stopped at relative residual " + std::to_string(inf.rel_res) +
                                      " above the tolerance " + std::to_string(so.tol));
  return GILA_OK;
}

}  // extern "C"
