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
// part[r][0][blk] = sum_i conj(a_r[i]) b_r[i]  (a_rs = 0: one a for all r)
template <typename CA, typename CB>
__global__ void __launch_bounds__(kT) k_dot(const CA* __restrict__ a, int64_t a_rs, const CB* __restrict__ b,
                                            int64_t n, double2* __restrict__ part) {
  const int r = blockIdx.y, nb = gridDim.x;
  a += a_rs * r;
  b += n * r;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)nb * kT)
    acc[0] = cadd(acc[0], cjmul(to_d(a[i]), to_d(b[i])));
  block_sum_store<1>(acc, 1, part + (int64_t)r * nb + blockIdx.x, nb);
}

// Gram matrix r_a^H r_b, a <= b <= ell, of the MR step (all kGram slots).
template <typename C>
__global__ void __launch_bounds__(kT) k_gram(KVec<C> v, int ell, int64_t n, double2* __restrict__ part) {
  const int r = blockIdx.y, nb = gridDim.x;
  const int64_t off = (int64_t)r * n;
  double2 acc[kGram];
#pragma unroll
  for (int k = 0; k < kGram; ++k) acc[k] = make_double2(0.0, 0.0);
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)nb * kT) {
    double2 e[kMaxEll + 1];
#pragma unroll
    for (int a = 0; a <= kMaxEll; ++a) e[a] = a <= ell ? to_d(v.r[a][off + i]) : make_double2(0.0, 0.0);
#pragma unroll
    for (int a = 0; a <= kMaxEll; ++a)
#pragma unroll
      for (int b = a; b <= kMaxEll; ++b)
        if (b <= ell) acc[gidx(a, b)] = cadd(acc[gidx(a, b)], cjmul(e[a], e[b]));
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
                                            double* __restrict__ nrm_out = nullptr) {
  const int r = blockIdx.x;
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
// BiCG part, step j (1-based): u_q = r_q - beta u_q, q < j, beta = rho / sigma
template <typename C>
__global__ void __launch_bounds__(kT) k_bicg_u(KVec<C> v, int j, int64_t n, const double2* __restrict__ sc,
                                               const Stat* __restrict__ st) {
  const int r = blockIdx.y;
  if (!st[r].act) return;
  const double2 beta = cdiv(sc[(int64_t)r * kSlots + S_RHO], sc[(int64_t)r * kSlots + S_SIG]);
  const int64_t off = (int64_t)r * n;
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT)
#pragma unroll
    for (int q = 0; q < kMaxEll; ++q)
      if (q < j) v.u[q][off + i] = from_d<C>(csub(to_d(v.r[q][off + i]), cmul(beta, to_d(v.u[q][off + i]))));
}

// BiCG part, step j: r_q -= alpha u_{q+1}, q < j; x += alpha u_0; alpha =
// rho / sigma; and the partial of |r_0|^2.  A residual that a BiCG step
// already brought to tolerance ends the solve there: continuing the cycle
// would divide rounding noise by rounding noise (sigma of the next step is
// rho - beta * rho_prev; with chi = 0 the first step converges exactly).
template <typename C>
__global__ void __launch_bounds__(kT) k_bicg_r(KVec<C> v, int j, int64_t n, const double2* __restrict__ sc,
                                               const Stat* __restrict__ st, double2* __restrict__ part) {
  const int r = blockIdx.y, nb = gridDim.x;
  if (!st[r].act) return;
  const double2 alpha = cdiv(sc[(int64_t)r * kSlots + S_RHO], sc[(int64_t)r * kSlots + S_SIG]);
  const int64_t off = (int64_t)r * n;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)nb * kT) {
#pragma unroll
    for (int q = 0; q < kMaxEll; ++q)
      if (q < j) {
        const C t = from_d<C>(csub(to_d(v.r[q][off + i]), cmul(alpha, to_d(v.u[q + 1][off + i]))));
        v.r[q][off + i] = t;
        if (q == 0) acc[0].x += cabs2(to_d(t));
      }
    v.x[off + i] = from_d<C>(cadd(to_d(v.x[off + i]), cmul(alpha, to_d(v.u[0][off + i]))));
  }
  block_sum_store<1>(acc, 1, part + (int64_t)r * nb + blockIdx.x, nb);
}

// MR part: u_0 -= sum_k gamma_k u_k, x += sum_k gamma_k r_{k-1},
// r_0 -= sum_k gamma_k r_k (k = 1..l), and the partial of |r_0|^2.
template <typename C>
__global__ void __launch_bounds__(kT) k_mr_update(KVec<C> v, int ell, int64_t n, const double2* __restrict__ sc,
                                                  const Stat* __restrict__ st, double2* __restrict__ part) {
  const int r = blockIdx.y, nb = gridDim.x;
  if (!st[r].act) return;
  double2 g[kMaxEll];
#pragma unroll
  for (int k = 0; k < kMaxEll; ++k)
    g[k] = k < ell ? sc[(int64_t)r * kSlots + S_GAM + k] : make_double2(0.0, 0.0);
  const int64_t off = (int64_t)r * n;
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)nb * kT) {
    double2 u0 = to_d(v.u[0][off + i]), r0 = to_d(v.r[0][off + i]), x = to_d(v.x[off + i]);
    x = cadd(x, cmul(g[0], r0));
#pragma unroll
    for (int k = 1; k <= kMaxEll; ++k)
      if (k <= ell) {
        const double2 rk = to_d(v.r[k][off + i]);
        u0 = csub(u0, cmul(g[k - 1], to_d(v.u[k][off + i])));
        r0 = csub(r0, cmul(g[k - 1], rk));
        if (k < ell) x = cadd(x, cmul(g[k], rk));
      }
    v.u[0][off + i] = from_d<C>(u0);
    v.r[0][off + i] = from_d<C>(r0);
    v.x[off + i] = from_d<C>(x);
    const double2 r0s = to_d(from_d<C>(r0));
    acc[0].x += cabs2(r0s);
  }
  block_sum_store<1>(acc, 1, part + (int64_t)r * nb + blockIdx.x, nb);
}

// Lippmann-Schwinger combine after out = G in: out = in - chi .* out, chi per
// cell broadcast over the three components (examples/GilaOperators.jl:94).
template <typename C>
__global__ void __launch_bounds__(kT) k_ls_combine(const C* __restrict__ in, C* __restrict__ out,
                                                   const C* __restrict__ chi, int64_t V,
                                                   const Stat* __restrict__ st) {
  const int r = blockIdx.y;
  if (st && !st[r].act) return;
  in += 3 * V * r;
  out += 3 * V * r;
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < V; i += (int64_t)gridDim.x * kT) {
    const double2 c = to_d(chi[i]);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int64_t j = q * V + i;
      out[j] = from_d<C>(csub(to_d(in[j]), cmul(c, to_d(out[j]))));
    }
  }
}

// ------------------------------------------------- refinement (FP64) steps
// r = b - (x - chi .* t) with t = G x held in r on entry; partial |r|^2
// (masked right-hand sides only when mask is set).
__global__ void __launch_bounds__(kT) k_resid(const double2* __restrict__ b, const double2* __restrict__ x,
                                              double2* __restrict__ r, const double2* __restrict__ chi, int64_t V,
                                              const int* __restrict__ mask, double2* __restrict__ part) {
  const int q = blockIdx.y, nb = gridDim.x;
  if (mask && !mask[q]) return;
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
template <typename C>
__global__ void __launch_bounds__(kT) k_inner_start(const double2* __restrict__ r64, KVec<C> v,
                                                    const double* __restrict__ inv, const int* __restrict__ mask,
                                                    int64_t n) {
  const int r = blockIdx.y;
  if (!mask[r]) return;
  const double s = inv[r];
  const int64_t off = (int64_t)r * n;
  const C zero = from_d<C>(make_double2(0.0, 0.0));
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT) {
    const double2 a = r64[off + i];
    v.r[0][off + i] = from_d<C>(make_double2(a.x * s, a.y * s));
    v.u[0][off + i] = zero;
    v.x[off + i] = zero;
  }
}

// Reliable update, first half: x64 += s * d and d = 0 for the masked
// right-hand sides (the correction leaves the low-precision iterate).
template <typename C>
__global__ void __launch_bounds__(kT) k_accum(double2* __restrict__ x, C* __restrict__ d,
                                              const double* __restrict__ scale, const int* __restrict__ mask,
                                              int64_t n) {
  const int r = blockIdx.y;
  if (!mask[r]) return;
  const double s = scale[r];
  const int64_t off = (int64_t)r * n;
  const C zero = from_d<C>(make_double2(0.0, 0.0));
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT) {
    const double2 a = to_d(d[off + i]);
    x[off + i] = make_double2(x[off + i].x + s * a.x, x[off + i].y + s * a.y);
    d[off + i] = zero;
  }
}

// Reliable update, second half: the recursive residual of the masked
// right-hand sides is replaced by the FP64 one, r_0 = (b - A64 x) * inv.
template <typename C>
__global__ void __launch_bounds__(kT) k_replace(const double2* __restrict__ r64, C* __restrict__ r0,
                                                const double* __restrict__ inv, const int* __restrict__ mask,
                                                int64_t n) {
  const int r = blockIdx.y;
  if (!mask[r]) return;
  const double s = inv[r];
  const int64_t off = (int64_t)r * n;
  for (int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x; i < n; i += (int64_t)gridDim.x * kT) {
    const double2 a = r64[off + i];
    r0[off + i] = from_d<C>(make_double2(a.x * s, a.y * s));
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
    cudaError_t e = cudaMalloc(p, bytes < 256 ? 256 : bytes);
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

struct Opts {
  double tol, delta;
  int ell, mixed, max_mv, max_restarts, x0, graph;
};

// blocks per right-hand side of the vector kernels: a function of n only, so
// that the reduction order never depends on the batch
int vec_blocks(int64_t n) {
  int64_t b = (n + kT * 4 - 1) / (kT * 4);
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 1024));
}

template <typename C>
cudaError_t ls_apply(Core& c, const C* chi, const C* in, C* out, int nrhs, const Stat* st, int nbv,
                     cudaStream_t s) {
  C one, zero;
  one.x = 1;
  one.y = 0;
  zero.x = 0;
  zero.y = 0;
  cudaError_t e = launch_matvec<C>(c.geom, devop<C>(c), c.launch, in, out, static_cast<C*>(c.A),
                                   static_cast<C*>(c.B), nrhs, false, one, zero, s);
  if (e != cudaSuccess) return e;
  const int64_t V = in_elems(c) / 3;
  k_ls_combine<C><<<dim3(nbv, nrhs), kT, 0, s>>>(in, out, chi, V, st);
  return cudaGetLastError();
}

// One batched solve.  Per right-hand side r the host keeps |b|, the FP64
// residual norm, the scale s of the current Krylov process and the largest
// recursive residual since the last reliable update; the device keeps the
// Krylov vectors, the scalars and the status (act / broke / nrm2).
template <typename CI>
struct Solver {
  Core& g64;
  Core& gi;  // Krylov operator (g64 itself when plain)
  const double2* chi64;
  const CI* chii;
  const double2* b;
  double2* x;
  int nrhs;
  int64_t n;
  Opts o;
  cudaStream_t s;
  int nb;
  DevArena mem;
  double2 *r64 = nullptr, *part = nullptr, *sc = nullptr;
  Stat *st_d = nullptr, *st_h = nullptr;
  // parameter block [tol2 | scale | inv | nrm] doubles then [mask] ints,
  // mirrored in pinned host memory
  char *pb_d = nullptr, *pb_h = nullptr;
  KVec<CI> kv{};
  CI* shadow = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool graph_ok = true;
  gila_solve_info info{};

  Solver(Core& a, Core& i, const double2* c64, const CI* ci, const double2* bb, double2* xx, int nr, const Opts& oo,
         cudaStream_t ss)
      : g64(a), gi(i), chi64(c64), chii(ci), b(bb), x(xx), nrhs(nr), n(in_elems(a)), o(oo), s(ss) {
    nb = vec_blocks(n);
  }
  ~Solver() {
    if (graph) cudaGraphExecDestroy(graph);
  }
  double* pd(int k) const { return reinterpret_cast<double*>(pb_d) + (size_t)k * nrhs; }
  double* ph(int k) const { return reinterpret_cast<double*>(pb_h) + (size_t)k * nrhs; }
  int* mask_d() const { return reinterpret_cast<int*>(pb_d + 4 * sizeof(double) * nrhs); }
  int* mask_h() const { return reinterpret_cast<int*>(pb_h + 4 * sizeof(double) * nrhs); }
  size_t pb_bytes() const { return (4 * sizeof(double) + sizeof(int)) * (size_t)nrhs; }

  cudaError_t setup() {
    cudaError_t e;
    const size_t vb = (size_t)nrhs * n;
    if ((e = mem.alloc((void**)&r64, vb * sizeof(double2))) != cudaSuccess) return e;
    if ((e = mem.alloc((void**)&part, (size_t)nrhs * kGram * nb * sizeof(double2))) != cudaSuccess) return e;
    if ((e = mem.alloc((void**)&sc, (size_t)nrhs * kSlots * sizeof(double2))) != cudaSuccess) return e;
    if ((e = mem.alloc((void**)&st_d, (size_t)nrhs * sizeof(Stat))) != cudaSuccess) return e;
    if ((e = mem.alloc((void**)&pb_d, pb_bytes())) != cudaSuccess) return e;
    if ((e = mem.alloc_host((void**)&st_h, (size_t)nrhs * sizeof(Stat))) != cudaSuccess) return e;
    if ((e = mem.alloc_host((void**)&pb_h, pb_bytes())) != cudaSuccess) return e;
    memset(pb_h, 0, pb_bytes());
    memset(st_h, 0, (size_t)nrhs * sizeof(Stat));
    CI* base = nullptr;
    const int nvec = 2 * o.ell + 3;
    if ((e = mem.alloc((void**)&base, (size_t)nvec * vb * sizeof(CI))) != cudaSuccess) return e;
    if ((e = mem.alloc((void**)&shadow, (size_t)n * sizeof(CI))) != cudaSuccess) return e;
    kv.x = base;
    for (int k = 0; k <= o.ell; ++k) {
      kv.r[k] = base + (size_t)(1 + k) * vb;
      kv.u[k] = base + (size_t)(2 + o.ell + k) * vb;
    }
    for (int k = o.ell + 1; k <= kMaxEll; ++k) kv.r[k] = kv.u[k] = nullptr;
    kv.shadow = shadow;
    // every Krylov vector starts finite, including those of right-hand sides
    // that never iterate (their matvecs still run inside the batch)
    if ((e = cudaMemsetAsync(base, 0, (size_t)nvec * vb * sizeof(CI), s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(st_d, st_h, (size_t)nrhs * sizeof(Stat), cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return e;
    k_shadow<CI><<<nb, kT, 0, s>>>(shadow, n, 0x5EEDull);
    return cudaGetLastError();
  }

  // squared norms of the nrhs vectors whose partials are in `part` -> host
  cudaError_t fetch_norms(std::vector<double>& out) {
    k_fin<<<nrhs, kT, 0, s>>>(part, 1, nb, sc, 0, st_d, pd(0), FIN_NORM, pd(3));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(ph(3), pd(3), nrhs * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    out.assign(ph(3), ph(3) + nrhs);
    return cudaSuccess;
  }

  // r64 = b - A64 x for the right-hand sides set in mask_h (all when null):
  // one batched FP64 matvec per run of consecutive masked right-hand sides.
  // Returns |r|^2 per right-hand side (entries of unmasked ones undefined).
  cudaError_t true_residual(std::vector<double>& rn2, const int* mh) {
    cudaError_t e;
    const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
    for (int r0 = 0; r0 < nrhs;) {
      if (mh && !mh[r0]) {
        ++r0;
        continue;
      }
      int r1 = r0 + 1;
      while (r1 < nrhs && (!mh || mh[r1])) ++r1;
      e = launch_matvec<double2>(g64.geom, devop<double2>(g64), g64.launch, x + (size_t)r0 * n, r64 + (size_t)r0 * n,
                                 static_cast<double2*>(g64.A), static_cast<double2*>(g64.B), r1 - r0, false, one,
                                 zero, s);
      if (e != cudaSuccess) return e;
      r0 = r1;
    }
    k_resid<<<dim3(nb, nrhs), kT, 0, s>>>(b, x, r64, chi64, n / 3, mh ? mask_d() : nullptr, part);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    ++info.matvecs_f64;
    return fetch_norms(rn2);
  }

  // Reliable update of the masked right-hand sides (mask_h set by the
  // caller): x64 += s d, d = 0, FP64 residual, r_0 = r64 / s.
  cudaError_t reliable_update(std::vector<double>& rn2) {
    cudaError_t e;
    if ((e = cudaMemcpyAsync(pb_d, pb_h, pb_bytes(), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    k_accum<CI><<<dim3(nb, nrhs), kT, 0, s>>>(x, kv.x, pd(1), mask_d(), n);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = true_residual(rn2, mask_h())) != cudaSuccess) return e;
    k_replace<CI><<<dim3(nb, nrhs), kT, 0, s>>>(r64, kv.r[0], pd(2), mask_d(), n);
    ++info.outer;
    return cudaGetLastError();
  }

  // One BiCGStab(l) cycle for every active right-hand side, ending with the
  // copy of the per-rhs status to the host.
  cudaError_t body() {
    cudaError_t e;
    const dim3 gv(nb, nrhs);
    const int sb = (nrhs + 127) / 128;
    double* tol2 = pd(0);
    k_iter_start<<<sb, 128, 0, s>>>(sc, st_d, nrhs);
    for (int j = 1; j <= o.ell; ++j) {
      k_dot<CI, CI><<<gv, kT, 0, s>>>(shadow, 0, kv.r[j - 1], n, part);
      k_fin<<<nrhs, kT, 0, s>>>(part, 1, nb, sc, S_RHO, st_d, tol2, FIN_CHECK);
      k_bicg_u<CI><<<gv, kT, 0, s>>>(kv, j, n, sc, st_d);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if ((e = ls_apply<CI>(gi, chii, kv.u[j - 1], kv.u[j], nrhs, st_d, nb, s)) != cudaSuccess) return e;
      k_dot<CI, CI><<<gv, kT, 0, s>>>(shadow, 0, kv.u[j], n, part);
      k_fin<<<nrhs, kT, 0, s>>>(part, 1, nb, sc, S_SIG, st_d, tol2, FIN_CHECK);
      k_bicg_r<CI><<<gv, kT, 0, s>>>(kv, j, n, sc, st_d, part);
      k_fin<<<nrhs, kT, 0, s>>>(part, 1, nb, sc, 0, st_d, tol2, FIN_RESID);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if ((e = ls_apply<CI>(gi, chii, kv.r[j - 1], kv.r[j], nrhs, st_d, nb, s)) != cudaSuccess) return e;
    }
    k_gram<CI><<<gv, kT, 0, s>>>(kv, o.ell, n, part);
    k_fin<<<nrhs, kT, 0, s>>>(part, kGram, nb, sc, S_GRAM, st_d, tol2, FIN_STORE);
    k_mr_solve<<<sb, 128, 0, s>>>(sc, st_d, o.ell, nrhs);
    k_mr_update<CI><<<gv, kT, 0, s>>>(kv, o.ell, n, sc, st_d, part);
    k_fin<<<nrhs, kT, 0, s>>>(part, 1, nb, sc, 0, st_d, tol2, FIN_RESID);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaMemcpyAsync(st_h, st_d, nrhs * sizeof(Stat), cudaMemcpyDeviceToHost, s);
  }

  cudaError_t iterate(bool first) {
    if (o.graph && graph_ok && !graph && !first) {
      // the first cycle ran directly (function attributes are set); capture the next
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t eb = body();
        e = cudaStreamEndCapture(s, &g);
        if (eb == cudaSuccess && e == cudaSuccess && g) e = cudaGraphInstantiate(&graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (eb != cudaSuccess || e != cudaSuccess) {
          graph = nullptr;
          graph_ok = false;
        }
      } else {
        graph_ok = false;
      }
      cudaGetLastError();
    }
    if (graph) return cudaGraphLaunch(graph, s);
    return body();
  }

  cudaError_t run(std::vector<double>& res) {
    cudaError_t e;
    const size_t vb = (size_t)nrhs * n;
    std::vector<double> bn2, rn2;
    k_dot<double2, double2><<<dim3(nb, nrhs), kT, 0, s>>>(b, n, b, n, part);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = fetch_norms(bn2)) != cudaSuccess) return e;
    if (o.x0) {
      if ((e = true_residual(rn2, nullptr)) != cudaSuccess) return e;
    } else {
      if ((e = cudaMemsetAsync(x, 0, vb * sizeof(double2), s)) != cudaSuccess) return e;
      if ((e = cudaMemcpyAsync(r64, b, vb * sizeof(double2), cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return e;
      rn2 = bn2;
    }
    std::vector<double> bn(nrhs), rn(nrhs), scale(nrhs, 0.0), maxr(nrhs, 0.0);
    std::vector<char> live(nrhs, 0), restart(nrhs, 0), broke(nrhs, 0), pending(nrhs, 0);
    std::vector<int> restarts(nrhs, 0);
    for (int r = 0; r < nrhs; ++r) {
      bn[r] = std::sqrt(bn2[r]);
      rn[r] = std::sqrt(rn2[r]);
    }
    auto done = [&](int r) { return bn[r] == 0.0 || rn[r] <= o.tol * bn[r]; };
    for (int r = 0; r < nrhs; ++r) restart[r] = !done(r) && std::isfinite(rn[r]);
    const double delta = o.mixed ? o.delta : 0.0;
    const int mv_iter = 2 * o.ell;
    int mv = 0;
    int* mh = mask_h();
    for (;;) {
      // (re)start the Krylov processes that need it, on A d = r / |r|
      int nstart = 0;
      for (int r = 0; r < nrhs; ++r) {
        mh[r] = 0;
        if (!restart[r]) continue;
        restart[r] = 0;
        if (restarts[r] >= o.max_restarts) continue;
        ++restarts[r];
        mh[r] = 1;
        ++nstart;
        live[r] = 1;
        scale[r] = rn[r];
        maxr[r] = 1.0;
        st_h[r].nrm2 = 1.0;
        st_h[r].act = 1;
        st_h[r].broke = 0;
      }
      if (nstart) {
        for (int r = 0; r < nrhs; ++r) {
          const double t = live[r] ? 0.9 * o.tol * bn[r] / scale[r] : 0.0;
          ph(0)[r] = t * t;
          ph(1)[r] = live[r] ? scale[r] : 0.0;
          ph(2)[r] = live[r] ? 1.0 / scale[r] : 0.0;
        }
        if ((e = cudaMemcpyAsync(pb_d, pb_h, pb_bytes(), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(st_d, st_h, nrhs * sizeof(Stat), cudaMemcpyHostToDevice, s)) != cudaSuccess)
          return e;
        k_inner_start<CI><<<dim3(nb, nrhs), kT, 0, s>>>(r64, kv, pd(2), mask_d(), n);
        k_scal_init<<<(nrhs + 127) / 128, 128, 0, s>>>(sc, mask_d(), nrhs);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
      int nlive = 0;
      for (int r = 0; r < nrhs; ++r) nlive += live[r];
      if (nlive == 0 || mv + mv_iter > o.max_mv) break;
      // one cycle; its status copy is read after the sync
      if ((e = iterate(info.iters == 0)) != cudaSuccess) return e;
      if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
      mv += mv_iter;
      ++info.iters;
      if (o.mixed)
        info.matvecs_f32 += mv_iter;
      else
        info.matvecs_f64 += mv_iter;
      // reliable updates: breakdown, claimed convergence, or (mixed) a
      // recursive residual below delta times its largest value since the last
      int nupd = 0;
      for (int r = 0; r < nrhs; ++r) {
        mh[r] = 0;
        if (!live[r]) continue;
        pending[r] = 1;
        const Stat& q = st_h[r];
        const double nr = std::sqrt(q.nrm2);
        if (q.broke || !q.act || nr < delta * maxr[r]) {
          mh[r] = 1;
          ++nupd;
        } else if (nr > maxr[r]) {
          maxr[r] = nr;
        }
      }
      if (nupd == 0) continue;
      if ((e = reliable_update(rn2)) != cudaSuccess) return e;
      for (int r = 0; r < nrhs; ++r) {
        if (!mh[r]) continue;
        pending[r] = 0;
        rn[r] = std::sqrt(rn2[r]);
        Stat& q = st_h[r];
        broke[r] |= (char)q.broke;
        if (done(r)) {
          live[r] = 0;
          q.act = 0;
        } else if (q.broke || !q.act || !std::isfinite(rn[r])) {
          // breakdown, or convergence the FP64 residual does not confirm:
          // restart from the FP64 residual
          live[r] = 0;
          q.act = 0;
          restart[r] = std::isfinite(rn[r]);
        } else {
          maxr[r] = rn[r] / scale[r];
          q.nrm2 = maxr[r] * maxr[r];
        }
      }
      if ((e = cudaMemcpyAsync(st_d, st_h, nrhs * sizeof(Stat), cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    }
    // fold the corrections still held by the Krylov iterates into x
    int npend = 0;
    for (int r = 0; r < nrhs; ++r) {
      mh[r] = pending[r];
      npend += pending[r];
    }
    if (npend) {
      if ((e = reliable_update(rn2)) != cudaSuccess) return e;
      for (int r = 0; r < nrhs; ++r)
        if (pending[r]) rn[r] = std::sqrt(rn2[r]);
    }
    res.resize(nrhs);
    info.converged = 0;
    info.rel_res = 0.0;
    info.breakdowns = 0;
    for (int r = 0; r < nrhs; ++r) {
      res[r] = bn[r] == 0.0 ? 0.0 : rn[r] / bn[r];
      info.rel_res = std::max(info.rel_res, res[r]);
      if (!std::isfinite(res[r])) info.rel_res = res[r];
      info.converged += done(r) ? 1 : 0;
      info.breakdowns += broke[r] ? 1 : 0;
    }
    return cudaSuccess;
  }
};

bool same_volume(const Core& a, const Core& b) {
  for (int k = 0; k < 3; ++k)
    if (a.geom.sc[k] != b.geom.sc[k] || a.geom.tc[k] != b.geom.tc[k]) return false;
  return a.geom.parT == b.geom.parT && a.parS == b.parS;
}

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
}  // namespace gila

using namespace gila;

extern "C" {

gila_status gila_opr_cast(gila_opr* opr, gila_dtype dtype, gila_opr** out) {
  if (!opr || !opr->core || !out) return fail(GILA_ERR_ARG, "null argument");
  if (dtype != GILA_C64 && dtype != GILA_C128) return fail(GILA_ERR_TYPE, "setTyp must be ComplexF32 or ComplexF64");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  const gila_vol trg = vol_to_abi(c.trg), src = vol_to_abi(c.src);
  std::shared_ptr<Core> core;
  gila_status s = init_core(opr->ctx, &trg, c.self ? nullptr : &src, &c.opt, dtype, core);
  if (s != GILA_OK) return s;
  const int64_t elems = (int64_t)(c.ker_bytes / csize(c.dtype));
  core->ker_bytes = (size_t)elems * csize(dtype);
  GILA_CUDA_TRY(cudaMalloc(&core->ker, core->ker_bytes));
  const int blocks = (int)std::min<int64_t>((elems + 255) / 256, 148 * 16);
  if (dtype == GILA_C128)
    k_cast_any<double2><<<blocks, 256, 0, c.stream>>>(c.ker, c.dtype == GILA_C128, static_cast<double2*>(core->ker),
                                                       elems);
  else
    k_cast_any<float2><<<blocks, 256, 0, c.stream>>>(c.ker, c.dtype == GILA_C128, static_cast<float2*>(core->ker),
                                                      elems);
  GILA_CUDA_TRY(cudaGetLastError());
  GILA_CUDA_TRY(cudaStreamSynchronize(c.stream));
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
  if (a.dtype != GILA_C128) return fail(GILA_ERR_TYPE, "the residual operator must be ComplexF64");
  if (!a.self || a.geom.parT != 1 || a.parS != 1 || in_elems(a) != out_elems(a))
    return fail(GILA_ERR_SIZE, "Green's operator and medium must have the same size (a self operator).");
  Opts o;
  o.tol = opts && opts->tol > 0 ? opts->tol : 1e-6;
  o.ell = opts && opts->ell > 0 ? opts->ell : 2;
  o.mixed = opts ? (opts->mixed != 0) : 0;
  o.max_mv = opts && opts->max_matvecs > 0 ? opts->max_matvecs : 4000;
  o.max_restarts = opts && opts->max_restarts > 0 ? opts->max_restarts : 20;
  o.delta = opts && opts->delta > 0 ? opts->delta : 0.1;
  o.x0 = opts ? (opts->x0 != 0) : 0;
  o.graph = opts ? (opts->no_graph == 0) : 1;
  if (const char* ev = getenv("GILA_SOLVE_GRAPH"))
    if (ev[0] == '0') o.graph = 0;
  if (o.ell > kMaxEll) return fail(GILA_ERR_ARG, "BiCGStab(l) degree must be 1..4");
  Core* inner = &a;
  if (o.mixed) {
    if (!g32 || !g32->core) return fail(GILA_ERR_ARG, "the mixed solve needs the ComplexF32 operator");
    inner = g32->core.get();
    if (inner->dtype != GILA_C64) return fail(GILA_ERR_TYPE, "the inner operator must be ComplexF32");
    if (!same_volume(a, *inner) || inner->device != a.device)
      return fail(GILA_ERR_SIZE, "the two operators describe different volumes");
  }
  std::unique_lock<std::mutex> la(a.mu, std::defer_lock), lb(inner->mu, std::defer_lock);
  if (inner != &a)
    std::lock(la, lb);
  else
    la.lock();
  GILA_CUDA_TRY(cudaSetDevice(a.device));
  for (Core* c : {&a, inner}) {
    gila_status s = ensure_work(*c, nrhs);
    if (s != GILA_OK) return s;
    if (!c->tuned) {
      c->launch = default_launch(*c);
      c->tuned = true;
    }
  }
  cudaStream_t st = a.stream;
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  DevArena mem;
  cudaEvent_t ev = nullptr;
  if (user) {
    GILA_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    GILA_CUDA_TRY(cudaEventRecord(ev, user));
    GILA_CUDA_TRY(cudaStreamWaitEvent(st, ev, 0));
  }
  const int64_t n = in_elems(a), V = n / 3, nv = n * nrhs;
  // device copies of chi, b and x
  double2 *chi64 = nullptr, *bd = nullptr, *xd = nullptr;
  GILA_CUDA_TRY(mem.alloc((void**)&chi64, V * sizeof(double2)));
  GILA_CUDA_TRY(cudaMemcpyAsync(chi64, chi, V * sizeof(double2), cudaMemcpyDefault, st));
  if (is_device_ptr(b)) {
    bd = const_cast<double2*>(static_cast<const double2*>(b));
  } else {
    GILA_CUDA_TRY(mem.alloc((void**)&bd, nv * sizeof(double2)));
    GILA_CUDA_TRY(cudaMemcpyAsync(bd, b, nv * sizeof(double2), cudaMemcpyHostToDevice, st));
  }
  GILA_CUDA_TRY(mem.alloc((void**)&xd, nv * sizeof(double2)));
  if (o.x0) GILA_CUDA_TRY(cudaMemcpyAsync(xd, x, nv * sizeof(double2), cudaMemcpyDefault, st));
  std::vector<double> res;
  gila_solve_info inf{};
  cudaError_t e;
  if (o.mixed) {
    float2* chi32 = nullptr;
    GILA_CUDA_TRY(mem.alloc((void**)&chi32, V * sizeof(float2)));
    k_cast<float2><<<vec_blocks(V), kT, 0, st>>>(chi64, chi32, V);
    GILA_CUDA_TRY(cudaGetLastError());
    Solver<float2> sv(a, *inner, chi64, chi32, bd, xd, (int)nrhs, o, st);
    if ((e = sv.setup()) != cudaSuccess || (e = sv.run(res)) != cudaSuccess) {
      cudaStreamSynchronize(st);
      return cuda_fail(e, "gila_ls_solve");
    }
    inf = sv.info;
  } else {
    Solver<double2> sv(a, a, chi64, chi64, bd, xd, (int)nrhs, o, st);
    if ((e = sv.setup()) != cudaSuccess || (e = sv.run(res)) != cudaSuccess) {
      cudaStreamSynchronize(st);
      return cuda_fail(e, "gila_ls_solve");
    }
    inf = sv.info;
  }
  GILA_CUDA_TRY(cudaMemcpyAsync(x, xd, nv * sizeof(double2), cudaMemcpyDefault, st));
  GILA_CUDA_TRY(cudaStreamSynchronize(st));
  if (ev) {
    cudaEventRecord(ev, st);
    cudaStreamWaitEvent(user, ev, 0);
    cudaEventDestroy(ev);
  }
  if (info) *info = inf;
  if (rhs_res)
    for (int64_t r = 0; r < nrhs; ++r) rhs_res[r] = res[r];
  if (inf.converged < nrhs)
    return fail(GILA_ERR_NOTCONV, "the solve stopped at relative residual " + std::to_string(inf.rel_res) +
                                      " above the tolerance " + std::to_string(o.tol));
  return GILA_OK;
}

}  // extern "C"
