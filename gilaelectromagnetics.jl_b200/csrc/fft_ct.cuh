// fft_ct.cuh -- compile-time specialised Stockham stages.
//
// Same algorithm as fft_run in fft.cuh, but the transform length, the radix
// schedule, the span of every stage and the line count are template
// constants, so all index arithmetic folds to shifts / immediates and every
// stage is unrolled.  Used for the circulant lengths the workloads use; other
// lengths run the runtime-sized path.
#pragma once
#include "fft.cuh"

namespace gila {

// greedy radix schedule: 8s, then a 4 or a 2, then 3s, 5s, 7s
constexpr int ct_pow2(int P) {
  int t = 0;
  while (P % 2 == 0) {
    P /= 2;
    ++t;
  }
  return t;
}
constexpr int ct_odd(int P) {
  while (P % 2 == 0) P /= 2;
  return P;
}
constexpr int ct_nst(int P) {
  int t = ct_pow2(P);
  int n = t / 3 + ((t % 3) ? 1 : 0);
  int o = ct_odd(P);
  for (int q : {3, 5, 7})
    while (o % q == 0) {
      o /= q;
      ++n;
    }
  return n;
}
constexpr int ct_radix(int P, int s) {
  int t = ct_pow2(P);
  int n8 = t / 3;
  if (s < n8) return 8;
  s -= n8;
  if (t % 3) {
    if (s == 0) return (t % 3 == 2) ? 4 : 2;
    --s;
  }
  int o = ct_odd(P);
  for (int q : {3, 5, 7})
    while (o % q == 0) {
      if (s == 0) return q;
      o /= q;
      --s;
    }
  return 1;
}
constexpr int ct_span(int P, int s) {
  int ns = 1;
  for (int k = 0; k < s; ++k) ns *= ct_radix(P, k);
  return ns;
}
constexpr bool ct_supported(int P) { return ct_odd(P) == 1 || ct_odd(P) == 3 || ct_odd(P) == 5 || ct_odd(P) == 9; }
// the same radices in reverse order (REV): the inverse transform of the z
// pass starts with the radix the forward transform ends with, so that the
// forward's last stage, the 3x3 multiply and the inverse's first stage run on
// the same registers
template <bool REV>
constexpr int ct_radix_o(int P, int s) {
  return REV ? ct_radix(P, ct_nst(P) - 1 - s) : ct_radix(P, s);
}
template <bool REV>
constexpr int ct_span_o(int P, int s) {
  int ns = 1;
  for (int k = 0; k < s; ++k) ns *= ct_radix_o<REV>(P, k);
  return ns;
}

// One stage; T = threads per CTA, M = lines.
template <typename C, int P, int S, int E, int T, int M, bool INV, bool LINE_FAST, bool REV, class Ld, class St>
__device__ __forceinline__ void ct_stage(const C* __restrict__ tw, const Ld& ld, const St& st, bool sync_mid) {
  constexpr int R = ct_radix_o<REV>(P, S);
  constexpr int NS = ct_span_o<REV>(P, S);
  constexpr int TPL = P / R;
  constexpr int NTASK = M * TPL;
  constexpr int K = (NTASK + T - 1) / T;
  constexpr int TWST = P / (NS * R);
  C v[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NTASK % T == 0 || task < NTASK) {
      int l, j;
      if (LINE_FAST) {
        l = task % M;
        j = task / M;
      } else {
        l = task / TPL;
        j = task % TPL;
      }
#pragma unroll
      for (int r = 0; r < R; ++r) v[k][r] = ld(l, j + r * TPL);
    }
  }
  if (sync_mid) __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NTASK % T == 0 || task < NTASK) {
      int l, j;
      if (LINE_FAST) {
        l = task % M;
        j = task / M;
      } else {
        l = task / TPL;
        j = task % TPL;
      }
      const int jm = j % NS;
      if (NS > 1) {
        C w[R];
        twiddles<R, INV>(tw, jm * TWST, w);
#pragma unroll
        for (int r = 1; r < R; ++r) v[k][r] = cmul(v[k][r], w[r]);
      }
      Bfly<R, INV, C>::run(v[k], tw, TPL);
      const int base = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) st(l, base + r * NS, v[k][r]);
    }
  }
}

// stages [S0, S1) of the schedule (S runs from S0); ld_first feeds stage
// S0, st_last takes the output of stage S1 - 1
template <typename C, int P, int S0, int S, int S1, int E, int T, int M, bool INV, bool LINE_FAST, bool REV,
          class LdF, class LdM, class StM, class StL>
__device__ __forceinline__ void ct_run_range(const C* __restrict__ tw, const LdF& ld_first, const LdM& ld_mid,
                                             const StM& st_mid, const StL& st_last, bool first_in_smem,
                                             bool last_in_smem) {
  if constexpr (S < S1) {
    constexpr bool first = (S == S0), last = (S == S1 - 1);
    const bool sync_mid = (first ? first_in_smem : true) && (last ? last_in_smem : true);
    if constexpr (first && last)
      ct_stage<C, P, S, E, T, M, INV, LINE_FAST, REV>(tw, ld_first, st_last, sync_mid);
    else if constexpr (first)
      ct_stage<C, P, S, E, T, M, INV, LINE_FAST, REV>(tw, ld_first, st_mid, sync_mid);
    else if constexpr (last)
      ct_stage<C, P, S, E, T, M, INV, LINE_FAST, REV>(tw, ld_mid, st_last, sync_mid);
    else
      ct_stage<C, P, S, E, T, M, INV, LINE_FAST, REV>(tw, ld_mid, st_mid, sync_mid);
    __syncthreads();
    ct_run_range<C, P, S0, S + 1, S1, E, T, M, INV, LINE_FAST, REV>(tw, ld_first, ld_mid, st_mid, st_last,
                                                                     first_in_smem, last_in_smem);
  }
}

template <typename C, int P, int E, int T, int M, bool INV, bool LINE_FAST, class LdF, class LdM, class StM, class StL>
__device__ __forceinline__ void ct_run(const C* __restrict__ tw, const LdF& ld_first, const LdM& ld_mid,
                                       const StM& st_mid, const StL& st_last, bool first_in_smem, bool last_in_smem) {
  ct_run_range<C, P, 0, 0, ct_nst(P), E, T, M, INV, LINE_FAST, false>(tw, ld_first, ld_mid, st_mid, st_last,
                                                                      first_in_smem, last_in_smem);
}

// ---------------------------------------------------------- line pairs
// FP32 passes whose lines are contiguous in shared memory ([index][line]):
// a task handles two adjacent lines, so each shared-memory access moves both
// lines' values in one 16-byte transaction and the two lines share the
// twiddles and the index arithmetic.  M2 = line pairs; ld / st take a pair
// index and a position and move float4 = (line 2p, line 2p + 1).  LF: pairs
// fastest across threads (y, z layouts [index][pair]) or positions fastest
// (x layout [pair][index]).
template <int P, int S, int T, int M2, bool INV, bool REV, bool LF, class Ld, class St>
__device__ __forceinline__ void ct_stage2(const float2* __restrict__ tw, const Ld& ld, const St& st, bool sync_mid) {
  constexpr int R = ct_radix_o<REV>(P, S);
  constexpr int NS = ct_span_o<REV>(P, S);
  constexpr int TPL = P / R;
  constexpr int NTASK = M2 * TPL;
  constexpr int K = (NTASK + T - 1) / T;
  constexpr int TWST = P / (NS * R);
  float2 a[K][R], b[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NTASK % T == 0 || task < NTASK) {
      const int lp = LF ? task % M2 : task / TPL, j = LF ? task / M2 : task % TPL;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float4 q = ld(lp, j + r * TPL);
        a[k][r] = make_float2(q.x, q.y);
        b[k][r] = make_float2(q.z, q.w);
      }
    }
  }
  if (sync_mid) __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NTASK % T == 0 || task < NTASK) {
      const int lp = LF ? task % M2 : task / TPL, j = LF ? task / M2 : task % TPL;
      const int jm = j % NS;
      if (NS > 1) {
        float2 w[R];
        twiddles<R, INV>(tw, jm * TWST, w);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          a[k][r] = cmul(a[k][r], w[r]);
          b[k][r] = cmul(b[k][r], w[r]);
        }
      }
      Bfly<R, INV, float2>::run(a[k], tw, TPL);
      Bfly<R, INV, float2>::run(b[k], tw, TPL);
      const int base = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r)
        st(lp, base + r * NS, make_float4(a[k][r].x, a[k][r].y, b[k][r].x, b[k][r].y));
    }
  }
}

template <int P, int S0, int S, int S1, int T, int M2, bool INV, bool REV, bool LF, class LdF, class LdM, class StM,
          class StL>
__device__ __forceinline__ void ct_run_range2(const float2* __restrict__ tw, const LdF& ld_first, const LdM& ld_mid,
                                              const StM& st_mid, const StL& st_last, bool first_in_smem,
                                              bool last_in_smem) {
  if constexpr (S < S1) {
    constexpr bool first = (S == S0), last = (S == S1 - 1);
    const bool sync_mid = (first ? first_in_smem : true) && (last ? last_in_smem : true);
    if constexpr (first && last)
      ct_stage2<P, S, T, M2, INV, REV, LF>(tw, ld_first, st_last, sync_mid);
    else if constexpr (first)
      ct_stage2<P, S, T, M2, INV, REV, LF>(tw, ld_first, st_mid, sync_mid);
    else if constexpr (last)
      ct_stage2<P, S, T, M2, INV, REV, LF>(tw, ld_mid, st_last, sync_mid);
    else
      ct_stage2<P, S, T, M2, INV, REV, LF>(tw, ld_mid, st_mid, sync_mid);
    __syncthreads();
    ct_run_range2<P, S0, S + 1, S1, T, M2, INV, REV, LF>(tw, ld_first, ld_mid, st_mid, st_last, first_in_smem,
                                                         last_in_smem);
  }
}

// ---------------------------------------------------------- launch shapes
// Shared by the kernels (template constants) and the host (launch config).
constexpr int ct_round32(int a) { return (a + 31) / 32 * 32; }
// rows per CTA of an x pass: 1024 values (measured against 512 and 2048 at
// 128x128x64 F64: 0.4134 / 0.4155 / 0.4201 ms per matvec, bit-identical)
template <int CS>
constexpr int ct_xlines(int P) {
  return P >= 1024 ? 1 : 1024 / P;
}
// kx tile of a y pass: 128-byte rows, at most 512 threads with E = 8
template <int CS>
constexpr int ct_ytile(int P) {
  int tx = 128 / CS;
  while (tx > 1 && ct_round32((tx * P + 7) / 8) > 512) tx /= 2;
  return tx;
}
// kx tile of the z pass: three components in shared memory (<= 100 KB)
template <int CS>
constexpr int ct_ztile(int P) {
  int tx = 128 / CS;
  while (tx > 1 && (ct_round32((tx * P + 7) / 8) > 512 || 3 * tx * P * CS > 100 * 1024)) tx /= 2;
  return tx;
}
constexpr int ct_threads(int M, int P) {
  int t = ct_round32((M * P + 7) / 8);
  return t < 32 ? 32 : t;
}
// threads of a line-pair kernel over M lines (8 pairs of values per thread)
constexpr int ct_threads2(int M, int P) { return ct_threads(M / 2, P); }
// rows per CTA of an FP32 x pass on row pairs: even
template <int CS>
constexpr int ct_xlines2(int P) {
  return ct_xlines<CS>(P) >= 2 ? ct_xlines<CS>(P) / 2 * 2 : 2;
}
// tile widths the y and z kernels are instantiated for (the autotuner picks
// among them per operator): at most 512 threads and the shared-memory budget
constexpr int kTileSet[3] = {4, 8, 16};
constexpr bool ct_y_ok(int CS, int P, int TX) {
  return ct_threads(TX, P) <= 512 && (long long)TX * P * CS <= 200 * 1024;
}
constexpr bool ct_z_ok(int CS, int P, int TX) {
  return ct_threads(TX, P) <= 512 && 3LL * TX * P * CS <= 100 * 1024;
}

}  // namespace gila
