// fft.cuh -- device building blocks for the pruned Stockham FFT passes of the
// Green-operator matvec.
//
// The reference applies the block-Toeplitz operator as a depth-3 recursion of
// even/odd parity branches with 1-D FFTW/CUFFT transforms on each
// (src/glaAct.jl:63-321).  Each level's split (src/glaActSup.jl:72-421) is the
// first radix-2 decimation-in-frequency stage of a zero-padded length-P DFT
// (P = srcCel + trgCel) and each merge (src/glaActSup.jl:425-667) is the last
// radix-2 stage of the truncated inverse.  Here the whole length-P transform
// runs as a mixed-radix Stockham FFT whose first stage reads only the nonzero
// input (zero padding is never stored) and whose last inverse stage writes
// only the target range (truncation fused).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gila {

// ---------------------------------------------------------------- complex ops
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by -i (fwd) or +i (inv)
template <bool INV> __device__ __forceinline__ double2 cmuli(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
template <bool INV> __device__ __forceinline__ float2 cmuli(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <typename C> struct Real;
template <> struct Real<double2> { using T = double; };
template <> struct Real<float2> { using T = float; };

template <typename C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }

template <typename C> __device__ __forceinline__ C cmake(double re, double im);
template <> __device__ __forceinline__ double2 cmake<double2>(double re, double im) { return make_double2(re, im); }
template <> __device__ __forceinline__ float2 cmake<float2>(double re, double im) {
  return make_float2((float)re, (float)im);
}

// twiddle w_P^m = exp(-2 pi i m / P) from the table (conjugated for inverse)
template <bool INV, typename C>
__device__ __forceinline__ C twid(const C* __restrict__ tw, int m) {
  C w = __ldg(tw + m);
  return INV ? cconj(w) : w;
}

// Twiddles w^(r*step), r = 1 .. R-1, of one butterfly into w[1..R).  FP64:
// w^step (and w^(4 step) for R = 8) from the table, the other powers by
// complex products (a few FP64 multiplies instead of table loads, which
// share the load/store pipe with the shared-memory transposes; the products
// add at most 3 roundings).  FP32: table loads (its pipes are issue-bound).
template <int R, bool INV, typename C>
__device__ __forceinline__ void twiddles(const C* __restrict__ tw, int step, C* w) {
  if constexpr (sizeof(C) == 16 && (R == 4 || R == 8)) {
    w[1] = twid<INV>(tw, step);
    w[2] = cmul(w[1], w[1]);
    w[3] = cmul(w[2], w[1]);
    if constexpr (R == 8) {
      w[4] = twid<INV>(tw, 4 * step);
      w[5] = cmul(w[4], w[1]);
      w[6] = cmul(w[4], w[2]);
      w[7] = cmul(w[4], w[3]);
    }
  } else {
#pragma unroll
    for (int r = 1; r < R; ++r) w[r] = twid<INV>(tw, r * step);
  }
}

// ------------------------------------------------------------- butterflies
// In-place R-point DFT of v[0..R): out[k] = sum_r v[r] exp(-+2 pi i r k / R)
// (minus sign forward, plus sign inverse), natural output order.
template <int R, bool INV, typename C> struct Bfly;

template <bool INV, typename C> struct Bfly<2, INV, C> {
  __device__ __forceinline__ static void run(C* v, const C* __restrict__, int) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV, typename C> struct Bfly<4, INV, C> {
  __device__ __forceinline__ static void run(C* v, const C* __restrict__, int) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = cmuli<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV, typename C> struct Bfly<8, INV, C> {
  __device__ __forceinline__ static void run(C* v, const C* __restrict__, int) {
    using T = typename Real<C>::T;
    const T h = (T)0.70710678118654752440084436210484903928;
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    Bfly<4, INV, C>::run(e, nullptr, 0);
    Bfly<4, INV, C>::run(o, nullptr, 0);
    // o[k] *= w8^k, w8 = exp(-+ i pi / 4)
    C o1 = o[1], o3 = o[3];
    if (!INV) {
      o[1] = cmake<C>(h * (o1.x + o1.y), h * (o1.y - o1.x));
      o[3] = cmake<C>(h * (o3.y - o3.x), -h * (o3.x + o3.y));
    } else {
      o[1] = cmake<C>(h * (o1.x - o1.y), h * (o1.x + o1.y));
      o[3] = cmake<C>(-h * (o3.x + o3.y), h * (o3.x - o3.y));
    }
    o[2] = cmuli<INV>(o[2]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
};

template <bool INV, typename C> struct Bfly<3, INV, C> {
  __device__ __forceinline__ static void run(C* v, const C* __restrict__, int) {
    using T = typename Real<C>::T;
    const T s3 = (T)0.86602540378443864676372317075293618347;
    C t = cadd(v[1], v[2]);
    C u = csub(v[1], v[2]);
    C m = cmake<C>(v[0].x - (T)0.5 * t.x, v[0].y - (T)0.5 * t.y);
    C w = cmuli<INV>(cscale(u, s3));  // -+ i s3 u
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, w);
    v[2] = csub(m, w);
  }
};

template <bool INV, typename C> struct Bfly<5, INV, C> {
  __device__ __forceinline__ static void run(C* v, const C* __restrict__, int) {
    using T = typename Real<C>::T;
    const T c1 = (T)0.30901699437494742410229341718281905886;   // cos(2pi/5)
    const T c2 = (T)-0.80901699437494742410229341718281905886;  // cos(4pi/5)
    const T s1 = (T)0.95105651629515357211643933337938214340;   // sin(2pi/5)
    const T s2 = (T)0.58778525229247312916870595463907276860;   // sin(4pi/5)
    C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    C x0 = v[0];
    C p1 = cmake<C>(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    C p2 = cmake<C>(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    C q1 = cmuli<INV>(cmake<C>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    C q2 = cmuli<INV>(cmake<C>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    v[0] = cadd(x0, cadd(a1, a2));
    v[1] = cadd(p1, q1);
    v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2);
    v[3] = csub(p2, q2);
  }
};

// radix 7 (and the general odd case): direct DFT with the P-point twiddle
// table, whose (P/7)-strided entries are the 7th roots of unity.
template <bool INV, typename C> struct Bfly<7, INV, C> {
  __device__ __forceinline__ static void run(C* v, const C* __restrict__ tw, int pr) {
    C out[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      C acc = v[0];
#pragma unroll
      for (int r = 1; r < 7; ++r) acc = cadd(acc, cmul(v[r], twid<INV>(tw, ((r * k) % 7) * pr)));
      out[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = out[k];
  }
};

// ------------------------------------------------------------ async copy
// Global -> shared copies that bypass registers (cp.async), so that a CTA
// can put its whole input tile in flight at once.
__device__ __forceinline__ void cp_async(double2* s, const double2* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async(float2* s, const float2* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async(float4* s, const float4* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// -------------------------------------------------------- fast division
// n / d for 0 <= n < 2^31 by multiply-high and shift (Granlund-Montgomery);
// the magic numbers are computed once on the host.
struct FDiv {
  uint32_t d, m, s;
  __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const { return (__umulhi_hd(n, m) + n) >> s; }
  __host__ __device__ __forceinline__ static uint32_t __umulhi_hd(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
  }
};

inline FDiv make_fdiv(uint32_t d) {
  FDiv f;
  f.d = d;
  uint32_t s = 0;
  while ((1ull << s) < d) ++s;
  f.s = s;
  f.m = (uint32_t)((((1ull << s) - d) << 32) / d + 1);
  if (d == 1) f.m = 0;
  return f;
}

// ------------------------------------------------------------- one stage
// Per-stage constants of a Stockham plan, precomputed on the host.
struct StageC {
  int R;      // radix
  int ns;     // span Ns = product of the previous radices
  int tpl;    // tasks per line = P / R
  int twst;   // twiddle stride P / (Ns * R)
  FDiv nsd;   // division by Ns
  FDiv tpld;  // division by tpl
};

// A plan for one axis: the radix of each stage (product = P).
struct AxisPlan {
  int P;
  int nst;
  int radix[12];
  StageC st[12];
};

// Stockham autosort stage of radix R and span Ns over M lines of length P.
// Task (l, j), j in [0, P/R), reads positions j + r*P/R of line l, applies
// the twiddles w_P^{r*(j mod Ns)*P/(Ns*R)}, runs the R-point butterfly and
// writes positions (j - j mod Ns)*R + j mod Ns + r*Ns.
// ld(l, i) / st(l, i, v) abstract the source and destination; for an
// in-place shared-memory stage the caller passes sync_mid = true so that all
// loads complete before any store.  E = complex values staged per thread.
template <typename C, int R, int E, bool INV, bool LINE_FAST, class Ld, class St>
__device__ __forceinline__ void fft_stage(int M, const FDiv& md, const StageC& sc, const C* __restrict__ tw,
                                          const Ld& ld, const St& st, bool sync_mid) {
  constexpr int K = (E + R - 1) / R;  // K*R >= E covers every task
  const int tpl = sc.tpl;
  const int ntask = M * tpl;
  C v[K][R];
  int tl[K], tj[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * (int)blockDim.x;
    tl[k] = -1;
    tj[k] = 0;
    if (task < ntask) {
      int l, j;
      if (LINE_FAST) {
        j = (int)md.div((uint32_t)task);
        l = task - j * M;
      } else {
        l = (int)sc.tpld.div((uint32_t)task);
        j = task - l * tpl;
      }
      tl[k] = l;
      tj[k] = j;
#pragma unroll
      for (int r = 0; r < R; ++r) v[k][r] = ld(l, j + r * tpl);
    }
  }
  if (sync_mid) __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (tl[k] >= 0) {
      const int j = tj[k];
      const int Ns = sc.ns;
      const int jm = j - (int)sc.nsd.div((uint32_t)j) * Ns;
      if (Ns > 1) {
        const int step = jm * sc.twst;
#pragma unroll
        for (int r = 1; r < R; ++r) v[k][r] = cmul(v[k][r], twid<INV>(tw, r * step));
      }
      Bfly<R, INV, C>::run(v[k], tw, tpl);
      const int base = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) st(tl[k], base + r * Ns, v[k][r]);
    }
  }
}

// Run all stages of a plan.  The first stage reads through ld_first, the last
// writes through st_last; intermediate stages work in place on shared memory
// through ld_mid / st_mid.  A __syncthreads() separates stages.  md divides
// by the line count M (used when lines are the fastest-varying task index).
__device__ __forceinline__ StageC load_stage(const AxisPlan* __restrict__ pl, int s) {
  const StageC* q = pl->st + s;
  StageC c;
  c.R = __ldg(&q->R);
  c.ns = __ldg(&q->ns);
  c.tpl = __ldg(&q->tpl);
  c.twst = __ldg(&q->twst);
  c.nsd.d = __ldg(&q->nsd.d);
  c.nsd.m = __ldg(&q->nsd.m);
  c.nsd.s = __ldg(&q->nsd.s);
  c.tpld.d = __ldg(&q->tpld.d);
  c.tpld.m = __ldg(&q->tpld.m);
  c.tpld.s = __ldg(&q->tpld.s);
  return c;
}

// The plan lives in device memory (read through the read-only cache): a
// kernel-parameter copy indexed by the runtime stage number would be spilled
// to per-thread local memory.
template <typename C, int E, bool INV, bool LINE_FAST, bool MIXED, class LdF, class LdM, class StM, class StL>
__device__ __forceinline__ void fft_run(const AxisPlan* __restrict__ pl, int M, const FDiv& md,
                                        const C* __restrict__ tw, const LdF& ld_first, const LdM& ld_mid,
                                        const StM& st_mid, const StL& st_last, bool first_in_smem,
                                        bool last_in_smem) {
  const int nst = __ldg(&pl->nst);
  for (int s = 0; s < nst; ++s) {
    const StageC sc = load_stage(pl, s);
    const bool first = (s == 0), last = (s == nst - 1);
    // in-place hazard only when both source and destination are shared memory
    const bool sync_mid = (first ? first_in_smem : true) && (last ? last_in_smem : true);
    auto ld = [&](int l, int i) { return first ? ld_first(l, i) : ld_mid(l, i); };
    auto st = [&](int l, int i, C v) {
      if (last)
        st_last(l, i, v);
      else
        st_mid(l, i, v);
    };
    switch (sc.R) {
      case 8: fft_stage<C, 8, E, INV, LINE_FAST>(M, md, sc, tw, ld, st, sync_mid); break;
      case 4: fft_stage<C, 4, E, INV, LINE_FAST>(M, md, sc, tw, ld, st, sync_mid); break;
      case 2: fft_stage<C, 2, E, INV, LINE_FAST>(M, md, sc, tw, ld, st, sync_mid); break;
      default:
        if constexpr (MIXED) {
          if (sc.R == 3) fft_stage<C, 3, E, INV, LINE_FAST>(M, md, sc, tw, ld, st, sync_mid);
          else if (sc.R == 5) fft_stage<C, 5, E, INV, LINE_FAST>(M, md, sc, tw, ld, st, sync_mid);
          else if (sc.R == 7) fft_stage<C, 7, E, INV, LINE_FAST>(M, md, sc, tw, ld, st, sync_mid);
        }
        break;
    }
    __syncthreads();
  }
}

}  // namespace gila
