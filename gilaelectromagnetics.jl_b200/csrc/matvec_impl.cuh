// matvec_impl.cuh -- kernels and launchers of the five matvec passes,
// instantiated once per precision by matvec_c128.cu / matvec_c64.cu (the two
// translation units compile in parallel).
#pragma once
#include <cstdio>
#include <cstdlib>

#include "fft_ct.cuh"
#include "matvec.cuh"

namespace gila {


template <bool MX> struct StageE { static constexpr int v = MX ? kEm : kE; };

// Shared-memory row of an x pass: element i sits at i + i/8, which spreads
// the stride-R accesses of the early Stockham stages over all banks.
__host__ __device__ __forceinline__ int row_stride(int P) { return P + (P + 7) / 8; }


// -------------------------------------------------------------------- xfwd
template <typename C>
struct XfParams {
  const C* in;
  C* A;
  const AxisPlan* pl;  // device copy
  int P;
  const C* tw;
  int nin;       // source x cells
  int M;         // rows per CTA
  int64_t rows;  // total rows = 3 * sy * sz * nrhs
  FDiv nind;     // division by nin
};

template <typename C, bool MX>
__global__ void __launch_bounds__(512) k_xfwd(const XfParams<C> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan* const pl = p.pl;
  const int P = p.P, M = p.M, nin = p.nin;
  const int64_t rows = p.rows;
  C* const A = p.A;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const int LS = row_stride(P);
  // stage the M input rows (nin values each) into shared memory
  {
    const int nl = (int)((rows - g0) < M ? (rows - g0) : M);
    const C* const src = p.in + g0 * nin;
    for (int q = threadIdx.x; q < nl * nin; q += blockDim.x) {
      const int l = (int)p.nind.div((uint32_t)q);
      const int i = q - l * nin;
      cp_async(sm + l * LS + i + (i >> 3), src + q);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  auto ldf = [=](int l, int i) -> C {
    if (i < nin) return sm[l * LS + i + (i >> 3)];
    return czero<C>();
  };
  auto lds = [=](int l, int i) -> C { return sm[l * LS + i + (i >> 3)]; };
  auto sts = [=](int l, int i, C v) { sm[l * LS + i + (i >> 3)] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g < rows) A[g * P + i] = v;
  };
  const FDiv md{1, 0, 0};  // unused: rows are not the fastest task index
  fft_run<C, StageE<MX>::v, false, false, MX>(pl, M, md, p.tw, ldf, lds, sts, stg, true, false);
}

// ---------------------------------------------------------------------- y
template <typename C>
struct YParams {
  const C* src;
  C* dst;
  const AxisPlan* pl;  // device copy
  int P;
  const C* tw;
  int Px;
  int TX;
  int ntiles;     // ceil(Px / TX)
  int nin, nout;  // rows read / written
  int nz;         // z planes per channel in this pass
  int src_z, dst_z;          // z planes per channel in the src / dst layouts
  int src_rows, dst_rows;    // y rows per plane in the src / dst layouts
  int64_t q0;                // first plane (ch*nz + z) of this launch
  int64_t src_sub, dst_sub;  // plane index of the first plane held by src / dst
  FDiv md;                   // division by the line count TX
  // kx tiles of this launch: nt tiles, the first nlo from lo0 on, the rest
  // from hi0 on (all tiles: nt = nlo = ntiles, lo0 = 0)
  int nt, nlo, lo0, hi0;
};

template <typename C, bool INV, bool MX>
__global__ void __launch_bounds__(512) k_y(const YParams<C> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan* const pl = p.pl;
  const int Px = p.Px, TX = p.TX, nin = p.nin, nout = p.nout;
  const int tl = blockIdx.x % p.nt;  // tile of the kx set: low range, then high range
  const int tile = tl < p.nlo ? p.lo0 + tl : p.hi0 + (tl - p.nlo);
  const int64_t slice = p.q0 + blockIdx.x / p.nt;  // ch*nz + z
  const int64_t rc = slice / p.nz;
  const int z = (int)(slice % p.nz);
  const int kx0 = tile * TX;
  const int M = TX;
  const C* const src = p.src + ((rc * p.src_z + z) - p.src_sub) * p.src_rows * (int64_t)Px + kx0;
  C* const dst = p.dst + ((rc * p.dst_z + z) - p.dst_sub) * p.dst_rows * (int64_t)Px + kx0;
  const int tmax = Px - kx0;
  // stage the TX x nin input tile into shared memory [i][t]
  for (int q = threadIdx.x; q < nin * TX; q += blockDim.x) {
    const int i = (int)p.md.div((uint32_t)q);
    const int t = q - i * TX;
    if (t < tmax) cp_async(sm + q, src + (int64_t)i * Px + t);
  }
  cp_async_wait_all();
  __syncthreads();
  auto ldf = [=](int t, int i) -> C {
    if (t < tmax && i < nin) return sm[i * M + t];
    return czero<C>();
  };
  auto lds = [=](int t, int i) -> C { return sm[i * M + t]; };
  auto sts = [=](int t, int i, C v) { sm[i * M + t] = v; };
  auto stg = [=](int t, int i, C v) {
    if (t < tmax && i < nout) dst[(int64_t)i * Px + t] = v;
  };
  fft_run<C, StageE<MX>::v, INV, true, MX>(pl, M, p.md, p.tw, ldf, lds, sts, stg, true, false);
}

// ---------------------------------------------------------------------- z
// Kernel address of frequency f on one axis (mirror rules of mulBrnDev!,
// src/glaActSup.jl:789-846), computed arithmetically: branch bit p = f & 1,
// stored index m, mirrored flag (sign flip of the off-diagonal components).
struct AxMap {
  int brn;   // P / 2
  int full;  // stored extent == brn (no mirror)
  int fe;    // forward count of the even branch: ceil(t/2) + iseven(t)
  int fo;    // forward count of the odd branch: ceil(t/2)
};
__device__ __forceinline__ void ax_map(const AxMap& a, int f, int& p, int& m, int& mir) {
  p = f & 1;
  const int k = f >> 1;
  if (a.full) {
    m = k;
    mir = 0;
  } else if (p == 0) {
    mir = k >= a.fe;
    m = mir ? a.brn - k : k;
  } else {
    mir = k >= a.fo;
    m = mir ? a.brn - 1 - k : k;
  }
}

template <typename C>
struct ZParams {
  C* B;
  const C* ker;
  const int* mapx;
  const int* mapy;
  const int* mapz;
  const AxisPlan* pl;  // device copy
  int P;
  const C* tw;
  int Px, Py;
  int TX, ntiles;
  int nin, nout;  // source / target z cells
  int zb;         // z planes per channel in B
  int tx, ty, tz; // stored kernel extents
  int parT;
  int nrhs;
  int zmir;  // fused z pass: one kernel load per mirror pair of z frequencies
  double scale;
  FDiv md;    // division by the tile width TX
  FDiv nind;  // division by nin
  AxMap ax[3];
  int ts0, nts;  // positions [ts0, ts0 + nts) of the mirror tile order (all: 0, ntiles)
  // spectrum rows of this launch: B holds Py rows, which are rows ky0 ..
  // ky0 + Py - 1 of the operator's spectrum (the kernel values and mirror
  // flags follow the operator's row); ky0 = 0 and Py = the full row count
  // except for the slab pieces of a slab-decomposed matvec
  int ky0;
};

// ky order that places each frequency next to its mirror Py - ky, and kx
// tile order that places tile i next to tile ntiles-1-i, so that the four
// CTAs reading the same stored (half-spectrum) kernel values run together and
// the re-reads are served from L2.
__device__ __forceinline__ int mirror_seq(int idx, int n) {
  if (idx == 0) return 0;
  if (n % 2 == 0) {
    if (idx == 1) return n / 2;
    const int k = (idx - 2) / 2 + 1;
    return (idx % 2 == 0) ? k : n - k;
  }
  const int k = (idx - 1) / 2 + 1;
  return (idx % 2 == 1) ? k : n - k;
}
__device__ __forceinline__ int tile_seq(int idx, int n) {
  const int k = idx / 2;
  return (idx % 2 == 0) ? k : n - 1 - k;
}

// FP64 kernel values are read once per column and their L2 lines are shared
// by the CTAs of the mirror columns, not by the threads of one CTA: the loads
// bypass L1 allocation (measured 3% faster z passes at 256x256x128 than
// cached loads, whose fills share the L1 data path with the transposes).
__device__ __forceinline__ double2 ld_nc_na(const double2* g) {
  double2 r;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(g));
  return r;
}
// FP32: cached (measured faster than loads past L1 here), since a line-pair
// thread reads the two x parities of one stored index, which sit side by
// side: one 16-byte load where both are unmirrored, two loads of one line
// otherwise
__device__ __forceinline__ float2 ld_nc_na(const float2* g) { return __ldg(g); }
template <typename C>
__device__ __forceinline__ C ker_ld(const C* __restrict__ g, int c, int tx) {
  return ld_nc_na(g + 2 * c * tx);
}
// Stored kernel layout: target-partition blocks laid out by ker_index
// ([py,pz][tz][ty][6][tx][px]); the threads of a warp (consecutive kx of a
// tile, alternating x parity) read consecutive entries of one component.
// Returns the address of component 0 of entry (eo, iz, iy, ix); component c
// is 2 * c * tx entries further (ker_ld).
template <typename C>
__device__ __forceinline__ const C* ker_at(const C* __restrict__ kpar, int eo, int iz, int iy, int ix, int tx, int ty,
                                           int tz) {
  // one partition holds 8 * tz * ty * 6 * tx < 2^31 entries (host-checked)
  return kpar + (((((eo & 3) * tz + iz) * ty + iy) * 6) * tx + ix) * 2 + (eo >> 2);
}


template <typename C, bool MX>
__global__ void __launch_bounds__(512) k_z(const ZParams<C> p) {
  using T = typename Real<C>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan* const pl = p.pl;
  const int P = p.P;
  const int nrhs = p.nrhs, ntiles = p.ntiles, TX = p.TX, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = p.ts0 + rest % p.nts;  // [ts0, ts0 + nts) of the mirror tile order
  const int yseq = rest / p.nts;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int tmax = Px - kx0;
  const int64_t plane = (int64_t)Py * Px;
  const int CH = P * TX;  // one component's spectra in shared memory: [kz][t]
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  // stage all three components' source z lines into shared memory [c][z][t]
  for (int q = threadIdx.x; q < 3 * nin * TX; q += blockDim.x) {
    const int row = (int)p.md.div((uint32_t)q);  // c * nin + z
    const int t = q - row * TX;
    const int c = (int)p.nind.div((uint32_t)row);
    const int i = row - c * nin;
    if (t < tmax) cp_async(sm + c * CH + i * TX + t, Bb + (int64_t)row * plane + t);
  }
  cp_async_wait_all();
  __syncthreads();
  // forward, one component at a time, in place in shared memory
  for (int c = 0; c < 3; ++c) {
    C* const smc = sm + c * CH;
    auto ldf = [=](int t, int i) -> C {
      if (t < tmax && i < nin) return smc[i * TX + t];
      return czero<C>();
    };
    auto lds = [=](int t, int i) -> C { return smc[i * TX + t]; };
    auto sts = [=](int t, int i, C v) { smc[i * TX + t] = v; };
    fft_run<C, StageE<MX>::v, false, true, MX>(pl, TX, p.md, p.tw, ldf, lds, sts, sts, true, true);
  }

  const int my = __ldg(p.mapy + ky + p.ky0);
  const int py = (my >> 29) & 1, ry = (my >> 30) & 1;
  const int iy = my & 0x1fffffff;
  const int tx = p.tx, ty = p.ty, tz = p.tz, parT = p.parT;
  const int* const mapx = p.mapx;
  const int* const mapz = p.mapz;
  const T s = (T)p.scale;
  C* const out3 = sm + 3 * CH;  // extra 3-component buffer (parT > 1 only)
  for (int t_par = 0; t_par < parT; ++t_par) {
    C* const dst = (parT == 1) ? sm : out3;
    const C* const kpar = p.ker + (int64_t)t_par * 8 * tz * ty * tx * 6;
    for (int task = threadIdx.x; task < CH; task += blockDim.x) {
      const int kz = (int)p.md.div((uint32_t)task);
      const int t = task - kz * TX;
      const int kx = kx0 + t;
      if (kx >= Px) continue;
      const int mx = __ldg(mapx + kx), mz = __ldg(mapz + kz);
      const int px = (mx >> 29) & 1, rx = (mx >> 30) & 1, ix = mx & 0x1fffffff;
      const int pz = (mz >> 29) & 1, rz = (mz >> 30) & 1, iz = mz & 0x1fffffff;
      const int eo = 4 * px + 2 * py + pz;
      const C* g = ker_at(kpar, eo, iz, iy, ix, tx, ty, tz);
      const T sxy = (rx ^ ry) ? (T)-1 : (T)1;
      const T sxz = (rx ^ rz) ? (T)-1 : (T)1;
      const T syz = (ry ^ rz) ? (T)-1 : (T)1;
      const C gxx = ker_ld(g, 0, tx), gyy = ker_ld(g, 1, tx), gzz = ker_ld(g, 2, tx);
      const C gxy = cscale(ker_ld(g, 3, tx), sxy), gxz = cscale(ker_ld(g, 4, tx), sxz),
              gyz = cscale(ker_ld(g, 5, tx), syz);
      const C x0 = sm[task], x1 = sm[CH + task], x2 = sm[2 * CH + task];
      C y0 = cadd(cadd(cmul(gxx, x0), cmul(gxy, x1)), cmul(gxz, x2));
      C y1 = cadd(cadd(cmul(gxy, x0), cmul(gyy, x1)), cmul(gyz, x2));
      C y2 = cadd(cadd(cmul(gxz, x0), cmul(gyz, x1)), cmul(gzz, x2));
      dst[task] = cscale(y0, s);
      dst[CH + task] = cscale(y1, s);
      dst[2 * CH + task] = cscale(y2, s);
    }
    __syncthreads();
    // inverse, one component at a time: shared -> global (target z), truncated
    for (int c = 0; c < 3; ++c) {
      C* const dc = dst + c * CH;
      C* const Bo = Bb + (int64_t)(t_par * 3 + c) * nout * plane;
      auto ldo = [=](int t, int i) -> C { return dc[i * TX + t]; };
      auto sto = [=](int t, int i, C v) { dc[i * TX + t] = v; };
      auto stg = [=](int t, int i, C v) {
        if (t < tmax && i < nout) Bo[(int64_t)i * plane + t] = v;
      };
      fft_run<C, StageE<MX>::v, true, true, MX>(pl, TX, p.md, p.tw, ldo, ldo, sto, stg, true, false);
    }
  }
}

// -------------------------------------------------------------------- xinv
template <typename C>
struct XiParams {
  const C* A;
  C* out;
  const AxisPlan* pl;  // device copy
  int P;
  const C* tw;
  int nout;  // target x cells
  int M;
  int64_t rows;   // rows in this launch
  int64_t g_off;  // global row index (over all rhs) of the first row
  int ty, tz, parT;
  int part_scatter;  // parT > 1
  int tdiv[3];
  int toff[64][3];
  int64_t full[3];
  C alpha, beta;
  FDiv pd;  // division by P
  // Lippmann-Schwinger epilogue (ls != 0): out = ls_in - chi .* value
  const C* ls_in;
  const C* ls_chi;
  int64_t ls_chi_rs;
  int ls;
  FDiv rows_rhs;  // division by 3 * tz * ty (rows per right-hand side)
  FDiv rows_zy;   // division by tz * ty
};

// the epilogue value at output index o of row gg, column i
template <typename C>
__device__ __forceinline__ C ls_value(const C* __restrict__ in, const C* __restrict__ chi, int64_t chi_rs, FDiv rr,
                                      FDiv rzy, int nout, int64_t gg, int i, int64_t o, C v) {
  const uint32_t rhs = rr.div((uint32_t)gg);
  const uint32_t rem = (uint32_t)gg - rhs * rr.d;
  const uint32_t zy = rem - rzy.div(rem) * rzy.d;
  const C c = chi[(int64_t)rhs * chi_rs + (int64_t)zy * nout + i];
  return csub(in[o], cmul(c, v));
}

template <typename C, bool AXPBY, bool MX>
__global__ void __launch_bounds__(512) k_xinv(const XiParams<C> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan* const pl = p.pl;
  const int P = p.P, M = p.M, nout = p.nout;
  const int64_t rows = p.rows;
  const C* const A = p.A;
  C* const out = p.out;
  const C alpha = p.alpha, beta = p.beta;
  const int ls = p.ls;
  const C* const ls_in = p.ls_in;
  const C* const ls_chi = p.ls_chi;
  const int64_t ls_chi_rs = p.ls_chi_rs;
  const FDiv rows_rhs = p.rows_rhs, rows_zy = p.rows_zy;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const bool scatter = p.part_scatter != 0;
  const int ty = p.ty, tz = p.tz, parT = p.parT;
  const int d0 = p.tdiv[0], d1 = p.tdiv[1], d2 = p.tdiv[2];
  const int64_t f0 = p.full[0], f1 = p.full[1], f2 = p.full[2];
  const int(*toff)[3] = p.toff;
  const int64_t g_off = p.g_off;
  const int LS = row_stride(P);
  // stage the M spectral rows (P values each) into shared memory
  {
    const int nl = (int)((rows - g0) < M ? (rows - g0) : M);
    const C* const src = A + g0 * P;
    for (int q = threadIdx.x; q < nl * P; q += blockDim.x) {
      const int l = (int)p.pd.div((uint32_t)q);
      const int i = q - l * P;
      cp_async(sm + l * LS + i + (i >> 3), src + q);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  auto ldg = [=](int l, int i) -> C { return sm[l * LS + i + (i >> 3)]; };
  auto lds = [=](int l, int i) -> C { return sm[l * LS + i + (i >> 3)]; };
  auto sts = [=](int l, int i, C v) { sm[l * LS + i + (i >> 3)] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g >= rows || i >= nout) return;
    int64_t o;
    const int64_t gg = g + g_off;
    if (!scatter) {
      o = gg * nout + i;
    } else {
      // gg = ((rhs*parT + t)*3 + c)*tz + z)*ty + y
      int64_t q = gg;
      const int y = (int)(q % ty); q /= ty;
      const int z = (int)(q % tz); q /= tz;
      const int c = (int)(q % 3); q /= 3;
      const int t = (int)(q % parT);
      const int64_t rhs = q / parT;
      const int64_t X = (int64_t)i * d0 + toff[t][0];
      const int64_t Y = (int64_t)y * d1 + toff[t][1];
      const int64_t Z = (int64_t)z * d2 + toff[t][2];
      o = (((rhs * 3 + c) * f2 + Z) * f1 + Y) * f0 + X;
    }
    if (AXPBY)
      out[o] = cadd(cmul(alpha, v), cmul(beta, out[o]));
    else if (ls)
      out[o] = ls_value(ls_in, ls_chi, ls_chi_rs, rows_rhs, rows_zy, nout, gg, i, o, v);
    else
      out[o] = v;
  };
  const FDiv md{1, 0, 0};
  fft_run<C, StageE<MX>::v, true, false, MX>(pl, M, md, p.tw, ldg, lds, sts, stg, true, false);
}

// ------------------------------------------------ compile-time specialised
// The same five passes with the transform length P, tile width and thread
// count as template constants (see fft_ct.cuh).

// CTAs per SM a pass kernel is compiled for: at power-of-two lengths,
// registers capped at 48 per thread (y passes: 0.4131 -> 0.4107 ms per
// matvec at 128x128x64 F64, 3.470 -> 3.439 ms at 256x256x128,
// bit-identical); lengths with a radix-3 stage would spill 300+ bytes at
// that cap and keep no hint
constexpr int pow2_min_blocks(int T, int P) {
  const int b = ct_odd(P) == 1 ? 65536 / (T * 48) : 1;
  return b < 1 ? 1 : (b > 32 ? 32 : b);  // at most 32 resident CTAs per SM
}

template <typename C, int P, bool REV>
__global__ void __launch_bounds__(ct_threads(ct_xlines<sizeof(C)>(P), P)) k_xfwd_ct(const XfParams<C> p) {
  constexpr int M = ct_xlines<sizeof(C)>(P);
  constexpr int T = ct_threads(M, P);
  constexpr int LS = P + (P + 7) / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nin = p.nin;
  const int64_t rows = p.rows;
  C* const A = p.A;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  {
    const int nl = (int)((rows - g0) < M ? (rows - g0) : M);
    const C* const src = p.in + g0 * nin;
    for (int q = threadIdx.x; q < nl * nin; q += T) {
      const int l = (int)p.nind.div((uint32_t)q);
      const int i = q - l * nin;
      cp_async(sm + l * LS + i + (i >> 3), src + q);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  auto ldf = [=](int l, int i) -> C {
    if (i < nin) return sm[l * LS + i + (i >> 3)];
    return czero<C>();
  };
  auto lds = [=](int l, int i) -> C { return sm[l * LS + i + (i >> 3)]; };
  auto sts = [=](int l, int i, C v) { sm[l * LS + i + (i >> 3)] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g < rows) A[g * P + i] = v;
  };
  ct_run_range<C, P, 0, 0, ct_nst(P), 8, T, M, false, false, REV>(p.tw, ldf, lds, sts, stg, true, false);
}

// FP32 x passes on row pairs: rows 2p and 2p+1 interleaved in shared memory
// (float4 slot = element i of both rows, slot i + i/8 of the pair's row), so
// every stage access is a conflict-free 16-byte transaction -- the access
// pattern of the FP64 passes -- and the two rows share twiddles.
template <int P, bool REV>
__global__ void __launch_bounds__(ct_threads2(ct_xlines2<8>(P), P)) k_xfwd2_ct(const XfParams<float2> p) {
  constexpr int M = ct_xlines2<8>(P);  // rows per CTA (even)
  constexpr int M2 = M / 2;
  constexpr int T = ct_threads2(M, P);
  constexpr int LS = P + (P + 7) / 8;  // float4 slots per pair row
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* const sm = reinterpret_cast<float4*>(smem_raw);
  const int nin = p.nin;
  const int64_t rows = p.rows;
  float2* const A = p.A;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const int nl = (int)((rows - g0) < M ? (rows - g0) : M);
  {
    // consecutive threads fill the two halves of consecutive slots
    const float2* const src = p.in + g0 * nin;
    for (int q = threadIdx.x; q < M2 * 2 * nin; q += T) {
      const int pr = q / (2 * nin), rem = q - pr * 2 * nin;
      const int i = rem >> 1, h = rem & 1;
      const int l = 2 * pr + h;
      if (l < nl) cp_async(reinterpret_cast<float2*>(sm + pr * LS + i + (i >> 3)) + h, src + (int64_t)l * nin + i);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  auto ldf = [=](int lp, int i) -> float4 {
    if (i < nin) return sm[lp * LS + i + (i >> 3)];
    return z4;
  };
  auto lds = [=](int lp, int i) -> float4 { return sm[lp * LS + i + (i >> 3)]; };
  auto sts = [=](int lp, int i, float4 v) { sm[lp * LS + i + (i >> 3)] = v; };
  auto stg = [=](int lp, int i, float4 v) {
    const int64_t g = g0 + 2 * lp;
    if (g < rows) A[g * P + i] = make_float2(v.x, v.y);
    if (g + 1 < rows) A[(g + 1) * P + i] = make_float2(v.z, v.w);
  };
  ct_run_range2<P, 0, 0, ct_nst(P), T, M2, false, REV, false>(p.tw, ldf, lds, sts, stg, true, false);
}

template <int P, bool REV>
__global__ void __launch_bounds__(ct_threads2(ct_xlines2<8>(P), P)) k_xinv2_ct(const XiParams<float2> p) {
  constexpr int M = ct_xlines2<8>(P);
  constexpr int M2 = M / 2;
  constexpr int T = ct_threads2(M, P);
  constexpr int LS = P + (P + 7) / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* const sm = reinterpret_cast<float4*>(smem_raw);
  const int nout = p.nout;
  const int64_t rows = p.rows;
  float2* const out = p.out;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const int64_t g_off = p.g_off;
  const int ls = p.ls;
  const float2* const ls_in = p.ls_in;
  const float2* const ls_chi = p.ls_chi;
  const int64_t ls_chi_rs = p.ls_chi_rs;
  const FDiv rows_rhs = p.rows_rhs, rows_zy = p.rows_zy;
  const int nl = (int)((rows - g0) < M ? (rows - g0) : M);
  {
    const float2* const src = p.A + g0 * P;
    for (int q = threadIdx.x; q < M2 * 2 * P; q += T) {
      const int pr = q / (2 * P), rem = q - pr * 2 * P;
      const int i = rem >> 1, h = rem & 1;
      const int l = 2 * pr + h;
      if (l < nl) cp_async(reinterpret_cast<float2*>(sm + pr * LS + i + (i >> 3)) + h, src + (int64_t)l * P + i);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  auto lds = [=](int lp, int i) -> float4 { return sm[lp * LS + i + (i >> 3)]; };
  auto sts = [=](int lp, int i, float4 v) { sm[lp * LS + i + (i >> 3)] = v; };
  auto stg = [=](int lp, int i, float4 v) {
    if (i >= nout) return;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t g = g0 + 2 * lp + h;
      if (g >= rows) return;
      const int64_t gg = g + g_off;
      const int64_t o = gg * nout + i;
      const float2 w = h ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
      out[o] = ls ? ls_value(ls_in, ls_chi, ls_chi_rs, rows_rhs, rows_zy, nout, gg, i, o, w) : w;
    }
  };
  ct_run_range2<P, 0, 0, ct_nst(P), T, M2, true, REV, false>(p.tw, lds, lds, sts, stg, true, false);
}

template <typename C, int P, bool INV, int TX, bool REV>
__global__ void __launch_bounds__(ct_threads(TX, P), pow2_min_blocks(ct_threads(TX, P), P)) k_y_ct(const YParams<C> p) {
  constexpr int T = ct_threads(TX, P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int Px = p.Px, nin = p.nin, nout = p.nout;
  const int tl = blockIdx.x % p.nt;  // tile of the kx set: low range, then high range
  const int tile = tl < p.nlo ? p.lo0 + tl : p.hi0 + (tl - p.nlo);
  const int64_t slice = p.q0 + blockIdx.x / p.nt;  // ch*nz + z
  const int64_t rc = slice / p.nz;
  const int z = (int)(slice % p.nz);
  const int kx0 = tile * TX;
  const C* const src = p.src + ((rc * p.src_z + z) - p.src_sub) * p.src_rows * (int64_t)Px + kx0;
  C* const dst = p.dst + ((rc * p.dst_z + z) - p.dst_sub) * p.dst_rows * (int64_t)Px + kx0;
  const int tmax = Px - kx0;
  for (int q = threadIdx.x; q < nin * TX; q += T) {
    const int i = q / TX, t = q % TX;
    if (t < tmax) cp_async(sm + q, src + (int64_t)i * Px + t);
  }
  cp_async_wait_all();
  __syncthreads();
  auto ldf = [=](int t, int i) -> C {
    if (t < tmax && i < nin) return sm[i * TX + t];
    return czero<C>();
  };
  auto lds = [=](int t, int i) -> C { return sm[i * TX + t]; };
  auto sts = [=](int t, int i, C v) { sm[i * TX + t] = v; };
  auto stg = [=](int t, int i, C v) {
    if (t < tmax && i < nout) dst[(int64_t)i * Px + t] = v;
  };
  ct_run_range<C, P, 0, 0, ct_nst(P), 8, T, TX, INV, true, REV>(p.tw, ldf, lds, sts, stg, true, false);
}

// FP32 y pass on line pairs (ct_stage2): two adjacent kx columns per task.
template <int P, bool INV, int TX, bool REV>
// (FP32 y passes with the same cap: 0.2517 -> 0.2426 ms per matvec at
// 128x128x64, 1.958 -> 1.946 ms at 256x256x128, bit-identical)
__global__ void __launch_bounds__(ct_threads2(TX, P), pow2_min_blocks(ct_threads2(TX, P), P)) k_y2_ct(const YParams<float2> p) {
  constexpr int T = ct_threads2(TX, P);
  constexpr int M2 = TX / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* const sm = reinterpret_cast<float4*>(smem_raw);
  const int Px = p.Px, nin = p.nin, nout = p.nout;
  const int tl = blockIdx.x % p.nt;  // tile of the kx set: low range, then high range
  const int tile = tl < p.nlo ? p.lo0 + tl : p.hi0 + (tl - p.nlo);
  const int64_t slice = p.q0 + blockIdx.x / p.nt;  // ch*nz + z
  const int64_t rc = slice / p.nz;
  const int z = (int)(slice % p.nz);
  const int kx0 = tile * TX;
  const float2* const src = p.src + ((rc * p.src_z + z) - p.src_sub) * p.src_rows * (int64_t)Px + kx0;
  float2* const dst = p.dst + ((rc * p.dst_z + z) - p.dst_sub) * p.dst_rows * (int64_t)Px + kx0;
  const int tmax = Px - kx0;  // even: Px and kx0 are even
  for (int q = threadIdx.x; q < nin * M2; q += T) {
    const int i = q / M2, t2 = q % M2;
    if (2 * t2 < tmax) cp_async(sm + q, reinterpret_cast<const float4*>(src + (int64_t)i * Px) + t2);
  }
  cp_async_wait_all();
  __syncthreads();
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
  auto ldf = [=](int t2, int i) -> float4 {
    if (2 * t2 < tmax && i < nin) return sm[i * M2 + t2];
    return z4;
  };
  auto lds = [=](int t2, int i) -> float4 { return sm[i * M2 + t2]; };
  auto sts = [=](int t2, int i, float4 v) { sm[i * M2 + t2] = v; };
  auto stg = [=](int t2, int i, float4 v) {
    if (2 * t2 < tmax && i < nout) reinterpret_cast<float4*>(dst + (int64_t)i * Px)[t2] = v;
  };
  ct_run_range2<P, 0, 0, ct_nst(P), T, M2, INV, REV, true>(p.tw, ldf, lds, sts, stg, true, false);
}

template <typename C, int P, int TX>
__global__ void __launch_bounds__(ct_threads(TX, P)) k_z_ct(const ZParams<C> p) {
  using Tr = typename Real<C>::T;
  constexpr int T = ct_threads(TX, P);
  constexpr int CH = P * TX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nrhs = p.nrhs, ntiles = p.ntiles, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = p.ts0 + rest % p.nts;  // [ts0, ts0 + nts) of the mirror tile order
  const int yseq = rest / p.nts;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int tmax = Px - kx0;
  const int64_t plane = (int64_t)Py * Px;
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  for (int q = threadIdx.x; q < 3 * nin * TX; q += T) {
    const int row = q / TX, t = q % TX;  // row = c * nin + z
    const int c = (int)p.nind.div((uint32_t)row);
    const int i = row - c * nin;
    if (t < tmax) cp_async(sm + c * CH + i * TX + t, Bb + (int64_t)row * plane + t);
  }
  cp_async_wait_all();
  __syncthreads();
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    C* const smc = sm + c * CH;
    auto ldf = [=](int t, int i) -> C {
      if (t < tmax && i < nin) return smc[i * TX + t];
      return czero<C>();
    };
    auto lds = [=](int t, int i) -> C { return smc[i * TX + t]; };
    auto sts = [=](int t, int i, C v) { smc[i * TX + t] = v; };
    ct_run<C, P, 8, T, TX, false, true>(p.tw, ldf, lds, sts, sts, true, true);
  }
  int py, iy, ry;
  ax_map(p.ax[1], ky + p.ky0, py, iy, ry);
  const int tx = p.tx, ty = p.ty, tz = p.tz, parT = p.parT;
  const Tr s = (Tr)p.scale;
  C* const out3 = sm + 3 * CH;
  // When the z axis is stored by symmetry, frequencies kz and P - kz read the
  // same stored kernel value (mirrored: off-diagonal signs flip), so one task
  // handles both.  Tasks: t = task % TX, kz = task / TX for kz <= P/2.
  const bool zpair = !p.ax[2].full;
  const int nzt = zpair ? (P / 2 + 1) : P;
  // kernel values in flight per thread: the loads of G tasks are issued
  // together before any of them is used, so their latency is paid once
#ifndef GILA_ZMUL_G
#define GILA_ZMUL_G 1
#endif
  constexpr int G = GILA_ZMUL_G;
  const int ntask = nzt * TX;
  for (int t_par = 0; t_par < parT; ++t_par) {
    C* const dst = (parT == 1) ? sm : out3;
    const C* const kpar = p.ker + (int64_t)t_par * 8 * tz * ty * tx * 6;
    for (int k0 = threadIdx.x; k0 < ntask; k0 += G * T) {
      C gv[G][6];
      int rxv[G], rzv[G];
      bool ok[G];
#pragma unroll
      for (int j = 0; j < G; ++j) {
        const int task = k0 + j * T;
        const int kz = task / TX, t = task % TX;
        ok[j] = task < ntask && kx0 + t < Px;
        if (ok[j]) {
          int px, ix, pz, iz;
          ax_map(p.ax[0], kx0 + t, px, ix, rxv[j]);
          ax_map(p.ax[2], kz, pz, iz, rzv[j]);
          const int eo = 4 * px + 2 * py + pz;
          const C* gp = ker_at(kpar, eo, iz, iy, ix, tx, ty, tz);
#pragma unroll
          for (int q = 0; q < 6; ++q) gv[j][q] = ker_ld(gp, q, tx);
        }
      }
#pragma unroll
      for (int j = 0; j < G; ++j) {
        if (!ok[j]) continue;
        const int task = k0 + j * T;
        const int kz = task / TX, t = task % TX;
        const int rx = rxv[j], rz = rzv[j];
        const C gxx = gv[j][0], gyy = gv[j][1], gzz = gv[j][2];
        const C gxy = cscale(gv[j][3], (rx ^ ry) ? (Tr)-1 : (Tr)1);
        const C g4 = gv[j][4], g5 = gv[j][5];
        // the task's own frequency, then (paired) its mirror with rz flipped
        const int nk = (zpair && kz != 0 && 2 * kz != P) ? 2 : 1;
#pragma unroll 1
        for (int h = 0; h < nk; ++h) {
          const int kk = h ? P - kz : kz;
          const int rzz = h ? (rz ^ 1) : rz;
          const C gxz = cscale(g4, (rx ^ rzz) ? (Tr)-1 : (Tr)1);
          const C gyz = cscale(g5, (ry ^ rzz) ? (Tr)-1 : (Tr)1);
          const int e = kk * TX + t;
          const C x0 = sm[e], x1 = sm[CH + e], x2 = sm[2 * CH + e];
          C y0 = cadd(cadd(cmul(gxx, x0), cmul(gxy, x1)), cmul(gxz, x2));
          C y1 = cadd(cadd(cmul(gxy, x0), cmul(gyy, x1)), cmul(gyz, x2));
          C y2 = cadd(cadd(cmul(gxz, x0), cmul(gyz, x1)), cmul(gzz, x2));
          dst[e] = cscale(y0, s);
          dst[CH + e] = cscale(y1, s);
          dst[2 * CH + e] = cscale(y2, s);
        }
      }
    }
    __syncthreads();
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      C* const dc = dst + c * CH;
      C* const Bo = Bb + (int64_t)(t_par * 3 + c) * nout * plane;
      auto ldo = [=](int t, int i) -> C { return dc[i * TX + t]; };
      auto sto = [=](int t, int i, C v) { dc[i * TX + t] = v; };
      auto stg = [=](int t, int i, C v) {
        if (t < tmax && i < nout) Bo[(int64_t)i * plane + t] = v;
      };
      ct_run<C, P, 8, T, TX, true, true>(p.tw, ldo, ldo, sto, stg, true, false);
    }
  }
}

// z pass with the forward transform's last stage, the 3x3 multiply and the
// inverse transform's first stage fused in registers (single target
// partition).  The inverse runs the forward's radices in reverse order, so
// the values a thread holds after the forward's last stage -- frequencies
// j + r*P/R of its line -- are exactly the inputs of its first inverse
// butterfly: three shared-memory passes per element fewer than
// transform -> store -> multiply -> load -> transform.
#ifndef GILA_ZF_KPRE
#define GILA_ZF_KPRE 0
#endif
// CTAs per SM the fused z kernel is compiled for: registers capped at 128
constexpr int zf_min_blocks(int T) { return 65536 / (T * 128) > 1 ? 65536 / (T * 128) : 1; }
// the fused stage holds 3 * 8 values per thread; with a last radix of 8 that
// does not fit 128 FP64 registers, so those lengths keep the unfused kernel
constexpr bool zf_ok(int CS, int P) { return CS == 8 || ct_radix(P, ct_nst(P) - 1) <= 4; }

// the 3x3 symmetric multiply of one frequency with stored kernel values g
// (xx, yy, zz, xy, xz, yz), off-diagonal signs by the mirror flags, scaled
template <typename C>
__device__ __forceinline__ void zmul3(C& x0, C& x1, C& x2, const C (&g)[6], int rx, int ry, int rz,
                                      typename Real<C>::T s) {
  using Tr = typename Real<C>::T;
  const C gxy = cscale(g[3], (rx ^ ry) ? (Tr)-1 : (Tr)1);
  const C gxz = cscale(g[4], (rx ^ rz) ? (Tr)-1 : (Tr)1);
  const C gyz = cscale(g[5], (ry ^ rz) ? (Tr)-1 : (Tr)1);
  const C a = x0, b = x1, c = x2;
  x0 = cscale(cadd(cadd(cmul(g[0], a), cmul(gxy, b)), cmul(gxz, c)), s);
  x1 = cscale(cadd(cadd(cmul(gxy, a), cmul(g[1], b)), cmul(gyz, c)), s);
  x2 = cscale(cadd(cadd(cmul(gxz, a), cmul(gyz, b)), cmul(g[2], c)), s);
}

// Lengths whose fused stage can hold two tasks' values (3 * 2 * RL per
// thread): the mirror-pair form of k_zf_ct
template <typename C, int P>
constexpr bool zm_ok() {
  return ct_radix(P, ct_nst(P) - 1) <= 2 && (P / ct_radix(P, ct_nst(P) - 1)) % 2 == 0;
}

template <typename C, int P, int TX>
__global__ void __launch_bounds__(ct_threads(TX, P), zf_min_blocks(ct_threads(TX, P))) k_zf_ct(const ZParams<C> p) {
  using Tr = typename Real<C>::T;
  constexpr int T = ct_threads(TX, P);
  constexpr int CH = P * TX;
  constexpr int NST = ct_nst(P);
  constexpr int RL = ct_radix(P, NST - 1);  // last forward radix = first inverse radix
  constexpr int TPL = P / RL;
  constexpr int NTASK = TX * TPL;
  constexpr int K = (NTASK + T - 1) / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nrhs = p.nrhs, ntiles = p.ntiles, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = p.ts0 + rest % p.nts;  // [ts0, ts0 + nts) of the mirror tile order
  const int yseq = rest / p.nts;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int tmax = Px - kx0;
  const int64_t plane = (int64_t)Py * Px;
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  for (int q = threadIdx.x; q < 3 * nin * TX; q += T) {
    const int row = q / TX, t = q % TX;  // row = c * nin + z
    const int c = (int)p.nind.div((uint32_t)row);
    const int i = row - c * nin;
    if (t < tmax) cp_async(sm + c * CH + i * TX + t, Bb + (int64_t)row * plane + t);
  }
  cp_async_wait_all();
  __syncthreads();
  // forward stages 0 .. NST-2 of each component, in shared memory
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    C* const smc = sm + c * CH;
    auto ldf = [=](int t, int i) -> C {
      if (t < tmax && i < nin) return smc[i * TX + t];
      return czero<C>();
    };
    auto lds = [=](int t, int i) -> C { return smc[i * TX + t]; };
    auto sts = [=](int t, int i, C v) { smc[i * TX + t] = v; };
    ct_run_range<C, P, 0, 0, NST - 1, 8, T, TX, false, true, false>(p.tw, ldf, lds, sts, sts, true, true);
  }
  int py, iy, ry;
  ax_map(p.ax[1], ky + p.ky0, py, iy, ry);
  const int tx = p.tx, ty = p.ty, tz = p.tz;
  const Tr s = (Tr)p.scale;
  const C* const tw = p.tw;
  bool paired = false;
  if constexpr (zm_ok<C, P>()) {
    if (p.zmir && !p.ax[2].full) {
      // Mirror pairs: frequency j + r*TPL (this task's r-th value) and
      // P - j - r*TPL = (TPL - j) + (RL-1-r)*TPL (task TPL - j, value
      // RL-1-r) read the same stored kernel entry with mirrored signs, so
      // one thread takes both tasks and loads each entry once.  Task pair
      // (0, TPL/2) holds two self-mirrored sets and loads for both.  The
      // arithmetic per frequency is the single-task form's.
      constexpr int NPT = TX * (TPL / 2);
      constexpr int K2 = (NPT + T - 1) / T;
#pragma unroll
      for (int k = 0; k < K2; ++k) {
        const int task = (int)threadIdx.x + k * T;
        if (NPT % T != 0 && task >= NPT) continue;
        const int l = task % TX, jp = task / TX;
        if (l >= tmax) continue;  // columns past Px are never stored
        const int jj[2] = {jp, jp ? TPL - jp : TPL / 2};
        C v[2][3][RL];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < RL; ++r) v[h][c][r] = sm[c * CH + (jj[h] + r * TPL) * TX + l];
          C w[RL];
          twiddles<RL, false>(tw, jj[h], w);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int r = 1; r < RL; ++r) v[h][c][r] = cmul(v[h][c][r], w[r]);
            Bfly<RL, false, C>::run(v[h][c], tw, TPL);
          }
        }
        int px, ix, rx;
        ax_map(p.ax[0], kx0 + l, px, ix, rx);
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int f0 = jj[0] + r * TPL, f1 = jj[1] + (RL - 1 - r) * TPL;
          int pz0, iz0, rz0, pz1, iz1, rz1;
          ax_map(p.ax[2], f0, pz0, iz0, rz0);
          ax_map(p.ax[2], f1, pz1, iz1, rz1);
          C g[6];
          const C* gp = ker_at(p.ker, 4 * px + 2 * py + pz0, iz0, iy, ix, tx, ty, tz);
#pragma unroll
          for (int q = 0; q < 6; ++q) g[q] = ker_ld(gp, q, tx);
          zmul3(v[0][0][r], v[0][1][r], v[0][2][r], g, rx, ry, rz0, s);
          if (pz1 != pz0 || iz1 != iz0) {
            gp = ker_at(p.ker, 4 * px + 2 * py + pz1, iz1, iy, ix, tx, ty, tz);
#pragma unroll
            for (int q = 0; q < 6; ++q) g[q] = ker_ld(gp, q, tx);
          }
          zmul3(v[1][0][RL - 1 - r], v[1][1][RL - 1 - r], v[1][2][RL - 1 - r], g, rx, ry, rz1, s);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Bfly<RL, true, C>::run(v[h][c], tw, TPL);
#pragma unroll
            for (int r = 0; r < RL; ++r) sm[c * CH + (jj[h] + r * TPL) * TX + l] = v[h][c][r];
          }
      }
      paired = true;
    }
  }
  if (!paired) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = (int)threadIdx.x + k * T;
      if (NTASK % T != 0 && task >= NTASK) continue;
      const int l = task % TX, j = task / TX;
      if (l >= tmax) continue;  // columns past Px are never stored
      C v[3][RL];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < RL; ++r) v[c][r] = sm[c * CH + (j + r * TPL) * TX + l];
      // forward last stage (span TPL: twiddle exponent r * j)
      {
        C w[RL];
        twiddles<RL, false>(tw, j, w);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
          for (int r = 1; r < RL; ++r) v[c][r] = cmul(v[c][r], w[r]);
          Bfly<RL, false, C>::run(v[c], tw, TPL);
        }
      }
      // v[c][r] is frequency kz = j + r * TPL: 3x3 symmetric multiply with the
      // stored kernel (mirror / sign rules of mulBrnDev!)
      int px, ix, rx;
      ax_map(p.ax[0], kx0 + l, px, ix, rx);
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int kz = j + r * TPL;
        int pz, iz, rz;
        ax_map(p.ax[2], kz, pz, iz, rz);
        const C* gp = ker_at(p.ker, 4 * px + 2 * py + pz, iz, iy, ix, tx, ty, tz);
        const C gxx = ker_ld(gp, 0, tx), gyy = ker_ld(gp, 1, tx), gzz = ker_ld(gp, 2, tx);
        const C gxy = cscale(ker_ld(gp, 3, tx), (rx ^ ry) ? (Tr)-1 : (Tr)1);
        const C gxz = cscale(ker_ld(gp, 4, tx), (rx ^ rz) ? (Tr)-1 : (Tr)1);
        const C gyz = cscale(ker_ld(gp, 5, tx), (ry ^ rz) ? (Tr)-1 : (Tr)1);
        const C x0 = v[0][r], x1 = v[1][r], x2 = v[2][r];
        v[0][r] = cscale(cadd(cadd(cmul(gxx, x0), cmul(gxy, x1)), cmul(gxz, x2)), s);
        v[1][r] = cscale(cadd(cadd(cmul(gxy, x0), cmul(gyy, x1)), cmul(gyz, x2)), s);
        v[2][r] = cscale(cadd(cadd(cmul(gxz, x0), cmul(gyz, x1)), cmul(gzz, x2)), s);
      }
      // inverse first stage (span 1: no twiddles).  Its output of natural
      // index j * RL + r goes back to the slot the thread read, j + r * TPL,
      // so no thread overwrites a value another one has not read yet; the next
      // stage reads through that permutation.
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Bfly<RL, true, C>::run(v[c], tw, TPL);
#pragma unroll
        for (int r = 0; r < RL; ++r) sm[c * CH + (j + r * TPL) * TX + l] = v[c][r];
      }
    }
  }
  __syncthreads();
  // inverse stages 1 .. NST-1 (reversed radix order), truncated to the target z
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    C* const dc = sm + c * CH;
    C* const Bo = Bb + (int64_t)c * nout * plane;
    auto ldp = [=](int t, int q) -> C { return dc[((q / RL) + (q % RL) * TPL) * TX + t]; };
    auto ldo = [=](int t, int i) -> C { return dc[i * TX + t]; };
    auto sto = [=](int t, int i, C v) { dc[i * TX + t] = v; };
    auto stg = [=](int t, int i, C v) {
      if (t < tmax && i < nout) Bo[(int64_t)i * plane + t] = v;
    };
    ct_run_range<C, P, 1, 1, NST, 8, T, TX, true, true, true>(p.tw, ldp, ldo, sto, stg, true, false);
  }
}

// Two-stage fused z pass (FP64, P = 64 = 8 * 8).  The transform runs as two
// radix-8 stages:
//   A   forward, span 1: reads the source z planes of B straight into
//       registers (all loads of a thread in flight at once), writes the
//       shared tile;
//   F   forward, span 8, the 3x3 multiply and the inverse's first stage on
//       the same registers (as k_zf_ct), kernel values two frequencies ahead;
//   B'  inverse, span 8: reads the shared tile, writes the target z planes.
// Each element crosses shared memory twice instead of four times.  The same
// two-stage form at P = 128 and 256 (radix 16 / 32 outer stages) needs about
// 168 registers per thread; the lower occupancy cost more than the shared
// traffic saved (measured 2% and 14% slower than k_zf_ct), so only P = 64
// uses it (4% faster).
constexpr int zr_r1(int P) { return P / 8; }
constexpr int zr_threads(int TX, int P) { return TX * zr_r1(P); }
constexpr int zr_min_blocks(int T) { return 65536 / (T * 168) > 1 ? 65536 / (T * 168) : 1; }
constexpr bool zr_ok(int CS, int P, int TX) {
  return CS == 16 && P == 64 && zr_threads(TX, P) >= 32 && zr_threads(TX, P) <= 256 &&
         3LL * TX * P * CS <= 100 * 1024;
}

template <typename C, int P, int TX>
__global__ void __launch_bounds__(zr_threads(TX, P), zr_min_blocks(zr_threads(TX, P))) k_zr_ct(const ZParams<C> p) {
  using Tr = typename Real<C>::T;
  constexpr int R2 = 8, R1 = zr_r1(P);
  constexpr int T = TX * R1;
  constexpr int CH = P * TX;
  constexpr int NA = 3 * TX * R2;  // tasks of stages A and B': (component, line, j < R2)
  constexpr int KA = (NA + T - 1) / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nrhs = p.nrhs, ntiles = p.ntiles, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = p.ts0 + rest % p.nts;  // [ts0, ts0 + nts) of the mirror tile order
  const int yseq = rest / p.nts;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int tmax = Px - kx0;
  const int64_t plane = (int64_t)Py * Px;
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  const C* const tw = p.tw;
  // A: task (c, l, j) reads z = j + r * R2, r < R1 (zero past the source);
  // output natural index j * R1 + r.  All tasks' loads go out first.
  {
    C v[KA][R1];
#pragma unroll
    for (int k = 0; k < KA; ++k) {
      const int task = (int)threadIdx.x + k * T;
      const int l = task % TX, q = task / TX, j = q % R2, c = q / R2;
      const bool ok = (NA % T == 0 || task < NA) && l < tmax;
      const C* const src = Bb + (int64_t)c * nin * plane + l;
#pragma unroll
      for (int r = 0; r < R1; ++r) {
        const int i = j + r * R2;
        v[k][r] = (ok && i < nin) ? __ldcs(src + (int64_t)i * plane) : czero<C>();
      }
    }
#pragma unroll
    for (int k = 0; k < KA; ++k) {
      const int task = (int)threadIdx.x + k * T;
      if (NA % T == 0 || task < NA) {
        const int l = task % TX, q = task / TX, j = q % R2, c = q / R2;
        Bfly<R1, false, C>::run(v[k], tw, 0);
        C* const dst = sm + c * CH + (j * R1) * TX + l;
#pragma unroll
        for (int r = 0; r < R1; ++r) dst[r * TX] = v[k][r];
      }
    }
  }
  int py, iy, ry;
  ax_map(p.ax[1], ky + p.ky0, py, iy, ry);
  const int tx = p.tx, ty = p.ty, tz = p.tz;
  const Tr s = (Tr)p.scale;
  // F: task (l, j), j < R1: frequencies kz = j + r * R1
  const int l = (int)threadIdx.x % TX, j = (int)threadIdx.x / TX;
  int px, ix, rx;
  ax_map(p.ax[0], kx0 + l, px, ix, rx);
  auto kload = [&](int r, C* dst, int& rzo) {
    int pz, iz;
    ax_map(p.ax[2], j + r * R1, pz, iz, rzo);
    const C* gp = ker_at(p.ker, 4 * px + 2 * py + pz, iz, iy, ix, tx, ty, tz);
#pragma unroll
    for (int q = 0; q < 6; ++q) dst[q] = ker_ld(gp, q, tx);
  };
  // kernel values: two frequencies in flight (48 values for all eight do
  // not fit); the first two go out before the barrier, under the forward
  // stage
  C ga[6], gb[6];
  int rza = 0, rzb = 0;
  if (l < tmax) {
    kload(0, ga, rza);
    kload(1, gb, rzb);
  }
  __syncthreads();
  {
    if (l < tmax) {
      C v[3][R2];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < R2; ++r) v[c][r] = sm[c * CH + (j + r * R1) * TX + l];
      {
        C w[R2];
        twiddles<R2, false>(tw, j, w);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
          for (int r = 1; r < R2; ++r) v[c][r] = cmul(v[c][r], w[r]);
          Bfly<R2, false, C>::run(v[c], tw, R1);
        }
      }
#pragma unroll
      for (int r = 0; r < R2; ++r) {
        C* const g = (r & 1) ? gb : ga;
        const int rz = (r & 1) ? rzb : rza;
        const C gxx = g[0], gyy = g[1], gzz = g[2];
        const C gxy = cscale(g[3], (rx ^ ry) ? (Tr)-1 : (Tr)1);
        const C gxz = cscale(g[4], (rx ^ rz) ? (Tr)-1 : (Tr)1);
        const C gyz = cscale(g[5], (ry ^ rz) ? (Tr)-1 : (Tr)1);
        const C x0 = v[0][r], x1 = v[1][r], x2 = v[2][r];
        v[0][r] = cscale(cadd(cadd(cmul(gxx, x0), cmul(gxy, x1)), cmul(gxz, x2)), s);
        v[1][r] = cscale(cadd(cadd(cmul(gxy, x0), cmul(gyy, x1)), cmul(gyz, x2)), s);
        v[2][r] = cscale(cadd(cadd(cmul(gxz, x0), cmul(gyz, x1)), cmul(gzz, x2)), s);
        // refill the set just used with frequency r + 2
        asm volatile("" ::: "memory");
        if (r + 2 < R2) {
          if (r & 1)
            kload(r + 2, gb, rzb);
          else
            kload(r + 2, ga, rza);
        }
      }
      // inverse radix 8 (span 1): output natural index j * R2 + r goes back
      // to the slot read, j + r * R1
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Bfly<R2, true, C>::run(v[c], tw, R1);
#pragma unroll
        for (int r = 0; r < R2; ++r) sm[c * CH + (j + r * R1) * TX + l] = v[c][r];
      }
    }
  }
  __syncthreads();
  // B': task (c, l, j), j < R2, reads natural indices j + r * R2, which sit
  // in slots j * R1 + r; twiddles w^(-r j); output z = j + r * R2
#pragma unroll 1
  for (int k = 0; k < KA; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NA % T == 0 || task < NA) {
      const int l = task % TX, q = task / TX, j = q % R2, c = q / R2;
      const C* const srcs = sm + c * CH + (j * R1) * TX + l;
      C v[R1];
#pragma unroll
      for (int r = 0; r < R1; ++r) v[r] = srcs[r * TX];
#pragma unroll
      for (int r = 1; r < R1; ++r) v[r] = cmul(v[r], twid<true>(tw, r * j));
      Bfly<R1, true, C>::run(v, tw, 0);
      if (l < tmax) {
        C* const Bo = Bb + (int64_t)c * nout * plane + l;
#pragma unroll
        for (int r = 0; r < R1; ++r) {
          const int i = j + r * R2;
          if (i < nout) Bo[(int64_t)i * plane] = v[r];
        }
      }
    }
  }
}

// ------------------------------------------------------------------------
// Fused z pass, FP64, for lines whose source and target each fill at most
// half of the padded length (self operators and external ones whose z
// extents do not exceed half of P).  Same transform as k_zf_ct with fewer
// shared-memory round trips, FP64 instructions and barriers:
//   * forward stage 0 (radix 8, span 1) reads the source z planes of B
//     straight into registers, all of a thread's loads in flight at once,
//     and runs radix-8 butterflies whose upper four inputs are the known
//     zero padding;
//   * the middle stages run the three components back to back with one set
//     of twiddles per task and one barrier per component;
//   * the fused stage (forward last stage, 3x3 multiply, inverse first
//     stage) multiplies with FMA chains, flips the off-diagonal signs of the
//     mirror rules with sign-bit XORs instead of FP64 multiplies, and keeps
//     the next frequency's kernel values in flight;
//   * the last inverse stage (radix 8) forms only the four outputs that fall
//     in the target half and writes them straight to B.
// Results agree with k_zf_ct to rounding (both are checked against the
// oracle); every tile width and both task forms give identical bits.

// radix-8 DFT of v[0..3] with v[4..7] == 0
template <bool INV, typename C>
__device__ __forceinline__ void bfly8_half_in(C* v) {
  using T = typename Real<C>::T;
  const T h = (T)0.70710678118654752440084436210484903928;
  const C a = v[0], b = v[2], c = v[1], d = v[3];
  const C ib = cmuli<INV>(b), id = cmuli<INV>(d);
  C e[4] = {cadd(a, b), cadd(a, ib), csub(a, b), csub(a, ib)};
  C o[4] = {cadd(c, d), cadd(c, id), csub(c, d), csub(c, id)};
  const C o1 = o[1], o3 = o[3];
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

// radix-8 DFT of v[0..7] whose outputs 0..3 only are needed (into v[0..3])
template <bool INV, typename C>
__device__ __forceinline__ void bfly8_half_out(C* v) {
  using T = typename Real<C>::T;
  const T h = (T)0.70710678118654752440084436210484903928;
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
  Bfly<4, INV, C>::run(e, nullptr, 0);
  Bfly<4, INV, C>::run(o, nullptr, 0);
  const C o1 = o[1], o3 = o[3];
  if (!INV) {
    o[1] = cmake<C>(h * (o1.x + o1.y), h * (o1.y - o1.x));
    o[3] = cmake<C>(h * (o3.y - o3.x), -h * (o3.x + o3.y));
  } else {
    o[1] = cmake<C>(h * (o1.x - o1.y), h * (o1.x + o1.y));
    o[3] = cmake<C>(-h * (o3.x + o3.y), h * (o3.x - o3.y));
  }
  o[2] = cmuli<INV>(o[2]);
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = cadd(e[k], o[k]);
}

// a with both parts' signs flipped when f != 0: a sign-bit XOR on the high
// words, no FP64 instruction
__device__ __forceinline__ double2 cflip(double2 a, int f) {
  const long long m = (long long)(f != 0) << 63;
  return make_double2(__longlong_as_double(__double_as_longlong(a.x) ^ m),
                      __longlong_as_double(__double_as_longlong(a.y) ^ m));
}

// s * (g0 a + g1 b + g2 c) as two FMA chains
__device__ __forceinline__ double2 mac3(const double2& g0, const double2& a, const double2& g1, const double2& b,
                                       const double2& g2, const double2& c, double s) {
  double re = g0.x * a.x;
  re = fma(-g0.y, a.y, re);
  re = fma(g1.x, b.x, re);
  re = fma(-g1.y, b.y, re);
  re = fma(g2.x, c.x, re);
  re = fma(-g2.y, c.y, re);
  double im = g0.x * a.y;
  im = fma(g0.y, a.x, im);
  im = fma(g1.x, b.y, im);
  im = fma(g1.y, b.x, im);
  im = fma(g2.x, c.y, im);
  im = fma(g2.y, c.x, im);
  return make_double2(re * s, im * s);
}

// the 3x3 symmetric multiply of one frequency (stored kernel g: xx, yy, zz,
// xy, xz, yz; mirror flags rx, ry, rz), scaled by s
__device__ __forceinline__ void zmul3f(double2& x0, double2& x1, double2& x2, const double2 (&g)[6], int rx, int ry,
                                       int rz, double s) {
  const double2 gxy = cflip(g[3], rx ^ ry), gxz = cflip(g[4], rx ^ rz), gyz = cflip(g[5], ry ^ rz);
  const double2 a = x0, b = x1, c = x2;
  x0 = mac3(g[0], a, gxy, b, gxz, c, s);
  x1 = mac3(gxy, a, g[1], b, gyz, c, s);
  x2 = mac3(gxz, a, gyz, b, g[2], c, s);
}

template <int P>
constexpr bool zg_ok() {
  return ct_nst(P) >= 3 && ct_radix(P, 0) == 8 && ct_radix(P, ct_nst(P) - 1) <= 4;
}

// One in-place middle stage S (radix order REV) over the three component
// blocks of the tile, twiddles computed once per task.  Input index q of a
// line sits in slot slot(q); outputs go to their natural slots.  One barrier
// per component, between its loads and its stores; the stores of one stage
// and the loads of the next are ordered by the barriers of the components
// in between (callers put a barrier before a stage that follows a stage
// writing all three components at once).
template <int P, int S, int T, int TX, bool INV, bool REV, class Slot>
__device__ __forceinline__ void zg_mid(double2* sm, const double2* __restrict__ tw, const Slot& slot) {
  constexpr int R = ct_radix_o<REV>(P, S), NS = ct_span_o<REV>(P, S), TPL = P / R, NT = TX * TPL;
  constexpr int K = (NT + T - 1) / T, TWST = P / (NS * R), CH = P * TX;
  double2 w[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    const int j = task / TX;
    if (NS > 1) twiddles<R, INV>(tw, (j % NS) * TWST, w[k]);
  }
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    double2* const smc = sm + c * CH;
    double2 v[K][R];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = (int)threadIdx.x + k * T;
      if (NT % T == 0 || task < NT) {
        const int l = task % TX, j = task / TX;
#pragma unroll
        for (int r = 0; r < R; ++r) v[k][r] = smc[slot(j + r * TPL) * TX + l];
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = (int)threadIdx.x + k * T;
      if (NT % T == 0 || task < NT) {
        const int l = task % TX, j = task / TX, jm = j % NS;
        if (NS > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) v[k][r] = cmul(v[k][r], w[k][r]);
        }
        Bfly<R, INV, double2>::run(v[k], tw, TPL);
        const int base = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) smc[(base + r * NS) * TX + l] = v[k][r];
      }
    }
  }
}

template <int P, int TX>
__global__ void __launch_bounds__(ct_threads(TX, P), zf_min_blocks(ct_threads(TX, P))) k_zg_ct(const ZParams<double2> p) {
  using C = double2;
  constexpr int T = ct_threads(TX, P);
  constexpr int CH = P * TX;
  constexpr int NST = ct_nst(P);
  constexpr int RL = ct_radix(P, NST - 1);  // last forward radix = first inverse radix
  constexpr int TPL = P / RL;
  constexpr int TPL0 = P / 8, NT0 = TX * TPL0, K0 = (NT0 + T - 1) / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nrhs = p.nrhs, ntiles = p.ntiles, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = p.ts0 + rest % p.nts;  // [ts0, ts0 + nts) of the mirror tile order
  const int yseq = rest / p.nts;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int tmax = Px - kx0;
  const int64_t plane = (int64_t)Py * Px;
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  const C* const tw = p.tw;
  // forward stage 0: task (l, j0) reads z = j0 + r * TPL0, r < 4 (the upper
  // half of the padded line is zero); output slot j0 * 8 + r
  {
    C v[3][K0][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < K0; ++k) {
        const int task = (int)threadIdx.x + k * T;
        const int l = task % TX, j0 = task / TX;
        const bool ok = (NT0 % T == 0 || task < NT0) && l < tmax;
        const C* const src = Bb + (int64_t)c * nin * plane + l;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = j0 + r * TPL0;
          v[c][k][r] = (ok && i < nin) ? __ldcs(src + (int64_t)i * plane) : czero<C>();
        }
      }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < K0; ++k) {
        const int task = (int)threadIdx.x + k * T;
        if (NT0 % T == 0 || task < NT0) {
          const int l = task % TX, j0 = task / TX;
          bfly8_half_in<false>(v[c][k]);
          C* const dst = sm + c * CH + (j0 * 8) * TX + l;
#pragma unroll
          for (int r = 0; r < 8; ++r) dst[r * TX] = v[c][k][r];
        }
      }
  }
  __syncthreads();
  // forward middle stages 1 .. NST-2
  {
    auto nat = [](int q) { return q; };
    if constexpr (NST >= 3) zg_mid<P, 1, T, TX, false, false>(sm, tw, nat);
    if constexpr (NST >= 4) zg_mid<P, 2, T, TX, false, false>(sm, tw, nat);
    if constexpr (NST >= 5) zg_mid<P, 3, T, TX, false, false>(sm, tw, nat);
  }
  int py, iy, ry;
  ax_map(p.ax[1], ky + p.ky0, py, iy, ry);
  const int tx = p.tx, ty = p.ty, tz = p.tz;
  const double s = p.scale;
  auto kload = [&](int px, int ix, int f, C (&g)[6], int& rz) {
    int pz, iz;
    ax_map(p.ax[2], f, pz, iz, rz);
    const C* gp = ker_at(p.ker, 4 * px + 2 * py + pz, iz, iy, ix, tx, ty, tz);
#pragma unroll
    for (int q = 0; q < 6; ++q) g[q] = ker_ld(gp, q, tx);
  };
  bool paired = false;
  if constexpr (zm_ok<C, P>()) {
    if (p.zmir && !p.ax[2].full) {
      // mirror pairs of z frequencies (see k_zf_ct): frequency j + r*TPL of
      // task j and P - j - r*TPL of task TPL - j read the same stored entry
      constexpr int NPT = TX * (TPL / 2);
      constexpr int K2 = (NPT + T - 1) / T;
#pragma unroll
      for (int k = 0; k < K2; ++k) {
        const int task = (int)threadIdx.x + k * T;
        const bool live = (NPT % T == 0 || task < NPT) && task % TX < tmax;
        const int l = task % TX, jp = task / TX;
        const int jj[2] = {jp, jp ? TPL - jp : TPL / 2};
        int px = 0, ix = 0, rx = 0;
        ax_map(p.ax[0], kx0 + l, px, ix, rx);
        // the first frequency's kernel values go out before the barrier
        C g[6];
        int rzg = 0;
        if (live) kload(px, ix, jj[0], g, rzg);
        if (k == 0) __syncthreads();
        if (!live) continue;
        C v[2][3][RL];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < RL; ++r) v[h][c][r] = sm[c * CH + (jj[h] + r * TPL) * TX + l];
          C w[RL];
          twiddles<RL, false>(tw, jj[h], w);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int r = 1; r < RL; ++r) v[h][c][r] = cmul(v[h][c][r], w[r]);
            Bfly<RL, false, C>::run(v[h][c], tw, TPL);
          }
        }
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const int f0 = jj[0] + r * TPL, f1 = jj[1] + (RL - 1 - r) * TPL;
          int pz0, iz0, rz0, pz1, iz1, rz1;
          ax_map(p.ax[2], f0, pz0, iz0, rz0);
          ax_map(p.ax[2], f1, pz1, iz1, rz1);
          zmul3f(v[0][0][r], v[0][1][r], v[0][2][r], g, rx, ry, rz0, s);
          if (pz1 != pz0 || iz1 != iz0) {
            // the self-mirrored pair (0, TPL/2): its own entry
            C g1[6];
            int rzx = 0;
            kload(px, ix, f1, g1, rzx);
            zmul3f(v[1][0][RL - 1 - r], v[1][1][RL - 1 - r], v[1][2][RL - 1 - r], g1, rx, ry, rz1, s);
          } else {
            zmul3f(v[1][0][RL - 1 - r], v[1][1][RL - 1 - r], v[1][2][RL - 1 - r], g, rx, ry, rz1, s);
          }
          // next frequency's entry (two tasks' values already fill the
          // registers: no second set in flight)
          if (r + 1 < RL) kload(px, ix, jj[0] + (r + 1) * TPL, g, rzg);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            Bfly<RL, true, C>::run(v[h][c], tw, TPL);
#pragma unroll
            for (int r = 0; r < RL; ++r) sm[c * CH + (jj[h] + r * TPL) * TX + l] = v[h][c][r];
          }
      }
      paired = true;
    }
  }
  if (!paired) {
    constexpr int NTASK = TX * TPL;
    constexpr int K = (NTASK + T - 1) / T;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = (int)threadIdx.x + k * T;
      const bool live = (NTASK % T == 0 || task < NTASK) && task % TX < tmax;
      const int l = task % TX, j = task / TX;
      int px = 0, ix = 0, rx = 0;
      ax_map(p.ax[0], kx0 + l, px, ix, rx);
      // the first frequency's kernel values go out before the barrier
      C g[6];
      int rz = 0;
      if (live) kload(px, ix, j, g, rz);
      if (k == 0) __syncthreads();
      if (!live) continue;
      C v[3][RL];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < RL; ++r) v[c][r] = sm[c * CH + (j + r * TPL) * TX + l];
      {
        C w[RL];
        twiddles<RL, false>(tw, j, w);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
          for (int r = 1; r < RL; ++r) v[c][r] = cmul(v[c][r], w[r]);
          Bfly<RL, false, C>::run(v[c], tw, TPL);
        }
      }
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        C gn[6];
        int rzn = 0;
        if (r + 1 < RL) kload(px, ix, j + (r + 1) * TPL, gn, rzn);
        zmul3f(v[0][r], v[1][r], v[2][r], g, rx, ry, rz, s);
        if (r + 1 < RL) {
#pragma unroll
          for (int q = 0; q < 6; ++q) g[q] = gn[q];
          rz = rzn;
        }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Bfly<RL, true, C>::run(v[c], tw, TPL);
#pragma unroll
        for (int r = 0; r < RL; ++r) sm[c * CH + (j + r * TPL) * TX + l] = v[c][r];
      }
    }
  }
  __syncthreads();
  // inverse middle stages 1 .. NST-2 (reversed radix order); stage 1 reads
  // through the fused stage's permutation (input q in slot q/RL + (q%RL)*TPL)
  {
    auto perm = [](int q) { return (q / RL) + (q % RL) * TPL; };
    auto nat = [](int q) { return q; };
    if constexpr (NST >= 3) zg_mid<P, 1, T, TX, true, true>(sm, tw, perm);
    if constexpr (NST >= 4) zg_mid<P, 2, T, TX, true, true>(sm, tw, nat);
    if constexpr (NST >= 5) zg_mid<P, 3, T, TX, true, true>(sm, tw, nat);
  }
  __syncthreads();
  // inverse last stage (radix 8, span TPL0): outputs z = j + r * TPL0, r < 4
  // (the target half), straight to the target z planes of B
  {
    constexpr int NSL = TPL0;
    double2 w[K0][8];
#pragma unroll
    for (int k = 0; k < K0; ++k) {
      const int task = (int)threadIdx.x + k * T;
      twiddles<8, true>(tw, task / TX, w[k]);
    }
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      const C* const smc = sm + c * CH;
      C* const Bo = Bb + (int64_t)c * nout * plane;
#pragma unroll
      for (int k = 0; k < K0; ++k) {
        const int task = (int)threadIdx.x + k * T;
        if (NT0 % T == 0 || task < NT0) {
          const int l = task % TX, j = task / TX;
          C v[8];
#pragma unroll
          for (int r = 0; r < 8; ++r) v[r] = smc[(j + r * NSL) * TX + l];
#pragma unroll
          for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], w[k][r]);
          bfly8_half_out<true>(v);
          if (l < tmax) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              const int i = j + r * NSL;
              if (i < nout) __stcs(Bo + (int64_t)i * plane + l, v[r]);
            }
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------------------
// x and y passes (FP64) whose first stage is fed from global memory and
// whose last stage forms only the target half: the forward passes load only
// the source half of each padded line (radix-R0 butterflies with the upper
// inputs known zero), every thread's loads in flight at once, instead of
// staging the line through shared memory; the inverse passes load the full
// spectrum line the same way and run a last butterfly that forms only the
// outputs inside the target.  One shared-memory round trip per element
// fewer than k_xfwd_ct / k_y_ct / k_xinv_ct, and fewer FP64 operations.

template <int R, bool INV, typename C>
__device__ __forceinline__ void bfly_half_in(C* v) {
  if constexpr (R == 8) {
    bfly8_half_in<INV>(v);
  } else if constexpr (R == 4) {
    const C a = v[0], b = v[1], ib = cmuli<INV>(v[1]);
    v[0] = cadd(a, b);
    v[1] = cadd(a, ib);
    v[2] = csub(a, b);
    v[3] = csub(a, ib);
  } else {
    static_assert(R == 2, "half-input butterflies: radix 2, 4, 8");
    v[1] = v[0];
  }
}

template <int R, bool INV, typename C>
__device__ __forceinline__ void bfly_half_out(C* v) {
  if constexpr (R == 8) {
    bfly8_half_out<INV>(v);
  } else if constexpr (R == 4) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const C t2 = cadd(v[1], v[3]), t3 = cmuli<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[1] = cadd(t1, t3);
  } else {
    static_assert(R == 2, "half-output butterflies: radix 2, 4, 8");
    v[0] = cadd(v[0], v[1]);
  }
}

constexpr bool pow2_radix(int r) { return r == 2 || r == 4 || r == 8; }
template <int P, bool REV>
constexpr bool xyg_in_ok() {
  return ct_nst(P) >= 2 && pow2_radix(ct_radix_o<REV>(P, 0));
}
template <int P, bool REV>
constexpr bool xyg_out_ok() {
  return ct_nst(P) >= 2 && pow2_radix(ct_radix_o<REV>(P, ct_nst(P) - 1));
}

// Stage 0 (span 1) fed from global memory: task (l, j) loads inputs j + r *
// (P / R0) with gld(l, i), r < R0 / 2 when HALF (the rest is the zero
// padding), then butterflies and st(l, j * R0 + r, v).
template <typename C, int P, int T, int M, bool INV, bool LINE_FAST, bool REV, bool HALF, class GLd, class St>
__device__ __forceinline__ void ct_first_g(const GLd& gld, const St& st) {
  constexpr int R = ct_radix_o<REV>(P, 0), TPL = P / R, NT = M * TPL, K = (NT + T - 1) / T;
  constexpr int RIN = HALF ? R / 2 : R;
  C v[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NT % T == 0 || task < NT) {
      const int l = LINE_FAST ? task % M : task / TPL, j = LINE_FAST ? task / M : task % TPL;
#pragma unroll
      for (int r = 0; r < RIN; ++r) v[k][r] = gld(l, j + r * TPL);
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NT % T == 0 || task < NT) {
      const int l = LINE_FAST ? task % M : task / TPL, j = LINE_FAST ? task / M : task % TPL;
      if constexpr (HALF)
        bfly_half_in<R, INV>(v[k]);
      else
        Bfly<R, INV, C>::run(v[k], nullptr, TPL);
#pragma unroll
      for (int r = 0; r < R; ++r) st(l, j * R + r, v[k][r]);
    }
  }
}

// Last stage (span P / R) forming outputs j + r * (P / R) for r < R / 2
// only: ld reads the stage input, st takes the outputs.
template <typename C, int P, int T, int M, bool INV, bool LINE_FAST, bool REV, class Ld, class St>
__device__ __forceinline__ void ct_last_half(const C* __restrict__ tw, const Ld& ld, const St& st) {
  constexpr int S = ct_nst(P) - 1;
  constexpr int R = ct_radix_o<REV>(P, S), NS = ct_span_o<REV>(P, S), TPL = P / R, NT = M * TPL;
  constexpr int K = (NT + T - 1) / T, TWST = P / (NS * R);
  static_assert(NS == TPL, "the last stage spans P / R");
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NT % T == 0 || task < NT) {
      const int l = LINE_FAST ? task % M : task / TPL, j = LINE_FAST ? task / M : task % TPL;
      C v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = ld(l, j + r * TPL);
      C w[R];
      twiddles<R, INV>(tw, j * TWST, w);
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
      bfly_half_out<R, INV>(v);
#pragma unroll
      for (int r = 0; r < R / 2; ++r) st(l, j + r * NS, v[r]);
    }
  }
}

template <int P, bool REV>
__global__ void __launch_bounds__(ct_threads(ct_xlines<16>(P), P)) k_xfwd_g(const XfParams<double2> p) {
  using C = double2;
  constexpr int M = ct_xlines<16>(P);
  constexpr int T = ct_threads(M, P);
  constexpr int LS = P + (P + 7) / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nin = p.nin;
  const int64_t rows = p.rows;
  C* const A = p.A;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const C* const src = p.in + g0 * nin;
  auto gld = [=](int l, int i) -> C {
    return (g0 + l < rows && i < nin) ? __ldcs(src + (int64_t)l * nin + i) : czero<C>();
  };
  auto lds = [=](int l, int i) -> C { return sm[l * LS + i + (i >> 3)]; };
  auto sts = [=](int l, int i, C v) { sm[l * LS + i + (i >> 3)] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g < rows) A[g * P + i] = v;
  };
  ct_first_g<C, P, T, M, false, false, REV, true>(gld, sts);
  __syncthreads();
  ct_run_range<C, P, 1, 1, ct_nst(P), 8, T, M, false, false, REV>(p.tw, lds, lds, sts, stg, true, false);
}

template <int P, bool INV, int TX, bool REV>
__global__ void __launch_bounds__(ct_threads(TX, P), pow2_min_blocks(ct_threads(TX, P), P)) k_y_g(const YParams<double2> p) {
  using C = double2;
  constexpr int T = ct_threads(TX, P);
  constexpr int NST = ct_nst(P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int Px = p.Px, nin = p.nin, nout = p.nout;
  const int tl = blockIdx.x % p.nt;  // tile of the kx set: low range, then high range
  const int tile = tl < p.nlo ? p.lo0 + tl : p.hi0 + (tl - p.nlo);
  const int64_t slice = p.q0 + blockIdx.x / p.nt;  // ch*nz + z
  const int64_t rc = slice / p.nz;
  const int z = (int)(slice % p.nz);
  const int kx0 = tile * TX;
  const C* const src = p.src + ((rc * p.src_z + z) - p.src_sub) * p.src_rows * (int64_t)Px + kx0;
  C* const dst = p.dst + ((rc * p.dst_z + z) - p.dst_sub) * p.dst_rows * (int64_t)Px + kx0;
  const int tmax = Px - kx0;
  auto gld = [=](int t, int i) -> C {
    return (t < tmax && i < nin) ? __ldcs(src + (int64_t)i * Px + t) : czero<C>();
  };
  auto lds = [=](int t, int i) -> C { return sm[i * TX + t]; };
  auto sts = [=](int t, int i, C v) { sm[i * TX + t] = v; };
  auto stg = [=](int t, int i, C v) {
    if (t < tmax && i < nout) {
      // the forward pass writes the spectrum B (streamed through L2), the
      // inverse pass the x/y slab that the x-inverse pass reads next
      if constexpr (!INV)
        __stcs(dst + (int64_t)i * Px + t, v);
      else
        dst[(int64_t)i * Px + t] = v;
    }
  };
  if constexpr (!INV) {
    ct_first_g<C, P, T, TX, false, true, REV, true>(gld, sts);
    __syncthreads();
    ct_run_range<C, P, 1, 1, NST, 8, T, TX, false, true, REV>(p.tw, lds, lds, sts, stg, true, false);
  } else {
    ct_first_g<C, P, T, TX, true, true, REV, false>(gld, sts);
    __syncthreads();
    ct_run_range<C, P, 1, 1, NST - 1, 8, T, TX, true, true, REV>(p.tw, lds, lds, sts, sts, true, true);
    ct_last_half<C, P, T, TX, true, true, REV>(p.tw, lds, stg);
  }
}

template <int P, bool AXPBY, bool REV>
__global__ void __launch_bounds__(ct_threads(ct_xlines<16>(P), P)) k_xinv_g(const XiParams<double2> p) {
  using C = double2;
  constexpr int M = ct_xlines<16>(P);
  constexpr int T = ct_threads(M, P);
  constexpr int LS = P + (P + 7) / 8;
  constexpr int NST = ct_nst(P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nout = p.nout;
  const int64_t rows = p.rows;
  C* const out = p.out;
  const C alpha = p.alpha, beta = p.beta;
  const int ls = p.ls;
  const C* const ls_in = p.ls_in;
  const C* const ls_chi = p.ls_chi;
  const int64_t ls_chi_rs = p.ls_chi_rs;
  const FDiv rows_rhs = p.rows_rhs, rows_zy = p.rows_zy;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const bool scatter = p.part_scatter != 0;
  const int ty = p.ty, tz = p.tz, parT = p.parT;
  const int d0 = p.tdiv[0], d1 = p.tdiv[1], d2 = p.tdiv[2];
  const int64_t f0 = p.full[0], f1 = p.full[1], f2 = p.full[2];
  const int(*toff)[3] = p.toff;
  const int64_t g_off = p.g_off;
  const C* const src = p.A + g0 * P;
  auto gld = [=](int l, int i) -> C { return g0 + l < rows ? __ldcs(src + (int64_t)l * P + i) : czero<C>(); };
  auto lds = [=](int l, int i) -> C { return sm[l * LS + i + (i >> 3)]; };
  auto sts = [=](int l, int i, C v) { sm[l * LS + i + (i >> 3)] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g >= rows || i >= nout) return;
    int64_t o;
    const int64_t gg = g + g_off;
    if (!scatter) {
      o = gg * nout + i;
    } else {
      int64_t q = gg;
      const int y = (int)(q % ty); q /= ty;
      const int z = (int)(q % tz); q /= tz;
      const int c = (int)(q % 3); q /= 3;
      const int t = (int)(q % parT);
      const int64_t rhs = q / parT;
      const int64_t X = (int64_t)i * d0 + toff[t][0];
      const int64_t Y = (int64_t)y * d1 + toff[t][1];
      const int64_t Z = (int64_t)z * d2 + toff[t][2];
      o = (((rhs * 3 + c) * f2 + Z) * f1 + Y) * f0 + X;
    }
    if (AXPBY)
      out[o] = cadd(cmul(alpha, v), cmul(beta, out[o]));
    else if (ls)
      __stcs(out + o, ls_value(ls_in, ls_chi, ls_chi_rs, rows_rhs, rows_zy, nout, gg, i, o, v));
    else
      __stcs(out + o, v);
  };
  ct_first_g<C, P, T, M, true, false, REV, false>(gld, sts);
  __syncthreads();
  ct_run_range<C, P, 1, 1, NST - 1, 8, T, M, true, false, REV>(p.tw, lds, lds, sts, sts, true, true);
  ct_last_half<C, P, T, M, true, false, REV>(p.tw, lds, stg);
}

// FP32 x / y passes on line pairs with the global-fed first stage and the
// half last stage of k_xfwd_g / k_y_g / k_xinv_g.
template <int P, int T, int M2, bool INV, bool LF, bool REV, bool HALF, class GLd, class St>
__device__ __forceinline__ void ct_first_g2(const GLd& gld, const St& st) {
  constexpr int R = ct_radix_o<REV>(P, 0), TPL = P / R, NT = M2 * TPL, K = (NT + T - 1) / T;
  constexpr int RIN = HALF ? R / 2 : R;
  float2 a[K][R], b[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NT % T == 0 || task < NT) {
      const int lp = LF ? task % M2 : task / TPL, j = LF ? task / M2 : task % TPL;
#pragma unroll
      for (int r = 0; r < RIN; ++r) {
        const float4 q = gld(lp, j + r * TPL);
        a[k][r] = make_float2(q.x, q.y);
        b[k][r] = make_float2(q.z, q.w);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NT % T == 0 || task < NT) {
      const int lp = LF ? task % M2 : task / TPL, j = LF ? task / M2 : task % TPL;
      if constexpr (HALF) {
        bfly_half_in<R, INV>(a[k]);
        bfly_half_in<R, INV>(b[k]);
      } else {
        Bfly<R, INV, float2>::run(a[k], nullptr, TPL);
        Bfly<R, INV, float2>::run(b[k], nullptr, TPL);
      }
#pragma unroll
      for (int r = 0; r < R; ++r) st(lp, j * R + r, make_float4(a[k][r].x, a[k][r].y, b[k][r].x, b[k][r].y));
    }
  }
}

template <int P, int T, int M2, bool INV, bool LF, bool REV, class Ld, class St>
__device__ __forceinline__ void ct_last_half2(const float2* __restrict__ tw, const Ld& ld, const St& st) {
  constexpr int S = ct_nst(P) - 1;
  constexpr int R = ct_radix_o<REV>(P, S), NS = ct_span_o<REV>(P, S), TPL = P / R, NT = M2 * TPL;
  constexpr int K = (NT + T - 1) / T, TWST = P / (NS * R);
  static_assert(NS == TPL, "the last stage spans P / R");
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NT % T == 0 || task < NT) {
      const int lp = LF ? task % M2 : task / TPL, j = LF ? task / M2 : task % TPL;
      float2 a[R], b[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float4 q = ld(lp, j + r * TPL);
        a[r] = make_float2(q.x, q.y);
        b[r] = make_float2(q.z, q.w);
      }
      float2 w[R];
      twiddles<R, INV>(tw, j * TWST, w);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        a[r] = cmul(a[r], w[r]);
        b[r] = cmul(b[r], w[r]);
      }
      bfly_half_out<R, INV>(a);
      bfly_half_out<R, INV>(b);
#pragma unroll
      for (int r = 0; r < R / 2; ++r) st(lp, j + r * NS, make_float4(a[r].x, a[r].y, b[r].x, b[r].y));
    }
  }
}

template <int P, bool REV>
__global__ void __launch_bounds__(ct_threads2(ct_xlines2<8>(P), P)) k_xfwd2_g(const XfParams<float2> p) {
  constexpr int M = ct_xlines2<8>(P);
  constexpr int M2 = M / 2;
  constexpr int T = ct_threads2(M, P);
  constexpr int LS = P + (P + 7) / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* const sm = reinterpret_cast<float4*>(smem_raw);
  const int nin = p.nin;
  const int64_t rows = p.rows;
  float2* const A = p.A;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const float2* const src = p.in + g0 * nin;
  const float2 z2 = make_float2(0.f, 0.f);
  auto gld = [=](int lp, int i) -> float4 {
    const bool in = i < nin;
    const float2 u = (in && g0 + 2 * lp < rows) ? __ldcs(src + (int64_t)(2 * lp) * nin + i) : z2;
    const float2 v = (in && g0 + 2 * lp + 1 < rows) ? __ldcs(src + (int64_t)(2 * lp + 1) * nin + i) : z2;
    return make_float4(u.x, u.y, v.x, v.y);
  };
  auto lds = [=](int lp, int i) -> float4 { return sm[lp * LS + i + (i >> 3)]; };
  auto sts = [=](int lp, int i, float4 v) { sm[lp * LS + i + (i >> 3)] = v; };
  auto stg = [=](int lp, int i, float4 v) {
    const int64_t g = g0 + 2 * lp;
    if (g < rows) A[g * P + i] = make_float2(v.x, v.y);
    if (g + 1 < rows) A[(g + 1) * P + i] = make_float2(v.z, v.w);
  };
  ct_first_g2<P, T, M2, false, false, REV, true>(gld, sts);
  __syncthreads();
  ct_run_range2<P, 1, 1, ct_nst(P), T, M2, false, REV, false>(p.tw, lds, lds, sts, stg, true, false);
}

template <int P, bool REV>
__global__ void __launch_bounds__(ct_threads2(ct_xlines2<8>(P), P)) k_xinv2_g(const XiParams<float2> p) {
  constexpr int M = ct_xlines2<8>(P);
  constexpr int M2 = M / 2;
  constexpr int T = ct_threads2(M, P);
  constexpr int LS = P + (P + 7) / 8;
  constexpr int NST = ct_nst(P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* const sm = reinterpret_cast<float4*>(smem_raw);
  const int nout = p.nout;
  const int64_t rows = p.rows;
  float2* const out = p.out;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const int64_t g_off = p.g_off;
  const int ls = p.ls;
  const float2* const ls_in = p.ls_in;
  const float2* const ls_chi = p.ls_chi;
  const int64_t ls_chi_rs = p.ls_chi_rs;
  const FDiv rows_rhs = p.rows_rhs, rows_zy = p.rows_zy;
  const float2* const src = p.A + g0 * P;
  const float2 z2 = make_float2(0.f, 0.f);
  auto gld = [=](int lp, int i) -> float4 {
    const float2 u = g0 + 2 * lp < rows ? __ldcs(src + (int64_t)(2 * lp) * P + i) : z2;
    const float2 v = g0 + 2 * lp + 1 < rows ? __ldcs(src + (int64_t)(2 * lp + 1) * P + i) : z2;
    return make_float4(u.x, u.y, v.x, v.y);
  };
  auto lds = [=](int lp, int i) -> float4 { return sm[lp * LS + i + (i >> 3)]; };
  auto sts = [=](int lp, int i, float4 v) { sm[lp * LS + i + (i >> 3)] = v; };
  auto stg = [=](int lp, int i, float4 v) {
    if (i >= nout) return;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t g = g0 + 2 * lp + h;
      if (g >= rows) return;
      const int64_t gg = g + g_off;
      const int64_t o = gg * nout + i;
      const float2 w = h ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
      __stcs(out + o, ls ? ls_value(ls_in, ls_chi, ls_chi_rs, rows_rhs, rows_zy, nout, gg, i, o, w) : w);
    }
  };
  ct_first_g2<P, T, M2, true, false, REV, false>(gld, sts);
  __syncthreads();
  ct_run_range2<P, 1, 1, NST - 1, T, M2, true, REV, false>(p.tw, lds, lds, sts, sts, true, true);
  ct_last_half2<P, T, M2, true, false, REV>(p.tw, lds, stg);
}

template <int P, bool INV, int TX, bool REV>
__global__ void __launch_bounds__(ct_threads2(TX, P), pow2_min_blocks(ct_threads2(TX, P), P)) k_y2_g(const YParams<float2> p) {
  constexpr int T = ct_threads2(TX, P);
  constexpr int M2 = TX / 2;
  constexpr int NST = ct_nst(P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* const sm = reinterpret_cast<float4*>(smem_raw);
  const int Px = p.Px, nin = p.nin, nout = p.nout;
  const int tl = blockIdx.x % p.nt;  // tile of the kx set: low range, then high range
  const int tile = tl < p.nlo ? p.lo0 + tl : p.hi0 + (tl - p.nlo);
  const int64_t slice = p.q0 + blockIdx.x / p.nt;  // ch*nz + z
  const int64_t rc = slice / p.nz;
  const int z = (int)(slice % p.nz);
  const int kx0 = tile * TX;
  const float2* const src = p.src + ((rc * p.src_z + z) - p.src_sub) * p.src_rows * (int64_t)Px + kx0;
  float2* const dst = p.dst + ((rc * p.dst_z + z) - p.dst_sub) * p.dst_rows * (int64_t)Px + kx0;
  const int tmax = Px - kx0;  // even: Px and kx0 are even
  auto gld = [=](int t2, int i) -> float4 {
    return (2 * t2 < tmax && i < nin) ? __ldcs(reinterpret_cast<const float4*>(src + (int64_t)i * Px) + t2)
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
  };
  auto lds = [=](int t2, int i) -> float4 { return sm[i * M2 + t2]; };
  auto sts = [=](int t2, int i, float4 v) { sm[i * M2 + t2] = v; };
  auto stg = [=](int t2, int i, float4 v) {
    if (2 * t2 < tmax && i < nout) {
      float4* const q = reinterpret_cast<float4*>(dst + (int64_t)i * Px) + t2;
      if constexpr (!INV)
        __stcs(q, v);
      else
        *q = v;
    }
  };
  if constexpr (!INV) {
    ct_first_g2<P, T, M2, false, true, REV, true>(gld, sts);
    __syncthreads();
    ct_run_range2<P, 1, 1, NST, T, M2, false, REV, true>(p.tw, lds, lds, sts, stg, true, false);
  } else {
    ct_first_g2<P, T, M2, true, true, REV, false>(gld, sts);
    __syncthreads();
    ct_run_range2<P, 1, 1, NST - 1, T, M2, true, REV, true>(p.tw, lds, lds, sts, sts, true, true);
    ct_last_half2<P, T, M2, true, true, REV>(p.tw, lds, stg);
  }
}

// The fused z pass for FP32 on line pairs (ct_stage2): same arithmetic as
// k_zf_ct, each task moving two adjacent kx lines per shared-memory access.
#ifndef GILA_ZF2_CAP
#define GILA_ZF2_CAP 1
#endif
// CTAs per SM the FP32 fused z kernel is compiled for: registers capped at
// 128 per thread, or at 168 where the fused stage is radix 3 (P = 96, 192,
// 384; measured z pass at P = 96, 96x96x48 cells: 0.0675 -> 0.0606 ms,
// unchanged at 192; at P = 256 the higher cap measured 16% slower)
constexpr int zf2_min_blocks(int T, int P) {
  const int regs = ct_radix(P, ct_nst(P) - 1) == 3 ? 168 : 128;
  return 65536 / (T * regs) > 1 ? 65536 / (T * regs) : 1;
}
template <int P, int TX>
__global__ void __launch_bounds__(ct_threads2(TX, P), GILA_ZF2_CAP ? zf2_min_blocks(ct_threads2(TX, P), P) : 1)
    k_zf2_ct(const ZParams<float2> p) {
  using C = float2;
  constexpr int T = ct_threads2(TX, P);
  constexpr int M2 = TX / 2;
  constexpr int CH = P * TX;
  constexpr int NST = ct_nst(P);
  constexpr int RL = ct_radix(P, NST - 1);
  constexpr int TPL = P / RL;
  constexpr int NTASK = M2 * TPL;
  constexpr int K = (NTASK + T - 1) / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nrhs = p.nrhs, ntiles = p.ntiles, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = p.ts0 + rest % p.nts;  // [ts0, ts0 + nts) of the mirror tile order
  const int yseq = rest / p.nts;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int tmax = Px - kx0;  // even: Px and kx0 are even
  const int64_t plane = (int64_t)Py * Px;
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  // stage the tile with 16-byte copies (pairs of columns)
  for (int q = threadIdx.x; q < 3 * nin * M2; q += T) {
    const int row = q / M2, t2 = q % M2;  // row = c * nin + z
    const int c = (int)p.nind.div((uint32_t)row);
    const int i = row - c * nin;
    if (2 * t2 < tmax) cp_async(reinterpret_cast<float4*>(sm + c * CH + i * TX) + t2,
                                reinterpret_cast<const float4*>(Bb + (int64_t)row * plane) + t2);
  }
  cp_async_wait_all();
  __syncthreads();
  const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    float4* const smc = reinterpret_cast<float4*>(sm + c * CH);
    auto ldf = [=](int t2, int i) -> float4 {
      if (2 * t2 < tmax && i < nin) return smc[i * M2 + t2];
      return z4;
    };
    auto lds = [=](int t2, int i) -> float4 { return smc[i * M2 + t2]; };
    auto sts = [=](int t2, int i, float4 v) { smc[i * M2 + t2] = v; };
    ct_run_range2<P, 0, 0, NST - 1, T, M2, false, false, true>(p.tw, ldf, lds, sts, sts, true, true);
  }
  int py, iy, ry;
  ax_map(p.ax[1], ky + p.ky0, py, iy, ry);
  const int tx = p.tx, ty = p.ty, tz = p.tz;
  const float s = (float)p.scale;
  const C* const tw = p.tw;
  const float4* const sm4 = reinterpret_cast<const float4*>(sm);
  float4* const smw = reinterpret_cast<float4*>(sm);
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    if (NTASK % T != 0 && task >= NTASK) continue;
    const int lp = task % M2, j = task / M2;
    if (2 * lp >= tmax) continue;
    C a[3][RL], b[3][RL];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const float4 q = sm4[(c * CH + (j + r * TPL) * TX) / 2 + lp];
        a[c][r] = make_float2(q.x, q.y);
        b[c][r] = make_float2(q.z, q.w);
      }
    {
      C w[RL];
      twiddles<RL, false>(tw, j, w);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int r = 1; r < RL; ++r) {
          a[c][r] = cmul(a[c][r], w[r]);
          b[c][r] = cmul(b[c][r], w[r]);
        }
        Bfly<RL, false, C>::run(a[c], tw, TPL);
        Bfly<RL, false, C>::run(b[c], tw, TPL);
      }
    }
    // the two columns kx0 + 2 lp (even parity) and kx0 + 2 lp + 1 (odd; on
    // an odd-length x axis the last pair's second column lies outside the
    // spectrum and reads the first column's entry, never stored)
    int pxa, ixa, rxa, pxb, ixb, rxb;
    ax_map(p.ax[0], kx0 + 2 * lp, pxa, ixa, rxa);
    if (2 * lp + 1 < tmax) {
      ax_map(p.ax[0], kx0 + 2 * lp + 1, pxb, ixb, rxb);
    } else {
      pxb = pxa;
      ixb = ixa;
      rxb = rxa;
    }
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const int kz = j + r * TPL;
      int pz, iz, rz;
      ax_map(p.ax[2], kz, pz, iz, rz);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int px = h ? pxb : pxa, ix = h ? ixb : ixa, rx = h ? rxb : rxa;
        const C* gp = ker_at(p.ker, 4 * px + 2 * py + pz, iz, iy, ix, tx, ty, tz);
        const C gxx = ker_ld(gp, 0, tx), gyy = ker_ld(gp, 1, tx), gzz = ker_ld(gp, 2, tx);
        const C gxy = cscale(ker_ld(gp, 3, tx), (rx ^ ry) ? -1.f : 1.f);
        const C gxz = cscale(ker_ld(gp, 4, tx), (rx ^ rz) ? -1.f : 1.f);
        const C gyz = cscale(ker_ld(gp, 5, tx), (ry ^ rz) ? -1.f : 1.f);
        C (*v)[RL] = h ? b : a;
        const C x0 = v[0][r], x1 = v[1][r], x2 = v[2][r];
        v[0][r] = cscale(cadd(cadd(cmul(gxx, x0), cmul(gxy, x1)), cmul(gxz, x2)), s);
        v[1][r] = cscale(cadd(cadd(cmul(gxy, x0), cmul(gyy, x1)), cmul(gyz, x2)), s);
        v[2][r] = cscale(cadd(cadd(cmul(gxz, x0), cmul(gyz, x1)), cmul(gzz, x2)), s);
      }
    }
    // inverse first stage, written back to the slots the task read
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Bfly<RL, true, C>::run(a[c], tw, TPL);
      Bfly<RL, true, C>::run(b[c], tw, TPL);
#pragma unroll
      for (int r = 0; r < RL; ++r)
        smw[(c * CH + (j + r * TPL) * TX) / 2 + lp] = make_float4(a[c][r].x, a[c][r].y, b[c][r].x, b[c][r].y);
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    float4* const dc = reinterpret_cast<float4*>(sm + c * CH);
    C* const Bo = Bb + (int64_t)c * nout * plane;
    auto ldp = [=](int t2, int q) -> float4 { return dc[((q / RL) + (q % RL) * TPL) * M2 + t2]; };
    auto ldo = [=](int t2, int i) -> float4 { return dc[i * M2 + t2]; };
    auto sto = [=](int t2, int i, float4 v) { dc[i * M2 + t2] = v; };
    auto stg = [=](int t2, int i, float4 v) {
      if (2 * t2 < tmax && i < nout) reinterpret_cast<float4*>(Bo + (int64_t)i * plane)[t2] = v;
    };
    ct_run_range2<P, 1, 1, NST, T, M2, true, true, true>(p.tw, ldp, ldo, sto, stg, true, false);
  }
}

// ------------------------------------------------------------------------
// FP32 fused z pass on line pairs, in the form of k_zg_ct: forward stage 0
// fed from global memory with the zero padding pruned, middle stages with
// twiddles shared by the three components and both lines of a pair, FMA-chain
// multiply with sign-bit flips, and a last inverse stage that forms only the
// target half.  Every tile width gives identical bits.

__device__ __forceinline__ float2 cflip(float2 a, int f) {
  const int m = (f != 0) << 31;
  return make_float2(__int_as_float(__float_as_int(a.x) ^ m), __int_as_float(__float_as_int(a.y) ^ m));
}

__device__ __forceinline__ float2 mac3(const float2& g0, const float2& a, const float2& g1, const float2& b,
                                      const float2& g2, const float2& c, float s) {
  float re = g0.x * a.x;
  re = fmaf(-g0.y, a.y, re);
  re = fmaf(g1.x, b.x, re);
  re = fmaf(-g1.y, b.y, re);
  re = fmaf(g2.x, c.x, re);
  re = fmaf(-g2.y, c.y, re);
  float im = g0.x * a.y;
  im = fmaf(g0.y, a.x, im);
  im = fmaf(g1.x, b.y, im);
  im = fmaf(g1.y, b.x, im);
  im = fmaf(g2.x, c.y, im);
  im = fmaf(g2.y, c.x, im);
  return make_float2(re * s, im * s);
}

__device__ __forceinline__ void zmul3f(float2& x0, float2& x1, float2& x2, const float2 (&g)[6], int rx, int ry,
                                       int rz, float s) {
  const float2 gxy = cflip(g[3], rx ^ ry), gxz = cflip(g[4], rx ^ rz), gyz = cflip(g[5], ry ^ rz);
  const float2 a = x0, b = x1, c = x2;
  x0 = mac3(g[0], a, gxy, b, gxz, c, s);
  x1 = mac3(gxy, a, g[1], b, gyz, c, s);
  x2 = mac3(gxz, a, gyz, b, g[2], c, s);
}

// middle stage on line pairs (float4 = element q of lines 2 lp, 2 lp + 1)
template <int P, int S, int T, int TX, bool INV, bool REV, class Slot>
__device__ __forceinline__ void zg_mid2(float2* sm, const float2* __restrict__ tw, const Slot& slot) {
  constexpr int R = ct_radix_o<REV>(P, S), NS = ct_span_o<REV>(P, S), TPL = P / R, M2 = TX / 2, NT = M2 * TPL;
  constexpr int K = (NT + T - 1) / T, TWST = P / (NS * R), CH = P * TX;
  float2 w[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = (int)threadIdx.x + k * T;
    const int j = task / M2;
    if (NS > 1) twiddles<R, INV>(tw, (j % NS) * TWST, w[k]);
  }
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    float4* const smc = reinterpret_cast<float4*>(sm + c * CH);
    float2 a[K][R], b[K][R];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = (int)threadIdx.x + k * T;
      if (NT % T == 0 || task < NT) {
        const int lp = task % M2, j = task / M2;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const float4 q = smc[slot(j + r * TPL) * M2 + lp];
          a[k][r] = make_float2(q.x, q.y);
          b[k][r] = make_float2(q.z, q.w);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = (int)threadIdx.x + k * T;
      if (NT % T == 0 || task < NT) {
        const int lp = task % M2, j = task / M2, jm = j % NS;
        if (NS > 1) {
#pragma unroll
          for (int r = 1; r < R; ++r) {
            a[k][r] = cmul(a[k][r], w[k][r]);
            b[k][r] = cmul(b[k][r], w[k][r]);
          }
        }
        Bfly<R, INV, float2>::run(a[k], tw, TPL);
        Bfly<R, INV, float2>::run(b[k], tw, TPL);
        const int base = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r)
          smc[(base + r * NS) * M2 + lp] = make_float4(a[k][r].x, a[k][r].y, b[k][r].x, b[k][r].y);
      }
    }
  }
}

template <int P, int TX>
__global__ void __launch_bounds__(ct_threads2(TX, P), zf2_min_blocks(ct_threads2(TX, P), P))
    k_zg2_ct(const ZParams<float2> p) {
  using C = float2;
  constexpr int T = ct_threads2(TX, P);
  constexpr int M2 = TX / 2;
  constexpr int CH = P * TX;
  constexpr int NST = ct_nst(P);
  constexpr int RL = ct_radix(P, NST - 1);
  constexpr int TPL = P / RL;
  constexpr int TPL0 = P / 8, NT0 = M2 * TPL0, K0 = (NT0 + T - 1) / T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nrhs = p.nrhs, ntiles = p.ntiles, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = p.ts0 + rest % p.nts;  // [ts0, ts0 + nts) of the mirror tile order
  const int yseq = rest / p.nts;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int tmax = Px - kx0;  // even: Px and kx0 are even
  const int64_t plane = (int64_t)Py * Px;
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  const C* const tw = p.tw;
  // forward stage 0 (radix 8, span 1): pair task (lp, j0) reads z = j0 + r
  // * TPL0, r < 4, as 16-byte loads of both lines
  {
    float2 a[3][K0][8], b[3][K0][8];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < K0; ++k) {
        const int task = (int)threadIdx.x + k * T;
        const int lp = task % M2, j0 = task / M2;
        const bool ok = (NT0 % T == 0 || task < NT0) && 2 * lp < tmax;
        const float4* const src = reinterpret_cast<const float4*>(Bb + (int64_t)c * nin * plane) + lp;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = j0 + r * TPL0;
          const float4 q = (ok && i < nin) ? __ldcs(reinterpret_cast<const float4*>(
                                                 reinterpret_cast<const C*>(src) + (int64_t)i * plane))
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
          a[c][k][r] = make_float2(q.x, q.y);
          b[c][k][r] = make_float2(q.z, q.w);
        }
      }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < K0; ++k) {
        const int task = (int)threadIdx.x + k * T;
        if (NT0 % T == 0 || task < NT0) {
          const int lp = task % M2, j0 = task / M2;
          bfly8_half_in<false>(a[c][k]);
          bfly8_half_in<false>(b[c][k]);
          float4* const dst = reinterpret_cast<float4*>(sm + c * CH) + (j0 * 8) * M2 + lp;
#pragma unroll
          for (int r = 0; r < 8; ++r) dst[r * M2] = make_float4(a[c][k][r].x, a[c][k][r].y, b[c][k][r].x, b[c][k][r].y);
        }
      }
  }
  __syncthreads();
  {
    auto nat = [](int q) { return q; };
    if constexpr (NST >= 3) zg_mid2<P, 1, T, TX, false, false>(sm, tw, nat);
    if constexpr (NST >= 4) zg_mid2<P, 2, T, TX, false, false>(sm, tw, nat);
    if constexpr (NST >= 5) zg_mid2<P, 3, T, TX, false, false>(sm, tw, nat);
  }
  int py, iy, ry;
  ax_map(p.ax[1], ky + p.ky0, py, iy, ry);
  const int tx = p.tx, ty = p.ty, tz = p.tz;
  const float s = (float)p.scale;
  const float4* const sm4 = reinterpret_cast<const float4*>(sm);
  float4* const smw = reinterpret_cast<float4*>(sm);
  {
    constexpr int NTASK = M2 * TPL;
    constexpr int K = (NTASK + T - 1) / T;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = (int)threadIdx.x + k * T;
      const bool live = (NTASK % T == 0 || task < NTASK) && 2 * (task % M2) < tmax;
      const int lp = task % M2, j = task / M2;
      // the two columns kx0 + 2 lp (even parity) and kx0 + 2 lp + 1 (odd)
      int pxa = 0, ixa = 0, rxa = 0, pxb = 0, ixb = 0, rxb = 0;
      ax_map(p.ax[0], kx0 + 2 * lp, pxa, ixa, rxa);
      // an odd-length x axis leaves the last pair's second column outside
      // the spectrum: it reads the first column's entry (never stored)
      if (2 * lp + 1 < tmax) {
        ax_map(p.ax[0], kx0 + 2 * lp + 1, pxb, ixb, rxb);
      } else {
        pxb = pxa;
        ixb = ixa;
        rxb = rxa;
      }
      // the first frequency's kernel values (both columns) go out before the barrier
      C ga[6], gb[6];
      int rz = 0;
      // both columns' kernel values for z frequency f: the even and odd x
      // parity of one unmirrored stored index are adjacent (one 16-byte load
      // per component), mirrored ones are not
      const bool adj = ixa == ixb && pxa == 0 && pxb == 1;
      auto kload2 = [&](int f, int& rzf) {
        int pz, iz;
        ax_map(p.ax[2], f, pz, iz, rzf);
        const C* gpa = ker_at(p.ker, 4 * pxa + 2 * py + pz, iz, iy, ixa, tx, ty, tz);
        if (adj) {
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(gpa + 2 * q * tx));
            ga[q] = make_float2(v.x, v.y);
            gb[q] = make_float2(v.z, v.w);
          }
        } else {
          const C* gpb = ker_at(p.ker, 4 * pxb + 2 * py + pz, iz, iy, ixb, tx, ty, tz);
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            ga[q] = ker_ld(gpa, q, tx);
            gb[q] = ker_ld(gpb, q, tx);
          }
        }
      };
      if (live) kload2(j, rz);
      if (k == 0) __syncthreads();
      if (!live) continue;
      C a[3][RL], b[3][RL];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < RL; ++r) {
          const float4 q = sm4[(c * CH + (j + r * TPL) * TX) / 2 + lp];
          a[c][r] = make_float2(q.x, q.y);
          b[c][r] = make_float2(q.z, q.w);
        }
      {
        C w[RL];
        twiddles<RL, false>(tw, j, w);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
          for (int r = 1; r < RL; ++r) {
            a[c][r] = cmul(a[c][r], w[r]);
            b[c][r] = cmul(b[c][r], w[r]);
          }
          Bfly<RL, false, C>::run(a[c], tw, TPL);
          Bfly<RL, false, C>::run(b[c], tw, TPL);
        }
      }
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        if (r > 0) kload2(j + r * TPL, rz);
        zmul3f(a[0][r], a[1][r], a[2][r], ga, rxa, ry, rz, s);
        zmul3f(b[0][r], b[1][r], b[2][r], gb, rxb, ry, rz, s);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        Bfly<RL, true, C>::run(a[c], tw, TPL);
        Bfly<RL, true, C>::run(b[c], tw, TPL);
#pragma unroll
        for (int r = 0; r < RL; ++r)
          smw[(c * CH + (j + r * TPL) * TX) / 2 + lp] = make_float4(a[c][r].x, a[c][r].y, b[c][r].x, b[c][r].y);
      }
    }
  }
  __syncthreads();
  {
    auto perm = [](int q) { return (q / RL) + (q % RL) * TPL; };
    auto nat = [](int q) { return q; };
    if constexpr (NST >= 3) zg_mid2<P, 1, T, TX, true, true>(sm, tw, perm);
    if constexpr (NST >= 4) zg_mid2<P, 2, T, TX, true, true>(sm, tw, nat);
    if constexpr (NST >= 5) zg_mid2<P, 3, T, TX, true, true>(sm, tw, nat);
  }
  __syncthreads();
  // inverse last stage (radix 8, span TPL0): the target half, straight to B
  {
    float2 w[K0][8];
#pragma unroll
    for (int k = 0; k < K0; ++k) {
      const int task = (int)threadIdx.x + k * T;
      twiddles<8, true>(tw, task / M2, w[k]);
    }
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      const float4* const smc = reinterpret_cast<const float4*>(sm + c * CH);
      C* const Bo = Bb + (int64_t)c * nout * plane;
#pragma unroll
      for (int k = 0; k < K0; ++k) {
        const int task = (int)threadIdx.x + k * T;
        if (NT0 % T == 0 || task < NT0) {
          const int lp = task % M2, j = task / M2;
          float2 a[8], b[8];
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            const float4 q = smc[(j + r * TPL0) * M2 + lp];
            a[r] = make_float2(q.x, q.y);
            b[r] = make_float2(q.z, q.w);
          }
#pragma unroll
          for (int r = 1; r < 8; ++r) {
            a[r] = cmul(a[r], w[k][r]);
            b[r] = cmul(b[r], w[k][r]);
          }
          bfly8_half_out<true>(a);
          bfly8_half_out<true>(b);
          if (2 * lp < tmax) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              const int i = j + r * TPL0;
              if (i < nout)
                __stcs(reinterpret_cast<float4*>(Bo + (int64_t)i * plane) + lp, make_float4(a[r].x, a[r].y, b[r].x, b[r].y));
            }
          }
        }
      }
    }
  }
}

template <typename C, int P, bool AXPBY, bool REV>
__global__ void __launch_bounds__(ct_threads(ct_xlines<sizeof(C)>(P), P)) k_xinv_ct(const XiParams<C> p) {
  constexpr int M = ct_xlines<sizeof(C)>(P);
  constexpr int T = ct_threads(M, P);
  constexpr int LS = P + (P + 7) / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const int nout = p.nout;
  const int64_t rows = p.rows;
  C* const out = p.out;
  const C alpha = p.alpha, beta = p.beta;
  const int ls = p.ls;
  const C* const ls_in = p.ls_in;
  const C* const ls_chi = p.ls_chi;
  const int64_t ls_chi_rs = p.ls_chi_rs;
  const FDiv rows_rhs = p.rows_rhs, rows_zy = p.rows_zy;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const bool scatter = p.part_scatter != 0;
  const int ty = p.ty, tz = p.tz, parT = p.parT;
  const int d0 = p.tdiv[0], d1 = p.tdiv[1], d2 = p.tdiv[2];
  const int64_t f0 = p.full[0], f1 = p.full[1], f2 = p.full[2];
  const int(*toff)[3] = p.toff;
  const int64_t g_off = p.g_off;
  {
    const int nl = (int)((rows - g0) < M ? (rows - g0) : M);
    const C* const src = p.A + g0 * P;
    for (int q = threadIdx.x; q < nl * P; q += T) {
      const int l = q / P, i = q % P;
      cp_async(sm + l * LS + i + (i >> 3), src + q);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  auto lds = [=](int l, int i) -> C { return sm[l * LS + i + (i >> 3)]; };
  auto sts = [=](int l, int i, C v) { sm[l * LS + i + (i >> 3)] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g >= rows || i >= nout) return;
    int64_t o;
    const int64_t gg = g + g_off;
    if (!scatter) {
      o = gg * nout + i;
    } else {
      int64_t q = gg;
      const int y = (int)(q % ty); q /= ty;
      const int z = (int)(q % tz); q /= tz;
      const int c = (int)(q % 3); q /= 3;
      const int t = (int)(q % parT);
      const int64_t rhs = q / parT;
      const int64_t X = (int64_t)i * d0 + toff[t][0];
      const int64_t Y = (int64_t)y * d1 + toff[t][1];
      const int64_t Z = (int64_t)z * d2 + toff[t][2];
      o = (((rhs * 3 + c) * f2 + Z) * f1 + Y) * f0 + X;
    }
    if (AXPBY)
      out[o] = cadd(cmul(alpha, v), cmul(beta, out[o]));
    else if (ls)
      out[o] = ls_value(ls_in, ls_chi, ls_chi_rs, rows_rhs, rows_zy, nout, gg, i, o, v);
    else
      out[o] = v;
  };
  ct_run_range<C, P, 0, 0, ct_nst(P), 8, T, M, true, false, REV>(p.tw, lds, lds, sts, stg, true, false);
}

// Lengths with specialised kernels.
#define GILA_CT_SIZES(X) X(64) X(96) X(128) X(192) X(256) X(384) X(512)
static bool ct_has(int P) {
#define GILA_CT_CASE(n) if (P == n) return true;
  GILA_CT_SIZES(GILA_CT_CASE)
#undef GILA_CT_CASE
  return false;
}

// ---------------------------------------------------------------- launchers
// fused z pass (GILA_ZFUSE=0 selects the unfused one); FP32 on line pairs
// (GILA_ZPAIR=0 selects one line per task)
static inline bool zfuse() {
  static const bool on = [] {
    const char* e = getenv("GILA_ZFUSE");
    return !(e && e[0] == '0');
  }();
  return on;
}
// FP64 fused z pass with register-fed first stage and pruned half
// butterflies (k_zg_ct) where it applies (GILA_ZG=0: k_zf_ct)
static inline bool zgo() {
  static const bool on = [] {
    const char* e = getenv("GILA_ZG");
    return !(e && e[0] == '0');
  }();
  return on;
}
// FP64 x / y passes with a global-fed first stage and a half last stage
// (k_xfwd_g, k_y_g, k_xinv_g) where they apply (GILA_XYG=0: the staged ones)
static inline bool xyg() {
  static const bool on = [] {
    const char* e = getenv("GILA_XYG");
    return !(e && e[0] == '0');
  }();
  return on;
}
// two-stage FP64 z pass (k_zr_ct) where it applies (GILA_ZTWO=0: k_zf_ct)
static inline bool ztwo() {
  static const bool on = [] {
    const char* e = getenv("GILA_ZTWO");
    return !(e && e[0] == '0');
  }();
  return on;
}
// mirror-pair tasks in the fused z pass where the launch shape asks for
// them (GILA_ZMIRROR=0: never, 2: always); read at every launch, results
// are identical either way
static inline int zmirror(int want) {
  const char* e = getenv("GILA_ZMIRROR");
  if (e && e[0] == '0') return 0;
  if (e && e[0] == '2') return 1;
  return want != 0;
}
static inline bool zpair() {
  static const bool on = [] {
    const char* e = getenv("GILA_ZPAIR");
    return !(e && e[0] == '0');
  }();
  return on;
}
template <typename C>
static inline const ZParams<float2>& zp32(const ZParams<C>& p) {
  return reinterpret_cast<const ZParams<float2>&>(p);
}
template <typename C>
static inline const YParams<float2>& yp32(const YParams<C>& p) {
  return reinterpret_cast<const YParams<float2>&>(p);
}
template <typename C>
static inline const XfParams<float2>& xfp32(const XfParams<C>& p) {
  return reinterpret_cast<const XfParams<float2>&>(p);
}
template <typename C>
static inline const XiParams<float2>& xip32(const XiParams<C>& p) {
  return reinterpret_cast<const XiParams<float2>&>(p);
}

static cudaError_t set_smem(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return cudaSuccess;
}

static bool is_mixed(const AxisPlan& pl) {
  for (int s = 0; s < pl.nst; ++s)
    if (pl.radix[s] != 2 && pl.radix[s] != 4 && pl.radix[s] != 8) return true;
  return false;
}

#define GILA_LAUNCH(MXV, KERNEL, ...)                                                        \
  do {                                                                                       \
    const void* fn__ = (const void*)KERNEL;                                                  \
    cudaError_t e__ = set_smem(fn__, sm);                                                    \
    if (e__ != cudaSuccess) return e__;                                                      \
    KERNEL<<<(unsigned)blocks, T, sm, st>>>(__VA_ARGS__);                                    \
  } while (0)

// launch of an FP32 line-pair kernel with T threads (returns from the caller)
#define GILA_LAUNCH2_SB(KERNEL, TT, SMB, NB, ARG)                  \
  do {                                                          \
    cudaError_t e__ = set_smem((const void*)KERNEL, SMB);       \
    if (e__ != cudaSuccess) return e__;                         \
    KERNEL<<<(unsigned)(NB), TT, SMB, st>>>(ARG);                \
    return cudaGetLastError();                                  \
  } while (0)
#define GILA_LAUNCH2(KERNEL, TT, ARG) GILA_LAUNCH2_SB(KERNEL, TT, sm, blocks, ARG)

// one launch of a compile-time x / y kernel in the chosen radix order
template <int P, bool REV>
static cudaError_t run_xfwd2(const XfParams<float2>& p, int T, size_t sm, int64_t blocks, cudaStream_t st) {
  cudaError_t e = set_smem((const void*)k_xfwd2_ct<P, REV>, sm);
  if (e != cudaSuccess) return e;
  k_xfwd2_ct<P, REV><<<(unsigned)blocks, T, sm, st>>>(p);
  return cudaGetLastError();
}
template <int P, bool REV>
static cudaError_t run_xinv2(const XiParams<float2>& p, int T, size_t sm, int64_t blocks, cudaStream_t st) {
  cudaError_t e = set_smem((const void*)k_xinv2_ct<P, REV>, sm);
  if (e != cudaSuccess) return e;
  k_xinv2_ct<P, REV><<<(unsigned)blocks, T, sm, st>>>(p);
  return cudaGetLastError();
}
template <int P, bool INV, int TX, bool REV>
static cudaError_t run_y2(const YParams<float2>& p, int T, size_t sm, int64_t blocks, cudaStream_t st) {
  cudaError_t e = set_smem((const void*)k_y2_ct<P, INV, TX, REV>, sm);
  if (e != cudaSuccess) return e;
  k_y2_ct<P, INV, TX, REV><<<(unsigned)blocks, T, sm, st>>>(p);
  return cudaGetLastError();
}

template <typename C>
cudaError_t launch_xfwd(const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* A, int64_t rows,
                        cudaStream_t st) {
  XfParams<C> p;
  p.in = in;
  p.A = A;
  p.pl = d.plan_d[0];
  p.P = d.plan[0].P;
  p.tw = d.tw[0];
  p.nin = g.sc[0];
  p.M = L.xf_lines;
  p.rows = rows;
  p.nind = make_fdiv((uint32_t)p.nin);
  if (ct_has(p.P)) {
#define GILA_CT_XF(n)                                                                  \
  if constexpr (sizeof(C) == 8) {                                                      \
    if (p.P == n && zpair()) {                                                         \
      constexpr int M = ct_xlines2<8>(n);                                              \
      const int T2 = ct_threads2(M, n);                                                \
      const size_t sm = (size_t)M * row_stride(n) * sizeof(C);                         \
      p.M = M;                                                                         \
      const int64_t blocks = (p.rows + M - 1) / M;                                     \
      if (xyg() && L.xy_g && 2 * p.nin <= n) {                                                   \
        if (L.x_rev) {                                                                 \
          if constexpr (xyg_in_ok<n, true>()) {                                        \
            GILA_LAUNCH2((k_xfwd2_g<n, true>), T2, xfp32(p));                            \
          }                                                                            \
        } else {                                                                       \
          if constexpr (xyg_in_ok<n, false>()) {                                       \
            GILA_LAUNCH2((k_xfwd2_g<n, false>), T2, xfp32(p));                           \
          }                                                                            \
        }                                                                              \
      }                                                                                \
      return L.x_rev ? run_xfwd2<n, true>(xfp32(p), T2, sm, blocks, st)               \
                     : run_xfwd2<n, false>(xfp32(p), T2, sm, blocks, st);             \
    }                                                                                  \
  }                                                                                    \
  if (p.P == n) {                                                                      \
    constexpr int M = ct_xlines<sizeof(C)>(n);                                         \
    const int T = ct_threads(M, n);                                                    \
    const size_t sm = (size_t)M * row_stride(n) * sizeof(C);                           \
    p.M = M;                                                                           \
    const int64_t blocks = (p.rows + M - 1) / M;                                       \
    if constexpr (sizeof(C) == 16) {                                                   \
      if (xyg() && L.xy_g && 2 * p.nin <= n) {                                                   \
        if (L.x_rev) {                                                                 \
          if constexpr (xyg_in_ok<n, true>()) {                                        \
            GILA_LAUNCH(false, (k_xfwd_g<n, true>), p);                                \
            return cudaGetLastError();                                                 \
          }                                                                            \
        } else {                                                                       \
          if constexpr (xyg_in_ok<n, false>()) {                                       \
            GILA_LAUNCH(false, (k_xfwd_g<n, false>), p);                               \
            return cudaGetLastError();                                                 \
          }                                                                            \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
    if (L.x_rev)                                                                       \
      GILA_LAUNCH(false, (k_xfwd_ct<C, n, true>), p);                                  \
    else                                                                               \
      GILA_LAUNCH(false, (k_xfwd_ct<C, n, false>), p);                                 \
    return cudaGetLastError();                                                         \
  }
    GILA_CT_SIZES(GILA_CT_XF)
#undef GILA_CT_XF
  }
  const int T = pass_threads(d.plan[0], p.M);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)p.M * row_stride(p.P) * sizeof(C);
  const int64_t blocks = (p.rows + p.M - 1) / p.M;
  if (is_mixed(d.plan[0]))
    GILA_LAUNCH(true, (k_xfwd<C, true>), p);
  else
    GILA_LAUNCH(false, (k_xfwd<C, false>), p);
  return cudaGetLastError();
}

template <typename C, bool INV>
static cudaError_t launch_y_one(const YParams<C>& p, bool mx, int T, size_t sm, int64_t blocks, bool rev, bool gform,
                                cudaStream_t st) {
  if (ct_has(p.P)) {
#define GILA_CT_Y2(n, tx)                                  \
  if constexpr (ct_y_ok(sizeof(C), n, tx)) {               \
    if (p.P == n && p.TX == tx) {                          \
      if constexpr (sizeof(C) == 8) {                      \
        if (zpair()) {                                     \
          const int T2 = ct_threads2(tx, n);               \
          if (xyg() && gform && (INV ? 2 * p.nout <= n : 2 * p.nin <= n)) { \
            if (rev) {                                     \
              if constexpr (INV ? xyg_out_ok<n, true>() : xyg_in_ok<n, true>()) { \
                GILA_LAUNCH2((k_y2_g<n, INV, tx, true>), T2, yp32(p)); \
              }                                            \
            } else {                                       \
              if constexpr (INV ? xyg_out_ok<n, false>() : xyg_in_ok<n, false>()) { \
                GILA_LAUNCH2((k_y2_g<n, INV, tx, false>), T2, yp32(p)); \
              }                                            \
            }                                              \
          }                                                \
          return rev ? run_y2<n, INV, tx, true>(yp32(p), T2, sm, blocks, st) \
                     : run_y2<n, INV, tx, false>(yp32(p), T2, sm, blocks, st); \
        }                                                  \
      }                                                    \
      if constexpr (sizeof(C) == 16) {                                                 \
        if (xyg() && gform && (INV ? 2 * p.nout <= n : 2 * p.nin <= n)) {                       \
          if (rev) {                                                                   \
            if constexpr (INV ? xyg_out_ok<n, true>() : xyg_in_ok<n, true>()) {        \
              GILA_LAUNCH(false, (k_y_g<n, INV, tx, true>), p);                        \
              return cudaSuccess;                                                      \
            }                                                                          \
          } else {                                                                     \
            if constexpr (INV ? xyg_out_ok<n, false>() : xyg_in_ok<n, false>()) {      \
              GILA_LAUNCH(false, (k_y_g<n, INV, tx, false>), p);                       \
              return cudaSuccess;                                                      \
            }                                                                          \
          }                                                                            \
        }                                                                              \
      }                                                                                \
      if (rev)                                             \
        GILA_LAUNCH(false, (k_y_ct<C, n, INV, tx, true>), p); \
      else                                                 \
        GILA_LAUNCH(false, (k_y_ct<C, n, INV, tx, false>), p); \
      return cudaSuccess;                                  \
    }                                                      \
  }
#define GILA_CT_Y(n) GILA_CT_Y2(n, 4) GILA_CT_Y2(n, 8) GILA_CT_Y2(n, 16)
    GILA_CT_SIZES(GILA_CT_Y)
#undef GILA_CT_Y
#undef GILA_CT_Y2
    return cudaErrorInvalidConfiguration;
  }
  if (mx)
    GILA_LAUNCH(true, (k_y<C, INV, true>), p);
  else
    GILA_LAUNCH(false, (k_y<C, INV, false>), p);
  return cudaSuccess;
}

// One y pass over planes [q0, q0 + nq) (plane = ch*nz + z) of one rhs.
// Forward: src = x-pass slab holding planes from src_sub on, dst = B of the
// rhs.  Inverse: src = B of the rhs, dst = slab holding planes from dst_sub.
// y tile ranges of a kx chunk: positions [ts0, ts0 + nts) of the z pass's
// mirror tile order are z tiles p0 .. p1 - 1 and ntz - p1 .. ntz - p0 - 1
// (p = ts0 / 2 ...), i.e. the kx ranges [p0 txz, p1 txz) and [Px - p1 txz,
// Px - p0 txz); false when they do not fall on y tile boundaries
static bool chunk_y_tiles(int Px, int txz, int txy, const KxChunk& ch, int& lo0, int& nlo, int& hi0, int& nt) {
  if (txz <= 0 || txy <= 0 || Px % txz || Px % txy || (Px / txz) % 2 || ch.ts0 % 2 || ch.nts % 2) return false;
  const int p0 = ch.ts0 / 2, p1 = (ch.ts0 + ch.nts) / 2;
  const int k0 = p0 * txz, k1 = p1 * txz;
  if (k0 % txy || k1 % txy || 2 * k1 > Px) return false;
  lo0 = k0 / txy;
  nlo = (k1 - k0) / txy;
  hi0 = (Px - k1) / txy;
  nt = 2 * nlo;
  return true;
}

template <typename C>
cudaError_t launch_y(const Geom& g, const DevOp<C>& d, const Launch& L, bool inv, const C* src, C* dst, int64_t q0,
                     int64_t nq, int64_t src_sub, int64_t dst_sub, cudaStream_t st, const KxChunk* ch) {
  YParams<C> p;
  p.src = src;
  p.dst = dst;
  p.pl = d.plan_d[1];
  p.P = d.plan[1].P;
  p.tw = d.tw[1];
  p.Px = g.P[0];
  p.TX = L.y_tx;
  if (!inv) {
    p.nin = g.sc[1];
    p.nout = g.P[1];
    p.nz = g.sc[2];
    p.src_z = g.sc[2];
    p.src_rows = g.sc[1];
    p.dst_z = g.sc[2];  // B planes: c*sz + z
    p.dst_rows = g.P[1];
  } else {
    p.nin = g.P[1];
    p.nout = g.tc[1];
    p.nz = g.tc[2];
    p.src_z = g.tc[2];  // B planes: ch*tz + z
    p.src_rows = g.P[1];
    p.dst_z = g.tc[2];
    p.dst_rows = g.tc[1];
  }
  p.q0 = q0;
  p.src_sub = src_sub;
  p.dst_sub = dst_sub;
  if (ct_has(p.P)) p.TX = ct_tile_pick(sizeof(C), p.P, L.y_tx, false);
  p.ntiles = (p.Px + p.TX - 1) / p.TX;
  p.md = make_fdiv((uint32_t)p.TX);
  p.nt = p.nlo = p.ntiles;
  p.lo0 = p.hi0 = 0;
  if (ch && ch->nts >= 0) {
    const int txz = ct_has(g.P[2]) ? ct_tile_pick(sizeof(C), g.P[2], L.z_tx, true) : L.z_tx;
    if (!chunk_y_tiles(p.Px, txz, p.TX, *ch, p.lo0, p.nlo, p.hi0, p.nt)) return cudaErrorInvalidValue;
  }
  const int T = ct_has(p.P) ? ct_threads(p.TX, p.P) : pass_threads(d.plan[1], p.TX);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)p.TX * p.P * sizeof(C);
  const bool mx = is_mixed(d.plan[1]);
  const int64_t blocks = (int64_t)p.nt * nq;
  cudaError_t e = inv ? launch_y_one<C, true>(p, mx, T, sm, blocks, L.y_rev != 0, L.xy_g != 0, st)
                      : launch_y_one<C, false>(p, mx, T, sm, blocks, L.y_rev != 0, L.xy_g != 0, st);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

template <typename C>
cudaError_t launch_z(const Geom& g, const DevOp<C>& d, const Launch& L, C* B, int nrhs, cudaStream_t st,
                     const KxChunk* ch, int ky0, int nky) {
  const Work w = work_sizes(g);
  ZParams<C> p;
  p.B = B;
  p.ker = d.ker;
  p.mapx = d.map[0];
  p.mapy = d.map[1];
  p.mapz = d.map[2];
  p.pl = d.plan_d[2];
  p.P = d.plan[2].P;
  p.tw = d.tw[2];
  p.Px = g.P[0];
  p.Py = g.P[1];
  p.ky0 = 0;
  if (nky >= 0) {
    if (ky0 < 0 || nky < 1 || ky0 + nky > g.P[1] || (ch && ch->nts >= 0)) return cudaErrorInvalidValue;
    p.Py = nky;
    p.ky0 = ky0;
  }
  p.TX = L.z_tx;
  p.nin = g.sc[2];
  p.nout = g.tc[2];
  p.zb = w.zb;
  p.tx = g.tru[0];
  p.ty = g.tru[1];
  p.tz = g.tru[2];
  p.parT = g.parT;
  p.nrhs = nrhs;
  p.zmir = zmirror(L.z_mir);
  p.scale = d.scale;
  for (int k = 0; k < 3; ++k) {
    p.ax[k].brn = g.P[k] / 2;
    p.ax[k].full = g.tru[k] == g.P[k] / 2;
    p.ax[k].fe = (g.tc[k] + 1) / 2 + (g.tc[k] % 2 == 0 ? 1 : 0);
    p.ax[k].fo = (g.tc[k] + 1) / 2;
  }
  if (ct_has(p.P)) p.TX = ct_tile_pick(sizeof(C), p.P, L.z_tx, true);
  p.ntiles = (p.Px + p.TX - 1) / p.TX;
  p.md = make_fdiv((uint32_t)p.TX);
  p.nind = make_fdiv((uint32_t)p.nin);
  p.ts0 = 0;
  p.nts = p.ntiles;
  if (ch && ch->nts >= 0) {
    if (ch->ts0 < 0 || ch->ts0 + ch->nts > p.ntiles) return cudaErrorInvalidValue;
    p.ts0 = ch->ts0;
    p.nts = ch->nts;
  }
  const int T = ct_has(p.P) ? ct_threads(p.TX, p.P) : pass_threads(d.plan[2], p.TX);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)3 * p.TX * p.P * sizeof(C) * (g.parT > 1 ? 2 : 1);
  const int64_t blocks = (int64_t)p.nts * p.Py * nrhs;
  if (ct_has(p.P)) {
#define GILA_CT_Z2(n, tx)                             \
  if constexpr (ct_z_ok(sizeof(C), n, tx)) {          \
    if (p.P == n && p.TX == tx) {                     \
      if constexpr (zr_ok(sizeof(C), n, tx)) {        \
        if (p.parT == 1 && zfuse() && ztwo()) {       \
          const void* fnr = (const void*)k_zr_ct<C, n, tx>; \
          cudaError_t er = set_smem(fnr, sm);         \
          if (er != cudaSuccess) return er;           \
          k_zr_ct<C, n, tx><<<(unsigned)blocks, zr_threads(tx, n), sm, st>>>(p); \
          return cudaGetLastError();                  \
        }                                             \
      }                                               \
      if constexpr (sizeof(C) == 16 && zg_ok<n>()) {  \
        if (p.parT == 1 && zfuse() && zgo() && 2 * p.nin <= n && 2 * p.nout <= n) { \
          GILA_LAUNCH(false, (k_zg_ct<n, tx>), p);    \
          return cudaGetLastError();                  \
        }                                             \
      }                                               \
      if constexpr (zf_ok(sizeof(C), n)) {            \
        if (p.parT == 1 && zfuse()) {                 \
          if constexpr (sizeof(C) == 8 && zg_ok<n>()) { \
            if (zpair() && zgo() && 2 * p.nin <= n && 2 * p.nout <= n) { \
              const int T2 = ct_threads2(tx, n);      \
              const void* fn2 = (const void*)k_zg2_ct<n, tx>; \
              cudaError_t e2 = set_smem(fn2, sm);     \
              if (e2 != cudaSuccess) return e2;       \
              k_zg2_ct<n, tx><<<(unsigned)blocks, T2, sm, st>>>(zp32(p)); \
              return cudaGetLastError();              \
            }                                         \
          }                                           \
          if constexpr (sizeof(C) == 8) {             \
            if (zpair()) {                            \
              const int T2 = ct_threads2(tx, n);      \
              const void* fn2 = (const void*)k_zf2_ct<n, tx>; \
              cudaError_t e2 = set_smem(fn2, sm);     \
              if (e2 != cudaSuccess) return e2;       \
              k_zf2_ct<n, tx><<<(unsigned)blocks, T2, sm, st>>>(zp32(p)); \
              return cudaGetLastError();              \
            }                                         \
          }                                           \
          GILA_LAUNCH(false, (k_zf_ct<C, n, tx>), p); \
          return cudaGetLastError();                  \
        }                                             \
      }                                               \
      GILA_LAUNCH(false, (k_z_ct<C, n, tx>), p);      \
      return cudaGetLastError();                      \
    }                                                 \
  }
#define GILA_CT_Z(n) GILA_CT_Z2(n, 4) GILA_CT_Z2(n, 8) GILA_CT_Z2(n, 16)
    GILA_CT_SIZES(GILA_CT_Z)
#undef GILA_CT_Z
#undef GILA_CT_Z2
    return cudaErrorInvalidConfiguration;
  }
  if (is_mixed(d.plan[2]))
    GILA_LAUNCH(true, (k_z<C, true>), p);
  else
    GILA_LAUNCH(false, (k_z<C, false>), p);
  return cudaGetLastError();
}

template <typename C, bool AXPBY>
static cudaError_t launch_xinv_one(const XiParams<C>& p, bool mx, int T, size_t sm, int64_t blocks, bool rev,
                                   bool gform, cudaStream_t st) {
  if (ct_has(p.P)) {
#define GILA_CT_XI(n)                                                    \
  if constexpr (sizeof(C) == 8 && !AXPBY) {                              \
    if (p.P == n && !p.part_scatter && zpair()) {                        \
      constexpr int M2r = ct_xlines2<8>(n);                              \
      const int T2 = ct_threads2(M2r, n);                                \
      const size_t sm2 = (size_t)M2r * row_stride(n) * sizeof(C);        \
      const int64_t blocks2 = (p.rows + M2r - 1) / M2r;                  \
      if (xyg() && gform && 2 * p.nout <= n) {                                  \
        if (rev) {                                                     \
          if constexpr (xyg_out_ok<n, true>()) {                       \
            GILA_LAUNCH2_SB((k_xinv2_g<n, true>), T2, sm2, blocks2, xip32(p)); \
          }                                                            \
        } else {                                                       \
          if constexpr (xyg_out_ok<n, false>()) {                      \
            GILA_LAUNCH2_SB((k_xinv2_g<n, false>), T2, sm2, blocks2, xip32(p)); \
          }                                                            \
        }                                                              \
      }                                                                \
      return rev ? run_xinv2<n, true>(xip32(p), T2, sm2, blocks2, st)    \
                 : run_xinv2<n, false>(xip32(p), T2, sm2, blocks2, st);  \
    }                                                                    \
  }                                                                      \
  if (p.P == n) {                                                        \
    if constexpr (sizeof(C) == 16) {                                                   \
      if (xyg() && gform && 2 * p.nout <= n) {                                                  \
        if (rev) {                                                                     \
          if constexpr (xyg_out_ok<n, true>()) {                                       \
            GILA_LAUNCH(false, (k_xinv_g<n, AXPBY, true>), p);                         \
            return cudaSuccess;                                                        \
          }                                                                            \
        } else {                                                                       \
          if constexpr (xyg_out_ok<n, false>()) {                                      \
            GILA_LAUNCH(false, (k_xinv_g<n, AXPBY, false>), p);                        \
            return cudaSuccess;                                                        \
          }                                                                            \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
    if (rev)                                                             \
      GILA_LAUNCH(false, (k_xinv_ct<C, n, AXPBY, true>), p);             \
    else                                                                 \
      GILA_LAUNCH(false, (k_xinv_ct<C, n, AXPBY, false>), p);            \
    return cudaSuccess;                                                  \
  }
    GILA_CT_SIZES(GILA_CT_XI)
#undef GILA_CT_XI
  }
  if (mx)
    GILA_LAUNCH(true, (k_xinv<C, AXPBY, true>), p);
  else
    GILA_LAUNCH(false, (k_xinv<C, AXPBY, false>), p);
  return cudaSuccess;
}

// x inverse over `rows` spectral rows of the slab A; g_off is the global row
// index (over all rhs) of the slab's first row, `out` the full output.
template <typename C>
cudaError_t launch_xinv(const Geom& g, const DevOp<C>& d, const Launch& L, const C* A, C* out, int64_t rows,
                        int64_t g_off, bool axpby, C alpha, C beta, cudaStream_t st, const LsEpi<C>* ls) {
  XiParams<C> p;
  p.ls = ls != nullptr;
  p.ls_in = ls ? ls->in : nullptr;
  p.ls_chi = ls ? ls->chi : nullptr;
  p.ls_chi_rs = ls ? ls->chi_rs : 0;
  p.rows_rhs = make_fdiv((uint32_t)(3 * g.tc[2] * g.tc[1]));
  p.rows_zy = make_fdiv((uint32_t)(g.tc[2] * g.tc[1]));
  if (ls && (g.parT != 1 || axpby)) return cudaErrorInvalidValue;
  p.A = A;
  p.out = out;
  p.pl = d.plan_d[0];
  p.P = d.plan[0].P;
  p.tw = d.tw[0];
  p.nout = g.tc[0];
  p.M = L.xi_lines;
  p.ty = g.tc[1];
  p.tz = g.tc[2];
  p.parT = g.parT;
  p.rows = rows;
  p.g_off = g_off;
  p.part_scatter = g.parT > 1;
  for (int k = 0; k < 3; ++k) {
    p.tdiv[k] = g.tdiv[k];
    p.full[k] = g.out_full[k];
  }
  for (int t = 0; t < g.parT && t < 64; ++t)
    for (int k = 0; k < 3; ++k) p.toff[t][k] = g.toff[t][k];
  p.alpha = alpha;
  p.beta = beta;
  p.pd = make_fdiv((uint32_t)p.P);
  if (ct_has(p.P)) {
    int m = 1;
#define GILA_CT_XL(n) if (p.P == n) m = ct_xlines<sizeof(C)>(n);
    GILA_CT_SIZES(GILA_CT_XL)
#undef GILA_CT_XL
    p.M = m;
  }
  const int T = ct_has(p.P) ? ct_threads(p.M, p.P) : pass_threads(d.plan[0], p.M);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)p.M * row_stride(p.P) * sizeof(C);
  const bool mx = is_mixed(d.plan[0]);
  const int64_t blocks = (p.rows + p.M - 1) / p.M;
  cudaError_t e =
      axpby ? launch_xinv_one<C, true>(p, mx, T, sm, blocks, L.x_rev != 0, L.xy_g != 0, st)
            : launch_xinv_one<C, false>(p, mx, T, sm, blocks, L.x_rev != 0, L.xy_g != 0, st);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

template <typename C>
cudaError_t launch_matvec_phase(int phase, const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* out,
                                C* A, C* B, int nrhs, bool axpby, C alpha, C beta, cudaStream_t st,
                                const LsEpi<C>* ls) {
  cudaError_t e;
  const Work w = work_sizes(g);
  const int64_t nq_slab = w.slab_planes;
  const int64_t in_rhs = (int64_t)3 * g.sc[0] * g.sc[1] * g.sc[2];
  // planes (rhs, ch, z) are one flat index when B is dense across rhs
  const int64_t fwd_planes = 3LL * g.sc[2];
  const bool fwd_flat = (int64_t)w.zb == g.sc[2];
  const int64_t inv_planes = 3LL * g.parT * g.tc[2];
  const bool inv_flat = (int64_t)w.zb == (int64_t)g.parT * g.tc[2];
  if (phase == 0) {
    const int64_t nr = fwd_flat ? 1 : nrhs;
    const int64_t span = fwd_flat ? fwd_planes * nrhs : fwd_planes;
    for (int64_t r = 0; r < nr; ++r)
      for (int64_t q0 = 0; q0 < span; q0 += nq_slab) {
        const int64_t nq = (span - q0) < nq_slab ? (span - q0) : nq_slab;
        const C* src = in + r * in_rhs + q0 * g.sc[1] * (int64_t)g.sc[0];
        if ((e = launch_xfwd<C>(g, d, L, src, A, nq * g.sc[1], st)) != cudaSuccess) return e;
        if ((e = launch_y<C>(g, d, L, false, A, B + r * w.b_rhs, q0, nq, q0, 0, st)) != cudaSuccess) return e;
      }
    return cudaSuccess;
  }
  if (phase == 1) return launch_z<C>(g, d, L, B, nrhs, st);
  const int64_t nr = inv_flat ? 1 : nrhs;
  const int64_t span = inv_flat ? inv_planes * nrhs : inv_planes;
  for (int64_t r = 0; r < nr; ++r)
    for (int64_t q0 = 0; q0 < span; q0 += nq_slab) {
      const int64_t nq = (span - q0) < nq_slab ? (span - q0) : nq_slab;
      if ((e = launch_y<C>(g, d, L, true, B + r * w.b_rhs, A, q0, nq, 0, q0, st)) != cudaSuccess) return e;
      const int64_t g_off = (r * inv_planes + q0) * g.tc[1];
      if ((e = launch_xinv<C>(g, d, L, A, out, nq * g.tc[1], g_off, axpby, alpha, beta, st, ls)) != cudaSuccess)
        return e;
    }
  return cudaSuccess;
}

// kx chunks of the pipelined matvec (GILA_KX_CHUNKS sets the count; off by
// default: at 256x256x128 F64 one apply took 3.34 ms unpipelined and 3.39 /
// 3.43 / 3.49 ms with 2 / 4 / 8 chunks, F32 1.80 vs 1.84-1.91 ms -- the z
// pass and the y passes contend for the same L1 / shared-memory pipe, and
// the smaller launches lose tail efficiency and the kernel's L2 reuse):
// self operators with specialised y / z lengths, one target partition, the
// x/y slab holding every plane of every vector, chunk boundaries on both
// tile widths
static inline int kx_chunks_wanted() {
  static const int n = [] {
    const char* e = getenv("GILA_KX_CHUNKS");
    const int v = e ? atoi(e) : 0;
    return v < 0 ? 0 : (v > kMaxKxChunks ? kMaxKxChunks : v);
  }();
  return n;
}

template <typename C>
int kx_chunks(const Geom& g, const DevOp<C>& d, const Launch& L, int nrhs) {
  const int want = kx_chunks_wanted();
  if (want < 2 || !d.pst[0] || !d.pst[1] || !d.pjoin || g.parT != 1) return 0;
  if (!ct_has(g.P[1]) || !ct_has(g.P[2])) return 0;
  const Work w = work_sizes(g);
  const int64_t fwd = 3LL * g.sc[2] * nrhs, inv = 3LL * g.tc[2] * nrhs;
  if ((int64_t)w.zb != g.sc[2] || (int64_t)w.zb != g.tc[2] || w.slab_planes < fwd || w.slab_planes < inv) return 0;
  const int txz = ct_tile_pick(sizeof(C), g.P[2], L.z_tx, true);
  const int txy = ct_tile_pick(sizeof(C), g.P[1], L.y_tx, false);
  const int Px = g.P[0];
  if (Px % txz || Px % txy || (Px / txz) % 2) return 0;
  const int pairs = Px / txz / 2;
  const int q = txy > txz ? txy / txz : 1;  // pairs per chunk boundary step
  int n = want;
  while (n > 1 && (pairs % n || (pairs / n) % q)) --n;
  return n > 1 ? n : 0;
}

// The pipelined matvec: x forward on st; per kx chunk c the forward y pass
// on st, the z pass on pst[0] after it, the inverse y pass on pst[1] after
// that; x inverse on st after the last inverse y pass.  Chunks touch
// disjoint kx columns of A and B, so the passes of different chunks run
// concurrently; stream capture records the same dependencies.
template <typename C>
static cudaError_t launch_matvec_pipe(const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* out, C* A,
                                      C* B, int nrhs, bool axpby, C alpha, C beta, cudaStream_t st,
                                      const LsEpi<C>* ls, int nch) {
  cudaError_t e;
  const int64_t fwd_planes = 3LL * g.sc[2] * nrhs, inv_planes = 3LL * g.tc[2] * nrhs;
  const int txz = ct_tile_pick(sizeof(C), g.P[2], L.z_tx, true);
  const int pairs = g.P[0] / txz / 2;
  if ((e = launch_xfwd<C>(g, d, L, in, A, fwd_planes * g.sc[1], st)) != cudaSuccess) return e;
  for (int c = 0; c < nch; ++c) {
    KxChunk ch;
    ch.ts0 = 2 * (pairs / nch) * c;
    ch.nts = 2 * (pairs / nch);
    if ((e = launch_y<C>(g, d, L, false, A, B, 0, fwd_planes, 0, 0, st, &ch)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(d.pev_y[c], st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(d.pst[0], d.pev_y[c], 0)) != cudaSuccess) return e;
    if ((e = launch_z<C>(g, d, L, B, nrhs, d.pst[0], &ch)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(d.pev_z[c], d.pst[0])) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(d.pst[1], d.pev_z[c], 0)) != cudaSuccess) return e;
    if ((e = launch_y<C>(g, d, L, true, B, A, 0, inv_planes, 0, 0, d.pst[1], &ch)) != cudaSuccess) return e;
  }
  if ((e = cudaEventRecord(d.pjoin, d.pst[1])) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(st, d.pjoin, 0)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(st, d.pev_z[nch - 1], 0)) != cudaSuccess) return e;
  return launch_xinv<C>(g, d, L, A, out, inv_planes * g.tc[1], 0, axpby, alpha, beta, st, ls);
}

template <typename C>
cudaError_t launch_matvec(const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* out, C* A, C* B,
                          int nrhs, bool axpby, C alpha, C beta, cudaStream_t st, const LsEpi<C>* ls) {
  const int nch = kx_chunks<C>(g, d, L, nrhs);
  if (nch > 1) return launch_matvec_pipe<C>(g, d, L, in, out, A, B, nrhs, axpby, alpha, beta, st, ls, nch);
  for (int ph = 0; ph < 3; ++ph) {
    cudaError_t e = launch_matvec_phase<C>(ph, g, d, L, in, out, A, B, nrhs, axpby, alpha, beta, st, ls);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

#define GILA_INST(C)                                                                                              \
  template cudaError_t launch_matvec_phase<C>(int, const Geom&, const DevOp<C>&, const Launch&, const C*, C*, C*, \
                                              C*, int, bool, C, C, cudaStream_t, const LsEpi<C>*);                                 \
  template cudaError_t launch_matvec<C>(const Geom&, const DevOp<C>&, const Launch&, const C*, C*, C*, C*, int,   \
                                        bool, C, C, cudaStream_t, const LsEpi<C>*);                                                \
  template cudaError_t launch_xfwd<C>(const Geom&, const DevOp<C>&, const Launch&, const C*, C*, int64_t,         \
                                      cudaStream_t);                                                              \
  template cudaError_t launch_y<C>(const Geom&, const DevOp<C>&, const Launch&, bool, const C*, C*, int64_t,      \
                                   int64_t, int64_t, int64_t, cudaStream_t, const KxChunk*);                      \
  template cudaError_t launch_z<C>(const Geom&, const DevOp<C>&, const Launch&, C*, int, cudaStream_t,            \
                                   const KxChunk*, int, int);                                                     \
  template int kx_chunks<C>(const Geom&, const DevOp<C>&, const Launch&, int);                                    \
  template cudaError_t launch_xinv<C>(const Geom&, const DevOp<C>&, const Launch&, const C*, C*, int64_t,         \
                                      int64_t, bool, C, C, cudaStream_t, const LsEpi<C>*);

}  // namespace gila
