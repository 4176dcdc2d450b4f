// matvec.cu -- the five passes of the Green-operator matvec on sm_100a.
//
// The reference's egoBrnDev! (src/glaAct.jl:191-321) walks a depth-3 binary
// tree of parity branches: split along x, 1-D FFT x, split y, FFT y, split z,
// FFT z, 3x3 multiply in each of the 8 leaves (src/glaActSup.jl:766-935),
// then inverse FFTs and merges back up, with a CUDA.synchronize and an
// allocation after nearly every step.  Arithmetically that is a zero-padded
// length-P convolution per axis, so here it runs as five bandwidth-bound
// passes over HBM, each a batched Stockham FFT with its pre/post-processing
// fused in:
//
//   xfwd : rows of the source (x contiguous) -> length-Px spectra (pad fused)
//   yfwd : columns along y of tiles of kx    -> length-Py spectra (pad fused)
//   z    : z pencils of a kx tile, all 3 components: forward length-Pz FFT
//          (pad fused), 3x3 complex-symmetric multiply with the stored
//          Fourier kernel (mirror/sign rules of mulBrnDev!, normalisation
//          1/(Px Py Pz) folded in), inverse FFT truncated to the target z
//   yinv : inverse along y, truncated to the target y
//   xinv : inverse along x, truncated to the target x; target partition
//          scatter (mrgPrtDev!, src/glaActSup.jl:956-1004) and the mul!
//          axpby epilogue (src/glaLinAlg.jl:61-69) fused into the store.
#include <cstdio>

#include "matvec.cuh"

namespace gila {

// complex values staged per thread per FFT stage: power-of-two plans (radix
// 2/4/8 only) and mixed plans (radix 3/5/7 too) are separate instantiations
// so that the common case carries no register pressure from the odd radices.
#ifndef GILA_KE_MIXED
#define GILA_KE_MIXED 4
#endif
constexpr int kE = 8;
constexpr int kEm = GILA_KE_MIXED;
template <bool MX> struct StageE { static constexpr int v = MX ? kEm : kE; };

static inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

Work work_sizes(const Geom& g) {
  Work w;
  const int64_t Px = g.P[0], Py = g.P[1];
  const int64_t fwd_rows = (int64_t)g.sc[2] * g.sc[1];
  const int64_t inv_rows = (int64_t)g.tc[2] * g.tc[1] * g.parT;
  w.a_rhs = 3 * (fwd_rows > inv_rows ? fwd_rows : inv_rows) * Px;
  w.zb = g.sc[2] > g.tc[2] * g.parT ? g.sc[2] : g.tc[2] * g.parT;
  w.b_rhs = 3 * (int64_t)w.zb * Py * Px;
  return w;
}

int smem_optin_bytes() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v;
}

// -------------------------------------------------------------------- xfwd
template <typename C>
struct XfParams {
  const C* in;
  C* A;
  AxisPlan pl;
  const C* tw;
  int nin;       // source x cells
  int M;         // rows per CTA
  int64_t rows;  // total rows = 3 * sy * sz * nrhs
};

template <typename C, bool MX>
__global__ void __launch_bounds__(512) k_xfwd(const XfParams<C> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan pl = p.pl;
  const int P = pl.P, M = p.M, nin = p.nin;
  const int64_t rows = p.rows;
  const C* const in = p.in;
  C* const A = p.A;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  auto ldg = [=](int l, int i) -> C {
    const int64_t g = g0 + l;
    if (g < rows && i < nin) return in[g * nin + i];
    return czero<C>();
  };
  auto lds = [=](int l, int i) -> C { return sm[l * P + i]; };
  auto sts = [=](int l, int i, C v) { sm[l * P + i] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g < rows) A[g * P + i] = v;
  };
  fft_run<C, StageE<MX>::v, false, false, MX>(pl, M, p.tw, ldg, lds, sts, stg, false, false);
}

// ---------------------------------------------------------------------- y
template <typename C>
struct YParams {
  const C* src;
  C* dst;
  AxisPlan pl;
  const C* tw;
  int Px;
  int TX;
  int ntiles;     // ceil(Px / TX)
  int nin, nout;  // rows read / written
  int nz;         // z planes per channel in this pass
  int src_z, dst_z;          // z planes per channel in the src / dst layouts
  int src_rows, dst_rows;    // y rows per plane in the src / dst layouts
};

template <typename C, bool INV, bool MX>
__global__ void __launch_bounds__(512) k_y(const YParams<C> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan pl = p.pl;
  const int Px = p.Px, TX = p.TX, nin = p.nin, nout = p.nout;
  const int tile = blockIdx.x % p.ntiles;
  const int64_t slice = blockIdx.x / p.ntiles;  // (rhs*nch + ch)*nz + z
  const int64_t rc = slice / p.nz;
  const int z = (int)(slice % p.nz);
  const int kx0 = tile * TX;
  const int M = TX;
  const C* const src = p.src + ((rc * p.src_z + z) * p.src_rows) * (int64_t)Px + kx0;
  C* const dst = p.dst + ((rc * p.dst_z + z) * p.dst_rows) * (int64_t)Px + kx0;
  const int tmax = Px - kx0;
  auto ldg = [=](int t, int i) -> C {
    if (t < tmax && i < nin) return src[(int64_t)i * Px + t];
    return czero<C>();
  };
  auto lds = [=](int t, int i) -> C { return sm[i * M + t]; };
  auto sts = [=](int t, int i, C v) { sm[i * M + t] = v; };
  auto stg = [=](int t, int i, C v) {
    if (t < tmax && i < nout) dst[(int64_t)i * Px + t] = v;
  };
  fft_run<C, StageE<MX>::v, INV, true, MX>(pl, M, p.tw, ldg, lds, sts, stg, false, false);
}

// ---------------------------------------------------------------------- z
template <typename C>
struct ZParams {
  C* B;
  const C* ker;
  const int* mapx;
  const int* mapy;
  const int* mapz;
  AxisPlan pl;
  const C* tw;
  int Px, Py;
  int TX, ntiles;
  int nin, nout;  // source / target z cells
  int zb;         // z planes per channel in B
  int tx, ty, tz; // stored kernel extents
  int parT;
  int nrhs;
  double scale;
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

template <typename C>
__device__ __forceinline__ C ker_ld(const C* __restrict__ g, int c) {
  return __ldg(g + c);
}

template <typename C, bool MX>
__global__ void __launch_bounds__(512) k_z(const ZParams<C> p) {
  using T = typename Real<C>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan pl = p.pl;
  const int P = pl.P;
  const int nrhs = p.nrhs, ntiles = p.ntiles, TX = p.TX, Px = p.Px, Py = p.Py;
  const int nin = p.nin, nout = p.nout;
  const int rhs = blockIdx.x % nrhs;
  const int rest = blockIdx.x / nrhs;
  const int tseq = rest % ntiles;
  const int yseq = rest / ntiles;
  const int kx0 = tile_seq(tseq, ntiles) * TX;
  const int ky = mirror_seq(yseq, Py);
  const int M = 3 * TX;  // lines: (c, t), t fastest
  const int tmax = Px - kx0;
  const int64_t plane = (int64_t)Py * Px;
  C* const Bb = p.B + (int64_t)rhs * 3 * p.zb * plane + (int64_t)ky * Px + kx0;
  // forward: global (source z) -> shared, all Pz frequencies
  auto ldg = [=](int l, int i) -> C {
    const int c = l / TX, t = l - c * TX;
    if (t < tmax && i < nin) return Bb[((int64_t)c * nin + i) * plane + t];
    return czero<C>();
  };
  auto lds = [=](int l, int i) -> C { return sm[i * M + l]; };
  auto sts = [=](int l, int i, C v) { sm[i * M + l] = v; };
  fft_run<C, StageE<MX>::v, false, true, MX>(pl, M, p.tw, ldg, lds, sts, sts, false, true);

  const int my = __ldg(p.mapy + ky);
  const int py = (my >> 29) & 1, ry = (my >> 30) & 1;
  const int iy = my & 0x1fffffff;
  const int tx = p.tx, ty = p.ty, tz = p.tz, parT = p.parT;
  const int* const mapx = p.mapx;
  const int* const mapz = p.mapz;
  const T s = (T)p.scale;
  C* const out3 = sm + (int64_t)P * M;  // extra 3-channel buffer (parT > 1 only)
  for (int t_par = 0; t_par < parT; ++t_par) {
    C* const dst = (parT == 1) ? sm : out3;
    const C* const kpar = p.ker + (int64_t)t_par * 8 * tz * ty * tx * 6;
    for (int task = threadIdx.x; task < TX * P; task += blockDim.x) {
      const int t = task % TX, kz = task / TX;
      const int kx = kx0 + t;
      if (kx >= Px) continue;
      const int mx = __ldg(mapx + kx), mz = __ldg(mapz + kz);
      const int px = (mx >> 29) & 1, rx = (mx >> 30) & 1, ix = mx & 0x1fffffff;
      const int pz = (mz >> 29) & 1, rz = (mz >> 30) & 1, iz = mz & 0x1fffffff;
      const int eo = 4 * px + 2 * py + pz;
      const C* g = kpar + ((((int64_t)eo * tz + iz) * ty + iy) * tx + ix) * 6;
      const T sxy = (rx ^ ry) ? (T)-1 : (T)1;
      const T sxz = (rx ^ rz) ? (T)-1 : (T)1;
      const T syz = (ry ^ rz) ? (T)-1 : (T)1;
      const C gxx = ker_ld(g, 0), gyy = ker_ld(g, 1), gzz = ker_ld(g, 2);
      const C gxy = cscale(ker_ld(g, 3), sxy), gxz = cscale(ker_ld(g, 4), sxz), gyz = cscale(ker_ld(g, 5), syz);
      const C x0 = sm[kz * M + t], x1 = sm[kz * M + TX + t], x2 = sm[kz * M + 2 * TX + t];
      C y0 = cadd(cadd(cmul(gxx, x0), cmul(gxy, x1)), cmul(gxz, x2));
      C y1 = cadd(cadd(cmul(gxy, x0), cmul(gyy, x1)), cmul(gyz, x2));
      C y2 = cadd(cadd(cmul(gxz, x0), cmul(gyz, x1)), cmul(gzz, x2));
      dst[kz * M + t] = cscale(y0, s);
      dst[kz * M + TX + t] = cscale(y1, s);
      dst[kz * M + 2 * TX + t] = cscale(y2, s);
    }
    __syncthreads();
    // inverse: shared -> global (target z), truncated
    C* const Bo = Bb + (int64_t)(t_par * 3) * nout * plane;
    auto ldo = [=](int l, int i) -> C { return dst[i * M + l]; };
    auto sto = [=](int l, int i, C v) { dst[i * M + l] = v; };
    auto stg = [=](int l, int i, C v) {
      const int c = l / TX, t = l - c * TX;
      if (t < tmax && i < nout) Bo[((int64_t)c * nout + i) * plane + t] = v;
    };
    fft_run<C, StageE<MX>::v, true, true, MX>(pl, M, p.tw, ldo, ldo, sto, stg, true, false);
  }
}

// -------------------------------------------------------------------- xinv
template <typename C>
struct XiParams {
  const C* A;
  C* out;
  AxisPlan pl;
  const C* tw;
  int nout;  // target x cells
  int M;
  int64_t rows;  // 3 * parT * ty * tz * nrhs
  int ty, tz, parT;
  int part_scatter;  // parT > 1
  int tdiv[3];
  int toff[64][3];
  int64_t full[3];
  C alpha, beta;
};

template <typename C, bool AXPBY, bool MX>
__global__ void __launch_bounds__(512) k_xinv(const XiParams<C> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* const sm = reinterpret_cast<C*>(smem_raw);
  const AxisPlan pl = p.pl;
  const int P = pl.P, M = p.M, nout = p.nout;
  const int64_t rows = p.rows;
  const C* const A = p.A;
  C* const out = p.out;
  const C alpha = p.alpha, beta = p.beta;
  const int64_t g0 = (int64_t)blockIdx.x * M;
  const bool scatter = p.part_scatter != 0;
  const int ty = p.ty, tz = p.tz, parT = p.parT;
  const int d0 = p.tdiv[0], d1 = p.tdiv[1], d2 = p.tdiv[2];
  const int64_t f0 = p.full[0], f1 = p.full[1], f2 = p.full[2];
  const int(*toff)[3] = p.toff;
  auto ldg = [=](int l, int i) -> C {
    const int64_t g = g0 + l;
    if (g < rows) return A[g * P + i];
    return czero<C>();
  };
  auto lds = [=](int l, int i) -> C { return sm[l * P + i]; };
  auto sts = [=](int l, int i, C v) { sm[l * P + i] = v; };
  auto stg = [=](int l, int i, C v) {
    const int64_t g = g0 + l;
    if (g >= rows || i >= nout) return;
    int64_t o;
    if (!scatter) {
      o = g * nout + i;
    } else {
      // g = ((rhs*parT + t)*3 + c)*tz + z)*ty + y
      int64_t q = g;
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
    else
      out[o] = v;
  };
  fft_run<C, StageE<MX>::v, true, false, MX>(pl, M, p.tw, ldg, lds, sts, stg, false, false);
}

// ---------------------------------------------------------------- launchers
static cudaError_t set_smem(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return cudaSuccess;
}

static bool is_mixed(const AxisPlan& pl) {
  for (int s = 0; s < pl.nst; ++s)
    if (pl.radix[s] != 2 && pl.radix[s] != 4 && pl.radix[s] != 8) return true;
  return false;
}

int pass_threads(const AxisPlan& pl, int M) {
  const int E = is_mixed(pl) ? kEm : kE;
  int t = round_up((M * pl.P + E - 1) / E, 32);
  return t < 32 ? 32 : t;
}

#define GILA_LAUNCH(MXV, KERNEL, ...)                                                        \
  do {                                                                                       \
    const void* fn__ = (const void*)KERNEL;                                                  \
    cudaError_t e__ = set_smem(fn__, sm);                                                    \
    if (e__ != cudaSuccess) return e__;                                                      \
    KERNEL<<<(unsigned)blocks, T, sm, st>>>(__VA_ARGS__);                                    \
  } while (0)

template <typename C>
cudaError_t launch_xfwd(const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* A, int nrhs,
                        cudaStream_t st) {
  XfParams<C> p;
  p.in = in;
  p.A = A;
  p.pl = d.plan[0];
  p.tw = d.tw[0];
  p.nin = g.sc[0];
  p.M = L.xf_lines;
  p.rows = (int64_t)3 * g.sc[1] * g.sc[2] * nrhs;
  const int T = pass_threads(p.pl, p.M);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)p.M * p.pl.P * sizeof(C);
  const int64_t blocks = (p.rows + p.M - 1) / p.M;
  if (is_mixed(p.pl))
    GILA_LAUNCH(true, (k_xfwd<C, true>), p);
  else
    GILA_LAUNCH(false, (k_xfwd<C, false>), p);
  return cudaGetLastError();
}

template <typename C, bool INV>
static cudaError_t launch_y_one(const YParams<C>& p, int T, size_t sm, int64_t blocks, cudaStream_t st) {
  if (is_mixed(p.pl))
    GILA_LAUNCH(true, (k_y<C, INV, true>), p);
  else
    GILA_LAUNCH(false, (k_y<C, INV, false>), p);
  return cudaSuccess;
}

template <typename C>
cudaError_t launch_y(const Geom& g, const DevOp<C>& d, const Launch& L, bool inv, const C* src, C* dst, int nrhs,
                     cudaStream_t st) {
  const Work w = work_sizes(g);
  YParams<C> p;
  p.src = src;
  p.dst = dst;
  p.pl = d.plan[1];
  p.tw = d.tw[1];
  p.Px = g.P[0];
  p.TX = L.y_tx;
  p.ntiles = (p.Px + p.TX - 1) / p.TX;
  int nch;
  if (!inv) {
    nch = 3;
    p.nin = g.sc[1];
    p.nout = g.P[1];
    p.nz = g.sc[2];
    p.src_z = g.sc[2];
    p.src_rows = g.sc[1];
    p.dst_z = g.sc[2];  // B planes: c*sz + z
    p.dst_rows = g.P[1];
  } else {
    nch = 3 * g.parT;
    p.nin = g.P[1];
    p.nout = g.tc[1];
    p.nz = g.tc[2];
    p.src_z = g.tc[2];  // B planes: ch*tz + z
    p.src_rows = g.P[1];
    p.dst_z = g.tc[2];
    p.dst_rows = g.tc[1];
  }
  const int T = pass_threads(p.pl, p.TX);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)p.TX * p.pl.P * sizeof(C);
  const int64_t src_rhs = inv ? w.b_rhs : w.a_rhs;
  const int64_t dst_rhs = inv ? w.a_rhs : w.b_rhs;
  const int64_t dense_src = (int64_t)nch * p.src_z * p.src_rows * p.Px;
  const int64_t dense_dst = (int64_t)nch * p.dst_z * p.dst_rows * p.Px;
  cudaError_t e = cudaSuccess;
  if (src_rhs == dense_src && dst_rhs == dense_dst) {
    const int64_t blocks = (int64_t)p.ntiles * nch * p.nz * nrhs;
    e = inv ? launch_y_one<C, true>(p, T, sm, blocks, st) : launch_y_one<C, false>(p, T, sm, blocks, st);
  } else {
    // per-rhs blocks are padded (workspace sized for the larger direction)
    const int64_t blocks = (int64_t)p.ntiles * nch * p.nz;
    for (int r = 0; r < nrhs && e == cudaSuccess; ++r) {
      YParams<C> q = p;
      q.src = src + (int64_t)r * src_rhs;
      q.dst = dst + (int64_t)r * dst_rhs;
      e = inv ? launch_y_one<C, true>(q, T, sm, blocks, st) : launch_y_one<C, false>(q, T, sm, blocks, st);
    }
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

template <typename C>
cudaError_t launch_z(const Geom& g, const DevOp<C>& d, const Launch& L, C* B, int nrhs, cudaStream_t st) {
  const Work w = work_sizes(g);
  ZParams<C> p;
  p.B = B;
  p.ker = d.ker;
  p.mapx = d.map[0];
  p.mapy = d.map[1];
  p.mapz = d.map[2];
  p.pl = d.plan[2];
  p.tw = d.tw[2];
  p.Px = g.P[0];
  p.Py = g.P[1];
  p.TX = L.z_tx;
  p.ntiles = (p.Px + p.TX - 1) / p.TX;
  p.nin = g.sc[2];
  p.nout = g.tc[2];
  p.zb = w.zb;
  p.tx = g.tru[0];
  p.ty = g.tru[1];
  p.tz = g.tru[2];
  p.parT = g.parT;
  p.nrhs = nrhs;
  p.scale = d.scale;
  const int M = 3 * p.TX;
  const int T = pass_threads(p.pl, M);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)M * p.pl.P * sizeof(C) * (g.parT > 1 ? 2 : 1);
  const int64_t blocks = (int64_t)p.ntiles * p.Py * nrhs;
  if (is_mixed(p.pl))
    GILA_LAUNCH(true, (k_z<C, true>), p);
  else
    GILA_LAUNCH(false, (k_z<C, false>), p);
  return cudaGetLastError();
}

template <typename C, bool AXPBY>
static cudaError_t launch_xinv_one(const XiParams<C>& p, int T, size_t sm, int64_t blocks, cudaStream_t st) {
  if (is_mixed(p.pl))
    GILA_LAUNCH(true, (k_xinv<C, AXPBY, true>), p);
  else
    GILA_LAUNCH(false, (k_xinv<C, AXPBY, false>), p);
  return cudaSuccess;
}

template <typename C>
cudaError_t launch_xinv(const Geom& g, const DevOp<C>& d, const Launch& L, const C* A, C* out, int nrhs, bool axpby,
                        C alpha, C beta, cudaStream_t st) {
  XiParams<C> p;
  p.A = A;
  p.out = out;
  p.pl = d.plan[0];
  p.tw = d.tw[0];
  p.nout = g.tc[0];
  p.M = L.xi_lines;
  p.ty = g.tc[1];
  p.tz = g.tc[2];
  p.parT = g.parT;
  p.rows = (int64_t)3 * g.parT * g.tc[1] * g.tc[2] * nrhs;
  p.part_scatter = g.parT > 1;
  for (int k = 0; k < 3; ++k) {
    p.tdiv[k] = g.tdiv[k];
    p.full[k] = g.out_full[k];
  }
  for (int t = 0; t < g.parT && t < 64; ++t)
    for (int k = 0; k < 3; ++k) p.toff[t][k] = g.toff[t][k];
  p.alpha = alpha;
  p.beta = beta;
  const int T = pass_threads(p.pl, p.M);
  if (T > 512) return cudaErrorInvalidConfiguration;
  const size_t sm = (size_t)p.M * p.pl.P * sizeof(C);
  // the A rows of one rhs are dense only when a_rhs matches the inverse layout
  const Work w = work_sizes(g);
  const int64_t rows_rhs = (int64_t)3 * g.parT * g.tc[1] * g.tc[2];
  cudaError_t e = cudaSuccess;
  if (w.a_rhs == rows_rhs * g.P[0]) {
    const int64_t blocks = (p.rows + p.M - 1) / p.M;
    e = axpby ? launch_xinv_one<C, true>(p, T, sm, blocks, st) : launch_xinv_one<C, false>(p, T, sm, blocks, st);
  } else {
    const int64_t out_rhs = 3 * g.out_full[0] * g.out_full[1] * g.out_full[2];
    for (int r = 0; r < nrhs && e == cudaSuccess; ++r) {
      XiParams<C> q = p;
      q.A = A + (int64_t)r * w.a_rhs;
      q.out = out + (int64_t)r * out_rhs;
      q.rows = rows_rhs;
      const int64_t blocks = (q.rows + q.M - 1) / q.M;
      e = axpby ? launch_xinv_one<C, true>(q, T, sm, blocks, st) : launch_xinv_one<C, false>(q, T, sm, blocks, st);
    }
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

template <typename C>
cudaError_t launch_matvec(const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* out, C* A, C* B,
                          int nrhs, bool axpby, C alpha, C beta, cudaStream_t st) {
  cudaError_t e;
  // xfwd writes A densely per rhs only when a_rhs equals the forward extent
  const Work w = work_sizes(g);
  const int64_t fwd_rhs = (int64_t)3 * g.sc[1] * g.sc[2] * g.P[0];
  if (w.a_rhs == fwd_rhs) {
    if ((e = launch_xfwd<C>(g, d, L, in, A, nrhs, st)) != cudaSuccess) return e;
  } else {
    const int64_t in_rhs = (int64_t)3 * g.sc[0] * g.sc[1] * g.sc[2];
    for (int r = 0; r < nrhs; ++r)
      if ((e = launch_xfwd<C>(g, d, L, in + r * in_rhs, A + r * w.a_rhs, 1, st)) != cudaSuccess) return e;
  }
  if ((e = launch_y<C>(g, d, L, false, A, B, nrhs, st)) != cudaSuccess) return e;
  if ((e = launch_z<C>(g, d, L, B, nrhs, st)) != cudaSuccess) return e;
  if ((e = launch_y<C>(g, d, L, true, B, A, nrhs, st)) != cudaSuccess) return e;
  return launch_xinv<C>(g, d, L, A, out, nrhs, axpby, alpha, beta, st);
}

#define GILA_INST(C)                                                                                              \
  template cudaError_t launch_matvec<C>(const Geom&, const DevOp<C>&, const Launch&, const C*, C*, C*, C*, int,   \
                                        bool, C, C, cudaStream_t);                                                \
  template cudaError_t launch_xfwd<C>(const Geom&, const DevOp<C>&, const Launch&, const C*, C*, int,             \
                                      cudaStream_t);                                                              \
  template cudaError_t launch_y<C>(const Geom&, const DevOp<C>&, const Launch&, bool, const C*, C*, int,          \
                                   cudaStream_t);                                                                 \
  template cudaError_t launch_z<C>(const Geom&, const DevOp<C>&, const Launch&, C*, int, cudaStream_t);           \
  template cudaError_t launch_xinv<C>(const Geom&, const DevOp<C>&, const Launch&, const C*, C*, int, bool, C, C, \
                                      cudaStream_t);
GILA_INST(double2)
GILA_INST(float2)

}  // namespace gila
