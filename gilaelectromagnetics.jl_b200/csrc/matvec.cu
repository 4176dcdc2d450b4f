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

#include "fft_ct.cuh"
#include "matvec.cuh"

namespace gila {

static inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

static bool is_mixed_plan(const AxisPlan& pl) {
  for (int s = 0; s < pl.nst; ++s)
    if (pl.radix[s] != 2 && pl.radix[s] != 4 && pl.radix[s] != 8) return true;
  return false;
}

Work work_sizes(const Geom& g) {
  const int64_t slab_bytes = g.slab_bytes > 0 ? g.slab_bytes : kSlabBytes;
  Work w;
  const int64_t Px = g.P[0], Py = g.P[1];
  const int64_t cs = g.csize;
  const int64_t rows_per_plane = g.sc[1] > g.tc[1] ? g.sc[1] : g.tc[1];
  const int64_t plane_bytes = rows_per_plane * Px * cs;
  int64_t nq = slab_bytes / plane_bytes;
  if (nq < 1) nq = 1;
  const int64_t max_planes = 3LL * (g.sc[2] > g.tc[2] * g.parT ? g.sc[2] : g.tc[2] * g.parT) * g.max_rhs;
  if (nq > max_planes) nq = max_planes;
  w.slab_planes = nq;
  w.a_elems = nq * rows_per_plane * Px;
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

int pass_threads(const AxisPlan& pl, int M) {
  const int E = is_mixed_plan(pl) ? kEm : kE;
  int t = round_up((M * pl.P + E - 1) / E, 32);
  return t < 32 ? 32 : t;
}

// The x and y passes run slab by slab over planes (ch, z) so that the slab
// buffer A between them stays resident in L2 and is overwritten there by the
// next slab: the x<->y intermediate then never reaches HBM.
int64_t matvec_launches(const Geom& g, int nrhs, int kx_chunks) {
  if (kx_chunks > 1) return 2 + 3LL * kx_chunks;
  const Work w = work_sizes(g);
  const int64_t fwd_planes = 3LL * g.sc[2], inv_planes = 3LL * g.parT * g.tc[2];
  const bool fwd_flat = (int64_t)w.zb == g.sc[2];
  const bool inv_flat = (int64_t)w.zb == (int64_t)g.parT * g.tc[2];
  auto slabs = [&](int64_t span) { return (span + w.slab_planes - 1) / w.slab_planes; };
  const int64_t nf = fwd_flat ? slabs(fwd_planes * nrhs) : nrhs * slabs(fwd_planes);
  const int64_t ni = inv_flat ? slabs(inv_planes * nrhs) : nrhs * slabs(inv_planes);
  return 2 * nf + 1 + 2 * ni;
}

static bool ct_len(int P) {
  for (int n : {64, 96, 128, 192, 256, 384, 512})
    if (P == n) return true;
  return false;
}

std::vector<int> ct_tiles(int cs, int P, bool z) {
  std::vector<int> v;
  if (!ct_len(P)) return v;
  for (int tx : kTileSet)
    if (z ? ct_z_ok(cs, P, tx) : ct_y_ok(cs, P, tx)) v.push_back(tx);
  return v;
}

int ct_tile_pick(int cs, int P, int want, bool z) {
  const std::vector<int> v = ct_tiles(cs, P, z);
  for (int tx : v)
    if (tx == want) return tx;
  // default: the widest up to 128-byte rows
  int best = v.empty() ? 1 : v.front();
  for (int tx : v)
    if (tx * cs <= 128) best = tx;
  return best;
}

}  // namespace gila
