// matvec.cuh -- geometry of one Green-operator matvec and the launchers of its
// five passes.  See matvec.cu for the kernels.
#pragma once
#include <vector>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft.cuh"

namespace gila {

// Everything the passes need to know about one operator.  Sizes follow
// GlaExtInf (src/glaMem.jl:39-47): sc / tc are srcCel / trgCel (cells of one
// partition), P = sc + tc is the circulant length per axis, tru the stored
// kernel extent per axis (src/glaMemSup.jl:121-136).
struct Geom {
  int sc[3];
  int tc[3];
  int P[3];
  int tru[3];
  int parT;   // target partitions (source partitions are rejected, see gila.cu)
  int tdiv[3];
  int toff[64][3];  // target partition offsets (x fastest), parT <= 64
  int64_t out_full[3];  // full target volume (tc * tdiv)
  int csize;            // bytes per complex element
  int slab_bytes;       // target size of the x/y slab buffer
  int max_rhs;          // right-hand sides the workspaces are sized for
};

// Workspaces (complex elements):
//   A : one slab of slab_planes planes (ch, z) of max(sy, ty) rows of Px,
//       shared by all rhs (the x and y passes run slab by slab)
//   B : per rhs [3*zb][Py][Px] planes, zb = max(sc_z, tc_z*parT)
struct Work {
  int64_t slab_planes;  // planes per slab
  int64_t a_elems;      // elements of the slab buffer A
  int64_t b_rhs;        // elements of B per rhs
  int zb;               // z planes per component in B
};

// complex values staged per thread per FFT stage: power-of-two plans (radix
// 2/4/8 only) and mixed plans (radix 3/5/7 too) are separate instantiations
// so that the common case carries no register pressure from the odd radices.
#ifndef GILA_KE_MIXED
#define GILA_KE_MIXED 4
#endif
constexpr int kE = 8;
constexpr int kEm = GILA_KE_MIXED;

// Default slab size.  Slabs small enough to stay L2-resident between the x
// and y passes cut HBM traffic but multiply the launch count; the default
// keeps one slab (whole volume) until the launches are graph-captured.
constexpr int kSlabBytes = 1 << 30;
Work work_sizes(const Geom& g);

// The y passes and the z pass of a self operator work on independent sets of
// kx columns, so a matvec can run them as a pipeline over kx chunks: the z
// pass of chunk c (bound by the L1 / shared-memory pipe) on its own stream
// while the y passes of chunks c + 1 (forward) and c - 1 (inverse) run on
// two others (bound by memory latency).  A chunk is a range of positions of
// the z pass's mirror tile order (z tiles i and ntiles - 1 - i side by side).
constexpr int kMaxKxChunks = 16;
struct KxChunk {
  int ts0 = 0;   // first position (even)
  int nts = -1;  // positions; < 0: all
};

// Index of stored kernel entry (branch eo = 4 px + 2 py + pz, iz, iy,
// component c, ix) in one target partition's block: the layout is
// [py,pz][tz][ty][6][tx][px] -- the two x parities of one stored x index side
// by side, so that the consecutive kx of a z-pass tile, whose parity
// alternates, read consecutive entries (whole 32-byte sectors) of one
// component.  A block holds 8 * tz * ty * 6 * tx entries.
__host__ __device__ inline int64_t ker_index(int eo, int iz, int iy, int c, int ix, int tx, int ty, int tz) {
  return (((((int64_t)(eo & 3) * tz + iz) * ty + iy) * 6 + c) * tx + ix) * 2 + (eo >> 2);
}

// Per-axis plan (radix list), twiddle tables and kernel-address maps live on
// the device; Dev bundles the pointers for one dtype.
template <typename C>
struct DevOp {
  const C* ker;      // [parT] blocks laid out by ker_index
  const int* map[3]; // per axis, per frequency f: m | p<<29 | mirrored<<30
  const C* tw[3];    // P-point twiddle tables
  AxisPlan plan[3];          // host copies (launch decisions)
  const AxisPlan* plan_d[3]; // device copies (read by the kernels)
  double scale;      // 1 / (Px Py Pz)
  // the operator's kx-chunk pipeline: z-pass and inverse-y streams, per-chunk
  // events after the forward y pass and after the z pass, the join event
  // (no pipeline when pst[0] is null)
  cudaStream_t pst[2] = {nullptr, nullptr};
  cudaEvent_t pev_y[kMaxKxChunks] = {}, pev_z[kMaxKxChunks] = {};
  cudaEvent_t pjoin = nullptr;
};

// Tile / launch parameters picked by the autotuner.
struct Launch {
  int xf_lines;  // lines per CTA, x forward
  int xi_lines;  // lines per CTA, x inverse
  int y_tx;      // kx tile, y passes
  int z_tx;      // kx tile, z pass
  int x_rev = 0;  // radix order of the x passes: 0 greedy (8s first), 1 reversed
  int y_rev = 0;  // radix order of the y passes
  int z_mir = 1;  // fused z pass: one task per mirror pair of z frequencies
  int xy_g = 1;   // x / y passes: first stage fed from global memory and half
                  // last stage (1) or the line staged in shared memory (0);
                  // the same arithmetic either way
};

// Lippmann-Schwinger epilogue of the last pass (self operators): out =
// in - chi .* (G in), chi per cell broadcast over the three components,
// chi_rs = 0 (one medium) or V (one per right-hand side of the launch).
template <typename C>
struct LsEpi {
  const C* in;
  const C* chi;
  int64_t chi_rs;
};

template <typename C>
cudaError_t launch_matvec(const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* out, C* A, C* B,
                          int nrhs, bool axpby, C alpha, C beta, cudaStream_t st, const LsEpi<C>* ls = nullptr);

// Individual passes (exposed for the autotuner and the profiler).
template <typename C>
cudaError_t launch_xfwd(const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* A, int64_t rows,
                        cudaStream_t st);
template <typename C>
cudaError_t launch_y(const Geom& g, const DevOp<C>& d, const Launch& L, bool inv, const C* src, C* dst, int64_t q0,
                     int64_t nq, int64_t src_sub, int64_t dst_sub, cudaStream_t st, const KxChunk* ch = nullptr);
// (ky0, nky >= 0: B holds only spectrum rows ky0 .. ky0 + nky - 1, each
// plane nky rows of Px; the slab pieces of a slab-decomposed matvec)
template <typename C>
cudaError_t launch_z(const Geom& g, const DevOp<C>& d, const Launch& L, C* B, int nrhs, cudaStream_t st,
                     const KxChunk* ch = nullptr, int ky0 = 0, int nky = -1);
// kx chunks the pipelined matvec uses for this operator and launch shape
// (0: no pipeline)
template <typename C>
int kx_chunks(const Geom& g, const DevOp<C>& d, const Launch& L, int nrhs);
template <typename C>
cudaError_t launch_xinv(const Geom& g, const DevOp<C>& d, const Launch& L, const C* A, C* out, int64_t rows,
                        int64_t g_off, bool axpby, C alpha, C beta, cudaStream_t st, const LsEpi<C>* ls = nullptr);

int smem_optin_bytes();

// Kernels one matvec of nrhs vectors launches (kx_chunks > 1: the
// pipelined form).
int64_t matvec_launches(const Geom& g, int nrhs, int kx_chunks = 0);

// The three phases of launch_matvec, for timing: forward x/y slabs, z pass,
// inverse y/x slabs.
template <typename C>
cudaError_t launch_matvec_phase(int phase, const Geom& g, const DevOp<C>& d, const Launch& L, const C* in, C* out,
                                C* A, C* B, int nrhs, bool axpby, C alpha, C beta, cudaStream_t st,
                                const LsEpi<C>* ls = nullptr);
// Threads per CTA of a pass over M lines of an axis plan.
int pass_threads(const AxisPlan& pl, int M);

// Tile widths (kx per CTA) of the compile-time specialised y (z = false) or
// z (z = true) kernels for transform length P and complex size cs; empty when
// P has no specialised kernels.  ct_tile_pick returns `want` when it is one
// of them, else the default (128-byte rows, or the widest that fits).
std::vector<int> ct_tiles(int cs, int P, bool z);
int ct_tile_pick(int cs, int P, int want, bool z);

}  // namespace gila
