// slab.cu -- the three pieces of a slab-decomposed matvec.
//
// A volume whose padded spectrum does not fit one GPU is split over several
// (one process per GPU, each holding the whole Fourier kernel): rank r keeps
// source z planes Zs_r and target z planes Zt_r of the vectors, and spectrum
// rows Y_r (ky) between the passes.  One matvec is
//   1. gila_opr_slab_fwd on Zs_r: the x and y passes of those planes, every
//      (component, plane) to its full 2-D spectrum (Py rows of Px);
//   2. an all-to-all: rank s receives rows Y_s of every rank's planes, so
//      that it holds the whole source z extent of its rows;
//   3. gila_opr_slab_z on Y_r: the fused z pass of those rows;
//   4. an all-to-all back: rank r receives target planes Zt_r of every
//      rank's rows;
//   5. gila_opr_slab_inv on Zt_r: the inverse y and x passes.
// The exchanges are the caller's (NCCL all-to-all through torch.distributed
// in the Python package).  Each piece runs the same per-line arithmetic as
// gila_opr_apply with the operator's launch choices, so a slab-decomposed
// matvec gives the bits of the single-GPU one.  The reference runs a volume
// on one device (src/glaAct.jl:191-321); the split is this library's.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace gila {

// device pointer on the operator's GPU, aligned to the element
static gila_status check_dev(const Core& c, const void* p, const char* what) {
  if (!p) return fail(GILA_ERR_ARG, std::string("null ") + what);
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return fail(GILA_ERR_ARG, std::string(what) + " is not device memory");
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return fail(GILA_ERR_ARG, std::string(what) + " is not device memory");
  if (a.type == cudaMemoryTypeDevice && a.device != c.device)
    return fail(GILA_ERR_ARG, std::string(what) + " lives on another GPU than the operator");
  if ((uintptr_t)p % csize(c.dtype)) return fail(GILA_ERR_ARG, std::string(what) + " is not element aligned");
  return GILA_OK;
}

static gila_status check_opr(gila_opr* opr, gila_dtype dtype) {
  if (!opr || !opr->core) return fail(GILA_ERR_ARG, "null operator");
  const Core& c = *opr->core;
  if (dtype != c.dtype) return fail(GILA_ERR_TYPE, "vector element type differs from the operator's");
  if (c.parS != 1 || c.geom.parT != 1)
    return fail(GILA_ERR_ARG, "slab pieces need an operator with one source and one target partition");
  return GILA_OK;
}

// x/y slab buffer of a slab geometry
static gila_status slab_a(Core& c, const Geom& g, void** out) {
  const Work w = work_sizes(g);
  if (c.slab_a_cap < w.a_elems) {
    cudaFree(c.slab_a);
    c.slab_a = nullptr;
    c.slab_a_cap = 0;
    GILA_CUDA_TRY(dev_malloc(&c.slab_a, (size_t)w.a_elems * csize(c.dtype)));
    c.slab_a_cap = w.a_elems;
  }
  *out = c.slab_a;
  return GILA_OK;
}

// the operator's geometry restricted to nz z planes of one vector (the x
// and y passes do not depend on z beyond the plane count)
static Geom slab_geom(const Core& c, int64_t nz, bool target) {
  Geom g = c.geom;
  g.max_rhs = 1;
  g.sc[2] = g.tc[2] = (int)nz;
  if (target) g.out_full[2] = nz;
  return g;
}

template <typename C>
static gila_status slab_fwd_t(Core& c, const C* in, int64_t nz, C* bslab, cudaStream_t st) {
  const Geom g = slab_geom(c, nz, false);
  void* A = nullptr;
  gila_status s = slab_a(c, g, &A);
  if (s != GILA_OK) return s;
  const Launch L = c.tuned ? c.launch : default_launch(c);
  C one, zero;
  one.x = 1;
  one.y = 0;
  zero.x = 0;
  zero.y = 0;
  GILA_CUDA_TRY(launch_matvec_phase<C>(0, g, devop<C>(c), L, in, nullptr, static_cast<C*>(A), bslab, 1, false, one,
                                       zero, st));
  return GILA_OK;
}

template <typename C>
static gila_status slab_z_t(Core& c, C* bz, int64_t ky0, int64_t nky, cudaStream_t st) {
  Geom g = c.geom;
  g.max_rhs = 1;
  const Launch L = c.tuned ? c.launch : default_launch(c);
  GILA_CUDA_TRY(launch_z<C>(g, devop<C>(c), L, bz, 1, st, nullptr, (int)ky0, (int)nky));
  return GILA_OK;
}

template <typename C>
static gila_status slab_inv_t(Core& c, const C* bslab, int64_t nz, C* out, cudaStream_t st) {
  const Geom g = slab_geom(c, nz, true);
  void* A = nullptr;
  gila_status s = slab_a(c, g, &A);
  if (s != GILA_OK) return s;
  const Launch L = c.tuned ? c.launch : default_launch(c);
  C one, zero;
  one.x = 1;
  one.y = 0;
  zero.x = 0;
  zero.y = 0;
  GILA_CUDA_TRY(launch_matvec_phase<C>(2, g, devop<C>(c), L, nullptr, out, static_cast<C*>(A), const_cast<C*>(bslab),
                                       1, false, one, zero, st));
  return GILA_OK;
}

}  // namespace gila

using namespace gila;

extern "C" {

gila_status gila_opr_slab_dims(const gila_opr* opr, int64_t dims[5]) {
  if (!opr || !opr->core || !dims) return fail(GILA_ERR_ARG, "null argument");
  const Geom& g = opr->core->geom;
  dims[0] = g.P[0];
  dims[1] = g.P[1];
  dims[2] = g.P[2];
  dims[3] = g.sc[2];
  dims[4] = g.tc[2];
  return GILA_OK;
}

gila_status gila_opr_slab_fwd(gila_opr* opr, gila_dtype dtype, const void* in, int64_t nz, void* bslab,
                              void* stream) {
  gila_status s = check_opr(opr, dtype);
  if (s != GILA_OK) return s;
  Core& c = *opr->core;
  if (nz < 1 || nz > c.geom.sc[2]) return fail(GILA_ERR_SIZE, "slab plane count out of range");
  if ((s = check_dev(c, in, "input slab")) != GILA_OK || (s = check_dev(c, bslab, "spectrum slab")) != GILA_OK)
    return s;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c.stream;
  s = c.dtype == GILA_C128 ? slab_fwd_t<double2>(c, static_cast<const double2*>(in), nz, static_cast<double2*>(bslab), st)
                           : slab_fwd_t<float2>(c, static_cast<const float2*>(in), nz, static_cast<float2*>(bslab), st);
  if (s == GILA_OK && !stream) GILA_CUDA_TRY(cudaStreamSynchronize(st));
  return s;
}

gila_status gila_opr_slab_z(gila_opr* opr, gila_dtype dtype, void* bz, int64_t ky0, int64_t nky, void* stream) {
  gila_status s = check_opr(opr, dtype);
  if (s != GILA_OK) return s;
  Core& c = *opr->core;
  if (ky0 < 0 || nky < 1 || ky0 + nky > c.geom.P[1]) return fail(GILA_ERR_SIZE, "spectrum rows out of range");
  if ((s = check_dev(c, bz, "row slab")) != GILA_OK) return s;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c.stream;
  s = c.dtype == GILA_C128 ? slab_z_t<double2>(c, static_cast<double2*>(bz), ky0, nky, st)
                           : slab_z_t<float2>(c, static_cast<float2*>(bz), ky0, nky, st);
  if (s == GILA_OK && !stream) GILA_CUDA_TRY(cudaStreamSynchronize(st));
  return s;
}

gila_status gila_opr_slab_inv(gila_opr* opr, gila_dtype dtype, const void* bslab, int64_t nz, void* out,
                              void* stream) {
  gila_status s = check_opr(opr, dtype);
  if (s != GILA_OK) return s;
  Core& c = *opr->core;
  if (nz < 1 || nz > c.geom.tc[2]) return fail(GILA_ERR_SIZE, "slab plane count out of range");
  if ((s = check_dev(c, bslab, "spectrum slab")) != GILA_OK || (s = check_dev(c, out, "output slab")) != GILA_OK)
    return s;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c.stream;
  s = c.dtype == GILA_C128
          ? slab_inv_t<double2>(c, static_cast<const double2*>(bslab), nz, static_cast<double2*>(out), st)
          : slab_inv_t<float2>(c, static_cast<const float2*>(bslab), nz, static_cast<float2*>(out), st);
  if (s == GILA_OK && !stream) GILA_CUDA_TRY(cudaStreamSynchronize(st));
  return s;
}

}  // extern "C"
