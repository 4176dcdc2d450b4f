// noalloc.cu -- a matvec entry point that allocates no device memory.
//
// gila_opr_apply sizes its scratch workspaces (the x/y slab and the padded
// spectrum between the passes) with cudaMalloc on first use.  Some callers
// cannot let a library allocate at that point: hosts whose own allocator owns
// every byte of device memory (a Julia CUDA.jl or framework memory pool that
// reserved the device at start-up, so a foreign cudaMalloc fails or steals
// memory the pool has promised elsewhere), and latency-critical loops that
// forbid allocation after start-up (cudaMalloc can synchronise the device and
// takes an unbounded time).  For them this entry point runs the same five
// passes with its scratch in one fixed, file-scope device array instead.
//
// The array is kNoAllocScratchBytes (64 MiB) and is reserved on every GPU that
// loads the library, for the life of the process.  It is shared by every call
// on that device and keeps the contents of the last call; nothing in it needs
// to start at zero, because every scratch element a matvec reads is written
// earlier in the same matvec.  Calls that overlap on the GPU (different
// streams, or different host threads without ordering) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

namespace gila {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch, looked up once per device (the first
// call on that device, with the device current) and kept for the process.
// In host code the symbol names a host-side stand-in, not a device address,
// so it is never handed to a kernel directly.  Like every operator's device
// memory, the kept address does not survive cudaDeviceReset.
static std::mutex g_na_mu;
static void* g_na_ptr[128] = {};

static gila_status noalloc_scratch(int device, void** out) {
  if (device < 0 || device >= 128) return fail(GILA_ERR_ARG, "device index out of range for the no-alloc scratch");
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_na_ptr[device] = p;
  }
  *out = g_na_ptr[device];
  return GILA_OK;
}

template <typename C>
static gila_status noalloc_t(Core& c, const void* in, void* out, cudaStream_t user_st) {
  void* scratch = nullptr;
  gila_status s = noalloc_scratch(c.device, &scratch);
  if (s != GILA_OK) return s;
  // Workspace plan: the whole padded spectrum B of one vector, plus an x/y
  // slab A sized to whatever room is left (at least one plane).
  Geom g = c.geom;
  g.max_rhs = 1;
  const size_t cs = sizeof(C);
  const Work w1 = work_sizes(g);
  const size_t b_bytes = ((size_t)w1.b_rhs * cs + 255) / 256 * 256;
  const int64_t plane_rows = g.sc[1] > g.tc[1] ? g.sc[1] : g.tc[1];
  const size_t plane_bytes = (size_t)plane_rows * g.P[0] * cs;
  if (b_bytes + plane_bytes > kNoAllocScratchBytes)
    return fail(GILA_ERR_SIZE, "operator too large for gila_opr_apply_noalloc: it needs " +
                                   std::to_string(b_bytes + plane_bytes) + " bytes of scratch, the fixed scratch holds " +
                                   std::to_string(kNoAllocScratchBytes) + " bytes; use gila_opr_apply");
  const size_t room = kNoAllocScratchBytes - b_bytes;
  g.slab_bytes = (int)(room < (size_t)(1u << 30) ? room : (size_t)(1u << 30));
  const Work w = work_sizes(g);
  if (b_bytes + (size_t)w.a_elems * cs > kNoAllocScratchBytes)
    return fail(GILA_ERR_INTERNAL, "no-alloc workspace plan exceeds the scratch");
  C* B = static_cast<C*>(scratch);
  C* A = reinterpret_cast<C*>(static_cast<unsigned char*>(scratch) + b_bytes);
  const DevOp<C> d = devop<C>(c);
  const Launch L = c.tuned ? c.launch : default_launch(c);
  cudaStream_t st = user_st ? user_st : c.stream;
  C one, zero;
  one.x = 1;
  one.y = 0;
  zero.x = 0;
  zero.y = 0;
  GILA_CUDA_TRY(launch_matvec<C>(g, d, L, static_cast<const C*>(in), static_cast<C*>(out), A, B, 1, false, one, zero,
                                 st));
  if (!user_st) GILA_CUDA_TRY(cudaStreamSynchronize(st));
  return GILA_OK;
}

}  // namespace gila

using namespace gila;

extern "C" gila_status gila_opr_apply_noalloc(gila_opr* opr, gila_dtype dtype, const void* in, int64_t in_len,
                                              void* out, int64_t out_len, void* stream) {
  if (!opr || !opr->core) return fail(GILA_ERR_ARG, "null operator");
  Core& c = *opr->core;
  if (dtype != c.dtype) return fail(GILA_ERR_TYPE, "vector element type differs from the operator's");
  const int64_t ni = 3LL * c.geom.sc[0] * c.geom.sc[1] * c.geom.sc[2];
  const int64_t no = 3LL * c.geom.out_full[0] * c.geom.out_full[1] * c.geom.out_full[2];
  if (c.parS != 1 || in_len != ni || out_len != no)
    return fail(GILA_ERR_SIZE,
                "Size of input vector does not match size of source volume. Required data layout is (srcCelX, "
                "srcCelY, srcCelZ, 3).");
  if (!in || !out) return fail(GILA_ERR_ARG, "null vector");
  // device vectors only: staging host vectors would need device buffers
  for (const void* p : {in, static_cast<const void*>(out)}) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return fail(GILA_ERR_ARG, "gila_opr_apply_noalloc takes device pointers only");
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
      return fail(GILA_ERR_ARG, "gila_opr_apply_noalloc takes device pointers only");
    if (a.type == cudaMemoryTypeDevice && a.device != c.device)
      return fail(GILA_ERR_ARG, "gila_opr_apply_noalloc: a vector lives on another GPU than the operator");
  }
  const size_t cs = csize(c.dtype);
  if ((uintptr_t)in % cs || (uintptr_t)out % cs)
    return fail(GILA_ERR_ARG, "device vectors must be aligned to their complex element size");
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (c.dtype == GILA_C128) return noalloc_t<double2>(c, in, out, st);
  return noalloc_t<float2>(c, in, out, st);
}
