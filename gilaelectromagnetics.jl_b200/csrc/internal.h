// internal.h -- host-side operator state shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gila_b200.h"
#include "matvec.cuh"

namespace gila {

void set_error(const std::string& msg);
gila_status fail(gila_status s, const std::string& msg);
gila_status cuda_fail(cudaError_t e, const char* where);

// Every device allocation of the library goes through dev_malloc, so that a
// test can make the n-th one fail (gila_debug_fail_alloc) without touching
// the GPU: the failure is returned before cudaMalloc is called.
cudaError_t dev_malloc_raw(void** p, size_t bytes);
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  return dev_malloc_raw(reinterpret_cast<void**>(p), bytes);
}

#define GILA_CUDA_TRY(expr)                                     \
  do {                                                          \
    cudaError_t e__ = (expr);                                   \
    if (e__ != cudaSuccess) return ::gila::cuda_fail(e__, #expr); \
  } while (0)

// Rational arithmetic on int64 num/den pairs (GlaVol uses Julia Rationals).
struct Rat {
  int64_t n, d;
};
Rat rat(int64_t n, int64_t d);
bool rat_eq(Rat a, Rat b);

// Volume in rational form (GlaVol, src/glaMem.jl:12-19).
struct Vol {
  int64_t cel[3];
  Rat scl[3], org[3], grd[3];
};
Vol vol_from_abi(const gila_vol& v);
gila_vol vol_to_abi(const Vol& v);
bool vol_eq(const Vol& a, const Vol& b);
Vol vol_even(const Vol& v);

struct ExtInf {  // GlaExtInf (src/glaMem.jl:39-47)
  Rat min_scl[3];
  int tdiv[3], sdiv[3];
  int tc[3], sc[3];
};
gila_status ext_inf(const Vol& trg, const Vol& src, ExtInf* out);

struct Ctx;
class LsBatch;

// Device-resident operator data, shared between an operator and its adjoint.
struct Core {
  Ctx* ctx = nullptr;
  int device = 0;
  gila_dtype dtype = GILA_C128;
  bool self = true;
  Vol trg{}, src{};  // volumes after even-cell regeneration
  ExtInf mix{};
  gila_kopt opt{};
  Geom geom{};
  int parS = 1;
  AxisPlan plan[3]{};
  void* ker = nullptr;  // device, complex, target-partition blocks laid out by ker_index (matvec.cuh)
  size_t ker_bytes = 0;
  int* maps[3] = {nullptr, nullptr, nullptr};
  AxisPlan* plan_d = nullptr;  // device copies of plan[3]
  const void* tw[3] = {nullptr, nullptr, nullptr};  // owned by ctx cache
  // workspaces
  void* A = nullptr;
  void* B = nullptr;
  int64_t cap_rhs = 0;
  void* stage_in = nullptr;
  void* stage_out = nullptr;
  int64_t stage_cap_in = 0, stage_cap_out = 0;
  // host-vector pipeline (several vectors in host memory): two staging
  // slots per direction (in stage_in / stage_out), upload and download
  // streams, per-slot events
  cudaStream_t st_h2d = nullptr, st_d2h = nullptr;
  cudaEvent_t ev_in_ready[2] = {nullptr, nullptr}, ev_in_free[2] = {nullptr, nullptr};
  cudaEvent_t ev_out_ready[2] = {nullptr, nullptr}, ev_out_free[2] = {nullptr, nullptr};
  Launch launch{};
  bool tuned = false;
  int64_t tuned_rhs = 0;  // batch size c.launch was picked for
  bool pinned = false;    // launch shapes forced by the caller (set_tiles / set_schedule)
  cudaStream_t stream = nullptr;
  // the kx-chunk pipeline of the matvec (matvec.cuh): z-pass and inverse-y
  // streams and their events, made with the operator so that no apply or
  // stream capture creates any
  cudaStream_t pipe_st[2] = {nullptr, nullptr};
  cudaEvent_t pipe_ev_y[kMaxKxChunks] = {}, pipe_ev_z[kMaxKxChunks] = {};
  cudaEvent_t pipe_join = nullptr;
  // x/y slab buffer of the slab pieces of a slab-decomposed matvec (sized
  // for the caller's z slabs, not the whole volume; gila_opr_slab_*)
  void* slab_a = nullptr;
  int64_t slab_a_cap = 0;
  std::mutex mu;
  // a solve batch kept resident between gila_ls_solve calls (opts->keep)
  std::shared_ptr<LsBatch> ls_keep;
  std::string ls_keep_key;
  std::weak_ptr<Core> ls_keep_inner;  // the ComplexF32 operator the kept batch uses
  ~Core();
};

struct Ctx {
  int device = 0;
  std::mutex mu;
  std::map<std::pair<int, int>, void*> tw_cache;  // (P, dtype) -> table
  std::map<std::string, Launch> tune_cache;
  ~Ctx();
};

size_t csize(gila_dtype t);
Launch default_launch(const Core& c);
// GPU FP64 Fourier-kernel build into c.ker (kerbuild.cu)
gila_status build_kernel(Core& c);
gila_status ensure_work(Core& c, int64_t nrhs);
void release_work(Core& c);  // frees the matvec workspaces (allocated again on demand)
// launch shapes: cached per context, else timed (autotune) at first use
gila_status ensure_tuned(Core& c, int64_t nrhs);
gila_status autotune(Core& c, int64_t nrhs);
// launch shapes for nrhs vectors laid out for g: the context's cached choice,
// else timed on the caller's buffers (din finite and read only, dout
// overwritten, workspaces A and B) on stream s and cached; c.launch unchanged
template <typename C>
gila_status tuned_launch(Core& c, const Geom& g, int64_t nrhs, const C* din, C* dout, C* A, C* B, cudaStream_t s,
                         Launch& L);
int64_t in_elems(const Core& c);
int64_t out_elems(const Core& c);
bool is_device_ptr(const void* p);
gila_status init_core(gila_ctx* ctx, const gila_vol* trg_abi, const gila_vol* src_abi, const gila_kopt* opt,
                      gila_dtype dtype, std::shared_ptr<Core>& core);

template <typename C>
inline DevOp<C> devop(const Core& c) {
  DevOp<C> d;
  d.ker = static_cast<const C*>(c.ker);
  for (int k = 0; k < 3; ++k) {
    d.map[k] = c.maps[k];
    d.tw[k] = static_cast<const C*>(c.tw[k]);
    d.plan[k] = c.plan[k];
    d.plan_d[k] = c.plan_d + k;
  }
  d.scale = 1.0 / ((double)c.geom.P[0] * c.geom.P[1] * c.geom.P[2]);
  d.pst[0] = c.pipe_st[0];
  d.pst[1] = c.pipe_st[1];
  for (int k = 0; k < kMaxKxChunks; ++k) {
    d.pev_y[k] = c.pipe_ev_y[k];
    d.pev_z[k] = c.pipe_ev_z[k];
  }
  d.pjoin = c.pipe_join;
  return d;
}
gila_status plan_axis(int P, AxisPlan* pl);
gila_status twiddle_table(Ctx* ctx, int P, gila_dtype dt, const void** out);

}  // namespace gila

struct gila_ctx {
  gila::Ctx* impl;
};

struct gila_opr {
  gila_ctx* ctx;
  std::shared_ptr<gila::Core> core;
  gila::Vol trg, src;  // as reported by glaSze (swapped for the adjoint)
  int adj;
};
