// solver.h -- batched Lippmann-Schwinger solves with one right-hand side per
// slot (solver.cu), shared by the synchronous entry point gila_ls_solve and
// the request server (server.cu).
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

#include "internal.h"

namespace gila {

// per right-hand side stopping rules
// cycles between two reliable updates triggered by the residual drop delta
// (at 8 instead of 3 the 64-dipole batch on 96^3 took 10 instead of 28
// update events and 1.77 instead of 1.82 s; the 256x256x128 film, whose
// residual drops by delta every few tens of cycles, is unaffected)
constexpr int kReliableGap = 8;

struct SlotOpts {
  double tol = 1e-6;     // FP64 relative residual target
  double delta = 0.1;    // mixed: recursive-residual drop that triggers a reliable update
  int max_mv = 4000;     // Krylov operator applications
  int max_restarts = 20; // Krylov (re)starts
  int x0 = 0;            // x_out holds an initial guess
};

// per batch structure (fixed for the batch's lifetime)
struct BatchCfg {
  int ell = 2;         // BiCGStab(l) degree
  int mixed = 0;       // Krylov process on the ComplexF32 operator
  int graph = 1;       // replay cycles from captured CUDA graphs
  int chi_shared = 0;  // one medium for all slots (set_shared_chi)
  int priority = 0;    // CUDA stream priority of the batch's stream (lower = more urgent)
  int tune = 0;        // time the launch shapes for the batch's own right-hand-side counts
};

struct SlotResult {
  int slot;
  uint64_t tag;
  double rel_res;  // final FP64 relative residual
  int converged;
  int cycles;      // BiCGStab(l) cycles this right-hand side took part in
  int updates;     // FP64 reliable updates
  int broke;       // a breakdown occurred
};

// A set of slots on one operator pair.  Every call is made from one host
// thread.  The state machine alternates between enqueueing one step (a
// Krylov cycle for every iterating slot, a reliable update, or the start of
// newly assigned slots) on the batch's stream and digesting the step's
// results once it completed; slots are assigned and released at those step
// boundaries, so new right-hand sides join a running batch.
class LsBatch {
 public:
  virtual ~LsBatch() {}
  virtual int slots() const = 0;
  virtual int free_slot() const = 0;   // -1 when none is free
  virtual int busy_slots() const = 0;  // assigned and not yet released
  // chi: V complex128 (ignored when the medium is shared); b: n complex128;
  // x_out: n complex128 receiving the solution (read as initial guess when
  // o.x0).  Host or device pointers; they must stay valid until the slot is
  // reported finished.
  virtual gila_status assign(int slot, const void* chi, const void* b, void* x_out, const SlotOpts& o,
                             uint64_t tag) = 0;
  virtual gila_status set_shared_chi(const void* chi) = 0;
  // Digest the completed step and enqueue the next; *enqueued = false when
  // nothing is left to do.  Call only when no step is in flight.
  virtual gila_status advance(bool* enqueued) = 0;
  virtual bool in_flight() const = 0;
  virtual bool ready() = 0;        // the step in flight completed (non-blocking)
  virtual gila_status wait() = 0;  // block until it completes
  virtual std::vector<SlotResult> take_finished() = 0;
  virtual const gila_solve_info& info() const = 0;
  virtual void reset_info() = 0;
  virtual cudaStream_t stream() const = 0;
};

// device bytes of a batch of `slots` slots
size_t ls_batch_bytes(const Core& g64, const Core* g32, int slots, const BatchCfg& cfg);
// g64: ComplexF64 self operator; g32: its ComplexF32 copy (mixed) or null
gila_status make_ls_batch(Core& g64, Core* g32, int slots, const BatchCfg& cfg, std::unique_ptr<LsBatch>& out);
bool same_volume(const Core& a, const Core& b);
// a copy of operator c in another precision (kernel cast on the device)
gila_status cast_core(gila_ctx* ctx, Core& c, gila_dtype dtype, std::shared_ptr<Core>& out);
gila_status check_ls_operator(const Core& a);
// GILA_ERR_NAN when any of n_complex complex doubles at p (host or device
// memory) is NaN or Inf; `what` names the input in the message
gila_status check_finite(const void* p, int64_t n_complex, const char* what);

}  // namespace gila
