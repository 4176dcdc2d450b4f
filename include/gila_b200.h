/*
 * gila_b200.h -- C ABI of libgila_b200, a B200 (sm_100a) implementation of the
 * discrete 3-D electromagnetic Green-operator matvec of GilaElectromagnetics.jl
 * (v1.0.3) and of the Fourier-kernel build it consumes.
 *
 * Every entry point below replaces one piece of the reference's Julia API; the
 * reference file:line of that piece is cited beside it.  A Julia shim
 * (gilaelectromagnetics.jl_b200/julia/GilaB200.jl) keeps the reference
 * signatures (GlaOprMem, GlaOpr, egoOpr!, mul!, *, adjoint, glaSze, size,
 * eltype, isadjoint, isselfoperator, isexternaloperator) and swaps their
 * bodies for ccalls into this library.
 *
 * Conventions
 *  - Vectors are (Nx, Ny, Nz, 3[, nrhs]) column-major (x fastest), complex
 *    interleaved (re, im): double2 for GILA_C128 (ComplexF64), float2 for
 *    GILA_C64 (ComplexF32).  Multi-RHS batches are contiguous, one vector after
 *    the other.
 *  - Pointers may be host or device memory; the library tells them apart with
 *    cudaPointerGetAttributes.  Host buffers are copied through device
 *    staging buffers (page-locked host buffers let the copies overlap).
 *  - No call aborts; every call returns a gila_status.  gila_last_error()
 *    returns a message for the last failure on the calling thread.
 *  - Calls that take a `stream` (a cudaStream_t; NULL = the operator's own
 *    stream) enqueue work and, for host pointers or stream == NULL, wait for
 *    it before returning.
 */
#ifndef GILA_B200_H
#define GILA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GILA_OK = 0,
  GILA_ERR_ARG = 1,       /* invalid argument / unsupported option          */
  GILA_ERR_SIZE = 2,      /* egoOpr! size check (src/glaAct.jl:37-45)       */
  GILA_ERR_TYPE = 3,      /* element type mismatch (src/glaLinAlg.jl:35)    */
  GILA_ERR_CUDA = 4,      /* CUDA runtime error                              */
  GILA_ERR_NOMEM = 5,     /* device / host allocation failed                 */
  GILA_ERR_NAN = 6,       /* non-numeric kernel (src/glaMemSup.jl:93,110,160)*/
  GILA_ERR_NODEV = 7,     /* no usable CUDA device (src/glaMemSup.jl:22-24)  */
  GILA_ERR_OVERLAP = 8,   /* overlapping volumes (src/glaGen.jl:77-79)       */
  GILA_ERR_SCALE = 9,     /* no common scale grid (src/glaMem.jl:192-209)    */
  GILA_ERR_NOTCONV = 10,  /* iterative solve hit its iteration cap           */
  GILA_ERR_TIMEOUT = 11,  /* a bounded device-side wait ran out              */
  GILA_ERR_INTERNAL = 12
} gila_status;

typedef enum {
  GILA_C64 = 0,  /* ComplexF32 */
  GILA_C128 = 1  /* ComplexF64 */
} gila_dtype;

/* GlaVol (src/glaMem.jl:12-19, constructor :136-148).  Rationals are
 * num/den pairs.  grd = cell pitch (equals scl unless partitioned). */
typedef struct {
  int64_t cel[3];
  int64_t scl_num[3], scl_den[3];
  int64_t org_num[3], org_den[3];
  int64_t grd_num[3], grd_den[3];
} gila_vol;

/* GlaKerOpt (src/glaMem.jl:62-70, defaults :226-233).  num_trd / num_blk are
 * accepted for ABI compatibility and ignored: launch shapes are chosen by the
 * library's autotuner. */
typedef struct {
  double frq_re, frq_im; /* frqPhz */
  int32_t int_ord;       /* intOrd, Gauss-Legendre order of singular terms */
  int32_t adj_mod;       /* adjMod */
  int32_t dev_mod;       /* devMod (must be 1: this library is the device path) */
  int32_t num_trd[3];
  int32_t num_blk[3];
} gila_kopt;

typedef struct gila_ctx gila_ctx;
typedef struct gila_opr gila_opr;

/* ---- context --------------------------------------------------------- */
/* One context per device: streams, twiddle tables, autotune cache.  Replaces
 * the CUDA.functional() gate of GlaOprMem (src/glaMemSup.jl:22-24). */
gila_status gila_ctx_create(int device, gila_ctx** out);
gila_status gila_ctx_destroy(gila_ctx* ctx);
const char* gila_last_error(void);
const char* gila_status_string(gila_status s);
/* Library version, e.g. "0.1.0". */
const char* gila_version(void);

/* ---- operator construction -------------------------------------------- */
/* GlaOprMem(cmpInf, trgVol, srcVol=nothing; setTyp) with egoFur == nothing
 * (src/glaMemSup.jl:16-171): builds the real-space circulant on the GPU in
 * FP64 (src/glaGen.jl, src/glaInt.jl, src/glaIntSup.jl), FFTs it in FP64,
 * extracts the 8 parity branches, casts to dtype.  src == NULL (or src equal
 * to trg) gives the self operator. */
gila_status gila_opr_create(gila_ctx* ctx, const gila_vol* trg, const gila_vol* src,
                            const gila_kopt* opt, gila_dtype dtype, gila_opr** out);

/* GlaOprMem(...; egoFur = fur) (src/glaMemSup.jl:16-20, :158-171): accept the
 * reference's egoFur layout.  fur[eo] (eo = 4*px + 2*py + pz) is a
 * (tx, ty, tz, 6, parSrc, parTrg) column-major complex array of fur_dtype,
 * component order (xx, yy, zz, xy, xz, yz), frequency 2k+p on each axis.
 * fur_dims[eo] gives its 6 extents.  Pointers may be host or device. */
gila_status gila_opr_create_from_fur(gila_ctx* ctx, const gila_vol* trg, const gila_vol* src,
                                     const gila_kopt* opt, gila_dtype dtype,
                                     const void* const fur[8], const int64_t fur_dims[8][6],
                                     gila_dtype fur_dtype, gila_opr** out);

/* Copy the operator's egoFur back out in the reference layout (host
 * pointers, each sized per gila_opr_fur_dims), in the operator's dtype. */
gila_status gila_opr_fur_dims(const gila_opr* opr, int64_t dims[8][6]);
gila_status gila_opr_export_fur(gila_opr* opr, void* const host_out[8]);

/* Kernel cache on disk.  The reference keeps egoFur between sessions with
 * Serialization files in a Scratch space (test/runtests.jl:38-98) or JLD2
 * files keyed by element type, cells and scale (examples/GilaOperators.jl:
 * 28-55); both are Julia-only formats.  gila_opr_save writes the operator's
 * egoFur (in the reference layout, the operator's dtype) with its volumes
 * and GlaKerOpt to one little-endian file, "GILAFUR1":
 *   0 "GILAFUR1" | 8 int32 version 1 | 12 int32 dtype (gila_dtype)
 *   16 int32 self | 20 int32 adjMod | 24 int32 intOrd | 28 int32 0
 *   32 double frqPhz re | 40 double frqPhz im
 *   48 int64[21] target gila_vol | 216 int64[21] source gila_vol
 *      (cel[3], scl_num[3], scl_den[3], org_num[3], org_den[3],
 *       grd_num[3], grd_den[3])
 *   384 int64[8][6] extents of fur[eo]: (tx, ty, tz, 6, parSrc, parTrg)
 *   768 fur[0] .. fur[7]: column-major complex arrays, (re, im) interleaved.
 * Volumes are stored after GlaOprMem's even-cell regeneration; an adjoint
 * handle saves the operator it shares.  gila_opr_load reads such a file and
 * creates the operator as gila_opr_create_from_fur would, casting the kernel
 * to `dtype`.  julia/GilaB200.jl reads and writes the same format in plain
 * Julia, so a cache moves between this library and the reference package. */
gila_status gila_opr_save(gila_opr* opr, const char* path);
gila_status gila_opr_load(gila_ctx* ctx, const char* path, gila_dtype dtype, gila_opr** out);

/* wekS / wekE / wekV (src/glaInt.jl:75-262), the weakly singular self, edge
 * and vertex face-pair integrals of a cell of size scl at Gauss-Legendre
 * order int_ord, evaluated on the GPU by the kernels the operator build uses;
 * the reference's quadrature-convergence check (test/intConTest.jl:6-35)
 * calls them directly.  out: 18 complex values as (re, im) pairs, unscaled:
 * wS[3], wE[9], wV[6]. */
gila_status gila_weak_integrals(gila_ctx* ctx, const int64_t scl_num[3], const int64_t scl_den[3], double frq_re,
                                double frq_im, int32_t int_ord, double out[36]);

/* adjoint(opr) (src/glaLinAlg.jl:16-29): a new handle that shares the
 * operator's device memory, with adjMod flipped and the volumes swapped.  As
 * in the reference, the matvec itself ignores adjMod. */
gila_status gila_opr_adjoint(gila_opr* opr, gila_opr** out);
gila_status gila_opr_destroy(gila_opr* opr);

/* ---- queries ---------------------------------------------------------- */
/* glaSze (src/glaMemSup.jl:359-371): trg = (trgVol.cel..., 3),
 * src = (srcVol.cel..., 3). */
gila_status gila_opr_sizes(const gila_opr* opr, int64_t trg[4], int64_t src[4]);
/* Input size egoOpr! accepts: (mixInf.srcCel..., 3) (src/glaAct.jl:37). */
gila_status gila_opr_input_size(const gila_opr* opr, int64_t in[4]);
gila_status gila_opr_output_size(const gila_opr* opr, int64_t out[4]);
/* flags: bit0 self operator, bit1 adjMod. */
gila_status gila_opr_info(const gila_opr* opr, gila_dtype* dtype, int32_t* flags);

/* ---- the hot path ------------------------------------------------------ */
/* egoOpr!(egoMem, actVec) (src/glaAct.jl:33-49) for nrhs vectors at once:
 * out = G * in.  `in` is not modified (the reference consumes its input;
 * callers must not rely on either behaviour).  in_len / out_len are element
 * counts (complex) of the buffers and are checked against the operator's
 * input and output sizes times nrhs (GILA_ERR_SIZE, as egoOpr!'s error).
 * `dtype` must match the operator (GILA_ERR_TYPE, as the eltype assertion of
 * src/glaLinAlg.jl:35).  Vectors may be in device or host memory; the call
 * returns when a host `out` holds the result.  With nrhs > 1 and a vector in
 * host memory the vectors go through the device one at a time, the upload of
 * the next and the download of the previous overlapping the passes of the
 * current one (pinned host memory lets both copy directions run at once). */
gila_status gila_opr_apply(gila_opr* opr, gila_dtype dtype, const void* in, int64_t in_len,
                           void* out, int64_t out_len, int64_t nrhs, void* stream);

/* LinearAlgebra.mul!(out, G, in, alpha, beta) (src/glaLinAlg.jl:61-69):
 * out = alpha * (G * in) + beta * out, with the axpby fused into the last
 * pass.  alpha/beta are (re, im) pairs. */
gila_status gila_opr_apply_axpby(gila_opr* opr, gila_dtype dtype, const double alpha[2],
                                 const void* in, int64_t in_len, const double beta[2],
                                 void* out, int64_t out_len, int64_t nrhs, void* stream);

/* Pre-size the operator's workspaces for nrhs vectors (so a later apply
 * allocates nothing) and pick launch shapes with the autotuner. */
gila_status gila_opr_reserve(gila_opr* opr, int64_t nrhs);

/* Device bytes the operator holds (kernel + workspaces). */
gila_status gila_opr_device_bytes(const gila_opr* opr, int64_t* bytes);

/* Profiling (no counterpart in the reference, which has no timers beyond
 * @time in the examples): device time of one apply on nrhs device-resident
 * vectors, averaged over `reps`, measured with CUDA events on the operator's
 * stream.  ms[0] = forward x/y passes, ms[1] = z pass (FFT, 3x3 multiply,
 * inverse FFT), ms[2] = inverse y/x passes, ms[3] = whole apply. */
gila_status gila_opr_time_passes(gila_opr* opr, int64_t nrhs, int reps, double ms[4]);

/* Launch shapes.  tiles = {x-forward lines per CTA, x-inverse lines per CTA,
 * y-pass kx tile, z-pass kx tile}.  No counterpart in the reference.  The
 * first apply of an operator picks the y and z tiles (with the radix order of
 * the x and y transforms, gila_opr_get_schedule, and the task form of the
 * fused z pass: one task per frequency or per mirror pair) by timing every compiled
 * candidate on the operator's workspaces (cached per context and geometry;
 * GILA_AUTOTUNE=0 keeps the defaults).  An apply with another number of
 * device-resident vectors re-times the tiles and the task form for that
 * count and keeps the radix order.  gila_opr_autotune re-runs the timing for
 * a batch of nrhs vectors; gila_opr_set_tiles forces tiles (entries <= 0 or
 * not compiled for the transform length are ignored) for every batch size.
 * Tiles never change results, only speed. */
gila_status gila_opr_autotune(gila_opr* opr, int64_t nrhs, int32_t tiles[4]);
gila_status gila_opr_get_tiles(gila_opr* opr, int32_t tiles[4]);
gila_status gila_opr_set_tiles(gila_opr* opr, const int32_t tiles[4]);

/* Radix order of the x and y transforms at the specialised lengths (no
 * counterpart in the reference, whose FFTs are FFTW / CUFFT plans): sched =
 * {x, y}, 0 = the greedy order (radix-8 stages first), 1 = its reverse.  Both
 * compute the same transform; results differ by rounding only.  The autotuner
 * picks them together with the tiles; set forces them (entries < 0 keep the
 * current value). */
gila_status gila_opr_get_schedule(gila_opr* opr, int32_t sched[2]);
gila_status gila_opr_set_schedule(gila_opr* opr, const int32_t sched[2]);

/* Number of kernels one apply of nrhs vectors launches. */
gila_status gila_opr_launches_per_apply(const gila_opr* opr, int64_t nrhs, int64_t* n);

/* ---- the scattering solve (examples/GilaOperators.jl:57-96) ------------ */
/* A copy of the operator in another precision (kernel cast on the device),
 * sharing nothing with the original.  Used to pair a ComplexF64 operator with
 * the ComplexF32 one of the mixed-precision solve. */
gila_status gila_opr_cast(gila_opr* opr, gila_dtype dtype, gila_opr** out);

typedef struct {
  double tol;           /* target FP64 relative residual ||b - A x|| / ||b||; <= 0 -> 1e-6 */
  int32_t ell;          /* BiCGStab(l) degree 1..4; 0 -> 2 (IterativeSolvers.bicgstabl's default) */
  int32_t mixed;        /* 0: FP64 Krylov process; 1: the Krylov process runs on the ComplexF32
                           operator and FP64 reliable updates (FP64 solution, residual replaced
                           by the FP64 b - A x) keep the result at FP64 accuracy */
  int32_t max_matvecs;  /* cap on Krylov operator applications; 0 -> 4000 */
  int32_t max_restarts; /* cap on Krylov (re)starts per right-hand side (breakdowns, convergence
                           the FP64 residual does not confirm); 0 -> 20 */
  double delta;         /* mixed: a reliable update follows a cycle whose recursive residual fell
                           below delta times its largest value since the last update, at least
                           8 cycles after that update; <= 0 -> 0.1 */
  int32_t x0;           /* 1: x holds an initial guess on entry; 0: start from zero (as
                           IterativeSolvers.bicgstabl(A, b) does) */
  int32_t no_graph;     /* 1: launch every Krylov cycle's kernels directly instead of replaying
                           one captured CUDA graph per cycle */
  int32_t keep;         /* 1: keep the solve's device state (Krylov vectors, workspaces, captured
                           graphs) with the operator for the next call with the same operators,
                           nrhs and structure (freed with the operator) */
} gila_solve_opts;

typedef struct {
  int32_t iters;        /* BiCGStab(l) cycles of the batch (2l matvecs each) */
  int32_t outer;        /* FP64 residual evaluations (reliable updates) */
  int32_t matvecs_f64;  /* batched FP64 operator applications */
  int32_t matvecs_f32;  /* batched ComplexF32 operator applications */
  double rel_res;       /* max over right-hand sides of the final FP64 relative residual */
  int32_t converged;    /* right-hand sides that reached tol */
  int32_t breakdowns;   /* right-hand sides whose Krylov recurrence broke down at least once */
} gila_solve_info;

/* Solve (I - chi G) x = b for nrhs right-hand sides at once: the
 * LippmannSchwinger operator of examples/GilaOperators.jl:89-96 (chi per
 * cell, broadcast over the 3 components) and its `solve`
 * (examples/scattering_film.jl:58-61, IterativeSolvers.bicgstabl) with
 * BiCGStab(l).  g64 is a ComplexF64 self operator; g32 a ComplexF32 operator
 * of the same volume (gila_opr_cast), required when opts->mixed.  chi:
 * (Nx,Ny,Nz) complex128; b, x: (Nx,Ny,Nz,3,nrhs) complex128, host or device
 * pointers.  opts may be NULL (defaults); info and rhs_res (nrhs final FP64
 * relative residuals) may be NULL.  Returns GILA_ERR_NOTCONV, with x holding
 * the last iterate, when a right-hand side missed the tolerance. */
gila_status gila_ls_solve(gila_opr* g64, gila_opr* g32, const void* chi, const void* b, void* x, int64_t nrhs,
                          const gila_solve_opts* opts, gila_solve_info* info, double* rhs_res, void* stream);

/* ---- the solve server: continuous batching of scattering solves -------- */
/* No counterpart in the reference (its solves are single blocking calls).
 * A server owns one scheduler thread per context.  Requests (a self volume,
 * its medium chi and incident field b) are queued on submit; the scheduler
 * keeps one batch of right-hand-side slots per volume shape on its own CUDA
 * stream, with the shape's ComplexF64 and ComplexF32 operators (built on the
 * GPU and cached) and all Krylov vectors resident in HBM.  A request joins
 * its shape's running batch at the next Krylov-cycle boundary as soon as a
 * slot is free and the HBM budget admits the batch; batches of different
 * shapes run concurrently on their streams.  Each right-hand side's result
 * does not depend on what else is batched with it. */
typedef struct gila_server gila_server;

typedef struct {
  int64_t hbm_budget;      /* device bytes for operators and batches; 0 -> free memory at
                              creation minus 4 GiB */
  int32_t slots;           /* right-hand-side slots of a shape's batch; 0 -> 8 */
  int32_t ell;             /* BiCGStab(l) degree of every solve; 0 -> 2 */
  int32_t mixed;           /* ComplexF32 Krylov process with FP64 reliable updates */
  int32_t int_ord;         /* GlaKerOpt intOrd of the operators built; 0 -> 32 */
  double frq_re, frq_im;   /* GlaKerOpt frqPhz; 0 + 0i -> 1 + 0i */
} gila_server_opts;

typedef struct {
  int64_t submitted, completed, queued, running;
  int64_t batches;         /* shape batches allocated */
  int64_t operators;       /* shapes whose operators are cached */
  int64_t bytes_in_use;    /* operators + batches, device bytes */
  int64_t hbm_budget;
} gila_server_stats;

gila_status gila_server_create(gila_ctx* ctx, const gila_server_opts* opts, gila_server** out);
gila_status gila_server_destroy(gila_server* srv);
/* vol: a self volume (cells, scale; origin ignored); chi: (Nx,Ny,Nz)
 * complex128; b, x: (Nx,Ny,Nz,3) complex128 host or device pointers that
 * stay valid until the request completes (x receives the solution).  opts:
 * tol, max_matvecs, max_restarts, delta of this request (ell / mixed are the
 * server's); NULL for defaults. */
gila_status gila_server_submit(gila_server* srv, const gila_vol* vol, const void* chi, const void* b, void* x,
                               const gila_solve_opts* opts, uint64_t* ticket);
/* Wait for a request (timeout_ms < 0: no limit; GILA_ERR_TIMEOUT when it
 * runs out).  info (may be NULL): that right-hand side's cycles (iters),
 * reliable updates (outer), rel_res, converged; latency_ms (may be NULL):
 * submit to completion on the host clock.  Returns GILA_ERR_NOTCONV when the
 * solve missed its tolerance. */
gila_status gila_server_wait(gila_server* srv, uint64_t ticket, int64_t timeout_ms, gila_solve_info* info,
                             double* latency_ms);
gila_status gila_server_stats_get(gila_server* srv, gila_server_stats* out);

/* Fault injection for tests (no counterpart in the reference): with n >= 1,
 * the n-th device allocation the library makes from now on fails as an
 * out-of-memory would (GILA_ERR_NOMEM), before cudaMalloc is called; n = 0
 * disarms.  Process-wide. */
gila_status gila_debug_fail_alloc(int64_t n);

/* Slab pieces of a matvec split over several GPUs (no counterpart in the
 * reference, which runs a volume on one device: src/glaAct.jl:191-321).  One
 * process per GPU holds the operator (the whole Fourier kernel); rank r
 * keeps source z planes [zs_r, zs_r + nzs_r) of the input, target z planes
 * [zt_r, zt_r + nzt_r) of the output and spectrum rows [ky_r, ky_r + nky_r)
 * between the passes.  A matvec is slab_fwd on the rank's source planes, an
 * all-to-all that gives every rank all source planes of its rows, slab_z on
 * its rows, an all-to-all that gives every rank all rows of its target
 * planes, and slab_inv on its target planes; the exchanges are the caller's
 * (gila_b200.SlabOpr uses NCCL through torch.distributed).  The pieces run
 * the per-line arithmetic of gila_opr_apply with the operator's launch
 * choices (its defaults until it is applied or autotuned), so the result
 * equals the single-GPU matvec bit for bit.  Operators with one source and
 * one target partition; every pointer is device memory on the operator's
 * GPU; pieces of one operator must be ordered (one stream): they share an
 * x/y buffer.  stream == NULL runs on the operator's stream and waits.
 *
 * dims: Px, Py, Pz (padded transform lengths), nin (source z planes), nout
 * (target z planes). */
gila_status gila_opr_slab_dims(const gila_opr* opr, int64_t dims[5]);
/* in: nz source planes, (srcCelX, srcCelY, nz, 3) column-major; bslab: 3 *
 * nz planes of Py x Px (component-major, then z, then ky, kx fastest)
 * receiving each plane's 2-D spectrum. */
gila_status gila_opr_slab_fwd(gila_opr* opr, gila_dtype dtype, const void* in, int64_t nz, void* bslab,
                              void* stream);
/* bz: spectrum rows ky0 .. ky0 + nky - 1 of every z plane, planes of nky x
 * Px; on entry component c's nin source planes start at c * nin planes, on
 * return its nout target planes start at c * nout planes (3 * max(nin,
 * nout) planes of room). */
gila_status gila_opr_slab_z(gila_opr* opr, gila_dtype dtype, void* bz, int64_t ky0, int64_t nky, void* stream);
/* bslab: 3 * nz target planes of Py x Px (component-major); out: nz target
 * planes, (trgCelX, trgCelY, nz, 3) column-major. */
gila_status gila_opr_slab_inv(gila_opr* opr, gila_dtype dtype, const void* bslab, int64_t nz, void* out,
                              void* stream);

/* A matvec that allocates no device memory.  This entry point has no
 * counterpart in the reference.  It computes out = G * in for one vector,
 * like gila_opr_apply, for callers that cannot let the library call
 * cudaMalloc at apply time: hosts whose own memory pool owns all device
 * memory (a foreign cudaMalloc there fails or takes memory the pool has
 * promised elsewhere), and loops that forbid allocation after start-up
 * (cudaMalloc can synchronise the device and take unbounded time).  The
 * scratch between the passes lives in one fixed 64 MiB device array that
 * every GPU loading the library holds until the process exits; operators
 * whose padded spectrum plus one x/y plane do not fit are rejected with
 * GILA_ERR_SIZE.  `in` and `out` must be device pointers on the operator's
 * GPU (host vectors would need staging buffers).  The first call on a device
 * looks up the array's device address and keeps it; make that first call
 * before any stream capture, and note that the kept address, like the
 * operators' own device memory, does not survive cudaDeviceReset.  All calls
 * on a device share the array, which keeps the last call's contents, and
 * calls that overlap on the GPU race on it.  stream == NULL runs on the
 * operator's stream and waits. */
gila_status gila_opr_apply_noalloc(gila_opr* opr, gila_dtype dtype, const void* in, int64_t in_len,
                                   void* out, int64_t out_len, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GILA_B200_H */
