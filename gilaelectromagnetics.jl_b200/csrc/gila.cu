// gila.cu -- C ABI of libgila_b200: contexts, operators, the matvec entry
// points.  Construction mirrors GlaOprMem / GlaOprPrp (src/glaMemSup.jl:16-269),
// the apply mirrors egoOpr! (src/glaAct.jl:33-49) and mul! (src/glaLinAlg.jl).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace gila {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }
gila_status fail(gila_status s, const std::string& msg) {
  g_err = msg;
  return s;
}
gila_status cuda_fail(cudaError_t e, const char* where) {
  g_err = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") at " + where;
  if (e == cudaErrorMemoryAllocation) return GILA_ERR_NOMEM;
  return GILA_ERR_CUDA;
}

size_t csize(gila_dtype t) { return t == GILA_C128 ? 16 : 8; }

// Fault injection for tests: when armed with n >= 1, the n-th device
// allocation from then on fails as an out-of-memory would, before cudaMalloc
// is called, and the countdown disarms.
static std::atomic<int64_t> g_fail_alloc{0};

cudaError_t dev_malloc_raw(void** p, size_t bytes) {
  *p = nullptr;
  int64_t n = g_fail_alloc.load();
  while (n > 0) {
    if (g_fail_alloc.compare_exchange_weak(n, n - 1)) {
      if (n == 1) return cudaErrorMemoryAllocation;
      break;
    }
  }
  return cudaMalloc(p, bytes);
}

// ------------------------------------------------------------- rationals
static int64_t gcd64(int64_t a, int64_t b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}
Rat rat(int64_t n, int64_t d) {
  if (d < 0) {
    n = -n;
    d = -d;
  }
  int64_t g = gcd64(n, d);
  if (g == 0) g = 1;
  return Rat{n / g, d / g};
}
bool rat_eq(Rat a, Rat b) { return a.n == b.n && a.d == b.d; }
static Rat rdiv(Rat a, Rat b) { return rat(a.n * b.d, a.d * b.n); }
static bool risint(Rat a) { return a.d == 1; }

Vol vol_from_abi(const gila_vol& v) {
  Vol o;
  for (int k = 0; k < 3; ++k) {
    o.cel[k] = v.cel[k];
    o.scl[k] = rat(v.scl_num[k], v.scl_den[k]);
    o.org[k] = rat(v.org_num[k], v.org_den[k]);
    if (v.grd_den[k] == 0)
      o.grd[k] = o.scl[k];
    else
      o.grd[k] = rat(v.grd_num[k], v.grd_den[k]);
  }
  return o;
}
gila_vol vol_to_abi(const Vol& v) {
  gila_vol o;
  for (int k = 0; k < 3; ++k) {
    o.cel[k] = v.cel[k];
    o.scl_num[k] = v.scl[k].n;
    o.scl_den[k] = v.scl[k].d;
    o.org_num[k] = v.org[k].n;
    o.org_den[k] = v.org[k].d;
    o.grd_num[k] = v.grd[k].n;
    o.grd_den[k] = v.grd[k].d;
  }
  return o;
}
bool vol_eq(const Vol& a, const Vol& b) {
  for (int k = 0; k < 3; ++k)
    if (a.cel[k] != b.cel[k] || !rat_eq(a.scl[k], b.scl[k]) || !rat_eq(a.org[k], b.org[k]) ||
        !rat_eq(a.grd[k], b.grd[k]))
      return false;
  return true;
}

// glaVolEveGen (src/glaMem.jl:152-175)
Vol vol_even(const Vol& v) {
  bool all_even = true;
  for (int k = 0; k < 3; ++k) all_even &= (v.cel[k] % 2 == 0);
  if (all_even) return v;
  Vol o = v;
  for (int k = 0; k < 3; ++k) {
    const int64_t par = v.cel[k] % 2;
    const int64_t nc = v.cel[k] + par;
    o.cel[k] = nc;
    o.scl[k] = rat(v.scl[k].n * v.cel[k], v.scl[k].d * nc);
    o.grd[k] = rat(v.grd[k].n * v.cel[k], v.grd[k].d * nc);
  }
  return o;
}

// GlaExtInf constructor (src/glaMem.jl:190-216)
gila_status ext_inf(const Vol& trg, const Vol& src, ExtInf* out) {
  int64_t ok = 1;
  for (int k = 0; k < 3; ++k) ok *= (int)risint(rdiv(src.scl[k], trg.scl[k])) + (int)risint(rdiv(trg.scl[k], src.scl[k]));
  if (ok == 0) return fail(GILA_ERR_SCALE, "Volume pair must share a common scale grid.");
  for (int k = 0; k < 3; ++k) {
    const Rat a = src.scl[k], b = trg.scl[k];
    const int64_t gn = gcd64(a.n, b.n), ld = a.d / gcd64(a.d, b.d) * b.d;
    out->min_scl[k] = rat(gn, ld);
    const int64_t ln = a.n / gcd64(a.n, b.n) * b.n, gd = gcd64(a.d, b.d);
    const Rat mx = rat(ln, gd);
    const Rat td = rdiv(mx, trg.scl[k]), sd = rdiv(mx, src.scl[k]);
    out->tdiv[k] = (int)(td.n / td.d);
    out->sdiv[k] = (int)(sd.n / sd.d);
    out->tc[k] = (int)(trg.cel[k] / out->tdiv[k]);
    out->sc[k] = (int)(src.cel[k] / out->sdiv[k]);
    if (out->tc[k] == 0 || out->sc[k] == 0)
      return fail(GILA_ERR_SCALE, "Volume sizes are incompatible---volume smaller than cell.");
  }
  return GILA_OK;
}

// ------------------------------------------------------------ FFT plans
gila_status plan_axis(int P, AxisPlan* pl) {
  pl->P = P;
  pl->nst = 0;
  int r = P;
  int twos = 0;
  while (r % 2 == 0) {
    r /= 2;
    ++twos;
  }
  while (twos >= 3) {
    pl->radix[pl->nst++] = 8;
    twos -= 3;
  }
  if (twos == 2) pl->radix[pl->nst++] = 4;
  if (twos == 1) pl->radix[pl->nst++] = 2;
  for (int q : {3, 5, 7}) {
    while (r % q == 0) {
      if (pl->nst >= 12) return fail(GILA_ERR_ARG, "axis length has too many factors");
      pl->radix[pl->nst++] = q;
      r /= q;
    }
  }
  if (r != 1)
    return fail(GILA_ERR_ARG, "circulant length " + std::to_string(P) +
                                  " has a prime factor above 7; supported lengths are 2^a 3^b 5^c 7^d");
  if (pl->nst == 0) pl->radix[pl->nst++] = 2;  // P == 1 cannot occur (P even)
  int ns = 1;
  for (int s = 0; s < pl->nst; ++s) {
    StageC& c = pl->st[s];
    c.R = pl->radix[s];
    c.ns = ns;
    c.tpl = P / c.R;
    c.twst = P / (ns * c.R);
    c.nsd = make_fdiv((uint32_t)ns);
    c.tpld = make_fdiv((uint32_t)c.tpl);
    ns *= c.R;
  }
  return GILA_OK;
}

gila_status twiddle_table(Ctx* ctx, int P, gila_dtype dt, const void** out) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto key = std::make_pair(P, (int)dt);
  auto it = ctx->tw_cache.find(key);
  if (it != ctx->tw_cache.end()) {
    *out = it->second;
    return GILA_OK;
  }
  // w_P^m = exp(-2 pi i m / P); angle reduced to the first octant for accuracy
  std::vector<double> re(P), im(P);
  for (int m = 0; m < P; ++m) {
    const long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)P;
    re[m] = (double)cosl(a);
    im[m] = (double)sinl(a);
  }
  void* d = nullptr;
  const size_t bytes = (size_t)P * csize(dt);
  GILA_CUDA_TRY(dev_malloc(&d, bytes));
  if (dt == GILA_C128) {
    std::vector<double2> h(P);
    for (int m = 0; m < P; ++m) h[m] = make_double2(re[m], im[m]);
    GILA_CUDA_TRY(cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice));
  } else {
    std::vector<float2> h(P);
    for (int m = 0; m < P; ++m) h[m] = make_float2((float)re[m], (float)im[m]);
    GILA_CUDA_TRY(cudaMemcpy(d, h.data(), bytes, cudaMemcpyHostToDevice));
  }
  ctx->tw_cache[key] = d;
  *out = d;
  return GILA_OK;
}

Ctx::~Ctx() {
  for (auto& kv : tw_cache) cudaFree(kv.second);
}

Core::~Core() {
  if (device >= 0) cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  cudaFree(ker);
  for (int k = 0; k < 3; ++k) cudaFree(maps[k]);
  cudaFree(plan_d);
  cudaFree(A);
  cudaFree(B);
  cudaFree(stage_in);
  cudaFree(stage_out);
  cudaFree(slab_a);
  for (cudaStream_t x : {st_h2d, st_d2h})
    if (x) {
      cudaStreamSynchronize(x);
      cudaStreamDestroy(x);
    }
  for (int k = 0; k < 2; ++k)
    for (cudaEvent_t x : {ev_in_ready[k], ev_in_free[k], ev_out_ready[k], ev_out_free[k]})
      if (x) cudaEventDestroy(x);
  for (cudaStream_t x : pipe_st)
    if (x) {
      cudaStreamSynchronize(x);
      cudaStreamDestroy(x);
    }
  for (int k = 0; k < kMaxKxChunks; ++k) {
    if (pipe_ev_y[k]) cudaEventDestroy(pipe_ev_y[k]);
    if (pipe_ev_z[k]) cudaEventDestroy(pipe_ev_z[k]);
  }
  if (pipe_join) cudaEventDestroy(pipe_join);
  if (stream) cudaStreamDestroy(stream);
}

// Stored kernel extents (src/glaMemSup.jl:121-136).
static void tru_inf(const Core& c, int tru[3]) {
  for (int d = 0; d < 3; ++d) {
    const int tot = c.mix.tc[d] + c.mix.sc[d];
    const bool one_par = (c.mix.sdiv[0] * c.mix.sdiv[1] * c.mix.sdiv[2] == 1) &&
                         (c.mix.tdiv[0] * c.mix.tdiv[1] * c.mix.tdiv[2] == 1);
    if (c.mix.tc[d] == c.mix.sc[d] && one_par && rat_eq(c.trg.org[d], c.src.org[d])) {
      const int n = c.mix.tc[d];
      const int v = (n + 1) / 2 + (n % 2 == 0 ? 1 : 0);
      tru[d] = v > 2 ? v : 2;
    } else {
      tru[d] = tot / 2;
    }
  }
}

// Per-frequency kernel address on one axis, following the forward / reverse
// quadrants of mulBrnDev! (src/glaActSup.jl:789-846): frequency f = 2k + p
// reads stored index m of branch p, mirrored (sign flip for off-diagonal
// components) in the reverse quadrant.
static std::vector<int> axis_map(int P, int tru, int tcel) {
  const int brn = P / 2;
  std::vector<int> m(P);
  for (int f = 0; f < P; ++f) {
    const int p = f % 2, k = f / 2;
    int idx = k, mir = 0;
    if (tru != brn) {
      const int fwd_even = (tcel + 1) / 2 + (tcel % 2 == 0 ? 1 : 0);
      const int fwd_odd = (tcel + 1) / 2;
      if (p == 0 && k >= fwd_even) {
        idx = brn - k;
        mir = 1;
      } else if (p == 1 && k >= fwd_odd) {
        idx = brn - 1 - k;
        mir = 1;
      }
    }
    m[f] = idx | (p << 29) | (mir << 30);
  }
  return m;
}

gila_status init_core(gila_ctx* ctx, const gila_vol* trg_abi, const gila_vol* src_abi, const gila_kopt* opt,
                             gila_dtype dtype, std::shared_ptr<Core>& core) {
  if (!ctx || !trg_abi) return fail(GILA_ERR_ARG, "null context or target volume");
  if (dtype != GILA_C64 && dtype != GILA_C128) return fail(GILA_ERR_TYPE, "setTyp must be ComplexF32 or ComplexF64");
  core = std::make_shared<Core>();
  core->ctx = ctx->impl;
  core->device = ctx->impl->device;
  core->dtype = dtype;
  if (opt)
    core->opt = *opt;
  else {
    core->opt.frq_re = 1.0;
    core->opt.frq_im = 0.0;
    core->opt.int_ord = 32;
    core->opt.dev_mod = 1;
  }
  Vol trg = vol_from_abi(*trg_abi);
  for (int k = 0; k < 3; ++k)
    if (trg.cel[k] <= 0) return fail(GILA_ERR_ARG, "cell counts must be positive");
  Vol src = src_abi ? vol_from_abi(*src_abi) : trg;
  // self / external detection and even-cell regeneration (src/glaMemSup.jl:26-43)
  if (!src_abi || vol_eq(trg, src)) {
    core->self = true;
    src = trg;
  } else {
    core->self = false;
    int64_t odd = 0;
    for (int k = 0; k < 3; ++k) odd += (trg.cel[k] + src.cel[k]) % 2;
    if (odd != 0) {
      fprintf(stderr,
              "Warning! A volume has been regenerated to have an even number of cells---the size of a cell has "
              "changed. The sum of the number of source and target cells must be even for the algorithm to "
              "function.\n");
      trg = vol_even(trg);
      src = vol_even(src);
    }
  }
  core->trg = trg;
  core->src = src;
  gila_status s = ext_inf(trg, src, &core->mix);
  if (s != GILA_OK) return s;
  core->parS = core->mix.sdiv[0] * core->mix.sdiv[1] * core->mix.sdiv[2];
  Geom& g = core->geom;
  int parT = core->mix.tdiv[0] * core->mix.tdiv[1] * core->mix.tdiv[2];
  if (parT > 64) return fail(GILA_ERR_ARG, "more than 64 target partitions are not supported");
  g.parT = parT;
  g.csize = (int)csize(dtype);
  g.max_rhs = 1;
  // GILA_SLAB_BYTES overrides the x/y slab size (tuning and tests)
  g.slab_bytes = kSlabBytes;
  if (const char* e = getenv("GILA_SLAB_BYTES")) {
    const long v = atol(e);
    if (v > 0) g.slab_bytes = (int)v;
  }
  for (int k = 0; k < 3; ++k) {
    g.sc[k] = core->mix.sc[k];
    g.tc[k] = core->mix.tc[k];
    g.P[k] = g.sc[k] + g.tc[k];
    g.tdiv[k] = core->mix.tdiv[k];
    g.out_full[k] = (int64_t)g.tc[k] * g.tdiv[k];
  }
  int t = 0;
  for (int z = 0; z < g.tdiv[2]; ++z)
    for (int y = 0; y < g.tdiv[1]; ++y)
      for (int x = 0; x < g.tdiv[0]; ++x, ++t) {
        g.toff[t][0] = x;
        g.toff[t][1] = y;
        g.toff[t][2] = z;
      }
  tru_inf(*core, g.tru);
  // the z pass addresses one partition's kernel with 32-bit offsets
  if ((int64_t)48 * g.tru[0] * g.tru[1] * g.tru[2] >= ((int64_t)1 << 31))
    return fail(GILA_ERR_SIZE, "Fourier kernel too large: more than 2^31 stored values per target partition");
  for (int k = 0; k < 3; ++k) {
    if ((s = plan_axis(g.P[k], &core->plan[k])) != GILA_OK) return s;
    if ((s = twiddle_table(ctx->impl, g.P[k], dtype, &core->tw[k])) != GILA_OK) return s;
    std::vector<int> m = axis_map(g.P[k], g.tru[k], g.tc[k]);
    GILA_CUDA_TRY(dev_malloc(&core->maps[k], m.size() * sizeof(int)));
    GILA_CUDA_TRY(cudaMemcpy(core->maps[k], m.data(), m.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  GILA_CUDA_TRY(dev_malloc(&core->plan_d, 3 * sizeof(AxisPlan)));
  GILA_CUDA_TRY(cudaMemcpy(core->plan_d, core->plan, 3 * sizeof(AxisPlan), cudaMemcpyHostToDevice));
  GILA_CUDA_TRY(cudaStreamCreateWithFlags(&core->stream, cudaStreamNonBlocking));
  for (int k = 0; k < 2; ++k) GILA_CUDA_TRY(cudaStreamCreateWithFlags(&core->pipe_st[k], cudaStreamNonBlocking));
  for (int k = 0; k < kMaxKxChunks; ++k) {
    GILA_CUDA_TRY(cudaEventCreateWithFlags(&core->pipe_ev_y[k], cudaEventDisableTiming));
    GILA_CUDA_TRY(cudaEventCreateWithFlags(&core->pipe_ev_z[k], cudaEventDisableTiming));
  }
  GILA_CUDA_TRY(cudaEventCreateWithFlags(&core->pipe_join, cudaEventDisableTiming));
  return GILA_OK;
}

bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Re-layout the reference egoFur (tx,ty,tz,6,parS,parT column-major, one
// array per branch eo) into target-partition blocks laid out by ker_index,
// in the operator dtype.
template <typename CT>
static gila_status load_fur(Core& c, const void* const fur[8], gila_dtype fdt, std::vector<CT>& out) {
  const Geom& g = c.geom;
  const int tx = g.tru[0], ty = g.tru[1], tz = g.tru[2];
  const int64_t per = (int64_t)tx * ty * tz * 6;
  out.assign((size_t)per * 8 * g.parT, CT{});
  const int64_t n_in = per * c.parS * g.parT;
  std::vector<unsigned char> host;
  for (int eo = 0; eo < 8; ++eo) {
    const void* src = fur[eo];
    if (!src) return fail(GILA_ERR_ARG, "null egoFur branch");
    const size_t bytes = (size_t)n_in * csize(fdt);
    const unsigned char* hp;
    if (is_device_ptr(src)) {
      host.resize(bytes);
      GILA_CUDA_TRY(cudaMemcpy(host.data(), src, bytes, cudaMemcpyDeviceToHost));
      hp = host.data();
    } else {
      hp = static_cast<const unsigned char*>(src);
    }
    for (int tp = 0; tp < g.parT; ++tp)
      for (int cc = 0; cc < 6; ++cc)
        for (int iz = 0; iz < tz; ++iz)
          for (int iy = 0; iy < ty; ++iy)
            for (int ix = 0; ix < tx; ++ix) {
              // source partition 0 only (parS > 1 operators cannot be applied)
              const int64_t si = ((((int64_t)tp * c.parS + 0) * 6 + cc) * tz + iz) * ty * (int64_t)tx +
                                 (int64_t)iy * tx + ix;
              double re, im;
              if (fdt == GILA_C128) {
                const double* q = reinterpret_cast<const double*>(hp) + 2 * si;
                re = q[0];
                im = q[1];
              } else {
                const float* q = reinterpret_cast<const float*>(hp) + 2 * si;
                re = q[0];
                im = q[1];
              }
              if (!std::isfinite(re) || !std::isfinite(im))
                return fail(GILA_ERR_NAN, "Fourier information contains non-numeric values.");
              const int64_t di = (int64_t)tp * 8 * per + ker_index(eo, iz, iy, cc, ix, tx, ty, tz);
              out[di].x = (decltype(out[di].x))re;
              out[di].y = (decltype(out[di].y))im;
            }
  }
  return GILA_OK;
}

// Launch shapes: the largest tiles whose thread count stays <= 512 with 8
// staged values per thread and whose shared memory stays within budget.
Launch default_launch(const Core& c) {
  const Geom& g = c.geom;
  const int cs = (int)csize(c.dtype);
  Launch L;
  auto lines = [&](const AxisPlan& pl) {
    int m = 2048 / pl.P;
    if (m < 1) m = 1;
    while (m > 1 && pass_threads(pl, m) > 512) --m;
    return m;
  };
  L.xf_lines = lines(c.plan[0]);
  L.xi_lines = lines(c.plan[0]);
  auto tile = [&](const AxisPlan& pl, int ch, int want, int smem_budget) {
    int tx = want;
    while (tx > 1 && (pass_threads(pl, ch * tx) > 512 || (int64_t)ch * tx * pl.P * cs > smem_budget)) tx /= 2;
    return tx < 1 ? 1 : tx;
  };
  const int want = c.dtype == GILA_C128 ? 8 : 16;
  L.y_tx = tile(c.plan[1], 1, want, 96 * 1024);
  // the z pass runs its FFTs one component at a time (threads for TX lines)
  // but keeps all three components' spectra in shared memory
  {
    int tx = want;
    const int64_t budget = (g.parT > 1 ? 55 : 110) * 1024;
    while (tx > 1 && (pass_threads(c.plan[2], tx) > 512 || 3LL * tx * c.plan[2].P * cs > budget)) tx /= 2;
    L.z_tx = tx < 1 ? 1 : tx;
  }
  return L;
}

gila_status ensure_work(Core& c, int64_t nrhs) {
  if (nrhs <= c.cap_rhs) return GILA_OK;
  c.geom.max_rhs = (int)nrhs;
  const Work w = work_sizes(c.geom);
  const size_t cs = csize(c.dtype);
  cudaFree(c.A);
  cudaFree(c.B);
  c.A = c.B = nullptr;
  c.cap_rhs = 0;
  GILA_CUDA_TRY(dev_malloc(&c.A, (size_t)w.a_elems * cs));
  GILA_CUDA_TRY(dev_malloc(&c.B, (size_t)(w.b_rhs * nrhs) * cs));
  c.cap_rhs = nrhs;
  return GILA_OK;
}

void release_work(Core& c) {
  cudaFree(c.A);
  cudaFree(c.B);
  c.A = c.B = nullptr;
  c.cap_rhs = 0;
}

int64_t in_elems(const Core& c) { return 3LL * c.geom.sc[0] * c.geom.sc[1] * c.geom.sc[2]; }
int64_t out_elems(const Core& c) {
  return 3LL * c.geom.out_full[0] * c.geom.out_full[1] * c.geom.out_full[2];
}

// ------------------------------------------------------------ autotuner
// Tile widths of the y and z passes (kx per CTA) are picked per operator
// geometry, precision and batch size by timing every compiled candidate on
// the operator's own workspaces; results are cached per context.  The tile
// does not change any arithmetic (each line's transform and each point's
// multiply are the same), only the launch shape.
static std::string tune_key(const Core& c, int64_t nrhs) {
  const Geom& g = c.geom;
  char b[256];
  snprintf(b, sizeof b, "%d|%d,%d,%d|%d,%d,%d|%d,%d,%d|%d|%lld", (int)c.dtype, g.P[0], g.P[1], g.P[2], g.sc[0],
           g.sc[1], g.sc[2], g.tc[0], g.tc[1], g.tc[2], g.parT, (long long)nrhs);
  return b;
}

static bool tune_debug() {
  const char* e = getenv("GILA_TUNE_DEBUG");
  return e && e[0] == '1';
}

// Times the candidates for nrhs vectors on the given buffers: din (finite,
// nrhs input vectors, read only), dout (nrhs output vectors, overwritten),
// workspaces A and B laid out for g, all on stream s.
template <typename C>
static gila_status tune_on(Core& c, const Geom& g, int64_t nrhs, const C* din, C* dout, C* A, C* B,
                           cudaStream_t s, Launch& best, const Launch* keep_radix = nullptr) {
  cudaError_t e = cudaSuccess;
  cudaEvent_t ev[2];
  GILA_CUDA_TRY(cudaEventCreate(&ev[0]));
  if ((e = cudaEventCreate(&ev[1])) != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    return cuda_fail(e, "cudaEventCreate");
  }
  const DevOp<C> d = devop<C>(c);
  C one, zero;
  one.x = 1;
  one.y = 0;
  zero.x = 0;
  zero.y = 0;
  // device ms of the given phases, best of 3 after a warm-up
  auto time_of = [&](const Launch& L, std::initializer_list<int> phases) -> float {
    float bt = 1e30f;
    for (int r = 0; r < 4 && e == cudaSuccess; ++r) {
      cudaEventRecord(ev[0], s);
      for (int ph : phases) {
        e = launch_matvec_phase<C>(ph, g, d, L, din, dout, A, B, (int)nrhs, false, one, zero, s);
        if (e != cudaSuccess) break;
      }
      cudaEventRecord(ev[1], s);
      cudaEventSynchronize(ev[1]);
      float t = 0;
      cudaEventElapsedTime(&t, ev[0], ev[1]);
      if (r > 0 && t < bt) bt = t;
    }
    return bt;
  };
  const int cs = (int)csize(c.dtype);
  best = default_launch(c);
  if (keep_radix) {
    best.x_rev = keep_radix->x_rev;
    best.y_rev = keep_radix->y_rev;
  }
  std::vector<int> zc = ct_tiles(cs, c.geom.P[2], true), yc = ct_tiles(cs, c.geom.P[1], false);
  // z tile width jointly with the task form of the fused z pass (one task
  // per thread slot, or one per mirror pair of z frequencies where the
  // kernel has that form; the same arithmetic either way)
  if (!zc.empty()) {
    float bt = 1e30f;
    int pick = best.z_tx, pick_mir = best.z_mir;
    for (int tx : zc)
      for (int mir = 0; mir < 2 && e == cudaSuccess; ++mir) {
        Launch L = best;
        L.z_tx = tx;
        L.z_mir = mir;
        const float t = time_of(L, {1});
        if (e != cudaSuccess) break;
        if (tune_debug())
          fprintf(stderr, "gila autotune dtype %d z tile %d mirror pairs %d: %.4f ms\n", (int)c.dtype, tx, mir, t);
        if (t < bt) {
          bt = t;
          pick = tx;
          pick_mir = mir;
        }
      }
    best.z_tx = pick;
    best.z_mir = pick_mir;
  }
  // y tile width jointly with the form of the x / y passes (first stage fed
  // from global memory, or staged through shared memory: the same
  // arithmetic, the faster one depends on length and precision)
  if (!yc.empty() && e == cudaSuccess) {
    float bt = 1e30f;
    int pick = best.y_tx, pick_g = best.xy_g;
    for (int tx : yc)
      for (int gf = 0; gf < 2 && e == cudaSuccess; ++gf) {
        Launch L = best;
        L.y_tx = tx;
        L.xy_g = gf;
        const float t = time_of(L, {0, 2});
        if (e != cudaSuccess) break;
        if (tune_debug())
          fprintf(stderr, "gila autotune dtype %d y tile %d global-fed x/y %d: %.4f ms\n", (int)c.dtype, tx, gf, t);
        if (t < bt) {
          bt = t;
          pick = tx;
          pick_g = gf;
        }
      }
    best.y_tx = pick;
    best.xy_g = pick_g;
  }
  // radix order of the x and y passes: the greedy one (radix-8 stages first)
  // or its reverse, where they differ (specialised lengths, radix list not a
  // palindrome); phases 0 and 2 hold both passes
  for (int ax = 0; ax < 2 && e == cudaSuccess && !keep_radix; ++ax) {
    const AxisPlan& pl = c.plan[ax];
    bool pal = true;
    for (int k = 0; k < pl.nst; ++k) pal = pal && pl.radix[k] == pl.radix[pl.nst - 1 - k];
    if (ct_tiles(cs, pl.P, false).empty() || pal) continue;
    float bt = 1e30f;
    int pick = 0;
    for (int rv = 0; rv < 2; ++rv) {
      Launch L = best;
      (ax == 0 ? L.x_rev : L.y_rev) = rv;
      const float t = time_of(L, {0, 2});
      if (e != cudaSuccess) break;
      if (tune_debug())
        fprintf(stderr, "gila autotune dtype %d %c radix order %d: %.4f ms\n", (int)c.dtype, ax ? 'y' : 'x', rv, t);
      if (t < bt) {
        bt = t;
        pick = rv;
      }
    }
    (ax == 0 ? best.x_rev : best.y_rev) = pick;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (e != cudaSuccess) return cuda_fail(e, "autotune");
  return GILA_OK;
}

// the operator's own workspaces and two scratch vectors
template <typename C>
static gila_status tune_t(Core& c, int64_t nrhs, Launch& best, const Launch* keep_radix) {
  const int64_t ni = in_elems(c) * nrhs, no = out_elems(c) * nrhs;
  C *din = nullptr, *dout = nullptr;
  GILA_CUDA_TRY(dev_malloc(&din, (size_t)ni * sizeof(C)));
  cudaError_t e = dev_malloc(&dout, (size_t)no * sizeof(C));
  if (e == cudaSuccess) e = cudaMemsetAsync(din, 0, (size_t)ni * sizeof(C), c.stream);
  if (e != cudaSuccess) {
    cudaFree(din);
    cudaFree(dout);
    return cuda_fail(e, "autotune buffers");
  }
  const gila_status s =
      tune_on<C>(c, c.geom, nrhs, din, dout, static_cast<C*>(c.A), static_cast<C*>(c.B), c.stream, best, keep_radix);
  cudaStreamSynchronize(c.stream);
  cudaFree(din);
  cudaFree(dout);
  return s;
}

static bool autotune_off() {
  const char* ev = getenv("GILA_AUTOTUNE");
  return ev && ev[0] == '0';
}

template <typename C>
gila_status tuned_launch(Core& c, const Geom& g, int64_t nrhs, const C* din, C* dout, C* A, C* B, cudaStream_t s,
                         Launch& L) {
  {
    std::lock_guard<std::mutex> lk(c.ctx->mu);
    auto it = c.ctx->tune_cache.find(tune_key(c, nrhs));
    if (it != c.ctx->tune_cache.end()) {
      L = it->second;
      return GILA_OK;
    }
  }
  if (autotune_off()) {
    L = default_launch(c);
    return GILA_OK;
  }
  const gila_status st = tune_on<C>(c, g, nrhs, din, dout, A, B, s, L);
  if (st != GILA_OK) return st;
  std::lock_guard<std::mutex> lk(c.ctx->mu);
  c.ctx->tune_cache[tune_key(c, nrhs)] = L;
  return GILA_OK;
}
template gila_status tuned_launch<double2>(Core&, const Geom&, int64_t, const double2*, double2*, double2*,
                                           double2*, cudaStream_t, Launch&);
template gila_status tuned_launch<float2>(Core&, const Geom&, int64_t, const float2*, float2*, float2*, float2*,
                                          cudaStream_t, Launch&);

// Batch size a tuning run times: nrhs, capped so that its two scratch
// vector sets stay within 512 MiB (beyond that the grids are large and the
// choice no longer moves).
static int64_t tune_rhs(const Core& c, int64_t nrhs) {
  const int64_t per = (in_elems(c) + out_elems(c)) * (int64_t)csize(c.dtype);
  const int64_t cap = std::max<int64_t>(1, (512LL << 20) / std::max<int64_t>(per, 1));
  return std::min(nrhs, cap);
}

// Cache key of a tuning run; a run that kept the operator's radix schedule
// (re-tuning for another batch size) records that schedule too.
static std::string tune_key_of(const Core& c, int64_t nb, const Launch* keep_radix) {
  std::string k = tune_key(c, nb);
  if (keep_radix) k += "|r" + std::to_string(keep_radix->x_rev) + std::to_string(keep_radix->y_rev);
  return k;
}

// A tuning run for nrhs vectors.  The operator's first run picks every
// launch choice; later runs for other batch sizes keep its radix schedule,
// the one choice that changes rounding, so that an operator's result for a
// vector never depends on the batch it came in.
static gila_status autotune_run(Core& c, int64_t nrhs, const Launch* keep_radix) {
  const int64_t nb = tune_rhs(c, nrhs);
  gila_status s = ensure_work(c, nb);
  if (s != GILA_OK) return s;
  Launch L;
  if (c.dtype == GILA_C128)
    s = tune_t<double2>(c, nb, L, keep_radix);
  else
    s = tune_t<float2>(c, nb, L, keep_radix);
  if (s != GILA_OK) return s;
  c.launch = L;
  c.tuned = true;
  c.tuned_rhs = nrhs;
  std::lock_guard<std::mutex> lk(c.ctx->mu);
  c.ctx->tune_cache[tune_key_of(c, nb, keep_radix)] = L;
  return GILA_OK;
}

gila_status autotune(Core& c, int64_t nrhs) {
  const Launch keep = c.launch;
  return autotune_run(c, nrhs, c.tuned ? &keep : nullptr);
}

// The launch shapes for a batch of nrhs vectors: those already in use when
// they were picked for this batch size (or forced by the caller), else the
// context's cached choice, else a tuning run (GILA_AUTOTUNE=0: the
// defaults).  Tile widths and the z task form are re-picked per batch size;
// the radix schedule stays the operator's first choice.
gila_status ensure_tuned(Core& c, int64_t nrhs) {
  if (c.tuned && (c.pinned || c.tuned_rhs == nrhs)) return GILA_OK;
  if (autotune_off()) {
    if (!c.tuned) c.launch = default_launch(c);
    c.tuned = true;
    c.tuned_rhs = nrhs;
    return GILA_OK;
  }
  const Launch keep = c.launch;
  const Launch* kr = c.tuned ? &keep : nullptr;
  {
    std::lock_guard<std::mutex> lk(c.ctx->mu);
    auto it = c.ctx->tune_cache.find(tune_key_of(c, tune_rhs(c, nrhs), kr));
    if (it != c.ctx->tune_cache.end()) {
      c.launch = it->second;
      c.tuned = true;
      c.tuned_rhs = nrhs;
      return GILA_OK;
    }
  }
  return autotune_run(c, nrhs, kr);
}

// staging buffer of at least n elements (contents not kept)
static gila_status ensure_stage(void*& buf, int64_t& cap, int64_t n, size_t cs) {
  if (cap >= n) return GILA_OK;
  cudaFree(buf);
  buf = nullptr;
  cap = 0;
  GILA_CUDA_TRY(dev_malloc(&buf, (size_t)n * cs));
  cap = n;
  return GILA_OK;
}

// Several vectors in host memory: one vector at a time, the upload of vector
// k + 1 and the download of vector k - 1 overlapping the passes of vector k
// (upload, compute and download streams; two staging slots per direction,
// events order each slot's reuse).  With pinned host memory the copies run
// on the copy engines in both directions at once; pageable memory still
// gives the right result, without the overlap.
template <typename C>
static gila_status apply_host_pipe(Core& c, const C* in, C* out, int64_t nrhs, bool din, bool dout, bool axpby, C a,
                                   C b, cudaStream_t st) {
  const int64_t ni = in_elems(c), no = out_elems(c);
  const size_t cs = sizeof(C);
  gila_status s;
  if ((s = ensure_work(c, 1)) != GILA_OK) return s;
  if ((s = ensure_tuned(c, 1)) != GILA_OK) return s;
  if (!din && (s = ensure_stage(c.stage_in, c.stage_cap_in, 2 * ni, cs)) != GILA_OK) return s;
  if (!dout && (s = ensure_stage(c.stage_out, c.stage_cap_out, 2 * no, cs)) != GILA_OK) return s;
  for (cudaStream_t* x : {&c.st_h2d, &c.st_d2h})
    if (!*x) GILA_CUDA_TRY(cudaStreamCreateWithFlags(x, cudaStreamNonBlocking));
  for (int k = 0; k < 2; ++k)
    for (cudaEvent_t* x : {&c.ev_in_ready[k], &c.ev_in_free[k], &c.ev_out_ready[k], &c.ev_out_free[k]})
      if (!*x) GILA_CUDA_TRY(cudaEventCreateWithFlags(x, cudaEventDisableTiming));
  const DevOp<C> d = devop<C>(c);
  // every exit waits for the copies in flight: the caller may free or reuse
  // its host buffers as soon as the call returns, on success or error
  struct Drain {
    cudaStream_t a, b, c;
    ~Drain() {
      cudaStreamSynchronize(a);
      cudaStreamSynchronize(b);
      cudaStreamSynchronize(c);
    }
  } drain{st, c.st_h2d, c.st_d2h};
  for (int64_t k = 0; k < nrhs; ++k) {
    const int sl = (int)(k & 1);
    const C* d_in = din ? in + k * ni : static_cast<const C*>(c.stage_in) + sl * ni;
    C* d_out = dout ? out + k * no : static_cast<C*>(c.stage_out) + sl * no;
    const bool up_out = !dout && axpby;  // beta * out needs the old values
    if (!din || up_out) {
      // the slots' previous vectors (k - 2) have been read by their passes
      // and downloaded
      GILA_CUDA_TRY(cudaStreamWaitEvent(c.st_h2d, c.ev_in_free[sl], 0));
      if (up_out) GILA_CUDA_TRY(cudaStreamWaitEvent(c.st_h2d, c.ev_out_free[sl], 0));
      if (!din)
        GILA_CUDA_TRY(cudaMemcpyAsync(const_cast<C*>(d_in), in + k * ni, (size_t)ni * cs, cudaMemcpyHostToDevice,
                                      c.st_h2d));
      if (up_out)
        GILA_CUDA_TRY(cudaMemcpyAsync(d_out, out + k * no, (size_t)no * cs, cudaMemcpyHostToDevice, c.st_h2d));
      GILA_CUDA_TRY(cudaEventRecord(c.ev_in_ready[sl], c.st_h2d));
      GILA_CUDA_TRY(cudaStreamWaitEvent(st, c.ev_in_ready[sl], 0));
    }
    if (!dout) GILA_CUDA_TRY(cudaStreamWaitEvent(st, c.ev_out_free[sl], 0));
    GILA_CUDA_TRY(launch_matvec<C>(c.geom, d, c.launch, d_in, d_out, static_cast<C*>(c.A), static_cast<C*>(c.B), 1,
                                   axpby, a, b, st));
    GILA_CUDA_TRY(cudaEventRecord(c.ev_in_free[sl], st));
    if (!dout) {
      GILA_CUDA_TRY(cudaEventRecord(c.ev_out_ready[sl], st));
      GILA_CUDA_TRY(cudaStreamWaitEvent(c.st_d2h, c.ev_out_ready[sl], 0));
      GILA_CUDA_TRY(cudaMemcpyAsync(out + k * no, d_out, (size_t)no * cs, cudaMemcpyDeviceToHost, c.st_d2h));
      GILA_CUDA_TRY(cudaEventRecord(c.ev_out_free[sl], c.st_d2h));
    }
  }
  GILA_CUDA_TRY(cudaStreamSynchronize(st));
  GILA_CUDA_TRY(cudaStreamSynchronize(c.st_d2h));
  GILA_CUDA_TRY(cudaStreamSynchronize(c.st_h2d));
  return GILA_OK;  // (the drain's waits are then no-ops)
}

template <typename C>
static gila_status apply_t(Core& c, const void* in, void* out, int64_t nrhs, bool axpby, const double* alpha,
                           const double* beta, cudaStream_t user_st) {
  const int64_t ni = in_elems(c) * nrhs, no = out_elems(c) * nrhs;
  const size_t cs = sizeof(C);
  cudaStream_t st = user_st ? user_st : c.stream;
  const bool din = is_device_ptr(in), dout = is_device_ptr(out);
  // element alignment (the passes copy with 16 / 8 byte cp.async)
  if ((din && ((uintptr_t)in % cs)) || (dout && ((uintptr_t)out % cs)))
    return fail(GILA_ERR_ARG, "device vectors must be aligned to their complex element size");
  C a, b;
  a.x = alpha ? (decltype(a.x))alpha[0] : 1;
  a.y = alpha ? (decltype(a.y))alpha[1] : 0;
  b.x = beta ? (decltype(b.x))beta[0] : 0;
  b.y = beta ? (decltype(b.y))beta[1] : 0;
  if ((!din || !dout) && nrhs > 1)
    return apply_host_pipe<C>(c, static_cast<const C*>(in), static_cast<C*>(out), nrhs, din, dout, axpby, a, b, st);
  gila_status s = ensure_work(c, nrhs);
  if (s != GILA_OK) return s;
  if ((s = ensure_tuned(c, nrhs)) != GILA_OK) return s;
  const C* d_in = static_cast<const C*>(in);
  C* d_out = static_cast<C*>(out);
  // host vectors: an error return also waits for the copies already queued
  struct Drain {
    cudaStream_t st;
    bool on;
    ~Drain() {
      if (on) cudaStreamSynchronize(st);
    }
  } drain{st, !din || !dout};
  if (!din) {
    if ((s = ensure_stage(c.stage_in, c.stage_cap_in, ni, cs)) != GILA_OK) return s;
    GILA_CUDA_TRY(cudaMemcpyAsync(c.stage_in, in, (size_t)ni * cs, cudaMemcpyHostToDevice, st));
    d_in = static_cast<const C*>(c.stage_in);
  }
  if (!dout) {
    if ((s = ensure_stage(c.stage_out, c.stage_cap_out, no, cs)) != GILA_OK) return s;
    if (axpby) GILA_CUDA_TRY(cudaMemcpyAsync(c.stage_out, out, (size_t)no * cs, cudaMemcpyHostToDevice, st));
    d_out = static_cast<C*>(c.stage_out);
  }
  GILA_CUDA_TRY(launch_matvec<C>(c.geom, devop<C>(c), c.launch, d_in, d_out, static_cast<C*>(c.A),
                                 static_cast<C*>(c.B), (int)nrhs, axpby, a, b, st));
  if (!dout) GILA_CUDA_TRY(cudaMemcpyAsync(out, c.stage_out, (size_t)no * cs, cudaMemcpyDeviceToHost, st));
  if (!user_st || !din || !dout) GILA_CUDA_TRY(cudaStreamSynchronize(st));
  return GILA_OK;
}

static gila_status apply_common(gila_opr* opr, gila_dtype dtype, const void* in, int64_t in_len, void* out,
                                int64_t out_len, int64_t nrhs, bool axpby, const double* alpha, const double* beta,
                                void* stream) {
  if (!opr || !opr->core) return fail(GILA_ERR_ARG, "null operator");
  Core& c = *opr->core;
  if (dtype != c.dtype)
    return fail(GILA_ERR_TYPE, std::string("Input array must have the same element type as the operator. eltype(opr) = ") +
                                   (c.dtype == GILA_C128 ? "ComplexF64" : "ComplexF32"));
  if (nrhs < 1) return fail(GILA_ERR_ARG, "nrhs must be >= 1");
  if (c.parS != 1 || in_len != in_elems(c) * nrhs || out_len != out_elems(c) * nrhs)
    return fail(GILA_ERR_SIZE,
                "Size of input vector does not match size of source volume. Required data layout is (srcCelX, "
                "srcCelY, srcCelZ, 3).");
  if (!in || !out) return fail(GILA_ERR_ARG, "null vector");
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  if (c.dtype == GILA_C128)
    return apply_t<double2>(c, in, out, nrhs, axpby, alpha, beta, static_cast<cudaStream_t>(stream));
  return apply_t<float2>(c, in, out, nrhs, axpby, alpha, beta, static_cast<cudaStream_t>(stream));
}

template <typename C>
gila_status time_passes_t(Core& c, int64_t nrhs, int reps, double ms[4]) {
  gila_status s = ensure_work(c, nrhs);
  if (s != GILA_OK) return s;
  if ((s = ensure_tuned(c, nrhs)) != GILA_OK) return s;
  const int64_t ni = in_elems(c) * nrhs, no = out_elems(c) * nrhs;
  C *din = nullptr, *dout = nullptr;
  GILA_CUDA_TRY(dev_malloc(&din, (size_t)ni * sizeof(C)));
  cudaError_t e = dev_malloc(&dout, (size_t)no * sizeof(C));
  if (e != cudaSuccess) {
    cudaFree(din);
    return cuda_fail(e, "cudaMalloc");
  }
  cudaMemsetAsync(din, 0, (size_t)ni * sizeof(C), c.stream);
  cudaEvent_t ev[4];
  for (auto& x : ev) cudaEventCreate(&x);
  double acc[3] = {0, 0, 0};
  const DevOp<C> d = devop<C>(c);
  C one, zero;
  one.x = 1;
  one.y = 0;
  zero.x = 0;
  zero.y = 0;
  for (int r = -1; r < reps && e == cudaSuccess; ++r) {
    cudaEventRecord(ev[0], c.stream);
    for (int ph = 0; ph < 3 && e == cudaSuccess; ++ph) {
      e = launch_matvec_phase<C>(ph, c.geom, d, c.launch, din, dout, static_cast<C*>(c.A), static_cast<C*>(c.B),
                                 (int)nrhs, false, one, zero, c.stream);
      cudaEventRecord(ev[ph + 1], c.stream);
    }
    cudaEventSynchronize(ev[3]);
    if (r >= 0)  // r = -1 is a warm-up
      for (int ph = 0; ph < 3; ++ph) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[ph], ev[ph + 1]);
        acc[ph] += t;
      }
  }
  for (auto& x : ev) cudaEventDestroy(x);
  cudaFree(din);
  cudaFree(dout);
  if (e != cudaSuccess) return cuda_fail(e, "time_passes");
  for (int ph = 0; ph < 3; ++ph) ms[ph] = acc[ph] / reps;
  ms[3] = ms[0] + ms[1] + ms[2];
  return GILA_OK;
}

}  // namespace gila

using namespace gila;

// =================================================================== C ABI
extern "C" {

const char* gila_last_error(void) { return g_err.c_str(); }

const char* gila_version(void) { return "0.1.0"; }

gila_status gila_debug_fail_alloc(int64_t n) {
  if (n < 0) return fail(GILA_ERR_ARG, "gila_debug_fail_alloc: n must be >= 0");
  g_fail_alloc.store(n);
  return GILA_OK;
}

const char* gila_status_string(gila_status s) {
  switch (s) {
    case GILA_OK: return "ok";
    case GILA_ERR_ARG: return "invalid argument";
    case GILA_ERR_SIZE: return "size mismatch";
    case GILA_ERR_TYPE: return "element type mismatch";
    case GILA_ERR_CUDA: return "CUDA error";
    case GILA_ERR_NOMEM: return "out of memory";
    case GILA_ERR_NAN: return "non-numeric values";
    case GILA_ERR_NODEV: return "no usable CUDA device";
    case GILA_ERR_OVERLAP: return "overlapping volumes";
    case GILA_ERR_SCALE: return "incompatible scales";
    case GILA_ERR_NOTCONV: return "not converged";
    case GILA_ERR_TIMEOUT: return "device wait timed out";
    default: return "internal error";
  }
}

gila_status gila_ctx_create(int device, gila_ctx** out) {
  if (!out) return fail(GILA_ERR_ARG, "null output");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(GILA_ERR_NODEV,
                "Device computation requested, but CUDA is not functional. For CPU computation use "
                "GlaKerOpt(false)---devMod = false---when declaring compute options.");
  }
  if (device < 0 || device >= n) return fail(GILA_ERR_ARG, "device index out of range");
  GILA_CUDA_TRY(cudaSetDevice(device));
  GILA_CUDA_TRY(cudaFree(0));
  auto* c = new gila_ctx;
  c->impl = new Ctx;
  c->impl->device = device;
  *out = c;
  return GILA_OK;
}

gila_status gila_ctx_destroy(gila_ctx* ctx) {
  if (!ctx) return GILA_OK;
  cudaSetDevice(ctx->impl->device);
  delete ctx->impl;
  delete ctx;
  return GILA_OK;
}

gila_status gila_opr_create_from_fur(gila_ctx* ctx, const gila_vol* trg, const gila_vol* src, const gila_kopt* opt,
                                     gila_dtype dtype, const void* const fur[8], const int64_t fur_dims[8][6],
                                     gila_dtype fur_dtype, gila_opr** out) {
  if (!out || !fur || !fur_dims) return fail(GILA_ERR_ARG, "null argument");
  if (!ctx) return fail(GILA_ERR_ARG, "null context");
  GILA_CUDA_TRY(cudaSetDevice(ctx->impl->device));
  std::shared_ptr<Core> core;
  gila_status s = init_core(ctx, trg, src, opt, dtype, core);
  if (s != GILA_OK) return s;
  const Geom& g = core->geom;
  for (int eo = 0; eo < 8; ++eo) {
    const int64_t want[6] = {g.tru[0], g.tru[1], g.tru[2], 6, core->parS, g.parT};
    for (int k = 0; k < 6; ++k)
      if (fur_dims[eo][k] != want[k])
        return fail(GILA_ERR_ARG, "egoFur branch " + std::to_string(eo) + " has extents that do not match the volumes");
  }
  const size_t bytes = (size_t)g.tru[0] * g.tru[1] * g.tru[2] * 6 * 8 * g.parT * csize(dtype);
  GILA_CUDA_TRY(dev_malloc(&core->ker, bytes));
  core->ker_bytes = bytes;
  if (dtype == GILA_C128) {
    std::vector<double2> h;
    if ((s = load_fur(*core, fur, fur_dtype, h)) != GILA_OK) return s;
    GILA_CUDA_TRY(cudaMemcpy(core->ker, h.data(), bytes, cudaMemcpyHostToDevice));
  } else {
    std::vector<float2> h;
    if ((s = load_fur(*core, fur, fur_dtype, h)) != GILA_OK) return s;
    GILA_CUDA_TRY(cudaMemcpy(core->ker, h.data(), bytes, cudaMemcpyHostToDevice));
  }
  auto* o = new gila_opr;
  o->ctx = ctx;
  o->core = core;
  o->trg = core->trg;
  o->src = core->src;
  o->adj = opt ? (opt->adj_mod != 0) : 0;
  *out = o;
  return GILA_OK;
}

gila_status gila_opr_fur_dims(const gila_opr* opr, int64_t dims[8][6]) {
  if (!opr || !dims) return fail(GILA_ERR_ARG, "null argument");
  const Core& c = *opr->core;
  for (int eo = 0; eo < 8; ++eo) {
    dims[eo][0] = c.geom.tru[0];
    dims[eo][1] = c.geom.tru[1];
    dims[eo][2] = c.geom.tru[2];
    dims[eo][3] = 6;
    dims[eo][4] = c.parS;
    dims[eo][5] = c.geom.parT;
  }
  return GILA_OK;
}

gila_status gila_opr_export_fur(gila_opr* opr, void* const host_out[8]) {
  if (!opr || !host_out) return fail(GILA_ERR_ARG, "null argument");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  const Geom& g = c.geom;
  const size_t cs = csize(c.dtype);
  std::vector<unsigned char> h(c.ker_bytes);
  GILA_CUDA_TRY(cudaMemcpy(h.data(), c.ker, c.ker_bytes, cudaMemcpyDeviceToHost));
  const int tx = g.tru[0], ty = g.tru[1], tz = g.tru[2];
  for (int eo = 0; eo < 8; ++eo) {
    unsigned char* dst = static_cast<unsigned char*>(host_out[eo]);
    if (!dst) return fail(GILA_ERR_ARG, "null output branch");
    const int64_t n = (int64_t)tx * ty * tz * 6 * c.parS * g.parT;
    memset(dst, 0, (size_t)n * cs);
    for (int tp = 0; tp < g.parT; ++tp)
      for (int cc = 0; cc < 6; ++cc)
        for (int iz = 0; iz < tz; ++iz)
          for (int iy = 0; iy < ty; ++iy)
            for (int ix = 0; ix < tx; ++ix) {
              const int64_t di = ((((int64_t)tp * c.parS) * 6 + cc) * tz + iz) * ty * (int64_t)tx + (int64_t)iy * tx + ix;
              const int64_t si = (int64_t)tp * 8 * tx * ty * tz * 6 + ker_index(eo, iz, iy, cc, ix, tx, ty, tz);
              memcpy(dst + di * cs, h.data() + si * cs, cs);
            }
  }
  return GILA_OK;
}

// ---- kernel cache on disk ------------------------------------------------
// File layout (little-endian), 768-byte header then the 8 egoFur arrays:
//   0 "GILAFUR1" | 8 int32 version (1) | 12 int32 dtype of the arrays
//   16 int32 self | 20 int32 adjMod | 24 int32 intOrd | 28 int32 0
//   32 f64 frqPhz re | 40 f64 frqPhz im
//   48 int64[21] target gila_vol | 216 int64[21] source gila_vol
//   384 int64[8][6] branch extents (tx, ty, tz, 6, parSrc, parTrg)
//   768 fur[0] ... fur[7], column-major complex (re, im) per element
static const char kFurMagic[8] = {'G', 'I', 'L', 'A', 'F', 'U', 'R', '1'};
constexpr size_t kFurHeader = 768;

static void vol_pack(const gila_vol& v, int64_t out[21]) {
  for (int k = 0; k < 3; ++k) {
    out[k] = v.cel[k];
    out[3 + k] = v.scl_num[k];
    out[6 + k] = v.scl_den[k];
    out[9 + k] = v.org_num[k];
    out[12 + k] = v.org_den[k];
    out[15 + k] = v.grd_num[k];
    out[18 + k] = v.grd_den[k];
  }
}
static gila_vol vol_unpack(const int64_t in[21]) {
  gila_vol v;
  for (int k = 0; k < 3; ++k) {
    v.cel[k] = in[k];
    v.scl_num[k] = in[3 + k];
    v.scl_den[k] = in[6 + k];
    v.org_num[k] = in[9 + k];
    v.org_den[k] = in[12 + k];
    v.grd_num[k] = in[15 + k];
    v.grd_den[k] = in[18 + k];
  }
  return v;
}

gila_status gila_opr_adjoint(gila_opr* opr, gila_opr** out) {
  if (!opr || !out) return fail(GILA_ERR_ARG, "null argument");
  auto* o = new gila_opr;
  o->ctx = opr->ctx;
  o->core = opr->core;
  o->trg = opr->src;
  o->src = opr->trg;
  o->adj = !opr->adj;
  *out = o;
  return GILA_OK;
}

gila_status gila_opr_save(gila_opr* opr, const char* path) {
  if (!opr || !opr->core || !path) return fail(GILA_ERR_ARG, "null argument");
  const Core& c = *opr->core;
  int64_t dims[8][6];
  gila_status s = gila_opr_fur_dims(opr, dims);
  if (s != GILA_OK) return s;
  const size_t cs = csize(c.dtype);
  std::vector<std::vector<unsigned char>> fur(8);
  void* ptrs[8];
  for (int eo = 0; eo < 8; ++eo) {
    int64_t n = 1;
    for (int k = 0; k < 6; ++k) n *= dims[eo][k];
    fur[eo].resize((size_t)n * cs);
    ptrs[eo] = fur[eo].data();
  }
  if ((s = gila_opr_export_fur(opr, ptrs)) != GILA_OK) return s;
  unsigned char hdr[kFurHeader];
  memset(hdr, 0, sizeof hdr);
  memcpy(hdr, kFurMagic, 8);
  const int32_t i32[6] = {1, (int32_t)c.dtype, c.self ? 1 : 0, (int32_t)(c.opt.adj_mod != 0),
                          c.opt.int_ord > 0 ? c.opt.int_ord : 32, 0};
  memcpy(hdr + 8, i32, sizeof i32);
  const double frq[2] = {c.opt.frq_re, c.opt.frq_im};
  memcpy(hdr + 32, frq, sizeof frq);
  int64_t tv[21], sv[21];
  vol_pack(vol_to_abi(c.trg), tv);
  vol_pack(vol_to_abi(c.self ? c.trg : c.src), sv);
  memcpy(hdr + 48, tv, sizeof tv);
  memcpy(hdr + 216, sv, sizeof sv);
  memcpy(hdr + 384, dims, sizeof dims);
  FILE* f = fopen(path, "wb");
  if (!f) return fail(GILA_ERR_ARG, std::string("cannot open ") + path + " for writing");
  bool ok = fwrite(hdr, 1, sizeof hdr, f) == sizeof hdr;
  for (int eo = 0; eo < 8 && ok; ++eo) ok = fwrite(fur[eo].data(), 1, fur[eo].size(), f) == fur[eo].size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(GILA_ERR_INTERNAL, std::string("short write to ") + path);
  return GILA_OK;
}

gila_status gila_opr_load(gila_ctx* ctx, const char* path, gila_dtype dtype, gila_opr** out) {
  if (!ctx || !path || !out) return fail(GILA_ERR_ARG, "null argument");
  if (dtype != GILA_C64 && dtype != GILA_C128) return fail(GILA_ERR_ARG, "unknown dtype");
  FILE* f = fopen(path, "rb");
  if (!f) return fail(GILA_ERR_ARG, std::string("cannot open ") + path);
  unsigned char hdr[kFurHeader];
  if (fread(hdr, 1, sizeof hdr, f) != sizeof hdr || memcmp(hdr, kFurMagic, 8) != 0) {
    fclose(f);
    return fail(GILA_ERR_ARG, std::string(path) + " is not a GILAFUR1 kernel file");
  }
  int32_t i32[6];
  double frq[2];
  int64_t tv[21], sv[21], dims[8][6];
  memcpy(i32, hdr + 8, sizeof i32);
  memcpy(frq, hdr + 32, sizeof frq);
  memcpy(tv, hdr + 48, sizeof tv);
  memcpy(sv, hdr + 216, sizeof sv);
  memcpy(dims, hdr + 384, sizeof dims);
  if (i32[0] != 1 || (i32[1] != GILA_C64 && i32[1] != GILA_C128)) {
    fclose(f);
    return fail(GILA_ERR_ARG, std::string(path) + ": unsupported GILAFUR version or dtype");
  }
  const gila_dtype fdt = (gila_dtype)i32[1];
  const size_t cs = csize(fdt);
  std::vector<std::vector<unsigned char>> fur(8);
  const void* ptrs[8];
  for (int eo = 0; eo < 8; ++eo) {
    int64_t n = 1;
    for (int k = 0; k < 6; ++k) {
      if (dims[eo][k] < 1 || dims[eo][k] > (int64_t)1 << 20) {
        fclose(f);
        return fail(GILA_ERR_ARG, std::string(path) + ": corrupt branch extents");
      }
      n *= dims[eo][k];
    }
    if (n > ((int64_t)1 << 36) / (int64_t)cs) {
      fclose(f);
      return fail(GILA_ERR_ARG, std::string(path) + ": corrupt branch extents");
    }
    fur[eo].resize((size_t)n * cs);
    if (fread(fur[eo].data(), 1, fur[eo].size(), f) != fur[eo].size()) {
      fclose(f);
      return fail(GILA_ERR_ARG, std::string(path) + ": file ends inside the kernel data");
    }
    ptrs[eo] = fur[eo].data();
  }
  fclose(f);
  const gila_vol trg = vol_unpack(tv), src = vol_unpack(sv);
  gila_kopt opt;
  memset(&opt, 0, sizeof opt);
  opt.frq_re = frq[0];
  opt.frq_im = frq[1];
  opt.int_ord = i32[4];
  opt.adj_mod = i32[3];
  opt.dev_mod = 1;
  return gila_opr_create_from_fur(ctx, &trg, i32[2] ? nullptr : &src, &opt, dtype, ptrs, dims, fdt, out);
}

gila_status gila_opr_destroy(gila_opr* opr) {
  delete opr;
  return GILA_OK;
}

gila_status gila_opr_sizes(const gila_opr* opr, int64_t trg[4], int64_t src[4]) {
  if (!opr) return fail(GILA_ERR_ARG, "null operator");
  for (int k = 0; k < 3; ++k) {
    if (trg) trg[k] = opr->trg.cel[k];
    if (src) src[k] = opr->src.cel[k];
  }
  if (trg) trg[3] = 3;
  if (src) src[3] = 3;
  return GILA_OK;
}

gila_status gila_opr_input_size(const gila_opr* opr, int64_t in[4]) {
  if (!opr || !in) return fail(GILA_ERR_ARG, "null argument");
  for (int k = 0; k < 3; ++k) in[k] = opr->core->geom.sc[k];
  in[3] = 3;
  return GILA_OK;
}

gila_status gila_opr_output_size(const gila_opr* opr, int64_t o[4]) {
  if (!opr || !o) return fail(GILA_ERR_ARG, "null argument");
  for (int k = 0; k < 3; ++k) o[k] = opr->core->geom.out_full[k];
  o[3] = 3;
  return GILA_OK;
}

gila_status gila_opr_info(const gila_opr* opr, gila_dtype* dtype, int32_t* flags) {
  if (!opr) return fail(GILA_ERR_ARG, "null operator");
  if (dtype) *dtype = opr->core->dtype;
  if (flags) *flags = (vol_eq(opr->trg, opr->src) ? 1 : 0) | (opr->adj ? 2 : 0);
  return GILA_OK;
}

gila_status gila_opr_apply(gila_opr* opr, gila_dtype dtype, const void* in, int64_t in_len, void* out,
                           int64_t out_len, int64_t nrhs, void* stream) {
  return apply_common(opr, dtype, in, in_len, out, out_len, nrhs, false, nullptr, nullptr, stream);
}

gila_status gila_opr_apply_axpby(gila_opr* opr, gila_dtype dtype, const double alpha[2], const void* in,
                                 int64_t in_len, const double beta[2], void* out, int64_t out_len, int64_t nrhs,
                                 void* stream) {
  return apply_common(opr, dtype, in, in_len, out, out_len, nrhs, true, alpha, beta, stream);
}

gila_status gila_opr_reserve(gila_opr* opr, int64_t nrhs) {
  if (!opr) return fail(GILA_ERR_ARG, "null operator");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  gila_status s = ensure_work(c, nrhs);
  if (s != GILA_OK) return s;
  return ensure_tuned(c, nrhs);
}

gila_status gila_opr_autotune(gila_opr* opr, int64_t nrhs, int32_t tiles[4]) {
  if (!opr || nrhs < 1) return fail(GILA_ERR_ARG, "invalid argument");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  c.pinned = false;
  gila_status s = autotune(c, nrhs);
  if (s != GILA_OK) return s;
  if (tiles) {
    tiles[0] = c.launch.xf_lines;
    tiles[1] = c.launch.xi_lines;
    tiles[2] = c.launch.y_tx;
    tiles[3] = c.launch.z_tx;
  }
  return GILA_OK;
}

gila_status gila_opr_get_tiles(gila_opr* opr, int32_t tiles[4]) {
  if (!opr || !tiles) return fail(GILA_ERR_ARG, "null argument");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  const Launch L = c.tuned ? c.launch : default_launch(c);
  tiles[0] = L.xf_lines;
  tiles[1] = L.xi_lines;
  tiles[2] = L.y_tx;
  tiles[3] = L.z_tx;
  return GILA_OK;
}

gila_status gila_opr_set_tiles(gila_opr* opr, const int32_t tiles[4]) {
  if (!opr || !tiles) return fail(GILA_ERR_ARG, "null argument");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  Launch L = c.tuned ? c.launch : default_launch(c);
  const int cs = (int)csize(c.dtype);
  if (tiles[2] > 0) L.y_tx = ct_tile_pick(cs, c.geom.P[1], tiles[2], false) == tiles[2] ? tiles[2] : L.y_tx;
  if (tiles[3] > 0) L.z_tx = ct_tile_pick(cs, c.geom.P[2], tiles[3], true) == tiles[3] ? tiles[3] : L.z_tx;
  c.launch = L;
  c.tuned = true;
  c.pinned = true;
  return GILA_OK;
}

gila_status gila_opr_get_schedule(gila_opr* opr, int32_t sched[2]) {
  if (!opr || !sched) return fail(GILA_ERR_ARG, "null argument");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  const Launch L = c.tuned ? c.launch : default_launch(c);
  sched[0] = L.x_rev;
  sched[1] = L.y_rev;
  return GILA_OK;
}

gila_status gila_opr_set_schedule(gila_opr* opr, const int32_t sched[2]) {
  if (!opr || !sched) return fail(GILA_ERR_ARG, "null argument");
  if (sched[0] > 1 || sched[1] > 1) return fail(GILA_ERR_ARG, "radix order is 0 (greedy) or 1 (reversed)");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  Launch L = c.tuned ? c.launch : default_launch(c);
  if (sched[0] >= 0) L.x_rev = sched[0];
  if (sched[1] >= 0) L.y_rev = sched[1];
  c.launch = L;
  c.tuned = true;
  c.pinned = true;
  return GILA_OK;
}

gila_status gila_opr_device_bytes(const gila_opr* opr, int64_t* bytes) {
  if (!opr || !bytes) return fail(GILA_ERR_ARG, "null argument");
  const Core& c = *opr->core;
  const Work w = work_sizes(c.geom);
  *bytes = (int64_t)c.ker_bytes + (w.a_elems + w.b_rhs * c.cap_rhs) * (int64_t)csize(c.dtype);
  return GILA_OK;
}

gila_status gila_opr_launches_per_apply(const gila_opr* opr, int64_t nrhs, int64_t* n) {
  if (!opr || !n || nrhs < 1) return fail(GILA_ERR_ARG, "invalid argument");
  const Core& c = *opr->core;
  Geom g = c.geom;
  if (nrhs > g.max_rhs) g.max_rhs = (int)nrhs;
  const Launch L = c.tuned ? c.launch : default_launch(c);
  const int nch = c.dtype == GILA_C128 ? kx_chunks<double2>(g, devop<double2>(c), L, (int)nrhs)
                                       : kx_chunks<float2>(g, devop<float2>(c), L, (int)nrhs);
  *n = matvec_launches(g, (int)nrhs, nch);
  return GILA_OK;
}

gila_status gila_opr_time_passes(gila_opr* opr, int64_t nrhs, int reps, double ms[4]) {
  if (!opr || !ms || nrhs < 1 || reps < 1) return fail(GILA_ERR_ARG, "invalid argument");
  Core& c = *opr->core;
  std::lock_guard<std::mutex> lk(c.mu);
  GILA_CUDA_TRY(cudaSetDevice(c.device));
  if (c.dtype == GILA_C128) return time_passes_t<double2>(c, nrhs, reps, ms);
  return time_passes_t<float2>(c, nrhs, reps, ms);
}

gila_status gila_opr_create(gila_ctx* ctx, const gila_vol* trg, const gila_vol* src, const gila_kopt* opt,
                            gila_dtype dtype, gila_opr** out) {
  if (!out) return fail(GILA_ERR_ARG, "null output");
  if (!ctx) return fail(GILA_ERR_ARG, "null context");
  GILA_CUDA_TRY(cudaSetDevice(ctx->impl->device));
  std::shared_ptr<Core> core;
  gila_status s = init_core(ctx, trg, src, opt, dtype, core);
  if (s != GILA_OK) return s;
  if ((s = build_kernel(*core)) != GILA_OK) return s;
  auto* o = new gila_opr;
  o->ctx = ctx;
  o->core = core;
  o->trg = core->trg;
  o->src = core->src;
  o->adj = opt ? (opt->adj_mod != 0) : 0;
  *out = o;
  return GILA_OK;
}

}  // extern "C"
