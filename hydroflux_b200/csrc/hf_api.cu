// hf_api.cu -- C ABI (include/hydroflux_gpu.h) over the sm_100a kernels.
//
// hf_sim mirrors `Simulation` (solver-2d/src/sim.rs:119-245): it owns the
// device mesh/state, one CUDA stream and pre-captured CUDA graphs of 1, 8 and
// 64 steps. A step is [control -> stage 1 -> stage 2 (+ epilogue)]; dt, the
// clock and the step budget live in a device control block, so run_until
// replays graph chunks and reads 64 bytes back per chunk.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hydroflux_gpu.h"
#include "hf_internal.h"

using namespace hf;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HF_OK;
  cudaGetLastError();
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return fail(e == cudaErrorMemoryAllocation ? HF_ERR_OUT_OF_MEMORY : HF_ERR_CUDA, m);
}

#define HF_CUDA(call)                                \
  do {                                               \
    cudaError_t _e = (call);                         \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

#define HF_TRY(expr)          \
  do {                        \
    int _rc = (expr);         \
    if (_rc != 0) return _rc; \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

BcDev to_bcdev(const hf_boundaries& b) {
  BcDev d;
  const hf_boundary* s[4] = {&b.north, &b.south, &b.west, &b.east};
  for (int k = 0; k < 4; ++k) {
    d.kind[k] = s[k]->kind;
    d.val[k] = s[k]->value;
  }
  return d;
}

int check_bcs(const hf_boundaries& b, int64_t nr, int64_t nc) {
  const hf_boundary* s[4] = {&b.north, &b.south, &b.west, &b.east};
  for (int k = 0; k < 4; ++k) {
    const int kind = s[k]->kind;
    if (kind < HF_BC_TRANSMISSIVE || kind > HF_BC_DEPTH)
      return fail(HF_ERR_INVALID_CONFIG, "unknown boundary kind");
    if ((kind == HF_BC_DISCHARGE || kind == HF_BC_DEPTH) && (k < 2 ? nr : nc) < 2)
      return fail(HF_ERR_INVALID_CONFIG,
                  "Discharge/Depth boundaries extend the bed linearly and need >= 2 cells "
                  "normal to the side");
  }
  return HF_OK;
}

int check_shape(int64_t nr, int64_t nc) {
  if (nr <= 0 || nc <= 0) return fail(HF_ERR_SHAPE_MISMATCH, "mesh must have at least one cell");
  if (nr > INT_MAX / 2 || nc > INT_MAX / 2 || nr * nc > (int64_t)INT_MAX * 8)
    return fail(HF_ERR_INVALID_ARG, "mesh too large");
  return HF_OK;
}

template <class T>
int dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  return cuda_fail(e, "cudaMalloc");
}

// The state fields of simulation handles come from one memory pool per
// device that keeps freed memory mapped (release threshold: never), so a
// handle created after another was destroyed reuses its memory instead of
// asking the driver for fresh pages (measured: 5-600 ms for 1 GB of new
// allocations, against under a millisecond from the pool).
// hf_release_cached_memory returns the pool's unused memory.
std::mutex g_pool_mu;
cudaMemPool_t g_pool[64] = {};

// Pinned host mirrors of control blocks (one Ctrl each) kept from destroyed
// simulation handles for the next ones: pinning a fresh page costs 1-3 ms.
// hf_release_cached_memory frees them.
std::vector<Ctrl*> g_pinned_ctrl;
constexpr size_t kPinnedCtrlKeep = 64;

int pinned_ctrl_get(Ctrl** p) {
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pinned_ctrl.empty()) {
      *p = g_pinned_ctrl.back();
      g_pinned_ctrl.pop_back();
      return HF_OK;
    }
  }
  return cuda_fail(cudaMallocHost((void**)p, sizeof(Ctrl)), "cudaMallocHost");
}

void pinned_ctrl_put(Ctrl* p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (g_pinned_ctrl.size() < kPinnedCtrlKeep) {
      g_pinned_ctrl.push_back(p);
      return;
    }
  }
  cudaFreeHost(p);
}

int state_pool(int device, cudaMemPool_t* out) {
  if (device < 0 || device >= 64) return fail(HF_ERR_INVALID_ARG, "bad device index");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[device]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolCreate");
    unsigned long long keep = ~0ull;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return cuda_fail(e, "cudaMemPoolSetAttribute");
    }
    g_pool[device] = pool;
  }
  *out = g_pool[device];
  return HF_OK;
}

// n doubles from the device's state pool, in order on `stream`.
int palloc(double** p, size_t n, int device, cudaStream_t stream) {
  cudaMemPool_t pool = nullptr;
  HF_TRY(state_pool(device, &pool));
  if (n == 0) n = 1;
  return cuda_fail(cudaMallocFromPoolAsync((void**)p, n * sizeof(double), pool, stream),
                   "cudaMallocFromPoolAsync");
}

void pfree(void* p, cudaStream_t stream) {
  if (p) cudaFreeAsync(p, stream);
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

// max_depth_exceeds_relief (sim.rs:248-271): device max/min reductions, then
// the reference's host expression on the three values.
int relief_check(int64_t ncell, const double* h, const double* z, double factor, Ctrl* d_ctrl,
                 Ctrl* h_ctrl, cudaStream_t st, int* exceeds) {
  unsigned long long* keys = d_ctrl->relief_keys;
  HF_CUDA(cudaMemsetAsync(keys, 0, 2 * sizeof(unsigned long long), st));
  HF_CUDA(cudaMemsetAsync(keys + 2, 0xff, sizeof(unsigned long long), st));
  if (launch_relief(ncell, h, z, d_ctrl, st)) return cuda_fail(failed_call_error(), "relief");
  HF_CUDA(cudaMemcpyAsync(h_ctrl->relief_keys, keys, 3 * sizeof(unsigned long long),
                          cudaMemcpyDeviceToHost, st));
  HF_CUDA(cudaStreamSynchronize(st));
  const double max_depth = relief_key_value(h_ctrl->relief_keys[0]);
  const double bed_max = relief_key_value(h_ctrl->relief_keys[1]);
  const double bed_min = relief_key_value(h_ctrl->relief_keys[2]);
  const double relief = std::fmax(bed_max - bed_min, 1.0);  // f64::max(NaN, 1) = 1
  *exceeds = max_depth > factor * relief ? 1 : 0;
  return HF_OK;
}

}  // namespace

int hf::record_error(int code, const char* msg) { return fail(code, msg ? msg : ""); }

BcDev hf::boundaries_dev(const hf_boundaries& b) { return to_bcdev(b); }

int hf::check_boundaries(const hf_boundaries& b, int64_t nr, int64_t nc) {
  return check_bcs(b, nr, nc);
}

// ---------------------------------------------------------------- forcing
void ForcingHost::release_rain() {
  dfree(d_rain_t);
  dfree(d_rain_v);
  d_rain_t = d_rain_v = nullptr;
  n_rain = 0;
}

void ForcingHost::release_src() {
  for (void* p : {(void*)d_row, (void*)d_col, (void*)d_off, (void*)d_st, (void*)d_sq,
                  (void*)d_tile_start[0], (void*)d_tile_order[0], (void*)d_tile_start[1],
                  (void*)d_tile_order[1], (void*)d_blk_start, (void*)d_blk_order, (void*)d_dh})
    dfree(p);
  d_row = d_col = d_off = d_blk_start = d_blk_order = nullptr;
  d_tile_start[0] = d_tile_order[0] = d_tile_start[1] = d_tile_order[1] = nullptr;
  d_st = d_sq = d_dh = nullptr;
  n_src = 0;
}

ForcingDev ForcingHost::dev(int geom) const {
  ForcingDev f;
  f.n_rain = n_rain;
  f.n_src = n_src;
  f.rain_t = d_rain_t;
  f.rain_v = d_rain_v;
  f.src_row = d_row;
  f.src_col = d_col;
  f.src_off = d_off;
  f.src_t = d_st;
  f.src_q = d_sq;
  f.tile_start = d_tile_start[geom];
  f.tile_order = d_tile_order[geom];
  f.blk_start = d_blk_start;
  f.blk_order = d_blk_order;
  f.src_dh = d_dh;
  f.rain_u = rain_u;
  f.src_u = src_u;
  return f;
}

int hf::forcing_set_rain(ForcingHost& f, int64_t n_points, const double* t, const double* rate) {
  if (n_points < 0 || (n_points > 0 && (!t || !rate)))
    return fail(HF_ERR_INVALID_ARG, "bad rain series");
  for (int64_t k = 1; k < n_points; ++k)
    if (!(t[k] >= t[k - 1])) return fail(HF_ERR_INVALID_ARG, "rain time stamps must be sorted");
  f.release_rain();
  if (n_points == 0) return HF_OK;
  HF_TRY(dalloc(&f.d_rain_t, (size_t)n_points));
  HF_TRY(dalloc(&f.d_rain_v, (size_t)n_points));
  HF_CUDA(cudaMemcpy(f.d_rain_t, t, n_points * sizeof(double), cudaMemcpyHostToDevice));
  HF_CUDA(cudaMemcpy(f.d_rain_v, rate, n_points * sizeof(double), cudaMemcpyHostToDevice));
  f.n_rain = (int)n_points;
  return HF_OK;
}

int hf::forcing_set_sources(ForcingHost& f, int64_t nr, int64_t nc, int64_t n_sources,
                            const int64_t* rows, const int64_t* cols, const int64_t* offsets,
                            const double* t, const double* q) {
  if (n_sources < 0) return fail(HF_ERR_INVALID_ARG, "bad point sources");
  if (n_sources > 0 && (!rows || !cols || !offsets || !t || !q))
    return fail(HF_ERR_INVALID_ARG, "null point-source arrays");
  for (int64_t k = 0; k < n_sources; ++k) {
    if (rows[k] < 0 || rows[k] >= nr || cols[k] < 0 || cols[k] >= nc)
      return fail(HF_ERR_INVALID_ARG, "point source outside the mesh");
    if (offsets[k + 1] <= offsets[k] || offsets[k] < 0)
      return fail(HF_ERR_INVALID_ARG, "each point source needs at least one (t, q) point");
    for (int64_t p = offsets[k] + 1; p < offsets[k + 1]; ++p)
      if (!(t[p] >= t[p - 1])) return fail(HF_ERR_INVALID_ARG, "source time stamps must be sorted");
  }
  f.release_src();
  if (n_sources == 0) return HF_OK;
  const int ns = (int)n_sources;
  const int npts = (int)offsets[ns];
  std::vector<int> r(ns), c(ns), off(ns + 1);
  for (int k = 0; k < ns; ++k) {
    r[k] = (int)rows[k];
    c[k] = (int)cols[k];
  }
  for (int k = 0; k <= ns; ++k) off[k] = (int)offsets[k];
  // Bucket the sources by the stage tiles of each geometry and by strip
  // block, keeping their order within a bucket (repeated cells accumulate in
  // the caller's order).
  auto bucket = [&](int nbuckets, auto key, std::vector<int>& start, std::vector<int>& order) {
    start.assign(nbuckets + 1, 0);
    order.assign(ns, 0);
    for (int k = 0; k < ns; ++k) start[key(k) + 1]++;
    for (int k = 0; k < nbuckets; ++k) start[k + 1] += start[k];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int k = 0; k < ns; ++k) order[fill[key(k)]++] = k;
  };
  std::vector<int> start[2], order[2], bstart, border;
  const int tiles_x = tiles_along(nc, TX);
  int ntiles[2];
  for (int g = 0; g < 2; ++g) {
    const int th = kGeomTileH[g];
    ntiles[g] = tiles_x * tiles_along(nr, th);
    bucket(ntiles[g], [&](int k) { return (r[k] / th) * tiles_x + c[k] / TX; }, start[g],
           order[g]);
  }
  const int nb = strip_blocks(nr), nblk = strip_count(nc) * nb;
  bucket(nblk, [&](int k) { return (c[k] / TX) * nb + r[k] / STRIP_ROWS; }, bstart, border);
  HF_TRY(dalloc(&f.d_row, ns));
  HF_TRY(dalloc(&f.d_col, ns));
  HF_TRY(dalloc(&f.d_off, ns + 1));
  HF_TRY(dalloc(&f.d_st, npts));
  HF_TRY(dalloc(&f.d_sq, npts));
  for (int g = 0; g < 2; ++g) {
    HF_TRY(dalloc(&f.d_tile_start[g], ntiles[g] + 1));
    HF_TRY(dalloc(&f.d_tile_order[g], ns));
  }
  HF_TRY(dalloc(&f.d_blk_start, nblk + 1));
  HF_TRY(dalloc(&f.d_blk_order, ns));
  HF_TRY(dalloc(&f.d_dh, ns));
  HF_CUDA(cudaMemcpy(f.d_row, r.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
  HF_CUDA(cudaMemcpy(f.d_col, c.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
  HF_CUDA(cudaMemcpy(f.d_off, off.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice));
  HF_CUDA(cudaMemcpy(f.d_st, t, npts * sizeof(double), cudaMemcpyHostToDevice));
  HF_CUDA(cudaMemcpy(f.d_sq, q, npts * sizeof(double), cudaMemcpyHostToDevice));
  for (int g = 0; g < 2; ++g) {
    HF_CUDA(cudaMemcpy(f.d_tile_start[g], start[g].data(), (ntiles[g] + 1) * sizeof(int),
                       cudaMemcpyHostToDevice));
    HF_CUDA(cudaMemcpy(f.d_tile_order[g], order[g].data(), ns * sizeof(int),
                       cudaMemcpyHostToDevice));
  }
  HF_CUDA(cudaMemcpy(f.d_blk_start, bstart.data(), (nblk + 1) * sizeof(int),
                     cudaMemcpyHostToDevice));
  HF_CUDA(cudaMemcpy(f.d_blk_order, border.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
  HF_CUDA(cudaMemset(f.d_dh, 0, ns * sizeof(double)));
  f.n_src = ns;
  return HF_OK;
}

struct hf_sim {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t nr = 0, nc = 0;
  double dx = 1.0, dy = 1.0;
  int tiles_x = 0, tiles_y = 0, grid = 1, elem_grid = 1;
  hf_config cfg;
  double *d_z = nullptr, *d_n = nullptr;
  double *d_h = nullptr, *d_hu = nullptr, *d_hv = nullptr;
  double *d_h1 = nullptr, *d_hu1 = nullptr, *d_hv1 = nullptr;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;  // pinned mirror
  ForcingHost forcing;
  GaugeDev gauge{};  // n == 0: no gauges
  cudaGraphExec_t graphs[3] = {nullptr, nullptr, nullptr};
  // Tile geometry of the tile-shaped kernels (kGeomSmall / kGeomLarge) and
  // its entry points; tiles_x, tiles_y and grid are in its tiles.
  int geom = kGeomSmall;
  const GeomOps* ops = nullptr;
  // Stage kernel: HF_STAGE_TILE / HF_STAGE_TILE32 (k_stage_pf of the 32 x 8
  // or 32 x 32 geometry) or HF_STAGE_STRIP (k_stage_strip, with the TMA
  // descriptors of stage 1's and stage 2's inputs).
  int stage_kind = HF_STAGE_TILE;
  int strip_grid = 0;
  StripMaps maps[2];
  bool cfl_dirty = true;
  double last_dt = 0.0;
  double t = 0.0;
  uint64_t steps = 0;
  double err_dt = 0.0, err_t = 0.0;
  uint64_t err_step = 0;
};

static const int kChunk[3] = {1, 8, 64};

namespace {

StageArgs stage_args(const hf_sim* s, bool second) {
  StageArgs a;
  a.nr = (int)s->nr;
  a.nc = (int)s->nc;
  a.tiles_x = s->tiles_x;
  a.tiles_y = s->tiles_y;
  a.dx = s->dx;
  a.dy = s->dy;
  a.rx = hfa::make_recip(a.dx);
  a.ry = hfa::make_recip(a.dy);
  a.z = s->d_z;
  a.n = s->d_n;
  a.bc = to_bcdev(s->cfg.boundaries);
  a.ctrl = s->d_ctrl;
  a.dry_tol = s->cfg.friction_dry_tol;
  a.f = s->forcing.dev(s->geom);
  const bool ssp = s->cfg.integrator == HF_SSPRK2;
  if (!second) {  // U -> U1
    a.in_h = s->d_h; a.in_hu = s->d_hu; a.in_hv = s->d_hv;
    a.out_h = s->d_h1; a.out_hu = s->d_hu1; a.out_hv = s->d_hv1;
    a.combine = 0;
    a.finalize = 0;
  } else {  // SSP stage 2: U1 -> U (combine with U in place); FE finalize: U1 -> U
    a.in_h = s->d_h1; a.in_hu = s->d_hu1; a.in_hv = s->d_hv1;
    a.out_h = s->d_h; a.out_hu = s->d_hu; a.out_hv = s->d_hv;
    a.combine = ssp ? 1 : 0;
    a.finalize = 1;
  }
  a.un_h = s->d_h;
  a.un_hu = s->d_hu;
  a.un_hv = s->d_hv;
  return a;
}

// One stage of the simulation's step on its stage kernel.
int launch_sim_stage(hf_sim* s, bool second) {
  const StageArgs a = stage_args(s, second);
  if (s->stage_kind == HF_STAGE_STRIP)
    return launch_stage_strip(a, s->maps[second ? 1 : 0], s->strip_grid, s->stream);
  return s->ops->stage(a, s->grid, s->stream);
}

// Puts the tile-shaped kernels of the simulation on geometry `geom`.
void set_geom(hf_sim* s, int geom) {
  s->geom = geom;
  s->ops = &geom_ops(geom);
  s->tiles_x = tiles_along(s->nc, TX);
  s->tiles_y = tiles_along(s->nr, s->ops->tile_h);
  s->grid = s->ops->grid_size(s->tiles_x * s->tiles_y, s->device);
}

// Picks the stage kernel: the strip kernel where it is asked for and its TMA
// descriptors can be made, else the tile kernel of the geometry asked for;
// auto takes the tile kernel of the grid's geometry (geom_for: on B200 the
// tile kernel measured faster than the strip kernel on wet grids and as fast
// on mostly dry ones). The strip kernel's grids keep the 32 x 8 geometry for
// the CFL reduction and the forward-Euler finalize.
int choose_stage_kernel(hf_sim* s, int kind) {
  const int geom = kind == HF_STAGE_TILE32   ? kGeomLarge
                   : kind == HF_STAGE_AUTO ? geom_for(s->nr, s->nc)
                                           : kGeomSmall;
  set_geom(s, geom);
  s->stage_kind = geom == kGeomLarge ? HF_STAGE_TILE32 : HF_STAGE_TILE;
  if (kind != HF_STAGE_STRIP) return HF_OK;
  int g = strip_grid_size(s->nr, s->nc, s->device);
  if (g == 0) {  // a small grid: one CTA per block at most
    g = strip_grid_size(1 << 20, 1 << 12, s->device);
    const long long nq = (long long)strip_count(s->nc) * strip_blocks(s->nr);
    if (nq < g) g = (int)nq;
  }
  if (!(g > 0 && strip_maps(stage_args(s, false), s->maps[0]) &&
        strip_maps(stage_args(s, true), s->maps[1]))) {
    choose_stage_kernel(s, HF_STAGE_AUTO);
    return fail(HF_ERR_UNSUPPORTED,
                "the strip stage kernel needs an even column count and 16-byte aligned fields");
  }
  s->stage_kind = HF_STAGE_STRIP;
  s->strip_grid = g;
  return HF_OK;
}

int enqueue_step(hf_sim* s) {
  HF_TRY(launch_control(s->d_ctrl, s->dx, s->dy, s->forcing.dev(s->geom), s->stream));
  HF_TRY(launch_sim_stage(s, false));
  if (s->cfg.integrator == HF_SSPRK2)
    HF_TRY(launch_sim_stage(s, true));
  else
    HF_TRY(s->ops->finalize(stage_args(s, true), s->grid, s->stream));
  if (s->gauge.n > 0) HF_TRY(launch_gauges(s->d_ctrl, s->d_h, s->gauge, 0, s->stream));
  return HF_OK;
}

void release_gauges(hf_sim* s) {
  GaugeDev& g = s->gauge;
  for (void* p : {(void*)g.cell, (void*)g.peak, (void*)g.last, (void*)g.ser_t, (void*)g.ser_h,
                  (void*)g.count})
    dfree(p);
  g = GaugeDev{};
}

void drop_graphs(hf_sim* s) {
  for (auto& g : s->graphs) {
    if (g) graph_destroy(g);
    g = nullptr;
  }
}

int build_graph(hf_sim* s, int which) {
  if (s->graphs[which]) return HF_OK;
  cudaGraph_t graph = nullptr;
  HF_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int rc = HF_OK;
  for (int k = 0; k < kChunk[which] && rc == HF_OK; ++k) rc = enqueue_step(s);
  cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
  if (rc != HF_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  HF_CUDA(e);
  e = graph_instantiate(&s->graphs[which], graph);
  cudaGraphDestroy(graph);
  HF_CUDA(e);
  return HF_OK;
}

int refresh_cfl(hf_sim* s) {
  if (!s->cfl_dirty) return HF_OK;
  HF_CUDA(cudaMemsetAsync(&s->d_ctrl->sx_bits, 0, 3 * sizeof(unsigned long long), s->stream));
  StageArgs a = stage_args(s, false);
  HF_TRY(s->ops->cfl(a, 1, s->grid, s->stream));
  s->cfl_dirty = false;
  return HF_OK;
}

int read_ctrl(hf_sim* s) {
  HF_CUDA(cudaMemcpyAsync(s->h_ctrl, s->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream));
  HF_CUDA(cudaStreamSynchronize(s->stream));
  s->t = s->h_ctrl->t;
  s->steps = (uint64_t)s->h_ctrl->steps;
  return HF_OK;
}

int ctrl_status(hf_sim* s) {
  const Ctrl& c = *s->h_ctrl;
  if (c.status == 0) return HF_OK;
  s->err_dt = c.err_dt;
  s->err_t = c.err_t;
  s->err_step = (uint64_t)c.err_step;
  char buf[200];
  switch (c.status) {
    case HF_ERR_DEGENERATE_DT:
      std::snprintf(buf, sizeof buf, "degenerate time step dt = %g at t = %g (step %llu)", c.err_dt,
                    c.err_t, (unsigned long long)c.err_step);
      break;
    case HF_ERR_STEP_BUDGET:
      std::snprintf(buf, sizeof buf, "step budget exhausted: %llu steps, t = %g of %g s",
                    (unsigned long long)c.err_step, c.err_t, c.t_target);
      break;
    case HF_ERR_NONFINITE:
      std::snprintf(buf, sizeof buf, "non-finite depth in the state at t = %g (step %llu)", c.err_t,
                    (unsigned long long)c.err_step);
      break;
    default:
      std::snprintf(buf, sizeof buf, "device status %d", c.status);
  }
  return fail(c.status, buf);
}

int validate_config(const hf_config* cfg) {
  if (!cfg) return fail(HF_ERR_INVALID_ARG, "null config");
  if (!(cfg->cfl > 0.0 && cfg->cfl <= 1.0)) {
    char buf[96];
    std::snprintf(buf, sizeof buf, "invalid configuration: cfl must be in (0, 1], got %g", cfg->cfl);
    return fail(HF_ERR_INVALID_CONFIG, buf);
  }
  if (!(cfg->max_dt > 0.0)) {
    char buf[96];
    std::snprintf(buf, sizeof buf, "invalid configuration: max_dt must be positive, got %g",
                  cfg->max_dt);
    return fail(HF_ERR_INVALID_CONFIG, buf);
  }
  if (cfg->integrator != HF_FORWARD_EULER && cfg->integrator != HF_SSPRK2)
    return fail(HF_ERR_INVALID_CONFIG, "invalid configuration: unknown integrator");
  return HF_OK;
}

int upload3(hf_sim* s, const double* h, const double* hu, const double* hv) {
  const size_t bytes = (size_t)(s->nr * s->nc) * sizeof(double);
  HF_CUDA(cudaMemcpyAsync(s->d_h, h, bytes, cudaMemcpyHostToDevice, s->stream));
  HF_CUDA(cudaMemcpyAsync(s->d_hu, hu, bytes, cudaMemcpyHostToDevice, s->stream));
  HF_CUDA(cudaMemcpyAsync(s->d_hv, hv, bytes, cudaMemcpyHostToDevice, s->stream));
  HF_CUDA(cudaStreamSynchronize(s->stream));
  s->cfl_dirty = true;
  return HF_OK;
}

void destroy_sim(hf_sim* s) {
  if (!s) return;
  DeviceGuard g(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  s->forcing.release_rain();
  s->forcing.release_src();
  release_gauges(s);
  for (void* p : {(void*)s->d_z, (void*)s->d_n, (void*)s->d_h, (void*)s->d_hu, (void*)s->d_hv,
                  (void*)s->d_h1, (void*)s->d_hu1, (void*)s->d_hv1})
    pfree(p, s->stream);
  pfree(s->d_ctrl, s->stream);
  if (s->stream) cudaStreamSynchronize(s->stream);  // the frees complete before the stream goes
  pinned_ctrl_put(s->h_ctrl);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

}  // namespace

int hf::check_grid_config(const hf_config* cfg, int64_t nr, int64_t nc) {
  HF_TRY(check_shape(nr, nc));
  HF_TRY(validate_config(cfg));
  return check_bcs(cfg->boundaries, nr, nc);
}

extern "C" {

const char* hf_last_error(void) { return g_err.c_str(); }

int hf_abi_version(void) { return HF_ABI_VERSION; }

int hf_kernel_launches(uint64_t* count) {
  if (!count) return fail(HF_ERR_INVALID_ARG, "null count");
  *count = kernel_launch_count();
  return HF_OK;
}

void hf_config_default(hf_config* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->cfl = 0.4;
  cfg->integrator = HF_SSPRK2;
  cfg->check_finite = 0;
  hf_boundary w{HF_BC_WALL, 0, 0.0};
  cfg->boundaries = hf_boundaries{w, w, w, w};
  cfg->max_steps = 10000000ull;
  cfg->max_dt = 60.0;
  cfg->friction_dry_tol = 1.0e-6;
}

int hf_sim_create(const hf_mesh_desc* mesh, const double* h, const double* hu, const double* hv,
                  const hf_config* cfg, int device, hf_sim** out) {
  if (!mesh || !h || !hu || !hv || !out || !mesh->bed)
    return fail(HF_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  HF_TRY(check_shape(mesh->n_rows, mesh->n_cols));
  HF_TRY(validate_config(cfg));
  if (!(mesh->dx > 0.0) || !(mesh->dy > 0.0))
    return fail(HF_ERR_INVALID_ARG, "dx and dy must be strictly positive");
  HF_TRY(check_bcs(cfg->boundaries, mesh->n_rows, mesh->n_cols));
  const int64_t ncell = mesh->n_rows * mesh->n_cols;
  if (!mesh->manning && !(mesh->manning_uniform >= 0.0))
    return fail(HF_ERR_INVALID_ARG, "Manning n must be non-negative");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return fail(HF_ERR_CUDA, "no such CUDA device");
  }
  DeviceGuard guard(device);
  hf_sim* s = new hf_sim();
  s->device = device;
  s->nr = mesh->n_rows;
  s->nc = mesh->n_cols;
  s->dx = mesh->dx;
  s->dy = mesh->dy;
  s->cfg = *cfg;
  set_geom(s, geom_for(s->nr, s->nc));
  int rc = HF_OK;
  auto done = [&](int code) {
    if (code != HF_OK) destroy_sim(s);
    return code;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return done(cuda_fail(failed_call_error(), "cudaStreamCreate"));
  double** bufs[8] = {&s->d_z, &s->d_n, &s->d_h, &s->d_hu, &s->d_hv, &s->d_h1, &s->d_hu1, &s->d_hv1};
  for (double** b : bufs)
    if ((rc = palloc(b, (size_t)ncell, device, s->stream)) != HF_OK) return done(rc);
  if ((rc = palloc(reinterpret_cast<double**>(&s->d_ctrl),
                   (sizeof(Ctrl) + sizeof(double) - 1) / sizeof(double), device, s->stream)) !=
      HF_OK)
    return done(rc);
  // Stream-ordered allocations: usable from any stream once this completes.
  if (cudaStreamSynchronize(s->stream) != cudaSuccess)
    return done(cuda_fail(failed_call_error(), "pool allocation"));
  if ((rc = pinned_ctrl_get(&s->h_ctrl)) != HF_OK) return done(rc);
  const size_t bytes = (size_t)ncell * sizeof(double);
  if (cudaMemcpy(s->d_z, mesh->bed, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
    return done(cuda_fail(failed_call_error(), "copy bed"));
  if (mesh->manning) {
    if (cudaMemcpy(s->d_n, mesh->manning, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      return done(cuda_fail(failed_call_error(), "copy manning"));
  } else {
    std::vector<double> nn((size_t)ncell, mesh->manning_uniform);
    if (cudaMemcpy(s->d_n, nn.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      return done(cuda_fail(failed_call_error(), "copy manning"));
  }
  Ctrl c;
  std::memset(&c, 0, sizeof c);
  c.cfl = cfg->cfl;
  c.max_dt = cfg->max_dt;
  c.check_finite = cfg->check_finite;
  if (cudaMemcpy(s->d_ctrl, &c, sizeof c, cudaMemcpyHostToDevice) != cudaSuccess)
    return done(cuda_fail(failed_call_error(), "init ctrl"));
  if (mesh->manning) {  // n >= 0 at every cell, counted on the device into ctrl.nonfinite
    unsigned long long bad = 0;
    if ((rc = launch_count_bad_manning(ncell, s->d_n, &s->d_ctrl->nonfinite, s->stream)) ||
        cudaMemcpyAsync(&bad, &s->d_ctrl->nonfinite, sizeof bad, cudaMemcpyDeviceToHost,
                        s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
      return done(rc ? fail(rc, "Manning check") : cuda_fail(failed_call_error(), "Manning check"));
    if (bad)
      return done(fail(HF_ERR_INVALID_ARG, "Manning n must be non-negative at every cell"));
    if (cudaMemcpy(s->d_ctrl, &c, sizeof c, cudaMemcpyHostToDevice) != cudaSuccess)
      return done(cuda_fail(failed_call_error(), "init ctrl"));
  }
  if ((rc = upload3(s, h, hu, hv)) != HF_OK) return done(rc);
  if ((rc = choose_stage_kernel(s, HF_STAGE_AUTO)) != HF_OK) return done(rc);
  *out = s;
  return HF_OK;
}

int hf_sim_create_aos(const hf_mesh_desc* mesh, const double* hhuhv, const hf_config* cfg,
                      int device, hf_sim** out) {
  if (!mesh || !hhuhv) return fail(HF_ERR_INVALID_ARG, "null argument");
  HF_TRY(check_shape(mesh->n_rows, mesh->n_cols));
  const int64_t n = mesh->n_rows * mesh->n_cols;
  std::vector<double> h(n), hu(n), hv(n);
  for (int64_t k = 0; k < n; ++k) {
    h[k] = hhuhv[3 * k];
    hu[k] = hhuhv[3 * k + 1];
    hv[k] = hhuhv[3 * k + 2];
  }
  return hf_sim_create(mesh, h.data(), hu.data(), hv.data(), cfg, device, out);
}

int hf_sim_destroy(hf_sim* sim) {
  destroy_sim(sim);
  return HF_OK;
}

int hf_sim_step(hf_sim* s, double dt_cap, double* dt_out) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard(s->device);
  HF_TRY(refresh_cfl(s));
  HF_TRY(build_graph(s, 0));
  HF_TRY(launch_set_step(s->d_ctrl, dt_cap, s->cfg.cfl, s->cfg.max_dt, s->cfg.check_finite,
                         s->stream));
  HF_CUDA(graph_launch(s->graphs[0], s->stream));
  HF_TRY(read_ctrl(s));
  HF_TRY(ctrl_status(s));
  s->last_dt = s->h_ctrl->dt;
  if (dt_out) *dt_out = s->h_ctrl->dt;
  return HF_OK;
}

int hf_sim_run_until(hf_sim* s, double t_target) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard(s->device);
  if (!(s->t < t_target)) return HF_OK;
  HF_TRY(refresh_cfl(s));
  const long long budget =
      s->cfg.max_steps > (uint64_t)LLONG_MAX ? LLONG_MAX : (long long)s->cfg.max_steps;
  HF_TRY(launch_set_run(s->d_ctrl, t_target, budget, s->cfg.cfl, s->cfg.max_dt,
                        s->cfg.check_finite, 0, s->stream));
  while (true) {
    int which = 1;
    if (s->last_dt > 0.0) {
      const double est = (t_target - s->t) / s->last_dt;
      which = est <= 1.5 ? 0 : (est <= 12.0 ? 1 : 2);
    }
    const uint64_t steps_before = s->steps;
    HF_TRY(build_graph(s, which));
    HF_CUDA(graph_launch(s->graphs[which], s->stream));
    HF_TRY(read_ctrl(s));
    HF_TRY(ctrl_status(s));
    if (s->h_ctrl->dt > 0.0) s->last_dt = s->h_ctrl->dt;
    if (!(s->t < t_target)) break;
    if (s->steps == steps_before)  // a chunk that takes no step would repeat forever
      return fail(HF_ERR_TIMEOUT, "run_until made no progress: no step was taken in a chunk");
  }
  return HF_OK;
}

int hf_sim_run_steps(hf_sim* s, uint64_t n_steps, double t_target) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard(s->device);
  if (n_steps == 0 || !(s->t < t_target)) return HF_OK;
  HF_TRY(refresh_cfl(s));
  const long long budget = n_steps > (uint64_t)LLONG_MAX ? LLONG_MAX : (long long)n_steps;
  HF_TRY(launch_set_run(s->d_ctrl, t_target, budget, s->cfg.cfl, s->cfg.max_dt,
                        s->cfg.check_finite, 1, s->stream));
  uint64_t left = n_steps;
  for (int which = 2; which >= 0; --which) {
    const uint64_t k = left / (uint64_t)kChunk[which];
    if (k == 0) continue;
    HF_TRY(build_graph(s, which));
    for (uint64_t r = 0; r < k; ++r) HF_CUDA(graph_launch(s->graphs[which], s->stream));
    left -= k * (uint64_t)kChunk[which];
  }
  HF_TRY(read_ctrl(s));
  HF_TRY(ctrl_status(s));
  if (s->h_ctrl->dt > 0.0) s->last_dt = s->h_ctrl->dt;
  return HF_OK;
}

int hf_sim_run_steps_timed(hf_sim* s, uint64_t n_steps, double t_target, double* stage_ms,
                           uint64_t* stage_launches, double* total_ms) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard(s->device);
  if (stage_ms) *stage_ms = 0.0;
  if (stage_launches) *stage_launches = 0;
  if (total_ms) *total_ms = 0.0;
  if (n_steps == 0 || !(s->t < t_target)) return HF_OK;
  if (n_steps > 1000000) return fail(HF_ERR_INVALID_ARG, "n_steps too large for the timed run");
  HF_TRY(refresh_cfl(s));
  HF_TRY(launch_set_run(s->d_ctrl, t_target, (long long)n_steps, s->cfg.cfl, s->cfg.max_dt,
                        s->cfg.check_finite, 1, s->stream));
  const bool ssp = s->cfg.integrator == HF_SSPRK2;
  std::vector<cudaEvent_t> ev(3 * n_steps);
  for (auto& e : ev) HF_CUDA(cudaEventCreate(&e));
  int rc = HF_OK;
  for (uint64_t k = 0; k < n_steps && rc == HF_OK; ++k) {
    rc = launch_control(s->d_ctrl, s->dx, s->dy, s->forcing.dev(s->geom), s->stream);
    if (rc) break;
    cudaEventRecord(ev[3 * k], s->stream);
    rc = launch_sim_stage(s, false);
    if (rc) break;
    cudaEventRecord(ev[3 * k + 1], s->stream);
    rc = ssp ? launch_sim_stage(s, true) : s->ops->finalize(stage_args(s, true), s->grid, s->stream);
    cudaEventRecord(ev[3 * k + 2], s->stream);
    if (rc == HF_OK && s->gauge.n > 0)
      rc = launch_gauges(s->d_ctrl, s->d_h, s->gauge, 0, s->stream);
  }
  if (rc == HF_OK) rc = read_ctrl(s);
  if (rc == HF_OK) {
    double st = 0.0;
    uint64_t launches = 0;
    for (uint64_t k = 0; k < n_steps; ++k) {
      float a = 0.f, b = 0.f;
      cudaEventElapsedTime(&a, ev[3 * k], ev[3 * k + 1]);
      cudaEventElapsedTime(&b, ev[3 * k + 1], ev[3 * k + 2]);
      st += a;
      launches += 1;
      if (ssp) {
        st += b;
        launches += 1;
      }
    }
    float tot = 0.f;
    cudaEventElapsedTime(&tot, ev[0], ev[3 * n_steps - 1]);
    if (stage_ms) *stage_ms = st;
    if (stage_launches) *stage_launches = launches;
    if (total_ms) *total_ms = tot;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (rc != HF_OK) return rc;
  HF_TRY(ctrl_status(s));
  if (s->h_ctrl->dt > 0.0) s->last_dt = s->h_ctrl->dt;
  return HF_OK;
}

int hf_sim_time(const hf_sim* s, double* t) {
  if (!s || !t) return fail(HF_ERR_INVALID_ARG, "null argument");
  *t = s->t;
  return HF_OK;
}

int hf_sim_steps(const hf_sim* s, uint64_t* steps) {
  if (!s || !steps) return fail(HF_ERR_INVALID_ARG, "null argument");
  *steps = s->steps;
  return HF_OK;
}

int hf_sim_get_state(hf_sim* s, double* h, double* hu, double* hv) {
  if (!s || !h || !hu || !hv) return fail(HF_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(s->device);
  const size_t bytes = (size_t)(s->nr * s->nc) * sizeof(double);
  HF_CUDA(cudaMemcpyAsync(h, s->d_h, bytes, cudaMemcpyDeviceToHost, s->stream));
  HF_CUDA(cudaMemcpyAsync(hu, s->d_hu, bytes, cudaMemcpyDeviceToHost, s->stream));
  HF_CUDA(cudaMemcpyAsync(hv, s->d_hv, bytes, cudaMemcpyDeviceToHost, s->stream));
  HF_CUDA(cudaStreamSynchronize(s->stream));
  return HF_OK;
}

int hf_sim_set_state(hf_sim* s, const double* h, const double* hu, const double* hv) {
  if (!s || !h || !hu || !hv) return fail(HF_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(s->device);
  return upload3(s, h, hu, hv);
}

int hf_sim_max_depth_exceeds_relief(hf_sim* s, double factor, int* exceeds) {
  if (!s || !exceeds) return fail(HF_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(s->device);
  *exceeds = 0;
  return relief_check(s->nr * s->nc, s->d_h, s->d_z, factor, s->d_ctrl, s->h_ctrl, s->stream,
                      exceeds);
}

int hf_sim_get_state_aos(hf_sim* s, double* hhuhv) {
  if (!s || !hhuhv) return fail(HF_ERR_INVALID_ARG, "null argument");
  const int64_t n = s->nr * s->nc;
  std::vector<double> h(n), hu(n), hv(n);
  HF_TRY(hf_sim_get_state(s, h.data(), hu.data(), hv.data()));
  for (int64_t k = 0; k < n; ++k) {
    hhuhv[3 * k] = h[k];
    hhuhv[3 * k + 1] = hu[k];
    hhuhv[3 * k + 2] = hv[k];
  }
  return HF_OK;
}

int hf_sim_set_state_aos(hf_sim* s, const double* hhuhv) {
  if (!s || !hhuhv) return fail(HF_ERR_INVALID_ARG, "null argument");
  const int64_t n = s->nr * s->nc;
  std::vector<double> h(n), hu(n), hv(n);
  for (int64_t k = 0; k < n; ++k) {
    h[k] = hhuhv[3 * k];
    hu[k] = hhuhv[3 * k + 1];
    hv[k] = hhuhv[3 * k + 2];
  }
  return hf_sim_set_state(s, h.data(), hu.data(), hv.data());
}

int hf_sim_set_boundaries(hf_sim* s, const hf_boundaries* bcs) {
  if (!s || !bcs) return fail(HF_ERR_INVALID_ARG, "null argument");
  HF_TRY(check_bcs(*bcs, s->nr, s->nc));
  DeviceGuard guard(s->device);
  cudaStreamSynchronize(s->stream);
  s->cfg.boundaries = *bcs;
  drop_graphs(s);
  s->cfl_dirty = true;  // ghost wave speeds depend on the boundaries
  return HF_OK;
}

int hf_sim_set_stage_kernel(hf_sim* s, int kind) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (kind != HF_STAGE_AUTO && kind != HF_STAGE_TILE && kind != HF_STAGE_STRIP &&
      kind != HF_STAGE_TILE32)
    return fail(HF_ERR_INVALID_ARG, "unknown stage kernel");
  DeviceGuard guard(s->device);
  cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  return choose_stage_kernel(s, kind);
}

int hf_sim_stage_kernel(const hf_sim* s, int* kind) {
  if (!s || !kind) return fail(HF_ERR_INVALID_ARG, "null argument");
  *kind = s->stage_kind;
  return HF_OK;
}

int hf_sim_error_detail(const hf_sim* s, double* dt, double* t, uint64_t* step) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (dt) *dt = s->err_dt;
  if (t) *t = s->err_t;
  if (step) *step = s->err_step;
  return HF_OK;
}

int hf_sim_device_state(hf_sim* s, double** h, double** hu, double** hv, void** stream) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (h) *h = s->d_h;
  if (hu) *hu = s->d_hu;
  if (hv) *hv = s->d_hv;
  if (stream) *stream = (void*)s->stream;
  return HF_OK;
}

int hf_sim_set_rain(hf_sim* s, int64_t n_points, const double* t, const double* rate) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard(s->device);
  cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  return forcing_set_rain(s->forcing, n_points, t, rate);
}

int hf_sim_set_point_sources(hf_sim* s, int64_t n_sources, const int64_t* rows,
                             const int64_t* cols, const int64_t* offsets, const double* t,
                             const double* q) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  DeviceGuard guard(s->device);
  cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  return forcing_set_sources(s->forcing, s->nr, s->nc, n_sources, rows,
                             cols, offsets, t, q);
}

int hf_sim_set_rain_units(hf_sim* s, double t_div, double v_mul, double v_div) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (!(std::isfinite(t_div) && t_div > 0.0 && std::isfinite(v_mul) && std::isfinite(v_div) &&
        v_div != 0.0))
    return fail(HF_ERR_INVALID_ARG, "series units: t_div must be finite and > 0, v_mul finite, "
                                    "v_div finite and non-zero");
  DeviceGuard guard(s->device);
  cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  s->forcing.rain_u = SeriesUnits{t_div, v_mul, v_div};
  return HF_OK;
}

int hf_sim_set_point_source_units(hf_sim* s, double t_div, double v_mul, double v_div) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (!(std::isfinite(t_div) && t_div > 0.0 && std::isfinite(v_mul) && std::isfinite(v_div) &&
        v_div != 0.0))
    return fail(HF_ERR_INVALID_ARG, "series units: t_div must be finite and > 0, v_mul finite, "
                                    "v_div finite and non-zero");
  DeviceGuard guard(s->device);
  cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  s->forcing.src_u = SeriesUnits{t_div, v_mul, v_div};
  return HF_OK;
}

int hf_sim_set_gauges(hf_sim* s, int64_t n_gauges, const int64_t* rows, const int64_t* cols,
                      int64_t capacity) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (n_gauges < 0 || n_gauges > (1 << 20) || capacity < 0 ||
      (n_gauges > 0 && (!rows || !cols)))
    return fail(HF_ERR_INVALID_ARG, "bad gauge arguments");
  if (n_gauges > 0 && capacity > (int64_t)(((size_t)1 << 40) / (size_t)(n_gauges + 1)))
    return fail(HF_ERR_INVALID_ARG, "gauge capacity too large");
  std::vector<long long> cell((size_t)n_gauges);
  for (int64_t k = 0; k < n_gauges; ++k) {
    if (rows[k] < 0 || rows[k] >= s->nr || cols[k] < 0 || cols[k] >= s->nc)
      return fail(HF_ERR_INVALID_ARG, "gauge " + std::to_string(k) + " (" +
                                          std::to_string(rows[k]) + ", " +
                                          std::to_string(cols[k]) + ") is outside the grid");
    cell[(size_t)k] = (long long)(rows[k] * s->nc + cols[k]);
  }
  DeviceGuard guard(s->device);
  cudaStreamSynchronize(s->stream);
  drop_graphs(s);
  release_gauges(s);
  if (n_gauges == 0) return HF_OK;
  GaugeDev g{};
  const size_t n = (size_t)n_gauges, cap = (size_t)capacity;
  int rc = dalloc((long long**)&g.cell, n);
  if (!rc) rc = dalloc(&g.peak, n);
  if (!rc) rc = dalloc(&g.last, n);
  if (!rc) rc = dalloc(&g.ser_t, std::max<size_t>(cap, 1));
  if (!rc) rc = dalloc(&g.ser_h, std::max<size_t>(cap * n, 1));
  if (!rc) rc = dalloc(&g.count, 1);
  g.n = (int)n_gauges;
  g.cap = (long long)capacity;
  s->gauge = g;
  if (rc) {
    release_gauges(s);
    return rc;
  }
  HF_CUDA(cudaMemcpyAsync((void*)g.cell, cell.data(), n * sizeof(long long),
                          cudaMemcpyHostToDevice, s->stream));
  HF_CUDA(cudaMemsetAsync(g.count, 0, sizeof(long long), s->stream));
  HF_TRY(launch_gauges(s->d_ctrl, s->d_h, s->gauge, 1, s->stream));
  HF_CUDA(cudaStreamSynchronize(s->stream));
  return HF_OK;
}

int hf_sim_gauge_peaks(hf_sim* s, double* peak, double* last) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (s->gauge.n == 0) return fail(HF_ERR_INVALID_ARG, "no gauges set");
  DeviceGuard guard(s->device);
  HF_CUDA(cudaStreamSynchronize(s->stream));
  const size_t bytes = (size_t)s->gauge.n * sizeof(double);
  if (peak) HF_CUDA(cudaMemcpy(peak, s->gauge.peak, bytes, cudaMemcpyDeviceToHost));
  if (last) HF_CUDA(cudaMemcpy(last, s->gauge.last, bytes, cudaMemcpyDeviceToHost));
  return HF_OK;
}

int hf_sim_gauge_series(hf_sim* s, double* t, double* h, int64_t* n_stored, int64_t* n_seen) {
  if (!s) return fail(HF_ERR_INVALID_ARG, "null handle");
  if (s->gauge.n == 0) return fail(HF_ERR_INVALID_ARG, "no gauges set");
  DeviceGuard guard(s->device);
  HF_CUDA(cudaStreamSynchronize(s->stream));
  long long count = 0;
  HF_CUDA(cudaMemcpy(&count, s->gauge.count, sizeof count, cudaMemcpyDeviceToHost));
  const long long stored = std::min(count, s->gauge.cap);
  if (n_stored) *n_stored = stored;
  if (n_seen) *n_seen = count;
  if (stored > 0 && t)
    HF_CUDA(cudaMemcpy(t, s->gauge.ser_t, (size_t)stored * sizeof(double),
                       cudaMemcpyDeviceToHost));
  if (stored > 0 && h)
    HF_CUDA(cudaMemcpy(h, s->gauge.ser_h, (size_t)stored * s->gauge.n * sizeof(double),
                       cudaMemcpyDeviceToHost));
  return HF_OK;
}

int hf_release_cached_memory(int device) {
  if (device < 0 || device >= 64) return fail(HF_ERR_INVALID_ARG, "bad device index");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (Ctrl* p : g_pinned_ctrl) cudaFreeHost(p);
  g_pinned_ctrl.clear();
  if (!g_pool[device]) return HF_OK;
  DeviceGuard guard(device);
  HF_CUDA(cudaDeviceSynchronize());
  HF_CUDA(cudaMemPoolTrimTo(g_pool[device], 0));
  return HF_OK;
}

// ------------------------------------------------------------ workspace
struct hf_workspace {
  int device = 0;
  int64_t nr = 0, nc = 0;
  double *d_h1 = nullptr, *d_hu1 = nullptr, *d_hv1 = nullptr;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;
};

int hf_workspace_create(int64_t n_rows, int64_t n_cols, int device, hf_workspace** out) {
  if (!out) return fail(HF_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  HF_TRY(check_shape(n_rows, n_cols));
  DeviceGuard guard(device);
  hf_workspace* w = new hf_workspace();
  w->device = device;
  w->nr = n_rows;
  w->nc = n_cols;
  const size_t n = (size_t)(n_rows * n_cols);
  int rc = HF_OK;
  if ((rc = dalloc(&w->d_h1, n)) || (rc = dalloc(&w->d_hu1, n)) || (rc = dalloc(&w->d_hv1, n)) ||
      (rc = dalloc(&w->d_ctrl, 1))) {
    hf_workspace_destroy(w);
    return rc;
  }
  if (cudaMallocHost((void**)&w->h_ctrl, sizeof(Ctrl)) != cudaSuccess) {
    hf_workspace_destroy(w);
    return cuda_fail(failed_call_error(), "cudaMallocHost");
  }
  Ctrl c;
  std::memset(&c, 0, sizeof c);
  cudaMemcpy(w->d_ctrl, &c, sizeof c, cudaMemcpyHostToDevice);
  *out = w;
  return HF_OK;
}

int hf_workspace_destroy(hf_workspace* w) {
  if (!w) return HF_OK;
  DeviceGuard guard(w->device);
  for (void* p : {(void*)w->d_h1, (void*)w->d_hu1, (void*)w->d_hv1, (void*)w->d_ctrl}) dfree(p);
  if (w->h_ctrl) cudaFreeHost(w->h_ctrl);
  delete w;
  return HF_OK;
}

namespace {

int check_grid(const hf_grid* g, hf_workspace* w) {
  if (!g) return fail(HF_ERR_INVALID_ARG, "null grid");
  HF_TRY(check_shape(g->n_rows, g->n_cols));
  // Mesh2D's own checks (geometry.rs:59, 93: dx, dy strictly positive).
  if (!(g->dx > 0.0) || !(g->dy > 0.0))
    return fail(HF_ERR_INVALID_ARG, "dx and dy must be strictly positive");
  if (w && (w->nr != g->n_rows || w->nc != g->n_cols)) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "workspace shape (%lld, %lld) must match mesh (%lld, %lld)",
                  (long long)w->nr, (long long)w->nc, (long long)g->n_rows, (long long)g->n_cols);
    return fail(HF_ERR_SHAPE_MISMATCH, buf);
  }
  return HF_OK;
}

// Stage arguments of a device grid in the tiles of geometry `o`.
StageArgs ws_args(const hf_grid* g, const hf_boundaries& bcs, hf_workspace* w,
                  const GeomOps& o) {
  StageArgs a;
  std::memset(&a, 0, sizeof a);
  a.nr = (int)g->n_rows;
  a.nc = (int)g->n_cols;
  a.tiles_x = tiles_along(g->n_cols, TX);
  a.tiles_y = tiles_along(g->n_rows, o.tile_h);
  a.dx = g->dx;
  a.dy = g->dy;
  a.rx = hfa::make_recip(a.dx);
  a.ry = hfa::make_recip(a.dy);
  a.z = g->bed;
  a.n = g->manning;
  a.bc = to_bcdev(bcs);
  a.ctrl = w ? w->d_ctrl : nullptr;
  return a;
}

hf_boundaries transmissive() {
  hf_boundary t{HF_BC_TRANSMISSIVE, 0, 0.0};
  return hf_boundaries{t, t, t, t};
}

int euler_like(const hf_grid* grid, double* h, double* hu, double* hv, const hf_boundaries* bcs,
               double dt, hf_workspace* w, void* stream, bool ssp) {
  HF_TRY(check_grid(grid, w));
  if (!w) return fail(HF_ERR_INVALID_ARG, "null workspace");
  if (!h || !hu || !hv || !grid->bed) return fail(HF_ERR_INVALID_ARG, "null buffer");
  const hf_boundaries b = bcs ? *bcs : transmissive();
  HF_TRY(check_bcs(b, grid->n_rows, grid->n_cols));
  DeviceGuard guard(w->device);
  const GeomOps& o = geom_ops(geom_for(grid->n_rows, grid->n_cols));
  StageArgs a = ws_args(grid, b, w, o);
  const int gsz = o.grid_size(a.tiles_x * a.tiles_y, w->device);
  HF_TRY(launch_set_fixed(w->d_ctrl, dt, stream));
  a.in_h = h; a.in_hu = hu; a.in_hv = hv;
  a.out_h = w->d_h1; a.out_hu = w->d_hu1; a.out_hv = w->d_hv1;
  a.un_h = h; a.un_hu = hu; a.un_hv = hv;
  HF_TRY(o.stage(a, gsz, stream));
  const size_t bytes = (size_t)(grid->n_rows * grid->n_cols) * sizeof(double);
  if (!ssp) {
    cudaStream_t st = (cudaStream_t)stream;
    HF_CUDA(cudaMemcpyAsync(h, w->d_h1, bytes, cudaMemcpyDeviceToDevice, st));
    HF_CUDA(cudaMemcpyAsync(hu, w->d_hu1, bytes, cudaMemcpyDeviceToDevice, st));
    HF_CUDA(cudaMemcpyAsync(hv, w->d_hv1, bytes, cudaMemcpyDeviceToDevice, st));
    return HF_OK;
  }
  a.in_h = w->d_h1; a.in_hu = w->d_hu1; a.in_hv = w->d_hv1;
  a.out_h = h; a.out_hu = hu; a.out_hv = hv;
  a.combine = 1;
  HF_TRY(o.stage(a, gsz, stream));
  return HF_OK;
}

}  // namespace

int hf_cfl_time_step(const hf_grid* grid, const double* h, const double* hu, const double* hv,
                     const hf_boundaries* bcs, double cfl, hf_workspace* w, void* stream,
                     double* dt_out) {
  HF_TRY(check_grid(grid, w));
  if (!w || !dt_out || !h || !hu || !hv) return fail(HF_ERR_INVALID_ARG, "null argument");
  if (bcs) {
    HF_TRY(check_bcs(*bcs, grid->n_rows, grid->n_cols));
    if (!grid->bed) return fail(HF_ERR_INVALID_ARG, "boundary ghosts need the bed");
  }
  DeviceGuard guard(w->device);
  cudaStream_t st = (cudaStream_t)stream;
  const GeomOps& o = geom_ops(geom_for(grid->n_rows, grid->n_cols));
  StageArgs a = ws_args(grid, bcs ? *bcs : transmissive(), w, o);
  a.in_h = h; a.in_hu = hu; a.in_hv = hv;
  HF_CUDA(cudaMemsetAsync(&w->d_ctrl->sx_bits, 0, 3 * sizeof(unsigned long long), st));
  HF_TRY(o.cfl(a, bcs ? 1 : 0, o.grid_size(a.tiles_x * a.tiles_y, w->device), stream));
  HF_CUDA(cudaMemcpyAsync(w->h_ctrl, w->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
  HF_CUDA(cudaStreamSynchronize(st));
  double sx, sy;
  std::memcpy(&sx, &w->h_ctrl->sx_bits, sizeof sx);
  std::memcpy(&sy, &w->h_ctrl->sy_bits, sizeof sy);
  const double denom = sx / grid->dx + sy / grid->dy;  // update.rs:152-158
  *dt_out = denom > 0.0 ? cfl / denom : INFINITY;
  return HF_OK;
}

int hf_max_depth_exceeds_relief(const hf_grid* grid, const double* h, double factor,
                                hf_workspace* w, void* stream, int* exceeds) {
  HF_TRY(check_grid(grid, w));
  if (!w || !h || !grid->bed || !exceeds) return fail(HF_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(w->device);
  *exceeds = 0;
  HF_TRY(relief_check(grid->n_rows * grid->n_cols, h, grid->bed, factor, w->d_ctrl, w->h_ctrl,
                      (cudaStream_t)stream, exceeds));
  return HF_OK;
}

int hf_forward_euler_step(const hf_grid* grid, double* h, double* hu, double* hv,
                          const hf_boundaries* bcs, double dt, hf_workspace* ws, void* stream) {
  return euler_like(grid, h, hu, hv, bcs, dt, ws, stream, false);
}

int hf_ssprk2_step(const hf_grid* grid, double* h, double* hu, double* hv,
                   const hf_boundaries* bcs, double dt, hf_workspace* ws, void* stream) {
  return euler_like(grid, h, hu, hv, bcs, dt, ws, stream, true);
}

int hf_manning_friction_step(const hf_grid* grid, double* h, double* hu, double* hv, double dt,
                             double dry_tol, void* stream) {
  HF_TRY(check_grid(grid, nullptr));
  if (!grid->manning || !h || !hu || !hv) return fail(HF_ERR_INVALID_ARG, "null buffer");
  return launch_friction(grid->n_rows * grid->n_cols, grid->manning, h, hu, hv, dt, dry_tol,
                         stream) ? cuda_fail(failed_call_error(), "friction") : HF_OK;
}

int hf_apply_rain(int64_t n_cells, double* h, double* hu, double* hv, double rate, double dt,
                  void* stream) {
  if (n_cells < 0 || (n_cells > 0 && (!h || !hu || !hv)))
    return fail(HF_ERR_INVALID_ARG, "bad arguments");
  return launch_rain(n_cells, h, hu, hv, rate, dt, stream) ? cuda_fail(failed_call_error(), "rain")
                                                           : HF_OK;
}

int hf_apply_point_sources(const hf_grid* grid, double* h, double* hu, double* hv,
                           int64_t n_sources, const int64_t* rows, const int64_t* cols,
                           const double* q_mass, double dt, void* stream) {
  HF_TRY(check_grid(grid, nullptr));
  if (n_sources < 0 || (n_sources > 0 && (!rows || !cols || !q_mass)))
    return fail(HF_ERR_INVALID_ARG, "bad point sources");
  for (int64_t k = 0; k < n_sources; ++k)
    if (rows[k] < 0 || rows[k] >= grid->n_rows || cols[k] < 0 || cols[k] >= grid->n_cols)
      return fail(HF_ERR_INVALID_ARG, "point source outside the mesh");
  if (n_sources > INT_MAX) return fail(HF_ERR_INVALID_ARG, "too many sources");
  return launch_point_sources(grid->n_cols, h, hu, hv, (int)n_sources, rows, cols, q_mass, dt,
                              grid->dx, grid->dy, stream)
             ? cuda_fail(failed_call_error(), "point sources")
             : HF_OK;
}

int hf_hllc_flux(int x_dir, int64_t n, const double* ul, const double* ur, double* flux,
                 void* stream) {
  if (n < 0 || (n > 0 && (!ul || !ur || !flux))) return fail(HF_ERR_INVALID_ARG, "bad arguments");
  return launch_hllc(x_dir, n, ul, ur, flux, stream) ? cuda_fail(failed_call_error(), "hllc")
                                                     : HF_OK;
}

}  // extern "C"

int hf::check_grid_desc(const hf_grid* g) { return check_grid(g, nullptr); }
