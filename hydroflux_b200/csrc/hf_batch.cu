// hf_batch.cu -- ensembles of independent scenarios in one launch per stage.
//
// All scenarios' fields live in one allocation (8 SoA fields x total cells,
// scenario k at offset off[k]); their tiles form one list, and a batch step
// is [per-scenario control -> stage 1 over every tile -> stage 2 over every
// tile -> per-scenario clock commit], replayed from CUDA graphs of 1, 8 and
// 64 batch steps. A small scenario no longer leaves most of the GPU idle or
// pays a launch per step: the persistent grid keeps every SM busy with tiles
// from whichever scenarios are still running.
//
// Schedules. How the CTAs walk the tile list is chosen by an online
// autotuner, since the best choice depends on the mix (sizes, wet fraction,
// horizons): {static stride, dynamic (atomic tile counter)} x {scenario
// order, largest scenarios first}. The first hf_batch_run with enough steps
// runs two rounds of 8-step graph chunks, one chunk per candidate in turn,
// timed with CUDA events, and keeps the fastest candidate. Tuning steps are
// real steps: the schedule changes no result.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydroflux_gpu.h"
#include "hf_internal.h"

using namespace hf;

namespace {

int bfail(int code, const std::string& m) { return record_error(code, m.c_str()); }

int bcuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HF_OK;
  cudaGetLastError();
  return bfail(e == cudaErrorMemoryAllocation ? HF_ERR_OUT_OF_MEMORY : HF_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}

#define B_CUDA(call)                              \
  do {                                            \
    cudaError_t _e = (call);                      \
    if (_e != cudaSuccess) return bcuda(_e, #call); \
  } while (0)
#define B_TRY(x)              \
  do {                        \
    int _rc = (x);            \
    if (_rc != 0) return _rc; \
  } while (0)

struct Guard {
  int prev = -1;
  explicit Guard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~Guard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

const int kBatchChunk[3] = {1, 8, 64};
constexpr int kSchedules = 4;  // bit 0: dynamic; bit 1: largest scenarios first

}  // namespace

struct hf_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  // Tile geometry of the batched kernels: 32 x 32 once the batched scenarios
  // have kLargeTilesMin such tiles between them, else 32 x 8.
  int geom = kGeomSmall;
  const GeomOps* ops = nullptr;
  // Scenarios of at least kSoloTilesMin tiles of 32 x 32 are not in the tile
  // lists: each stage runs them as their own k_stage_pf launches on 32 x 32
  // tiles, with these arguments (batched = 1) and grids.
  std::vector<int> solo;
  std::vector<StageArgs> solo_a1, solo_a2;
  std::vector<int> solo_grid;
  int n = 0;
  int64_t total_cells = 0;
  int total_tiles = 0;
  int grid = 1;
  double* buf = nullptr;
  double *h = nullptr, *hu = nullptr, *hv = nullptr, *h1 = nullptr, *hu1 = nullptr,
         *hv1 = nullptr, *z = nullptr, *nman = nullptr;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;
  StageArgs* d_args1 = nullptr;
  StageArgs* d_args2 = nullptr;
  int* d_tile_scn = nullptr;
  int* d_n_tiles = nullptr;  // device copy of total_tiles (read by the stage kernel)
  std::vector<ForcingHost> forcing;
  std::vector<int64_t> off, nr, nc;
  std::vector<double> t_end;
  // schedule tables: order 1 lists the scenarios largest first
  int* d_tile_scn_lpt = nullptr;
  int* d_tile_local = nullptr;      // tile index within its scenario, order 0
  int* d_tile_local_lpt = nullptr;  // order 1
  int* d_counters = nullptr;        // dynamic schedule: stage 1 / stage 2 tile counters
  // Scenarios still running when the tile lists were last built: finished
  // scenarios' tiles are dropped from the lists (they would only be skipped).
  int64_t listed = -1;
  std::vector<int> tiles_of;  // tiles per scenario
  cudaGraphExec_t graphs[kSchedules][3] = {};
  int schedule = -1;  // -1: not tuned yet
  int forced = -1;    // hf_batch_set_schedule
  double tune_ms[kSchedules] = {0.0, 0.0, 0.0, 0.0};
};

namespace {

void destroy_batch(hf_batch* b) {
  if (!b) return;
  Guard g(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& row : b->graphs)
    for (auto& ge : row)
      if (ge) graph_destroy(ge);
  for (auto& f : b->forcing) {
    f.release_rain();
    f.release_src();
  }
  for (void* p : {(void*)b->buf, (void*)b->d_ctrl, (void*)b->d_args1, (void*)b->d_args2,
                  (void*)b->d_tile_scn, (void*)b->d_n_tiles, (void*)b->d_tile_scn_lpt,
                  (void*)b->d_tile_local, (void*)b->d_tile_local_lpt, (void*)b->d_counters})
    if (p) cudaFree(p);
  if (b->h_ctrl) cudaFreeHost(b->h_ctrl);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int enqueue_batch_step(hf_batch* b, int sched) {
  const bool dynamic = sched & 1, lpt = sched & 2;
  const int* scn = lpt ? b->d_tile_scn_lpt : b->d_tile_scn;
  const int* local = lpt ? b->d_tile_local_lpt : b->d_tile_local;
  int* c1 = dynamic ? b->d_counters : nullptr;
  int* c2 = dynamic ? b->d_counters + 1 : nullptr;
  if (launch_batch_control(b->d_ctrl, b->d_args1, b->n, b->stream, dynamic ? b->d_counters : nullptr))
    return bcuda(failed_call_error(), "control");
  const GeomOps& large = geom_ops(kGeomLarge);
  if (b->ops->stage_batch(b->d_args1, scn, b->d_n_tiles, b->grid, b->stream, local, c1))
    return bcuda(failed_call_error(), "stage 1");
  for (size_t k = 0; k < b->solo.size(); ++k)
    if (large.stage(b->solo_a1[k], b->solo_grid[k], b->stream))
      return bcuda(failed_call_error(), "stage 1");
  if (b->ops->stage_batch(b->d_args2, scn, b->d_n_tiles, b->grid, b->stream, local, c2))
    return bcuda(failed_call_error(), "stage 2");
  for (size_t k = 0; k < b->solo.size(); ++k)
    if (large.stage(b->solo_a2[k], b->solo_grid[k], b->stream))
      return bcuda(failed_call_error(), "stage 2");
  if (launch_batch_commit(b->d_ctrl, b->n, b->stream)) return bcuda(failed_call_error(), "commit");
  return HF_OK;
}

int build_batch_graph(hf_batch* b, int sched, int which) {
  if (b->graphs[sched][which]) return HF_OK;
  cudaGraph_t graph = nullptr;
  B_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = HF_OK;
  for (int k = 0; k < kBatchChunk[which] && rc == HF_OK; ++k) rc = enqueue_batch_step(b, sched);
  cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (rc != HF_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  B_CUDA(e);
  e = graph_instantiate(&b->graphs[sched][which], graph);
  cudaGraphDestroy(graph);
  B_CUDA(e);
  return HF_OK;
}

long long total_steps(const hf_batch* b) {
  long long k = 0;
  for (int s = 0; s < b->n; ++s) k += b->h_ctrl[s].steps;
  return k;
}

int64_t count_unfinished(const hf_batch* b) {
  int64_t k = 0;
  for (int s = 0; s < b->n; ++s)
    if (b->h_ctrl[s].status == 0 && b->h_ctrl[s].t < b->t_end[s]) ++k;
  return k;
}

// Rebuilds the two tile lists (scenario order; largest first) over the
// scenarios that are still running, in place: the graphs read the lists and
// their length from device memory, so they stay valid. Results do not
// change: a finished scenario's tiles are skipped by the kernel anyway.
int compact_tile_lists(hf_batch* b) {
  std::vector<int> order0, order1, scn0, loc0, scn1, loc1;
  for (int s = 0; s < b->n; ++s)
    if (b->h_ctrl[s].status == 0 && b->h_ctrl[s].t < b->t_end[s]) order0.push_back(s);
  order1 = order0;
  std::stable_sort(order1.begin(), order1.end(),
                   [&](int x, int y) { return b->tiles_of[x] > b->tiles_of[y]; });
  for (int s : order0)
    for (int t = 0; t < b->tiles_of[s]; ++t) {
      scn0.push_back(s);
      loc0.push_back(t);
    }
  for (int s : order1)
    for (int t = 0; t < b->tiles_of[s]; ++t) {
      scn1.push_back(s);
      loc1.push_back(t);
    }
  const int nt = (int)scn0.size();
  if (nt > 0 &&
      (cudaMemcpy(b->d_tile_scn, scn0.data(), nt * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(b->d_tile_local, loc0.data(), nt * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(b->d_tile_scn_lpt, scn1.data(), nt * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(b->d_tile_local_lpt, loc1.data(), nt * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess))
    return bcuda(failed_call_error(), "compact tile lists");
  if (cudaMemcpy(b->d_n_tiles, &nt, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return bcuda(failed_call_error(), "compact tile lists");
  return HF_OK;
}

// One graph chunk of schedule `sched`, then the control blocks read back.
// elapsed_ms (optional): device time of the chunk.
int run_chunk(hf_batch* b, int sched, int which, int64_t* running, float* elapsed_ms) {
  const long long steps_before = total_steps(b);
  B_TRY(build_batch_graph(b, sched, which));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (elapsed_ms) {
    B_CUDA(cudaEventCreate(&e0));
    B_CUDA(cudaEventCreate(&e1));
    B_CUDA(cudaEventRecord(e0, b->stream));
  }
  B_CUDA(graph_launch(b->graphs[sched][which], b->stream));
  if (elapsed_ms) B_CUDA(cudaEventRecord(e1, b->stream));
  B_CUDA(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, b->n * sizeof(Ctrl), cudaMemcpyDeviceToHost, b->stream));
  B_CUDA(cudaStreamSynchronize(b->stream));
  if (elapsed_ms) {
    cudaEventElapsedTime(elapsed_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  *running = count_unfinished(b);
  if (*running > 0 && total_steps(b) == steps_before)  // would repeat forever
    return bfail(HF_ERR_TIMEOUT, "ensemble made no progress: no scenario took a step");
  if (*running > 0 && *running < b->listed) {
    B_TRY(compact_tile_lists(b));
    b->listed = *running;
  }
  return HF_OK;
}

}  // namespace

extern "C" {

int hf_batch_create(int64_t n_scenarios, const hf_scenario_desc* sc, int device, hf_batch** out) {
  if (!out || !sc || n_scenarios <= 0) return bfail(HF_ERR_INVALID_ARG, "bad arguments");
  if (n_scenarios > (1 << 24)) return bfail(HF_ERR_INVALID_ARG, "too many scenarios");
  *out = nullptr;
  int64_t total = 0, tiles = 0, tiles_large = 0;
  for (int64_t k = 0; k < n_scenarios; ++k) {
    const hf_scenario_desc& d = sc[k];
    if (!d.mesh.bed || !d.h || !d.hu || !d.hv) return bfail(HF_ERR_INVALID_ARG, "null scenario arrays");
    B_TRY(check_grid_config(&d.cfg, d.mesh.n_rows, d.mesh.n_cols));
    if (d.cfg.integrator != HF_SSPRK2)
      return bfail(HF_ERR_UNSUPPORTED, "ensembles run the SSP-RK2 integrator only");
    if (!(d.mesh.dx > 0.0) || !(d.mesh.dy > 0.0))
      return bfail(HF_ERR_INVALID_ARG, "dx and dy must be strictly positive");
    const int64_t nc = d.mesh.n_rows * d.mesh.n_cols;
    if (d.mesh.manning) {
      for (int64_t c = 0; c < nc; ++c)
        if (!(d.mesh.manning[c] >= 0.0))
          return bfail(HF_ERR_INVALID_ARG, "Manning n must be non-negative at every cell");
    } else if (!(d.mesh.manning_uniform >= 0.0)) {
      return bfail(HF_ERR_INVALID_ARG, "Manning n must be non-negative");
    }
    total += nc;
    const int64_t tx = tiles_along(d.mesh.n_cols, TX);
    const int64_t t32 = tx * tiles_along(d.mesh.n_rows, kGeomTileH[kGeomLarge]);
    if (t32 >= kSoloTilesMin) continue;  // runs its own launches
    tiles += tx * tiles_along(d.mesh.n_rows, kGeomTileH[kGeomSmall]);
    tiles_large += t32;
  }
  const int geom = tiles_large >= kLargeTilesMin ? kGeomLarge : kGeomSmall;
  if (geom == kGeomLarge) tiles = tiles_large;
  if (tiles > INT_MAX / 2) return bfail(HF_ERR_INVALID_ARG, "ensemble too large");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return bfail(HF_ERR_CUDA, "no such CUDA device");
  }
  Guard guard(device);
  hf_batch* b = new hf_batch();
  auto done = [&](int code) {
    if (code != HF_OK) destroy_batch(b);
    return code;
  };
  b->device = device;
  b->n = (int)n_scenarios;
  b->total_cells = total;
  b->total_tiles = (int)tiles;
  b->geom = geom;
  b->ops = &geom_ops(geom);
  b->grid = b->ops->grid_size(std::max(b->total_tiles, 1), device);
  b->forcing.resize(b->n);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return done(bcuda(failed_call_error(), "cudaStreamCreate"));
  if (cudaMalloc((void**)&b->buf, 8 * (size_t)total * sizeof(double)) != cudaSuccess)
    return done(bcuda(failed_call_error(), "cudaMalloc(ensemble fields)"));
  double* f = b->buf;
  b->h = f; b->hu = f + total; b->hv = f + 2 * total; b->h1 = f + 3 * total;
  b->hu1 = f + 4 * total; b->hv1 = f + 5 * total; b->z = f + 6 * total; b->nman = f + 7 * total;
  const size_t list_len = (size_t)std::max(b->total_tiles, 1);  // solo scenarios only: empty lists
  if (cudaMalloc((void**)&b->d_ctrl, b->n * sizeof(Ctrl)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_args1, b->n * sizeof(StageArgs)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_args2, b->n * sizeof(StageArgs)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_tile_scn, list_len * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_tile_scn_lpt, list_len * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_tile_local, list_len * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_tile_local_lpt, list_len * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_counters, 2 * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&b->d_n_tiles, sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void**)&b->h_ctrl, b->n * sizeof(Ctrl)) != cudaSuccess)
    return done(bcuda(failed_call_error(), "cudaMalloc(ensemble tables)"));
  std::vector<StageArgs> a1(b->n), a2(b->n);
  std::vector<int> tile_scn(b->total_tiles), tile_local(b->total_tiles);
  std::memset(b->h_ctrl, 0, b->n * sizeof(Ctrl));
  int64_t o = 0;
  int tb = 0;
  for (int s = 0; s < b->n; ++s) {
    const hf_scenario_desc& d = sc[s];
    const int64_t nr = d.mesh.n_rows, nc = d.mesh.n_cols, ncell = nr * nc;
    const size_t bytes = (size_t)ncell * sizeof(double);
    b->off.push_back(o);
    b->nr.push_back(nr);
    b->nc.push_back(nc);
    b->t_end.push_back(d.t_end);
    if (cudaMemcpy(b->z + o, d.mesh.bed, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->h + o, d.h, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->hu + o, d.hu, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->hv + o, d.hv, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      return done(bcuda(failed_call_error(), "upload scenario"));
    if (d.mesh.manning) {
      if (cudaMemcpy(b->nman + o, d.mesh.manning, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return done(bcuda(failed_call_error(), "upload manning"));
    } else {
      std::vector<double> nn((size_t)ncell, d.mesh.manning_uniform);
      if (cudaMemcpy(b->nman + o, nn.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return done(bcuda(failed_call_error(), "upload manning"));
    }
    const bool solo = (int64_t)tiles_along(nc, TX) * tiles_along(nr, kGeomTileH[kGeomLarge]) >=
                      kSoloTilesMin;
    const GeomOps& go = solo ? geom_ops(kGeomLarge) : *b->ops;
    const int tx = tiles_along(nc, TX), ty = tiles_along(nr, go.tile_h);
    int rc = forcing_set_rain(b->forcing[s], d.n_rain, d.rain_t, d.rain_rate);
    if (rc == HF_OK)
      rc = forcing_set_sources(b->forcing[s], nr, nc, d.n_sources, d.src_rows, d.src_cols,
                               d.src_offsets, d.src_t, d.src_q);
    if (rc != HF_OK) return done(rc);
    Ctrl& c = b->h_ctrl[s];
    c.cfl = d.cfg.cfl;
    c.max_dt = d.cfg.max_dt;
    c.check_finite = d.cfg.check_finite;
    c.mode = MODE_RUN;
    c.t_target = d.t_end;
    c.budget = d.cfg.max_steps > (uint64_t)LLONG_MAX ? LLONG_MAX : (long long)d.cfg.max_steps;
    StageArgs& x = a1[s];
    std::memset(&x, 0, sizeof x);
    x.nr = (int)nr;
    x.nc = (int)nc;
    x.tiles_x = tx;
    x.tiles_y = ty;
    x.tile_base = solo ? 0 : tb;
    x.batched = 1;
    x.dx = d.mesh.dx;
    x.dy = d.mesh.dy;
    x.rx = hfa::make_recip(x.dx);
    x.ry = hfa::make_recip(x.dy);
    x.z = b->z + o;
    x.n = b->nman + o;
    x.bc = boundaries_dev(d.cfg.boundaries);
    x.ctrl = b->d_ctrl + s;
    x.dry_tol = d.cfg.friction_dry_tol;
    x.f = b->forcing[s].dev(solo ? kGeomLarge : b->geom);
    StageArgs y = x;
    x.in_h = b->h + o; x.in_hu = b->hu + o; x.in_hv = b->hv + o;
    x.out_h = b->h1 + o; x.out_hu = b->hu1 + o; x.out_hv = b->hv1 + o;
    x.un_h = b->h + o; x.un_hu = b->hu + o; x.un_hv = b->hv + o;
    y.in_h = b->h1 + o; y.in_hu = b->hu1 + o; y.in_hv = b->hv1 + o;
    y.out_h = b->h + o; y.out_hu = b->hu + o; y.out_hv = b->hv + o;
    y.un_h = b->h + o; y.un_hu = b->hu + o; y.un_hv = b->hv + o;
    y.combine = 1;
    y.finalize = 1;
    a2[s] = y;
    o += ncell;
    if (solo) {
      b->solo.push_back(s);
      b->solo_a1.push_back(x);
      b->solo_a2.push_back(y);
      b->solo_grid.push_back(go.grid_size(tx * ty, device));
      b->tiles_of.push_back(0);
      continue;
    }
    for (int t = 0; t < tx * ty; ++t) {
      tile_scn[tb + t] = s;
      tile_local[tb + t] = t;
    }
    b->tiles_of.push_back(tx * ty);
    tb += tx * ty;
  }
  b->listed = b->n;
  // Order 1: the same tiles, scenarios by decreasing tile count (stable).
  std::vector<int> by_size(b->n), tile_scn_lpt, tile_local_lpt;
  for (int s = 0; s < b->n; ++s) by_size[s] = s;
  std::stable_sort(by_size.begin(), by_size.end(),
                   [&](int x, int y) { return b->tiles_of[x] > b->tiles_of[y]; });
  tile_scn_lpt.reserve(b->total_tiles);
  tile_local_lpt.reserve(b->total_tiles);
  for (int s : by_size)
    for (int t = 0; t < b->tiles_of[s]; ++t) {
      tile_scn_lpt.push_back(s);
      tile_local_lpt.push_back(t);
    }
  if (cudaMemcpy(b->d_args1, a1.data(), b->n * sizeof(StageArgs), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_args2, a2.data(), b->n * sizeof(StageArgs), cudaMemcpyHostToDevice) != cudaSuccess ||
      (b->total_tiles > 0 &&
       (cudaMemcpy(b->d_tile_scn, tile_scn.data(), b->total_tiles * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_tile_local, tile_local.data(), b->total_tiles * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_tile_scn_lpt, tile_scn_lpt.data(), b->total_tiles * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_tile_local_lpt, tile_local_lpt.data(), b->total_tiles * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)) ||
      cudaMemset(b->d_counters, 0, 2 * sizeof(int)) != cudaSuccess ||
      cudaMemcpy(b->d_n_tiles, &b->total_tiles, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_ctrl, b->h_ctrl, b->n * sizeof(Ctrl), cudaMemcpyHostToDevice) != cudaSuccess)
    return done(bcuda(failed_call_error(), "upload ensemble tables"));
  // CFL accumulators of every scenario from its initial state (with ghosts).
  if (b->ops->cfl_batch(b->d_args1, b->d_tile_scn, 0, b->total_tiles, b->grid, b->stream))
    return done(bcuda(failed_call_error(), "initial CFL"));
  for (size_t k = 0; k < b->solo.size(); ++k)
    if (geom_ops(kGeomLarge).cfl(b->solo_a1[k], 1, b->solo_grid[k], b->stream))
      return done(bcuda(failed_call_error(), "initial CFL"));
  if (cudaStreamSynchronize(b->stream) != cudaSuccess)
    return done(bcuda(failed_call_error(), "initial CFL"));
  *out = b;
  return HF_OK;
}

int hf_batch_destroy(hf_batch* b) {
  destroy_batch(b);
  return HF_OK;
}

int hf_batch_run(hf_batch* b, uint64_t max_batch_steps, int64_t* n_unfinished) {
  if (!b) return bfail(HF_ERR_INVALID_ARG, "null handle");
  Guard guard(b->device);
  uint64_t left = max_batch_steps;
  B_CUDA(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, b->n * sizeof(Ctrl), cudaMemcpyDeviceToHost, b->stream));
  B_CUDA(cudaStreamSynchronize(b->stream));
  int64_t running = count_unfinished(b);
  if (b->schedule < 0 && b->forced >= 0) b->schedule = b->forced;
  if (b->schedule < 0 && left >= (uint64_t)(2 * kSchedules * kBatchChunk[1]) && running > 0) {
    // Autotune: two rounds of one 8-step chunk per candidate, alternating so
    // that the flow's slow change over the rounds weighs on all of them.
    double ms[kSchedules] = {0.0, 0.0, 0.0, 0.0};
    int done_rounds = 0;
    for (int r = 0; r < 2 && running > 0; ++r) {
      double round_ms[kSchedules] = {0.0, 0.0, 0.0, 0.0};
      int ran = 0;
      for (int c = 0; c < kSchedules && running > 0; ++c, ++ran) {
        float el = 0.f;
        B_TRY(run_chunk(b, c, 1, &running, &el));
        left -= (uint64_t)kBatchChunk[1];
        round_ms[c] = el;
      }
      if (ran < kSchedules) break;  // the ensemble finished inside the round
      for (int c = 0; c < kSchedules; ++c) ms[c] += round_ms[c];
      ++done_rounds;
    }
    if (done_rounds > 0) {
      int best = 0;
      for (int c = 1; c < kSchedules; ++c)
        if (ms[c] < ms[best]) best = c;
      b->schedule = best;
      for (int c = 0; c < kSchedules; ++c) b->tune_ms[c] = ms[c];
    }
  }
  const int sched = b->schedule >= 0 ? b->schedule : 0;
  while (left > 0 && running > 0) {
    const int which = left >= 64 ? 2 : (left >= 8 ? 1 : 0);
    B_TRY(run_chunk(b, sched, which, &running, nullptr));
    left -= (uint64_t)kBatchChunk[which];
  }
  if (n_unfinished) *n_unfinished = running;
  return HF_OK;
}

int hf_batch_set_schedule(hf_batch* b, int schedule) {
  if (!b) return bfail(HF_ERR_INVALID_ARG, "null handle");
  if (schedule < -1 || schedule >= kSchedules)
    return bfail(HF_ERR_INVALID_ARG, "schedule must be -1 (autotune) or 0..3");
  b->forced = schedule;
  b->schedule = schedule;
  return HF_OK;
}

int hf_batch_schedule(const hf_batch* b, int* schedule, double* tune_ms) {
  if (!b) return bfail(HF_ERR_INVALID_ARG, "null handle");
  if (schedule) *schedule = b->schedule;
  if (tune_ms)
    for (int c = 0; c < kSchedules; ++c) tune_ms[c] = b->tune_ms[c];
  return HF_OK;
}

int hf_batch_scenario_info(const hf_batch* b, int64_t k, double* t, uint64_t* steps, int* status) {
  if (!b || k < 0 || k >= b->n) return bfail(HF_ERR_INVALID_ARG, "bad scenario index");
  const Ctrl& c = b->h_ctrl[k];
  if (t) *t = c.t;
  if (steps) *steps = (uint64_t)c.steps;
  if (status) *status = c.status;
  return HF_OK;
}

int hf_batch_get_state(hf_batch* b, int64_t k, double* h, double* hu, double* hv) {
  if (!b || k < 0 || k >= b->n || !h || !hu || !hv)
    return bfail(HF_ERR_INVALID_ARG, "bad arguments");
  Guard guard(b->device);
  const size_t bytes = (size_t)(b->nr[k] * b->nc[k]) * sizeof(double);
  const int64_t o = b->off[k];
  B_CUDA(cudaMemcpyAsync(h, b->h + o, bytes, cudaMemcpyDeviceToHost, b->stream));
  B_CUDA(cudaMemcpyAsync(hu, b->hu + o, bytes, cudaMemcpyDeviceToHost, b->stream));
  B_CUDA(cudaMemcpyAsync(hv, b->hv + o, bytes, cudaMemcpyDeviceToHost, b->stream));
  B_CUDA(cudaStreamSynchronize(b->stream));
  return HF_OK;
}

}  // extern "C"
