// hf_serve.cu -- continuous batching of flood scenarios (hf_server_*).
//
// A server owns max_slots scenario slots. Per slot the device holds a control
// block and stage-1 / stage-2 arguments; the tiles of every admitted scenario
// form one device list whose length is also device-resident, so the CUDA
// graph of a batch step ([control over all slots -> stage 1 over the list ->
// stage 2 -> commit]) is captured once and serves any mix: admitting or
// collecting a scenario only rewrites the tables between graph chunks. Empty
// slots have a control block in MODE_FIXED, for which the control kernel
// never starts a step.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydroflux_gpu.h"
#include "hf_internal.h"

using namespace hf;

namespace {

int sfail(int code, const std::string& m) { return record_error(code, m.c_str()); }

int scuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HF_OK;
  cudaGetLastError();
  return sfail(e == cudaErrorMemoryAllocation ? HF_ERR_OUT_OF_MEMORY : HF_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}

#define S_CUDA(call)                               \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return scuda(_e, #call); \
  } while (0)
#define S_TRY(x)              \
  do {                        \
    int _rc = (x);            \
    if (_rc != 0) return _rc; \
  } while (0)

struct SGuard {
  int prev = -1;
  explicit SGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~SGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

const int kServeChunk[3] = {1, 8, 64};

struct Slot {
  bool used = false;
  bool finished = false;
  int64_t nr = 0, nc = 0;
  int tiles_x = 0, tiles_y = 0;
  double t_end = 0.0;
  size_t bytes = 0;
  double* buf = nullptr;  // h, hu, hv, h1, hu1, hv1, z, n
  ForcingHost forcing;
  StageArgs a1, a2;
  // At least kSoloTilesMin tiles: the stages run as the slot's own
  // k_stage_pf launches (grid solo_grid) instead of through the tile list.
  bool solo = false;
  int solo_grid = 0;
};

}  // namespace

struct hf_server {
  int device = 0;
  cudaStream_t stream = nullptr;
  // The server's batched kernels run on 32 x 32 tiles: a served mix is
  // dominated by the grids large enough to fill the GPU.
  int geom = kGeomLarge;
  const GeomOps* ops = nullptr;
  uint64_t budget = 0, in_use = 0;
  int max_slots = 0;
  int grid = 1;
  int tile_cap = 0;
  int n_tiles = 0;
  std::vector<Slot> slots;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;
  StageArgs* d_args1 = nullptr;
  StageArgs* d_args2 = nullptr;
  int* d_tile_scn = nullptr;
  int* d_n_tiles = nullptr;
  int* d_counters = nullptr;  // dynamic tile schedule: stage 1 / stage 2 counters
  cudaGraphExec_t graphs[3] = {nullptr, nullptr, nullptr};
  // Running solo slots; the graphs launch their stages, so they are rebuilt
  // when this set changes.
  std::vector<int> solo_set;
};

namespace {

void free_slot(Slot& s) {
  if (s.buf) cudaFree(s.buf);
  s.buf = nullptr;
  s.forcing.release_rain();
  s.forcing.release_src();
  s.used = false;
  s.finished = false;
}

void destroy_server(hf_server* v) {
  if (!v) return;
  SGuard g(v->device);
  if (v->stream) cudaStreamSynchronize(v->stream);
  for (auto& ge : v->graphs)
    if (ge) graph_destroy(ge);
  for (auto& s : v->slots) free_slot(s);
  for (void* p : {(void*)v->d_ctrl, (void*)v->d_args1, (void*)v->d_args2, (void*)v->d_tile_scn,
                  (void*)v->d_n_tiles, (void*)v->d_counters})
    if (p) cudaFree(p);
  if (v->h_ctrl) cudaFreeHost(v->h_ctrl);
  if (v->stream) cudaStreamDestroy(v->stream);
  delete v;
}

// Rebuild the tile list from the admitted, unfinished slots and upload the
// tables (no work in flight: called between graph chunks).
int rebuild_tiles(hf_server* v) {
  std::vector<int> scn, solo;
  scn.reserve(v->n_tiles + 1024);
  std::vector<StageArgs> a1(v->max_slots), a2(v->max_slots);
  for (int k = 0; k < v->max_slots; ++k) {
    Slot& s = v->slots[k];
    std::memset(&a1[k], 0, sizeof(StageArgs));
    std::memset(&a2[k], 0, sizeof(StageArgs));
    a1[k].ctrl = a2[k].ctrl = v->d_ctrl + k;
    if (!s.used) continue;
    s.a1.tile_base = s.a2.tile_base = s.solo ? 0 : (int)scn.size();
    if (!s.finished) {
      if (s.solo)
        solo.push_back(k);
      else
        for (int t = 0; t < s.tiles_x * s.tiles_y; ++t) scn.push_back(k);
    }
    a1[k] = s.a1;
    a2[k] = s.a2;
  }
  if (solo != v->solo_set) {  // the graphs launch the solo slots' stages: capture them again
    S_CUDA(cudaStreamSynchronize(v->stream));
    for (auto& ge : v->graphs) {
      if (ge) graph_destroy(ge);
      ge = nullptr;
    }
    v->solo_set = solo;
  }
  if ((int)scn.size() > v->tile_cap) return sfail(HF_ERR_CAPACITY, "tile list capacity exceeded");
  v->n_tiles = (int)scn.size();
  S_CUDA(cudaMemcpy(v->d_args1, a1.data(), v->max_slots * sizeof(StageArgs), cudaMemcpyHostToDevice));
  S_CUDA(cudaMemcpy(v->d_args2, a2.data(), v->max_slots * sizeof(StageArgs), cudaMemcpyHostToDevice));
  if (!scn.empty())
    S_CUDA(cudaMemcpy(v->d_tile_scn, scn.data(), scn.size() * sizeof(int), cudaMemcpyHostToDevice));
  S_CUDA(cudaMemcpy(v->d_n_tiles, &v->n_tiles, sizeof(int), cudaMemcpyHostToDevice));
  return HF_OK;
}

// The dynamic tile schedule (CTAs take tiles from a counter): on mixed
// ensembles it measured 5% faster than the static stride, and the mix of a
// server changes all the time.
int enqueue_serve_step(hf_server* v) {
  if (launch_batch_control(v->d_ctrl, v->d_args1, v->max_slots, v->stream, v->d_counters) ||
      v->ops->stage_batch(v->d_args1, v->d_tile_scn, v->d_n_tiles, v->grid, v->stream, nullptr,
                          v->d_counters))
    return scuda(failed_call_error(), "enqueue serve step");
  for (int k : v->solo_set)
    if (v->ops->stage(v->slots[k].a1, v->slots[k].solo_grid, v->stream))
      return scuda(failed_call_error(), "enqueue serve step");
  if (v->ops->stage_batch(v->d_args2, v->d_tile_scn, v->d_n_tiles, v->grid, v->stream, nullptr,
                          v->d_counters + 1))
    return scuda(failed_call_error(), "enqueue serve step");
  for (int k : v->solo_set)
    if (v->ops->stage(v->slots[k].a2, v->slots[k].solo_grid, v->stream))
      return scuda(failed_call_error(), "enqueue serve step");
  if (launch_batch_commit(v->d_ctrl, v->max_slots, v->stream))
    return scuda(failed_call_error(), "enqueue serve step");
  return HF_OK;
}

int build_serve_graph(hf_server* v, int which) {
  if (v->graphs[which]) return HF_OK;
  cudaGraph_t graph = nullptr;
  S_CUDA(cudaStreamBeginCapture(v->stream, cudaStreamCaptureModeThreadLocal));
  int rc = HF_OK;
  for (int k = 0; k < kServeChunk[which] && rc == HF_OK; ++k) rc = enqueue_serve_step(v);
  cudaError_t e = cudaStreamEndCapture(v->stream, &graph);
  if (rc != HF_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  S_CUDA(e);
  e = graph_instantiate(&v->graphs[which], graph);
  cudaGraphDestroy(graph);
  S_CUDA(e);
  return HF_OK;
}

// Marks newly finished slots from the host mirror; returns how many await collection.
int refresh_finished(hf_server* v) {
  int waiting = 0;
  for (int k = 0; k < v->max_slots; ++k) {
    Slot& s = v->slots[k];
    if (!s.used) continue;
    if (!s.finished && (v->h_ctrl[k].status != 0 || !(v->h_ctrl[k].t < s.t_end))) s.finished = true;
    if (s.finished) ++waiting;
  }
  return waiting;
}

}  // namespace

extern "C" {

int hf_server_create(int device, uint64_t hbm_budget_bytes, int max_slots, hf_server** out) {
  if (!out || max_slots <= 0 || max_slots > (1 << 20) || hbm_budget_bytes == 0)
    return sfail(HF_ERR_INVALID_ARG, "bad server arguments");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return sfail(HF_ERR_CUDA, "no such CUDA device");
  }
  SGuard guard(device);
  hf_server* v = new hf_server();
  auto done = [&](int code) {
    if (code != HF_OK) destroy_server(v);
    return code;
  };
  v->device = device;
  v->budget = hbm_budget_bytes;
  v->max_slots = max_slots;
  v->slots.resize(max_slots);
  v->ops = &geom_ops(v->geom);
  // Every tile holds at most TX * tile_h cells of 64 B; partial edge tiles
  // add at most (rows / tile_h + cols / TX + 1) per scenario, bounded here
  // generously.
  const uint64_t full_tiles = hbm_budget_bytes / (64ull * TX * v->ops->tile_h);
  const uint64_t cap = full_tiles + 4096ull * (uint64_t)max_slots;
  v->tile_cap = (int)std::min<uint64_t>(cap, (uint64_t)INT_MAX / 2);
  v->grid = v->ops->grid_size(std::max(v->tile_cap, 1), device);
  if (cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking) != cudaSuccess)
    return done(scuda(failed_call_error(), "cudaStreamCreate"));
  if (cudaMalloc((void**)&v->d_ctrl, max_slots * sizeof(Ctrl)) != cudaSuccess ||
      cudaMalloc((void**)&v->d_args1, max_slots * sizeof(StageArgs)) != cudaSuccess ||
      cudaMalloc((void**)&v->d_args2, max_slots * sizeof(StageArgs)) != cudaSuccess ||
      cudaMalloc((void**)&v->d_tile_scn, (size_t)v->tile_cap * sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&v->d_n_tiles, sizeof(int)) != cudaSuccess ||
      cudaMalloc((void**)&v->d_counters, 2 * sizeof(int)) != cudaSuccess ||
      cudaMallocHost((void**)&v->h_ctrl, max_slots * sizeof(Ctrl)) != cudaSuccess)
    return done(scuda(failed_call_error(), "cudaMalloc(server tables)"));
  std::memset(v->h_ctrl, 0, max_slots * sizeof(Ctrl));  // MODE_FIXED: empty
  if (cudaMemcpy(v->d_ctrl, v->h_ctrl, max_slots * sizeof(Ctrl), cudaMemcpyHostToDevice) != cudaSuccess)
    return done(scuda(failed_call_error(), "init slots"));
  int rc = rebuild_tiles(v);
  if (rc != HF_OK) return done(rc);
  *out = v;
  return HF_OK;
}

int hf_server_destroy(hf_server* v) {
  destroy_server(v);
  return HF_OK;
}

int hf_server_admit(hf_server* v, const hf_scenario_desc* d, int* slot_out) {
  if (!v || !d || !slot_out) return sfail(HF_ERR_INVALID_ARG, "null argument");
  if (!d->mesh.bed || !d->h || !d->hu || !d->hv) return sfail(HF_ERR_INVALID_ARG, "null scenario arrays");
  S_TRY(check_grid_config(&d->cfg, d->mesh.n_rows, d->mesh.n_cols));
  if (d->cfg.integrator != HF_SSPRK2)
    return sfail(HF_ERR_UNSUPPORTED, "the server runs the SSP-RK2 integrator only");
  if (!(d->mesh.dx > 0.0) || !(d->mesh.dy > 0.0))
    return sfail(HF_ERR_INVALID_ARG, "dx and dy must be strictly positive");
  const int64_t nr = d->mesh.n_rows, nc = d->mesh.n_cols, ncell = nr * nc;
  if (d->mesh.manning) {
    for (int64_t c = 0; c < ncell; ++c)
      if (!(d->mesh.manning[c] >= 0.0))
        return sfail(HF_ERR_INVALID_ARG, "Manning n must be non-negative at every cell");
  } else if (!(d->mesh.manning_uniform >= 0.0)) {
    return sfail(HF_ERR_INVALID_ARG, "Manning n must be non-negative");
  }
  const size_t bytes = 8 * (size_t)ncell * sizeof(double);
  int k = -1;
  for (int i = 0; i < v->max_slots; ++i)
    if (!v->slots[i].used) {
      k = i;
      break;
    }
  if (k < 0) return sfail(HF_ERR_CAPACITY, "no free slot");
  if (v->in_use + bytes > v->budget) return sfail(HF_ERR_CAPACITY, "over the HBM budget");
  SGuard guard(v->device);
  Slot& s = v->slots[k];
  if (cudaMalloc((void**)&s.buf, bytes) != cudaSuccess) {
    cudaGetLastError();
    return sfail(HF_ERR_CAPACITY, "device allocation failed");
  }
  s.used = true;
  s.finished = false;
  s.nr = nr;
  s.nc = nc;
  s.bytes = bytes;
  s.t_end = d->t_end;
  s.tiles_x = tiles_along(nc, TX);
  s.tiles_y = tiles_along(nr, v->ops->tile_h);
  s.solo = (int64_t)s.tiles_x * s.tiles_y >= kSoloTilesMin;
  s.solo_grid = s.solo ? v->ops->grid_size(s.tiles_x * s.tiles_y, v->device) : 0;
  auto undo = [&](int code) {
    free_slot(s);
    return code;
  };
  double* f = s.buf;
  double *h = f, *hu = f + ncell, *hv = f + 2 * ncell, *h1 = f + 3 * ncell, *hu1 = f + 4 * ncell,
         *hv1 = f + 5 * ncell, *z = f + 6 * ncell, *nm = f + 7 * ncell;
  const size_t fb = (size_t)ncell * sizeof(double);
  if (cudaMemcpy(z, d->mesh.bed, fb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h, d->h, fb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(hu, d->hu, fb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(hv, d->hv, fb, cudaMemcpyHostToDevice) != cudaSuccess)
    return undo(scuda(failed_call_error(), "upload scenario"));
  if (d->mesh.manning) {
    if (cudaMemcpy(nm, d->mesh.manning, fb, cudaMemcpyHostToDevice) != cudaSuccess)
      return undo(scuda(failed_call_error(), "upload manning"));
  } else {
    std::vector<double> nn((size_t)ncell, d->mesh.manning_uniform);
    if (cudaMemcpy(nm, nn.data(), fb, cudaMemcpyHostToDevice) != cudaSuccess)
      return undo(scuda(failed_call_error(), "upload manning"));
  }
  int rc = forcing_set_rain(s.forcing, d->n_rain, d->rain_t, d->rain_rate);
  if (rc == HF_OK)
    rc = forcing_set_sources(s.forcing, nr, nc, d->n_sources, d->src_rows,
                             d->src_cols, d->src_offsets, d->src_t, d->src_q);
  if (rc != HF_OK) return undo(rc);
  StageArgs& x = s.a1;
  std::memset(&x, 0, sizeof x);
  x.nr = (int)nr;
  x.nc = (int)nc;
  x.tiles_x = s.tiles_x;
  x.tiles_y = s.tiles_y;
  x.dx = d->mesh.dx;
  x.dy = d->mesh.dy;
  x.rx = hfa::make_recip(x.dx);
  x.ry = hfa::make_recip(x.dy);
  x.z = z;
  x.n = nm;
  x.bc = boundaries_dev(d->cfg.boundaries);
  x.ctrl = v->d_ctrl + k;
  x.batched = 1;
  x.dry_tol = d->cfg.friction_dry_tol;
  x.f = s.forcing.dev(v->geom);
  StageArgs y = x;
  x.in_h = h; x.in_hu = hu; x.in_hv = hv;
  x.out_h = h1; x.out_hu = hu1; x.out_hv = hv1;
  x.un_h = h; x.un_hu = hu; x.un_hv = hv;
  y.in_h = h1; y.in_hu = hu1; y.in_hv = hv1;
  y.out_h = h; y.out_hu = hu; y.out_hv = hv;
  y.un_h = h; y.un_hu = hu; y.un_hv = hv;
  y.combine = 1;
  y.finalize = 1;
  s.a2 = y;
  Ctrl c;
  std::memset(&c, 0, sizeof c);
  c.cfl = d->cfg.cfl;
  c.max_dt = d->cfg.max_dt;
  c.check_finite = d->cfg.check_finite;
  c.mode = MODE_RUN;
  c.t_target = d->t_end;
  c.budget = d->cfg.max_steps > (uint64_t)LLONG_MAX ? LLONG_MAX : (long long)d->cfg.max_steps;
  v->h_ctrl[k] = c;
  if (cudaMemcpy(v->d_ctrl + k, &c, sizeof c, cudaMemcpyHostToDevice) != cudaSuccess)
    return undo(scuda(failed_call_error(), "init slot"));
  rc = rebuild_tiles(v);
  if (rc != HF_OK) {
    undo(rc);
    rebuild_tiles(v);
    return rc;
  }
  // CFL accumulators of the new scenario from its initial state.
  const int tb = s.a1.tile_base;
  if ((s.solo ? v->ops->cfl(s.a1, 1, s.solo_grid, v->stream)
              : v->ops->cfl_batch(v->d_args1, v->d_tile_scn, tb, tb + s.tiles_x * s.tiles_y,
                                  v->grid, v->stream)) ||
      cudaStreamSynchronize(v->stream) != cudaSuccess)
    return scuda(failed_call_error(), "initial CFL");
  v->in_use += bytes;
  *slot_out = k;
  return HF_OK;
}

int hf_server_advance(hf_server* v, uint64_t n_batch_steps, int* n_finished) {
  if (!v) return sfail(HF_ERR_INVALID_ARG, "null handle");
  SGuard guard(v->device);
  int waiting = refresh_finished(v);
  uint64_t left = n_batch_steps;
  while (left > 0 && waiting == 0) {
    bool any = false;
    for (int k = 0; k < v->max_slots; ++k) any = any || (v->slots[k].used && !v->slots[k].finished);
    if (!any) break;
    const int which = left >= 64 ? 2 : (left >= 8 ? 1 : 0);
    long long before = 0;
    for (int k = 0; k < v->max_slots; ++k) before += v->h_ctrl[k].steps;
    S_TRY(build_serve_graph(v, which));
    S_CUDA(graph_launch(v->graphs[which], v->stream));
    left -= (uint64_t)kServeChunk[which];
    int top = 0;  // control blocks past the highest used slot are idle
    for (int k = 0; k < v->max_slots; ++k)
      if (v->slots[k].used) top = k + 1;
    S_CUDA(cudaMemcpyAsync(v->h_ctrl, v->d_ctrl, top * sizeof(Ctrl), cudaMemcpyDeviceToHost,
                           v->stream));
    S_CUDA(cudaStreamSynchronize(v->stream));
    waiting = refresh_finished(v);
    long long after = 0;
    for (int k = 0; k < v->max_slots; ++k) after += v->h_ctrl[k].steps;
    if (waiting == 0 && after == before)
      return sfail(HF_ERR_TIMEOUT, "server made no progress: no scenario took a step");
  }
  if (n_finished) *n_finished = waiting;
  return HF_OK;
}

int hf_server_finished(hf_server* v, int* slots, int cap, int* n) {
  if (!v || !n || (cap > 0 && !slots)) return sfail(HF_ERR_INVALID_ARG, "bad arguments");
  int m = 0;
  for (int k = 0; k < v->max_slots; ++k)
    if (v->slots[k].used && v->slots[k].finished) {
      if (m < cap) slots[m] = k;
      ++m;
    }
  *n = std::min(m, std::max(cap, 0));
  return HF_OK;
}

int hf_server_collect(hf_server* v, int k, double* h, double* hu, double* hv, double* t,
                      uint64_t* steps, int* status) {
  if (!v || k < 0 || k >= v->max_slots || !v->slots[k].used || !v->slots[k].finished)
    return sfail(HF_ERR_INVALID_ARG, "slot is not a finished scenario");
  SGuard guard(v->device);
  Slot& s = v->slots[k];
  const size_t fb = (size_t)(s.nr * s.nc) * sizeof(double);
  if (h) S_CUDA(cudaMemcpy(h, s.buf, fb, cudaMemcpyDeviceToHost));
  if (hu) S_CUDA(cudaMemcpy(hu, s.buf + s.nr * s.nc, fb, cudaMemcpyDeviceToHost));
  if (hv) S_CUDA(cudaMemcpy(hv, s.buf + 2 * s.nr * s.nc, fb, cudaMemcpyDeviceToHost));
  if (t) *t = v->h_ctrl[k].t;
  if (steps) *steps = (uint64_t)v->h_ctrl[k].steps;
  if (status) *status = v->h_ctrl[k].status;
  v->in_use -= s.bytes;
  free_slot(s);
  Ctrl c;
  std::memset(&c, 0, sizeof c);  // MODE_FIXED: the slot is empty again
  v->h_ctrl[k] = c;
  S_CUDA(cudaMemcpy(v->d_ctrl + k, &c, sizeof c, cudaMemcpyHostToDevice));
  return rebuild_tiles(v);
}

int hf_server_usage(const hf_server* v, uint64_t* bytes_in_use, int* occupied) {
  if (!v) return sfail(HF_ERR_INVALID_ARG, "null handle");
  if (bytes_in_use) *bytes_in_use = v->in_use;
  if (occupied) {
    int m = 0;
    for (const auto& s : v->slots) m += s.used ? 1 : 0;
    *occupied = m;
  }
  return HF_OK;
}

}  // extern "C"
