// hf_calib.cu -- gauge-misfit runs and their derivatives (hf_calib_*,
// hf_tangent, hf_grad_manning).
//
// One problem owns the device mesh, initial state, forcings, gauge cells and
// observations. A run is the same step sequence as hf_sim_run_until
// (control -> stage 1 -> stage 2 with the epilogue), plus two tiny record
// kernels per step (dt / start time before, gauge depths after).
//
// Tangent: the same sequence with the DualD stage kernels (values and
// tangents of h, hu, hv; the Manning tangent in the epilogue).
//
// Gradient: a primal run stores the state every C steps. The backward sweep
// takes the segments last to first: it replays the segment's steps from its
// checkpoint with the recorded dt (MODE_REPLAY), keeping every state U^k and
// stage-1 result U1^k of the segment, then walks the segment's steps
// backwards. Step k+1 in reverse is: rewind the control block to step k
// (which restores dt, rain and source increments) -> adjoint of stage 2
// (epilogue, combination, stage) -> gather into lambda(U1) and grad_n ->
// adjoint of stage 1 -> gather into lambda(U^k), adding the combination's
// share -> misfit seeds of step k. The replay of segment j-1 runs on its own
// stream (own control block and source increments) while segment j is
// reversed, in two alternating buffers: both kernels are latency-bound, so
// their CTAs share the SMs. Memory: checkpoints 24 B x cells x K / C, two
// segments 24 B x cells x (2C + 1) each, the adjoint buffers ~270 B per cell.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hydroflux_gpu.h"
#include "hf_internal.h"

using namespace hf;

// A calibration handle runs every kernel (forward solve, tangent, adjoint)
// on the 32 x 8 tiles of this build, with one tile numbering and one
// forcing table for all of them.
static_assert(TY == kGeomTileH[kGeomSmall], "calibration handles use the 32 x 8 geometry");

namespace {

int cfail(int code, const std::string& m) { return record_error(code, m.c_str()); }

int ccuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HF_OK;
  cudaGetLastError();
  return cfail(e == cudaErrorMemoryAllocation ? HF_ERR_OUT_OF_MEMORY : HF_ERR_CUDA,
               std::string(what) + ": " + cudaGetErrorString(e));
}

#define C_CUDA(call)                               \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return ccuda(_e, #call); \
  } while (0)
#define C_TRY(x)              \
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

// Device buffer of n elements (at least one), not initialised.
template <class T>
int alloc_dev(T** p, size_t n) {
  if (n == 0) n = 1;
  C_CUDA(cudaMalloc((void**)p, n * sizeof(T)));
  return HF_OK;
}

}  // namespace

struct hf_calib {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t nr = 0, nc = 0, ncell = 0;
  int tiles_x = 0, tiles_y = 0, ntiles = 0;
  int grid = 1, grid_dual = 1, grid_adj = 1;
  int grid_tiles = 1;  // one CTA per tile: the two backward streams share the SMs
  double dx = 1.0, dy = 1.0, t_end = 0.0;
  hf_config cfg;
  int64_t K = 0, G = 0, C = 1;
  double *z = nullptr, *n = nullptr, *dn = nullptr;
  double *h0 = nullptr, *hu0 = nullptr, *hv0 = nullptr;
  double* U[3] = {nullptr, nullptr, nullptr};
  double* U1[3] = {nullptr, nullptr, nullptr};
  double* dU[3] = {nullptr, nullptr, nullptr};
  double* dU1[3] = {nullptr, nullptr, nullptr};
  int64_t* cells = nullptr;
  double *gh = nullptr, *gdh = nullptr, *obs = nullptr;
  double *dts = nullptr, *ts = nullptr;
  Ctrl* ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;
  ForcingHost forcing;
  // adjoint buffers (allocated by the first gradient)
  double* ckpt = nullptr;
  double* seg = nullptr;   // segment buffers, alternating between segments
  double* seg2 = nullptr;
  cudaStream_t s_rec = nullptr, s_rev = nullptr;  // recompute / reverse streams
  Ctrl* ctrl_rec = nullptr;
  Ctrl* ctrl_rev = nullptr;
  double* dh_rev = nullptr;  // point-source increments of the reverse stream
  cudaEvent_t ev_primal = nullptr;
  cudaEvent_t ev_rec[2] = {nullptr, nullptr};
  cudaEvent_t ev_rev[2] = {nullptr, nullptr};
  double* lam[3] = {nullptr, nullptr, nullptr};
  double* lam1[3] = {nullptr, nullptr, nullptr};
  double* lamun[3] = {nullptr, nullptr, nullptr};
  double* grad = nullptr;
  double* halo = nullptr;
  int64_t last_run = 0;  // steps of the last run without replay
  bool have_dts = false;
  std::vector<double> obs_host;
  // vector-mode tangent (hf_tangent_lanes): lanes x cells per array
  int lanes_cap = 0, last_lanes = 0;
  double* dUL[3] = {nullptr, nullptr, nullptr};
  double* dU1L[3] = {nullptr, nullptr, nullptr};
  double* dnL = nullptr;
  double* gdhL = nullptr;                      // [lane][K][G]
  double* Ualt[3] = {nullptr, nullptr, nullptr};  // second value buffer (no in-place stage 2)
  // forward runs replayed from CUDA graphs: [mode][checkpoints][1 / 8 / 64 steps]
  cudaGraphExec_t fgraphs[3][2][3] = {};
  // vector-mode runs replayed from CUDA graphs of 2 / 8 / 64 steps, captured
  // for `lgraph_lanes` lanes. Every chunk is an even number of steps, so it
  // starts and ends with the values in U (the steps alternate U and Ualt).
  cudaGraphExec_t lgraphs[3] = {};
  int lgraph_lanes = 0;
};

namespace {

StageArgs calib_args(const hf_calib* c, double* const in[3], double* const out[3],
                     double* const un[3], int combine, int finalize, Ctrl* ctrl,
                     const ForcingDev& fd) {
  StageArgs a;
  a.nr = (int)c->nr;
  a.nc = (int)c->nc;
  a.tiles_x = c->tiles_x;
  a.tiles_y = c->tiles_y;
  a.tile_base = 0;
  a.batched = 0;
  a.dx = c->dx;
  a.dy = c->dy;
  a.rx = hfa::make_recip(a.dx);
  a.ry = hfa::make_recip(a.dy);
  a.z = c->z;
  a.n = c->n;
  a.in_h = in[0]; a.in_hu = in[1]; a.in_hv = in[2];
  a.out_h = out ? out[0] : nullptr;
  a.out_hu = out ? out[1] : nullptr;
  a.out_hv = out ? out[2] : nullptr;
  a.un_h = un ? un[0] : nullptr;
  a.un_hu = un ? un[1] : nullptr;
  a.un_hv = un ? un[2] : nullptr;
  a.bc = boundaries_dev(c->cfg.boundaries);
  a.ctrl = ctrl;
  a.combine = combine;
  a.finalize = finalize;
  a.dry_tol = c->cfg.friction_dry_tol;
  a.f = fd;
  return a;
}

void with_tangent(StageArgs& a, const hf_calib* c, double* const din[3], double* const dout[3],
                  double* const dun[3]) {
  a.tan.in_h = din[0]; a.tan.in_hu = din[1]; a.tan.in_hv = din[2];
  a.tan.out_h = dout[0]; a.tan.out_hu = dout[1]; a.tan.out_hv = dout[2];
  if (dun) {
    a.tan.un_h = dun[0]; a.tan.un_hu = dun[1]; a.tan.un_hv = dun[2];
  }
  a.tan.n = c->dn;
}

double* slot(double* base, int64_t k, int64_t f, int64_t ncell) {
  return base + (k * 3 + f) * ncell;
}

// Control block at the start of a run: MODE_RUN to t_end / K steps, or
// MODE_REPLAY of the recorded dt sequence.
int init_ctrl_on(hf_calib* c, Ctrl* ctrl, bool replay, cudaStream_t stream) {
  Ctrl h;
  std::memset(&h, 0, sizeof h);
  h.cfl = c->cfg.cfl;
  h.max_dt = c->cfg.max_dt;
  h.t_target = c->t_end;
  h.budget = (long long)c->K;
  h.mode = replay ? MODE_REPLAY : MODE_RUN;
  h.quiet_budget = 1;
  h.check_finite = c->cfg.check_finite;
  h.replay_dt = c->dts;
  h.replay_n = replay ? (long long)c->last_run : 0;
  C_CUDA(cudaMemcpyAsync(ctrl, &h, sizeof h, cudaMemcpyHostToDevice, stream));
  return HF_OK;
}

int init_ctrl(hf_calib* c, bool replay) { return init_ctrl_on(c, c->ctrl, replay, c->stream); }

int upload_manning(hf_calib* c, const double* manning) {
  if (!manning) return cfail(HF_ERR_INVALID_ARG, "null Manning field");
  for (int64_t k = 0; k < c->ncell; ++k)
    if (!(manning[k] >= 0.0) || !std::isfinite(manning[k]))
      return cfail(HF_ERR_INVALID_ARG, "Manning values must be finite and >= 0");
  C_CUDA(cudaMemcpyAsync(c->n, manning, c->ncell * sizeof(double), cudaMemcpyHostToDevice,
                         c->stream));
  return HF_OK;
}

int status_of_run(hf_calib* c, int64_t* n_run) {
  C_CUDA(cudaMemcpyAsync(c->h_ctrl, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, c->stream));
  C_CUDA(cudaStreamSynchronize(c->stream));
  const Ctrl& h = *c->h_ctrl;
  if (n_run) *n_run = (int64_t)h.steps;
  if (h.status != 0) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "misfit run failed with status %d at t = %g (step %lld)",
                  h.status, h.err_t, (long long)h.err_step);
    return cfail(h.status, buf);
  }
  return HF_OK;
}

// One forward run from the initial state. mode 0: primal with CFL dt (dt
// recorded), 1: replay of the recorded dt, 2: DualD tangent (dU holds the
// initial tangent; CFL dt from values, recorded). With checkpoints the state
// before every C-th step is stored.
const int kFwdChunk[3] = {1, 8, 64};
const int kLaneChunk[3] = {2, 8, 64};

// The launches of one forward step (see forward_run).
int enqueue_forward_step(hf_calib* c, int mode, bool checkpoints, const StageArgs& a1,
                         const StageArgs& a2, const ForcingDev& fd) {
  const bool replay = mode == 1, dual = mode == 2;
  const bool ssp = c->cfg.integrator == HF_SSPRK2;
  if (checkpoints)
    C_TRY(launch_calib_ckpt(c->ctrl, c->U[0], c->U[1], c->U[2], c->ckpt, (long long)c->C,
                            (long long)c->K, (long long)c->ncell, c->stream));
  C_TRY(launch_control(c->ctrl, c->dx, c->dy, fd, c->stream));
  if (!replay) C_TRY(launch_calib_pre(c->ctrl, c->dts, c->ts, (long long)c->K, c->stream));
  if (dual) {
    C_TRY(launch_stage_dual(a1, c->grid_dual, c->stream));
    if (ssp)
      C_TRY(launch_stage_dual(a2, c->grid_dual, c->stream));
    else
      C_TRY(launch_finalize_dual(a2, c->grid, c->stream));
  } else {
    C_TRY(launch_stage(a1, c->grid, c->stream));
    if (ssp)
      C_TRY(launch_stage(a2, c->grid, c->stream));
    else
      C_TRY(launch_finalize(a2, c->grid, c->stream));
  }
  C_TRY(launch_calib_post(c->ctrl, c->U[0], dual ? c->dU[0] : nullptr, c->cells, (int)c->G,
                          c->gh, c->gdh, (long long)c->K, c->stream));
  return HF_OK;
}

// One forward run from the initial state. mode 0: primal with CFL dt (dt
// recorded), 1: replay of the recorded dt, 2: DualD tangent (dU holds the
// initial tangent; CFL dt from values, recorded). With checkpoints the state
// before every C-th step is stored. The steps run from CUDA graphs of 64, 8
// and 1 steps (the buffers are fixed per problem, so a graph is captured
// once per mode); the control block is read back between graphs, and the
// launches stop once the run has ended.
int forward_run(hf_calib* c, int mode, bool checkpoints, int64_t* n_run) {
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  double* h0[3] = {c->h0, c->hu0, c->hv0};
  for (int f = 0; f < 3; ++f)
    C_CUDA(cudaMemcpyAsync(c->U[f], h0[f], bytes, cudaMemcpyDeviceToDevice, c->stream));
  const bool replay = mode == 1;
  const bool dual = mode == 2;
  C_TRY(init_ctrl(c, replay));
  const ForcingDev fd = c->forcing.dev(kGeomSmall);
  StageArgs a1 = calib_args(c, c->U, c->U1, nullptr, 0, 0, c->ctrl, fd);
  const bool ssp = c->cfg.integrator == HF_SSPRK2;
  StageArgs a2 = calib_args(c, c->U1, c->U, c->U, ssp ? 1 : 0, 1, c->ctrl, fd);
  if (dual) {
    with_tangent(a1, c, c->dU, c->dU1, nullptr);
    with_tangent(a2, c, c->dU1, c->dU, c->dU);
  }
  if (!replay) C_TRY(launch_cfl(a1, 1, c->grid, c->stream));
  const int64_t steps = replay ? c->last_run : c->K;
  int64_t k = 0;
  while (k < steps) {
    const int which = steps - k >= 64 ? 2 : (steps - k >= 8 ? 1 : 0);
    cudaGraphExec_t& ge = c->fgraphs[mode][checkpoints ? 1 : 0][which];
    if (!ge) {
      cudaGraph_t graph = nullptr;
      C_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int rc = HF_OK;
      for (int i = 0; i < kFwdChunk[which] && rc == HF_OK; ++i)
        rc = enqueue_forward_step(c, mode, checkpoints, a1, a2, fd);
      cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
      if (rc != HF_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      C_CUDA(e);
      e = graph_instantiate(&ge, graph);
      cudaGraphDestroy(graph);
      C_CUDA(e);
    }
    C_CUDA(graph_launch(ge, c->stream));
    k += kFwdChunk[which];
    if (k < steps) {  // stop launching once the run has ended
      C_CUDA(cudaMemcpyAsync(c->h_ctrl, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                             c->stream));
      C_CUDA(cudaStreamSynchronize(c->stream));
      if (!c->h_ctrl->active || c->h_ctrl->status != 0) break;
    }
  }
  int64_t run = 0;
  C_TRY(status_of_run(c, &run));
  if (!replay) {
    c->last_run = run;
    c->have_dts = true;
  }
  if (n_run) *n_run = run;
  return HF_OK;
}

// J (and dJ from gauge tangents) over `run` steps, summed on the host in
// step-major, gauge-minor order.
int misfit(hf_calib* c, int64_t run, bool with_tangent_, double* J, double* dJ,
           double* gauge_h_out) {
  const size_t n = (size_t)(run * c->G);
  std::vector<double> gh(n ? n : 1), gdh(with_tangent_ ? (n ? n : 1) : 1);
  if (n) {
    C_CUDA(cudaMemcpyAsync(gh.data(), c->gh, n * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    if (with_tangent_)
      C_CUDA(cudaMemcpyAsync(gdh.data(), c->gdh, n * sizeof(double), cudaMemcpyDeviceToHost,
                             c->stream));
    C_CUDA(cudaStreamSynchronize(c->stream));
  }
  double j = 0.0, dj = 0.0;
  for (int64_t k = 0; k < run; ++k)
    for (int64_t g = 0; g < c->G; ++g) {
      const size_t i = (size_t)(k * c->G + g);
      const double r = gh[i] - c->obs_host[i];
      j += r * r;
      if (with_tangent_) dj += 2.0 * r * gdh[i];
    }
  if (J) *J = j;
  if (dJ) *dJ = dj;
  if (gauge_h_out && n) std::memcpy(gauge_h_out, gh.data(), n * sizeof(double));
  return HF_OK;
}

int alloc_adjoint(hf_calib* c) {
  if (c->seg) return HF_OK;
  const int64_t n_ckpt = (c->K + c->C - 1) / c->C;
  C_TRY(alloc_dev(&c->ckpt, (size_t)(n_ckpt * 3 * c->ncell)));
  C_TRY(alloc_dev(&c->seg, (size_t)((2 * c->C + 1) * 3 * c->ncell)));
  C_TRY(alloc_dev(&c->seg2, (size_t)((2 * c->C + 1) * 3 * c->ncell)));
  C_TRY(alloc_dev(&c->ctrl_rec, 1));
  C_TRY(alloc_dev(&c->ctrl_rev, 1));
  C_TRY(alloc_dev(&c->dh_rev, (size_t)std::max(c->forcing.n_src, 1)));
  C_CUDA(cudaStreamCreateWithFlags(&c->s_rec, cudaStreamNonBlocking));
  C_CUDA(cudaStreamCreateWithFlags(&c->s_rev, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&c->ev_primal, &c->ev_rec[0], &c->ev_rec[1], &c->ev_rev[0], &c->ev_rev[1]})
    C_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  for (int f = 0; f < 3; ++f) {
    C_TRY(alloc_dev(&c->lam[f], (size_t)c->ncell));
    C_TRY(alloc_dev(&c->lam1[f], (size_t)c->ncell));
    C_TRY(alloc_dev(&c->lamun[f], (size_t)c->ncell));
  }
  C_TRY(alloc_dev(&c->grad, (size_t)c->ncell));
  C_TRY(alloc_dev(&c->halo, (size_t)c->ntiles * adj_halo_doubles_per_tile()));
  return HF_OK;
}

// Segment j of the last primal run covers steps [j C, min((j + 1) C, run)).
// Its buffer holds U^{k0+i} at slot i (i = 0..C) and the stage-1 result of
// step k0+i+1 at slot C+1+i.
double* seg_buf(hf_calib* c, int b) { return b ? c->seg2 : c->seg; }

// Replays segment j from its checkpoint into buffer b on the recompute
// stream (own control block and point-source increments).
int recompute_segment(hf_calib* c, int64_t j, int b) {
  const int64_t nb = c->ncell, k0 = j * c->C, k1 = std::min(k0 + c->C, c->last_run);
  const size_t bytes = (size_t)nb * sizeof(double);
  const bool ssp = c->cfg.integrator == HF_SSPRK2;
  double* buf = seg_buf(c, b);
  const ForcingDev fd = c->forcing.dev(kGeomSmall);
  cudaStream_t st = c->s_rec;
  for (int f = 0; f < 3; ++f)
    C_CUDA(cudaMemcpyAsync(slot(buf, 0, f, nb), slot(c->ckpt, j, f, nb), bytes,
                           cudaMemcpyDeviceToDevice, st));
  C_TRY(launch_calib_rewind(c->ctrl_rec, c->ts, (long long)k0, st));
  double *su[3], *su_next[3], *s1[3];
  for (int64_t i = 0; i < k1 - k0; ++i) {
    for (int f = 0; f < 3; ++f) {
      su[f] = slot(buf, i, f, nb);
      su_next[f] = slot(buf, i + 1, f, nb);
      s1[f] = slot(buf, c->C + 1 + i, f, nb);
    }
    C_TRY(launch_control(c->ctrl_rec, c->dx, c->dy, fd, st));
    C_TRY(launch_stage(calib_args(c, su, s1, nullptr, 0, 0, c->ctrl_rec, fd), c->grid_tiles, st));
    if (ssp)  // stage 2 writes U^{k+1} to the next slot (combining with U^k of this slot)
      C_TRY(launch_stage(calib_args(c, s1, su_next, su, 1, 1, c->ctrl_rec, fd), c->grid_tiles,
                         st));
    else
      C_TRY(launch_finalize(calib_args(c, s1, su_next, nullptr, 0, 1, c->ctrl_rec, fd),
                            c->grid_tiles, st));
  }
  C_CUDA(cudaEventRecord(c->ev_rec[b], st));
  return HF_OK;
}

// Walks segment j (in buffer b) backwards on the reverse stream.
int reverse_segment(hf_calib* c, int64_t j, int b) {
  const int64_t nb = c->ncell, k0 = j * c->C, k1 = std::min(k0 + c->C, c->last_run);
  const bool ssp = c->cfg.integrator == HF_SSPRK2;
  double* buf = seg_buf(c, b);
  ForcingDev fd = c->forcing.dev(kGeomSmall);
  fd.src_dh = c->dh_rev;
  cudaStream_t st = c->s_rev;
  const int nr = (int)c->nr, nc = (int)c->nc;
  C_CUDA(cudaStreamWaitEvent(st, c->ev_rec[b], 0));
  double *su[3], *s1[3];
  for (int64_t i = k1 - k0 - 1; i >= 0; --i) {
    const int64_t k = k0 + i;
    for (int f = 0; f < 3; ++f) {
      su[f] = slot(buf, i, f, nb);
      s1[f] = slot(buf, c->C + 1 + i, f, nb);
    }
    C_TRY(launch_calib_rewind(c->ctrl_rev, c->ts, (long long)k, st));
    C_TRY(launch_control(c->ctrl_rev, c->dx, c->dy, fd, st));
    if (ssp) {
      C_TRY(launch_stage_adj(calib_args(c, s1, nullptr, su, 1, 1, c->ctrl_rev, fd), c->lam[0],
                             c->lam[1], c->lam[2], c->lamun[0], c->lamun[1], c->lamun[2],
                             c->halo, c->grid_tiles, st));
      C_TRY(launch_adj_gather(nr, nc, c->tiles_x, c->tiles_y, c->halo, nullptr, nullptr, nullptr,
                              c->lam1[0], c->lam1[1], c->lam1[2], c->grad, st));
      C_TRY(launch_stage_adj(calib_args(c, su, nullptr, nullptr, 0, 0, c->ctrl_rev, fd),
                             c->lam1[0], c->lam1[1], c->lam1[2], nullptr, nullptr, nullptr,
                             c->halo, c->grid_tiles, st));
      C_TRY(launch_adj_gather(nr, nc, c->tiles_x, c->tiles_y, c->halo, c->lamun[0], c->lamun[1],
                              c->lamun[2], c->lam[0], c->lam[1], c->lam[2], c->grad, st));
    } else {
      C_TRY(launch_stage_adj(calib_args(c, su, nullptr, nullptr, 0, 1, c->ctrl_rev, fd),
                             c->lam[0], c->lam[1], c->lam[2], nullptr, nullptr, nullptr, c->halo,
                             c->grid_tiles, st));
      C_TRY(launch_adj_gather(nr, nc, c->tiles_x, c->tiles_y, c->halo, nullptr, nullptr, nullptr,
                              c->lam[0], c->lam[1], c->lam[2], c->grad, st));
    }
    if (k >= 1)
      C_TRY(launch_adj_seed(c->lam[0], c->cells, (int)c->G, c->gh + (k - 1) * c->G,
                            c->obs + (k - 1) * c->G, st));
  }
  C_CUDA(cudaEventRecord(c->ev_rev[b], st));
  return HF_OK;
}

// Backward sweep over the last primal run (checkpoints stored). Segments
// are taken last to first; segment j-1 is recomputed on the recompute
// stream while segment j is reversed, in alternating buffers.
int backward(hf_calib* c) {
  const int64_t run = c->last_run;
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  C_CUDA(cudaEventRecord(c->ev_primal, c->stream));
  C_CUDA(cudaStreamWaitEvent(c->s_rev, c->ev_primal, 0));
  C_CUDA(cudaStreamWaitEvent(c->s_rec, c->ev_primal, 0));
  for (int f = 0; f < 3; ++f) C_CUDA(cudaMemsetAsync(c->lam[f], 0, bytes, c->s_rev));
  C_CUDA(cudaMemsetAsync(c->grad, 0, bytes, c->s_rev));
  if (run > 0) {
    C_TRY(launch_adj_seed(c->lam[0], c->cells, (int)c->G, c->gh + (run - 1) * c->G,
                          c->obs + (run - 1) * c->G, c->s_rev));
    C_TRY(init_ctrl_on(c, c->ctrl_rec, true, c->s_rec));
    C_TRY(init_ctrl_on(c, c->ctrl_rev, true, c->s_rev));
    const int64_t n_seg = (run + c->C - 1) / c->C;
    bool used[2] = {false, false};
    C_TRY(recompute_segment(c, n_seg - 1, (int)((n_seg - 1) % 2)));
    for (int64_t j = n_seg - 1; j >= 0; --j) {
      if (j >= 1) {
        const int b = (int)((j - 1) % 2);
        if (used[b]) C_CUDA(cudaStreamWaitEvent(c->s_rec, c->ev_rev[b], 0));
        C_TRY(recompute_segment(c, j - 1, b));
      }
      C_TRY(reverse_segment(c, j, (int)(j % 2)));
      used[j % 2] = true;
    }
  }
  C_CUDA(cudaStreamSynchronize(c->s_rev));
  C_CUDA(cudaStreamSynchronize(c->s_rec));
  C_CUDA(cudaGetLastError());
  return HF_OK;
}

void destroy_calib(hf_calib* c) {
  if (!c) return;
  Guard g(c->device);
  for (cudaStream_t s : {c->stream, c->s_rec, c->s_rev})
    if (s) cudaStreamSynchronize(s);
  for (auto& m : c->fgraphs)
    for (auto& k : m)
      for (auto& g : k)
        if (g) graph_destroy(g);
  for (auto& g : c->lgraphs)
    if (g) graph_destroy(g);
  c->forcing.release_rain();
  c->forcing.release_src();
  std::vector<void*> ptrs = {c->z,    c->n,    c->dn,   c->h0,   c->hu0,  c->hv0,  c->cells,
                             c->gh,   c->gdh,  c->obs,  c->dts,  c->ts,   c->ctrl, c->ckpt,
                             c->seg,  c->seg2, c->grad, c->halo, c->ctrl_rec, c->ctrl_rev,
                             c->dh_rev};
  for (cudaEvent_t e : {c->ev_primal, c->ev_rec[0], c->ev_rec[1], c->ev_rev[0], c->ev_rev[1]})
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : {c->s_rec, c->s_rev})
    if (s) cudaStreamDestroy(s);
  for (int f = 0; f < 3; ++f)
    for (void* p : {(void*)c->U[f], (void*)c->U1[f], (void*)c->dU[f], (void*)c->dU1[f],
                    (void*)c->lam[f], (void*)c->lam1[f], (void*)c->lamun[f], (void*)c->dUL[f],
                    (void*)c->dU1L[f], (void*)c->Ualt[f]})
      ptrs.push_back(p);
  ptrs.push_back(c->dnL);
  ptrs.push_back(c->gdhL);
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->h_ctrl) cudaFreeHost(c->h_ctrl);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int upload_tangent_init(hf_calib* c, const double* dh0, const double* dhu0, const double* dhv0) {
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  const double* src[3] = {dh0, dhu0, dhv0};
  for (int f = 0; f < 3; ++f) {
    if (src[f])
      C_CUDA(cudaMemcpyAsync(c->dU[f], src[f], bytes, cudaMemcpyHostToDevice, c->stream));
    else
      C_CUDA(cudaMemsetAsync(c->dU[f], 0, bytes, c->stream));
  }
  return HF_OK;
}

void drop_lane_graphs(hf_calib* c) {
  for (auto& g : c->lgraphs)
    if (g) {
      graph_destroy(g);
      g = nullptr;
    }
  c->lgraph_lanes = 0;
}

void free_lanes(hf_calib* c) {
  drop_lane_graphs(c);  // they hold the lane buffers' addresses
  for (int f = 0; f < 3; ++f) {
    for (double** p : {&c->dUL[f], &c->dU1L[f]})
      if (*p) {
        cudaFree(*p);
        *p = nullptr;
      }
  }
  for (double** p : {&c->dnL, &c->gdhL})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  c->lanes_cap = 0;
}

int alloc_lanes(hf_calib* c, int lanes) {
  if (c->lanes_cap >= lanes) return HF_OK;
  C_CUDA(cudaStreamSynchronize(c->stream));
  free_lanes(c);
  const size_t n = (size_t)lanes * (size_t)c->ncell;
  for (int f = 0; f < 3; ++f) {
    C_TRY(alloc_dev(&c->dUL[f], n));
    C_TRY(alloc_dev(&c->dU1L[f], n));
    if (!c->Ualt[f]) C_TRY(alloc_dev(&c->Ualt[f], (size_t)c->ncell));
  }
  C_TRY(alloc_dev(&c->dnL, n));
  C_TRY(alloc_dev(&c->gdhL, (size_t)lanes * (size_t)std::max<int64_t>(c->K * c->G, 1)));
  c->lanes_cap = lanes;
  return HF_OK;
}

// Vector-mode tangent run: the mode-2 run of forward_run with `lanes`
// tangents at once (grid.y = lane). Lane 0 writes the values; stage 2
// writes them into the other value buffer (no in-place combination, since
// other lanes still read U^n), and the buffers swap after every step.
int forward_run_lanes(hf_calib* c, int lanes, int64_t* n_run) {
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  double* h0[3] = {c->h0, c->hu0, c->hv0};
  for (int f = 0; f < 3; ++f)
    C_CUDA(cudaMemcpyAsync(c->U[f], h0[f], bytes, cudaMemcpyDeviceToDevice, c->stream));
  C_TRY(init_ctrl(c, false));
  const ForcingDev fd = c->forcing.dev(kGeomSmall);
  const bool ssp = c->cfg.integrator == HF_SSPRK2;
  const long long stride = (long long)c->ncell;
  // One wave: lanes x grid CTAs within the resident capacity (a second,
  // partial wave would double the stage time).
  const int cap = stage_dual_grid_size(1 << 30, c->device);
  const int grid = std::max(1, std::min(c->ntiles, cap / lanes));
  double* const vU[3] = {c->U[0], c->U[1], c->U[2]};
  double* const vA[3] = {c->Ualt[0], c->Ualt[1], c->Ualt[2]};
  {
    StageArgs a0 = calib_args(c, vU, c->U1, nullptr, 0, 0, c->ctrl, fd);
    C_TRY(launch_cfl(a0, 1, c->grid, c->stream));
  }
  // One step from the values in `cur` to `nxt`.
  auto enqueue_lane_step = [&](double* const cur[3], double* const nxt[3]) -> int {
    StageArgs a1 = calib_args(c, cur, c->U1, nullptr, 0, 0, c->ctrl, fd);
    StageArgs a2 = calib_args(c, c->U1, nxt, cur, ssp ? 1 : 0, 1, c->ctrl, fd);
    with_tangent(a1, c, c->dUL, c->dU1L, nullptr);
    with_tangent(a2, c, c->dU1L, c->dUL, c->dUL);
    a1.tan.n = a2.tan.n = c->dnL;
    a1.tan.lane_stride = a2.tan.lane_stride = stride;
    C_TRY(launch_control(c->ctrl, c->dx, c->dy, fd, c->stream));
    C_TRY(launch_calib_pre(c->ctrl, c->dts, c->ts, (long long)c->K, c->stream));
    C_TRY(launch_stage_dual(a1, grid, c->stream, lanes));
    if (ssp)
      C_TRY(launch_stage_dual(a2, grid, c->stream, lanes));
    else
      C_TRY(launch_finalize_dual(a2, grid, c->stream, lanes));
    C_TRY(launch_calib_post(c->ctrl, nxt[0], c->dUL[0], c->cells, (int)c->G, c->gh, c->gdhL,
                            (long long)c->K, c->stream, lanes, stride));
    return HF_OK;
  };
  if (c->lgraph_lanes != lanes) {
    drop_lane_graphs(c);
    c->lgraph_lanes = lanes;
  }
  // Steps that find the run ended return at once and leave the buffers as
  // they are; the launches stop at the next chunk boundary.
  int64_t k = 0;
  while (k < c->K) {
    const int64_t left = c->K - k;
    if (left >= 2) {
      const int which = left >= 64 ? 2 : (left >= 8 ? 1 : 0);
      cudaGraphExec_t& ge = c->lgraphs[which];
      if (!ge) {
        cudaGraph_t graph = nullptr;
        C_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = HF_OK;
        for (int i = 0; i < kLaneChunk[which] && rc == HF_OK; ++i)
          rc = (i % 2 == 0) ? enqueue_lane_step(vU, vA) : enqueue_lane_step(vA, vU);
        cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
        if (rc != HF_OK) {
          if (graph) cudaGraphDestroy(graph);
          return rc;
        }
        C_CUDA(e);
        e = graph_instantiate(&ge, graph);
        cudaGraphDestroy(graph);
        C_CUDA(e);
      }
      C_CUDA(graph_launch(ge, c->stream));
      k += kLaneChunk[which];
    } else {  // the last step of an odd count; k is even, so the values are in U
      C_TRY(enqueue_lane_step(vU, vA));
      k += 1;
    }
    if (k < c->K) {
      C_CUDA(cudaMemcpyAsync(c->h_ctrl, c->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                             c->stream));
      C_CUDA(cudaStreamSynchronize(c->stream));
      if (!c->h_ctrl->active || c->h_ctrl->status != 0) break;
    }
  }
  int64_t run = 0;
  C_TRY(status_of_run(c, &run));
  c->last_run = run;
  c->have_dts = true;
  // The values after the last step taken: step j wrote buffer (j odd ? Ualt : U).
  if (run % 2 == 1)
    for (int f = 0; f < 3; ++f)
      C_CUDA(cudaMemcpyAsync(c->U[f], c->Ualt[f], bytes, cudaMemcpyDeviceToDevice, c->stream));
  if (n_run) *n_run = run;
  return HF_OK;
}

}  // namespace

extern "C" {

int hf_calib_create(const hf_scenario_desc* d, int64_t n_steps, int64_t n_gauges,
                    const int64_t* gauge_cells, int64_t checkpoint_every, int device,
                    hf_calib** out) {
  if (!d || !out) return cfail(HF_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (!d->h || !d->hu || !d->hv || !d->mesh.bed)
    return cfail(HF_ERR_INVALID_ARG, "scenario needs bed and initial state arrays");
  if (n_steps < 1) return cfail(HF_ERR_INVALID_ARG, "n_steps must be >= 1");
  if (n_gauges < 0 || (n_gauges > 0 && !gauge_cells))
    return cfail(HF_ERR_INVALID_ARG, "bad gauge list");
  if (checkpoint_every < 1) return cfail(HF_ERR_INVALID_ARG, "checkpoint_every must be >= 1");
  if (!(d->mesh.dx > 0.0) || !(d->mesh.dy > 0.0))
    return cfail(HF_ERR_INVALID_ARG, "cell sizes must be positive");
  C_TRY(check_grid_config(&d->cfg, d->mesh.n_rows, d->mesh.n_cols));
  const int64_t nr = d->mesh.n_rows, nc = d->mesh.n_cols, ncell = nr * nc;
  for (int64_t g = 0; g < n_gauges; ++g)
    if (gauge_cells[g] < 0 || gauge_cells[g] >= ncell)
      return cfail(HF_ERR_INVALID_ARG, "gauge cell outside the mesh");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return cfail(HF_ERR_CUDA, "no such CUDA device");
  }
  Guard guard(device);
  hf_calib* c = new hf_calib();
  c->device = device;
  c->nr = nr;
  c->nc = nc;
  c->ncell = ncell;
  c->dx = d->mesh.dx;
  c->dy = d->mesh.dy;
  c->t_end = d->t_end;
  c->cfg = d->cfg;
  c->K = n_steps;
  c->G = n_gauges;
  c->C = checkpoint_every;
  c->tiles_x = (int)((nc + TX - 1) / TX);
  c->tiles_y = (int)((nr + TY - 1) / TY);
  c->ntiles = c->tiles_x * c->tiles_y;
  c->obs_host.assign((size_t)(n_steps * n_gauges), 0.0);
  auto bail = [&](int rc) {
    destroy_calib(c);
    return rc;
  };
  const size_t bytes = (size_t)ncell * sizeof(double);
  int rc = HF_OK;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(ccuda(cudaErrorUnknown, "cudaStreamCreate"));
  for (double** p : {&c->z, &c->n, &c->dn, &c->h0, &c->hu0, &c->hv0})
    if ((rc = alloc_dev(p, (size_t)ncell))) return bail(rc);
  for (int f = 0; f < 3; ++f)
    for (double** p : {&c->U[f], &c->U1[f], &c->dU[f], &c->dU1[f]})
      if ((rc = alloc_dev(p, (size_t)ncell))) return bail(rc);
  const size_t kg = (size_t)(n_steps * n_gauges);
  if ((rc = alloc_dev(&c->cells, (size_t)n_gauges)) || (rc = alloc_dev(&c->gh, kg)) ||
      (rc = alloc_dev(&c->gdh, kg)) || (rc = alloc_dev(&c->obs, kg)) ||
      (rc = alloc_dev(&c->dts, (size_t)n_steps)) || (rc = alloc_dev(&c->ts, (size_t)n_steps)) ||
      (rc = alloc_dev(&c->ctrl, 1)))
    return bail(rc);
  if (cudaMallocHost((void**)&c->h_ctrl, sizeof(Ctrl)) != cudaSuccess)
    return bail(ccuda(cudaErrorMemoryAllocation, "cudaMallocHost"));
  std::vector<double> nn;
  const double* nptr = d->mesh.manning;
  if (!nptr) {
    nn.assign((size_t)ncell, d->mesh.manning_uniform);
    nptr = nn.data();
  }
  if (cudaMemcpy(c->z, d->mesh.bed, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->n, nptr, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->h0, d->h, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->hu0, d->hu, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->hv0, d->hv, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      (n_gauges && cudaMemcpy(c->cells, gauge_cells, n_gauges * sizeof(int64_t),
                              cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemset(c->obs, 0, (kg ? kg : 1) * sizeof(double)) != cudaSuccess ||
      cudaMemset(c->dn, 0, bytes) != cudaSuccess)
    return bail(ccuda(cudaErrorUnknown, "upload"));
  if ((rc = forcing_set_rain(c->forcing, d->n_rain, d->rain_t, d->rain_rate))) return bail(rc);
  if ((rc = forcing_set_sources(c->forcing, nr, nc, d->n_sources,
                                d->src_rows, d->src_cols, d->src_offsets, d->src_t, d->src_q)))
    return bail(rc);
  c->grid = stage_grid_size(c->ntiles, device);
  c->grid_dual = stage_dual_grid_size(c->ntiles, device);
  c->grid_adj = adj_grid_size(c->ntiles, device);  // also sets the kernel's smem limit
  c->grid_tiles = c->ntiles;
  if (cudaGetLastError() != cudaSuccess) return bail(cfail(HF_ERR_CUDA, "kernel attributes"));
  *out = c;
  return HF_OK;
}

int hf_calib_destroy(hf_calib* c) {
  destroy_calib(c);
  return HF_OK;
}

int hf_calib_set_observations(hf_calib* c, const double* h_obs) {
  if (!c || !h_obs) return cfail(HF_ERR_INVALID_ARG, "null argument");
  Guard g(c->device);
  const size_t n = (size_t)(c->K * c->G);
  std::memcpy(c->obs_host.data(), h_obs, n * sizeof(double));
  if (n) C_CUDA(cudaMemcpy(c->obs, h_obs, n * sizeof(double), cudaMemcpyHostToDevice));
  return HF_OK;
}

int hf_calib_run(hf_calib* c, const double* manning, int replay_dt, double* J, double* gauge_h,
                 int64_t* n_run) {
  if (!c) return cfail(HF_ERR_INVALID_ARG, "null problem");
  if (replay_dt && !c->have_dts)
    return cfail(HF_ERR_INVALID_ARG, "no recorded dt sequence to replay (run once without replay)");
  Guard g(c->device);
  C_TRY(upload_manning(c, manning));
  int64_t run = 0;
  C_TRY(forward_run(c, replay_dt ? 1 : 0, false, &run));
  if (n_run) *n_run = run;
  return misfit(c, run, false, J, nullptr, gauge_h);
}

int hf_tangent(hf_calib* c, const double* manning, const double* dn, const double* dh0,
               const double* dhu0, const double* dhv0, double* J, double* dJ) {
  if (!c) return cfail(HF_ERR_INVALID_ARG, "null problem");
  Guard g(c->device);
  C_TRY(upload_manning(c, manning));
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  if (dn)
    C_CUDA(cudaMemcpyAsync(c->dn, dn, bytes, cudaMemcpyHostToDevice, c->stream));
  else
    C_CUDA(cudaMemsetAsync(c->dn, 0, bytes, c->stream));
  C_TRY(upload_tangent_init(c, dh0, dhu0, dhv0));
  int64_t run = 0;
  C_TRY(forward_run(c, 2, false, &run));
  return misfit(c, run, true, J, dJ, nullptr);
}

int hf_tangent_lanes(hf_calib* c, const double* manning, int64_t n_lanes, const double* dn,
                     const double* dh0, const double* dhu0, const double* dhv0, double* J,
                     double* dJ) {
  if (!c) return cfail(HF_ERR_INVALID_ARG, "null problem");
  if (n_lanes < 1 || n_lanes > 1024)
    return cfail(HF_ERR_INVALID_ARG, "n_lanes must be in 1..1024");
  Guard g(c->device);
  C_TRY(upload_manning(c, manning));
  const int L = (int)n_lanes;
  C_TRY(alloc_lanes(c, L));
  const size_t n = (size_t)L * (size_t)c->ncell, bytes = n * sizeof(double);
  if (dn)
    C_CUDA(cudaMemcpyAsync(c->dnL, dn, bytes, cudaMemcpyHostToDevice, c->stream));
  else
    C_CUDA(cudaMemsetAsync(c->dnL, 0, bytes, c->stream));
  const double* src[3] = {dh0, dhu0, dhv0};
  for (int f = 0; f < 3; ++f) {
    if (src[f])
      C_CUDA(cudaMemcpyAsync(c->dUL[f], src[f], bytes, cudaMemcpyHostToDevice, c->stream));
    else
      C_CUDA(cudaMemsetAsync(c->dUL[f], 0, bytes, c->stream));
  }
  int64_t run = 0;
  C_TRY(forward_run_lanes(c, L, &run));
  c->last_lanes = L;
  // J from the gauge values, dJ per lane from that lane's gauge tangents,
  // in the same step-major, gauge-minor order as hf_tangent.
  const size_t m = (size_t)(run * c->G);
  std::vector<double> gh(m ? m : 1), gdh(m ? m * (size_t)L : 1);
  if (m) {
    C_CUDA(cudaMemcpyAsync(gh.data(), c->gh, m * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    for (int l = 0; l < L; ++l)
      C_CUDA(cudaMemcpyAsync(gdh.data() + (size_t)l * m, c->gdhL + (size_t)l * c->K * c->G,
                             m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    C_CUDA(cudaStreamSynchronize(c->stream));
  }
  double j = 0.0;
  for (size_t i = 0; i < m; ++i) {
    const double r = gh[i] - c->obs_host[i];
    j += r * r;
  }
  if (J) *J = j;
  if (dJ)
    for (int l = 0; l < L; ++l) {
      double dj = 0.0;
      for (size_t i = 0; i < m; ++i) dj += 2.0 * (gh[i] - c->obs_host[i]) * gdh[(size_t)l * m + i];
      dJ[l] = dj;
    }
  return HF_OK;
}

int hf_calib_lane_state(hf_calib* c, int64_t lane, double* dh, double* dhu, double* dhv) {
  if (!c) return cfail(HF_ERR_INVALID_ARG, "null problem");
  if (lane < 0 || lane >= c->last_lanes)
    return cfail(HF_ERR_INVALID_ARG, "no such lane in the last hf_tangent_lanes run");
  Guard g(c->device);
  C_CUDA(cudaStreamSynchronize(c->stream));
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  double* outs[3] = {dh, dhu, dhv};
  for (int f = 0; f < 3; ++f)
    if (outs[f])
      C_CUDA(cudaMemcpy(outs[f], c->dUL[f] + (size_t)lane * c->ncell, bytes,
                        cudaMemcpyDeviceToHost));
  return HF_OK;
}

int hf_grad_manning(hf_calib* c, const double* manning, double* J, double* grad_n,
                    double* grad_h0, double* grad_hu0, double* grad_hv0) {
  if (!c) return cfail(HF_ERR_INVALID_ARG, "null problem");
  Guard g(c->device);
  C_TRY(upload_manning(c, manning));
  C_TRY(alloc_adjoint(c));
  int64_t run = 0;
  C_TRY(forward_run(c, 0, true, &run));
  C_TRY(misfit(c, run, false, J, nullptr, nullptr));
  C_TRY(backward(c));
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  if (grad_n) C_CUDA(cudaMemcpy(grad_n, c->grad, bytes, cudaMemcpyDeviceToHost));
  double* outs[3] = {grad_h0, grad_hu0, grad_hv0};
  for (int f = 0; f < 3; ++f)
    if (outs[f]) C_CUDA(cudaMemcpy(outs[f], c->lam[f], bytes, cudaMemcpyDeviceToHost));
  return HF_OK;
}

int hf_calib_final_state(hf_calib* c, double* h, double* hu, double* hv, double* dh, double* dhu,
                         double* dhv) {
  if (!c) return cfail(HF_ERR_INVALID_ARG, "null problem");
  Guard g(c->device);
  const size_t bytes = (size_t)c->ncell * sizeof(double);
  double* outs[6] = {h, hu, hv, dh, dhu, dhv};
  double* srcs[6] = {c->U[0], c->U[1], c->U[2], c->dU[0], c->dU[1], c->dU[2]};
  C_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 6; ++k)
    if (outs[k]) C_CUDA(cudaMemcpy(outs[k], srcs[k], bytes, cudaMemcpyDeviceToHost));
  return HF_OK;
}

int hf_calib_dt(hf_calib* c, double* dts, int64_t* n) {
  if (!c) return cfail(HF_ERR_INVALID_ARG, "null problem");
  Guard g(c->device);
  if (n) *n = c->have_dts ? c->last_run : 0;
  if (dts && c->have_dts && c->last_run > 0)
    C_CUDA(cudaMemcpy(dts, c->dts, c->last_run * sizeof(double), cudaMemcpyDeviceToHost));
  return HF_OK;
}

}  // extern "C"
