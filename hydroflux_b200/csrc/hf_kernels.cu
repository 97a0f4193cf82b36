// hf_kernels.cu -- sm_100a kernels of the solver-2d explicit step.
//
// The reference (franciscoparrao/hydroflux, solver-2d/src/update.rs:805-1211)
// runs one forward-Euler stage as eleven full-grid passes over a ~241 B/cell
// workspace. Here one stage is ONE kernel: a CTA stages a 32x8 tile plus a
// 4-cell halo of (h, z, eta, u, v) in shared memory and runs every pass of
// the stage on it -- dry snapshot, primitives, limited slopes, face beds,
// Audusse+HLLC faces, alpha rescaling, FV update with the bed source and the
// moisture floor -- so a stage reads the state once and writes it once. The
// last stage of a step also folds in the SSP-RK2 combination, Manning
// friction, rain, point sources and the next step's CFL reduction, and the
// step size never leaves the device (Ctrl).
//
// Compiled with --fmad=false and IEEE division / square root: every floating
// point operation rounds like the reference's Rust f64 code.
#include <cuda_runtime.h>

#include <type_traits>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "hf_device.cuh"
#include "hf_internal.h"
#include "hf_stage.cuh"
#include "hf_strip.cuh"

namespace hf {

// Blocks per SM the stage kernel is compiled for: the f64 tile takes 66 KB
// of shared memory (three CTAs per SM), the DualD tile 112 KB (two).
template <class T> struct StageOcc { static constexpr int value = HF_MIN_BLOCKS; };
template <> struct StageOcc<DualD> { static constexpr int value = 2; };

// The arguments of tangent lane `lane`: its tangent arrays, and no value
// outputs unless it is lane 0 (the values are the same in every lane).
__device__ void lane_args(const StageArgs& A, int lane, StageArgs& L) {
  L = A;
  if (lane == 0) return;
  const long long o = (long long)lane * A.tan.lane_stride;
  auto shift = [o](const double* p) { return p ? p + o : p; };
  auto shift_w = [o](double* p) { return p ? p + o : p; };
  L.tan.in_h = shift(A.tan.in_h);
  L.tan.in_hu = shift(A.tan.in_hu);
  L.tan.in_hv = shift(A.tan.in_hv);
  L.tan.out_h = shift_w(A.tan.out_h);
  L.tan.out_hu = shift_w(A.tan.out_hu);
  L.tan.out_hv = shift_w(A.tan.out_hv);
  L.tan.un_h = shift(A.tan.un_h);
  L.tan.un_hu = shift(A.tan.un_hu);
  L.tan.un_hv = shift(A.tan.un_hv);
  L.tan.n = shift(A.tan.n);
  L.out_h = L.out_hu = L.out_hv = nullptr;
}

template <class T>
__device__ __forceinline__ void stage_tile_any(const StageArgs& A, StageSmemT<T>& S, int tile,
                                               double& sxm, double& sym,
                                               unsigned long long& nonfin) {
  if (interior_tile(A, tile))
    stage_tile<T, false, true>(A, S, tile, sxm, sym, nonfin);
  else
    stage_tile<T>(A, S, tile, sxm, sym, nonfin);
}

// One stage of one grid over a persistent tile loop. For T = DualD,
// blockIdx.y is the tangent lane (vector mode); the CFL reduction and the
// clock belong to lane 0.
template <class T>
__global__ void __launch_bounds__(NTHREADS, StageOcc<T>::value) k_stage(const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StageSmemT<T>& S = *reinterpret_cast<StageSmemT<T>*>(smem_raw);
  if (!A.ctrl->active) return;
  const int ntiles = A.tiles_x * A.tiles_y;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
  if constexpr (std::is_same<T, DualD>::value) {
    __shared__ __align__(16) unsigned char lane_raw[sizeof(StageArgs)];
    StageArgs& L = *reinterpret_cast<StageArgs*>(lane_raw);
    if (threadIdx.x == 0) lane_args(A, blockIdx.y, L);
    __syncthreads();
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
      stage_tile_any<T>(L, S, tile, sxm, sym, nonfin);
  } else {
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
      stage_tile_any<T>(A, S, tile, sxm, sym, nonfin);
  }
  if (A.finalize && blockIdx.y == 0) {
    block_reduce_speeds(sxm, sym, nonfin, A.ctrl);
    if (blockIdx.x == 0 && threadIdx.x == 0) commit_clock(A.ctrl);
  }
}

// The f64 stage of one grid, software-pipelined: while a CTA computes the
// alpha and update phases of one tile, the raw inputs of its next tile are
// already being copied into shared memory (cp.async), so the next tile
// starts without waiting on global memory. Results are those of k_stage.
__global__ void __launch_bounds__(NTHREADS, HF_MIN_BLOCKS) k_stage_pf(const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StagePfSmem& P = *reinterpret_cast<StagePfSmem*>(smem_raw);
  if (!A.ctrl->active) return;
  const int ntiles = A.tiles_x * A.tiles_y;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
  if ((int)blockIdx.x < ntiles) stage_prefetch(A, P.s, P.hst, blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();
    const int next = tile + (int)gridDim.x < ntiles ? tile + (int)gridDim.x : -1;
    if (interior_tile(A, tile))
      stage_tile<double, true, true>(A, P.s, tile, sxm, sym, nonfin, P.hst, next);
    else
      stage_tile<double, true>(A, P.s, tile, sxm, sym, nonfin, P.hst, next);
  }
  if (A.finalize) {
    block_reduce_speeds(sxm, sym, nonfin, A.ctrl);
    if (blockIdx.x == 0 && threadIdx.x == 0) commit_clock(A.ctrl);
  }
}

// The f64 stage of one grid as a streaming walk down 32-column strips in
// blocks of STRIP_ROWS rows (hf_strip.cuh): a CTA takes a contiguous range
// of the strip-major block sequence, computes only the rows a block adds to
// the previous one, and fetches the next block's new input rows with TMA
// while it computes. Results are those of k_stage_pf.
//
// Schedule: while the grid is mostly wet, each CTA takes one equal range
// (no atomics, one cold block per range). When the previous step skipped
// more than 1/16 of the blocks as dry, the cost of a block depends on where
// the water is, so CTAs claim ranges of STRIP_CHUNK blocks from a counter
// instead. Either way every block is computed once, the same way.
constexpr int STRIP_CHUNK = 16;

__device__ __forceinline__ bool strip_range(const StageArgs& A, const StripMaps& M,
                                            StripSmem& S, long long q, long long q_end, int nb,
                                            unsigned& parity, double dt, double dt_dx,
                                            double dt_dy, double& sxm, double& sym,
                                            unsigned long long& nonfin) {
  bool cold = true;
  while (q < q_end) {
    const int strip = (int)(q / nb), b = (int)(q - (long long)strip * nb);
    const int gi0 = b * SR, gj0 = strip * TX;
    const bool in = interior_block(A, gi0, gj0);
    const bool next_warm = q + 1 < q_end && b + 1 < nb;
    if (cold) {
      if (next_warm && threadIdx.x == 0) strip_fetch(S, M, gi0 + SR, gj0);
      if (in) strip_cold<true>(A, S, gi0, gj0); else strip_cold<false>(A, S, gi0, gj0);
    }
    if (next_warm) {
      if (!strip_wait(S, parity, A.ctrl)) return false;
      parity ^= 1;
    }
    if (in) strip_alpha_prims<true>(A, S, gi0, gj0, cold ? -1 : 1, next_warm, dt_dx, dt_dy);
    else strip_alpha_prims<false>(A, S, gi0, gj0, cold ? -1 : 1, next_warm, dt_dx, dt_dy);
    __syncthreads();
    if (in) strip_update<true>(A, S, gi0, gj0, q, dt, dt_dx, dt_dy, sxm, sym, nonfin);
    else strip_update<false>(A, S, gi0, gj0, q, dt, dt_dx, dt_dy, sxm, sym, nonfin);
    __syncthreads();
    ++q;
    cold = !next_warm;
    if (cold) continue;
    strip_shift(S);
    __syncthreads();
    if (q + 1 < q_end && b + 2 < nb && threadIdx.x == 0) strip_fetch(S, M, gi0 + 2 * SR, gj0);
    if (interior_block(A, gi0 + SR, gj0)) strip_new_rows<true>(A, S, gi0 + SR, gj0);
    else strip_new_rows<false>(A, S, gi0 + SR, gj0);
  }
  return true;
}

__global__ void __launch_bounds__(NTHREADS, HF_MIN_BLOCKS)
    k_stage_strip(const StageArgs A, const __grid_constant__ StripMaps M) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StripSmem& S = *reinterpret_cast<StripSmem*>(
      smem_raw + ((128 - (smem_addr(smem_raw) & 127)) & 127));
  __shared__ long long s_claim;
  Ctrl* ctrl = A.ctrl;
  if (!ctrl->active) return;
  const int nb = strip_blocks(A.nr);
  const long long nq = (long long)strip_count(A.nc) * nb;
  const double dt = ctrl->dt;
  const double dt_dx = dt / A.dx;  // update.rs:930-931
  const double dt_dy = dt / A.dy;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
  if (threadIdx.x == 0) mbar_init(&S.mbar);
  __syncthreads();
  unsigned parity = 0;
  const bool dynamic = 16ull * ctrl->strip_dry_last > 2ull * (unsigned long long)nq;
  unsigned long long* counter = &ctrl->strip_claim[A.finalize ? 1 : 0];
  for (int round = 0;; ++round) {
    long long q0, q1;
    if (!dynamic) {
      if (round > 0) break;
      q0 = nq * blockIdx.x / gridDim.x;
      q1 = nq * (blockIdx.x + 1) / gridDim.x;
    } else {
      if (threadIdx.x == 0) s_claim = (long long)atomicAdd(counter, (unsigned long long)STRIP_CHUNK);
      __syncthreads();
      q0 = s_claim;
      __syncthreads();  // s_claim is read before the next claim overwrites it
      if (q0 >= nq) break;
      q1 = q0 + STRIP_CHUNK < nq ? q0 + STRIP_CHUNK : nq;
    }
    if (!strip_range(A, M, S, q0, q1, nb, parity, dt, dt_dx, dt_dy, sxm, sym, nonfin)) return;
  }
  if (A.finalize) {
    block_reduce_speeds(sxm, sym, nonfin, ctrl);
    if (blockIdx.x == 0 && threadIdx.x == 0) commit_clock(ctrl);
  }
}

// One stage of every grid of an ensemble in one launch: the persistent grid
// walks the concatenated tile list of all scenarios; tile t belongs to
// scenario tile_scn[t], whose arguments (own sizes, dt, forcings, control
// block) are args[tile_scn[t]]. Finished scenarios' tiles are skipped; each
// scenario's clock is committed afterwards by k_batch_commit.
//
// Schedules (the ensemble's autotuner picks one): tile_local == nullptr
// means tile t is tile t - tile_base of its scenario, else tile_local[t]
// (any order of the list); counter == nullptr strides the list statically
// (tile blockIdx.x, + gridDim.x, ...), else CTAs take the next tile from the
// counter (dynamic; k_batch_control zeroes it before each step). Results do
// not depend on the schedule: tiles are independent and the CFL reduction is
// a max.
//
// Either way the walk is software-pipelined like k_stage_pf: a CTA knows its
// next tile before it computes the current one, and the next tile's inputs
// (of whichever scenario it belongs to) are copied into shared memory while
// the current tile's alpha and update phases run. The arguments of the
// scenario in hand sit in shared memory (copied when the walk enters another
// scenario: consecutive tiles of a CTA mostly share one), and its CFL maxima
// are reduced into its control block once per run of its tiles, not per tile.
static_assert(sizeof(StageArgs) % 8 == 0, "StageArgs is copied in 8-byte words");

__global__ void __launch_bounds__(NTHREADS, HF_MIN_BLOCKS)
    k_stage_batch(const StageArgs* __restrict__ args, const int* __restrict__ tile_scn,
                  const int* __restrict__ tile_local, const int* __restrict__ n_tiles,
                  int* counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StagePfSmem& P = *reinterpret_cast<StagePfSmem*>(smem_raw);
  __shared__ __align__(16) unsigned char args_raw[sizeof(StageArgs)];
  StageArgs& A = *reinterpret_cast<StageArgs*>(args_raw);
  __shared__ int claimed;
  const int total_tiles = *n_tiles;  // device-resident: a graph serves any set of scenarios
  int t = blockIdx.x;
  if (counter) {
    if (threadIdx.x == 0) claimed = atomicAdd(counter, 1);
    __syncthreads();
    t = claimed;
  }
  if (t < total_tiles) {
    const StageArgs& A0 = args[tile_scn[t]];
    if (A0.ctrl->active) stage_prefetch(A0, P.s, P.hst, tile_local ? tile_local[t] : t - A0.tile_base);
  }
  __syncthreads();  // every thread has read `claimed`
  int cur = -1;     // scenario whose arguments are in A
  bool live = false;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
  while (t < total_tiles) {
    const int scn = tile_scn[t];
    if (scn != cur) {  // uniform over the CTA
      if (live && A.finalize) block_reduce_speeds(sxm, sym, nonfin, A.ctrl);
      sxm = sym = 0.0;
      nonfin = 0;
      __syncthreads();  // nobody reads the old arguments any more
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&args[scn]);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(args_raw);
      for (int w = threadIdx.x; w < (int)(sizeof(StageArgs) / 8); w += NTHREADS) dst[w] = src[w];
      cur = scn;
    }
    if (counter && threadIdx.x == 0) claimed = atomicAdd(counter, 1);
    cp_async_wait_all();
    __syncthreads();  // this tile's inputs and A are in shared memory; the claim is visible
    live = A.ctrl->active != 0;  // uniform over the CTA
    const int tn = counter ? claimed : t + (int)gridDim.x;
    const StageArgs* An = nullptr;
    if (tn < total_tiles) {
      const int sn = tile_scn[tn];
      An = sn == cur ? &A : &args[sn];
      if (!An->ctrl->active) An = nullptr;  // finished scenario: nothing to fetch
    }
    const int ln = An ? (tile_local ? tile_local[tn] : tn - An->tile_base) : -1;
    if (live) {
      const int tile = tile_local ? tile_local[t] : t - A.tile_base;
      if (interior_tile(A, tile))
        stage_tile<double, true, true>(A, P.s, tile, sxm, sym, nonfin, P.hst, ln, An);
      else
        stage_tile<double, true>(A, P.s, tile, sxm, sym, nonfin, P.hst, ln, An);
    } else if (An) {
      stage_prefetch(*An, P.s, P.hst, ln);
    }
    __syncthreads();  // every thread has read `claimed` before thread 0 takes another
    t = tn;
  }
  if (live && A.finalize) block_reduce_speeds(sxm, sym, nonfin, A.ctrl);
}

// Epilogue of a forward-Euler step: friction, forcings and the CFL
// reduction of the stage result (in_*) into the state (out_*).
// The forward-Euler finalize of one grid over its tiles (friction, forcings,
// CFL contributions); returns the CTA's speed maxima.
template <class T>
__device__ void finalize_tiles(const StageArgs& A, Ctrl* ctrl, double& sxm, double& sym,
                               unsigned long long& nonfin) {
  const double dt = ctrl->dt;
  const int ntiles = A.tiles_x * A.tiles_y;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int tyi = tile / A.tiles_x;
    const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;
    int src_lo = 0, src_hi = 0;
    if (A.f.n_src > 0) {
      src_lo = A.f.tile_start[tile];
      src_hi = A.f.tile_start[tile + 1];
    }
    for (int q = 0; q < CELLS_PER_THREAD; ++q) {
      const int gi = gi0 + threadIdx.x / TX + ROWS_PER_PASS * q, gj = gj0 + threadIdx.x % TX;
      if (gi >= A.nr || gj >= A.nc) continue;
      const int64_t g = (int64_t)gi * A.nc + gj;
      T h = Field<T>::ld(A.in_h, A.tan.in_h, g);
      T hu = Field<T>::ld(A.in_hu, A.tan.in_hu, g);
      T hv = Field<T>::ld(A.in_hv, A.tan.in_hv, g);
      finalize_cell<T>(A, ctrl, dt, gi, gj, g, A.f.tile_order, src_lo, src_hi, h, hu, hv);
      cfl_cell(A, gi, gj, g, val(h), val(hu), val(hv), sxm, sym);
      if (ctrl->check_finite && !isfinite(val(h))) ++nonfin;
      Field<T>::st(A.out_h, A.tan.out_h, g, h);
      Field<T>::st(A.out_hu, A.tan.out_hu, g, hu);
      Field<T>::st(A.out_hv, A.tan.out_hv, g, hv);
    }
  }
}

// Forward-Euler finalize kernel. For T = DualD, blockIdx.y is the tangent
// lane, as in k_stage.
template <class T>
__global__ void __launch_bounds__(NTHREADS) k_finalize(const StageArgs A) {
  Ctrl* ctrl = A.ctrl;
  if (!ctrl->active) return;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
  if constexpr (std::is_same<T, DualD>::value) {
    __shared__ __align__(16) unsigned char lane_raw[sizeof(StageArgs)];
    StageArgs& L = *reinterpret_cast<StageArgs*>(lane_raw);
    if (threadIdx.x == 0) lane_args(A, blockIdx.y, L);
    __syncthreads();
    finalize_tiles<T>(L, ctrl, sxm, sym, nonfin);
  } else {
    finalize_tiles<T>(A, ctrl, sxm, sym, nonfin);
  }
  if (blockIdx.y != 0) return;  // the CFL reduction and the clock belong to lane 0
  block_reduce_speeds(sxm, sym, nonfin, ctrl);
  if (blockIdx.x == 0 && threadIdx.x == 0) commit_clock(ctrl);
}

// CFL reduction of a state (max_wave_speeds + ghost speeds when with_ghosts).
__global__ void __launch_bounds__(NTHREADS) k_cfl(const StageArgs A, int with_ghosts) {
  Ctrl* ctrl = A.ctrl;
  const int ntiles = A.tiles_x * A.tiles_y;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int tyi = tile / A.tiles_x;
    const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;
    for (int q = 0; q < CELLS_PER_THREAD; ++q) {
      const int gi = gi0 + threadIdx.x / TX + ROWS_PER_PASS * q, gj = gj0 + threadIdx.x % TX;
      if (gi >= A.nr || gj >= A.nc) continue;
      const int64_t g = (int64_t)gi * A.nc + gj;
      const double h = A.in_h[g], hu = A.in_hu[g], hv = A.in_hv[g];
      if (with_ghosts)
        cfl_cell(A, gi, gj, g, h, hu, hv, sxm, sym);
      else
        cell_speeds(h, hu, hv, sxm, sym);
      if (!isfinite(h)) ++nonfin;
    }
  }
  block_reduce_speeds(sxm, sym, nonfin, ctrl);
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->cfl_valid = 1;
}

// Step control of one grid (sim.rs:204-215, 231-245): dt = min(cfl /
// (sx/dx + sy/dy), max_dt, cap), validity, rain at t_new. Returns whether the
// step runs (also stored in c->active).
__device__ int control_step(Ctrl* c, double dx, double dy, const ForcingDev& f) {
  {
    int go = 0;
    if (c->status == 0) {
      go = 1;
      if (c->mode == MODE_RUN) {
        if (!(c->t < c->t_target)) {
          go = 0;
        } else if (c->budget <= 0) {
          if (!c->quiet_budget) {
            c->status = -4;  // HF_ERR_STEP_BUDGET
            c->err_t = c->t;
            c->err_step = c->steps;
          }
          go = 0;
        }
      } else if (c->mode == MODE_STEP) {
        go = c->pending;
      } else if (c->mode == MODE_REPLAY) {
        go = c->steps < c->replay_n;
      } else {
        go = 0;
      }
      if (go && c->check_finite && c->nonfinite) {
        c->status = -5;  // HF_ERR_NONFINITE
        c->err_t = c->t;
        c->err_step = c->steps;
        go = 0;
      }
      if (go) {
        const double sx = __longlong_as_double((long long)c->sx_bits);
        const double sy = __longlong_as_double((long long)c->sy_bits);
        const double denom = sx / dx + sy / dy;
        double dt = denom > 0.0 ? c->cfl / denom : __longlong_as_double(0x7ff0000000000000LL);
        dt = fmin(dt, c->max_dt);
        dt = fmin(dt, c->mode == MODE_RUN ? c->t_target - c->t : c->dt_cap);
        if (c->mode == MODE_REPLAY) dt = c->replay_dt[c->steps];  // a recorded (frozen) step
        if (!(isfinite(dt) && dt > 0.0)) {
          c->status = -3;  // HF_ERR_DEGENERATE_DT
          c->err_dt = dt;
          c->err_t = c->t;
          c->err_step = c->steps;
          go = 0;
        } else {
          c->dt = dt;
          c->t_new = c->t + dt;
          const double rate =
              f.n_rain > 0 ? series_eval_u(f.rain_t, f.rain_v, f.n_rain, c->t_new, f.rain_u) : 0.0;
          c->rain_on = rate != 0.0;
          c->rain_dh = rate * dt;
          c->sx_bits = 0ull;
          c->sy_bits = 0ull;
          c->nonfinite = 0ull;
          c->cfl_valid = 0;
          c->pending = 0;
        }
      }
    }
    c->active = go;
    return go;
  }
}

// Point-source depth increments Q_k(t_new) * dt / (dx * dy) (source.rs:58-60).
__device__ __forceinline__ void source_increment(const Ctrl* c, double dx, double dy,
                                                 const ForcingDev& f, int k) {
  const int a = f.src_off[k], b = f.src_off[k + 1];
  const double q = series_eval_u(f.src_t + a, f.src_q + a, b - a, c->t_new, f.src_u);
  f.src_dh[k] = q * c->dt / (dx * dy);
}

__global__ void k_control(Ctrl* c, double dx, double dy, ForcingDev f) {
  __shared__ int s_go;
  if (threadIdx.x == 0) {
    c->strip_dry_last = c->strip_dry;
    c->strip_dry = 0;
    c->strip_claim[0] = c->strip_claim[1] = 0;
    s_go = control_step(c, dx, dy, f);
  }
  __syncthreads();
  if (s_go)
    for (int k = threadIdx.x; k < f.n_src; k += blockDim.x) source_increment(c, dx, dy, f, k);
}

// Gauge row after a step: the series the reference's urban example keeps at
// its control points (solver-2d/examples/uk_ea_test8a_official.rs:219-222)
// and their peaks (fold(0.0, f64::max), ibid. 243-246; fmax ignores NaN as
// f64::max does).
__global__ void k_gauges(const Ctrl* c, const double* __restrict__ h, GaugeDev g, int init) {
  if (!init && !c->active) return;
  const long long row = *g.count;
  for (int k = threadIdx.x; k < g.n; k += blockDim.x) {
    const double v = h[g.cell[k]];
    g.peak[k] = fmax(init ? 0.0 : g.peak[k], v);
    g.last[k] = v;
    if (row < g.cap) g.ser_h[row * g.n + k] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (row < g.cap) g.ser_t[row] = c->t;
    *g.count = row + 1;
  }
}

// Per-scenario control of an ensemble: one thread per scenario.
__global__ void k_batch_control(Ctrl* ctrls, const StageArgs* __restrict__ args, int n,
                                int* counters) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (counters && s == 0) {  // the dynamic schedule's tile counters of this step's two stages
    counters[0] = 0;
    counters[1] = 0;
  }
  if (s >= n) return;
  const StageArgs& A = args[s];
  if (control_step(&ctrls[s], A.dx, A.dy, A.f))
    for (int k = 0; k < A.f.n_src; ++k) source_increment(&ctrls[s], A.dx, A.dy, A.f, k);
}

// Per-scenario clock commit after the ensemble's last stage.
__global__ void k_batch_commit(Ctrl* ctrls, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n && ctrls[s].active) commit_clock(&ctrls[s]);
}

// Ensemble CFL reduction (with ghosts), reduced per tile into its scenario.
__global__ void __launch_bounds__(NTHREADS)
    k_cfl_batch(const StageArgs* __restrict__ args, const int* __restrict__ tile_scn,
                int first_tile, int last_tile) {
  for (int t = first_tile + blockIdx.x; t < last_tile; t += gridDim.x) {
    const StageArgs& A = args[tile_scn[t]];
    const int tile = t - A.tile_base;
    const int tyi = tile / A.tiles_x;
    const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;
    double sxm = 0.0, sym = 0.0;
    unsigned long long nonfin = 0;
    for (int q = 0; q < CELLS_PER_THREAD; ++q) {
      const int gi = gi0 + threadIdx.x / TX + ROWS_PER_PASS * q, gj = gj0 + threadIdx.x % TX;
      if (gi >= A.nr || gj >= A.nc) continue;
      const int64_t g = (int64_t)gi * A.nc + gj;
      const double h = A.in_h[g], hu = A.in_hu[g], hv = A.in_hv[g];
      cfl_cell(A, gi, gj, g, h, hu, hv, sxm, sym);
      if (!isfinite(h)) ++nonfin;
    }
    block_reduce_speeds(sxm, sym, nonfin, A.ctrl);
  }
}

__global__ void k_set_fixed(Ctrl* c, double dt) {
  c->mode = MODE_FIXED;
  c->dt = dt;
  c->t_new = c->t + dt;
  c->active = 1;
  c->status = 0;
  c->rain_on = 0;
  c->sx_bits = 0ull;
  c->sy_bits = 0ull;
  c->nonfinite = 0ull;
}

__global__ void k_set_step(Ctrl* c, double dt_cap, double cfl, double max_dt, int check_finite) {
  c->mode = MODE_STEP;
  c->dt_cap = dt_cap;
  c->pending = 1;
  c->status = 0;
  c->cfl = cfl;
  c->max_dt = max_dt;
  c->check_finite = check_finite;
}

__global__ void k_set_run(Ctrl* c, double t_target, long long budget, double cfl, double max_dt,
                          int check_finite, int quiet_budget) {
  c->mode = MODE_RUN;
  c->quiet_budget = quiet_budget;
  c->t_target = t_target;
  c->budget = budget;
  c->status = 0;
  c->cfl = cfl;
  c->max_dt = max_dt;
  c->check_finite = check_finite;
}

__global__ void k_friction(int64_t ncell, const double* __restrict__ n, double* h, double* hu,
                           double* hv, double dt, double dry_tol) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ncell;
       k += (int64_t)gridDim.x * blockDim.x) {
    double a = hu[k], b = hv[k];
    const double hh = h[k];
    friction_cell(hh, a, b, n[k], dt, dry_tol);
    hu[k] = a;
    hv[k] = b;
  }
}

__global__ void k_rain(int64_t ncell, double* h, double* hu, double* hv, double dh) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ncell;
       k += (int64_t)gridDim.x * blockDim.x) {
    const double nh = h[k] + dh;
    if (nh <= 0.0) {
      h[k] = 0.0;
      hu[k] = 0.0;
      hv[k] = 0.0;
    } else {
      h[k] = nh;
    }
  }
}

constexpr int PS_CHUNK = 32;
struct PointChunk {
  int n;
  long long cell[PS_CHUNK];
  double dh[PS_CHUNK];
};

// Sources in order on one thread: repeated cells accumulate like the
// reference's loop (source.rs:60-68).
__global__ void k_point_sources(PointChunk pc, double* h, double* hu, double* hv) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < pc.n; ++k) {
    const long long g = pc.cell[k];
    const double nh = fmax(h[g] + pc.dh[k], 0.0);
    h[g] = nh;
    if (nh == 0.0) {
      hu[g] = 0.0;
      hv[g] = 0.0;
    }
  }
}

// Counts cells whose Manning value is negative or NaN (Mesh2D's requirement
// n >= 0), checked on the device after the upload.
__global__ void k_count_bad_manning(int64_t ncell, const double* __restrict__ n,
                                    unsigned long long* count) {
  unsigned long long bad = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ncell;
       k += (int64_t)gridDim.x * blockDim.x)
    bad += !(n[k] >= 0.0);
  for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
  if ((threadIdx.x & 31) == 0 && bad) atomicAdd(count, bad);
}

// max_depth_exceeds_relief (sim.rs:248-271): the largest depth folded from
// 0.0 and the bed's max and min, NaN skipped on every side as f64::max/min
// do (fmax/fmin return the other operand). Max and min are order-independent,
// so block partials are combined with atomics on order-preserving keys.
__device__ __forceinline__ unsigned long long order_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void k_relief(int64_t ncell, const double* __restrict__ h,
                         const double* __restrict__ z, Ctrl* c) {
  double hm = 0.0, zmax = -INFINITY, zmin = INFINITY;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ncell;
       k += (int64_t)gridDim.x * blockDim.x) {
    hm = fmax(hm, h[k]);
    const double zk = z[k];
    zmax = fmax(zmax, zk);
    zmin = fmin(zmin, zk);
  }
  for (int o = 16; o > 0; o >>= 1) {
    hm = fmax(hm, __shfl_xor_sync(0xffffffffu, hm, o));
    zmax = fmax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
    zmin = fmin(zmin, __shfl_xor_sync(0xffffffffu, zmin, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&c->relief_keys[0], order_key(hm));
    atomicMax(&c->relief_keys[1], order_key(zmax));
    atomicMin(&c->relief_keys[2], order_key(zmin));
  }
}

__global__ void k_hllc(int x_dir, int64_t n, const double* ul, const double* ur, double* out) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const double* l = ul + 3 * k;
    const double* r = ur + 3 * k;
    double m, nn, t;
    if (x_dir) {
      hllc_normal(l[0], l[1], l[2], r[0], r[1], r[2], m, nn, t);
      out[3 * k] = m; out[3 * k + 1] = nn; out[3 * k + 2] = t;
    } else {
      hllc_normal(l[0], l[2], l[1], r[0], r[2], r[1], m, nn, t);
      out[3 * k] = m; out[3 * k + 1] = t; out[3 * k + 2] = nn;
    }
  }
}

// ------------------------------------------------------------- launchers
namespace {
thread_local cudaError_t g_launch_error = cudaSuccess;
int cuda_rc(cudaError_t e) {
  if (e == cudaSuccess) return 0;
  g_launch_error = e;
  return -7;
}
struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    if (dev >= 0 && prev != dev) cudaSetDevice(dev);
  }
  ~DevGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};
int elem_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}
}  // namespace

cudaError_t last_launch_error() { return g_launch_error; }

namespace {
std::atomic<unsigned long long> g_kernel_launches{0};
std::mutex g_graph_mu;
std::unordered_map<cudaGraphExec_t, unsigned long long> g_graph_kernels;  // kernel nodes

unsigned long long kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
  unsigned long long k = 0;
  for (size_t i = 0; i < n; ++i) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}
}  // namespace

int launched(void* stream) {
  const int rc = cuda_rc(cudaGetLastError());
  if (rc != 0) return rc;
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing((cudaStream_t)stream, &st) != cudaSuccess) {
    cudaGetLastError();  // the query failed: count the launch
    st = cudaStreamCaptureStatusNone;
  }
  if (st == cudaStreamCaptureStatusNone) g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  return 0;
}

cudaError_t graph_instantiate(cudaGraphExec_t* exec, cudaGraph_t graph) {
  const cudaError_t e = cudaGraphInstantiate(exec, graph, 0);
  if (e == cudaSuccess) {
    const unsigned long long k = kernel_nodes(graph);
    cudaGetLastError();  // a failed node query only leaves the count at 0
    std::lock_guard<std::mutex> lock(g_graph_mu);
    g_graph_kernels[*exec] = k;
  }
  return e;
}

cudaError_t graph_launch(cudaGraphExec_t exec, cudaStream_t stream) {
  unsigned long long k = 0;
  {
    std::lock_guard<std::mutex> lock(g_graph_mu);
    const auto it = g_graph_kernels.find(exec);
    if (it != g_graph_kernels.end()) k = it->second;
  }
  const cudaError_t e = cudaGraphLaunch(exec, stream);
  if (e == cudaSuccess) g_kernel_launches.fetch_add(k, std::memory_order_relaxed);
  return e;
}

void graph_destroy(cudaGraphExec_t exec) {
  {
    std::lock_guard<std::mutex> lock(g_graph_mu);
    g_graph_kernels.erase(exec);
  }
  cudaGraphExecDestroy(exec);
}

unsigned long long kernel_launch_count() { return g_kernel_launches.load(); }

size_t stage_smem_bytes() { return sizeof(StageSmem); }

int stage_grid_size(int tiles, int device) {
  static int cached[64] = {0};
  int per_sm = 0, sms = 0;
  if (device >= 0 && device < 64 && cached[device] > 0) {
    per_sm = cached[device];
  } else {
    DevGuard dg(device);
    cudaFuncSetAttribute(k_stage_pf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(StagePfSmem));
    cudaFuncSetAttribute(k_stage_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(StagePfSmem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_pf, NTHREADS,
                                                  sizeof(StagePfSmem));
    if (per_sm < 1) per_sm = 1;
    if (device >= 0 && device < 64) cached[device] = per_sm;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int g = per_sm * (sms > 0 ? sms : 148);
  return tiles < g ? (tiles < 1 ? 1 : tiles) : g;
}

// ---- strip kernel: descriptors, grid size, launch
namespace {
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}
// An nr x nc row-major f64 array, boxes of 40 columns x `rows` rows; cells
// outside the array read as zeros.
bool encode_rows(CUtensorMap& m, const double* base, int64_t nr, int64_t nc, int rows) {
  EncodeTiled enc = encode_tiled();
  if (!enc || !base || ((uintptr_t)base & 15) || (nc * sizeof(double)) % 16) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)nc, (cuuint64_t)nr};
  const cuuint64_t strides[1] = {(cuuint64_t)nc * sizeof(double)};
  const cuuint32_t box[2] = {40u, (cuuint32_t)rows};
  const cuuint32_t estr[2] = {1u, 1u};
  return enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides,
             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}
constexpr size_t kStripSmemBytes = sizeof(StripSmem) + 128;  // + alignment of the base
}  // namespace

bool strip_maps(const StageArgs& a, StripMaps& m) {
  return encode_rows(m.h, a.in_h, a.nr, a.nc, STRIP_ROWS + 1) &&
         encode_rows(m.z, a.z, a.nr, a.nc, STRIP_ROWS) &&
         encode_rows(m.hu, a.in_hu, a.nr, a.nc, STRIP_ROWS) &&
         encode_rows(m.hv, a.in_hv, a.nr, a.nc, STRIP_ROWS);
}

int strip_grid_size(int64_t nr, int64_t nc, int device) {
  static int cached[64] = {0};
  int per_sm = 0, sms = 0;
  if (device >= 0 && device < 64 && cached[device] > 0) {
    per_sm = cached[device];
  } else {
    DevGuard dg(device);
    cudaFuncSetAttribute(k_stage_strip, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kStripSmemBytes);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_strip, NTHREADS,
                                                  kStripSmemBytes);
    cudaGetLastError();
    if (per_sm < 1) return 0;
    if (device >= 0 && device < 64) cached[device] = per_sm;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const long long g = (long long)per_sm * (sms > 0 ? sms : 148);
  const long long nq = (long long)strip_count(nc) * strip_blocks(nr);
  return nq >= 4 * g ? (int)g : 0;
}

int launch_stage_strip(const StageArgs& a, const StripMaps& m, int grid, void* stream) {
  k_stage_strip<<<grid, NTHREADS, kStripSmemBytes, (cudaStream_t)stream>>>(a, m);
  return launched(stream);
}

int stage_dual_grid_size(int tiles, int device) {
  static int cached[64] = {0};
  int per_sm = 0, sms = 0;
  if (device >= 0 && device < 64 && cached[device] > 0) {
    per_sm = cached[device];
  } else {
    DevGuard dg(device);
    cudaFuncSetAttribute(k_stage<DualD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(StageSmemT<DualD>));
    // two 112 KB tiles per SM need the largest shared-memory carveout
    cudaFuncSetAttribute(k_stage<DualD>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage<DualD>, NTHREADS,
                                                  sizeof(StageSmemT<DualD>));
    if (per_sm < 1) per_sm = 1;
    if (device >= 0 && device < 64) cached[device] = per_sm;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  int g = per_sm * (sms > 0 ? sms : 148);
  return tiles < g ? (tiles < 1 ? 1 : tiles) : g;
}

// Callers size the grid with stage_grid_size() first, which also raises the
// kernel's dynamic shared-memory limit on this device (never inside a
// stream capture).
int launch_stage(const StageArgs& a, int grid, void* stream) {
  k_stage_pf<<<grid, NTHREADS, sizeof(StagePfSmem), (cudaStream_t)stream>>>(a);
  return launched(stream);
}

int launch_finalize(const StageArgs& a, int grid, void* stream) {
  k_finalize<double><<<grid, NTHREADS, 0, (cudaStream_t)stream>>>(a);
  return launched(stream);
}

// DualD (tangent) stage and finalize: value arrays in a.in_* / a.out_* /
// a.un_* / a.n, tangent arrays in a.tan. Grid from stage_dual_grid_size().
int launch_stage_dual(const StageArgs& a, int grid, void* stream, int lanes) {
  k_stage<DualD><<<dim3(grid, lanes), NTHREADS, sizeof(StageSmemT<DualD>),
                   (cudaStream_t)stream>>>(a);
  return launched(stream);
}

int launch_finalize_dual(const StageArgs& a, int grid, void* stream, int lanes) {
  k_finalize<DualD><<<dim3(grid, lanes), NTHREADS, 0, (cudaStream_t)stream>>>(a);
  return launched(stream);
}

int launch_stage_batch(const StageArgs* args, const int* tile_scn, const int* n_tiles, int grid,
                       void* stream, const int* tile_local, int* counter) {
  k_stage_batch<<<grid, NTHREADS, sizeof(StagePfSmem), (cudaStream_t)stream>>>(
      args, tile_scn, tile_local, n_tiles, counter);
  return launched(stream);
}

int launch_cfl_batch(const StageArgs* args, const int* tile_scn, int first_tile, int last_tile,
                     int grid, void* stream) {
  if (last_tile <= first_tile) return 0;
  k_cfl_batch<<<grid, NTHREADS, 0, (cudaStream_t)stream>>>(args, tile_scn, first_tile, last_tile);
  return launched(stream);
}

int launch_batch_control(Ctrl* ctrls, const StageArgs* args, int n, void* stream,
                         int* counters) {
  k_batch_control<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ctrls, args, n, counters);
  return launched(stream);
}

int launch_batch_commit(Ctrl* ctrls, int n, void* stream) {
  k_batch_commit<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ctrls, n);
  return launched(stream);
}

int launch_cfl(const StageArgs& a, int with_ghosts, int grid, void* stream) {
  k_cfl<<<grid, NTHREADS, 0, (cudaStream_t)stream>>>(a, with_ghosts);
  return launched(stream);
}

int launch_control(Ctrl* ctrl, double dx, double dy, const ForcingDev& f, void* stream) {
  k_control<<<1, 256, 0, (cudaStream_t)stream>>>(ctrl, dx, dy, f);
  return launched(stream);
}

int launch_gauges(const Ctrl* ctrl, const double* h, const GaugeDev& g, int init, void* stream) {
  k_gauges<<<1, 128, 0, (cudaStream_t)stream>>>(ctrl, h, g, init);
  return launched(stream);
}

int launch_set_fixed(Ctrl* ctrl, double dt, void* stream) {
  k_set_fixed<<<1, 1, 0, (cudaStream_t)stream>>>(ctrl, dt);
  return launched(stream);
}

int launch_set_step(Ctrl* ctrl, double dt_cap, double cfl, double max_dt, int check_finite,
                    void* stream) {
  k_set_step<<<1, 1, 0, (cudaStream_t)stream>>>(ctrl, dt_cap, cfl, max_dt, check_finite);
  return launched(stream);
}

int launch_set_run(Ctrl* ctrl, double t_target, long long budget, double cfl, double max_dt,
                   int check_finite, int quiet_budget, void* stream) {
  k_set_run<<<1, 1, 0, (cudaStream_t)stream>>>(ctrl, t_target, budget, cfl, max_dt, check_finite,
                                               quiet_budget);
  return launched(stream);
}

int launch_friction(int64_t ncell, const double* n, double* h, double* hu, double* hv, double dt,
                    double dry_tol, void* stream) {
  if (ncell <= 0) return 0;
  k_friction<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(ncell, n, h, hu, hv, dt, dry_tol);
  return launched(stream);
}

int launch_rain(int64_t ncell, double* h, double* hu, double* hv, double rate, double dt,
                void* stream) {
  if (rate == 0.0 || ncell <= 0) return 0;  // source.rs:89-91
  const double dh = rate * dt;
  k_rain<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(ncell, h, hu, hv, dh);
  return launched(stream);
}

int launch_point_sources(int64_t nc, double* h, double* hu, double* hv, int n,
                         const int64_t* rows, const int64_t* cols, const double* q, double dt,
                         double dx, double dy, void* stream) {
  const double area = dx * dy;
  for (int base = 0; base < n; base += PS_CHUNK) {
    PointChunk pc;
    pc.n = n - base < PS_CHUNK ? n - base : PS_CHUNK;
    for (int k = 0; k < pc.n; ++k) {
      pc.cell[k] = (long long)rows[base + k] * nc + cols[base + k];
      pc.dh[k] = q[base + k] * dt / area;
    }
    k_point_sources<<<1, 32, 0, (cudaStream_t)stream>>>(pc, h, hu, hv);
    int rc = launched(stream);
    if (rc) return rc;
  }
  return 0;
}

int launch_count_bad_manning(int64_t ncell, const double* n, unsigned long long* count,
                             void* stream) {
  if (ncell <= 0) return 0;
  k_count_bad_manning<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(ncell, n, count);
  return launched(stream);
}

int launch_relief(int64_t ncell, const double* h, const double* z, Ctrl* c, void* stream) {
  if (ncell <= 0) return 0;
  k_relief<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(ncell, h, z, c);
  return launched(stream);
}

int launch_hllc(int x_dir, int64_t n, const double* ul, const double* ur, double* out,
                void* stream) {
  if (n <= 0) return 0;
  k_hllc<<<elem_grid(n), 256, 0, (cudaStream_t)stream>>>(x_dir, n, ul, ur, out);
  return launched(stream);
}

}  // namespace hf
