// hf_internal.h -- structures shared by the kernels and the C-ABI layer.
#pragma once

#include <cuda.h>  // CUtensorMap (types only; the driver is reached through the runtime)

#include <cstdint>
#include <cstring>

#include "../../include/hydroflux_gpu.h"
#include "hf_arith.h"

namespace hf {

// Tile geometry of the fused stage kernels: a CTA advances a TX x TY block
// of cells, one cell per thread; its shared-memory halo is 4 cells (two-cell
// dry buffer of the slope limiter + one neighbour slope + one neighbour
// alpha). Two geometries are built (hf_tiles.cu is compiled once for each;
// its symbols sit in the geometry's inline namespace):
// - 32 x 8 (g8, kGeomSmall): 256 threads, 71 KB of shared memory, three CTAs
//   (24 warps) per SM. Many tiles per grid, so small grids still spread over
//   every SM. The DualD tangent, the adjoint, the strip kernel and the
//   calibration handle's runs use this geometry only.
// - 32 x 32 (g32, kGeomLarge): 1024 threads, 211 KB of shared memory, one
//   CTA (32 warps) per SM. The halo is a smaller share of the tile (2.32
//   Audusse+HLLC faces and 2.39 limited-slope cells per cell against 2.83
//   and 3.0) and an SM runs more warps; a stage launch on the 4096^2 valley
//   takes 2.06 ms against 2.36 ms. Grids with at least kLargeTilesMin tiles
//   of it take it (geom_for).
// Both compute every cell with the same operations: results are identical.
constexpr int TX = 32;
constexpr int kGeomSmall = 0, kGeomLarge = 1;
#ifndef HF_LARGE_TILE_Y
#define HF_LARGE_TILE_Y 32  // the large geometry's tile height (build.py passes the same)
#endif
constexpr int kGeomTileH[2] = {8, HF_LARGE_TILE_Y};
constexpr int kLargeTilesMin = 100;
// A scenario of an ensemble or server with at least this many 32 x 32 tiles
// (about 3.5 waves of the 148 SMs; from 724 x 724 cells on) fills the GPU
// by itself: it runs its stages as its own k_stage_pf launches (arguments
// as kernel parameters) beside the batched launch of the other scenarios.
constexpr int kSoloTilesMin = 512;
#ifndef HF_GEOM
#define HF_GEOM g8
#define HF_GEOM_INDEX 0
#define HF_TILE_Y 8
#define HF_THREADS 256
#define HF_MIN_BLOCKS 3
#endif
// The build of the 32 x 8 geometry also carries the kernels that exist in
// one geometry only (strip, DualD, adjoint) and the host code.
#define HF_GEOM_PRIMARY (HF_GEOM_INDEX == 0)
#define HF_CAT2(a, b) a##b
#define HF_CAT(a, b) HF_CAT2(a, b)
#define HF_GEOM_OPS HF_CAT(geom_ops_, HF_GEOM)
inline namespace HF_GEOM {
constexpr int TY = HF_TILE_Y;
constexpr int NTHREADS = HF_THREADS;
constexpr int ROWS_PER_PASS = NTHREADS / TX;  // tile rows one pass of the CTA covers
// Cells a thread updates per tile. When the tile height is not a multiple of
// the rows of a pass, the last pass is partial (kPartialPass) and the threads
// past the tile's last row skip it.
constexpr int CELLS_PER_THREAD = (TY + ROWS_PER_PASS - 1) / ROWS_PER_PASS;
constexpr bool kPartialPass = TY % ROWS_PER_PASS != 0;
static_assert(NTHREADS % TX == 0, "tile / thread shape");
static_assert(TY == kGeomTileH[HF_GEOM_INDEX], "geometry index and tile height");
}  // namespace HF_GEOM

// Strip geometry of the streaming stage kernel (hf_strip.cuh): a CTA walks
// down a TX-wide column of blocks of STRIP_ROWS rows, carrying the halo rows
// of one block into the next. Blocks are numbered strip-major:
// q = (column / TX) * strip_blocks(nr) + row / STRIP_ROWS.
constexpr int STRIP_ROWS = 7;
HF_ARITH_HD int strip_blocks(int64_t nr) { return (int)((nr + STRIP_ROWS - 1) / STRIP_ROWS); }
HF_ARITH_HD int strip_count(int64_t nc) { return (int)((nc + TX - 1) / TX); }

// Boundary descriptor in kernel arguments; sides in Boundaries2D order.
struct BcDev {
  int kind[4];    // north, south, west, east
  double val[4];  // q for Discharge, h for Depth
};

// MODE_REPLAY takes step k's dt from replay_dt[k] (a recorded dt sequence)
// for steps < replay_n.
enum CtrlMode { MODE_FIXED = 0, MODE_STEP = 1, MODE_RUN = 2, MODE_REPLAY = 3 };

// Device-resident step control block. dt, the simulation clock and the CFL
// accumulators live here, so a step needs no host round trip.
struct Ctrl {
  double t;         // simulation time
  double dt;        // dt of the step in flight
  double t_new;     // t + dt
  double t_target;  // MODE_RUN target
  double dt_cap;    // MODE_STEP cap
  double cfl;
  double max_dt;
  double rain_dh;   // rate(t_new) * dt
  unsigned long long sx_bits;    // max |u| + c over the current state (bits of a double >= 0)
  unsigned long long sy_bits;
  unsigned long long nonfinite;  // cells with non-finite depth (opt-in check)
  long long steps;
  long long budget;  // MODE_RUN step budget left
  int mode;
  int active;        // 1 while the step in flight runs
  int status;        // 0 or an hf_status_code
  int rain_on;       // rate(t_new) != 0
  int pending;       // MODE_STEP: one step requested
  int check_finite;
  int cfl_valid;     // accumulators describe the current state
  int quiet_budget;  // MODE_RUN: an exhausted budget ends the run without error
  double err_dt;
  double err_t;
  long long err_step;
  const double* replay_dt;  // MODE_REPLAY
  long long replay_n;
  // max_depth_exceeds_relief accumulators (order-preserving keys of doubles):
  // max depth (from 0), max bed, min bed.
  unsigned long long relief_keys[3];
  // Strip stage kernel: block counters of the dynamic schedule of stage 1 /
  // stage 2, and the blocks its stages skipped as dry in the current and the
  // previous step (which picks the schedule). The control kernel rolls them
  // over at the start of every step.
  unsigned long long strip_claim[2];
  unsigned long long strip_dry, strip_dry_last;
};

struct SeriesUnits {
  double t_div = 1.0;
  double v_mul = 1.0;
  double v_div = 1.0;
};

// Forcing tables on the device (piecewise-linear series). Point sources are
// bucketed by stage tile: sources of tile t are tile_order[tile_start[t] ..
// tile_start[t+1]) in their original order.
struct ForcingDev {
  int n_rain;
  int n_src;
  const double* rain_t;
  const double* rain_v;
  const int* src_row;
  const int* src_col;
  const int* src_off;  // n_src + 1 offsets into src_t / src_q
  const double* src_t;
  const double* src_q;
  const int* tile_start;
  const int* tile_order;
  // The same sources bucketed by strip block (blk_start has one entry per
  // strip block + 1).
  const int* blk_start;
  const int* blk_order;
  double* src_dh;  // per source, set each step by the control kernel
  // Series units: a series is sampled at t / t_div and its value converted
  // as (v * v_mul) / v_div (identity by default; see hf_sim_set_rain_units).
  SeriesUnits rain_u;
  SeriesUnits src_u;
};

// Control-point (gauge) recorder of a simulation: after every step taken,
// the depth at each gauge cell is folded into its running maximum and stored
// as one row of the series while rows remain.
struct GaugeDev {
  int n;
  const long long* cell;  // row-major cell index of each gauge
  double* peak;           // fold(0.0, f64::max) over the recorded depths
  double* last;
  double* ser_t;          // cap rows: time of the row
  double* ser_h;          // cap x n depths
  long long cap;
  long long* count;       // rows seen (stored: min(count, cap))
};

// Tangent arrays of a DualD (forward-mode) stage, parallel to the value
// arrays of StageArgs; the f64 kernels never read them. A null input
// tangent is a zero tangent.
struct TanPtrs {
  const double* in_h = nullptr;
  const double* in_hu = nullptr;
  const double* in_hv = nullptr;
  double* out_h = nullptr;
  double* out_hu = nullptr;
  double* out_hv = nullptr;
  const double* un_h = nullptr;
  const double* un_hu = nullptr;
  const double* un_hv = nullptr;
  const double* n = nullptr;  // Manning tangent
  // Vector mode: blockIdx.y is the tangent lane; lane l's tangent arrays
  // start lane_stride doubles after lane l-1's (0: one lane).
  long long lane_stride = 0;
};

struct StageArgs {
  int nr, nc;
  int tiles_x, tiles_y;
  int tile_base;  // first tile of this grid in an ensemble's tile list (0 alone)
  // 1 for a grid of an ensemble or server that runs k_stage_pf on its own:
  // its clock is committed by k_batch_commit, not by the stage kernel.
  int batched = 0;
  double dx, dy;
  // 1/dx and 1/dy for the divisions by the spacing (hfa::div_recip); a
  // default (ok = false) falls back to the IEEE division.
  hfa::RecipD rx, ry;
  const double* z;
  const double* n;
  const double* in_h;
  const double* in_hu;
  const double* in_hv;
  double* out_h;
  double* out_hu;
  double* out_hv;
  const double* un_h;  // SSP-RK2 U^n (may alias out_*)
  const double* un_hu;
  const double* un_hv;
  BcDev bc;
  Ctrl* ctrl;
  int combine;   // SSP-RK2 convex combination + floor with U^n
  int finalize;  // friction + forcings + CFL reduction + clock commit
  double dry_tol;
  ForcingDev f;
  TanPtrs tan;   // DualD kernels only
};

// Launchers of the step control and standalone kernels (hf_kernels.cu).
int launch_control(Ctrl* ctrl, double dx, double dy, const ForcingDev& f, void* stream);
// Records one gauge row when the step ran (init: unconditionally, the peak
// starting from 0).
int launch_gauges(const Ctrl* ctrl, const double* h, const GaugeDev& g, int init, void* stream);
int launch_set_fixed(Ctrl* ctrl, double dt, void* stream);
int launch_set_step(Ctrl* ctrl, double dt_cap, double cfl, double max_dt, int check_finite,
                    void* stream);
int launch_set_run(Ctrl* ctrl, double t_target, long long budget, double cfl, double max_dt,
                   int check_finite, int quiet_budget, void* stream);
int launch_friction(int64_t ncell, const double* n, double* h, double* hu, double* hv, double dt,
                    double dry_tol, void* stream);
int launch_rain(int64_t ncell, double* h, double* hu, double* hv, double rate, double dt,
                void* stream);
int launch_point_sources(int64_t nc, double* h, double* hu, double* hv, int n,
                         const int64_t* rows, const int64_t* cols, const double* q, double dt,
                         double dx, double dy, void* stream);
// max_depth_exceeds_relief reduction (sim.rs:248-271) into c->relief_keys,
// which the caller presets to {0, 0, ~0}. Decode with relief_key_value.
int launch_relief(int64_t ncell, const double* h, const double* z, Ctrl* c, void* stream);
inline double relief_key_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k ^ 0x8000000000000000ull) : ~k;
  double d;
  std::memcpy(&d, &b, sizeof d);
  return d;
}
// *count += cells with !(n >= 0) (count is device memory, zeroed by the caller).
int launch_count_bad_manning(int64_t ncell, const double* n, unsigned long long* count,
                             void* stream);
int launch_hllc(int x_dir, int64_t n, const double* ul, const double* ur, double* out,
                void* stream);

// TMA descriptors of one stage's inputs for the strip kernel (hf_strip.cuh):
// depth rows (box 40 x (STRIP_ROWS + 1)), bed, hu, hv (40 x STRIP_ROWS).
struct StripMaps {
  CUtensorMap h, z, hu, hv;
};

// The tile-shaped kernels of one geometry (hf_tiles.cu), reached from host
// code that serves grids of either geometry through geom_ops().
struct GeomOps {
  int tile_h;   // TY of the geometry (the width is TX)
  int threads;  // CTA size
  // CTAs for `tiles` tiles on `device` (also raises the kernels' shared-memory
  // limits; never inside a stream capture).
  int (*grid_size)(int tiles, int device);
  int (*stage)(const StageArgs& a, int grid, void* stream);
  int (*finalize)(const StageArgs& a, int grid, void* stream);
  int (*cfl)(const StageArgs& a, int with_ghosts, int grid, void* stream);
  int (*stage_batch)(const StageArgs* args, const int* tile_scn, const int* n_tiles, int grid,
                     void* stream, const int* tile_local, int* counter);
  int (*cfl_batch)(const StageArgs* args, const int* tile_scn, int first_tile, int last_tile,
                   int grid, void* stream);
};
const GeomOps& geom_ops_g8();
const GeomOps& geom_ops_g32();
const GeomOps& geom_ops(int geom);
// The geometry of an nr x nc grid: kGeomLarge once it has kLargeTilesMin
// tiles of 32 x 32, else kGeomSmall.
int geom_for(int64_t nr, int64_t nc);
inline int tiles_along(int64_t n, int tile) { return (int)((n + tile - 1) / tile); }

inline namespace HF_GEOM {
// The single-grid stage (k_stage_pf), the forward-Euler finalize and the CFL
// reduction of this geometry. Callers size the grid with stage_grid_size()
// first, which also raises the kernels' shared-memory limits on the device.
int launch_stage(const StageArgs& a, int grid, void* stream);
int launch_finalize(const StageArgs& a, int grid, void* stream);
int launch_cfl(const StageArgs& a, int with_ghosts, int grid, void* stream);
int stage_grid_size(int tiles, int device);
size_t stage_smem_bytes();

// Encodes the descriptors of a stage's inputs (a.in_h, a.z, a.in_hu,
// a.in_hv); false when the grid cannot be fetched that way (an odd column
// count gives rows that do not start on 16 bytes; an unaligned buffer; no
// driver entry point), in which case the tile kernel runs.
bool strip_maps(const StageArgs& a, StripMaps& m);
// CTAs of the strip kernel for an nr x nc grid on `device` (also raises its
// shared-memory limit; never inside a stream capture); 0 when the grid has
// too few strip blocks per CTA for streaming to pay.
int strip_grid_size(int64_t nr, int64_t nc, int device);
int launch_stage_strip(const StageArgs& a, const StripMaps& m, int grid, void* stream);
// DualD tangent stage / finalize (same arguments; tangent arrays in a.tan).
int stage_dual_grid_size(int tiles, int device);
// lanes > 1 (vector mode): one grid of `grid` CTAs per tangent lane
// (blockIdx.y), a.tan.lane_stride apart; lane 0 alone writes the values, so
// a.out_* must not alias a.in_* or a.un_* then.
int launch_stage_dual(const StageArgs& a, int grid, void* stream, int lanes = 1);
int launch_finalize_dual(const StageArgs& a, int grid, void* stream, int lanes = 1);

// Adjoint of one stage (hf_adjoint.cu). `a` is the stage's forward arguments
// (with combine / finalize as run); lam_* the adjoint of its output. Writes
// halo[tile][4][..] (adjoint of the input h, hu, hv and of n over each tile
// and its 3-cell halo) and, with a.combine, 0.5 * the combination's adjoint
// into lam_un_*. Grid from adj_grid_size().
size_t adj_halo_doubles_per_tile();
int adj_grid_size(int tiles, int device);
int launch_stage_adj(const StageArgs& a, const double* lam_h, const double* lam_hu,
                     const double* lam_hv, double* lam_un_h, double* lam_un_hu,
                     double* lam_un_hv, double* halo, int grid, void* stream);
// out = sum of the halo contributions (+ add when non-null); grad_n += the
// Manning part.
int launch_adj_gather(int nr, int nc, int tiles_x, int tiles_y, const double* halo,
                      const double* add_h, const double* add_hu, const double* add_hv,
                      double* out_h, double* out_hu, double* out_hv, double* grad_n,
                      void* stream);
int launch_adj_seed(double* lam_h, const int64_t* cells, int n_gauges, const double* gauge_h,
                    const double* obs, void* stream);
int launch_calib_pre(const Ctrl* c, double* dts, double* ts, long long cap, void* stream);
// gauge_dh of lane l at [l][cap][n_gauges], read from dh + l * lane_stride.
int launch_calib_post(const Ctrl* c, const double* h, const double* dh, const int64_t* cells,
                      int n_gauges, double* gauge_h, double* gauge_dh, long long cap,
                      void* stream, int lanes = 1, long long lane_stride = 0);
int launch_calib_rewind(Ctrl* c, const double* ts, long long k, void* stream);
// State checkpoint before the current step when c->steps % every == 0.
int launch_calib_ckpt(const Ctrl* c, const double* h, const double* hu, const double* hv,
                      double* ckpt, long long every, long long cap, long long ncell,
                      void* stream);
}  // namespace HF_GEOM

// Sets the calling thread's hf_last_error() message and returns `code`.
int record_error(int code, const char* msg);
// Shape, SimulationConfig (sim.rs:130-165) and boundary checks of one grid.
int check_grid_config(const hf_config* cfg, int64_t nr, int64_t nc);
// The boundary-set check alone (kinds; Discharge/Depth need >= 2 cells
// normal to their side) and the low-level grid check (shape; dx, dy > 0 as
// Mesh2D::new asserts, geometry.rs:59, 93), shared by every entry point.
int check_boundaries(const hf_boundaries& b, int64_t nr, int64_t nc);
int check_grid_desc(const hf_grid* g);
BcDev boundaries_dev(const hf_boundaries& b);
// The error of this thread's last failed kernel launch in the launchers
// (launched() returns -7 and keeps the cudaError_t here).
cudaError_t last_launch_error();
// The error to report once a runtime call or a launcher has failed: the
// runtime's pending error, else the launch error the launcher consumed, else
// cudaErrorUnknown, so that a failure is never reported as success.
inline cudaError_t failed_call_error() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const cudaError_t l = last_launch_error();
  return l != cudaSuccess ? l : cudaErrorUnknown;
}

// Kernel launch accounting (hf_kernel_launches): every launcher ends with
// launched(stream), which returns 0 or -7 like the launch check and counts
// the launch unless the stream is being captured into a graph. Graphs are
// instantiated, launched and destroyed through the three graph_* calls,
// which count each launch as the kernel nodes of its graph.
int launched(void* stream);
cudaError_t graph_instantiate(cudaGraphExec_t* exec, cudaGraph_t graph);
cudaError_t graph_launch(cudaGraphExec_t exec, cudaStream_t stream);
void graph_destroy(cudaGraphExec_t exec);
unsigned long long kernel_launch_count();

// Device copies of one grid's forcing tables (host-side owner).
struct ForcingHost {
  int n_rain = 0, n_src = 0;
  double* d_rain_t = nullptr;
  double* d_rain_v = nullptr;
  int* d_row = nullptr;
  int* d_col = nullptr;
  int* d_off = nullptr;
  double* d_st = nullptr;
  double* d_sq = nullptr;
  int* d_tile_start[2] = {nullptr, nullptr};  // per geometry (kGeomSmall, kGeomLarge)
  int* d_tile_order[2] = {nullptr, nullptr};
  int* d_blk_start = nullptr;
  int* d_blk_order = nullptr;
  double* d_dh = nullptr;
  SeriesUnits rain_u, src_u;
  void release_rain();
  void release_src();
  // The device tables, with the point sources bucketed by the tiles of
  // geometry `geom`.
  ForcingDev dev(int geom) const;
};
// Validate and upload a rain series / point-source series (see
// hf_sim_set_rain / hf_sim_set_point_sources); sources are bucketed by the
// tiles of both geometries and by strip block.
int forcing_set_rain(ForcingHost& f, int64_t n_points, const double* t, const double* rate);
int forcing_set_sources(ForcingHost& f, int64_t nr, int64_t nc, int64_t n_sources,
                        const int64_t* rows, const int64_t* cols, const int64_t* offsets,
                        const double* t, const double* q);

// Ensemble launchers: args1/args2 are per-scenario device arrays of stage-1 /
// stage-2 arguments, ctrls the per-scenario control blocks. n_tiles is a
// device int (the tile list length, read at launch time); the CFL reduction
// covers tiles [first_tile, last_tile). tile_local / counter select the
// schedule (see k_stage_batch): nullptr gives the static stride over
// scenario-contiguous tiles. The stage and CFL launchers are per geometry
// (hf_tiles.cu, GeomOps::stage_batch / cfl_batch); control and commit are
// not (hf_kernels.cu).
inline namespace HF_GEOM {
int launch_stage_batch(const StageArgs* args, const int* tile_scn, const int* n_tiles, int grid,
                       void* stream, const int* tile_local, int* counter);
int launch_cfl_batch(const StageArgs* args, const int* tile_scn, int first_tile, int last_tile,
                     int grid, void* stream);
}  // namespace HF_GEOM
// counters (2 ints, may be NULL) are zeroed for the dynamic schedule.
int launch_batch_control(Ctrl* ctrls, const StageArgs* args, int n, void* stream,
                         int* counters = nullptr);
int launch_batch_commit(Ctrl* ctrls, int n, void* stream);

}  // namespace hf
