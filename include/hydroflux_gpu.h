/*
 * hydroflux_gpu.h -- C ABI of the B200 (sm_100a) implementation of hydroflux
 * solver-2d's explicit time step.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (HF_OK = 0, negative on failure; the message is in
 * hf_last_error()). Nothing here names a torch or CUDA C++ type: a CUDA
 * stream is passed as `void*` (a cudaStream_t / CUstream handle, NULL for the
 * legacy default stream).
 *
 * The surface mirrors the reference crate (franciscoparrao/hydroflux,
 * crate hydroflux-solver-2d) so that a Rust `extern "C"` shim can sit behind
 * its existing API:
 *   - hf_sim_*    <-> `Simulation` (solver-2d/src/sim.rs:119-245)
 *   - hf_cfl_time_step, hf_forward_euler_step, hf_ssprk2_step,
 *     hf_manning_friction_step, hf_apply_rain, hf_apply_point_sources
 *                 <-> the free functions re-exported at solver-2d/src/lib.rs:74-91
 *   - hf_workspace_* <-> `StepWorkspace2D` (solver-2d/src/update.rs:743-777)
 * Layout: the reference stores `Array2<Conserved2D>` (AoS {h,hu,hv}, row-major
 * (n_rows, n_cols), row i along y, column j along x). Here the state is SoA:
 * three row-major double arrays h, hu, hv of n_rows*n_cols; the hf_sim API
 * also accepts/returns the AoS {h,hu,hv} layout of `Conserved2D`.
 */
#ifndef HYDROFLUX_GPU_H
#define HYDROFLUX_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HF_ABI_VERSION 1

/* Status codes. The first four mirror `SimError` (solver-2d/src/sim.rs:81-115). */
enum hf_status_code {
  HF_OK = 0,
  HF_ERR_SHAPE_MISMATCH = -1, /* SimError::ShapeMismatch (sim.rs:83-91) */
  HF_ERR_INVALID_CONFIG = -2, /* SimError::InvalidConfig (sim.rs:93-94) */
  HF_ERR_DEGENERATE_DT = -3,  /* SimError::DegenerateDt (sim.rs:96-104) */
  HF_ERR_STEP_BUDGET = -4,    /* SimError::StepBudgetExhausted (sim.rs:106-114) */
  HF_ERR_NONFINITE = -5,      /* non-finite depth seen by the CFL reduction (opt-in) */
  HF_ERR_TIMEOUT = -6,        /* a bounded device-side wait gave up */
  HF_ERR_CUDA = -7,           /* CUDA runtime failure */
  HF_ERR_INVALID_ARG = -8,    /* bad pointer / index; the reference panics here */
  HF_ERR_OUT_OF_MEMORY = -9,  /* device allocation failed */
  HF_ERR_UNSUPPORTED = -10,   /* feature not available for this configuration */
  HF_ERR_CAPACITY = -11       /* server: no free slot or over the HBM budget (retry later) */
};

/* Boundary kinds (solver-2d/src/boundary.rs:80-104). */
enum hf_bc_kind {
  HF_BC_TRANSMISSIVE = 0,
  HF_BC_WALL = 1,
  HF_BC_DISCHARGE = 2, /* value = q [m^2/s], coordinate-axis sign convention */
  HF_BC_DEPTH = 3      /* value = h [m] */
};

/* Integrators (solver-2d/src/sim.rs:38-46). */
enum hf_integrator { HF_FORWARD_EULER = 0, HF_SSPRK2 = 1 };

typedef struct hf_boundary {
  int32_t kind;  /* enum hf_bc_kind */
  int32_t reserved;
  double value;
} hf_boundary;

/* Boundaries2D (boundary.rs:131-140): same field order. */
typedef struct hf_boundaries {
  hf_boundary north; /* i = 0 */
  hf_boundary south; /* i = n_rows - 1 */
  hf_boundary west;  /* j = 0 */
  hf_boundary east;  /* j = n_cols - 1 */
} hf_boundaries;

/* SimulationConfig (sim.rs:49-77) plus the friction threshold the driver
 * passes to manning_friction_step (sim.rs:224, H_DRY) and an opt-in
 * non-finite guard. */
typedef struct hf_config {
  double cfl;              /* (0, 1]; default 0.4 */
  int32_t integrator;      /* enum hf_integrator; default HF_SSPRK2 */
  int32_t check_finite;    /* 0 (default): reference behaviour; 1: HF_ERR_NONFINITE */
  hf_boundaries boundaries;/* default: four walls */
  uint64_t max_steps;      /* run_until budget; default 10,000,000 */
  double max_dt;           /* default 60 s */
  double friction_dry_tol; /* default 1e-6 (H_DRY) */
} hf_config;

/* Mesh2D (geometry.rs:31-47), host memory. */
typedef struct hf_mesh_desc {
  int64_t n_rows;
  int64_t n_cols;
  double dx;
  double dy;
  const double* bed;     /* n_rows*n_cols, row-major */
  const double* manning; /* n_rows*n_cols, or NULL for manning_uniform everywhere */
  double manning_uniform;
} hf_mesh_desc;

/* A device-resident mesh for the low-level entry points (caller-owned). */
typedef struct hf_grid {
  int64_t n_rows;
  int64_t n_cols;
  double dx;
  double dy;
  const double* bed;     /* device, n_rows*n_cols */
  const double* manning; /* device, n_rows*n_cols (may be NULL when unused) */
} hf_grid;

/* Last error message of the calling thread ("" when none). */
const char* hf_last_error(void);
/* ABI version (HF_ABI_VERSION). */
int hf_abi_version(void);
/* Fills the reference defaults (SimulationConfig::default, sim.rs:67-77). */
void hf_config_default(hf_config* cfg);
/* Kernels this library has launched in this process, over every handle and
 * thread: direct launches (not those captured into graphs) plus each kernel
 * node of every graph launch. Read it before and after a region to count
 * the region's kernels. HF_ERR_INVALID_ARG for a NULL count. */
int hf_kernel_launches(uint64_t* count);

/* ---------------------------------------------------------------------------
 * Simulation handle (replaces `Simulation`, sim.rs:119-245). Owns device
 * copies of the mesh and state, one CUDA stream and the step graphs. Not
 * thread-safe: one caller thread per handle.
 * ------------------------------------------------------------------------- */
typedef struct hf_sim hf_sim;

/* Simulation::new (sim.rs:130-165). h/hu/hv are host SoA arrays. */
int hf_sim_create(const hf_mesh_desc* mesh, const double* h, const double* hu,
                  const double* hv, const hf_config* cfg, int device, hf_sim** out);
/* Same with the AoS {h,hu,hv} layout of Conserved2D. */
int hf_sim_create_aos(const hf_mesh_desc* mesh, const double* hhuhv, const hf_config* cfg,
                      int device, hf_sim** out);
int hf_sim_destroy(hf_sim* sim);
/* Simulation::step (sim.rs:204-228), then the attached forcings at t_new. */
int hf_sim_step(hf_sim* sim, double dt_cap, double* dt_out);
/* Simulation::run_until (sim.rs:231-245), forcings applied after every step. */
int hf_sim_run_until(hf_sim* sim, double t_target);
/* Advances exactly n_steps steps with run_until semantics toward t_target
 * (each dt is also capped by t_target - t), stopping early if t_target is
 * reached or a step fails. Steps are replayed from CUDA-graph chunks with no
 * host round trip between them; the clock is read back once at the end.
 * No counterpart in the reference: its callers loop over Simulation::step
 * (sim.rs:204) one step at a time. */
int hf_sim_run_steps(hf_sim* sim, uint64_t n_steps, double t_target);
/* hf_sim_run_steps with every kernel launched directly and CUDA events on the
 * handle's stream around each stage kernel: returns the summed stage-kernel
 * time [ms], the number of stage launches and the whole region's time [ms].
 * Used to measure the stage kernel against its roofline. */
int hf_sim_run_steps_timed(hf_sim* sim, uint64_t n_steps, double t_target, double* stage_ms,
                           uint64_t* stage_launches, double* total_ms);
/* Simulation::time / steps (sim.rs:167-175). */
int hf_sim_time(const hf_sim* sim, double* t);
int hf_sim_steps(const hf_sim* sim, uint64_t* steps);
/* Simulation::states / states_mut (sim.rs:177-186): host copies. */
int hf_sim_get_state(hf_sim* sim, double* h, double* hu, double* hv);
/* max_depth_exceeds_relief(sim.states(), sim.mesh(), factor) (sim.rs:262):
 * the same check on the simulation's current state and bed, on its stream. */
int hf_sim_max_depth_exceeds_relief(hf_sim* sim, double factor, int* exceeds);
int hf_sim_set_state(hf_sim* sim, const double* h, const double* hu, const double* hv);
int hf_sim_get_state_aos(hf_sim* sim, double* hhuhv);
int hf_sim_set_state_aos(hf_sim* sim, const double* hhuhv);
/* Simulation::set_boundaries (sim.rs:194-196). */
int hf_sim_set_boundaries(hf_sim* sim, const hf_boundaries* bcs);
/* Which kernel runs the stages of a simulation; no counterpart in the
 * reference (its passes are fixed). HF_STAGE_TILE computes every 32 x 8
 * tile with its halo (three 256-thread CTAs per SM); HF_STAGE_TILE32 every
 * 32 x 32 tile (one 1024-thread CTA per SM: a smaller halo share, more warps
 * per SM; faster once a grid has enough tiles to fill the GPU);
 * HF_STAGE_STRIP walks 32-column strips in 7-row blocks and carries the halo
 * rows from block to block (fewer faces and slopes per cell, TMA row
 * fetches; needs an even column count). HF_STAGE_AUTO (the default at
 * creation) takes HF_STAGE_TILE32 for grids of at least 100 tiles of 32 x 32
 * and HF_STAGE_TILE below; hf_sim_stage_kernel reports the kernel in use.
 * Results are bit-identical; this is a tuning and diagnostic knob. Forcing
 * HF_STAGE_STRIP where it cannot run returns HF_ERR_UNSUPPORTED (the auto
 * choice stays selected). */
enum { HF_STAGE_AUTO = 0, HF_STAGE_TILE = 1, HF_STAGE_STRIP = 2, HF_STAGE_TILE32 = 3 };
int hf_sim_set_stage_kernel(hf_sim* sim, int kind);
int hf_sim_stage_kernel(const hf_sim* sim, int* kind);
/* The state fields of simulation handles come from a per-device memory pool
 * that keeps the memory of destroyed handles for the next ones (no driver
 * allocation on re-creation). This returns the pool's unused memory to the
 * device. */
int hf_release_cached_memory(int device);
/* Details of the last HF_ERR_DEGENERATE_DT / HF_ERR_STEP_BUDGET (the fields
 * of SimError::DegenerateDt {dt,t,step} / StepBudgetExhausted {steps,t}). */
int hf_sim_error_detail(const hf_sim* sim, double* dt, double* t, uint64_t* step);
/* Device pointers of the resident state (valid until hf_sim_destroy) and the
 * handle's stream, for zero-copy interop. */
int hf_sim_device_state(hf_sim* sim, double** h, double** hu, double** hv, void** stream);
/* Forcings applied after each step at t_new, in this order (the order of
 * solver-2d/examples/uk_ea_test8a_official.rs:203-217):
 *   apply_rain(rate(t_new), dt)          (source.rs:88-101)
 *   apply_point_sources(Q_k(t_new), dt)  (source.rs:52-69)
 * rate(t) and Q_k(t) are piecewise-linear series, held constant outside
 * their first/last stamps; equal stamps make a step. n_points = 0 clears. */
int hf_sim_set_rain(hf_sim* sim, int64_t n_points, const double* t, const double* rate);
/* Source k has rows[k], cols[k] and the series t/q[offsets[k] .. offsets[k+1]). */
int hf_sim_set_point_sources(hf_sim* sim, int64_t n_sources, const int64_t* rows,
                             const int64_t* cols, const int64_t* offsets, const double* t,
                             const double* q);
/* Units of the rain / point-source series: the series is sampled at
 * t / t_div and its value converted as (v * v_mul) / v_div, the arithmetic of
 * a caller that keeps a hyetograph in minutes and mm/h
 * (uk_ea_test8a_official.rs:119-134: t_div = 60, v_mul = 1e-3, v_div = 3600;
 * its inflow: v_mul = cellsize). Default (1, 1, 1) is the identity. */
int hf_sim_set_rain_units(hf_sim* sim, double t_div, double v_mul, double v_div);
int hf_sim_set_point_source_units(hf_sim* sim, double t_div, double v_mul, double v_div);
/* Control points (gauges): after every step the depth at each gauge cell is
 * recorded (the series and fold(0.0, f64::max) peaks the reference's urban
 * example keeps, uk_ea_test8a_official.rs:187-246). Row 0 is the current
 * state; rows beyond `capacity` are counted but not stored. n_gauges = 0
 * clears. */
int hf_sim_set_gauges(hf_sim* sim, int64_t n_gauges, const int64_t* rows, const int64_t* cols,
                      int64_t capacity);
int hf_sim_gauge_peaks(hf_sim* sim, double* peak, double* last);
/* t: n_stored times; h: n_stored x n_gauges depths (either may be NULL). */
int hf_sim_gauge_series(hf_sim* sim, double* t, double* h, int64_t* n_stored, int64_t* n_seen);

/* ---------------------------------------------------------------------------
 * Ensembles: many independent scenarios (different grid sizes, beds,
 * roughness, forcings and horizons) advanced together. No counterpart in the
 * reference, whose callers run one `Simulation` per scenario. Every scenario
 * keeps run_until semantics (sim.rs:231-245) with its own CFL dt, clock,
 * step budget and errors; one batch step advances every unfinished scenario
 * by one of its own steps in a single persistent launch per stage (the tiles
 * of all scenarios in one list), replayed from CUDA graphs. Results are
 * bit-identical to solving each scenario alone with hf_sim_*.
 * Supports the SSP-RK2 integrator (HF_ERR_UNSUPPORTED otherwise).
 * ------------------------------------------------------------------------- */
typedef struct hf_batch hf_batch;

typedef struct hf_scenario_desc {
  hf_mesh_desc mesh;           /* host arrays */
  const double* h;             /* host SoA initial state */
  const double* hu;
  const double* hv;
  hf_config cfg;
  double t_end;                /* horizon: the scenario runs until t >= t_end */
  int64_t n_rain;              /* rain series (see hf_sim_set_rain) */
  const double* rain_t;
  const double* rain_rate;
  int64_t n_sources;           /* point sources (see hf_sim_set_point_sources) */
  const int64_t* src_rows;
  const int64_t* src_cols;
  const int64_t* src_offsets;
  const double* src_t;
  const double* src_q;
} hf_scenario_desc;

int hf_batch_create(int64_t n_scenarios, const hf_scenario_desc* scenarios, int device,
                    hf_batch** out);
int hf_batch_destroy(hf_batch* batch);
/* Up to max_batch_steps batch steps; stops early when every scenario has
 * reached its horizon or failed. n_unfinished (optional) receives the count
 * still running. A scenario's failure (DegenerateDt, budget) stops only it:
 * read it with hf_batch_scenario_info. */
int hf_batch_run(hf_batch* batch, uint64_t max_batch_steps, int64_t* n_unfinished);
/* Clock, step count and status (0 or an hf_status_code) of scenario k. */
int hf_batch_scenario_info(const hf_batch* batch, int64_t k, double* t, uint64_t* steps,
                           int* status);
/* Host copy of scenario k's state. */
int hf_batch_get_state(hf_batch* batch, int64_t k, double* h, double* hu, double* hv);
/* Tile schedule of the batched stage kernel. 0: static stride over the tiles
 * in scenario order; 1: dynamic (CTAs take the next tile from an atomic
 * counter); 2 / 3: the same with the scenarios largest first. -1 (default):
 * the first hf_batch_run with at least 64 steps times two 8-step chunks of
 * each and keeps the fastest (those are real steps). No schedule changes any
 * result. */
int hf_batch_set_schedule(hf_batch* batch, int schedule);
/* The schedule in use (-1 before tuning) and, after tuning, the measured
 * milliseconds of each candidate's two chunks (tune_ms[4], may be NULL). */
int hf_batch_schedule(const hf_batch* batch, int* schedule, double* tune_ms);

/* ---------------------------------------------------------------------------
 * Serving: continuous batching of flood scenarios on one GPU. No counterpart
 * in the reference. Scenarios are admitted into slots while a slot is free
 * and their fields (64 B per cell) fit the HBM budget, stay resident on the
 * device between steps, and advance together with every other admitted
 * scenario (one persistent launch per stage over all their tiles, one
 * captured CUDA graph for any mix). A scenario finishes at its horizon (or on
 * its own error) and is collected, which frees its slot and memory for the
 * next request. Each scenario's result is bit-identical to solving it alone.
 * ------------------------------------------------------------------------- */
typedef struct hf_server hf_server;

int hf_server_create(int device, uint64_t hbm_budget_bytes, int max_slots, hf_server** out);
int hf_server_destroy(hf_server* server);
/* Copies the scenario to the device and admits it (*slot receives its id), or
 * returns HF_ERR_CAPACITY when no slot is free or it would exceed the budget. */
int hf_server_admit(hf_server* server, const hf_scenario_desc* scenario, int* slot);
/* Up to n_batch_steps batch steps over the admitted scenarios; returns early
 * once some scenario finishes. n_finished receives the count awaiting
 * collection. */
int hf_server_advance(hf_server* server, uint64_t n_batch_steps, int* n_finished);
/* Ids of finished, uncollected slots (up to cap). */
int hf_server_finished(hf_server* server, int* slots, int cap, int* n);
/* Result of a finished slot (state may be NULL to skip it), then frees it. */
int hf_server_collect(hf_server* server, int slot, double* h, double* hu, double* hv, double* t,
                      uint64_t* steps, int* status);
/* Bytes of the budget in use and occupied slots. */
int hf_server_usage(const hf_server* server, uint64_t* bytes_in_use, int* occupied);

/* ---------------------------------------------------------------------------
 * Differentiation with respect to the per-cell Manning field.
 *
 * The reference differentiates by running its generic step with T = Dual
 * (autograd/src/dual.rs; e.g. examples/m1_inverse_manning_demo.rs): forward
 * mode, one direction per run, dt taken from values (update.rs:113-136).
 * hf_tangent is that forward mode on the GPU with the same Dual rules
 * (branches on values, max/min ties average the derivatives, sqrt(0) has
 * derivative 0, powf's n x^(n-1)). hf_grad_manning is reverse mode, which the
 * reference does not have: the gradient with respect to every Manning value
 * (and the initial state) from one forward and one backward sweep, with
 * checkpoints every `checkpoint_every` steps and the steps in between
 * recomputed. It is the transpose of the tangent map: for any direction v,
 * dot(gradient, v) equals hf_tangent's dJ along v up to rounding.
 *
 * A problem is a scenario (mesh, initial state, config, forcings, horizon
 * t_end) and gauge cells (row-major indices). A run takes steps like
 * hf_sim_run_until (dt = min(cfl dt, max_dt, t_end - t)) until t_end or
 * n_steps steps, and its misfit is
 *   J = sum over steps k = 1..K and gauges g of (h_k[cell_g] - h_obs[k-1][g])^2
 * with h_obs an [n_steps][n_gauges] table (zeros until set).
 * ------------------------------------------------------------------------- */
typedef struct hf_calib hf_calib;

int hf_calib_create(const hf_scenario_desc* scenario, int64_t n_steps, int64_t n_gauges,
                    const int64_t* gauge_cells, int64_t checkpoint_every, int device,
                    hf_calib** out);
int hf_calib_destroy(hf_calib* calib);
int hf_calib_set_observations(hf_calib* calib, const double* h_obs);
/* Forward run with the Manning field `manning` (one value per cell). J and
 * the gauge depths of each step ([K][n_gauges], K = *n_run) are optional
 * outputs. With replay_dt = 0 the steps take their CFL dt and the sequence is
 * recorded; with replay_dt != 0 they take the dt sequence recorded by the
 * last such run (frozen dt, as the tangent and the gradient see it). */
int hf_calib_run(hf_calib* calib, const double* manning, int replay_dt, double* J,
                 double* gauge_h, int64_t* n_run);
/* Forward-mode (Dual) run along the direction (dn, dh0, dhu0, dhv0); any may
 * be NULL (zero). Returns J and its directional derivative dJ. */
int hf_tangent(hf_calib* calib, const double* manning, const double* dn, const double* dh0,
               const double* dhu0, const double* dhv0, double* J, double* dJ);
/* Vector mode (DualN<N>, autograd/src/dual_n.rs; used by
 * solver-2d/examples/m1_forward_scaling.rs): n_lanes directions in one run.
 * dn, dh0, dhu0 and dhv0 hold n_lanes consecutive arrays of one value per
 * cell (any may be NULL: zero); dJ receives n_lanes values. Each lane is
 * bit-identical to hf_tangent along that direction. The lanes run side by
 * side in one launch per stage (a grid per lane), so on grids too small to
 * fill the GPU the extra lanes cost little. 1 <= n_lanes <= 1024. */
int hf_tangent_lanes(hf_calib* calib, const double* manning, int64_t n_lanes, const double* dn,
                     const double* dh0, const double* dhu0, const double* dhv0, double* J,
                     double* dJ);
/* Final tangent of one lane of the last hf_tangent_lanes run (any pointer
 * may be NULL). */
int hf_calib_lane_state(hf_calib* calib, int64_t lane, double* dh, double* dhu, double* dhv);
/* Reverse mode: J and dJ/dn (one value per cell); the gradient with respect
 * to the initial state is written when grad_h0 / grad_hu0 / grad_hv0 are
 * non-NULL. */
int hf_grad_manning(hf_calib* calib, const double* manning, double* J, double* grad_n,
                    double* grad_h0, double* grad_hu0, double* grad_hv0);
/* Final state of the last run, and the final tangent of the last hf_tangent
 * (any pointer may be NULL). */
int hf_calib_final_state(hf_calib* calib, double* h, double* hu, double* hv, double* dh,
                         double* dhu, double* dhv);
/* dt sequence recorded by the last run without replay (*n values). */
int hf_calib_dt(hf_calib* calib, double* dts, int64_t* n);

/* ---------------------------------------------------------------------------
 * Rasters on the host: ESRI ASCII grids (solver-2d/src/ascii_grid.rs) and the
 * depth raster / land-cover roughness helpers of solver-2d/src/io.rs.
 * ------------------------------------------------------------------------- */
typedef struct hf_ascii_grid_header {
  int64_t ncols;
  int64_t nrows;
  double xllcorner;     /* south-west corner of the grid */
  double yllcorner;
  double cellsize;
  double nodata_value;
} hf_ascii_grid_header;

/* read_ascii_grid (ascii_grid.rs:101-160): the six header lines in order
 * (ncols, nrows, xllcorner, yllcorner, cellsize, NODATA_value; keys matched
 * case-insensitively), then exactly ncols * nrows numbers in any line layout,
 * row 0 = the first data row (north). A path ending in ".gz" is gunzipped.
 * *data receives a malloc'd row-major array (free with hf_free_buffer).
 * Errors: HF_ERR_INVALID_ARG (I/O, header, unparsable value),
 * HF_ERR_SHAPE_MISMATCH (value count). */
int hf_read_ascii_grid(const char* path, hf_ascii_grid_header* header, double** data);
void hf_free_buffer(void* p);
/* Writes an ESRI ASCII grid (gzip when the path ends in ".gz") whose values
 * hf_read_ascii_grid returns bit for bit (%.17g). No counterpart in the
 * reference, which writes GeoTIFF through surtgis. */
int hf_write_ascii_grid(const char* path, const hf_ascii_grid_header* header, const double* data);
/* depth_raster_from_states (io.rs:216-234): out[k] = h[k], or nodata where
 * h[k] <= H_DRY when use_nodata != 0. */
int hf_depth_raster(int64_t ncell, const double* h, int use_nodata, double nodata, double* out);
/* esa_worldcover_to_manning (io.rs:192-207): Manning n of an ESA WorldCover
 * land-cover class (0.040 for unlisted codes). */
double hf_worldcover_manning(int code);

/* ---------------------------------------------------------------------------
 * Low-level entry points on caller-owned device buffers, mirroring the
 * reference's free functions. All run on `stream` and are asynchronous
 * unless they return a host value (hf_cfl_time_step synchronizes it).
 * ------------------------------------------------------------------------- */
typedef struct hf_workspace hf_workspace;
/* StepWorkspace2D::new (update.rs:758): stage buffer + reduction scratch. */
int hf_workspace_create(int64_t n_rows, int64_t n_cols, int device, hf_workspace** out);
int hf_workspace_destroy(hf_workspace* ws);

/* cfl_time_step (update.rs:148) when bcs == NULL, cfl_time_step_with_bcs
 * (update.rs:170) otherwise. Writes +inf for a dry domain. */
int hf_cfl_time_step(const hf_grid* grid, const double* h, const double* hu, const double* hv,
                     const hf_boundaries* bcs, double cfl, hf_workspace* ws, void* stream,
                     double* dt_out);
/* forward_euler_step_with (update.rs:805): in place on h/hu/hv. */
int hf_forward_euler_step(const hf_grid* grid, double* h, double* hu, double* hv,
                          const hf_boundaries* bcs, double dt, hf_workspace* ws, void* stream);
/* ssprk2_step_with (update.rs:1255): in place on h/hu/hv. */
int hf_ssprk2_step(const hf_grid* grid, double* h, double* hu, double* hv,
                   const hf_boundaries* bcs, double dt, hf_workspace* ws, void* stream);
/* manning_friction_step (source.rs:130): reads grid->manning. */
int hf_manning_friction_step(const hf_grid* grid, double* h, double* hu, double* hv, double dt,
                             double dry_tol, void* stream);
/* apply_rain (source.rs:88). */
int hf_apply_rain(int64_t n_cells, double* h, double* hu, double* hv, double rate, double dt,
                  void* stream);
/* apply_point_sources (source.rs:52): rows/cols/q_mass are HOST arrays,
 * applied in order (repeated cells accumulate like the reference's loop). */
int hf_apply_point_sources(const hf_grid* grid, double* h, double* hu, double* hv,
                           int64_t n_sources, const int64_t* rows, const int64_t* cols,
                           const double* q_mass, double dt, void* stream);
/* max_depth_exceeds_relief (sim.rs:248-271): the reference's plausibility
 * check for a finite blow-up. *exceeds = 1 when the largest depth (folded
 * from 0, NaN skipped) exceeds factor * max(bed.max() - bed.min(), 1 m),
 * else 0. The max/min reductions run on the device over h and the bed
 * (device arrays of the grid's shape); the workspace supplies the
 * accumulators and the pinned readback. Synchronizes `stream`. */
int hf_max_depth_exceeds_relief(const hf_grid* grid, const double* h, double factor,
                                hf_workspace* ws, void* stream, int* exceeds);
/* ssprk2_step without allocating: no counterpart in the reference (whose
 * StepWorkspace2D is always caller-allocated host memory). Same result as
 * hf_ssprk2_step, but the stage buffer and control block live in a fixed
 * array inside this library instead of an hf_workspace, so the call never
 * runs cudaMalloc/cudaFree. It is meant for callers that cannot allocate
 * device memory: hosts that reserve nearly all GPU memory for their own
 * caching allocator up front, and latency-critical loops that must not
 * trigger the device-wide synchronization cudaMalloc/cudaFree can cause.
 * - Grids of at most HF_NOALLOC_MAX_CELLS cells (larger: HF_ERR_INVALID_ARG).
 *   The array costs every GPU that loads the library 24 MiB + 512 B, held
 *   until the process exits.
 * - The first call on a device resolves the array's device address
 *   (cudaGetSymbolAddress, with `device` current); make that first call
 *   before any stream capture. The address is kept for the life of the
 *   process: after cudaDeviceReset on that device it is stale, so do not
 *   call this entry point again in that process.
 * - All calls on a device share the array and see the previous call's
 *   leftovers (the control block is cleared each call): calls whose GPU work
 *   overlaps, e.g. on two streams, race. Serialize them. */
#define HF_NOALLOC_MAX_CELLS (1 << 20)
int hf_ssprk2_step_noalloc(const hf_grid* grid, double* h, double* hu, double* hv,
                           const hf_boundaries* bcs, double dt, int device, void* stream);
/* hllc_flux_x / hllc_flux_y (riemann.rs:80, 97) over n faces (device
 * arrays, 3 doubles per state {h,hu,hv}, 3 per flux {mass,x_mom,y_mom}). */
int hf_hllc_flux(int x_dir, int64_t n, const double* ul, const double* ur, double* flux,
                 void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HYDROFLUX_GPU_H */
