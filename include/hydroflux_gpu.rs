//! Rust FFI declarations of include/hydroflux_gpu.h: the module a maintainer
//! adds to hydroflux-solver-2d (as src/ffi.rs of a `-b200` crate) to put the
//! crate's `Simulation`, free functions and calibration loop on the B200
//! library. Every item mirrors the C header one to one; status codes map
//! onto `SimError` as the header states. There is no Rust toolchain in the
//! build image, so this file is not compiled here; tests/
//! test_integration_shim.py checks every declaration against the header
//! (names, parameter and return types, struct fields in order).
//!
//! Linking: build.rs emits `cargo:rustc-link-search=<repo>/hydroflux_b200`
//! and `cargo:rustc-link-lib=dylib=hydroflux_gpu`. The library links the
//! CUDA runtime statically and needs only the NVIDIA driver at run time.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

pub const HF_ABI_VERSION: c_int = 1;

// Status codes (enum hf_status_code): 0 = OK; -1..-4 are SimError's variants.
pub const HF_OK: c_int = 0;
pub const HF_ERR_SHAPE_MISMATCH: c_int = -1;
pub const HF_ERR_INVALID_CONFIG: c_int = -2;
pub const HF_ERR_DEGENERATE_DT: c_int = -3;
pub const HF_ERR_STEP_BUDGET: c_int = -4;
pub const HF_ERR_NONFINITE: c_int = -5;
pub const HF_ERR_TIMEOUT: c_int = -6;
pub const HF_ERR_CUDA: c_int = -7;
pub const HF_ERR_INVALID_ARG: c_int = -8;
pub const HF_ERR_OUT_OF_MEMORY: c_int = -9;
pub const HF_ERR_UNSUPPORTED: c_int = -10;
pub const HF_ERR_CAPACITY: c_int = -11;

// Boundary kinds (BoundaryKind, boundary.rs:35-48), integrators, stage kernels.
pub const HF_BC_TRANSMISSIVE: i32 = 0;
pub const HF_BC_WALL: i32 = 1;
pub const HF_BC_DISCHARGE: i32 = 2;
pub const HF_BC_DEPTH: i32 = 3;
pub const HF_FORWARD_EULER: i32 = 0;
pub const HF_SSPRK2: i32 = 1;
pub const HF_STAGE_AUTO: c_int = 0;
pub const HF_STAGE_TILE: c_int = 1;
pub const HF_STAGE_STRIP: c_int = 2;
pub const HF_STAGE_TILE32: c_int = 3;
pub const HF_NOALLOC_MAX_CELLS: i64 = 1 << 20;

#[repr(C)] #[derive(Clone, Copy)]
pub struct HfBoundary { pub kind: i32, pub reserved: i32, pub value: f64 }

#[repr(C)] #[derive(Clone, Copy)]
pub struct HfBoundaries { pub north: HfBoundary, pub south: HfBoundary,
                          pub west: HfBoundary, pub east: HfBoundary }

#[repr(C)] #[derive(Clone, Copy)]
pub struct HfConfig { pub cfl: f64, pub integrator: i32, pub check_finite: i32,
                      pub boundaries: HfBoundaries, pub max_steps: u64,
                      pub max_dt: f64, pub friction_dry_tol: f64 }

#[repr(C)] #[derive(Clone, Copy)]
pub struct HfMeshDesc { pub n_rows: i64, pub n_cols: i64, pub dx: f64, pub dy: f64,
                        pub bed: *const f64, pub manning: *const f64,
                        pub manning_uniform: f64 }

#[repr(C)] #[derive(Clone, Copy)]
pub struct HfGrid { pub n_rows: i64, pub n_cols: i64, pub dx: f64, pub dy: f64,
                    pub bed: *const f64, pub manning: *const f64 }

#[repr(C)] #[derive(Clone, Copy)]
pub struct HfScenarioDesc {
    pub mesh: HfMeshDesc, pub h: *const f64, pub hu: *const f64, pub hv: *const f64,
    pub cfg: HfConfig, pub t_end: f64,
    pub n_rain: i64, pub rain_t: *const f64, pub rain_rate: *const f64,
    pub n_sources: i64, pub src_rows: *const i64, pub src_cols: *const i64,
    pub src_offsets: *const i64, pub src_t: *const f64, pub src_q: *const f64,
}

#[repr(C)] #[derive(Clone, Copy)]
pub struct HfAsciiGridHeader { pub ncols: i64, pub nrows: i64, pub xllcorner: f64,
                               pub yllcorner: f64, pub cellsize: f64, pub nodata_value: f64 }

// Opaque handles.
pub enum HfSim {}
pub enum HfBatch {}
pub enum HfServer {}
pub enum HfCalib {}
pub enum HfWorkspace {}

#[link(name = "hydroflux_gpu")]
extern "C" {
    pub fn hf_last_error() -> *const c_char;
    pub fn hf_abi_version() -> c_int;
    pub fn hf_config_default(cfg: *mut HfConfig);
    pub fn hf_kernel_launches(count: *mut u64) -> c_int;
    pub fn hf_sim_create(mesh: *const HfMeshDesc, h: *const f64, hu: *const f64, hv: *const f64,
                         cfg: *const HfConfig, device: c_int, out: *mut *mut HfSim) -> c_int;
    pub fn hf_sim_create_aos(mesh: *const HfMeshDesc, hhuhv: *const f64, cfg: *const HfConfig,
                             device: c_int, out: *mut *mut HfSim) -> c_int;
    pub fn hf_sim_destroy(sim: *mut HfSim) -> c_int;
    pub fn hf_sim_step(sim: *mut HfSim, dt_cap: f64, dt_out: *mut f64) -> c_int;
    pub fn hf_sim_run_until(sim: *mut HfSim, t_target: f64) -> c_int;
    pub fn hf_sim_run_steps(sim: *mut HfSim, n_steps: u64, t_target: f64) -> c_int;
    pub fn hf_sim_run_steps_timed(sim: *mut HfSim, n_steps: u64, t_target: f64, stage_ms: *mut f64,
                                  stage_launches: *mut u64, total_ms: *mut f64) -> c_int;
    pub fn hf_sim_time(sim: *const HfSim, t: *mut f64) -> c_int;
    pub fn hf_sim_steps(sim: *const HfSim, steps: *mut u64) -> c_int;
    pub fn hf_sim_get_state(sim: *mut HfSim, h: *mut f64, hu: *mut f64, hv: *mut f64) -> c_int;
    pub fn hf_sim_max_depth_exceeds_relief(sim: *mut HfSim, factor: f64,
                                           exceeds: *mut c_int) -> c_int;
    pub fn hf_sim_set_state(sim: *mut HfSim, h: *const f64, hu: *const f64,
                            hv: *const f64) -> c_int;
    pub fn hf_sim_get_state_aos(sim: *mut HfSim, hhuhv: *mut f64) -> c_int;
    pub fn hf_sim_set_state_aos(sim: *mut HfSim, hhuhv: *const f64) -> c_int;
    pub fn hf_sim_set_boundaries(sim: *mut HfSim, bcs: *const HfBoundaries) -> c_int;
    pub fn hf_sim_set_stage_kernel(sim: *mut HfSim, kind: c_int) -> c_int;
    pub fn hf_sim_stage_kernel(sim: *const HfSim, kind: *mut c_int) -> c_int;
    pub fn hf_release_cached_memory(device: c_int) -> c_int;
    pub fn hf_sim_error_detail(sim: *const HfSim, dt: *mut f64, t: *mut f64,
                               step: *mut u64) -> c_int;
    pub fn hf_sim_device_state(sim: *mut HfSim, h: *mut *mut f64, hu: *mut *mut f64,
                               hv: *mut *mut f64, stream: *mut *mut c_void) -> c_int;
    pub fn hf_sim_set_rain(sim: *mut HfSim, n_points: i64, t: *const f64,
                           rate: *const f64) -> c_int;
    pub fn hf_sim_set_point_sources(sim: *mut HfSim, n_sources: i64, rows: *const i64,
                                    cols: *const i64, offsets: *const i64, t: *const f64,
                                    q: *const f64) -> c_int;
    pub fn hf_sim_set_rain_units(sim: *mut HfSim, t_div: f64, v_mul: f64, v_div: f64) -> c_int;
    pub fn hf_sim_set_point_source_units(sim: *mut HfSim, t_div: f64, v_mul: f64,
                                         v_div: f64) -> c_int;
    pub fn hf_sim_set_gauges(sim: *mut HfSim, n_gauges: i64, rows: *const i64, cols: *const i64,
                             capacity: i64) -> c_int;
    pub fn hf_sim_gauge_peaks(sim: *mut HfSim, peak: *mut f64, last: *mut f64) -> c_int;
    pub fn hf_sim_gauge_series(sim: *mut HfSim, t: *mut f64, h: *mut f64, n_stored: *mut i64,
                               n_seen: *mut i64) -> c_int;
    pub fn hf_batch_create(n_scenarios: i64, scenarios: *const HfScenarioDesc, device: c_int,
                           out: *mut *mut HfBatch) -> c_int;
    pub fn hf_batch_destroy(batch: *mut HfBatch) -> c_int;
    pub fn hf_batch_run(batch: *mut HfBatch, max_batch_steps: u64,
                        n_unfinished: *mut i64) -> c_int;
    pub fn hf_batch_scenario_info(batch: *const HfBatch, k: i64, t: *mut f64, steps: *mut u64,
                                  status: *mut c_int) -> c_int;
    pub fn hf_batch_get_state(batch: *mut HfBatch, k: i64, h: *mut f64, hu: *mut f64,
                              hv: *mut f64) -> c_int;
    pub fn hf_batch_set_schedule(batch: *mut HfBatch, schedule: c_int) -> c_int;
    pub fn hf_batch_schedule(batch: *const HfBatch, schedule: *mut c_int,
                             tune_ms: *mut f64) -> c_int;
    pub fn hf_server_create(device: c_int, hbm_budget_bytes: u64, max_slots: c_int,
                            out: *mut *mut HfServer) -> c_int;
    pub fn hf_server_destroy(server: *mut HfServer) -> c_int;
    pub fn hf_server_admit(server: *mut HfServer, scenario: *const HfScenarioDesc,
                           slot: *mut c_int) -> c_int;
    pub fn hf_server_advance(server: *mut HfServer, n_batch_steps: u64,
                             n_finished: *mut c_int) -> c_int;
    pub fn hf_server_finished(server: *mut HfServer, slots: *mut c_int, cap: c_int,
                              n: *mut c_int) -> c_int;
    pub fn hf_server_collect(server: *mut HfServer, slot: c_int, h: *mut f64, hu: *mut f64,
                             hv: *mut f64, t: *mut f64, steps: *mut u64,
                             status: *mut c_int) -> c_int;
    pub fn hf_server_usage(server: *const HfServer, bytes_in_use: *mut u64,
                           occupied: *mut c_int) -> c_int;
    pub fn hf_calib_create(scenario: *const HfScenarioDesc, n_steps: i64, n_gauges: i64,
                           gauge_cells: *const i64, checkpoint_every: i64, device: c_int,
                           out: *mut *mut HfCalib) -> c_int;
    pub fn hf_calib_destroy(calib: *mut HfCalib) -> c_int;
    pub fn hf_calib_set_observations(calib: *mut HfCalib, h_obs: *const f64) -> c_int;
    pub fn hf_calib_run(calib: *mut HfCalib, manning: *const f64, replay_dt: c_int, J: *mut f64,
                        gauge_h: *mut f64, n_run: *mut i64) -> c_int;
    pub fn hf_tangent(calib: *mut HfCalib, manning: *const f64, dn: *const f64, dh0: *const f64,
                      dhu0: *const f64, dhv0: *const f64, J: *mut f64, dJ: *mut f64) -> c_int;
    pub fn hf_tangent_lanes(calib: *mut HfCalib, manning: *const f64, n_lanes: i64, dn: *const f64,
                            dh0: *const f64, dhu0: *const f64, dhv0: *const f64, J: *mut f64,
                            dJ: *mut f64) -> c_int;
    pub fn hf_calib_lane_state(calib: *mut HfCalib, lane: i64, dh: *mut f64, dhu: *mut f64,
                               dhv: *mut f64) -> c_int;
    pub fn hf_grad_manning(calib: *mut HfCalib, manning: *const f64, J: *mut f64, grad_n: *mut f64,
                           grad_h0: *mut f64, grad_hu0: *mut f64, grad_hv0: *mut f64) -> c_int;
    pub fn hf_calib_final_state(calib: *mut HfCalib, h: *mut f64, hu: *mut f64, hv: *mut f64,
                                dh: *mut f64, dhu: *mut f64, dhv: *mut f64) -> c_int;
    pub fn hf_calib_dt(calib: *mut HfCalib, dts: *mut f64, n: *mut i64) -> c_int;
    pub fn hf_read_ascii_grid(path: *const c_char, header: *mut HfAsciiGridHeader,
                              data: *mut *mut f64) -> c_int;
    pub fn hf_free_buffer(p: *mut c_void);
    pub fn hf_write_ascii_grid(path: *const c_char, header: *const HfAsciiGridHeader,
                               data: *const f64) -> c_int;
    pub fn hf_depth_raster(ncell: i64, h: *const f64, use_nodata: c_int, nodata: f64,
                           out: *mut f64) -> c_int;
    pub fn hf_worldcover_manning(code: c_int) -> f64;
    pub fn hf_workspace_create(n_rows: i64, n_cols: i64, device: c_int,
                               out: *mut *mut HfWorkspace) -> c_int;
    pub fn hf_workspace_destroy(ws: *mut HfWorkspace) -> c_int;
    pub fn hf_cfl_time_step(grid: *const HfGrid, h: *const f64, hu: *const f64, hv: *const f64,
                            bcs: *const HfBoundaries, cfl: f64, ws: *mut HfWorkspace,
                            stream: *mut c_void, dt_out: *mut f64) -> c_int;
    pub fn hf_forward_euler_step(grid: *const HfGrid, h: *mut f64, hu: *mut f64, hv: *mut f64,
                                 bcs: *const HfBoundaries, dt: f64, ws: *mut HfWorkspace,
                                 stream: *mut c_void) -> c_int;
    pub fn hf_ssprk2_step(grid: *const HfGrid, h: *mut f64, hu: *mut f64, hv: *mut f64,
                          bcs: *const HfBoundaries, dt: f64, ws: *mut HfWorkspace,
                          stream: *mut c_void) -> c_int;
    pub fn hf_manning_friction_step(grid: *const HfGrid, h: *mut f64, hu: *mut f64, hv: *mut f64,
                                    dt: f64, dry_tol: f64, stream: *mut c_void) -> c_int;
    pub fn hf_apply_rain(n_cells: i64, h: *mut f64, hu: *mut f64, hv: *mut f64, rate: f64, dt: f64,
                         stream: *mut c_void) -> c_int;
    pub fn hf_apply_point_sources(grid: *const HfGrid, h: *mut f64, hu: *mut f64, hv: *mut f64,
                                  n_sources: i64, rows: *const i64, cols: *const i64,
                                  q_mass: *const f64, dt: f64, stream: *mut c_void) -> c_int;
    pub fn hf_max_depth_exceeds_relief(grid: *const HfGrid, h: *const f64, factor: f64,
                                       ws: *mut HfWorkspace, stream: *mut c_void,
                                       exceeds: *mut c_int) -> c_int;
    pub fn hf_ssprk2_step_noalloc(grid: *const HfGrid, h: *mut f64, hu: *mut f64, hv: *mut f64,
                                  bcs: *const HfBoundaries, dt: f64, device: c_int,
                                  stream: *mut c_void) -> c_int;
    pub fn hf_hllc_flux(x_dir: c_int, n: i64, ul: *const f64, ur: *const f64, flux: *mut f64,
                        stream: *mut c_void) -> c_int;
}
