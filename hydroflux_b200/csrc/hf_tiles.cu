// hf_tiles.cu -- the tile-shaped stage kernels of the solver-2d explicit
// step, compiled once per tile geometry.
//
// A CTA stages a TX x TY tile plus a 4-cell halo of (h, z, eta, u, v) in
// shared memory and runs every pass of a forward-Euler stage on it (the
// phases are in hf_stage.cuh). This file holds the kernels whose work is cut
// into those tiles -- the single-grid stage (k_stage_pf), the ensemble stage
// (k_stage_batch), the forward-Euler finalize and the CFL reductions -- and
// their launchers. The build compiles it twice: with the 32 x 8 geometry
// (namespace g8, 256 threads, three CTAs per SM), which also carries the
// strip kernel and the DualD tangent kernels, and with the 32 x 32 geometry
// (namespace g32, 1024 threads, one CTA per SM). The geometry's symbols live
// in its inline namespace, so both builds link into one library; the host
// code reaches the one a grid uses through geom_ops().
#include <cuda_runtime.h>

#include <type_traits>

#include "hf_device.cuh"
#include "hf_internal.h"
#include "hf_stage.cuh"
#if HF_GEOM_PRIMARY
#include "hf_strip.cuh"
#endif

namespace hf {
inline namespace HF_GEOM {

namespace {
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
}  // namespace

// Blocks per SM the stage kernel is compiled for: in the 32 x 8 geometry the
// f64 tile takes 71 KB of shared memory (three CTAs per SM) and the DualD
// tile 112 KB (two); in the 32 x 32 geometry the f64 tile takes 211 KB (one).
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

#if HF_GEOM_PRIMARY
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
#endif  // HF_GEOM_PRIMARY

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
    if (blockIdx.x == 0 && threadIdx.x == 0 && !A.batched) commit_clock(A.ctrl);
  }
}

#if HF_GEOM_PRIMARY
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
#endif  // HF_GEOM_PRIMARY

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
      if (kPartialPass && (int)threadIdx.x / TX + ROWS_PER_PASS * q >= TY) continue;
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
      if (kPartialPass && (int)threadIdx.x / TX + ROWS_PER_PASS * q >= TY) continue;
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
      if (kPartialPass && (int)threadIdx.x / TX + ROWS_PER_PASS * q >= TY) continue;
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

// ------------------------------------------------------------- launchers
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

#if HF_GEOM_PRIMARY
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
#endif  // HF_GEOM_PRIMARY

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

int launch_cfl(const StageArgs& a, int with_ghosts, int grid, void* stream) {
  k_cfl<<<grid, NTHREADS, 0, (cudaStream_t)stream>>>(a, with_ghosts);
  return launched(stream);
}

}  // namespace HF_GEOM

// The geometry's entry points, for geom_ops().
const GeomOps& HF_GEOM_OPS() {
  static const GeomOps ops = {TY, NTHREADS, &stage_grid_size, &launch_stage, &launch_finalize,
                              &launch_cfl, &launch_stage_batch, &launch_cfl_batch};
  return ops;
}

}  // namespace hf
