// hf_noalloc.cu -- SSP-RK2 step that allocates no device memory.
//
// hf_ssprk2_step needs scratch on the GPU: the stage-1 state (three arrays
// of n_rows*n_cols doubles) and a small control block carrying dt. Normally
// the caller provides it through an hf_workspace, which calls cudaMalloc.
// Some callers cannot do that: a host that hands almost all GPU memory to its
// own caching allocator up front (so a library's cudaMalloc fails, or
// fragments that pool), and a latency-critical loop that must not call
// cudaMalloc/cudaFree because they can synchronize the whole device. For
// them, hf_ssprk2_step_noalloc keeps its scratch in the file-scope array
// below, which the CUDA runtime reserves on every GPU that loads this library
// and keeps until the process exits.
//
// Limits and rules (also stated in include/hydroflux_gpu.h):
//   * at most HF_NOALLOC_MAX_CELLS cells per call (2^20: e.g. 1024 x 1024),
//     i.e. 24 MiB of stage buffer + 512 B of control block per GPU;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current);
//     make that first call before any stream capture. The address is kept
//     for the life of the process: after cudaDeviceReset on that device it
//     is stale, and the entry point must not be called again;
//   * all calls on a device share the one array, which keeps the last call's
//     contents: calls whose work overlaps on the GPU (other streams, other
//     host threads) race and corrupt each other, so serialize them;
//   * nothing here calls cudaMalloc, cudaFree or any allocating routine.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/hydroflux_gpu.h"
#include "hf_internal.h"

using namespace hf;

namespace {

// Control block (first 64 doubles = 512 bytes), then h1, hu1, hv1.
constexpr size_t kCtrlDoubles = 64;
constexpr size_t kScratchDoubles = kCtrlDoubles + 3 * (size_t)HF_NOALLOC_MAX_CELLS;
static_assert(sizeof(Ctrl) <= kCtrlDoubles * sizeof(double), "control block does not fit");

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

namespace {

std::mutex g_setup_mu;
double* g_scratch_ptr[64] = {nullptr};

// Message goes to hf_last_error(), like every other entry point.
int noalloc_fail(int code, const std::string& msg) { return record_error(code, msg.c_str()); }

// The launchers keep the launch's own error (cudaGetLastError has cleared it).
int launch_failed() {
  return noalloc_fail(HF_ERR_CUDA, std::string("kernel launch: ") +
                                       cudaGetErrorString(last_launch_error()));
}

struct CurrentDevice {
  int prev = -1;
  bool ok = false;
  explicit CurrentDevice(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = (prev == dev) || cudaSetDevice(dev) == cudaSuccess;
  }
  ~CurrentDevice() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Device address of the scratch array on `device` (current), looked up once.
int scratch_on(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return noalloc_fail(HF_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                           cudaGetErrorString(e));
    }
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[device];
  return HF_OK;
}

}  // namespace

extern "C" int hf_ssprk2_step_noalloc(const hf_grid* grid, double* h, double* hu, double* hv,
                                      const hf_boundaries* bcs, double dt, int device,
                                      void* stream) {
  if (!grid || !h || !hu || !hv || !grid->bed)
    return noalloc_fail(HF_ERR_INVALID_ARG, "null argument");
  if (grid->n_rows > (int64_t)HF_NOALLOC_MAX_CELLS || grid->n_cols > (int64_t)HF_NOALLOC_MAX_CELLS ||
      grid->n_rows * grid->n_cols > (int64_t)HF_NOALLOC_MAX_CELLS) {
    char buf[200];
    std::snprintf(buf, sizeof buf,
                  "grid of %lld x %lld cells exceeds the no-allocation step's fixed scratch of "
                  "%d cells; use hf_ssprk2_step with an hf_workspace",
                  (long long)grid->n_rows, (long long)grid->n_cols, HF_NOALLOC_MAX_CELLS);
    return noalloc_fail(HF_ERR_INVALID_ARG, buf);
  }
  if (device < 0 || device >= 64) return noalloc_fail(HF_ERR_INVALID_ARG, "bad device index");
  // The same shape, spacing and boundary checks as hf_ssprk2_step.
  int rc = check_grid_desc(grid);
  if (rc != HF_OK) return rc;
  hf_boundary t{HF_BC_TRANSMISSIVE, 0, 0.0};
  const hf_boundaries b = bcs ? *bcs : hf_boundaries{t, t, t, t};
  rc = check_boundaries(b, grid->n_rows, grid->n_cols);
  if (rc != HF_OK) return rc;
  CurrentDevice cur(device);
  if (!cur.ok) return noalloc_fail(HF_ERR_CUDA, "cannot make the device current");
  double* base = nullptr;
  rc = scratch_on(device, &base);
  if (rc != HF_OK) return rc;
  Ctrl* ctrl = reinterpret_cast<Ctrl*>(base);
  double* h1 = base + kCtrlDoubles;
  double* hu1 = h1 + HF_NOALLOC_MAX_CELLS;
  double* hv1 = hu1 + HF_NOALLOC_MAX_CELLS;
  cudaStream_t st = (cudaStream_t)stream;
  // The control block keeps the previous call's values: start it from zero.
  cudaError_t e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(HF_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  }
  const GeomOps& o = geom_ops(geom_for(grid->n_rows, grid->n_cols));
  StageArgs a;
  std::memset(&a, 0, sizeof a);
  a.nr = (int)grid->n_rows;
  a.nc = (int)grid->n_cols;
  a.tiles_x = tiles_along(grid->n_cols, TX);
  a.tiles_y = tiles_along(grid->n_rows, o.tile_h);
  a.dx = grid->dx;
  a.dy = grid->dy;
  a.rx = hfa::make_recip(a.dx);
  a.ry = hfa::make_recip(a.dy);
  a.z = grid->bed;
  a.n = grid->manning;
  a.bc = boundaries_dev(b);
  a.ctrl = ctrl;
  const int gsz = o.grid_size(a.tiles_x * a.tiles_y, device);
  if (launch_set_fixed(ctrl, dt, stream)) return launch_failed();
  // Stage 1: U -> scratch (every real cell of h1/hu1/hv1 is written before
  // stage 2 reads it, so the stale stage buffer needs no clearing).
  a.in_h = h; a.in_hu = hu; a.in_hv = hv;
  a.out_h = h1; a.out_hu = hu1; a.out_hv = hv1;
  a.un_h = h; a.un_hu = hu; a.un_hv = hv;
  if (o.stage(a, gsz, stream)) return launch_failed();
  // Stage 2 + convex combination, in place on the caller's state.
  a.in_h = h1; a.in_hu = hu1; a.in_hv = hv1;
  a.out_h = h; a.out_hu = hu; a.out_hv = hv;
  a.combine = 1;
  if (o.stage(a, gsz, stream)) return launch_failed();
  return HF_OK;
}
