// hf_kernels.cu -- sm_100a kernels of the solver-2d explicit step that do not
// depend on the stage tile's shape, and the launch bookkeeping.
//
// The reference (franciscoparrao/hydroflux, solver-2d/src/update.rs:805-1211)
// runs one forward-Euler stage as eleven full-grid passes over a ~241 B/cell
// workspace. Here one stage is ONE kernel (hf_tiles.cu): a CTA stages a tile
// plus a 4-cell halo of (h, z, eta, u, v) in shared memory and runs every
// pass of the stage on it -- dry snapshot, primitives, limited slopes, face
// beds, Audusse+HLLC faces, alpha rescaling, FV update with the bed source
// and the moisture floor -- so a stage reads the state once and writes it
// once. The last stage of a step also folds in the SSP-RK2 combination,
// Manning friction, rain, point sources and the next step's CFL reduction,
// and the step size never leaves the device (Ctrl). This file holds the step
// control kernels around those stages (dt, clock, forcing increments,
// gauges), the standalone free-function kernels (friction, rain, point
// sources, HLLC, the relief check), the launch accounting and geom_ops().
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

namespace hf {

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

const GeomOps& geom_ops(int geom) { return geom == kGeomLarge ? geom_ops_g32() : geom_ops_g8(); }

int geom_for(int64_t nr, int64_t nc) {
  const int64_t t = (int64_t)tiles_along(nc, TX) * tiles_along(nr, kGeomTileH[kGeomLarge]);
  return t >= kLargeTilesMin ? kGeomLarge : kGeomSmall;
}

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

int launch_batch_control(Ctrl* ctrls, const StageArgs* args, int n, void* stream,
                         int* counters) {
  k_batch_control<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ctrls, args, n, counters);
  return launched(stream);
}

int launch_batch_commit(Ctrl* ctrls, int n, void* stream) {
  k_batch_commit<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ctrls, n);
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
