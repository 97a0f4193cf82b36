// hf_strip.cuh -- the streaming f64 stage kernel.
//
// k_stage_pf computes a 32 x 8 tile with a 4-cell halo from scratch: 2.83
// Audusse+HLLC faces, 3.0 limited-slope cells and 2.1 primitive cells per
// cell, most of the excess in the halo rows above and below the tile (on
// its 32 x 32 tiles: 2.32, 2.39 and 1.41). This kernel is built with the
// 32 x 8 geometry's 256-thread CTAs only. Here a
// CTA instead walks DOWN a 32-column strip in blocks of STRIP_ROWS (7) rows:
// every array (depth, primitives, slopes, faces, alpha) keeps the rows the
// next block shares with this one, which are shifted to the top of their
// buffers, and a block computes only its new rows: 2.16 faces, 2.19 slope
// cells and 1.19 primitive cells per cell. With 7-row blocks each phase of a
// block is close to a whole number of passes of the 256 threads (slopes 490
// items, faces 483, alpha + the next block's primitives 504, update 224).
//
// The new input rows of the next block (depth, bed, hu, hv; 40 columns,
// out-of-grid cells zero-filled by the copy engine) are fetched with TMA
// (cp.async.bulk.tensor, no multicast) into staging buffers while the
// current block computes; completion is an mbarrier with a bounded wait.
//
// Work is split into contiguous ranges of the strip-major sequence of blocks
// (q = strip * blocks_per_strip + block): one equal range per CTA while the
// grid is wet, ranges of 16 blocks claimed from a counter once many blocks
// are dry (k_stage_strip). A CTA starts from scratch (a "cold" block, as
// k_stage_pf does for a tile) only at the start of a range and where the
// range enters a new strip. Interior blocks whose depths are all at or
// below H_DRY write their zero slopes and faces instead of computing them.
//
// Every cell is computed by the same item functions as k_stage_pf's
// (slope_at, face_at, alpha_at, update_at in hf_stage.cuh), on the same
// values: results are bit-identical.
#pragma once

#include <cuda_runtime.h>

#include "hf_stage.cuh"

namespace hf {
inline namespace HF_GEOM {

namespace {

constexpr int SR = STRIP_ROWS;
constexpr int SH4 = SR + 8;   // depth rows [-4, SR + 4)
constexpr int SH3 = SR + 6;   // z, eta, u, v rows [-3, SR + 3)
constexpr int SHX = SR + 2;   // x slope rows [-1, SR + 1)
constexpr int SHY = SR + 4;   // y slope rows [-2, SR + 2)
constexpr int SHFX = SR + 2;  // x face rows [-1, SR + 1)
constexpr int SHFY = SR + 3;  // y faces [-1, SR + 2)
constexpr int SHA = SR + 2;   // alpha rows [-1, SR + 1)
constexpr int STW = 40;       // a staged row: columns [-4, 36)
constexpr int STH = SR + 1;   // staged depth rows: [3, SR + 4) of the next block
constexpr int STQ = SR;       // staged bed / hu / hv rows: [3, SR + 3) of the next block
constexpr unsigned STRIP_TX_BYTES = (STH + 3 * STQ) * STW * sizeof(double);
static_assert(STW == R4W && SR * TX <= NTHREADS, "strip geometry");

// Same row widths and row / column offsets as StageSmem (i4, i3, isx, ...),
// fewer rows, plus the staging buffers (TMA destinations, 128-byte aligned).
struct StripSmem {
  alignas(128) double st_h[STH * STW];
  alignas(128) double st_z[STQ * STW];
  alignas(128) double st_u[STQ * STW];  // hu, then u once converted
  alignas(128) double st_v[STQ * STW];  // hv, then v
  alignas(16) double h[SH4 * R4W];
  double z[SH3 * R3W], eta[SH3 * R3W], u[SH3 * R3W], v[SH3 * R3W];
  double sxe[SHX * SXW], sxu[SHX * SXW], sxv[SHX * SXW];
  double sye[SHY * SYW], syu[SHY * SYW], syv[SHY * SYW];
  double fxm[SHFX * FXW], fxnm[SHFX * FXW], fxnp[SHFX * FXW], fxt[SHFX * FXW];
  double fym[SHFY * FYW], fynm[SHFY * FYW], fynp[SHFY * FYW], fyt[SHFY * FYW];
  double a[SHA * AW];
  unsigned long long mbar;
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(b)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ void tma_load_rows(double* dst, const CUtensorMap* map, int col,
                                              int row, unsigned long long* b) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(col), "r"(row), "r"(smem_addr(b))
      : "memory");
}

// Thread 0: fetch the new input rows of the block whose first row is gi0n
// (strip columns from gj0) into the staging buffers. The caller has passed a
// barrier since the staging buffers were last read.
__device__ __forceinline__ void strip_fetch(StripSmem& S, const StripMaps& M, int gi0n,
                                            int gj0) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                   smem_addr(&S.mbar)),
               "r"(STRIP_TX_BYTES)
               : "memory");
  tma_load_rows(S.st_h, &M.h, gj0 - 4, gi0n + 3, &S.mbar);
  tma_load_rows(S.st_z, &M.z, gj0 - 4, gi0n + 3, &S.mbar);
  tma_load_rows(S.st_u, &M.hu, gj0 - 4, gi0n + 3, &S.mbar);
  tma_load_rows(S.st_v, &M.hv, gj0 - 4, gi0n + 3, &S.mbar);
}

// Every thread: wait (bounded) for the fetch of the given phase parity. A
// wait that gives up is reported in the control block; the CTA then stops
// (the decision is uniform over the CTA).
__device__ __forceinline__ bool strip_wait(StripSmem& S, unsigned parity, Ctrl* ctrl) {
  bool ok = false;
  for (int it = 0; it < (1 << 22) && !ok; ++it) ok = mbar_try_wait(&S.mbar, parity);
  const bool any_fail = __syncthreads_or(!ok);
  if (any_fail && threadIdx.x == 0) atomicCAS(&ctrl->status, 0, -6);  // HF_ERR_TIMEOUT
  return !any_fail;
}

__device__ __forceinline__ bool interior_block(const StageArgs& A, int gi0, int gj0) {
  return gi0 >= 4 && gj0 >= 4 && gi0 + SR + 4 <= A.nr && gj0 + TX + 4 <= A.nc;
}

// Dry blocks. When every depth a block's slopes and faces read is at or
// below H_DRY and the block reaches no side, every slope is the limiter's
// zero (a dry cell within two cells, update.rs:459-540) and every face is a
// dry-dry face with zero flux (update.rs:890-926): the block writes those
// zeros instead of computing them, and its cells then take the isolated-dry
// update. Votes over the depth buffer entries [k0, k1) (with a barrier);
// a dry block is counted for the schedule of the next step.
__device__ __forceinline__ bool strip_all_dry(StripSmem& S, int k0, int k1, Ctrl* ctrl) {
  bool dry = true;
  for (int k = k0 + threadIdx.x; k < k1; k += NTHREADS) dry &= S.h[k] <= H_DRY;
  const bool all = __syncthreads_and(dry);
  if (all && threadIdx.x == 0) atomicAdd(&ctrl->strip_dry, 1ull);
  return all;
}
__device__ __forceinline__ void zero_rows(double* a, double* b, double* c, int k0, int k1) {
  for (int k = k0 + threadIdx.x; k < k1; k += NTHREADS) a[k] = b[k] = c[k] = 0.0;
}
__device__ __forceinline__ void zero_faces(StripSmem& S, int x0, int x1, int y0, int y1) {
  for (int k = x0 + threadIdx.x; k < x1; k += NTHREADS)
    S.fxm[k] = S.fxnm[k] = S.fxnp[k] = S.fxt[k] = 0.0;
  for (int k = y0 + threadIdx.x; k < y1; k += NTHREADS)
    S.fym[k] = S.fynm[k] = S.fynp[k] = S.fyt[k] = 0.0;
}

// A block from scratch: inputs (plain loads, zeros outside the grid),
// primitives, slopes and faces of every row of its buffers.
template <bool IN>
__device__ void strip_cold(const StageArgs& A, StripSmem& S, int gi0, int gj0) {
  const int nr = A.nr, nc = A.nc;
  const int tid = threadIdx.x;
  for (int k = tid; k < SH4 * R4W; k += NTHREADS) {
    const int r = k / R4W, cc = k - r * R4W;
    const int gi = gi0 + r - 4, gj = gj0 + cc - 4;
    const bool real = IN || (gi >= 0 && gi < nr && gj >= 0 && gj < nc);
    const int64_t g = (int64_t)gi * nc + gj;
    const double hh = real ? A.in_h[g] : 0.0;
    S.h[k] = hh;
    if (r >= 1 && r < SH4 - 1 && cc >= 1 && cc < R4W - 1) {
      const int k3 = (r - 1) * R3W + (cc - 1);
      double zz = 0.0, e = 0.0, uu = 0.0, vv = 0.0;
      if (real) {
        zz = A.z[g];
        e = hh + zz;
        if (hh > H_VEL) {
          uu = hfa::div_rn_pos(A.in_hu[g], hh);
          vv = hfa::div_rn_pos(A.in_hv[g], hh);
        }
      }
      S.z[k3] = zz;
      S.eta[k3] = e;
      S.u[k3] = uu;
      S.v[k3] = vv;
    }
  }
  if constexpr (IN) {  // the vote is also the barrier after the loads
    if (strip_all_dry(S, 0, SH4 * R4W, A.ctrl)) {
      zero_rows(S.sxe, S.sxu, S.sxv, 0, SHX * SXW);
      zero_rows(S.sye, S.syu, S.syv, 0, SHY * SYW);
      zero_faces(S, 0, SHFX * FXW, 0, SHFY * FYW);
      __syncthreads();
      return;
    }
  } else {
    __syncthreads();
  }
  for (int k = tid; k < SHX * SXW + SHY * SYW; k += NTHREADS) {
    if (k < SHX * SXW) {
      const int r = k / SXW;
      slope_at<double, IN>(A, S, gi0, gj0, r - 1, k - r * SXW - 2, true);
    } else {
      const int kk = k - SHX * SXW, r = kk / SYW;
      slope_at<double, IN>(A, S, gi0, gj0, r - 2, kk - r * SYW - 1, false);
    }
  }
  __syncthreads();
  for (int k = tid; k < SHFX * FXW + SHFY * FYW; k += NTHREADS) {
    if (k < SHFX * FXW) {
      const int r = k / FXW;
      face_at<double, IN>(A, S, gi0, gj0, r - 1, k - r * FXW - 1, true);
    } else {
      const int kk = k - SHFX * FXW, r = kk / FYW;
      face_at<double, IN>(A, S, gi0, gj0, r - 1, kk - r * FYW - 1, false);
    }
  }
  __syncthreads();
}

// Alpha of rows [a0, SR + 1) of the current block (every column of its
// buffer: the corners of the last row are the ring columns of the next
// block's first row) and, when the next block is streamed, the primitives
// of its staged rows (u = hu / h, v = hv / h in place; 0 at h <= H_VEL).
template <bool IN>
__device__ __forceinline__ void strip_alpha_prims(const StageArgs& A, StripSmem& S, int gi0,
                                                  int gj0, int a0, bool prims, double dt_dx,
                                                  double dt_dy) {
  const int na = (SR + 1 - a0) * AW;
  const int n = na + (prims ? STQ * (STW - 2) : 0);
  for (int k = threadIdx.x; k < n; k += NTHREADS) {
    if (k < na) {
      const int r = k / AW;
      alpha_at<double, IN>(A, S, gi0, gj0, a0 + r, k - r * AW - 1, dt_dx, dt_dy);
    } else {
      const int kk = k - na, r = kk / (STW - 2);
      const int s = r * STW + (kk - r * (STW - 2)) + 1;  // staged columns [-3, 35)
      const double hh = S.st_h[s];
      double uu = 0.0, vv = 0.0;
      if (hh > H_VEL) {
        uu = hfa::div_rn_pos(S.st_u[s], hh);
        vv = hfa::div_rn_pos(S.st_v[s], hh);
      }
      S.st_u[s] = uu;
      S.st_v[s] = vv;
    }
  }
}

__device__ __forceinline__ void copy_rows(double* dst, const double* src, int n) {
  for (int k = threadIdx.x; k < n; k += NTHREADS) dst[k] = src[k];
}

// Rows the next block shares with this one move to the top of each buffer
// (row r + SR -> row r), then the staged rows fill the rows below them.
__device__ __forceinline__ void strip_shift(StripSmem& S) {
  // carried rows; sources and destinations are disjoint within each buffer
  copy_rows(S.h, S.h + SR * R4W, (SH4 - SR - 1) * R4W);  // rows [-4, 3); row 3 is staged
  copy_rows(S.z, S.z + SR * R3W, (SH3 - SR) * R3W);
  copy_rows(S.eta, S.eta + SR * R3W, (SH3 - SR) * R3W);
  copy_rows(S.u, S.u + SR * R3W, (SH3 - SR) * R3W);
  copy_rows(S.v, S.v + SR * R3W, (SH3 - SR) * R3W);
  copy_rows(S.sxe, S.sxe + SR * SXW, (SHX - SR) * SXW);
  copy_rows(S.sxu, S.sxu + SR * SXW, (SHX - SR) * SXW);
  copy_rows(S.sxv, S.sxv + SR * SXW, (SHX - SR) * SXW);
  copy_rows(S.sye, S.sye + SR * SYW, (SHY - SR) * SYW);
  copy_rows(S.syu, S.syu + SR * SYW, (SHY - SR) * SYW);
  copy_rows(S.syv, S.syv + SR * SYW, (SHY - SR) * SYW);
  copy_rows(S.fxm, S.fxm + SR * FXW, (SHFX - SR) * FXW);
  copy_rows(S.fxnm, S.fxnm + SR * FXW, (SHFX - SR) * FXW);
  copy_rows(S.fxnp, S.fxnp + SR * FXW, (SHFX - SR) * FXW);
  copy_rows(S.fxt, S.fxt + SR * FXW, (SHFX - SR) * FXW);
  copy_rows(S.fym, S.fym + SR * FYW, (SHFY - SR) * FYW);
  copy_rows(S.fynm, S.fynm + SR * FYW, (SHFY - SR) * FYW);
  copy_rows(S.fynp, S.fynp + SR * FYW, (SHFY - SR) * FYW);
  copy_rows(S.fyt, S.fyt + SR * FYW, (SHFY - SR) * FYW);
  copy_rows(S.a, S.a + SR * AW, (SHA - SR) * AW);
  __syncthreads();
  // staged rows: depth rows [3, SR + 4), primitives rows [3, SR + 3)
  copy_rows(S.h + (SH4 - SR - 1) * R4W, S.st_h, STH * STW);
  for (int k = threadIdx.x; k < STQ * (STW - 2); k += NTHREADS) {
    const int r = k / (STW - 2), c = k - r * (STW - 2);
    const int s = r * STW + c + 1, d = (SH3 - SR + r) * R3W + c;
    const double zz = S.st_z[s];
    S.z[d] = zz;
    S.eta[d] = S.st_h[s] + zz;
    S.u[d] = S.st_u[s];
    S.v[d] = S.st_v[s];
  }
}

// Slopes (x rows [1, SR + 1), y rows [2, SR + 2)) and then faces (x rows
// [1, SR + 1), y faces [2, SR + 2)) of the rows a streamed block adds.
template <bool IN>
__device__ __forceinline__ void strip_new_rows(const StageArgs& A, StripSmem& S, int gi0,
                                               int gj0) {
  constexpr int NX = SR * SXW, NY = SR * SYW;
  // new slopes and faces read the depths of rows [0, SR + 4)
  if constexpr (IN) {
    if (strip_all_dry(S, 4 * R4W, SH4 * R4W, A.ctrl)) {
      zero_rows(S.sxe, S.sxu, S.sxv, isx(1, -2), isx(SR + 1, -2));
      zero_rows(S.sye, S.syu, S.syv, isy(2, -1), isy(SR + 2, -1));
      zero_faces(S, ifx(1, -1), ifx(SR + 1, -1), ify(2, -1), ify(SR + 2, -1));
      __syncthreads();
      return;
    }
  }
  for (int k = threadIdx.x; k < NX + NY; k += NTHREADS) {
    if (k < NX) {
      const int r = k / SXW;
      slope_at<double, IN>(A, S, gi0, gj0, 1 + r, k - r * SXW - 2, true);
    } else {
      const int kk = k - NX, r = kk / SYW;
      slope_at<double, IN>(A, S, gi0, gj0, 2 + r, kk - r * SYW - 1, false);
    }
  }
  __syncthreads();
  constexpr int FX = SR * FXW, FY = SR * FYW;
  for (int k = threadIdx.x; k < FX + FY; k += NTHREADS) {
    if (k < FX) {
      const int r = k / FXW;
      face_at<double, IN>(A, S, gi0, gj0, 1 + r, k - r * FXW - 1, true);
    } else {
      const int kk = k - FX, r = kk / FYW;
      face_at<double, IN>(A, S, gi0, gj0, 2 + r, kk - r * FYW - 1, false);
    }
  }
  __syncthreads();
}

template <bool IN>
__device__ __forceinline__ void strip_update(const StageArgs& A, StripSmem& S, int gi0, int gj0,
                                             long long q, double dt, double dt_dx, double dt_dy,
                                             double& sxm, double& sym,
                                             unsigned long long& nonfin) {
  int src_lo = 0, src_hi = 0;
  if (A.finalize && A.f.n_src > 0) {
    src_lo = A.f.blk_start[q];
    src_hi = A.f.blk_start[q + 1];
  }
  if (threadIdx.x < SR * TX)
    update_at<double, IN>(A, S, gi0, gj0, threadIdx.x / TX, threadIdx.x % TX, dt, dt_dx, dt_dy,
                          A.f.blk_order, src_lo, src_hi, sxm, sym, nonfin);
}

}  // namespace

}  // namespace HF_GEOM
}  // namespace hf
