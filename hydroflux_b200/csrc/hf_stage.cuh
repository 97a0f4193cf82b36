// hf_stage.cuh -- the fused stage tile shared by the forward kernels
// (hf_tiles.cu) and the adjoint kernels (hf_adjoint.cu): shared-memory
// layout of a tile and its halo, the forward phases of one stage on a tile
// (generic over the scalar: double or DualD), the per-cell epilogue
// (friction, forcings) and the CFL reduction helpers.
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

#include <type_traits>

#include "hf_device.cuh"
#include "hf_internal.h"

namespace hf {
inline namespace HF_GEOM {

namespace {

// Shared-memory regions of the stage kernel, relative to the tile origin.
constexpr int R4W = TX + 8, R4H = TY + 8, R4N = R4W * R4H;  // h: rows/cols [-4, T+4)
constexpr int R3W = TX + 6, R3H = TY + 6, R3N = R3W * R3H;  // z, eta, u, v: [-3, T+3)
constexpr int SXW = TX + 4, SXH = TY + 2, SXN = SXW * SXH;  // x slopes: rows [-1,TY], cols [-2,TX+1]
constexpr int SYW = TX + 2, SYH = TY + 4, SYN = SYW * SYH;  // y slopes: rows [-2,TY+1], cols [-1,TX]
constexpr int FXW = TX + 3, FXH = TY + 2, FXN = FXW * FXH;  // x faces: rows [-1,TY], faces [-1,TX+1]
constexpr int FYW = TX + 2, FYH = TY + 3, FYN = FYW * FYH;  // y faces: faces [-1,TY+1], cols [-1,TX]
constexpr int AW = TX + 2, AH = TY + 2, AN = AW * AH;       // alpha: rows [-1,TY], cols [-1,TX]

template <class T> struct StageSmemT {
  T h[R4N];
  double z[R3N];
  // eta, u and v start 8 bytes past a 16-byte boundary: the pipelined stage
  // stages z, hu and hv there with 16-byte copies of column pairs (even
  // global column, odd halo index), which then land on 16-byte boundaries.
  double pad_;
  T eta[R3N], u[R3N], v[R3N];
  T sxe[SXN], sxu[SXN], sxv[SXN];
  T sye[SYN], syu[SYN], syv[SYN];
  T fxm[FXN], fxnm[FXN], fxnp[FXN], fxt[FXN];  // mass, normal(minus), normal(plus), tangential
  T fym[FYN], fynm[FYN], fynp[FYN], fyt[FYN];
  T a[AN];
};
using StageSmem = StageSmemT<double>;

// The DualD tile would take 129 KB in the layout above: one CTA per SM. It
// runs the x faces before the y faces (SplitFaces), so the y faces can be
// written over the x momentum slopes (dead once the x faces are done) and
// alpha over the y momentum slopes (dead once the y faces are done): 112 KB,
// two CTAs per SM. The eta slopes of both directions stay (the bed source
// reads them).
template <> struct StageSmemT<DualD> {
  DualD h[R4N];
  double z[R3N];
  DualD eta[R3N], u[R3N], v[R3N];
  DualD sxe[SXN], sye[SYN];
  DualD fxm[FXN], fxnm[FXN], fxnp[FXN], fxt[FXN];
  union {
    struct { DualD sxu[SXN], sxv[SXN]; };
    struct { DualD fym[FYN], fynm[FYN], fynp[FYN], fyt[FYN]; };
  };
  union {
    struct { DualD syu[SYN], syv[SYN]; };
    DualD a[AN];
  };
};
template <class T> struct SplitFaces { static constexpr bool value = false; };
template <> struct SplitFaces<DualD> { static constexpr bool value = true; };

__device__ __forceinline__ int i4(int li, int lj) { return (li + 4) * R4W + (lj + 4); }
__device__ __forceinline__ int i3(int li, int lj) { return (li + 3) * R3W + (lj + 3); }
__device__ __forceinline__ int isx(int li, int lj) { return (li + 1) * SXW + (lj + 2); }
__device__ __forceinline__ int isy(int li, int lj) { return (li + 2) * SYW + (lj + 1); }
__device__ __forceinline__ int ifx(int li, int f) { return (li + 1) * FXW + (f + 1); }
__device__ __forceinline__ int ify(int g, int lj) { return (g + 1) * FYW + (lj + 1); }
__device__ __forceinline__ int ia(int li, int lj) { return (li + 1) * AW + (lj + 1); }

// Ghost bed only (boundary.rs:335-367), for the face beds of the source term.
__device__ __forceinline__ double ghost_bed(int kind, double z0, double z1) {
  return (kind == BC_TRANSMISSIVE || kind == BC_WALL) ? z0 : z0 * 2.0 - z1;
}

// Reduce (sx, sy) over the block and fold into the control block.
__device__ void block_reduce_speeds(double sx, double sy, unsigned long long nonfin, Ctrl* c) {
  __shared__ double wx[NTHREADS / 32], wy[NTHREADS / 32];
  __shared__ unsigned long long wn[NTHREADS / 32];
  for (int o = 16; o > 0; o >>= 1) {
    sx = fmax(sx, __shfl_xor_sync(0xffffffffu, sx, o));
    sy = fmax(sy, __shfl_xor_sync(0xffffffffu, sy, o));
    nonfin += __shfl_xor_sync(0xffffffffu, nonfin, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    wx[warp] = sx;
    wy[warp] = sy;
    wn[warp] = nonfin;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NTHREADS / 32; ++w) {
      sx = fmax(sx, wx[w]);
      sy = fmax(sy, wy[w]);
      nonfin += wn[w];
    }
    // Non-negative doubles order like their bit patterns.
    atomicMax(&c->sx_bits, (unsigned long long)__double_as_longlong(sx));
    atomicMax(&c->sy_bits, (unsigned long long)__double_as_longlong(sy));
    if (nonfin) atomicAdd(&c->nonfinite, nonfin);
  }
  __syncthreads();  // wx/wy/wn may be written again by the next call
}

// Final state of a cell for the next step: friction (source.rs:130-165),
// rain (source.rs:88-101) and the point sources of the cell
// (source.rs:52-69), in the reference caller's order
// (examples/uk_ea_test8a_official.rs:203-217).
template <class T>
__device__ __forceinline__ void finalize_cell(const StageArgs& A, const Ctrl* c, double dt,
                                              int gi, int gj, int64_t g, const int* order,
                                              int src_lo, int src_hi, T& h, T& hu, T& hv) {
  friction_cell<T>(h, hu, hv, Field<T>::ld(A.n, A.tan.n, g), dt, A.dry_tol);
  if (c->rain_on) {
    const T nh = h + c->rain_dh;
    if (val(nh) <= 0.0) {
      h = cst<T>(0.0); hu = cst<T>(0.0); hv = cst<T>(0.0);
    } else {
      h = nh;
    }
  }
  for (int s = src_lo; s < src_hi; ++s) {
    const int k = order[s];
    if (A.f.src_row[k] == gi && A.f.src_col[k] == gj) {
      h = r_max(h + A.f.src_dh[k], cst<T>(0.0));
      if (val(h) == 0.0) {
        hu = cst<T>(0.0);
        hv = cst<T>(0.0);
      }
    }
  }
}

// CFL contribution of one cell of the final state, with the ghost cells of
// the sides it touches (cfl_time_step_with_bcs, update.rs:170-208).
// IN: the cell is known not to touch a side (an interior tile).
template <bool IN = false>
__device__ __forceinline__ void cfl_cell(const StageArgs& A, int gi, int gj, int64_t g, double h,
                                         double hu, double hv, double& sx, double& sy) {
  cell_speeds(h, hu, hv, sx, sy);
  if constexpr (IN) return;
  const int nr = A.nr, nc = A.nc;
  const double* dn = nullptr;
  if (gj == 0)
    ghost_speeds(ghost_cell<double>(SIDE_WEST, A.bc, h, hu, hv, A.z, A.n, dn, g, g + 1, A.dx), sx, sy);
  if (gj == nc - 1)
    ghost_speeds(ghost_cell<double>(SIDE_EAST, A.bc, h, hu, hv, A.z, A.n, dn, g, g - 1, A.dx), sx, sy);
  if (gi == 0)
    ghost_speeds(ghost_cell<double>(SIDE_NORTH, A.bc, h, hu, hv, A.z, A.n, dn, g, g + nc, A.dy), sx, sy);
  if (gi == nr - 1)
    ghost_speeds(ghost_cell<double>(SIDE_SOUTH, A.bc, h, hu, hv, A.z, A.n, dn, g, g - nc, A.dy), sx, sy);
}

__device__ __forceinline__ void commit_clock(Ctrl* c) {
  c->t = c->t_new;
  c->steps += 1;
  if (c->mode == MODE_RUN) c->budget -= 1;
  c->cfl_valid = 1;
}

}  // namespace

// 8-byte asynchronous global -> shared copy; `valid` false zero-fills the
// destination without reading `gmem` (which must still be a valid address).
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
  const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(gmem),
               "r"(bytes)
               : "memory");
}
// 16-byte copy of a column pair (both addresses 16-byte aligned); valid ==
// false zero-fills.
__device__ __forceinline__ void cp_async16(double* smem, const double* gmem, bool valid) {
  const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gmem),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Shared memory of the pipelined f64 stage: the tile plus a staging buffer
// for the next tile's depth (its z, hu and hv are staged in eta, u and v,
// which are dead once the faces are done).
struct StagePfSmem {
  StageSmem s;
  alignas(16) double hst[R4N];
};
static_assert(R3W % 2 == 0 && R4W % 2 == 0 && TX % 2 == 0, "column pairs");
static_assert(offsetof(StageSmem, h) % 16 == 0 && offsetof(StageSmem, eta) % 16 == 8 &&
                  offsetof(StageSmem, u) % 16 == 8 && offsetof(StageSmem, v) % 16 == 8 &&
                  offsetof(StagePfSmem, hst) % 16 == 0,
              "16-byte staging copies");

// Starts the copies of a tile's raw inputs: h (4-cell halo) into hst and z,
// hu, hv (3-cell halo) into S.eta, S.u, S.v; cells outside the grid read as
// zeros. Completed by cp_async_wait_all() and a barrier.
//
// With an even column count and 16-byte aligned fields, the copies move
// column pairs (16 bytes; the halo's first column gj0 - 4 is even, so every
// pair starts on an even global column and lies wholly inside or wholly
// outside the grid). The 3-cell halo rows (columns gj0-3 .. gj0+TX+2) take
// TX/2 + 1 pairs and one single column at each end. Otherwise every element
// is copied alone.
__device__ __forceinline__ void stage_prefetch(const StageArgs& A, StageSmem& S, double* hst,
                                               int tile) {
  const int nr = A.nr, nc = A.nc;
  const int tyi = tile / A.tiles_x;
  const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;
  const uintptr_t any = (uintptr_t)A.in_h | (uintptr_t)A.z | (uintptr_t)A.in_hu |
                        (uintptr_t)A.in_hv;
  if (((nc & 1) | (int)(any & 15)) == 0) {
    constexpr int PW = R4W / 2;  // pairs per 4-cell halo row
    for (int k = threadIdx.x; k < R4H * PW; k += NTHREADS) {
      const int r = k / PW, cc = 2 * (k - r * PW);
      const int gi = gi0 + r - 4, gj = gj0 + cc - 4;
      const bool real = gi >= 0 && gi < nr && gj >= 0 && gj < nc;
      cp_async16(&hst[r * R4W + cc], A.in_h + (real ? (int64_t)gi * nc + gj : 0), real);
    }
    constexpr int NP = (R3W - 2) / 2;  // pairs per 3-cell halo row (columns 2 .. R3W-1)
    for (int k = threadIdx.x; k < R3H * (NP + 2); k += NTHREADS) {
      const int r3 = k / (NP + 2), j = k - r3 * (NP + 2);
      const int cc = j < NP ? 2 + 2 * j : (j == NP ? 1 : R4W - 2);  // column of the 4-halo row
      const int gi = gi0 + r3 - 3, gj = gj0 + cc - 4;
      const bool real = gi >= 0 && gi < nr && gj >= 0 && gj < nc;
      const int64_t g = real ? (int64_t)gi * nc + gj : 0;
      const int k3 = r3 * R3W + (cc - 1);
      if (j < NP) {
        cp_async16(&S.eta[k3], A.z + g, real);
        cp_async16(&S.u[k3], A.in_hu + g, real);
        cp_async16(&S.v[k3], A.in_hv + g, real);
      } else {
        cp_async8(&S.eta[k3], A.z + g, real);
        cp_async8(&S.u[k3], A.in_hu + g, real);
        cp_async8(&S.v[k3], A.in_hv + g, real);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    return;
  }
  for (int k = threadIdx.x; k < R4N; k += NTHREADS) {
    const int r = k / R4W, cc = k - r * R4W;
    const int gi = gi0 + r - 4, gj = gj0 + cc - 4;
    const bool real = gi >= 0 && gi < nr && gj >= 0 && gj < nc;
    const int64_t g = real ? (int64_t)gi * nc + gj : 0;
    cp_async8(&hst[k], A.in_h + g, real);
    if (r >= 1 && r < R4H - 1 && cc >= 1 && cc < R4W - 1) {
      const int k3 = (r - 1) * R3W + (cc - 1);
      cp_async8(&S.eta[k3], A.z + g, real);
      cp_async8(&S.u[k3], A.in_hu + g, real);
      cp_async8(&S.v[k3], A.in_hv + g, real);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Per-item work of one forward-Euler stage for the strip kernel (a column of
// blocks that carries the halo rows from one block to the next). The same
// arithmetic, in the same order, as the tile phases further below, which
// keep it inline (written as one function per item, the tile kernel
// measured 6% slower). The strip buffers use the tile's row widths and
// offsets of row and column 0 (i4, i3, isx, ...); SM is the layout's type.
// (gi0, gj0) is the grid cell of local (0, 0).
// ---------------------------------------------------------------------------

// Limited slopes of cell (li, lj) along x (xd) or y: update.rs:459-540.
template <class T, bool IN, class SM>
__device__ __forceinline__ void slope_at(const StageArgs& A, SM& S, int gi0, int gj0, int li,
                                         int lj, bool xd) {
  const int nr = A.nr, nc = A.nc;
  const T Z = cst<T>(0.0);
  const int gi = gi0 + li, gj = gj0 + lj;
  if (!IN && (gi < 0 || gi >= nr || gj < 0 || gj >= nc)) return;
  const int ga = xd ? gj : gi;
  const int na = xd ? nc : nr;
  const int st4 = xd ? 1 : R4W;
  const int st3 = xd ? 1 : R3W;
  const hfa::RecipD& rd = xd ? A.rx : A.ry;
  T se = Z, su = Z, sv = Z;
  if (IN || na >= 2) {
    const int lo = IN ? -2 : max(ga - 2, 0) - ga, hi = IN ? 2 : min(ga + 2, na - 1) - ga;
    const int c4 = i4(li, lj);
    bool anyd = false;
    for (int o = lo; o <= hi; ++o) anyd |= val(S.h[c4 + o * st4]) <= H_DRY;
    if (!anyd) {
      const int c3 = i3(li, lj);
      if (!IN && ga == 0) {
        const int r3 = c3 + st3;
        se = dvr(S.eta[r3] - S.eta[c3], rd);  // / dx or / dy
        su = dvr(S.u[r3] - S.u[c3], rd);
        sv = dvr(S.v[r3] - S.v[c3], rd);
      } else if (!IN && ga == na - 1) {
        const int l3 = c3 - st3;
        se = dvr(S.eta[c3] - S.eta[l3], rd);
        su = dvr(S.u[c3] - S.u[l3], rd);
        sv = dvr(S.v[c3] - S.v[l3], rd);
      } else {
        const int l3 = c3 - st3, r3 = c3 + st3;
        se = minmod_div<T>(S.eta[c3] - S.eta[l3], S.eta[r3] - S.eta[c3], rd);
        su = minmod_div<T>(S.u[c3] - S.u[l3], S.u[r3] - S.u[c3], rd);
        sv = minmod_div<T>(S.v[c3] - S.v[l3], S.v[r3] - S.v[c3], rd);
      }
    }
  }
  if (xd) {
    const int k = isx(li, lj);
    S.sxe[k] = se;
    S.sxu[k] = su;
    S.sxv[k] = sv;
  } else {
    const int k = isy(li, lj);
    S.sye[k] = se;
    S.syu[k] = su;
    S.syv[k] = sv;
  }
}

// Face fluxes: update.rs:676-728 (face beds), 890-926 (fluxes). x face
// (xd): row li, face lj (between cells lj - 1 and lj); y face: face li
// (between rows li - 1 and li), column lj.
template <class T, bool IN, class SM>
__device__ __forceinline__ void face_at(const StageArgs& A, SM& S, int gi0, int gj0, int li,
                                        int lj, bool xd) {
  const int nr = A.nr, nc = A.nc;
  const T Z = cst<T>(0.0);
  const int gf = xd ? gj0 + lj : gi0 + li;  // face index along the normal
  const int na = xd ? nc : nr;
  const int gx = xd ? gi0 + li : gj0 + lj;  // index across
  const int nx = xd ? nr : nc;
  if (!IN && (gx < 0 || gx >= nx || gf < 0 || gf > na)) return;
  const int mi = xd ? li : li - 1, mj = xd ? lj - 1 : lj;  // minus (left/top) cell
  const int pi = li, pj = lj;                               // plus (right/bottom) cell
  T m, nmn, npl, tg;
  if (!IN && (gf == 0 || gf == na)) {
    const bool lo_side = gf == 0;
    const int ci = lo_side ? pi : mi, cj = lo_side ? pj : mj;
    const int64_t g0 = (int64_t)(gi0 + ci) * nc + (gj0 + cj);
    const T h = S.h[i4(ci, cj)];
    const T hu = Field<T>::ld(A.in_hu, A.tan.in_hu, g0);
    const T hv = Field<T>::ld(A.in_hv, A.tan.in_hv, g0);
    int side;
    int64_t g1;
    double dn;
    if (xd) {
      side = lo_side ? SIDE_WEST : SIDE_EAST;
      g1 = lo_side ? g0 + 1 : g0 - 1;
      dn = A.dx;
    } else {
      side = lo_side ? SIDE_NORTH : SIDE_SOUTH;
      g1 = lo_side ? g0 + nc : g0 - nc;
      dn = A.dy;
    }
    const GhostT<T> G = ghost_cell<T>(side, A.bc, h, hu, hv, A.z, A.n, A.tan.n, g0, g1, dn);
    const double zc = S.z[i3(ci, cj)];
    const double zf = lo_side ? (G.z + zc) * 0.5 : (zc + G.z) * 0.5;
    const T qn = xd ? hu : hv, qt = xd ? hv : hu;
    const T gqn = xd ? G.hu : G.hv, gqt = xd ? G.hv : G.hu;
    if (lo_side)
      wb_face<T>(G.h, gqn, gqt, h, qn, qt, zf, m, nmn, npl, tg);
    else
      wb_face<T>(h, qn, qt, G.h, gqn, gqt, zf, m, nmn, npl, tg);
  } else {
    const T hm = S.h[i4(mi, mj)], hp = S.h[i4(pi, pj)];
    const bool dm = val(hm) <= H_DRY, dp = val(hp) <= H_DRY;
    if (dm && dp) {
      m = Z; nmn = Z; npl = Z; tg = Z;
    } else {
      const int m3 = i3(mi, mj), p3 = i3(pi, pj);
      const double zm = S.z[m3], zp = S.z[p3];
      const double zf = (dm != dp) ? fmax(zm, zp) : (zm + zp) * 0.5;  // update.rs:650-656
      const double half = xd ? 0.5 * A.dx : 0.5 * A.dy;
      T se_m, sn_m, st_m, se_p, sn_p, st_p;
      if (xd) {
        const int a = isx(mi, mj), b = isx(pi, pj);
        se_m = S.sxe[a]; sn_m = S.sxu[a]; st_m = S.sxv[a];
        se_p = S.sxe[b]; sn_p = S.sxu[b]; st_p = S.sxv[b];
      } else {
        const int a = isy(mi, mj), b = isy(pi, pj);
        se_m = S.sye[a]; sn_m = S.syv[a]; st_m = S.syu[a];
        se_p = S.sye[b]; sn_p = S.syv[b]; st_p = S.syu[b];
      }
      const T un_mc = xd ? S.u[m3] : S.v[m3], ut_mc = xd ? S.v[m3] : S.u[m3];
      const T un_pc = xd ? S.u[p3] : S.v[p3], ut_pc = xd ? S.v[p3] : S.u[p3];
      // reconstruct_x/y_face_states (update.rs:560-623)
      const T eta_m = S.eta[m3] + se_m * half;
      const T un_m = un_mc + sn_m * half;
      const T ut_m = ut_mc + st_m * half;
      const T eta_p = S.eta[p3] - se_p * half;
      const T un_p = un_pc - sn_p * half;
      const T ut_p = ut_pc - st_p * half;
      const T h_m = r_max(eta_m - zf, Z);
      const T h_p = r_max(eta_p - zf, Z);
      wb_face<T>(h_m, h_m * un_m, h_m * ut_m, h_p, h_p * un_p, h_p * ut_p, zf, m, nmn, npl, tg);
    }
  }
  if (xd) {
    const int k = ifx(li, lj);
    S.fxm[k] = m; S.fxnm[k] = nmn; S.fxnp[k] = npl; S.fxt[k] = tg;
  } else {
    const int k = ify(li, lj);
    S.fym[k] = m; S.fynm[k] = nmn; S.fynp[k] = npl; S.fyt[k] = tg;
  }
}

// Alpha mass rescaling factor of cell (li, lj): update.rs:953-982.
template <class T, bool IN, class SM>
__device__ __forceinline__ void alpha_at(const StageArgs& A, SM& S, int gi0, int gj0, int li,
                                         int lj, double dt_dx, double dt_dy) {
  const int gi = gi0 + li, gj = gj0 + lj;
  if (!IN && (gi < 0 || gi >= A.nr || gj < 0 || gj >= A.nc)) return;
  const T Z = cst<T>(0.0);
  const T fr = S.fxm[ifx(li, lj + 1)], fl = S.fxm[ifx(li, lj)];
  const T fb = S.fym[ify(li + 1, lj)], ft = S.fym[ify(li, lj)];
  T out = Z;
  if (val(fr) > 0.0) out = out + fr * dt_dx;
  if (val(fl) < 0.0) out = out + (-fl) * dt_dx;
  if (val(fb) > 0.0) out = out + fb * dt_dy;
  if (val(ft) < 0.0) out = out + (-ft) * dt_dy;
  const T avail = r_max(S.h[i4(li, lj)] - H_DRY, Z);
  S.a[ia(li, lj)] = (val(out) > val(avail) && val(out) > 0.0) ? dvp(avail, out) : cst<T>(1.0);
}

// Face beds of a tile cell's four faces (update.rs:676-728, 650-656).
template <bool IN = false>
__device__ __forceinline__ void cell_face_beds(const StageArgs& A, const double* Sz, bool dc,
                                               bool dl, bool dr, bool dt_, bool db, int c3,
                                               int gi, int gj, double& zfl, double& zfr,
                                               double& zft, double& zfb) {
  const double zc = Sz[c3];
  if (!IN && gj == 0)
    zfl = (ghost_bed(A.bc.kind[SIDE_WEST], zc, Sz[c3 + 1]) + zc) * 0.5;
  else
    zfl = (dl != dc) ? fmax(Sz[c3 - 1], zc) : (Sz[c3 - 1] + zc) * 0.5;
  if (!IN && gj + 1 == A.nc)
    zfr = (zc + ghost_bed(A.bc.kind[SIDE_EAST], zc, Sz[c3 - 1])) * 0.5;
  else
    zfr = (dc != dr) ? fmax(zc, Sz[c3 + 1]) : (zc + Sz[c3 + 1]) * 0.5;
  if (!IN && gi == 0)
    zft = (ghost_bed(A.bc.kind[SIDE_NORTH], zc, Sz[c3 + R3W]) + zc) * 0.5;
  else
    zft = (dt_ != dc) ? fmax(Sz[c3 - R3W], zc) : (Sz[c3 - R3W] + zc) * 0.5;
  if (!IN && gi + 1 == A.nr)
    zfb = (zc + ghost_bed(A.bc.kind[SIDE_SOUTH], zc, Sz[c3 - R3W])) * 0.5;
  else
    zfb = (dc != db) ? fmax(zc, Sz[c3 + R3W]) : (zc + Sz[c3 + R3W]) * 0.5;
}

// FV update + bed source + floor of cell (li, lj) (update.rs:1071-1210),
// then the SSP-RK2 combination (update.rs:1271-1286) and, in the last
// stage, friction, forcings and the CFL contribution; writes the cell.
// Sources of the cell's tile or block are order[src_lo, src_hi).
template <class T, bool IN, class SM>
__device__ __forceinline__ void update_at(const StageArgs& A, SM& S, int gi0, int gj0, int li,
                                          int lj, double dt, double dt_dx, double dt_dy,
                                          const int* order, int src_lo, int src_hi, double& sxm,
                                          double& sym, unsigned long long& nonfin) {
  const int nr = A.nr, nc = A.nc;
  const double dx = A.dx, dy = A.dy;
  const T Z = cst<T>(0.0);
  const int gi = gi0 + li, gj = gj0 + lj;
  if (!IN && (gi >= nr || gj >= nc)) return;
  const int64_t g = (int64_t)gi * nc + gj;
  const int c4 = i4(li, lj), c3 = i3(li, lj);
  const T hc = S.h[c4];
  const bool dc = val(hc) <= H_DRY;
  T nh, nhu, nhv;
  if (dc && (IN || (gi > 0 && gi + 1 < nr && gj > 0 && gj + 1 < nc)) && val(S.h[c4 - R4W]) <= H_DRY &&
      val(S.h[c4 + R4W]) <= H_DRY && val(S.h[c4 - 1]) <= H_DRY && val(S.h[c4 + 1]) <= H_DRY) {
    nh = hc;  // isolated-dry fast path (update.rs:1072-1088)
    nhu = Z;
    nhv = Z;
  } else {
    const int fr = ifx(li, lj + 1), fl = ifx(li, lj), fb = ify(li + 1, lj), ft = ify(li, lj);
    const T mr = S.fxm[fr], ml = S.fxm[fl], mb = S.fym[fb], mt = S.fym[ft];
    const T ac = S.a[ia(li, lj)];
    const T one = cst<T>(1.0);
    // Upstream alpha per face (update.rs:992-1053). Dry-dry interior faces
    // are exact zeros; scaling them by an alpha in [0, 1] keeps them +0.
    const T ar = (!IN && gj + 1 == nc) ? (val(mr) > 0.0 ? ac : one) : (val(mr) > 0.0 ? ac : S.a[ia(li, lj + 1)]);
    const T al = (!IN && gj == 0) ? (val(ml) < 0.0 ? ac : one) : (val(ml) > 0.0 ? S.a[ia(li, lj - 1)] : ac);
    const T ab = (!IN && gi + 1 == nr) ? (val(mb) > 0.0 ? ac : one) : (val(mb) > 0.0 ? ac : S.a[ia(li + 1, lj)]);
    const T at = (!IN && gi == 0) ? (val(mt) < 0.0 ? ac : one) : (val(mt) > 0.0 ? S.a[ia(li - 1, lj)] : ac);
    const T fxr_m = mr * ar, fxr_n = S.fxnm[fr] * ar, fxr_t = S.fxt[fr] * ar;
    const T fxl_m = ml * al, fxl_n = S.fxnp[fl] * al, fxl_t = S.fxt[fl] * al;
    const T fyb_m = mb * ab, fyb_n = S.fynm[fb] * ab, fyb_t = S.fyt[fb] * ab;
    const T fyt_m = mt * at, fyt_n = S.fynp[ft] * at, fyt_t = S.fyt[ft] * at;
    const T dh = (fxr_m - fxl_m) * dt_dx + (fyb_m - fyt_m) * dt_dy;
    const T new_h = hc - dh;
    const T dhu = (fxr_n - fxl_n) * dt_dx + (fyb_t - fyt_t) * dt_dy;
    const T dhv = (fxr_t - fxl_t) * dt_dx + (fyb_n - fyt_n) * dt_dy;

    double zfl, zfr, zft, zfb;
    cell_face_beds<IN>(A, S.z, dc, val(S.h[c4 - 1]) <= H_DRY, val(S.h[c4 + 1]) <= H_DRY,
                       val(S.h[c4 - R4W]) <= H_DRY, val(S.h[c4 + R4W]) <= H_DRY, c3, gi, gj, zfl,
                       zfr, zft, zfb);

    // Explicit bed-slope source on the reconstructed face states (update.rs:1140-1180).
    const double zc = S.z[c3];
    const T eta_cell = hc + zc;
    const T sex = S.sxe[isx(li, lj)];
    const T eta_left = (IN || gj > 0) ? eta_cell - sex * (0.5 * dx) : eta_cell;
    const T eta_right = (IN || gj + 1 < nc) ? eta_cell + sex * (0.5 * dx) : eta_cell;
    const T hfl = r_max(eta_left - zfl, Z);
    const T hfr = r_max(eta_right - zfr, Z);
    const T s_hu = dvr((hfl + hfr) * ((eta_left - hfl) - (eta_right - hfr)) * (0.5 * GRAVITY), A.rx);
    const T sey = S.sye[isy(li, lj)];
    const T eta_top = (IN || gi > 0) ? eta_cell - sey * (0.5 * dy) : eta_cell;
    const T eta_bot = (IN || gi + 1 < nr) ? eta_cell + sey * (0.5 * dy) : eta_cell;
    const T hft = r_max(eta_top - zft, Z);
    const T hfb = r_max(eta_bot - zfb, Z);
    const T s_hv = dvr((hft + hfb) * ((eta_top - hft) - (eta_bot - hfb)) * (0.5 * GRAVITY), A.ry);

    if (val(new_h) <= H_VEL) {
      nh = r_max(new_h, Z);  // moisture floor keeps the mass
      nhu = Z;
      nhv = Z;
    } else {
      T hu_old = Z, hv_old = Z;
      if (val(hc) > H_VEL) {
        hu_old = Field<T>::ld(A.in_hu, A.tan.in_hu, g);
        hv_old = Field<T>::ld(A.in_hv, A.tan.in_hv, g);
      }
      nh = new_h;
      nhu = hu_old - dhu + s_hu * dt;
      nhv = hv_old - dhv + s_hv * dt;
    }
  }
  if (A.combine) {  // SSP-RK2 convex combination + floor (update.rs:1271-1286)
    const T ph = Field<T>::ld(A.un_h, A.tan.un_h, g);
    const T phu = Field<T>::ld(A.un_hu, A.tan.un_hu, g);
    const T phv = Field<T>::ld(A.un_hv, A.tan.un_hv, g);
    nh = (ph + nh) * 0.5;
    nhu = (phu + nhu) * 0.5;
    nhv = (phv + nhv) * 0.5;
    if (val(nh) <= H_VEL) {
      nh = r_max(nh, Z);
      nhu = Z;
      nhv = Z;
    }
  }
  if (A.finalize) {
    finalize_cell<T>(A, A.ctrl, dt, gi, gj, g, order, src_lo, src_hi, nh, nhu, nhv);
    cfl_cell<IN>(A, gi, gj, g, val(nh), val(nhu), val(nhv), sxm, sym);
    if (A.ctrl->check_finite && !isfinite(val(nh))) ++nonfin;
  }
  Field<T>::st(A.out_h, A.tan.out_h, g, nh);
  Field<T>::st(A.out_hu, A.tan.out_hu, g, nhu);
  Field<T>::st(A.out_hv, A.tan.out_hv, g, nhv);
}

// Phases 1-4 of one forward-Euler stage (update.rs:805-1053) on one tile:
// depth snapshot, primitives, limited slopes, face fluxes and the alpha
// rescaling factors of the tile and its one-cell ring, all in shared memory.
// Called by every thread of the CTA; ends with a barrier.
// With PF (f64 only) the tile's raw inputs are already in shared memory
// (stage_prefetch into hst, S.eta, S.u, S.v, completed by the caller), and
// once the faces are done the copies of tile `next` (if >= 0) are started,
// overlapping the alpha and update phases of this tile. `next` is a tile of
// the grid described by *next_args (another scenario's, in an ensemble), or
// of A when next_args is null.
// DRY (forward stages of interior tiles only): when every depth of the tile
// and its halo is at or below H_DRY, every cell of the tile takes the
// isolated-dry update (update.rs:1072-1088), which reads no slope, face or
// alpha: those phases are skipped and the function returns true. The vote
// rides on the barrier that ends the primitives phase.
template <class T, bool PF = false, bool IN = false, bool DRY = false>
__device__ __forceinline__ bool stage_tile_faces(const StageArgs& A, StageSmemT<T>& S, int gi0,
                                                 int gj0, double dt, double* hst = nullptr,
                                                 int next = -1,
                                                 const StageArgs* next_args = nullptr) {
  constexpr bool SKIP = DRY && IN;
  bool dry = true;
  const int nr = A.nr, nc = A.nc;
  const double dx = A.dx, dy = A.dy;
  const double dt_dx = dt / dx;  // update.rs:930-931
  const double dt_dy = dt / dy;
  const double half_dx = 0.5 * dx, half_dy = 0.5 * dy;
  const int tid = threadIdx.x;
  const T Z = cst<T>(0.0);
  if constexpr (PF) {
    // ---- depth snapshot and primitives from the staged inputs. Cells outside
    // the grid were zero-filled, so they get h = z = eta = u = v = +0 as below.
    for (int k = tid; k < R4N; k += NTHREADS) {
      const int r = k / R4W, cc = k - r * R4W;
      const double hh = hst[k];
      S.h[k] = hh;
      if constexpr (SKIP) dry &= hh <= H_DRY;
      if (r >= 1 && r < R4H - 1 && cc >= 1 && cc < R4W - 1) {
        const int k3 = (r - 1) * R3W + (cc - 1);
        const double zz = S.eta[k3], qu = S.u[k3], qv = S.v[k3];
        double uu = 0.0, vv = 0.0;
        if (hh > H_VEL) dvp2(qu, qv, hh, uu, vv);
        S.z[k3] = zz;
        S.eta[k3] = hh + zz;
        S.u[k3] = uu;
        S.v[k3] = vv;
      }
    }
    if constexpr (SKIP) {
      if (__syncthreads_and(dry)) {
        if (next >= 0) stage_prefetch(next_args ? *next_args : A, S, hst, next);
        return true;
      }
    } else {
      __syncthreads();
    }
  } else {
    // ---- depth snapshot (halo 4) and primitives (halo 3): update.rs:853-858, 405-426
    for (int k = tid; k < R4N; k += NTHREADS) {
      const int r = k / R4W, cc = k - r * R4W;
      const int gi = gi0 + r - 4, gj = gj0 + cc - 4;
      const bool real = IN || (gi >= 0 && gi < nr && gj >= 0 && gj < nc);
      const int64_t g = (int64_t)gi * nc + gj;
      const T hh = real ? Field<T>::ld(A.in_h, A.tan.in_h, g) : Z;
      S.h[k] = hh;
      if (r >= 1 && r < R4H - 1 && cc >= 1 && cc < R4W - 1) {
        const int k3 = (r - 1) * R3W + (cc - 1);
        double zz = 0.0;
        T e = Z, uu = Z, vv = Z;
        if (real) {
          zz = A.z[g];
          e = hh + zz;
          if (val(hh) > H_VEL) {
            uu = dvp(Field<T>::ld(A.in_hu, A.tan.in_hu, g), hh);  // hh > H_VEL
            vv = dvp(Field<T>::ld(A.in_hv, A.tan.in_hv, g), hh);
          }
        }
        S.z[k3] = zz;
        S.eta[k3] = e;
        S.u[k3] = uu;
        S.v[k3] = vv;
      }
      if constexpr (SKIP) dry &= val(hh) <= H_DRY;
    }
    if constexpr (SKIP) {
      if (__syncthreads_and(dry)) return true;
    } else {
      __syncthreads();
    }
  }
  {
    // ---- limited slopes: update.rs:459-540 (item k < SXN: x slope, else y)
    auto slope_item = [&](int k) {
      const bool xd = k < SXN;
      int li, lj;
      if (xd) {
        const int r = k / SXW;
        li = r - 1;
        lj = k - r * SXW - 2;
      } else {
        const int kk = k - SXN, r = kk / SYW;
        li = r - 2;
        lj = kk - r * SYW - 1;
      }
      const int gi = gi0 + li, gj = gj0 + lj;
      if (!IN && (gi < 0 || gi >= nr || gj < 0 || gj >= nc)) return;
      const int ga = xd ? gj : gi;
      const int na = xd ? nc : nr;
      const int st4 = xd ? 1 : R4W;
      const int st3 = xd ? 1 : R3W;
      const hfa::RecipD& rd = xd ? A.rx : A.ry;
      T se = Z, su = Z, sv = Z;
      if (IN || na >= 2) {
        const int lo = IN ? -2 : max(ga - 2, 0) - ga, hi = IN ? 2 : min(ga + 2, na - 1) - ga;
        const int c4 = i4(li, lj);
        bool anyd = false;
        for (int o = lo; o <= hi; ++o) anyd |= val(S.h[c4 + o * st4]) <= H_DRY;
        if (!anyd) {
          const int c3 = i3(li, lj);
          if (!IN && ga == 0) {
            const int r3 = c3 + st3;
            se = dvr(S.eta[r3] - S.eta[c3], rd);  // / dx or / dy
            su = dvr(S.u[r3] - S.u[c3], rd);
            sv = dvr(S.v[r3] - S.v[c3], rd);
          } else if (!IN && ga == na - 1) {
            const int l3 = c3 - st3;
            se = dvr(S.eta[c3] - S.eta[l3], rd);
            su = dvr(S.u[c3] - S.u[l3], rd);
            sv = dvr(S.v[c3] - S.v[l3], rd);
          } else {
            const int l3 = c3 - st3, r3 = c3 + st3;
            se = minmod_div<T>(S.eta[c3] - S.eta[l3], S.eta[r3] - S.eta[c3], rd);
            su = minmod_div<T>(S.u[c3] - S.u[l3], S.u[r3] - S.u[c3], rd);
            sv = minmod_div<T>(S.v[c3] - S.v[l3], S.v[r3] - S.v[c3], rd);
          }
        }
      }
      if (xd) {
        S.sxe[k] = se;
        S.sxu[k] = su;
        S.sxv[k] = sv;
      } else {
        S.sye[k - SXN] = se;
        S.syu[k - SXN] = su;
        S.syv[k - SXN] = sv;
      }
    };

    // ---- faces: update.rs:676-728 (face beds), 890-926 (fluxes) (item k < FXN: x face)
    auto face_item = [&](int k) {
      const bool xd = k < FXN;
      int li, lj;  // x face: (row li, face lj); y face: (face li, column lj)
      if (xd) {
        const int r = k / FXW;
        li = r - 1;
        lj = k - r * FXW - 1;
      } else {
        const int kk = k - FXN, r = kk / FYW;
        li = r - 1;
        lj = kk - r * FYW - 1;
      }
      const int gf = xd ? gj0 + lj : gi0 + li;  // face index along the normal
      const int na = xd ? nc : nr;
      const int gx = xd ? gi0 + li : gj0 + lj;  // index across
      const int nx = xd ? nr : nc;
      if (!IN && (gx < 0 || gx >= nx || gf < 0 || gf > na)) return;
      const int mi = xd ? li : li - 1, mj = xd ? lj - 1 : lj;  // minus (left/top) cell
      const int pi = li, pj = lj;                               // plus (right/bottom) cell
      T m, nmn, npl, tg;
      if (!IN && (gf == 0 || gf == na)) {
        const bool lo_side = gf == 0;
        const int ci = lo_side ? pi : mi, cj = lo_side ? pj : mj;
        const int64_t g0 = (int64_t)(gi0 + ci) * nc + (gj0 + cj);
        const T h = S.h[i4(ci, cj)];
        const T hu = Field<T>::ld(A.in_hu, A.tan.in_hu, g0);
        const T hv = Field<T>::ld(A.in_hv, A.tan.in_hv, g0);
        int side;
        int64_t g1;
        double dn;
        if (xd) {
          side = lo_side ? SIDE_WEST : SIDE_EAST;
          g1 = lo_side ? g0 + 1 : g0 - 1;
          dn = dx;
        } else {
          side = lo_side ? SIDE_NORTH : SIDE_SOUTH;
          g1 = lo_side ? g0 + nc : g0 - nc;
          dn = dy;
        }
        const GhostT<T> G = ghost_cell<T>(side, A.bc, h, hu, hv, A.z, A.n, A.tan.n, g0, g1, dn);
        const double zc = S.z[i3(ci, cj)];
        const double zf = lo_side ? (G.z + zc) * 0.5 : (zc + G.z) * 0.5;
        const T qn = xd ? hu : hv, qt = xd ? hv : hu;
        const T gqn = xd ? G.hu : G.hv, gqt = xd ? G.hv : G.hu;
        if (lo_side)
          wb_face<T>(G.h, gqn, gqt, h, qn, qt, zf, m, nmn, npl, tg);
        else
          wb_face<T>(h, qn, qt, G.h, gqn, gqt, zf, m, nmn, npl, tg);
      } else {
        const T hm = S.h[i4(mi, mj)], hp = S.h[i4(pi, pj)];
        const bool dm = val(hm) <= H_DRY, dp = val(hp) <= H_DRY;
        if (dm && dp) {
          m = Z; nmn = Z; npl = Z; tg = Z;
        } else {
          const int m3 = i3(mi, mj), p3 = i3(pi, pj);
          const double zm = S.z[m3], zp = S.z[p3];
          const double zf = (dm != dp) ? fmax(zm, zp) : (zm + zp) * 0.5;  // update.rs:650-656
          const double half = xd ? half_dx : half_dy;
          T se_m, sn_m, st_m, se_p, sn_p, st_p;
          if (xd) {
            const int a = isx(mi, mj), b = isx(pi, pj);
            se_m = S.sxe[a]; sn_m = S.sxu[a]; st_m = S.sxv[a];
            se_p = S.sxe[b]; sn_p = S.sxu[b]; st_p = S.sxv[b];
          } else {
            const int a = isy(mi, mj), b = isy(pi, pj);
            se_m = S.sye[a]; sn_m = S.syv[a]; st_m = S.syu[a];
            se_p = S.sye[b]; sn_p = S.syv[b]; st_p = S.syu[b];
          }
          const T un_mc = xd ? S.u[m3] : S.v[m3], ut_mc = xd ? S.v[m3] : S.u[m3];
          const T un_pc = xd ? S.u[p3] : S.v[p3], ut_pc = xd ? S.v[p3] : S.u[p3];
          // reconstruct_x/y_face_states (update.rs:560-623)
          const T eta_m = S.eta[m3] + se_m * half;
          const T un_m = un_mc + sn_m * half;
          const T ut_m = ut_mc + st_m * half;
          const T eta_p = S.eta[p3] - se_p * half;
          const T un_p = un_pc - sn_p * half;
          const T ut_p = ut_pc - st_p * half;
          const T h_m = r_max(eta_m - zf, Z);
          const T h_p = r_max(eta_p - zf, Z);
          wb_face<T>(h_m, h_m * un_m, h_m * ut_m, h_p, h_p * un_p, h_p * ut_p, zf, m, nmn, npl, tg);
        }
      }
      if (xd) {
        S.fxm[k] = m; S.fxnm[k] = nmn; S.fxnp[k] = npl; S.fxt[k] = tg;
      } else {
        const int kk = k - FXN;
        S.fym[kk] = m; S.fynm[kk] = nmn; S.fynp[kk] = npl; S.fyt[kk] = tg;
      }
    };

    if constexpr (!SplitFaces<T>::value) {
      for (int k = tid; k < SXN + SYN; k += NTHREADS) slope_item(k);
      __syncthreads();
      for (int k = tid; k < FXN + FYN; k += NTHREADS) face_item(k);
      __syncthreads();
    } else {  // slopes, x faces, then y faces (over the x momentum slopes)
      for (int k = tid; k < SXN + SYN; k += NTHREADS) slope_item(k);
      __syncthreads();
      for (int k = tid; k < FXN; k += NTHREADS) face_item(k);
      __syncthreads();
      for (int k = FXN + tid; k < FXN + FYN; k += NTHREADS) face_item(k);
      __syncthreads();
    }
    if constexpr (PF) {
      if (next >= 0)  // eta, u, v and hst are dead now
        stage_prefetch(next_args ? *next_args : A, S, hst, next);
    }

    // ---- alpha mass rescaling factors: update.rs:953-982 (tile + 1-cell ring)
    for (int k = tid; k < AN; k += NTHREADS) {
      const int r = k / AW;
      const int li = r - 1, lj = k - r * AW - 1;
      if ((li < 0 || li >= TY) && (lj < 0 || lj >= TX)) continue;
      const int gi = gi0 + li, gj = gj0 + lj;
      if (!IN && (gi < 0 || gi >= nr || gj < 0 || gj >= nc)) continue;
      const T fr = S.fxm[ifx(li, lj + 1)], fl = S.fxm[ifx(li, lj)];
      const T fb = S.fym[ify(li + 1, lj)], ft = S.fym[ify(li, lj)];
      T out = Z;
      if (val(fr) > 0.0) out = out + fr * dt_dx;
      if (val(fl) < 0.0) out = out + (-fl) * dt_dx;
      if (val(fb) > 0.0) out = out + fb * dt_dy;
      if (val(ft) < 0.0) out = out + (-ft) * dt_dy;
      const T avail = r_max(S.h[i4(li, lj)] - H_DRY, Z);
      S.a[k] = (val(out) > val(avail) && val(out) > 0.0) ? dvp(avail, out) : cst<T>(1.0);
    }
    __syncthreads();
  }
  return false;
}

// One forward-Euler stage (update.rs:805-1211) on one tile of one grid. Called
// by every thread of the CTA; accumulates the CTA's CFL maxima for the
// finalize epilogue into (sxm, sym, nonfin).
// IN: the tile and its 4-cell halo lie inside the grid (no side is reached),
// so the boundary branches compile away; the arithmetic is the same.
template <class T, bool PF = false, bool IN = false>
__device__ __forceinline__ void stage_tile(const StageArgs& A, StageSmemT<T>& S, int tile,
                                           double& sxm, double& sym, unsigned long long& nonfin,
                                           double* hst = nullptr, int next = -1,
                                           const StageArgs* next_args = nullptr) {
  Ctrl* ctrl = A.ctrl;
  const double dt = ctrl->dt;
  const int nr = A.nr, nc = A.nc;
  const double dx = A.dx, dy = A.dy;
  const double dt_dx = dt / dx;  // update.rs:930-931
  const double dt_dy = dt / dy;
  const int tid = threadIdx.x;
  const T Z = cst<T>(0.0);
  {
    const int tyi = tile / A.tiles_x;
    const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;
    // Dry interior tiles skip their slopes, faces and alpha (f64 forward stage).
  stage_tile_faces<T, PF, IN, std::is_same<T, double>::value>(A, S, gi0, gj0, dt, hst, next,
                                                                 next_args);

    // ---- FV update + bed source + floor: update.rs:1071-1210
    int src_lo = 0, src_hi = 0;
    if (A.finalize && A.f.n_src > 0) {
      src_lo = A.f.tile_start[tile];
      src_hi = A.f.tile_start[tile + 1];
    }
#pragma unroll 1
    for (int q = 0; q < CELLS_PER_THREAD; ++q) {
      const int li = tid / TX + ROWS_PER_PASS * q, lj = tid % TX;
      if (kPartialPass && li >= TY) continue;
      const int gi = gi0 + li, gj = gj0 + lj;
      if (!IN && (gi >= nr || gj >= nc)) continue;
      const int64_t g = (int64_t)gi * nc + gj;
      const int c4 = i4(li, lj), c3 = i3(li, lj);
      const T hc = S.h[c4];
      const bool dc = val(hc) <= H_DRY;
      T nh, nhu, nhv;
      if (dc && (IN || (gi > 0 && gi + 1 < nr && gj > 0 && gj + 1 < nc)) && val(S.h[c4 - R4W]) <= H_DRY &&
          val(S.h[c4 + R4W]) <= H_DRY && val(S.h[c4 - 1]) <= H_DRY && val(S.h[c4 + 1]) <= H_DRY) {
        nh = hc;  // isolated-dry fast path (update.rs:1072-1088)
        nhu = Z;
        nhv = Z;
      } else {
        const int fr = ifx(li, lj + 1), fl = ifx(li, lj), fb = ify(li + 1, lj), ft = ify(li, lj);
        const T mr = S.fxm[fr], ml = S.fxm[fl], mb = S.fym[fb], mt = S.fym[ft];
        const T ac = S.a[ia(li, lj)];
        const T one = cst<T>(1.0);
        // Upstream alpha per face (update.rs:992-1053). Dry-dry interior faces
        // are exact zeros; scaling them by an alpha in [0, 1] keeps them +0.
        const T ar = (!IN && gj + 1 == nc) ? (val(mr) > 0.0 ? ac : one) : (val(mr) > 0.0 ? ac : S.a[ia(li, lj + 1)]);
        const T al = (!IN && gj == 0) ? (val(ml) < 0.0 ? ac : one) : (val(ml) > 0.0 ? S.a[ia(li, lj - 1)] : ac);
        const T ab = (!IN && gi + 1 == nr) ? (val(mb) > 0.0 ? ac : one) : (val(mb) > 0.0 ? ac : S.a[ia(li + 1, lj)]);
        const T at = (!IN && gi == 0) ? (val(mt) < 0.0 ? ac : one) : (val(mt) > 0.0 ? S.a[ia(li - 1, lj)] : ac);
        const T fxr_m = mr * ar, fxr_n = S.fxnm[fr] * ar, fxr_t = S.fxt[fr] * ar;
        const T fxl_m = ml * al, fxl_n = S.fxnp[fl] * al, fxl_t = S.fxt[fl] * al;
        const T fyb_m = mb * ab, fyb_n = S.fynm[fb] * ab, fyb_t = S.fyt[fb] * ab;
        const T fyt_m = mt * at, fyt_n = S.fynp[ft] * at, fyt_t = S.fyt[ft] * at;
        const T dh = (fxr_m - fxl_m) * dt_dx + (fyb_m - fyt_m) * dt_dy;
        const T new_h = hc - dh;
        const T dhu = (fxr_n - fxl_n) * dt_dx + (fyb_t - fyt_t) * dt_dy;
        const T dhv = (fxr_t - fxl_t) * dt_dx + (fyb_n - fyt_n) * dt_dy;

        double zfl, zfr, zft, zfb;
        cell_face_beds<IN>(A, S.z, dc, val(S.h[c4 - 1]) <= H_DRY, val(S.h[c4 + 1]) <= H_DRY,
                       val(S.h[c4 - R4W]) <= H_DRY, val(S.h[c4 + R4W]) <= H_DRY, c3, gi, gj, zfl,
                       zfr, zft, zfb);

        // Explicit bed-slope source on the reconstructed face states (update.rs:1140-1180).
        const double zc = S.z[c3];
        const T eta_cell = hc + zc;
        const T sex = S.sxe[isx(li, lj)];
        const T eta_left = (IN || gj > 0) ? eta_cell - sex * (0.5 * dx) : eta_cell;
        const T eta_right = (IN || gj + 1 < nc) ? eta_cell + sex * (0.5 * dx) : eta_cell;
        const T hfl = r_max(eta_left - zfl, Z);
        const T hfr = r_max(eta_right - zfr, Z);
        const T s_hu = dvr((hfl + hfr) * ((eta_left - hfl) - (eta_right - hfr)) * (0.5 * GRAVITY), A.rx);
        const T sey = S.sye[isy(li, lj)];
        const T eta_top = (IN || gi > 0) ? eta_cell - sey * (0.5 * dy) : eta_cell;
        const T eta_bot = (IN || gi + 1 < nr) ? eta_cell + sey * (0.5 * dy) : eta_cell;
        const T hft = r_max(eta_top - zft, Z);
        const T hfb = r_max(eta_bot - zfb, Z);
        const T s_hv = dvr((hft + hfb) * ((eta_top - hft) - (eta_bot - hfb)) * (0.5 * GRAVITY), A.ry);

        if (val(new_h) <= H_VEL) {
          nh = r_max(new_h, Z);  // moisture floor keeps the mass
          nhu = Z;
          nhv = Z;
        } else {
          T hu_old = Z, hv_old = Z;
          if (val(hc) > H_VEL) {
            hu_old = Field<T>::ld(A.in_hu, A.tan.in_hu, g);
            hv_old = Field<T>::ld(A.in_hv, A.tan.in_hv, g);
          }
          nh = new_h;
          nhu = hu_old - dhu + s_hu * dt;
          nhv = hv_old - dhv + s_hv * dt;
        }
      }
      if (A.combine) {  // SSP-RK2 convex combination + floor (update.rs:1271-1286)
        const T ph = Field<T>::ld(A.un_h, A.tan.un_h, g);
        const T phu = Field<T>::ld(A.un_hu, A.tan.un_hu, g);
        const T phv = Field<T>::ld(A.un_hv, A.tan.un_hv, g);
        nh = (ph + nh) * 0.5;
        nhu = (phu + nhu) * 0.5;
        nhv = (phv + nhv) * 0.5;
        if (val(nh) <= H_VEL) {
          nh = r_max(nh, Z);
          nhu = Z;
          nhv = Z;
        }
      }
      if (A.finalize) {
        finalize_cell<T>(A, ctrl, dt, gi, gj, g, A.f.tile_order, src_lo, src_hi, nh, nhu, nhv);
        cfl_cell<IN>(A, gi, gj, g, val(nh), val(nhu), val(nhv), sxm, sym);
        if (ctrl->check_finite && !isfinite(val(nh))) ++nonfin;
      }
      Field<T>::st(A.out_h, A.tan.out_h, g, nh);
      Field<T>::st(A.out_hu, A.tan.out_hu, g, nhu);
      Field<T>::st(A.out_hv, A.tan.out_hv, g, nhv);
    }
    __syncthreads();
  }
}

// A tile whose 4-cell halo lies inside the grid reaches no side: it runs the
// stage with the boundary branches compiled out (same arithmetic).
__device__ __forceinline__ bool interior_tile(const StageArgs& A, int tile) {
  const int tyi = tile / A.tiles_x;
  const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;
  return gi0 >= 4 && gj0 >= 4 && gi0 + TY + 4 <= A.nr && gj0 + TX + 4 <= A.nc;
}

}  // namespace HF_GEOM
}  // namespace hf
