// hf_kernels.cu -- sm_100a kernels of the solver-2d explicit step.
//
// The reference (franciscoparrao/hydroflux, solver-2d/src/update.rs:805-1211)
// runs one forward-Euler stage as eleven full-grid passes over a ~241 B/cell
// workspace. Here one stage is ONE kernel: a CTA stages a 32x16 tile plus a
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

#include <cstdio>

#include "hf_device.cuh"
#include "hf_internal.h"

namespace hf {

namespace {

// Shared-memory regions of the stage kernel, relative to the tile origin.
constexpr int R4W = TX + 8, R4H = TY + 8, R4N = R4W * R4H;  // h: rows/cols [-4, T+4)
constexpr int R3W = TX + 6, R3H = TY + 6, R3N = R3W * R3H;  // z, eta, u, v: [-3, T+3)
constexpr int SXW = TX + 4, SXH = TY + 2, SXN = SXW * SXH;  // x slopes: rows [-1,TY], cols [-2,TX+1]
constexpr int SYW = TX + 2, SYH = TY + 4, SYN = SYW * SYH;  // y slopes: rows [-2,TY+1], cols [-1,TX]
constexpr int FXW = TX + 3, FXH = TY + 2, FXN = FXW * FXH;  // x faces: rows [-1,TY], faces [-1,TX+1]
constexpr int FYW = TX + 2, FYH = TY + 3, FYN = FYW * FYH;  // y faces: faces [-1,TY+1], cols [-1,TX]
constexpr int AW = TX + 2, AH = TY + 2, AN = AW * AH;       // alpha: rows [-1,TY], cols [-1,TX]

struct StageSmem {
  double h[R4N];
  double z[R3N], eta[R3N], u[R3N], v[R3N];
  double sxe[SXN], sxu[SXN], sxv[SXN];
  double sye[SYN], syu[SYN], syv[SYN];
  double fxm[FXN], fxnm[FXN], fxnp[FXN], fxt[FXN];  // mass, normal(minus), normal(plus), tangential
  double fym[FYN], fynm[FYN], fynp[FYN], fyt[FYN];
  double a[AN];
};

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
__device__ __forceinline__ void finalize_cell(const StageArgs& A, const Ctrl* c, double dt,
                                              int gi, int gj, int64_t g, int src_lo, int src_hi,
                                              double& h, double& hu, double& hv) {
  friction_cell(h, hu, hv, A.n[g], dt, A.dry_tol);
  if (c->rain_on) {
    const double nh = h + c->rain_dh;
    if (nh <= 0.0) {
      h = 0.0; hu = 0.0; hv = 0.0;
    } else {
      h = nh;
    }
  }
  for (int s = src_lo; s < src_hi; ++s) {
    const int k = A.f.tile_order[s];
    if (A.f.src_row[k] == gi && A.f.src_col[k] == gj) {
      h = fmax(h + A.f.src_dh[k], 0.0);
      if (h == 0.0) {
        hu = 0.0;
        hv = 0.0;
      }
    }
  }
}

// CFL contribution of one cell of the final state, with the ghost cells of
// the sides it touches (cfl_time_step_with_bcs, update.rs:170-208).
__device__ __forceinline__ void cfl_cell(const StageArgs& A, int gi, int gj, int64_t g, double h,
                                         double hu, double hv, double& sx, double& sy) {
  cell_speeds(h, hu, hv, sx, sy);
  const int nr = A.nr, nc = A.nc;
  if (gj == 0) ghost_speeds(ghost_cell(SIDE_WEST, A.bc, h, hu, hv, A.z, A.n, g, g + 1, A.dx), sx, sy);
  if (gj == nc - 1)
    ghost_speeds(ghost_cell(SIDE_EAST, A.bc, h, hu, hv, A.z, A.n, g, g - 1, A.dx), sx, sy);
  if (gi == 0) ghost_speeds(ghost_cell(SIDE_NORTH, A.bc, h, hu, hv, A.z, A.n, g, g + nc, A.dy), sx, sy);
  if (gi == nr - 1)
    ghost_speeds(ghost_cell(SIDE_SOUTH, A.bc, h, hu, hv, A.z, A.n, g, g - nc, A.dy), sx, sy);
}

__device__ __forceinline__ void commit_clock(Ctrl* c) {
  c->t = c->t_new;
  c->steps += 1;
  if (c->mode == MODE_RUN) c->budget -= 1;
  c->cfl_valid = 1;
}

}  // namespace

// One forward-Euler stage (update.rs:805-1211) on one tile of one grid. Called
// by every thread of the CTA; accumulates the CTA's CFL maxima for the
// finalize epilogue into (sxm, sym, nonfin).
__device__ __forceinline__ void stage_tile(const StageArgs& A, StageSmem& S, int tile,
                                           double& sxm, double& sym, unsigned long long& nonfin) {
  Ctrl* ctrl = A.ctrl;
  const double dt = ctrl->dt;
  const int nr = A.nr, nc = A.nc;
  const double dx = A.dx, dy = A.dy;
  const double dt_dx = dt / dx;  // update.rs:930-931
  const double dt_dy = dt / dy;
  const double half_dx = 0.5 * dx, half_dy = 0.5 * dy;
  const int tid = threadIdx.x;
  {
    const int tyi = tile / A.tiles_x;
    const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;

    // ---- depth snapshot (halo 4) and primitives (halo 3): update.rs:853-858, 405-426
    for (int k = tid; k < R4N; k += NTHREADS) {
      const int r = k / R4W, cc = k - r * R4W;
      const int gi = gi0 + r - 4, gj = gj0 + cc - 4;
      const bool real = gi >= 0 && gi < nr && gj >= 0 && gj < nc;
      const int64_t g = (int64_t)gi * nc + gj;
      const double hh = real ? A.in_h[g] : 0.0;
      S.h[k] = hh;
      if (r >= 1 && r < R4H - 1 && cc >= 1 && cc < R4W - 1) {
        const int k3 = (r - 1) * R3W + (cc - 1);
        double zz = 0.0, e = 0.0, uu = 0.0, vv = 0.0;
        if (real) {
          zz = A.z[g];
          e = hh + zz;
          if (hh > H_VEL) {
            uu = hfa::div_rn(A.in_hu[g], hh);
            vv = hfa::div_rn(A.in_hv[g], hh);
          }
        }
        S.z[k3] = zz;
        S.eta[k3] = e;
        S.u[k3] = uu;
        S.v[k3] = vv;
      }
    }
    __syncthreads();

    // ---- limited slopes: update.rs:459-540
    for (int k = tid; k < SXN + SYN; k += NTHREADS) {
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
      if (gi < 0 || gi >= nr || gj < 0 || gj >= nc) continue;
      const int ga = xd ? gj : gi;
      const int na = xd ? nc : nr;
      const int st4 = xd ? 1 : R4W;
      const int st3 = xd ? 1 : R3W;
      const double d = xd ? dx : dy;
      double se = 0.0, su = 0.0, sv = 0.0;
      if (na >= 2) {
        const int lo = max(ga - 2, 0) - ga, hi = min(ga + 2, na - 1) - ga;
        const int c4 = i4(li, lj);
        bool anyd = false;
        for (int o = lo; o <= hi; ++o) anyd |= S.h[c4 + o * st4] <= H_DRY;
        if (!anyd) {
          const int c3 = i3(li, lj);
          if (ga == 0) {
            const int r3 = c3 + st3;
            se = hfa::div_rn(S.eta[r3] - S.eta[c3], d);
            su = hfa::div_rn(S.u[r3] - S.u[c3], d);
            sv = hfa::div_rn(S.v[r3] - S.v[c3], d);
          } else if (ga == na - 1) {
            const int l3 = c3 - st3;
            se = hfa::div_rn(S.eta[c3] - S.eta[l3], d);
            su = hfa::div_rn(S.u[c3] - S.u[l3], d);
            sv = hfa::div_rn(S.v[c3] - S.v[l3], d);
          } else {
            const int l3 = c3 - st3, r3 = c3 + st3;
            se = minmod_div(S.eta[c3] - S.eta[l3], S.eta[r3] - S.eta[c3], d);
            su = minmod_div(S.u[c3] - S.u[l3], S.u[r3] - S.u[c3], d);
            sv = minmod_div(S.v[c3] - S.v[l3], S.v[r3] - S.v[c3], d);
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
    }
    __syncthreads();

    // ---- faces: update.rs:676-728 (face beds), 890-926 (fluxes)
    for (int k = tid; k < FXN + FYN; k += NTHREADS) {
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
      if (gx < 0 || gx >= nx || gf < 0 || gf > na) continue;
      const int mi = xd ? li : li - 1, mj = xd ? lj - 1 : lj;  // minus (left/top) cell
      const int pi = li, pj = lj;                               // plus (right/bottom) cell
      double m, nmn, npl, tg;
      if (gf == 0 || gf == na) {
        const bool lo_side = gf == 0;
        const int ci = lo_side ? pi : mi, cj = lo_side ? pj : mj;
        const int64_t g0 = (int64_t)(gi0 + ci) * nc + (gj0 + cj);
        const double h = S.h[i4(ci, cj)];
        const double hu = A.in_hu[g0], hv = A.in_hv[g0];
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
        const Ghost G = ghost_cell(side, A.bc, h, hu, hv, A.z, A.n, g0, g1, dn);
        const double zc = S.z[i3(ci, cj)];
        const double zf = lo_side ? (G.z + zc) * 0.5 : (zc + G.z) * 0.5;
        const double qn = xd ? hu : hv, qt = xd ? hv : hu;
        const double gqn = xd ? G.hu : G.hv, gqt = xd ? G.hv : G.hu;
        if (lo_side)
          wb_face(G.h, gqn, gqt, h, qn, qt, zf, m, nmn, npl, tg);
        else
          wb_face(h, qn, qt, G.h, gqn, gqt, zf, m, nmn, npl, tg);
      } else {
        const double hm = S.h[i4(mi, mj)], hp = S.h[i4(pi, pj)];
        const bool dm = hm <= H_DRY, dp = hp <= H_DRY;
        if (dm && dp) {
          m = 0.0; nmn = 0.0; npl = 0.0; tg = 0.0;
        } else {
          const int m3 = i3(mi, mj), p3 = i3(pi, pj);
          const double zm = S.z[m3], zp = S.z[p3];
          const double zf = (dm != dp) ? fmax(zm, zp) : (zm + zp) * 0.5;  // update.rs:650-656
          const double half = xd ? half_dx : half_dy;
          double se_m, sn_m, st_m, se_p, sn_p, st_p;
          if (xd) {
            const int a = isx(mi, mj), b = isx(pi, pj);
            se_m = S.sxe[a]; sn_m = S.sxu[a]; st_m = S.sxv[a];
            se_p = S.sxe[b]; sn_p = S.sxu[b]; st_p = S.sxv[b];
          } else {
            const int a = isy(mi, mj), b = isy(pi, pj);
            se_m = S.sye[a]; sn_m = S.syv[a]; st_m = S.syu[a];
            se_p = S.sye[b]; sn_p = S.syv[b]; st_p = S.syu[b];
          }
          const double un_mc = xd ? S.u[m3] : S.v[m3], ut_mc = xd ? S.v[m3] : S.u[m3];
          const double un_pc = xd ? S.u[p3] : S.v[p3], ut_pc = xd ? S.v[p3] : S.u[p3];
          // reconstruct_x/y_face_states (update.rs:560-623)
          const double eta_m = S.eta[m3] + se_m * half;
          const double un_m = un_mc + sn_m * half;
          const double ut_m = ut_mc + st_m * half;
          const double eta_p = S.eta[p3] - se_p * half;
          const double un_p = un_pc - sn_p * half;
          const double ut_p = ut_pc - st_p * half;
          const double h_m = fmax(eta_m - zf, 0.0);
          const double h_p = fmax(eta_p - zf, 0.0);
          wb_face(h_m, h_m * un_m, h_m * ut_m, h_p, h_p * un_p, h_p * ut_p, zf, m, nmn, npl, tg);
        }
      }
      if (xd) {
        S.fxm[k] = m; S.fxnm[k] = nmn; S.fxnp[k] = npl; S.fxt[k] = tg;
      } else {
        const int kk = k - FXN;
        S.fym[kk] = m; S.fynm[kk] = nmn; S.fynp[kk] = npl; S.fyt[kk] = tg;
      }
    }
    __syncthreads();

    // ---- alpha mass rescaling factors: update.rs:953-982 (tile + 1-cell ring)
    for (int k = tid; k < AN; k += NTHREADS) {
      const int r = k / AW;
      const int li = r - 1, lj = k - r * AW - 1;
      if ((li < 0 || li >= TY) && (lj < 0 || lj >= TX)) continue;
      const int gi = gi0 + li, gj = gj0 + lj;
      if (gi < 0 || gi >= nr || gj < 0 || gj >= nc) continue;
      const double fr = S.fxm[ifx(li, lj + 1)], fl = S.fxm[ifx(li, lj)];
      const double fb = S.fym[ify(li + 1, lj)], ft = S.fym[ify(li, lj)];
      double out = 0.0;
      if (fr > 0.0) out = out + fr * dt_dx;
      if (fl < 0.0) out = out + (-fl) * dt_dx;
      if (fb > 0.0) out = out + fb * dt_dy;
      if (ft < 0.0) out = out + (-ft) * dt_dy;
      const double avail = fmax(S.h[i4(li, lj)] - H_DRY, 0.0);
      S.a[k] = (out > avail && out > 0.0) ? hfa::div_rn(avail, out) : 1.0;
    }
    __syncthreads();

    // ---- FV update + bed source + floor: update.rs:1071-1210
    int src_lo = 0, src_hi = 0;
    if (A.finalize && A.f.n_src > 0) {
      src_lo = A.f.tile_start[tile];
      src_hi = A.f.tile_start[tile + 1];
    }
#pragma unroll 1
    for (int q = 0; q < CELLS_PER_THREAD; ++q) {
      const int li = tid / TX + ROWS_PER_PASS * q, lj = tid % TX;
      const int gi = gi0 + li, gj = gj0 + lj;
      if (gi >= nr || gj >= nc) continue;
      const int64_t g = (int64_t)gi * nc + gj;
      const int c4 = i4(li, lj), c3 = i3(li, lj);
      const double hc = S.h[c4];
      const bool dc = hc <= H_DRY;
      double nh, nhu, nhv;
      if (dc && gi > 0 && gi + 1 < nr && gj > 0 && gj + 1 < nc && S.h[c4 - R4W] <= H_DRY &&
          S.h[c4 + R4W] <= H_DRY && S.h[c4 - 1] <= H_DRY && S.h[c4 + 1] <= H_DRY) {
        nh = hc;  // isolated-dry fast path (update.rs:1072-1088)
        nhu = 0.0;
        nhv = 0.0;
      } else {
        const int fr = ifx(li, lj + 1), fl = ifx(li, lj), fb = ify(li + 1, lj), ft = ify(li, lj);
        const double mr = S.fxm[fr], ml = S.fxm[fl], mb = S.fym[fb], mt = S.fym[ft];
        const double ac = S.a[ia(li, lj)];
        // Upstream alpha per face (update.rs:992-1053). Dry-dry interior faces
        // are exact zeros; scaling them by an alpha in [0, 1] keeps them +0.
        const double ar = (gj + 1 == nc) ? (mr > 0.0 ? ac : 1.0) : (mr > 0.0 ? ac : S.a[ia(li, lj + 1)]);
        const double al = (gj == 0) ? (ml < 0.0 ? ac : 1.0) : (ml > 0.0 ? S.a[ia(li, lj - 1)] : ac);
        const double ab = (gi + 1 == nr) ? (mb > 0.0 ? ac : 1.0) : (mb > 0.0 ? ac : S.a[ia(li + 1, lj)]);
        const double at = (gi == 0) ? (mt < 0.0 ? ac : 1.0) : (mt > 0.0 ? S.a[ia(li - 1, lj)] : ac);
        const double fxr_m = mr * ar, fxr_n = S.fxnm[fr] * ar, fxr_t = S.fxt[fr] * ar;
        const double fxl_m = ml * al, fxl_n = S.fxnp[fl] * al, fxl_t = S.fxt[fl] * al;
        const double fyb_m = mb * ab, fyb_n = S.fynm[fb] * ab, fyb_t = S.fyt[fb] * ab;
        const double fyt_m = mt * at, fyt_n = S.fynp[ft] * at, fyt_t = S.fyt[ft] * at;
        const double dh = (fxr_m - fxl_m) * dt_dx + (fyb_m - fyt_m) * dt_dy;
        const double new_h = hc - dh;
        const double dhu = (fxr_n - fxl_n) * dt_dx + (fyb_t - fyt_t) * dt_dy;
        const double dhv = (fxr_t - fxl_t) * dt_dx + (fyb_n - fyt_n) * dt_dy;

        // Face beds on the cell's four faces (update.rs:676-728).
        const double zc = S.z[c3];
        double zfl, zfr, zft, zfb;
        if (gj == 0)
          zfl = (ghost_bed(A.bc.kind[SIDE_WEST], zc, S.z[c3 + 1]) + zc) * 0.5;
        else
          zfl = ((S.h[c4 - 1] <= H_DRY) != dc) ? fmax(S.z[c3 - 1], zc) : (S.z[c3 - 1] + zc) * 0.5;
        if (gj + 1 == nc)
          zfr = (zc + ghost_bed(A.bc.kind[SIDE_EAST], zc, S.z[c3 - 1])) * 0.5;
        else
          zfr = (dc != (S.h[c4 + 1] <= H_DRY)) ? fmax(zc, S.z[c3 + 1]) : (zc + S.z[c3 + 1]) * 0.5;
        if (gi == 0)
          zft = (ghost_bed(A.bc.kind[SIDE_NORTH], zc, S.z[c3 + R3W]) + zc) * 0.5;
        else
          zft = ((S.h[c4 - R4W] <= H_DRY) != dc) ? fmax(S.z[c3 - R3W], zc) : (S.z[c3 - R3W] + zc) * 0.5;
        if (gi + 1 == nr)
          zfb = (zc + ghost_bed(A.bc.kind[SIDE_SOUTH], zc, S.z[c3 - R3W])) * 0.5;
        else
          zfb = (dc != (S.h[c4 + R4W] <= H_DRY)) ? fmax(zc, S.z[c3 + R3W]) : (zc + S.z[c3 + R3W]) * 0.5;

        // Explicit bed-slope source on the reconstructed face states (update.rs:1140-1180).
        const double eta_cell = hc + zc;
        const double sex = S.sxe[isx(li, lj)];
        const double eta_left = gj > 0 ? eta_cell - sex * (0.5 * dx) : eta_cell;
        const double eta_right = gj + 1 < nc ? eta_cell + sex * (0.5 * dx) : eta_cell;
        const double hfl = fmax(eta_left - zfl, 0.0);
        const double hfr = fmax(eta_right - zfr, 0.0);
        const double s_hu =
            hfa::div_rn((hfl + hfr) * ((eta_left - hfl) - (eta_right - hfr)) * (0.5 * GRAVITY), dx);
        const double sey = S.sye[isy(li, lj)];
        const double eta_top = gi > 0 ? eta_cell - sey * (0.5 * dy) : eta_cell;
        const double eta_bot = gi + 1 < nr ? eta_cell + sey * (0.5 * dy) : eta_cell;
        const double hft = fmax(eta_top - zft, 0.0);
        const double hfb = fmax(eta_bot - zfb, 0.0);
        const double s_hv =
            hfa::div_rn((hft + hfb) * ((eta_top - hft) - (eta_bot - hfb)) * (0.5 * GRAVITY), dy);

        if (new_h <= H_VEL) {
          nh = fmax(new_h, 0.0);  // moisture floor keeps the mass
          nhu = 0.0;
          nhv = 0.0;
        } else {
          double hu_old = 0.0, hv_old = 0.0;
          if (hc > H_VEL) {
            hu_old = A.in_hu[g];
            hv_old = A.in_hv[g];
          }
          nh = new_h;
          nhu = hu_old - dhu + s_hu * dt;
          nhv = hv_old - dhv + s_hv * dt;
        }
      }
      if (A.combine) {  // SSP-RK2 convex combination + floor (update.rs:1271-1286)
        const double ph = A.un_h[g], phu = A.un_hu[g], phv = A.un_hv[g];
        nh = (ph + nh) * 0.5;
        nhu = (phu + nhu) * 0.5;
        nhv = (phv + nhv) * 0.5;
        if (nh <= H_VEL) {
          nh = fmax(nh, 0.0);
          nhu = 0.0;
          nhv = 0.0;
        }
      }
      if (A.finalize) {
        finalize_cell(A, ctrl, dt, gi, gj, g, src_lo, src_hi, nh, nhu, nhv);
        cfl_cell(A, gi, gj, g, nh, nhu, nhv, sxm, sym);
        if (ctrl->check_finite && !isfinite(nh)) ++nonfin;
      }
      A.out_h[g] = nh;
      A.out_hu[g] = nhu;
      A.out_hv[g] = nhv;
    }
    __syncthreads();
  }
}

// One stage of one grid over a persistent tile loop.
__global__ void __launch_bounds__(NTHREADS, HF_MIN_BLOCKS) k_stage(const StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StageSmem& S = *reinterpret_cast<StageSmem*>(smem_raw);
  if (!A.ctrl->active) return;
  const int ntiles = A.tiles_x * A.tiles_y;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    stage_tile(A, S, tile, sxm, sym, nonfin);
  if (A.finalize) {
    block_reduce_speeds(sxm, sym, nonfin, A.ctrl);
    if (blockIdx.x == 0 && threadIdx.x == 0) commit_clock(A.ctrl);
  }
}

// One stage of every grid of an ensemble in one launch: the persistent grid
// walks the concatenated tile list of all scenarios; tile t belongs to
// scenario tile_scn[t], whose arguments (own sizes, dt, forcings, control
// block) are args[tile_scn[t]]. Finished scenarios' tiles are skipped. The
// CFL maxima are reduced per tile into the tile's scenario; each scenario's
// clock is committed afterwards by k_batch_commit.
__global__ void __launch_bounds__(NTHREADS, HF_MIN_BLOCKS)
    k_stage_batch(const StageArgs* __restrict__ args, const int* __restrict__ tile_scn,
                  const int* __restrict__ n_tiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StageSmem& S = *reinterpret_cast<StageSmem*>(smem_raw);
  const int total_tiles = *n_tiles;  // device-resident: a graph serves any set of scenarios
  for (int t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    const StageArgs& A = args[tile_scn[t]];
    if (!A.ctrl->active) continue;  // uniform over the CTA
    double sxm = 0.0, sym = 0.0;
    unsigned long long nonfin = 0;
    stage_tile(A, S, t - A.tile_base, sxm, sym, nonfin);
    if (A.finalize) block_reduce_speeds(sxm, sym, nonfin, A.ctrl);
  }
}

// Epilogue of a forward-Euler step: friction, forcings and the CFL
// reduction of the stage result (in_*) into the state (out_*).
__global__ void __launch_bounds__(NTHREADS) k_finalize(const StageArgs A) {
  Ctrl* ctrl = A.ctrl;
  if (!ctrl->active) return;
  const double dt = ctrl->dt;
  const int ntiles = A.tiles_x * A.tiles_y;
  double sxm = 0.0, sym = 0.0;
  unsigned long long nonfin = 0;
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
      double h = A.in_h[g], hu = A.in_hu[g], hv = A.in_hv[g];
      finalize_cell(A, ctrl, dt, gi, gj, g, src_lo, src_hi, h, hu, hv);
      cfl_cell(A, gi, gj, g, h, hu, hv, sxm, sym);
      if (ctrl->check_finite && !isfinite(h)) ++nonfin;
      A.out_h[g] = h;
      A.out_hu[g] = hu;
      A.out_hv[g] = hv;
    }
  }
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
        if (!(isfinite(dt) && dt > 0.0)) {
          c->status = -3;  // HF_ERR_DEGENERATE_DT
          c->err_dt = dt;
          c->err_t = c->t;
          c->err_step = c->steps;
          go = 0;
        } else {
          c->dt = dt;
          c->t_new = c->t + dt;
          const double rate = f.n_rain > 0 ? series_eval(f.rain_t, f.rain_v, f.n_rain, c->t_new) : 0.0;
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
  const double q = series_eval(f.src_t + a, f.src_q + a, b - a, c->t_new);
  f.src_dh[k] = q * c->dt / (dx * dy);
}

__global__ void k_control(Ctrl* c, double dx, double dy, ForcingDev f) {
  __shared__ int s_go;
  if (threadIdx.x == 0) s_go = control_step(c, dx, dy, f);
  __syncthreads();
  if (s_go)
    for (int k = threadIdx.x; k < f.n_src; k += blockDim.x) source_increment(c, dx, dy, f, k);
}

// Per-scenario control of an ensemble: one thread per scenario.
__global__ void k_batch_control(Ctrl* ctrls, const StageArgs* __restrict__ args, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
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
int cuda_rc(cudaError_t e) { return e == cudaSuccess ? 0 : -7; }
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

size_t stage_smem_bytes() { return sizeof(StageSmem); }

int stage_grid_size(int tiles, int device) {
  static int cached[64] = {0};
  int per_sm = 0, sms = 0;
  if (device >= 0 && device < 64 && cached[device] > 0) {
    per_sm = cached[device];
  } else {
    DevGuard dg(device);
    cudaFuncSetAttribute(k_stage, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(StageSmem));
    cudaFuncSetAttribute(k_stage_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(StageSmem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage, NTHREADS, sizeof(StageSmem));
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
  k_stage<<<grid, NTHREADS, sizeof(StageSmem), (cudaStream_t)stream>>>(a);
  return cuda_rc(cudaGetLastError());
}

int launch_finalize(const StageArgs& a, int grid, void* stream) {
  k_finalize<<<grid, NTHREADS, 0, (cudaStream_t)stream>>>(a);
  return cuda_rc(cudaGetLastError());
}

int launch_stage_batch(const StageArgs* args, const int* tile_scn, const int* n_tiles, int grid,
                       void* stream) {
  k_stage_batch<<<grid, NTHREADS, sizeof(StageSmem), (cudaStream_t)stream>>>(args, tile_scn,
                                                                             n_tiles);
  return cuda_rc(cudaGetLastError());
}

int launch_cfl_batch(const StageArgs* args, const int* tile_scn, int first_tile, int last_tile,
                     int grid, void* stream) {
  if (last_tile <= first_tile) return 0;
  k_cfl_batch<<<grid, NTHREADS, 0, (cudaStream_t)stream>>>(args, tile_scn, first_tile, last_tile);
  return cuda_rc(cudaGetLastError());
}

int launch_batch_control(Ctrl* ctrls, const StageArgs* args, int n, void* stream) {
  k_batch_control<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ctrls, args, n);
  return cuda_rc(cudaGetLastError());
}

int launch_batch_commit(Ctrl* ctrls, int n, void* stream) {
  k_batch_commit<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ctrls, n);
  return cuda_rc(cudaGetLastError());
}

int launch_cfl(const StageArgs& a, int with_ghosts, int grid, void* stream) {
  k_cfl<<<grid, NTHREADS, 0, (cudaStream_t)stream>>>(a, with_ghosts);
  return cuda_rc(cudaGetLastError());
}

int launch_control(Ctrl* ctrl, double dx, double dy, const ForcingDev& f, void* stream) {
  k_control<<<1, 256, 0, (cudaStream_t)stream>>>(ctrl, dx, dy, f);
  return cuda_rc(cudaGetLastError());
}

int launch_set_fixed(Ctrl* ctrl, double dt, void* stream) {
  k_set_fixed<<<1, 1, 0, (cudaStream_t)stream>>>(ctrl, dt);
  return cuda_rc(cudaGetLastError());
}

int launch_set_step(Ctrl* ctrl, double dt_cap, double cfl, double max_dt, int check_finite,
                    void* stream) {
  k_set_step<<<1, 1, 0, (cudaStream_t)stream>>>(ctrl, dt_cap, cfl, max_dt, check_finite);
  return cuda_rc(cudaGetLastError());
}

int launch_set_run(Ctrl* ctrl, double t_target, long long budget, double cfl, double max_dt,
                   int check_finite, int quiet_budget, void* stream) {
  k_set_run<<<1, 1, 0, (cudaStream_t)stream>>>(ctrl, t_target, budget, cfl, max_dt, check_finite,
                                               quiet_budget);
  return cuda_rc(cudaGetLastError());
}

int launch_friction(int64_t ncell, const double* n, double* h, double* hu, double* hv, double dt,
                    double dry_tol, void* stream) {
  if (ncell <= 0) return 0;
  k_friction<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(ncell, n, h, hu, hv, dt, dry_tol);
  return cuda_rc(cudaGetLastError());
}

int launch_rain(int64_t ncell, double* h, double* hu, double* hv, double rate, double dt,
                void* stream) {
  if (rate == 0.0 || ncell <= 0) return 0;  // source.rs:89-91
  const double dh = rate * dt;
  k_rain<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(ncell, h, hu, hv, dh);
  return cuda_rc(cudaGetLastError());
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
    int rc = cuda_rc(cudaGetLastError());
    if (rc) return rc;
  }
  return 0;
}

int launch_hllc(int x_dir, int64_t n, const double* ul, const double* ur, double* out,
                void* stream) {
  if (n <= 0) return 0;
  k_hllc<<<elem_grid(n), 256, 0, (cudaStream_t)stream>>>(x_dir, n, ul, ur, out);
  return cuda_rc(cudaGetLastError());
}

}  // namespace hf
