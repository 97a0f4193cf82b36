// hf_adjoint.cu -- reverse-mode (adjoint) kernels of the explicit step.
//
// The reference differentiates its step only in forward mode (T = Dual,
// autograd/src/dual.rs). The adjoint here is the exact transpose of that
// tangent map for one stage: the same branches (decided on values), dt frozen
// to the primal run, max/min ties split the adjoint in halves, sqrt(0)
// passes none, powf's n * x^(n-1) derivative. So <lambda, J v> computed by the
// adjoint equals the Dual tangent's <lambda, J v> up to rounding.
//
// k_stage_adj handles one tile of output cells per CTA: it recomputes the
// forward stage of the tile and its halo in shared memory (the same phases as
// the forward kernel), then propagates the adjoint of the tile's outputs back
// through, in reverse order: the epilogue (point sources, rain, Manning
// friction, with the Manning gradient), the SSP-RK2 combination, the floors
// and the finite-volume update with its bed source, the alpha mass
// rescaling, the Audusse + HLLC faces, the limited slopes and the
// primitives. The adjoint of the stage input over the tile and its 3-cell
// halo goes to a per-tile buffer; k_adj_gather sums each cell's
// contributions from the (up to nine) tiles that touch it in a fixed order,
// so the gradient is deterministic without atomics.
#include <cuda_runtime.h>

#include "hf_device.cuh"
#include "hf_internal.h"
#include "hf_adjoint_math.cuh"
#include "hf_stage.cuh"

namespace hf {
inline namespace HF_GEOM {

namespace {

// Adjoint shared memory beside the forward tile (StageSmem). Face and slope
// adjoints reuse the forward face / slope arrays in place once their values
// are dead; the cell's bed-source slope adjoints ride in lprim until the
// cell gather replaces them.
struct AdjSmem {
  double lpre[3][TX * TY];  // adjoint of the cell's flux divergence (dh, dhu, dhv)
  double ldir[4][AN];       // direct adjoint of (h, hu, hv, n) per alpha-region cell
  double lout[AN];          // adjoint of alpha's outgoing-mass sum
  double lf4[FXN + FYN];    // face adjoint slots 4 and 5 (slots 0-3 live in the forward
  double lf5[FXN + FYN];    //   face arrays): x faces first, then y faces
  double lprim[3][R3N];     // adjoint of (eta, u, v)
};

// Which tile cells and faces exist: tile cell (li, lj) in [0,TY) x [0,TX).
__device__ __forceinline__ bool in_tile(int li, int lj) {
  return li >= 0 && li < TY && lj >= 0 && lj < TX;
}
__device__ __forceinline__ int icell(int li, int lj) { return li * TX + lj; }
// alpha region: tile plus a one-cell ring without corners
__device__ __forceinline__ bool in_alpha(int li, int lj) {
  const bool ri = li >= -1 && li <= TY, rj = lj >= -1 && lj <= TX;
  return ri && rj && !((li < 0 || li >= TY) && (lj < 0 || lj >= TX));
}

// Adjoint of the scaled flux G = alpha_up * F of a face, from the flux
// divergence adjoints of its minus cell (M) and plus cell (P) when they are
// tile cells (update.rs:1089-1092 in reverse). Components (mass, normal seen
// by M, normal seen by P, tangential).
__device__ __forceinline__ void face_lg(const AdjSmem& R, bool xd, int mi, int mj, int pi, int pj,
                                        double dt_d, double& g0, double& g1, double& g2,
                                        double& g3) {
  double mh = 0.0, mn = 0.0, mt = 0.0, ph = 0.0, pn = 0.0, pt = 0.0;
  if (in_tile(mi, mj)) {
    const int c = icell(mi, mj);
    mh = R.lpre[0][c];
    mn = xd ? R.lpre[1][c] : R.lpre[2][c];
    mt = xd ? R.lpre[2][c] : R.lpre[1][c];
  }
  if (in_tile(pi, pj)) {
    const int c = icell(pi, pj);
    ph = R.lpre[0][c];
    pn = xd ? R.lpre[1][c] : R.lpre[2][c];
    pt = xd ? R.lpre[2][c] : R.lpre[1][c];
  }
  g0 = (mh - ph) * dt_d;
  g1 = mn * dt_d;
  g2 = -pn * dt_d;
  g3 = (mt - pt) * dt_d;
}

}  // namespace

// Reverse of one stage for every tile. A holds the forward arguments of the
// stage (inputs, U^n for the combination, forcings, ctrl->dt of the step);
// lam_* is the adjoint of the stage's output (after the combination and
// epilogue when A.combine / A.finalize are set). Writes per tile the adjoint
// of the stage input (h, hu, hv) and of the Manning field over the tile and
// its 3-cell halo into halo[tile][4][R3N], and, with A.combine, 0.5 * the
// adjoint of the combination into lam_un_* (own cells).
struct AdjArgs {
  const double* lam_h;
  const double* lam_hu;
  const double* lam_hv;
  double* lam_un_h;
  double* lam_un_hu;
  double* lam_un_hv;
  double* halo;
};

__global__ void __launch_bounds__(NTHREADS, 2) k_stage_adj(const StageArgs A, const AdjArgs J) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StageSmem& S = *reinterpret_cast<StageSmem*>(smem_raw);
  AdjSmem& R = *reinterpret_cast<AdjSmem*>(smem_raw + sizeof(StageSmem));
  const Ctrl* ctrl = A.ctrl;
  const double dt = ctrl->dt;
  const int nr = A.nr, nc = A.nc;
  const double dx = A.dx, dy = A.dy;
  const double dt_dx = dt / dx;
  const double dt_dy = dt / dy;
  const double half_dx = 0.5 * dx, half_dy = 0.5 * dy;
  const double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy;
  const int tid = threadIdx.x;
  const int ntiles = A.tiles_x * A.tiles_y;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int tyi = tile / A.tiles_x;
    const int gi0 = tyi * TY, gj0 = (tile - tyi * A.tiles_x) * TX;
    if (interior_tile(A, tile))
      stage_tile_faces<double, false, true>(A, S, gi0, gj0, dt);
    else
      stage_tile_faces<double>(A, S, gi0, gj0, dt);

    // ---- A: per tile cell, epilogue / combination / update in reverse
    int src_lo = 0, src_hi = 0;
    if (A.finalize && A.f.n_src > 0) {
      src_lo = A.f.tile_start[tile];
      src_hi = A.f.tile_start[tile + 1];
    }
    for (int k = tid; k < AN; k += NTHREADS) {
      R.ldir[0][k] = 0.0; R.ldir[1][k] = 0.0; R.ldir[2][k] = 0.0; R.ldir[3][k] = 0.0;
    }
    __syncthreads();
    for (int q = 0; q < CELLS_PER_THREAD; ++q) {
      const int li = tid / TX + ROWS_PER_PASS * q, lj = tid % TX;
      if (kPartialPass && li >= TY) continue;
      const int gi = gi0 + li, gj = gj0 + lj;
      const int ce = icell(li, lj), c3 = i3(li, lj), c4 = i4(li, lj), ca = ia(li, lj);
      R.lprim[0][c3] = 0.0;  // bed-source adjoint of the cell's x / y eta slopes
      R.lprim[1][c3] = 0.0;
      R.lpre[0][ce] = 0.0; R.lpre[1][ce] = 0.0; R.lpre[2][ce] = 0.0;
      if (gi >= nr || gj >= nc) continue;
      const int64_t g = (int64_t)gi * nc + gj;
      const double hc = S.h[c4];
      const bool dc = hc <= H_DRY;
      // forward recompute of the cell update (values)
      const bool isolated = dc && gi > 0 && gi + 1 < nr && gj > 0 && gj + 1 < nc &&
                            S.h[c4 - R4W] <= H_DRY && S.h[c4 + R4W] <= H_DRY &&
                            S.h[c4 - 1] <= H_DRY && S.h[c4 + 1] <= H_DRY;
      double nh, nhu = 0.0, nhv = 0.0, new_h = 0.0;
      double zfl = 0, zfr = 0, zft = 0, zfb = 0, eta_cell = 0, sex = 0, sey = 0;
      double eta_left = 0, eta_right = 0, eta_top = 0, eta_bot = 0;
      double hfl = 0, hfr = 0, hft = 0, hfb = 0;
      bool floor1 = false;
      if (isolated) {
        nh = hc;
      } else {
        const int fr = ifx(li, lj + 1), fl = ifx(li, lj), fb = ify(li + 1, lj), ft = ify(li, lj);
        const double mr = S.fxm[fr], ml = S.fxm[fl], mb = S.fym[fb], mt = S.fym[ft];
        const double ac = S.a[ca];
        const double ar = (gj + 1 == nc) ? (mr > 0.0 ? ac : 1.0) : (mr > 0.0 ? ac : S.a[ia(li, lj + 1)]);
        const double al = (gj == 0) ? (ml < 0.0 ? ac : 1.0) : (ml > 0.0 ? S.a[ia(li, lj - 1)] : ac);
        const double ab = (gi + 1 == nr) ? (mb > 0.0 ? ac : 1.0) : (mb > 0.0 ? ac : S.a[ia(li + 1, lj)]);
        const double at = (gi == 0) ? (mt < 0.0 ? ac : 1.0) : (mt > 0.0 ? S.a[ia(li - 1, lj)] : ac);
        const double dh = (mr * ar - ml * al) * dt_dx + (mb * ab - mt * at) * dt_dy;
        new_h = hc - dh;
        const double dhu = (S.fxnm[fr] * ar - S.fxnp[fl] * al) * dt_dx + (S.fyt[fb] * ab - S.fyt[ft] * at) * dt_dy;
        const double dhv = (S.fxt[fr] * ar - S.fxt[fl] * al) * dt_dx + (S.fynm[fb] * ab - S.fynp[ft] * at) * dt_dy;
        cell_face_beds(A, S.z, dc, S.h[c4 - 1] <= H_DRY, S.h[c4 + 1] <= H_DRY,
                       S.h[c4 - R4W] <= H_DRY, S.h[c4 + R4W] <= H_DRY, c3, gi, gj, zfl, zfr, zft,
                       zfb);
        eta_cell = hc + S.z[c3];
        sex = S.sxe[isx(li, lj)];
        eta_left = gj > 0 ? eta_cell - sex * (0.5 * dx) : eta_cell;
        eta_right = gj + 1 < nc ? eta_cell + sex * (0.5 * dx) : eta_cell;
        hfl = fmax(eta_left - zfl, 0.0);
        hfr = fmax(eta_right - zfr, 0.0);
        const double s_hu = hfa::div_rn((hfl + hfr) * ((eta_left - hfl) - (eta_right - hfr)) * (0.5 * GRAVITY), dx);
        sey = S.sye[isy(li, lj)];
        eta_top = gi > 0 ? eta_cell - sey * (0.5 * dy) : eta_cell;
        eta_bot = gi + 1 < nr ? eta_cell + sey * (0.5 * dy) : eta_cell;
        hft = fmax(eta_top - zft, 0.0);
        hfb = fmax(eta_bot - zfb, 0.0);
        const double s_hv = hfa::div_rn((hft + hfb) * ((eta_top - hft) - (eta_bot - hfb)) * (0.5 * GRAVITY), dy);
        floor1 = new_h <= H_VEL;
        if (floor1) {
          nh = fmax(new_h, 0.0);
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
      double ch = nh, chu = nhu, chv = nhv, ch_pre = nh;
      if (A.combine) {
        ch_pre = (A.un_h[g] + nh) * 0.5;
        chu = (A.un_hu[g] + nhu) * 0.5;
        chv = (A.un_hv[g] + nhv) * 0.5;
        ch = ch_pre;
        if (ch_pre <= H_VEL) {
          ch = fmax(ch_pre, 0.0);
          chu = 0.0;
          chv = 0.0;
        }
      }
      // adjoint of the stage output
      double Lh = J.lam_h[g], Lhu = J.lam_hu[g], Lhv = J.lam_hv[g], Ln = 0.0;
      if (A.finalize) {
        // forward values through friction and rain
        double fh = ch, fhu = chu, fhv = chv;
        friction_cell<double>(fh, fhu, fhv, A.n[g], dt, A.dry_tol);
        double rh = fh;
        bool rain_zero = false;
        if (ctrl->rain_on) {
          const double x = fh + ctrl->rain_dh;
          if (x <= 0.0) rain_zero = true; else rh = x;
        }
        // point sources of this cell, last first (source.rs:60-68 in reverse)
        for (int s = src_hi - 1; s >= src_lo; --s) {
          const int k = A.f.tile_order[s];
          if (A.f.src_row[k] != gi || A.f.src_col[k] != gj) continue;
          double hb = rain_zero ? 0.0 : rh;  // depth before source s
          for (int s2 = src_lo; s2 < s; ++s2) {
            const int k2 = A.f.tile_order[s2];
            if (A.f.src_row[k2] == gi && A.f.src_col[k2] == gj) hb = fmax(hb + A.f.src_dh[k2], 0.0);
          }
          const double x = hb + A.f.src_dh[k];
          if (fmax(x, 0.0) == 0.0) {
            Lhu = 0.0;
            Lhv = 0.0;
          }
          Lh *= dmax0(x);
        }
        if (rain_zero) {
          Lh = 0.0; Lhu = 0.0; Lhv = 0.0;
        }
        friction_rev(ch, chu, chv, A.n[g], dt, A.dry_tol, Lh, Lhu, Lhv, Ln);
      }
      if (A.combine) {
        if (ch_pre <= H_VEL) {
          Lh *= dmax0(ch_pre);
          Lhu = 0.0;
          Lhv = 0.0;
        }
        Lh *= 0.5; Lhu *= 0.5; Lhv *= 0.5;
        J.lam_un_h[g] = Lh;
        J.lam_un_hu[g] = Lhu;
        J.lam_un_hv[g] = Lhv;
      }
      double Ldh_c = Lh;  // direct adjoint of the stage input depth
      double Lhu_c = 0.0, Lhv_c = 0.0;
      if (!isolated) {
        double L_new = Lh, L_dhu = 0.0, L_dhv = 0.0, L_shu = 0.0, L_shv = 0.0;
        if (floor1) {
          L_new = Lh * dmax0(new_h);
        } else {
          if (hc > H_VEL) {
            Lhu_c = Lhu;
            Lhv_c = Lhv;
          }
          L_dhu = -Lhu;
          L_dhv = -Lhv;
          L_shu = Lhu * dt;
          L_shv = Lhv * dt;
        }
        Ldh_c = L_new;  // new_h = hc - dh
        R.lpre[0][ce] = -L_new;
        R.lpre[1][ce] = L_dhu;
        R.lpre[2][ce] = L_dhv;
        // bed source s = (hfl + hfr) ((eta_l - hfl) - (eta_r - hfr)) (g/2) / dx
        double L_eta = 0.0, L_sex = 0.0, L_sey = 0.0;
        {
          const double kx = L_shu * (0.5 * GRAVITY) * inv_dx;
          const double Aa = hfl + hfr, Bb = (eta_left - hfl) - (eta_right - hfr);
          const double LA = kx * Bb, LB = kx * Aa;
          const double L_hfl = LA - LB, L_hfr = LA + LB;
          const double L_el = LB + L_hfl * dmax0(eta_left - zfl);
          const double L_er = -LB + L_hfr * dmax0(eta_right - zfr);
          L_eta += L_el + L_er;
          if (gj > 0) L_sex -= L_el * (0.5 * dx);
          if (gj + 1 < nc) L_sex += L_er * (0.5 * dx);
        }
        {
          const double ky = L_shv * (0.5 * GRAVITY) * inv_dy;
          const double Aa = hft + hfb, Bb = (eta_top - hft) - (eta_bot - hfb);
          const double LA = ky * Bb, LB = ky * Aa;
          const double L_hft = LA - LB, L_hfb = LA + LB;
          const double L_et = LB + L_hft * dmax0(eta_top - zft);
          const double L_eb = -LB + L_hfb * dmax0(eta_bot - zfb);
          L_eta += L_et + L_eb;
          if (gi > 0) L_sey -= L_et * (0.5 * dy);
          if (gi + 1 < nr) L_sey += L_eb * (0.5 * dy);
        }
        Ldh_c += L_eta;  // eta_cell = hc + z
        R.lprim[0][c3] = L_sex;
        R.lprim[1][c3] = L_sey;
      }
      R.ldir[0][ca] = Ldh_c;
      R.ldir[1][ca] = Lhu_c;
      R.ldir[2][ca] = Lhv_c;
      R.ldir[3][ca] = Ln;
    }
    __syncthreads();

    // ---- B2: adjoint of alpha for the tile and its ring
    for (int k = tid; k < AN; k += NTHREADS) {
      const int r = k / AW;
      const int li = r - 1, lj = k - r * AW - 1;
      R.lout[k] = 0.0;
      if (!in_alpha(li, lj)) continue;
      const int gi = gi0 + li, gj = gj0 + lj;
      if (gi < 0 || gi >= nr || gj < 0 || gj >= nc) continue;
      const int fr = ifx(li, lj + 1), fl = ifx(li, lj), fb = ify(li + 1, lj), ft = ify(li, lj);
      const double mr = S.fxm[fr], ml = S.fxm[fl], mb = S.fym[fb], mt = S.fym[ft];
      double L_a = 0.0, g0, g1, g2, g3;
      // faces used by some tile cell's update, whose upstream alpha is this cell's
      if (li >= 0 && li < TY && lj <= TX - 1 && mr > 0.0) {
        face_lg(R, true, li, lj, li, lj + 1, dt_dx, g0, g1, g2, g3);
        L_a += mr * g0 + S.fxnm[fr] * g1 + S.fxnp[fr] * g2 + S.fxt[fr] * g3;
      }
      if (li >= 0 && li < TY && lj >= 0 && (gj == 0 ? ml < 0.0 : !(ml > 0.0))) {
        face_lg(R, true, li, lj - 1, li, lj, dt_dx, g0, g1, g2, g3);
        L_a += ml * g0 + S.fxnm[fl] * g1 + S.fxnp[fl] * g2 + S.fxt[fl] * g3;
      }
      if (lj >= 0 && lj < TX && li <= TY - 1 && mb > 0.0) {
        face_lg(R, false, li, lj, li + 1, lj, dt_dy, g0, g1, g2, g3);
        L_a += mb * g0 + S.fynm[fb] * g1 + S.fynp[fb] * g2 + S.fyt[fb] * g3;
      }
      if (lj >= 0 && lj < TX && li >= 0 && (gi == 0 ? mt < 0.0 : !(mt > 0.0))) {
        face_lg(R, false, li - 1, lj, li, lj, dt_dy, g0, g1, g2, g3);
        L_a += mt * g0 + S.fynm[ft] * g1 + S.fynp[ft] * g2 + S.fyt[ft] * g3;
      }
      double out = 0.0;
      if (mr > 0.0) out = out + mr * dt_dx;
      if (ml < 0.0) out = out + (-ml) * dt_dx;
      if (mb > 0.0) out = out + mb * dt_dy;
      if (mt < 0.0) out = out + (-mt) * dt_dy;
      const double xa = S.h[i4(li, lj)] - H_DRY;
      const double avail = fmax(xa, 0.0);
      if (out > avail && out > 0.0) {  // alpha = avail / out
        const double inv_out = 1.0 / out;
        R.ldir[0][k] += L_a * inv_out * dmax0(xa);
        R.lout[k] = -L_a * avail * inv_out * inv_out;
      }
    }
    __syncthreads();

    // ---- B3: faces in reverse; slots 0-5 replace the forward face values
    for (int k = tid; k < FXN + FYN; k += NTHREADS) {
      const bool xd = k < FXN;
      const int kk = xd ? k : k - FXN;
      int li, lj;
      if (xd) {
        const int r = kk / FXW;
        li = r - 1;
        lj = kk - r * FXW - 1;
      } else {
        const int r = kk / FYW;
        li = r - 1;
        lj = kk - r * FYW - 1;
      }
      double* f0 = xd ? S.fxm : S.fym;
      double* f1 = xd ? S.fxnm : S.fynm;
      double* f2 = xd ? S.fxnp : S.fynp;
      double* f3 = xd ? S.fxt : S.fyt;
      const int gf = xd ? gj0 + lj : gi0 + li;
      const int na = xd ? nc : nr;
      const int gx = xd ? gi0 + li : gj0 + lj;
      const int nx = xd ? nr : nc;
      const int mi = xd ? li : li - 1, mj = xd ? lj - 1 : lj;
      const int pi = li, pj = lj;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, s5 = 0.0;
      if (!(gx < 0 || gx >= nx || gf < 0 || gf > na)) {
        const double m = f0[kk];
        const double dt_d = xd ? dt_dx : dt_dy;
        // adjoint of the unscaled flux F
        double lm = 0.0, ln1 = 0.0, ln2 = 0.0, lt = 0.0;
        const bool tile_face = in_tile(mi, mj) || in_tile(pi, pj);
        if (tile_face) {
          double g0, g1, g2, g3;
          face_lg(R, xd, mi, mj, pi, pj, dt_d, g0, g1, g2, g3);
          double a_up;
          if (gf == 0) a_up = m < 0.0 ? S.a[ia(pi, pj)] : 1.0;
          else if (gf == na) a_up = m > 0.0 ? S.a[ia(mi, mj)] : 1.0;
          else a_up = m > 0.0 ? S.a[ia(mi, mj)] : S.a[ia(pi, pj)];
          lm = a_up * g0; ln1 = a_up * g1; ln2 = a_up * g2; lt = a_up * g3;
        }
        if (m > 0.0 && gf > 0 && in_alpha(mi, mj)) lm += R.lout[ia(mi, mj)] * dt_d;
        if (m < 0.0 && gf < na && in_alpha(pi, pj)) lm -= R.lout[ia(pi, pj)] * dt_d;
        if (lm != 0.0 || ln1 != 0.0 || ln2 != 0.0 || lt != 0.0) {
          if (gf == 0 || gf == na) {
            const bool lo_side = gf == 0;
            const int ci = lo_side ? pi : mi, cj = lo_side ? pj : mj;
            const int64_t g0i = (int64_t)(gi0 + ci) * nc + (gj0 + cj);
            const double h = S.h[i4(ci, cj)];
            const double hu = A.in_hu[g0i], hv = A.in_hv[g0i];
            int side;
            int64_t g1i;
            double dn;
            if (xd) {
              side = lo_side ? SIDE_WEST : SIDE_EAST;
              g1i = lo_side ? g0i + 1 : g0i - 1;
              dn = dx;
            } else {
              side = lo_side ? SIDE_NORTH : SIDE_SOUTH;
              g1i = lo_side ? g0i + nc : g0i - nc;
              dn = dy;
            }
            const double* nodn = nullptr;
            const Ghost G = ghost_cell<double>(side, A.bc, h, hu, hv, A.z, A.n, nodn, g0i, g1i, dn);
            const double zc = S.z[i3(ci, cj)];
            const double zf = lo_side ? (G.z + zc) * 0.5 : (zc + G.z) * 0.5;
            const double qn = xd ? hu : hv, qt = xd ? hv : hu;
            const double gqn = xd ? G.hu : G.hv, gqt = xd ? G.hv : G.hu;
            double Lc0 = 0, Lc1 = 0, Lc2 = 0, Lg0 = 0, Lg1 = 0, Lg2 = 0;
            if (lo_side)
              wb_face_rev(G.h, gqn, gqt, h, qn, qt, zf, lm, ln1, ln2, lt, Lg0, Lg1, Lg2, Lc0, Lc1, Lc2);
            else
              wb_face_rev(h, qn, qt, G.h, gqn, gqt, zf, lm, ln1, ln2, lt, Lc0, Lc1, Lc2, Lg0, Lg1, Lg2);
            double Lh = Lc0, Lhu = xd ? Lc1 : Lc2, Lhv = xd ? Lc2 : Lc1, Ln = 0.0;
            ghost_rev(side, A.bc, h, A.z, A.n, g0i, g1i, dn, Lg0, Lg1, Lg2, Lh, Lhu, Lhv, Ln);
            s0 = Lh; s1 = Lhu; s2 = Lhv; s3 = Ln;
          } else {
            const double hm = S.h[i4(mi, mj)], hp = S.h[i4(pi, pj)];
            const bool dm = hm <= H_DRY, dp = hp <= H_DRY;
            if (!(dm && dp)) {
              const int m3 = i3(mi, mj), p3 = i3(pi, pj);
              const double zm = S.z[m3], zp = S.z[p3];
              const double zf = (dm != dp) ? fmax(zm, zp) : (zm + zp) * 0.5;
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
              const double un_m = (xd ? S.u[m3] : S.v[m3]) + sn_m * half;
              const double ut_m = (xd ? S.v[m3] : S.u[m3]) + st_m * half;
              const double un_p = (xd ? S.u[p3] : S.v[p3]) - sn_p * half;
              const double ut_p = (xd ? S.v[p3] : S.u[p3]) - st_p * half;
              const double xm = (S.eta[m3] + se_m * half) - zf;
              const double xp = (S.eta[p3] - se_p * half) - zf;
              const double h_m = fmax(xm, 0.0), h_p = fmax(xp, 0.0);
              double a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
              wb_face_rev(h_m, h_m * un_m, h_m * ut_m, h_p, h_p * un_p, h_p * ut_p, zf, lm, ln1,
                          ln2, lt, a0, a1, a2, b0, b1, b2);
              // (h, h un, h ut) from (eta, un, ut): h = max(eta - zf, 0)
              s0 = (a0 + a1 * un_m + a2 * ut_m) * dmax0(xm);
              s1 = a1 * h_m;
              s2 = a2 * h_m;
              s3 = (b0 + b1 * un_p + b2 * ut_p) * dmax0(xp);
              s4 = b1 * h_p;
              s5 = b2 * h_p;
            }
          }
        }
      }
      f0[kk] = s0; f1[kk] = s1; f2[kk] = s2; f3[kk] = s3;
      R.lf4[k] = s4;
      R.lf5[k] = s5;
    }
    __syncthreads();

    // ---- C1: per cell, gather the face adjoints into (eta, u, v) and slopes
    for (int k = tid; k < R3N; k += NTHREADS) {
      const int r = k / R3W;
      const int li = r - 3, lj = k - r * R3W - 3;
      const int gi = gi0 + li, gj = gj0 + lj;
      const bool real = gi >= 0 && gi < nr && gj >= 0 && gj < nc;
      const bool sx_in = li >= -1 && li <= TY && lj >= -2 && lj <= TX + 1;
      const bool sy_in = li >= -2 && li <= TY + 1 && lj >= -1 && lj <= TX;
      double le = 0.0, lu = 0.0, lv = 0.0;
      double lsxe = 0.0, lsxu = 0.0, lsxv = 0.0, lsye = 0.0, lsyu = 0.0, lsyv = 0.0;
      double dh = 0.0, dhu = 0.0, dhv = 0.0, dn = 0.0;  // boundary faces: raw state
      if (real) {
        if (in_tile(li, lj)) {
          lsxe = R.lprim[0][k];
          lsye = R.lprim[1][k];
        }
        if (li >= -1 && li <= TY) {
          if (lj + 1 <= TX + 1 && lj + 1 >= -1) {  // right x face: this cell is M
            const int f = ifx(li, lj + 1);
            if (gj + 1 == nc) {
              dh += S.fxm[f]; dhu += S.fxnm[f]; dhv += S.fxnp[f]; dn += S.fxt[f];
            } else {
              le += S.fxm[f]; lu += S.fxnm[f]; lv += S.fxnp[f];
              lsxe += half_dx * S.fxm[f]; lsxu += half_dx * S.fxnm[f]; lsxv += half_dx * S.fxnp[f];
            }
          }
          if (lj >= -1 && lj <= TX + 1) {  // left x face: this cell is P
            const int f = ifx(li, lj);
            if (gj == 0) {
              dh += S.fxm[f]; dhu += S.fxnm[f]; dhv += S.fxnp[f]; dn += S.fxt[f];
            } else {
              le += S.fxt[f]; lu += R.lf4[f]; lv += R.lf5[f];
              lsxe -= half_dx * S.fxt[f]; lsxu -= half_dx * R.lf4[f]; lsxv -= half_dx * R.lf5[f];
            }
          }
        }
        if (lj >= -1 && lj <= TX) {
          if (li + 1 >= -1 && li + 1 <= TY + 1) {  // bottom y face: this cell is M
            const int f = ify(li + 1, lj);
            if (gi + 1 == nr) {
              dh += S.fym[f]; dhu += S.fynm[f]; dhv += S.fynp[f]; dn += S.fyt[f];
            } else {
              le += S.fym[f]; lv += S.fynm[f]; lu += S.fynp[f];
              lsye += half_dy * S.fym[f]; lsyv += half_dy * S.fynm[f]; lsyu += half_dy * S.fynp[f];
            }
          }
          if (li >= -1 && li <= TY + 1) {  // top y face: this cell is P
            const int f = ify(li, lj);
            if (gi == 0) {
              dh += S.fym[f]; dhu += S.fynm[f]; dhv += S.fynp[f]; dn += S.fyt[f];
            } else {
              le += S.fyt[f]; lv += R.lf4[FXN + f]; lu += R.lf5[FXN + f];
              lsye -= half_dy * S.fyt[f]; lsyv -= half_dy * R.lf4[FXN + f];
              lsyu -= half_dy * R.lf5[FXN + f];
            }
          }
        }
      }
      if (in_alpha(li, lj)) {
        const int ca = ia(li, lj);
        R.ldir[0][ca] += dh;
        R.ldir[1][ca] += dhu;
        R.ldir[2][ca] += dhv;
        R.ldir[3][ca] += dn;
      }
      R.lprim[0][k] = le;
      R.lprim[1][k] = lu;
      R.lprim[2][k] = lv;
      if (sx_in) {
        const int s = isx(li, lj);
        S.sxe[s] = lsxe; S.sxu[s] = lsxu; S.sxv[s] = lsxv;
      }
      if (sy_in) {
        const int s = isy(li, lj);
        S.sye[s] = lsye; S.syu[s] = lsyu; S.syv[s] = lsyv;
      }
    }
    __syncthreads();

    // ---- C2: slopes and primitives in reverse; adjoint of the stage input
    double* halo_t = J.halo + (size_t)tile * 4 * R3N;
    for (int k = tid; k < R3N; k += NTHREADS) {
      const int r = k / R3W;
      const int li = r - 3, lj = k - r * R3W - 3;
      const int gi = gi0 + li, gj = gj0 + lj;
      double oh = 0.0, ohu = 0.0, ohv = 0.0, on = 0.0;
      if (gi >= 0 && gi < nr && gj >= 0 && gj < nc) {
        double le = R.lprim[0][k], lu = R.lprim[1][k], lv = R.lprim[2][k];
        // slopes of this cell and its neighbours along x (o = -1, 0, 1) and y
        for (int dir = 0; dir < 2; ++dir) {
          const bool xd = dir == 0;
          const int na = xd ? nc : nr;
          if (na < 2) continue;
          const double d = xd ? dx : dy;
          const double inv_d = xd ? inv_dx : inv_dy;
          for (int o = -1; o <= 1; ++o) {
            const int si = xd ? li : li + o, sj = xd ? lj + o : lj;  // slope cell
            const bool in_reg = xd ? (si >= -1 && si <= TY && sj >= -2 && sj <= TX + 1)
                                   : (si >= -2 && si <= TY + 1 && sj >= -1 && sj <= TX);
            if (!in_reg) continue;
            const int ga = xd ? gj + o : gi + o;
            if (ga < 0 || ga >= na) continue;
            const int st4 = xd ? 1 : R4W, st3 = xd ? 1 : R3W;
            const int s4 = i4(si, sj), s3 = i3(si, sj);
            const int lo = max(ga - 2, 0) - ga, hi = min(ga + 2, na - 1) - ga;
            bool anyd = false;
            for (int w = lo; w <= hi; ++w) anyd |= S.h[s4 + w * st4] <= H_DRY;
            if (anyd) continue;
            const int sidx = xd ? isx(si, sj) : isy(si, sj);
            const double Le = xd ? S.sxe[sidx] : S.sye[sidx];
            const double Lu = xd ? S.sxu[sidx] : S.syu[sidx];
            const double Lv = xd ? S.sxv[sidx] : S.syv[sidx];
            // coefficient of this cell (offset -o from the slope cell) in each slope
            const int rel = -o;  // -1: left neighbour of the slope cell, 0: itself, 1: right
            double ce, cu, cv;
            if (ga == 0) {  // (q[+1] - q[0]) / d
              ce = cu = cv = rel == 1 ? 1.0 : (rel == 0 ? -1.0 : 0.0);
            } else if (ga == na - 1) {  // (q[0] - q[-1]) / d
              ce = cu = cv = rel == 0 ? 1.0 : (rel == -1 ? -1.0 : 0.0);
            } else {
              const double* fe = S.eta;
              const double* fu = xd ? S.u : S.u;
              const double* fv = xd ? S.v : S.v;
              double cc[3];
              const double* fld[3] = {fe, fu, fv};
              for (int q = 0; q < 3; ++q) {
                const double* F = fld[q];
                const int pk = minmod_pick(F[s3] - F[s3 - st3], F[s3 + st3] - F[s3], d);
                if (pk == 0) cc[q] = rel == 0 ? 1.0 : (rel == -1 ? -1.0 : 0.0);
                else if (pk == 1) cc[q] = rel == 1 ? 1.0 : (rel == 0 ? -1.0 : 0.0);
                else cc[q] = 0.0;
              }
              ce = cc[0]; cu = cc[1]; cv = cc[2];
            }
            le += ce * Le * inv_d;
            lu += cu * Lu * inv_d;
            lv += cv * Lv * inv_d;
          }
        }
        // primitives: eta = h + z, u = hu / h, v = hv / h (when h > H_VEL)
        const double hh = S.h[i4(li, lj)];
        oh = le;
        if (hh > H_VEL) {
          const double uu = S.u[k], vv = S.v[k];
          const double inv = 1.0 / hh;
          ohu = lu * inv;
          ohv = lv * inv;
          oh -= (lu * uu + lv * vv) * inv;
        }
        if (in_alpha(li, lj)) {
          const int ca = ia(li, lj);
          oh += R.ldir[0][ca];
          ohu += R.ldir[1][ca];
          ohv += R.ldir[2][ca];
          on = R.ldir[3][ca];
        }
      }
      halo_t[k] = oh;
      halo_t[R3N + k] = ohu;
      halo_t[2 * R3N + k] = ohv;
      halo_t[3 * R3N + k] = on;
    }
    __syncthreads();
  }
}

// Sum of the per-tile halo adjoints of every cell (in a fixed tile order),
// plus `add_*` when given: out = sum (+ add); grad_n += sum of the Manning
// part.
__global__ void k_adj_gather(int nr, int nc, int tiles_x, int tiles_y, const double* __restrict__ halo,
                             const double* __restrict__ add_h, const double* __restrict__ add_hu,
                             const double* __restrict__ add_hv, double* __restrict__ out_h,
                             double* __restrict__ out_hu, double* __restrict__ out_hv,
                             double* __restrict__ grad_n) {
  const int64_t ncell = (int64_t)nr * nc;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ncell;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int gi = (int)(g / nc), gj = (int)(g - (int64_t)gi * nc);
    const int ti = gi / TY, tj = gj / TX;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int a = -1; a <= 1; ++a) {
      const int t_i = ti + a;
      if (t_i < 0 || t_i >= tiles_y) continue;
      const int li = gi - t_i * TY;
      if (li < -3 || li >= TY + 3) continue;
      for (int b = -1; b <= 1; ++b) {
        const int t_j = tj + b;
        if (t_j < 0 || t_j >= tiles_x) continue;
        const int lj = gj - t_j * TX;
        if (lj < -3 || lj >= TX + 3) continue;
        const double* hb = halo + (size_t)(t_i * tiles_x + t_j) * 4 * R3N + i3(li, lj);
        s0 += hb[0];
        s1 += hb[R3N];
        s2 += hb[2 * R3N];
        s3 += hb[3 * R3N];
      }
    }
    if (add_h) {
      s0 += add_h[g];
      s1 += add_hu[g];
      s2 += add_hv[g];
    }
    out_h[g] = s0;
    out_hu[g] = s1;
    out_hv[g] = s2;
    grad_n[g] += s3;
  }
}

// Misfit seeds of one step: lam_h[cell_g] += 2 (h_g - obs_g), gauges in order.
__global__ void k_adj_seed(double* lam_h, const int64_t* __restrict__ cells, int n_gauges,
                           const double* __restrict__ gauge_h, const double* __restrict__ obs) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int k = 0; k < n_gauges; ++k) lam_h[cells[k]] += 2.0 * (gauge_h[k] - obs[k]);
}

// Records of a misfit run. Before the stages of a step: its dt and start
// time (index = steps so far). After them: the gauge depths (and tangents)
// of the new state (index = steps - 1). Inactive steps record nothing.
__global__ void k_calib_pre(const Ctrl* c, double* dts, double* ts, long long cap) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || !c->active || c->steps >= cap) return;
  dts[c->steps] = c->dt;
  ts[c->steps] = c->t;
}

// Checkpoint of the state before step c->steps when that is a multiple of
// `every` (the first step included; nothing once the run has ended).
__global__ void k_calib_ckpt(const Ctrl* c, const double* __restrict__ h,
                             const double* __restrict__ hu, const double* __restrict__ hv,
                             double* ckpt, long long every, long long cap, long long ncell) {
  const long long s = c->steps;
  if (s % every != 0 || s >= cap || (s > 0 && !c->active)) return;
  double* dst = ckpt + (s / every) * 3 * ncell;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ncell;
       i += (long long)gridDim.x * blockDim.x) {
    dst[i] = h[i];
    dst[ncell + i] = hu[i];
    dst[2 * ncell + i] = hv[i];
  }
}

__global__ void k_calib_post(const Ctrl* c, const double* __restrict__ h,
                             const double* __restrict__ dh, const int64_t* __restrict__ cells,
                             int n_gauges, double* gauge_h, double* gauge_dh, long long cap,
                             int lanes, long long lane_stride) {
  if (!c->active) return;
  const long long k = c->steps - 1;
  if (k < 0 || k >= cap) return;
  for (int g = threadIdx.x; g < n_gauges; g += blockDim.x) {
    gauge_h[k * n_gauges + g] = h[cells[g]];
    if (dh)
      for (int l = 0; l < lanes; ++l)
        gauge_dh[((long long)l * cap + k) * n_gauges + g] = dh[l * lane_stride + cells[g]];
  }
}

// Rewinds a control block to the start of recorded step k (replay mode).
__global__ void k_calib_rewind(Ctrl* c, const double* __restrict__ ts, long long k) {
  c->t = ts[k];
  c->steps = k;
  c->status = 0;
}

namespace {
int elem_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}
}  // namespace

size_t adj_halo_doubles_per_tile() { return (size_t)4 * R3N; }
size_t adj_smem_bytes() { return sizeof(StageSmem) + sizeof(AdjSmem); }

int adj_grid_size(int tiles, int device) {
  static int cached[64] = {0};
  int per_sm = 0, sms = 0;
  if (device >= 0 && device < 64 && cached[device] > 0) {
    per_sm = cached[device];
  } else {
    cudaFuncSetAttribute(k_stage_adj, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)adj_smem_bytes());
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_adj, NTHREADS, adj_smem_bytes());
    if (per_sm < 1) per_sm = 1;
    if (device >= 0 && device < 64) cached[device] = per_sm;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int g = per_sm * (sms > 0 ? sms : 148);
  return tiles < g ? (tiles < 1 ? 1 : tiles) : g;
}

int launch_stage_adj(const StageArgs& a, const double* lam_h, const double* lam_hu,
                     const double* lam_hv, double* lam_un_h, double* lam_un_hu,
                     double* lam_un_hv, double* halo, int grid, void* stream) {
  AdjArgs j{lam_h, lam_hu, lam_hv, lam_un_h, lam_un_hu, lam_un_hv, halo};
  k_stage_adj<<<grid, NTHREADS, adj_smem_bytes(), (cudaStream_t)stream>>>(a, j);
  return launched(stream);
}

int launch_adj_gather(int nr, int nc, int tiles_x, int tiles_y, const double* halo,
                      const double* add_h, const double* add_hu, const double* add_hv,
                      double* out_h, double* out_hu, double* out_hv, double* grad_n,
                      void* stream) {
  const int64_t ncell = (int64_t)nr * nc;
  k_adj_gather<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(
      nr, nc, tiles_x, tiles_y, halo, add_h, add_hu, add_hv, out_h, out_hu, out_hv, grad_n);
  return launched(stream);
}

int launch_adj_seed(double* lam_h, const int64_t* cells, int n_gauges, const double* gauge_h,
                    const double* obs, void* stream) {
  if (n_gauges <= 0) return 0;
  k_adj_seed<<<1, 32, 0, (cudaStream_t)stream>>>(lam_h, cells, n_gauges, gauge_h, obs);
  return launched(stream);
}

int launch_calib_pre(const Ctrl* c, double* dts, double* ts, long long cap, void* stream) {
  k_calib_pre<<<1, 32, 0, (cudaStream_t)stream>>>(c, dts, ts, cap);
  return launched(stream);
}

int launch_calib_post(const Ctrl* c, const double* h, const double* dh, const int64_t* cells,
                      int n_gauges, double* gauge_h, double* gauge_dh, long long cap,
                      void* stream, int lanes, long long lane_stride) {
  if (n_gauges <= 0) return 0;
  k_calib_post<<<1, 128, 0, (cudaStream_t)stream>>>(c, h, dh, cells, n_gauges, gauge_h, gauge_dh,
                                                    cap, lanes, lane_stride);
  return launched(stream);
}

int launch_calib_ckpt(const Ctrl* c, const double* h, const double* hu, const double* hv,
                      double* ckpt, long long every, long long cap, long long ncell,
                      void* stream) {
  k_calib_ckpt<<<elem_grid(ncell), 256, 0, (cudaStream_t)stream>>>(c, h, hu, hv, ckpt, every,
                                                                    cap, ncell);
  return launched(stream);
}

int launch_calib_rewind(Ctrl* c, const double* ts, long long k, void* stream) {
  k_calib_rewind<<<1, 1, 0, (cudaStream_t)stream>>>(c, ts, k);
  return launched(stream);
}

}  // namespace HF_GEOM
}  // namespace hf
