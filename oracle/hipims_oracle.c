/*
 * hipims_oracle.c -- CPU FP64 restatement of the HiPIMS shallow-water step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may
 * load it, and only as the checker or the timed CPU baseline.  The product
 * path (the CUDA library) never calls into it.
 *
 * Every function restates one reference kernel or Python routine, in the same
 * operation order so that, compiled with gcc -O2 (no FMA contraction, no fast
 * math), it reproduces the reference's own kernels built for the host bit for
 * bit.  Paths are relative to the reference project root:
 *   HC = CHANS-HiPIMS/hipims/cuda, HP = CHANS-HiPIMS/hipims/pythonHipims.
 *
 * Parity is pinned by tests/test_oracle_pin.py against (a) the reference
 * kernels compiled for the host (oracle/_ref, built by oracle/build_ref.py)
 * and (b) golden fixtures generated from that build (tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_H_SMALL 1.0e-6
#define OR_G 9.81

typedef struct {
  double h, wl, qx, qy, z;
} or_cell;

/* HC/flucCal_2ndOrder_jh_improved_Kernel.cu:74-81 (identical in the 1st-order
 * file :321-328). */
static inline double or_minmod(double x, double y) {
  if (x * y <= 0.0) return 0.0;
  return fabs(x) < fabs(y) ? x : y;
}

static inline or_cell or_load(const double *h, const double *wl,
                              const double *qx, const double *qy,
                              const double *z, int64_t i) {
  or_cell c;
  c.h = h[i];
  c.wl = wl[i];
  c.qx = qx[i];
  c.qy = qy[i];
  c.z = z[i];
  return c;
}

/* Boundary-type decode: leading decimal digit = type, the rest = id.
 * HC/flucCal_2ndOrder_jh_improved_Kernel.cu:430-438. */
void or_decode_bc(int32_t code, int32_t *type, int32_t *id) {
  int32_t bt = code;
  int n = 0;
  while (bt >= 10) {
    bt = (bt - (bt % 10)) / 10;
    n++;
  }
  *type = bt;
  *id = (int32_t)(code - bt * powf(10.0f, (float)n));
}

/* Ghost state of a missing neighbour.  Returns 0 when the type has no ghost
 * rule (the reference leaves field_r stale in that case; we skip the face).
 * HC/flucCal_2ndOrder_jh_improved_Kernel.cu:197-332 and, for type 9,
 * HC/fluxCal_jh_modified_surface_Kernel.cu:389-396. */
static int or_ghost(int type, int allow_fall, const or_cell *c, const double *n,
                    double hb, double wlb, double qxb, double qyb, or_cell *b) {
  switch (type) {
  case 3: /* RIGID / wall non-slip :199-207 */
    b->h = c->h;
    b->wl = c->wl;
    b->z = c->z;
    b->qx = (n[1] * n[1] - n[0] * n[0]) * c->qx;
    b->qy = -(n[0] * n[0] - n[1] * n[1]) * c->qy;
    return 1;
  case 4: /* WALL_SLIP :210-217 */
    b->h = c->h;
    b->wl = c->wl;
    b->z = c->z;
    b->qx = (n[1] * n[1] - n[0] * n[0]) * c->qx;
    b->qy = (n[0] * n[0] - n[1] * n[1]) * c->qy;
    return 1;
  case 5: /* OPEN :220-227 */
    *b = *c;
    return 1;
  case 6: /* H_GIVEN :278-286 */
    b->h = hb;
    b->z = c->z;
    b->wl = b->z + b->h;
    b->qx = c->qx;
    b->qy = c->qy;
    return 1;
  case 7: /* Q_GIVEN :266-275 */
    b->h = c->h;
    b->z = c->z;
    b->wl = b->z + b->h;
    b->qx = qxb;
    b->qy = qyb;
    return 1;
  case 8: /* WL_GIVEN :289-298 */
    b->z = c->z;
    b->wl = wlb > b->z ? wlb : b->z;
    b->h = b->wl - b->z;
    b->qx = c->qx;
    b->qy = c->qy;
    return 1;
  case 9: /* FALL, first order only: fluxCal_jh_modified_surface :389-396 */
    if (!allow_fall) return 0;
    b->h = 0.0;
    b->wl = c->wl;
    b->z = c->z;
    b->qx = 0.0;
    b->qy = 0.0;
    return 1;
  default:
    return 0;
  }
}

/* Step-function lookup of a boundary table row: the first row whose time is
 * not below t, clamped to the last row.  HC/flucCal_2ndOrder...:355-366. */
static int or_timelevel(double t, const double *tab, int rows, int cols) {
  int tl = 0;
  while ((t > tab[(int64_t)tl * cols]) && (tl < rows - 1)) tl++;
  return tl;
}

/* MUSCL edge value, HC/flucCal_2ndOrder_jh_improved_Kernel.cu:83-107.  The
 * edge wl it computes is overwritten by the hydrostatic reconstruction
 * (:48, :51) before any use, so it is not formed here. */
static inline void or_muscl(const or_cell *c, const or_cell *l, const or_cell *r,
                            or_cell *e) {
  e->h = c->h + 0.5 * or_minmod(c->h - l->h, r->h - c->h);
  e->wl = c->wl;
  e->z = c->z + 0.5 * or_minmod(c->z - l->z, r->z - c->z);
  if (c->h < OR_H_SMALL) {
    e->qx = 0.0;
    e->qy = 0.0;
  } else {
    e->qx = c->qx + 0.5 * or_minmod(c->qx - l->qx, r->qx - c->qx);
    e->qy = c->qy + 0.5 * or_minmod(c->qy - l->qy, r->qy - c->qy);
  }
}

/* Hydrostatic reconstruction, 2nd-order variant.
 * HC/flucCal_2ndOrder_jh_improved_Kernel.cu:43-72.  wl_cl, wl_cr are the
 * stored free-surface levels of the two cells (or of the ghost). */
static inline void or_hydro2(double wl_cl, double wl_cr, or_cell *L, or_cell *R) {
  double hi = fmax(wl_cl, wl_cr), lo = fmin(wl_cl, wl_cr);
  L->wl = L->h + L->z;
  L->wl = fmin(L->wl, hi);
  L->wl = fmax(L->wl, lo);
  R->wl = R->h + R->z;
  R->wl = fmin(R->wl, hi);
  R->wl = fmax(R->wl, lo);
  if (wl_cl > wl_cr)
    L->wl = fmax(L->wl, R->wl);
  else
    R->wl = fmax(L->wl, R->wl);
  L->z = L->wl - L->h;
  R->z = R->wl - R->h;
  double zbm = fmax(L->z, R->z);
  L->h = fmax(L->wl - zbm, 0.0);
  R->h = fmax(R->wl - zbm, 0.0);
  L->z = L->wl - L->h;
  R->z = R->wl - R->h;
}

/* Hydrostatic reconstruction, 1st-order ("jiaheng paper") variant.
 * HC/fluxCal_jh_modified_surface_Kernel.cu:96-139.  eta_c, eta_r are h+z of
 * the raw cells (field_c_h_z[0] + field_c_h_z[1]). */
static inline void or_hydro1(double hc, double zc, double hr, double zr,
                             or_cell *L, or_cell *R) {
  double ec = hc + zc, er = hr + zr;
  L->wl = L->h + L->z;
  L->wl = fmin(L->wl, fmax(ec, er));
  L->wl = fmax(L->wl, fmin(ec, er));
  R->wl = R->h + R->z;
  R->wl = fmin(R->wl, fmax(ec, er));
  R->wl = fmax(R->wl, fmin(ec, er));
  if ((ec - er) * (L->wl - R->wl) < 0.0) {
    double tmp = (L->wl + R->wl) / 2.0;
    L->wl = tmp;
    R->wl = tmp;
  }
  L->z = L->wl - L->h;
  R->z = R->wl - R->h;
  double zbm = fmax(L->z, R->z);
  L->h = fmax(L->wl - zbm, 0.0);
  R->h = fmax(R->wl - zbm, 0.0);
  L->z = L->wl - L->h;
  R->z = R->wl - R->h;
}

/* HLLC flux after the hydrostatic step; accumulates -dt/dx * F.
 * HC/flucCal_2ndOrder_jh_improved_Kernel.cu:109-195 (the 1st-order file
 * :173-260 differs only in the reconstruction it calls). */
static inline void or_hllc(int order, const or_cell *cc, const or_cell *cr,
                           or_cell *L, or_cell *R, const double *n,
                           const double *tn, double *fh, double *fqx,
                           double *fqy, double dx, double dt) {
  const double hs = OR_H_SMALL, g = OR_G;
  double ux_l = L->h < hs ? 0.0 : L->qx / L->h;
  double uy_l = L->h < hs ? 0.0 : L->qy / L->h;
  double ux_r = R->h < hs ? 0.0 : R->qx / R->h;
  double uy_r = R->h < hs ? 0.0 : R->qy / R->h;

  if (order == 2)
    or_hydro2(cc->wl, cr->wl, L, R);
  else
    or_hydro1(cc->h, cc->z, cr->h, cr->z, L, R);

  if (L->h < hs && R->h < hs) return;

  double u_L = ux_l * n[0] + uy_l * n[1];
  double u_R = ux_r * n[0] + uy_r * n[1];
  double v_L = -ux_l * n[1] + uy_l * n[0];
  double v_R = -ux_r * n[1] + uy_r * n[0];
  double qx_L = u_L * L->h;
  double qy_L = v_L * L->h;
  double qx_R = u_R * R->h;
  double qy_R = v_R * R->h;
  double a_L = sqrt(g * L->h);
  double a_R = sqrt(g * R->h);
  double h_star = pow((a_L + a_R) / 2.0 + (u_L - u_R) / 4.0, 2.0) / g;
  double u_star = (u_L + u_R) / 2.0 + a_L - a_R;
  double a_star = sqrt(g * h_star);
  double s_L = L->h <= hs ? u_R - 2.0 * a_R : fmin(u_L - a_L, u_star - a_star);
  double s_R = R->h <= hs ? u_L + 2.0 * a_L : fmax(u_R + a_R, u_star + a_star);
  double s_M = (s_L * R->h * (u_R - s_R) - s_R * L->h * (u_L - s_L)) /
               (R->h * (u_R - s_R) - L->h * (u_L - s_L));
  double h_flux_L = qx_L;
  double qx_flux_L = u_L * qx_L + 0.5 * g * L->h * L->h;
  double qy_flux_L = u_L * qy_L;
  double h_flux_R = qx_R;
  double qx_flux_R = u_R * qx_R + 0.5 * g * R->h * R->h;
  double qy_flux_R = u_R * qy_R;
  double h_flux_M =
      (s_R * h_flux_L - s_L * h_flux_R + s_L * s_R * (R->h - L->h)) / (s_R - s_L);
  double qx_flux_M =
      (s_R * qx_flux_L - s_L * qx_flux_R + s_L * s_R * (qx_R - qx_L)) / (s_R - s_L);
  double hf, qf, tf;
  if (0.0 <= s_L) {
    hf = h_flux_L;
    qf = qx_flux_L;
    tf = qy_flux_L;
  } else if (s_L < 0.0 && 0.0 <= s_M) {
    hf = h_flux_M;
    qf = qx_flux_M;
    tf = h_flux_M * v_L;
  } else if (s_M < 0.0 && 0.0 <= s_R) {
    hf = h_flux_M;
    qf = qx_flux_M;
    tf = h_flux_M * v_R;
  } else {
    hf = h_flux_R;
    qf = qx_flux_R;
    tf = qy_flux_R;
  }
  *fh -= (hf / dx) * dt;
  *fqx -= ((qf * n[0] + tf * tn[0]) / dx) * dt;
  *fqy -= ((qf * n[1] + tf * tn[1]) / dx) * dt;
}

/* Flux accumulation over the active list.  order 2 restates
 * HC/flucCal_2ndOrder_jh_improved_Kernel.cu:334-506, order 1 restates
 * HC/fluxCal_jh_modified_surface_Kernel.cu:437-615. */
void or_flux(int order, int64_t M, int64_t N, const int32_t *wetMask,
             double *h_flux, double *qx_flux, double *qy_flux, const double *h,
             const double *wl, const double *z, const double *qx,
             const double *qy, const int32_t *index, const double *normal,
             const double *given_depth, int depth_rows, int depth_cols,
             const double *given_wl, int wl_rows, int wl_cols,
             const double *given_q, int q_rows, int q_cols, double dx, double t,
             double dt) {
  const double hs = OR_H_SMALL, g = OR_G;
  int tl_d = or_timelevel(t, given_depth, depth_rows, depth_cols);
  int tl_w = or_timelevel(t, given_wl, wl_rows, wl_cols);
  int tl_q = or_timelevel(t, given_q, q_rows, q_cols);
#pragma omp parallel for schedule(static)
  for (int64_t w = 0; w < M; w++) {
    int32_t i = wetMask[w];
    int32_t c_type = index[i];
    for (int j = 0; j < 4; j++) {
      or_cell c = or_load(h, wl, qx, qy, z, i);
      double nrm[2] = {normal[j * 2], normal[j * 2 + 1]};
      double tan_[2] = {-nrm[1], nrm[0]};
      int rdir = j + 1;
      int ldir = (rdir + 2) > 4 ? rdir - 2 : rdir + 2;
      int32_t l_id = index[(int64_t)ldir * N + i];
      int32_t r_id = index[(int64_t)rdir * N + i];
      or_cell r, eL, eR;
      if (order == 2) {
        or_cell l = (l_id == -1) ? c : or_load(h, wl, qx, qy, z, l_id);
        if (r_id == -1) {
          int32_t bt, bid;
          or_decode_bc(c_type, &bt, &bid);
          double hb = given_depth[(int64_t)tl_d * depth_cols + bid + 1];
          double wlb = given_wl[(int64_t)tl_w * wl_cols + bid + 1];
          double qxb = given_q[(int64_t)tl_q * q_cols + 1 + 2 * bid];
          double qyb = given_q[(int64_t)tl_q * q_cols + 2 + 2 * bid];
          if (!or_ghost(bt, 0, &c, nrm, hb, wlb, qxb, qyb, &r)) continue;
          eL = c;
          eR = r;
        } else {
          int32_t rr_id = index[(int64_t)rdir * N + r_id];
          or_cell rr = (rr_id == -1) ? or_load(h, wl, qx, qy, z, r_id)
                                     : or_load(h, wl, qx, qy, z, rr_id);
          r = or_load(h, wl, qx, qy, z, r_id);
          or_muscl(&c, &l, &r, &eL);
          or_muscl(&r, &rr, &c, &eR);
        }
        if (c.h < hs && r.h < hs) continue;
        or_hllc(2, &c, &r, &eL, &eR, nrm, tan_, &h_flux[i], &qx_flux[i],
                &qy_flux[i], dx, dt);
        qx_flux[i] -= ((0.5 * g * (c.h + eL.h) * (eL.z - c.z) * nrm[0]) / dx) * dt;
        qy_flux[i] -= ((0.5 * g * (c.h + eL.h) * (eL.z - c.z) * nrm[1]) / dx) * dt;
      } else {
        double c_h = c.h, c_z = c.z; /* field_c_h_z */
        double l_z = (l_id == -1) ? z[i] : z[l_id];
        double r_h, r_z; /* field_r_h_z: taken before the bed slope is added */
        if (r_id == -1) {
          int32_t bt, bid;
          or_decode_bc(c_type, &bt, &bid);
          double hb = given_depth[(int64_t)tl_d * depth_cols + bid + 1];
          double wlb = given_wl[(int64_t)tl_w * wl_cols + bid + 1];
          double qxb = given_q[(int64_t)tl_q * q_cols + 1 + 2 * bid];
          double qyb = given_q[(int64_t)tl_q * q_cols + 2 + 2 * bid];
          if (!or_ghost(bt, 1, &c, nrm, hb, wlb, qxb, qyb, &r)) continue;
          r_h = r.h;
          r_z = r.z;
        } else {
          int32_t rr_id = index[(int64_t)rdir * N + r_id];
          double rr_z = (rr_id == -1) ? z[r_id] : z[rr_id];
          r = or_load(h, wl, qx, qy, z, r_id);
          r_h = r.h;
          r_z = r.z;
          double rb = or_minmod(c.z - l_z, r.z - c.z);
          if (r.h > hs) c.z += 0.5 * rb;
          rb = or_minmod(r.z - rr_z, c_z - r.z);
          if (c.h > hs) r.z += 0.5 * rb;
        }
        if (c.h < hs && r.h < hs) continue;
        or_cell ccell = {c_h, 0.0, 0.0, 0.0, c_z};
        or_cell rcell = {r_h, 0.0, 0.0, 0.0, r_z};
        eL = c;
        eR = r;
        or_hllc(1, &ccell, &rcell, &eL, &eR, nrm, tan_, &h_flux[i], &qx_flux[i],
                &qy_flux[i], dx, dt);
        qx_flux[i] -= ((0.5 * g * (eL.h + c_h) * (eL.z - c_z) * nrm[0]) / dx) * dt;
        qy_flux[i] -= ((0.5 * g * (eL.h + c_h) * (eL.z - c_z) * nrm[1]) / dx) * dt;
      }
    }
  }
}

/* Implicit Manning friction fused with the Euler update.
 * HC/friction_implicit_andUpdate_jh_Kernel.cu:22-146. */
void or_friction_update(int64_t M, const int32_t *wetMask, double *h_update,
                        double *qx_update, double *qy_update, double *z_update,
                        const uint8_t *landuse, double *h, double *wl,
                        double *qx, double *qy, double *z, const double *manning,
                        double dt) {
  const double hs = OR_H_SMALL, g = OR_G;
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < M; j++) {
    int32_t i = wetMask[j];
    h[i] += h_update[i];
    if (h[i] < hs) {
      qx[i] = 0.0;
      qy[i] = 0.0;
    } else {
      double n = manning[landuse[i]];
      double C_f = g * n * n * pow(h[i], -1.0 / 3.0);
      qx[i] += qx_update[i];
      qy[i] += qy_update[i];
      double q_norm = sqrt(qx[i] * qx[i] + qy[i] * qy[i]);
      if (n > 0.0) {
        if (fabs(qx[i]) > 1.0e-10) {
          double temp = (1.0 - sqrt(1.0 + (4.0 * dt * C_f) / (h[i] * h[i]) * q_norm)) /
                        (-2.0 * dt * C_f / (h[i] * h[i]) * (q_norm / qx[i]));
          if (fabs(temp) > 5.0 * h[i] * sqrt(h[i] * g)) {
            qx[i] = 2.0 * temp - qx[i];
            if (qx[i] * temp <= 0.0) qx[i] = 0.0;
          } else {
            qx[i] = temp;
          }
        }
        if (fabs(qy[i]) > 1.0e-10) {
          double temp = (1.0 - sqrt(1.0 + (4.0 * dt * C_f) / (h[i] * h[i]) * q_norm)) /
                        (-2.0 * dt * C_f / (h[i] * h[i]) * (q_norm / qy[i]));
          if (fabs(temp) > 5.0 * h[i] * sqrt(h[i] * g)) {
            qy[i] = 2.0 * temp - qy[i];
            if (qy[i] * temp <= 0.0) qy[i] = 0.0;
          } else {
            qy[i] = temp;
          }
        }
      }
    }
    z[i] += z_update[i];
    wl[i] = z[i] + h[i];
    h_update[i] = 0.0;
    qx_update[i] = 0.0;
    qy_update[i] = 0.0;
    z_update[i] = 0.0;
  }
}

/* Per-cell CFL time step and running maximum depth.
 * HC/timeControl_Kernel.cu:164-198 (sqrtf is single precision there too). */
void or_timestep(int64_t M, const int32_t *wetMask, double *accel,
                 double *h_max, const double *h, const double *qx,
                 const double *qy, double dx, double cfl) {
  const double hs = OR_H_SMALL, g = OR_G;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; i++) {
    int32_t j = wetMask[i];
    h_max[j] = fmax(h[j], h_max[j]);
    accel[i] = h[j] > hs ? cfl * dx /
                               ((double)sqrtf((float)(g * h[j])) +
                                fmax(fabs(qx[j]), fabs(qy[j])) / h[j])
                         : 60.0;
  }
}

/* Station rainfall source. HC/stationPrecipitation_Kernel.cu:18-29. */
void or_rain_station(int64_t N, double *h_update, const int16_t *mask,
                     const double *data, double dt) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; i++) h_update[i] += data[mask[i]] * dt;
}

/* Flux-active mask, including the reference's `n_index > 0` test that never
 * lets cell 0 activate its neighbours.  HC/fluxMaskGenerator_Kernel.cu:19-42. */
void or_flux_mask(int64_t N, uint8_t *out, const double *h, const int32_t *index,
                  double t) {
  const double hs = OR_H_SMALL;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; i++) {
    if (t == 0.0) {
      out[i] = 1;
    } else {
      int m = h[i] > hs;
      for (int nei = 1; nei < 5; nei++) {
        int32_t k = index[(int64_t)nei * N + i];
        if (k > 0) m = m || (h[k] > hs);
      }
      out[i] = (uint8_t)m;
    }
  }
}

/* Frictionless Euler update. HC/euler_update_Kernel.cu:18-36. */
void or_euler_update(int64_t M, const int32_t *mask, const double *h_update,
                     const double *qx_update, const double *qy_update,
                     const double *z_update, double *h, double *wl, double *z,
                     double *qx, double *qy) {
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < M; j++) {
    int32_t i = mask[j];
    h[i] += h_update[i];
    qx[i] += qx_update[i];
    qy[i] += qy_update[i];
    z[i] += z_update[i];
    wl[i] = h[i] + z[i];
  }
}

/* Green-Ampt infiltration. HC/infiltrationCUDA_Kernel.cu:20-46. */
void or_infiltration(int64_t M, const int32_t *wetMask, double *h_update,
                     const uint8_t *landuse, const double *h, const double *ks,
                     const double *psi, const double *dtheta, double *cum,
                     double dt) {
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < M; j++) {
    int32_t i = wetMask[j];
    uint8_t lt = landuse[i];
    double hh = h[i];
    double K_s = ks[lt], phi_s = psi[lt], dth = dtheta[lt];
    double F_0 = cum[i];
    double total_head = phi_s + hh;
    double F_1 = 0.5 * (F_0 + dt * K_s +
                        sqrt((F_0 + dt * K_s) * (F_0 + dt * K_s) +
                             4.0 * dt * K_s * total_head * dth));
    double dF = fmin(hh, F_1 - F_0);
    cum[i] += dF;
    h_update[i] -= dF;
  }
}

/* Neighbour table of a raster mask (row-major, valid = mask > 0).
 * HP/SWE_CUDA.py:173-222: row 0 = type code, rows 1-4 = E, N(row-1), W,
 * S(row+1) compacted ids, -1 where the neighbour is nodata.  torch.roll wraps
 * around the raster edge; so does this restatement.  Returns N. */
int64_t or_build_index(int64_t rows, int64_t cols, const int32_t *mask,
                       int32_t *index_out) {
  int32_t *id = (int32_t *)malloc(sizeof(int32_t) * rows * cols);
  int64_t N = 0;
  for (int64_t k = 0; k < rows * cols; k++) id[k] = mask[k] > 0 ? (int32_t)N++ : -1;
  if (index_out) {
    int64_t n = 0;
    for (int64_t y = 0; y < rows; y++)
      for (int64_t x = 0; x < cols; x++) {
        int64_t k = y * cols + x;
        if (mask[k] <= 0) continue;
        int64_t xe = (x + 1) % cols, xw = (x - 1 + cols) % cols;
        int64_t yn = (y - 1 + rows) % rows, ys = (y + 1) % rows;
        index_out[n] = mask[k];
        index_out[1 * N + n] = id[y * cols + xe];
        index_out[2 * N + n] = id[yn * cols + x];
        index_out[3 * N + n] = id[y * cols + xw];
        index_out[4 * N + n] = id[ys * cols + x];
        n++;
      }
  }
  free(id);
  return N;
}

/* ------------------------------------------------------------------------
 * One Godunov step in the order of the server loop
 * (CHANS-HiPIMS/CHANS-HiPIMS_server.py:246-256):
 *   addFlux            HP/SWE_CUDA.py:339-424  (fluxMask -> nonzero -> flux)
 *   rain               HP/SWE_CUDA.py:472-502  (station) or :517-549 (uniform)
 *   friction + dt      HP/SWE_CUDA.py:780-831
 * ------------------------------------------------------------------------ */
/* Kernel entry points of the reference's own kernels built for the host
 * (oracle/build_ref.py).  When or_godunov.ref is set, the step below drives
 * those instead of the restatement, which makes it the timed "reference" CPU
 * baseline: the reference's arithmetic under the reference's step order. */
typedef void (*or_ref_flux_fn)(int, int, int, int, int, int, int, int, int32_t *,
                               double *, double *, double *, double *, double *,
                               const int32_t *, const double *, double *, double *,
                               double *, double *, double *, double *, double *,
                               double *, double *);
typedef void (*or_ref_friction_fn)(int, int32_t *, double *, double *, double *,
                                   double *, uint8_t *, double *, double *,
                                   double *, double *, double *, double *, double *);
typedef void (*or_ref_timestep_fn)(int, int32_t *, double *, double *, double *,
                                   double *, double *, double *, double *, double *,
                                   double *);
typedef void (*or_ref_rain_fn)(int, double *, int16_t *, double *, double *);
typedef void (*or_ref_mask_fn)(int, uint8_t *, double *, const int32_t *, double *);
typedef void (*or_ref_infil_fn)(int, int32_t *, double *, uint8_t *, double *, double *,
                                double *, double *, double *, double *);
typedef struct {
  or_ref_flux_fn flux2, flux1;
  or_ref_friction_fn friction;
  or_ref_timestep_fn timestep;
  or_ref_rain_fn rain;
  or_ref_mask_fn mask;
  or_ref_infil_fn infil;
} or_ref_kernels;

typedef struct {
  int64_t N;
  int order;               /* 1 or 2 */
  double dx, cfl;
  double export_step;      /* Export_timeStep */
  int export_n;            /* export counter */
  double t, dt;
  /* state */
  double *h, *wl, *qx, *qy, *z, *h_max;
  double *h_upd, *qx_upd, *qy_upd, *z_upd;
  const int32_t *index;
  const uint8_t *landuse;
  const double *manning;
  const double *normal;
  const double *given_depth; int depth_rows, depth_cols;
  const double *given_wl; int wl_rows, wl_cols;
  const double *given_q; int q_rows, q_cols;
  /* rain: table [rain_rows, 1 + n_stations] with times in column 0 */
  const double *rain; int rain_rows, rain_cols;
  const int16_t *rain_mask; /* NULL = uniform rain (add_uniform_Precipitation) */
  int rain_index;          /* _rainfall_station_time_index */
  double *rain_rate;       /* [rain_cols-1] current interpolated rates */
  int exports;             /* number of export clips taken */
  /* scratch */
  int32_t *list;
  uint8_t *fmask;
  double *accel;
  const or_ref_kernels *ref; /* NULL: use the restatement */
  /* Green-Ampt infiltration (NULL cum: none): per-zone K_s, capillary head,
   * water-content difference; per-cell cumulative infiltrated depth */
  const double *ks, *psi, *dtheta;
  double *cum;
} or_godunov;

/* Rain table interpolation with the reference's monotone row cursor.
 * Station form HP/SWE_CUDA.py:472-495; the uniform form :520-544 gives the
 * same rates for increasing table times. */
static void or_rain_interp(or_godunov *s) {
  const double *R = s->rain;
  int C = s->rain_cols, T = s->rain_rows;
  double t = s->t;
  if (t < R[(int64_t)(T - 1) * C]) {
    for (;;) {
      if (t < R[(int64_t)(s->rain_index + 1) * C]) {
        const double *r0 = R + (int64_t)s->rain_index * C;
        const double *r1 = r0 + C;
        double per = (t - r0[0]) / (r1[0] - r0[0]);
        for (int k = 1; k < C; k++) s->rain_rate[k - 1] = r0[k] + per * (r1[k] - r0[k]);
        return;
      }
      s->rain_index++;
    }
  } else {
    for (int k = 1; k < C; k++) s->rain_rate[k - 1] -= s->rain_rate[k - 1];
  }
}

void or_godunov_step(or_godunov *s) {
  int64_t N = s->N;
  const or_ref_kernels *k = s->ref;
  double dx = s->dx, cfl = s->cfl, t = s->t, dt0 = s->dt;
  /* addFlux: fluxMask.update + nonzero */
  if (k)
    k->mask((int)N, s->fmask, s->h, s->index, &t);
  else
    or_flux_mask(N, s->fmask, s->h, s->index, s->t);
  int64_t M = 0;
  for (int64_t i = 0; i < N; i++)
    if (s->fmask[i]) s->list[M++] = (int32_t)i;
  if (M > 0) {
    if (k) {
      or_ref_flux_fn f = s->order == 2 ? k->flux2 : k->flux1;
      f((int)M, (int)N, s->depth_cols, s->depth_rows, s->wl_cols, s->wl_rows,
        s->q_cols, s->q_rows, s->list, s->h, s->wl, s->z, s->qx, s->qy, s->index,
        s->normal, (double *)s->given_depth, (double *)s->given_wl,
        (double *)s->given_q, &dx, &t, &dt0, s->h_upd, s->qx_upd, s->qy_upd);
    } else {
      or_flux(s->order, M, N, s->list, s->h_upd, s->qx_upd, s->qy_upd, s->h, s->wl,
              s->z, s->qx, s->qy, s->index, s->normal, s->given_depth,
              s->depth_rows, s->depth_cols, s->given_wl, s->wl_rows, s->wl_cols,
              s->given_q, s->q_rows, s->q_cols, s->dx, s->t, s->dt);
    }
  }
  /* rain */
  if (s->rain) {
    or_rain_interp(s);
    if (s->rain_mask) {
      if (k)
        k->rain((int)N, s->h_upd, (int16_t *)s->rain_mask, s->rain_rate, &dt0);
      else
        or_rain_station(N, s->h_upd, s->rain_mask, s->rain_rate, s->dt);
    } else {
      double rdt = s->rain_rate[0] * s->dt;
      for (int64_t i = 0; i < N; i++) s->h_upd[i] += rdt;
    }
  }
  /* infiltration on the flux list (HP/CatchFlood_main.py:164-170 order:
   * addFlux, rain, addInfiltrationSource, friction; HP/SWE_CUDA.py:439-443) */
  if (s->cum && M > 0) {
    if (k && k->infil)
      k->infil((int)M, s->list, s->h_upd, (uint8_t *)s->landuse, s->h, (double *)s->ks,
               (double *)s->psi, (double *)s->dtheta, s->cum, &dt0);
    else
      or_infiltration(M, s->list, s->h_upd, s->landuse, s->h, s->ks, s->psi, s->dtheta,
                      s->cum, s->dt);
  }
  /* time_friction_euler_update_cuda */
  double time_upper = s->dt * 10.0;
  M = 0;
  for (int64_t i = 0; i < N; i++)
    if (fabs(s->h_upd[i]) > 0.0 || s->h[i] >= 0.0) s->list[M++] = (int32_t)i;
  if (k)
    k->friction((int)M, s->list, s->h_upd, s->qx_upd, s->qy_upd, s->z_upd,
                (uint8_t *)s->landuse, s->h, s->wl, s->qx, s->qy, s->z,
                (double *)s->manning, &dt0);
  else
    or_friction_update(M, s->list, s->h_upd, s->qx_upd, s->qy_upd, s->z_upd,
                       s->landuse, s->h, s->wl, s->qx, s->qy, s->z, s->manning,
                       s->dt);
  memset(s->h_upd, 0, sizeof(double) * N);
  memset(s->qx_upd, 0, sizeof(double) * N);
  memset(s->qy_upd, 0, sizeof(double) * N);
  memset(s->z_upd, 0, sizeof(double) * N);
  for (int64_t i = 0; i < M; i++) s->accel[i] = 60.0;
  if (k)
    k->timestep((int)M, s->list, s->h_max, s->h, s->qx, s->qy, s->accel, &dx, &cfl,
                &t, &dt0);
  else
    or_timestep(M, s->list, s->accel, s->h_max, s->h, s->qx, s->qy, s->dx, s->cfl);
  double dt = s->dt;
  if (M > 0) {
    dt = s->accel[0];
    for (int64_t i = 1; i < M; i++)
      if (s->accel[i] < dt) dt = s->accel[i];
  }
  /* Python min(self.dt, time_upper): the second argument wins only when it
   * is strictly smaller. */
  if (time_upper < dt) dt = time_upper;
  double next_export = (double)(s->export_n + 1) * s->export_step;
  if (dt + s->t >= next_export) {
    dt = next_export - s->t;
    s->export_n += 1;
    s->exports += 1;
  }
  s->dt = dt;
  s->t += dt;
}

/* Run n steps, or until t >= t_end (whichever first); returns steps taken. */
int64_t or_godunov_run(or_godunov *s, int64_t n, double t_end) {
  int64_t k = 0;
  for (; k < n && s->t < t_end; k++) or_godunov_step(s);
  return k;
}

size_t or_godunov_sizeof(void) { return sizeof(or_godunov); }

void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
