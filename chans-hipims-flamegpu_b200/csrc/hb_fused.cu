// hb_fused.cu -- the fused dense-tile HiPIMS step for sm_100a.
//
// One kernel launch advances every instance of a batch by one time step.  It
// replaces, per step, the reference's
//   fluxMask -> nonzero -> fluxCalculation (HP/SWE_CUDA.py:339-424)
//   station / uniform rain                  (HP/SWE_CUDA.py:497-549)
//   friction + Euler update, timeControl, torch.min, 10x cap, export clip
//                                           (HP/SWE_CUDA.py:780-831)
// with the same decisions on a dense raster:
//  * a CTA owns a TY x TX tile; the tile plus a 2-cell halo (4 columns on the
//    x sides, for 16-byte alignment) of h, qx, qy, z and the cell code is
//    staged in shared memory;
//  * every face touching the tile is evaluated ONCE (MUSCL edges, hydrostatic
//    reconstruction, HLLC, both sides' bed-slope terms) into shared memory;
//    the reference evaluates each face twice, once from each cell;
//  * each cell then gathers its four faces in the reference's E, N, W, S
//    order, applies rain, implicit Manning friction and the update, tracks
//    h_max, its CFL wave speed and the FP64 volume;
//  * per-tile partials go to the workspace; the last tile of an instance to
//    finish (atomic counter, no spinning) reduces them and advances the
//    instance's control block: dt, t, export clip, rain rate and boundary
//    values for the next step.  dt and t never leave the device.
// The fluxMask activity rule is reproduced per cell, including the
// reference's neglect of the wetness of compacted cell 0
// (HC/fluxMaskGenerator_Kernel.cu:36).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <cuda.h>
#include <cuda/atomic>

#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "hb_common.cuh"
#include "hb_datum_halo.cuh"
#include "hb_once.h"
#include "hb_physics.cuh"
#include "hipims_b200_fused.h"

namespace hb {
namespace {

constexpr int kNT = 256;  // threads per CTA
// Tiles per reduction group of the rows kernel: the last tile of a group to
// finish sums the group's partials (one per thread of a 128-thread CTA), and
// the last group of an instance finalizes the step from the group sums.
constexpr int kGroupTiles = 128;

struct TilePartial {
  double smax;     // max CFL wave speed sqrt(g h) + max(|qx|, |qy|) / h over wet cells
  double volume;   // sum of h over valid cells
  double outflow;  // sum over boundary faces of the outward mass flux
  int32_t any_dry; // a valid cell had h <= h_small (its dt candidate is 60 s)
  int32_t pad;
};

template <typename T, int TY, int TX>
struct Smem {
  static constexpr int SW = TX + 8;   // staged row width (4 halo columns each side)
  static constexpr int SH = TY + 4;   // staged rows (2 halo rows each side)
  static constexpr int NXF = TY * (TX + 1);
  static constexpr int NYF = (TY + 1) * TX;
  T h[SH * SW], qx[SH * SW], qy[SH * SW], z[SH * SW];
  uint8_t code[SH * SW];
  // face results: mass flux, x/y momentum flux (global frame, from the side
  // of the west/south cell A), bed-slope term of side A and of side B
  T xf[5][NXF];
  T yf[5][NYF];
  double bc[HB_MAX_CLASSES][4];
  int bctype[HB_MAX_CLASSES];
  T ddatum[9];
  // per-tile reductions
  double red_d[2][kNT / 32];
  double red_s[kNT / 32];
  int red_i[kNT / 32];
  int last;
};

// ---------------------------------------------------------------------------
// Face evaluation
// ---------------------------------------------------------------------------
template <typename T>
struct FaceOut {
  T fh, fx, fy, sa, sb;
};

template <typename T, int TY, int TX>
__device__ __forceinline__ Cell<T> sm_cell(const Smem<T, TY, TX> &s, int k) {
  Cell<T> c;
  c.h = s.h[k];
  c.qx = s.qx[k];
  c.qy = s.qy[k];
  c.z = s.z[k];
  c.wl = c.z + c.h;  // the reference stores wl = z + h after every update
  return c;
}

__device__ __forceinline__ bool is_valid(uint8_t code) { return (code >> 4) != HB_NODATA_CLASS; }

template <bool B>
struct BoolTag {
  static constexpr bool value = B;
};

// Interior face between valid cells A (west/south) and B (east/north),
// evaluated from A's side with normal +x (DIR 0) or +y (DIR 1, towards the
// row above).  kl / krr: opposite neighbours of A / B (may be no-data).
template <typename T, bool FAST, int DIR, int TY, int TX>
__device__ __forceinline__ FaceOut<T> interior_face(const Smem<T, TY, TX> &s, int ka,
                                                    int kb, int kl, int krr) {
  const T hs = T(kHSmall), g = T(kG);
  FaceOut<T> o{T(0), T(0), T(0), T(0), T(0)};
  Cell<T> A = sm_cell(s, ka), B = sm_cell(s, kb);
  if (A.h < hs && B.h < hs) return o;
  Cell<T> L = is_valid(s.code[kl]) ? sm_cell(s, kl) : A;
  Cell<T> R = is_valid(s.code[krr]) ? sm_cell(s, krr) : B;
  Cell<T> eL, eR;
  muscl(A, L, B, eL);
  muscl(B, R, A, eR);
  T ux_l, uy_l, ux_r, uy_r;
  if constexpr (FAST) {
    const T il = eL.h < hs ? T(0) : T(1) / eL.h;
    const T ir = eR.h < hs ? T(0) : T(1) / eR.h;
    ux_l = eL.qx * il; uy_l = eL.qy * il;
    ux_r = eR.qx * ir; uy_r = eR.qy * ir;
  } else {
    ux_l = eL.h < hs ? T(0) : eL.qx / eL.h;
    uy_l = eL.h < hs ? T(0) : eL.qy / eL.h;
    ux_r = eR.h < hs ? T(0) : eR.qx / eR.h;
    uy_r = eR.h < hs ? T(0) : eR.qy / eR.h;
  }
  hydro2(A.wl, B.wl, eL, eR);
  T Fh, Fn, Ft;
  if (DIR == 0) {
    // n = (1, 0), t = (0, 1)
    if (hllc<T, FAST>(eL.h, eR.h, ux_l, ux_r, uy_l, uy_r, Fh, Fn, Ft)) {
      o.fh = Fh; o.fx = Fn; o.fy = Ft;
    }
  } else {
    // n = (0, 1), t = (-1, 0): u = uy, v = -ux; Fx = -Ft, Fy = Fn
    if (hllc<T, FAST>(eL.h, eR.h, uy_l, uy_r, -ux_l, -ux_r, Fh, Fn, Ft)) {
      o.fh = Fh; o.fx = -Ft; o.fy = Fn;
    }
  }
  o.sa = T(0.5) * g * (A.h + eL.h) * (eL.z - A.z);
  o.sb = T(0.5) * g * (B.h + eR.h) * (eR.z - B.z);
  return o;
}

// Face with exactly one valid side: the valid cell C sees a ghost built from
// its boundary class, along its outward normal (n0, n1).  Returns the flux
// from C's side and C's bed-slope term.
template <typename T, bool FAST, int TY, int TX>
__device__ __noinline__ void boundary_face(const Smem<T, TY, TX> &s, int kc, T n0, T n1,
                                           T datum, T &fh, T &fx, T &fy, T &sc) {
  const T hs = T(kHSmall), g = T(kG);
  fh = fx = fy = sc = T(0);
  Cell<T> C = sm_cell(s, kc);
  const int cls = s.code[kc] >> 4;
  const int type = s.bctype[cls];
  Cell<T> G;
  const T hb = (T)s.bc[cls][0], wlb = (T)(s.bc[cls][1] - (double)datum);
  const T qxb = (T)s.bc[cls][2], qyb = (T)s.bc[cls][3];
  if (!ghost(type, false, C, n0, n1, hb, wlb, qxb, qyb, G)) return;
  if (C.h < hs && G.h < hs) return;
  Cell<T> eL = C, eR = G;
  // the same arithmetic as interior faces, so that a state symmetric about a
  // wall gives bitwise the same pressure flux on both sides of a cell
  T ux_l, uy_l, ux_r, uy_r;
  if constexpr (FAST) {
    const T il = eL.h < hs ? T(0) : T(1) / eL.h;
    const T ir = eR.h < hs ? T(0) : T(1) / eR.h;
    ux_l = eL.qx * il; uy_l = eL.qy * il;
    ux_r = eR.qx * ir; uy_r = eR.qy * ir;
  } else {
    ux_l = eL.h < hs ? T(0) : eL.qx / eL.h;
    uy_l = eL.h < hs ? T(0) : eL.qy / eL.h;
    ux_r = eR.h < hs ? T(0) : eR.qx / eR.h;
    uy_r = eR.h < hs ? T(0) : eR.qy / eR.h;
  }
  hydro2(C.wl, G.wl, eL, eR);
  const T u_L = ux_l * n0 + uy_l * n1, u_R = ux_r * n0 + uy_r * n1;
  const T v_L = -ux_l * n1 + uy_l * n0, v_R = -ux_r * n1 + uy_r * n0;
  T Fh, Fn, Ft;
  if (hllc<T, FAST>(eL.h, eR.h, u_L, u_R, v_L, v_R, Fh, Fn, Ft)) {
    fh = Fh;
    fx = Fn * n0 + Ft * (-n1);
    fy = Fn * n1 + Ft * n0;
  }
  sc = T(0.5) * g * (C.h + eL.h) * (eL.z - C.z);
}

// ---------------------------------------------------------------------------
// Block reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------------------
// Control-block helpers (single thread)
// ---------------------------------------------------------------------------

// Rain rate at t with the reference's monotone row cursor
// (HP/SWE_CUDA.py:472-495): linear interpolation, zero after the last row.
// The cursor and multiplier are read from `rd` (the control block or a
// snapshot of it) and the moved cursor is written to `wr`.
__device__ double rain_rate_at(const hb_instance &in, const hb_ctrl *rd, hb_ctrl *wr, double t) {
  if (!in.rain_tab || in.rain_rows < 2) return 0.0;
  const double *R = in.rain_tab;
  const int C = in.rain_cols;
  if (!(t < R[(int64_t)(in.rain_rows - 1) * C])) return 0.0;
  int idx = min(max(rd->rain_index, 0), in.rain_rows - 2);
  while (idx + 2 < in.rain_rows && !(t < R[(int64_t)(idx + 1) * C])) idx++;
  wr->rain_index = idx;
  const double *r0 = R + (int64_t)idx * C, *r1 = r0 + C;
  const double per = (t - r0[0]) / (r1[0] - r0[0]);
  return (r0[1] + per * (r1[1] - r0[1])) * rd->rain_mult;
}

// Rates of every rain station at t (HP/SWE_CUDA.py:472-502: the row cursor
// rain_rate_at left in the control block, linear interpolation per station
// column, zero from the last row on), stations first, first + stride, ...
__device__ void station_rates_at(const hb_instance &in, const hb_ctrl *c, double t, int first,
                                 int stride) {
  if (!in.rain_station) return;
  const double *R = in.rain_tab;
  const int C = in.rain_cols;
  const bool inside = R && in.rain_rows >= 2 && t < R[(int64_t)(in.rain_rows - 1) * C];
  const double *r0 = inside ? R + (int64_t)c->rain_index * C : nullptr;
  const double per = inside ? (t - r0[0]) / (r0[C] - r0[0]) : 0.0;
  for (int k = first; k < in.n_stations; k += stride) {
    double rate = 0.0;
    if (inside && k + 1 < C) rate = (r0[k + 1] + per * (r0[C + k + 1] - r0[k + 1])) * c->rain_mult;
    in.station_rate[k] = rate;
  }
}

// Boundary values of every class at t (step-function lookup,
// HC/flucCal_2ndOrder_jh_improved_Kernel.cu:355-366, 441-446).
__device__ void bc_values_at(const hb_instance &in, hb_ctrl *c, double t) {
  const int tl_d = in.given_depth ? timelevel(t, in.given_depth, in.depth_rows, in.depth_cols) : 0;
  const int tl_w = in.given_wl ? timelevel(t, in.given_wl, in.wl_rows, in.wl_cols) : 0;
  const int tl_q = in.given_q ? timelevel(t, in.given_q, in.q_rows, in.q_cols) : 0;
  for (int k = 0; k < HB_MAX_CLASSES; k++) {
    const int id = in.bc_id[k];
    double hb = 0, wlb = 0, qxb = 0, qyb = 0;
    if (in.given_depth && id + 1 < in.depth_cols)
      hb = in.given_depth[(int64_t)tl_d * in.depth_cols + id + 1];
    if (in.given_wl && id + 1 < in.wl_cols)
      wlb = in.given_wl[(int64_t)tl_w * in.wl_cols + id + 1];
    if (in.given_q && 2 + 2 * id < in.q_cols) {
      qxb = in.given_q[(int64_t)tl_q * in.q_cols + 1 + 2 * id];
      qyb = in.given_q[(int64_t)tl_q * in.q_cols + 2 + 2 * id];
    }
    c->bc_vals[k][0] = (float)hb;
    c->bc_vals[k][1] = (float)wlb;
    c->bc_vals[k][2] = (float)qxb;
    c->bc_vals[k][3] = (float)qyb;
  }
}

}  // namespace

// Exact boundary values are kept in a double side table: bc_vals in hb_ctrl
// is the float copy the host reads; the kernels read this table.
struct BcTable {
  double v[HB_MAX_CLASSES][4];
};

namespace {

__device__ void bc_values_exact(const hb_instance &in, double t, BcTable *out) {
  const int tl_d = in.given_depth ? timelevel(t, in.given_depth, in.depth_rows, in.depth_cols) : 0;
  const int tl_w = in.given_wl ? timelevel(t, in.given_wl, in.wl_rows, in.wl_cols) : 0;
  const int tl_q = in.given_q ? timelevel(t, in.given_q, in.q_rows, in.q_cols) : 0;
  for (int k = 0; k < HB_MAX_CLASSES; k++) {
    const int id = in.bc_id[k];
    double hb = 0, wlb = 0, qxb = 0, qyb = 0;
    if (in.given_depth && id + 1 < in.depth_cols)
      hb = in.given_depth[(int64_t)tl_d * in.depth_cols + id + 1];
    if (in.given_wl && id + 1 < in.wl_cols)
      wlb = in.given_wl[(int64_t)tl_w * in.wl_cols + id + 1];
    if (in.given_q && 2 + 2 * id < in.q_cols) {
      qxb = in.given_q[(int64_t)tl_q * in.q_cols + 1 + 2 * id];
      qyb = in.given_q[(int64_t)tl_q * in.q_cols + 2 + 2 * id];
    }
    out->v[k][0] = hb;
    out->v[k][1] = wlb;
    out->v[k][2] = qxb;
    out->v[k][3] = qyb;
  }
}


// Last tile of an instance in a step: reduce the tiles' partials and advance
// the control block (HP/SWE_CUDA.py:818-831): dt = min over cells of
// CFL * dx / speed (60 s for dry cells), the 10x growth cap, the clip to the
// next export time, t += dt, FP64 volume / outflow / rain totals, and the rain
// rate and boundary values of the next step.  Called by every thread of the
// CTA that finished the instance's last tile.
// The clock after a step: dt of the next step from the largest wave speed SM
// and the any-dry flag D (HC/timeControl_Kernel.cu:164-198 per cell, torch.min,
// then HP/SWE_CUDA.py:818-831: 10x cap, export clip, t += dt), the rain rate
// and the boundary values at the new t.  All threads of the block call it;
// thread 0 owns the control block.  The step's clock fields are read from
// `snap` (the control block itself, or a copy taken at the start of the
// finalize) and the new values are written to the control block.
template <typename T, int NT>
__device__ void advance_clock(const hb_instance &in, int ii, BcTable *bct, double SM, int D,
                              const hb_ctrl *snap) {
  const int tid = threadIdx.x;
  hb_ctrl *ctrl = in.ctrl;
  __shared__ double s_tnew;
  if (tid == 0) {
    const double dtn = snap->dt, tn = snap->t;
    // min over cells of CFL*dx/speed; the division is monotone, so dividing
    // once by the largest speed gives the same value.
    double cand = INFINITY;
    if (SM > 0.0) cand = (double)((T)in.cfl * (T)in.dx / (T)SM);
    if (D) cand = fmin(cand, 60.0);
    double dtnew = (cand == INFINITY) ? dtn : cand;
    const double upper = dtn * 10.0;
    if (upper < dtnew) dtnew = upper;  // Python min(self.dt, time_upper)
    const double next_export = (double)(snap->export_n + 1) * snap->export_step;
    if (snap->export_step > 0.0 && dtnew + tn >= next_export) {
      dtnew = next_export - tn;
      ctrl->export_n = snap->export_n + 1;
      ctrl->exports = snap->exports + 1;
      if (snap->halt_on_export) ctrl->halted = 1;
    }
    const int64_t step = snap->step;
    if (in.dt_replay && step < in.n_replay) dtnew = in.dt_replay[step];
    if (!isfinite(dtnew)) atomicOr(&ctrl->status, 1);
    const double tnew = tn + dtnew;
    ctrl->dt = dtnew;
    ctrl->t = tnew;
    ctrl->step = step + 1;
    if (tnew >= snap->t_end) ctrl->halted = 1;
    s_tnew = tnew;
  }
  __syncthreads();
  const double tnew = s_tnew;
  // boundary values of the next step, one class per thread (step-function
  // lookup, HC/flucCal_2ndOrder_jh_improved_Kernel.cu:355-366, 441-446)
  if (tid < HB_MAX_CLASSES) {
    const int k = tid, id = in.bc_id[k];
    double hb = 0, wlb = 0, qxb = 0, qyb = 0;
    if (in.given_depth && id + 1 < in.depth_cols) {
      const int tl = timelevel(tnew, in.given_depth, in.depth_rows, in.depth_cols);
      hb = in.given_depth[(int64_t)tl * in.depth_cols + id + 1];
    }
    if (in.given_wl && id + 1 < in.wl_cols) {
      const int tl = timelevel(tnew, in.given_wl, in.wl_rows, in.wl_cols);
      wlb = in.given_wl[(int64_t)tl * in.wl_cols + id + 1];
    }
    if (in.given_q && 2 + 2 * id < in.q_cols) {
      const int tl = timelevel(tnew, in.given_q, in.q_rows, in.q_cols);
      qxb = in.given_q[(int64_t)tl * in.q_cols + 1 + 2 * id];
      qyb = in.given_q[(int64_t)tl * in.q_cols + 2 + 2 * id];
    }
    bct[ii].v[k][0] = hb;
    bct[ii].v[k][1] = wlb;
    bct[ii].v[k][2] = qxb;
    bct[ii].v[k][3] = qyb;
    ctrl->bc_vals[k][0] = (float)hb;
    ctrl->bc_vals[k][1] = (float)wlb;
    ctrl->bc_vals[k][2] = (float)qxb;
    ctrl->bc_vals[k][3] = (float)qyb;
  } else if (tid == 32) {
    ctrl->rain_rate = rain_rate_at(in, snap, ctrl, tnew);
  }
  if (in.rain_station) {
    __syncthreads();  // the rain cursor
    station_rates_at(in, ctrl, tnew, tid, NT);
  }
}

// Last tile of an instance: reduce the per-tile partials (FP64 volume and
// outflow, largest wave speed, any dry cell), account the step's volumes,
// flip the state buffer and advance the clock -- or, with external_dt,
// leave the clock to hb_fused_finish and publish the speed and dry flag.
// Sum of partials within a block, in a fixed order (lanes by a butterfly,
// then warps in index order): the result is in thread 0.
template <int NT>
__device__ TilePartial block_partial_sum(double v, double o, double sm, int dry,
                                         double (*red_d)[NT / 32], double *red_s, int *red_i) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  v = warp_sum(v);
  o = warp_sum(o);
  sm = warp_max(sm);
  dry = __any_sync(0xffffffffu, dry);
  if (lane == 0) {
    red_d[0][wid] = v;
    red_d[1][wid] = o;
    red_s[wid] = sm;
    red_i[wid] = dry;
  }
  __syncthreads();
  TilePartial p;
  p.volume = p.outflow = p.smax = 0.0;
  p.any_dry = 0;
  p.pad = 0;
  if (tid == 0) {
    for (int w = 0; w < NT / 32; w++) {
      p.volume += red_d[0][w];
      p.outflow += red_d[1][w];
      p.smax = fmax(p.smax, red_s[w]);
      p.any_dry |= red_i[w];
    }
  }
  return p;
}

// The instance's step is complete: reduce its `np` partials (per tile, or
// per group of tiles), account the step's volumes, flip the state buffer
// and advance the clock -- or, with external_dt, leave the clock to
// hb_fused_finish and publish the speed and dry flag.  The control block is
// copied to shared memory first (one load per thread) so that the clock
// logic does not wait on a chain of dependent global loads.
template <typename T, int NT>
__device__ void finalize_instance(const hb_instance &in, int ii, const TilePartial *parts,
                                  int np, BcTable *bct, double (*red_d)[NT / 32], double *red_s,
                                  int *red_i) {
  static_assert(sizeof(hb_ctrl) % 8 == 0 && sizeof(hb_ctrl) / 8 <= NT, "control block copy");
  const int tid = threadIdx.x;
  hb_ctrl *ctrl = in.ctrl;
  __shared__ hb_ctrl s_snap;
  __threadfence();
  if (tid < (int)(sizeof(hb_ctrl) / 8))
    reinterpret_cast<unsigned long long *>(&s_snap)[tid] =
        __ldcg(reinterpret_cast<const unsigned long long *>(ctrl) + tid);
  double v = 0, o = 0, sm = 0;
  int dry = 0;
  for (int k = tid; k < np; k += NT) {
    const TilePartial *pp = parts + k;
    v += __ldcg(&pp->volume);
    o += __ldcg(&pp->outflow);
    sm = fmax(sm, __ldcg(&pp->smax));
    dry |= __ldcg(&pp->any_dry);
  }
  const TilePartial P = block_partial_sum<NT>(v, o, sm, dry, red_d, red_s, red_i);
  __shared__ double s_sm;
  __shared__ int s_dry, s_ext;
  if (tid == 0) {
    const hb_ctrl &c = s_snap;
    const double V = P.volume, O = P.outflow, SM = P.smax;
    const int D = P.any_dry;
    const double dtn = c.dt, dxd = in.dx;
    if (!isfinite(V)) atomicOr(&ctrl->status, 4);  // a NaN / inf depth somewhere in the raster
    ctrl->volume = V * dxd * dxd;
    ctrl->outflow_volume = c.outflow_volume + O * dtn * dxd;
    if (in.rain_station) {
      double rv = 0.0;
      for (int k = 0; k < in.n_stations; k++) rv += in.station_rate[k] * in.station_cells[k];
      ctrl->rain_volume = c.rain_volume + rv * dtn * dxd * dxd;
    } else {
      ctrl->rain_volume = c.rain_volume + c.rain_rate * dtn * dxd * dxd * (double)in.n_valid;
    }
    ctrl->cur = 1 - c.cur;
    s_ext = c.external_dt;
    if (s_ext) {
      ctrl->ext[0] = SM;
      ctrl->ext[1] = D ? 1.0 : 0.0;
    }
    s_sm = SM;
    s_dry = D;
  }
  __syncthreads();
  if (!s_ext) advance_clock<T, NT>(in, ii, bct, s_sm, s_dry, &s_snap);
  if (tid == 0) ctrl->tiles_done = 0u;
}

// The last tile of a group to finish: sum the group's `n` tile partials
// (one per thread), store the group sum and count the group; the
// instance's last group finalizes the step from the group sums.
template <typename T, int NT>
__device__ void close_group(const hb_instance &in, int ii, const TilePartial *tiles, int n,
                            TilePartial *gparts, unsigned *gcount, int gi, int gbase, int ng,
                            BcTable *bct, double (*red_d)[NT / 32], double *red_s, int *red_i,
                            int *flag) {
  static_assert(kGroupTiles <= NT, "one tile partial per thread");
  const int tid = threadIdx.x;
  __threadfence();
  double v = 0, o = 0, sm = 0;
  int dry = 0;
  if (tid < n) {
    const TilePartial *pp = tiles + tid;
    v = __ldcg(&pp->volume);
    o = __ldcg(&pp->outflow);
    sm = __ldcg(&pp->smax);
    dry = __ldcg(&pp->any_dry);
  }
  const TilePartial P = block_partial_sum<NT>(v, o, sm, dry, red_d, red_s, red_i);
  if (tid == 0) {
    gparts[gi] = P;
    gcount[gi] = 0u;  // every tile of the group has counted: ready for the next step
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> done(in.ctrl->tiles_done);
    *flag = (done.fetch_add(1u, cuda::memory_order_acq_rel) == (unsigned)(ng - 1));
  }
  __syncthreads();
  if (*flag) finalize_instance<T, NT>(in, ii, gparts + gbase, ng, bct, red_d, red_s, red_i);
}

// hb_fused_finish: one block per instance advances the clock from the
// speed / dry flag reduced over all strips, ext = [n_instances][2].
template <typename T>
__global__ void __launch_bounds__(kNT)
finish_kernel(const hb_instance *__restrict__ insts, BcTable *__restrict__ bct,
              const double *__restrict__ ext, int n_instances) {
  const hb_instance &in = insts[blockIdx.x];
  if (in.ctrl->halted) return;
  double sm, dry;
  if (ext) {
    sm = ext[2 * blockIdx.x];
    dry = ext[2 * blockIdx.x + 1];
  } else {
    // the batch's instances are the strips of one catchment: the maximum of
    // what every instance published (order-independent)
    sm = 0.0;
    dry = 0.0;
    for (int k = 0; k < n_instances; k++) {
      sm = fmax(sm, __ldcg(&insts[k].ctrl->ext[0]));
      dry = fmax(dry, __ldcg(&insts[k].ctrl->ext[1]));
    }
  }
  advance_clock<T, kNT>(in, blockIdx.x, bct, sm, dry != 0.0 ? 1 : 0, in.ctrl);
}

// Workspace layout (each part 256-byte aligned): [n_tiles] TilePartial,
// [n_groups] TilePartial (sums of groups of kGroupTiles tiles), [n_groups]
// unsigned group counters, [n_tiles] int32 tile order (rows kernel: general
// tiles, then all-valid tiles), [2] int32 counts of the two, [n_tiles] uint8
// all-valid flags, 64-wide tiles only: [n_tiles] TileEntry in the order's
// order, then [n_instances] BcTable, then [n_instances][kMapsPerInstance]
// CUtensorMap.  Instance i's groups start at tile_begin / kGroupTiles + i,
// which never overlaps instance i + 1's.
inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
inline size_t ws_partials_bytes(int n_tiles) { return align256((size_t)n_tiles * sizeof(TilePartial)); }
inline int ws_n_groups(const hb_fused_batch *b) {
  return b->n_tiles / kGroupTiles + b->n_instances + 1;
}
inline size_t ws_gcount_offset(const hb_fused_batch *b) {
  return ws_partials_bytes(b->n_tiles) + align256((size_t)ws_n_groups(b) * sizeof(TilePartial));
}
inline size_t ws_order_offset(const hb_fused_batch *b) {
  return ws_gcount_offset(b) + align256((size_t)ws_n_groups(b) * sizeof(unsigned));
}
inline size_t ws_counts_offset(const hb_fused_batch *b) {
  return ws_order_offset(b) + align256((size_t)b->n_tiles * sizeof(int32_t));
}
inline size_t ws_flags_offset(const hb_fused_batch *b) { return ws_counts_offset(b) + 256; }
// What a tile of the two-cells-per-lane step needs before it can issue its
// tile loads, in one 16-byte record: the tile (~tile when it holds no valid
// cell), its instance and that instance's control block.
struct alignas(16) TileEntry {
  int32_t tile;
  int32_t inst;
  hb_ctrl *ctrl;
};
static_assert(sizeof(TileEntry) == 16, "one 16-byte load per tile");
inline size_t ws_entries_offset(const hb_fused_batch *b) {
  return ws_flags_offset(b) + align256((size_t)b->n_tiles);
}
inline size_t ws_entries_bytes(const hb_fused_batch *b) {
  return b->tile_x == 64 ? align256((size_t)b->n_tiles * sizeof(TileEntry)) : 0;
}
inline size_t ws_bct_offset(const hb_fused_batch *b) {
  return ws_entries_offset(b) + ws_entries_bytes(b);
}
inline size_t ws_maps_offset(const hb_fused_batch *b) {
  return align256(ws_bct_offset(b) + (size_t)b->n_instances * sizeof(BcTable));
}

// ---------------------------------------------------------------------------
// The step kernel
// ---------------------------------------------------------------------------
template <typename T, int TY, int TX, bool FAST>
__global__ void __launch_bounds__(kNT)
fused_step_kernel(const hb_instance *__restrict__ insts, const int32_t *__restrict__ tile_inst,
                  int n_tiles, TilePartial *__restrict__ partials, BcTable *__restrict__ bct) {
  using S = Smem<T, TY, TX>;
  constexpr int SW = S::SW, SH = S::SH;
  constexpr int V = 16 / sizeof(T);  // elements per 16-byte vector
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  const int tid = threadIdx.x;
  const T hs = T(kHSmall), g = T(kG);

  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int ii = tile_inst[tile];
    const hb_instance &in = insts[ii];
    hb_ctrl *ctrl = in.ctrl;
    if (ctrl->halted) continue;  // uniform across the CTA
    const int lt = tile - in.tile_begin;
    const int ty = lt / in.tiles_x, tx = lt - ty * in.tiles_x;
    const int y0 = ty * TY, x0 = tx * TX;  // raster origin of the tile
    const int cur = ctrl->cur;
    const double t = ctrl->t;
    const T dt = (T)ctrl->dt;
    const T dx = (T)in.dx;
    const T rain = (T)ctrl->rain_rate;
    const bool first = (t == 0.0);
    const T *hin = (const T *)in.h[cur];
    const T *qxin = (const T *)in.qx[cur];
    const T *qyin = (const T *)in.qy[cur];
    const T *zin = (const T *)in.z;
    const int P = in.pitch;

    // --- boundary tables and datum differences
    if (tid < HB_MAX_CLASSES) {
      s.bctype[tid] = in.bc_type[tid];
      for (int q = 0; q < 4; q++) s.bc[tid][q] = bct[ii].v[tid][q];
    }
    T datum_tile = T(0);
    if (in.datum) {
      const int by = y0 / HB_DATUM_BLOCK, bx = x0 / HB_DATUM_BLOCK;
      datum_tile = (T)in.datum[by * in.datum_nx + bx];
      if (tid >= 32 && tid < 41) {
        const int k = tid - 32, dy = k / 3 - 1, dxb = k % 3 - 1;
        const int yy = min(max(by + dy, 0), in.datum_ny - 1);
        const int xx = min(max(bx + dxb, 0), in.datum_nx - 1);
        s.ddatum[k] = (T)in.datum[yy * in.datum_nx + xx] - datum_tile;
      }
    }

    // --- stage the tile + halo (16-byte vector loads, all aligned)
    {
      constexpr int VPR = SW / V;  // vectors per staged row
      const size_t base = (size_t)y0 * P + x0;  // storage (y0, x0) = raster (y0-2, x0-4)
      for (int k = tid; k < SH * VPR; k += kNT) {
        const int r = k / VPR, cv = k - r * VPR;
        const size_t off = base + (size_t)r * P + cv * V;
        const int so = r * SW + cv * V;
        *reinterpret_cast<uint4 *>(&s.h[so]) = __ldg(reinterpret_cast<const uint4 *>(hin + off));
        *reinterpret_cast<uint4 *>(&s.qx[so]) = __ldg(reinterpret_cast<const uint4 *>(qxin + off));
        *reinterpret_cast<uint4 *>(&s.qy[so]) = __ldg(reinterpret_cast<const uint4 *>(qyin + off));
        *reinterpret_cast<uint4 *>(&s.z[so]) = __ldg(reinterpret_cast<const uint4 *>(zin + off));
      }
      constexpr int WPR = SW / 4;  // 32-bit words of codes per row
      const size_t cbase = (size_t)y0 * in.code_pitch + (x0 + HB_CODE_PAD_X - HB_PAD_X);
      for (int k = tid; k < SH * WPR; k += kNT) {
        const int r = k / WPR, cw = k - r * WPR;
        *reinterpret_cast<uint32_t *>(&s.code[r * SW + cw * 4]) =
            __ldg(reinterpret_cast<const uint32_t *>(in.code + cbase + (size_t)r * in.code_pitch) + cw);
      }
    }
    __syncthreads();
    if (in.datum) {
      // halo cells of neighbouring 64x64 datum blocks move into this tile's frame
      const int by0 = (y0 / HB_DATUM_BLOCK) * HB_DATUM_BLOCK;
      const int bx0 = (x0 / HB_DATUM_BLOCK) * HB_DATUM_BLOCK;
      for (int k = tid; k < SH * SW; k += kNT) {
        const int r = k / SW, c = k - r * SW;
        const int ry = y0 - 2 + r, rx = x0 - 4 + c;
        const int dyb = ry < by0 ? 0 : (ry >= by0 + HB_DATUM_BLOCK ? 2 : 1);
        const int dxb = rx < bx0 ? 0 : (rx >= bx0 + HB_DATUM_BLOCK ? 2 : 1);
        if (dyb != 1 || dxb != 1) s.z[k] += s.ddatum[dyb * 3 + dxb];
      }
      __syncthreads();
    }

    // --- faces
    for (int f = tid; f < S::NXF + S::NYF; f += kNT) {
      FaceOut<T> o{T(0), T(0), T(0), T(0), T(0)};
      if (f < S::NXF) {
        const int fi = f / (TX + 1), fj = f - fi * (TX + 1);
        // face between tile cells (fi, fj-1) = A and (fi, fj) = B
        const int ka = (fi + 2) * SW + (fj + 3);
        const int kb = ka + 1;
        const bool va = is_valid(s.code[ka]), vb = is_valid(s.code[kb]);
        if (va && vb) {
          o = interior_face<T, FAST, 0>(s, ka, kb, ka - 1, kb + 1);
        } else if (va) {
          boundary_face<T, FAST>(s, ka, T(1), T(0), datum_tile, o.fh, o.fx, o.fy, o.sa);
        } else if (vb) {
          T fh, fx, fy, sc;
          boundary_face<T, FAST>(s, kb, T(-1), T(0), datum_tile, fh, fx, fy, sc);
          o.fh = -fh; o.fx = -fx; o.fy = -fy; o.sb = sc;
        }
        s.xf[0][f] = o.fh; s.xf[1][f] = o.fx; s.xf[2][f] = o.fy;
        s.xf[3][f] = o.sa; s.xf[4][f] = o.sb;
      } else {
        const int q = f - S::NXF;
        const int fi = q / TX, fj = q - fi * TX;
        // face between tile cells (fi, fj) = A (south) and (fi-1, fj) = B (north)
        const int ka = (fi + 2) * SW + (fj + 4);
        const int kb = ka - SW;
        const bool va = is_valid(s.code[ka]), vb = is_valid(s.code[kb]);
        if (va && vb) {
          o = interior_face<T, FAST, 1>(s, ka, kb, ka + SW, kb - SW);
        } else if (va) {
          boundary_face<T, FAST>(s, ka, T(0), T(1), datum_tile, o.fh, o.fx, o.fy, o.sa);
        } else if (vb) {
          T fh, fx, fy, sc;
          boundary_face<T, FAST>(s, kb, T(0), T(-1), datum_tile, fh, fx, fy, sc);
          o.fh = -fh; o.fx = -fx; o.fy = -fy; o.sb = sc;
        }
        s.yf[0][q] = o.fh; s.yf[1][q] = o.fx; s.yf[2][q] = o.fy;
        s.yf[3][q] = o.sa; s.yf[4][q] = o.sb;
      }
    }
    __syncthreads();

    // --- cells: gather, rain, friction + update, h_max, CFL, volume
    double vol = 0.0, outf = 0.0;
    double smax = 0.0;
    int any_dry = 0;
    T *hout = (T *)in.h[1 - cur];
    T *qxout = (T *)in.qx[1 - cur];
    T *qyout = (T *)in.qy[1 - cur];
    T *hmax = (T *)in.h_max;
    for (int k = tid; k < TY * TX; k += kNT) {
      const int i = k / TX, j = k - i * TX;
      const int ry = y0 + i, rx = x0 + j;
      const int kc = (i + 2) * SW + (j + 4);
      const uint8_t code = s.code[kc];
      if (!is_valid(code) || ry >= in.rows || rx >= in.cols) continue;
      const T hc = s.h[kc];
      // fluxMask activity (HC/fluxMaskGenerator_Kernel.cu:19-42)
      bool active = first || hc > hs;
      if (!active) {
        const int kn[4] = {kc + 1, kc - SW, kc - 1, kc + SW};
        const int ny[4] = {ry, ry - 1, ry, ry + 1};
        const int nx[4] = {rx + 1, rx, rx - 1, rx};
#pragma unroll
        for (int d = 0; d < 4; d++) {
          const bool is_bug = (ny[d] == in.bug_y && nx[d] == in.bug_x);
          if (is_valid(s.code[kn[d]]) && !is_bug && s.h[kn[d]] > hs) active = true;
        }
      }
      T hu = T(0), qxu = T(0), qyu = T(0);
      if (active) {
        const int fe = i * (TX + 1) + (j + 1), fw = i * (TX + 1) + j;
        const int fn = i * TX + j, fs = (i + 1) * TX + j;
        const bool bE = !is_valid(s.code[kc + 1]), bW = !is_valid(s.code[kc - 1]);
        const bool bN = !is_valid(s.code[kc - SW]), bS = !is_valid(s.code[kc + SW]);
        if constexpr (FAST) {
          const T r = dt / dx;
          const T Fh = (s.xf[0][fw] + s.yf[0][fs]) - (s.xf[0][fe] + s.yf[0][fn]);
          const T Fx = (s.xf[1][fw] + s.yf[1][fs]) - (s.xf[1][fe] + s.yf[1][fn]);
          const T Fy = (s.xf[2][fw] + s.yf[2][fs]) - (s.xf[2][fe] + s.yf[2][fn]);
          hu = Fh * r;
          qxu = (Fx - s.xf[3][fe] + s.xf[4][fw]) * r;
          qyu = (Fy - s.yf[3][fn] + s.yf[4][fs]) * r;
        } else {
          // E (this cell is A of x-face fe)
          hu -= (s.xf[0][fe] / dx) * dt;
          qxu -= (s.xf[1][fe] / dx) * dt;
          qyu -= (s.xf[2][fe] / dx) * dt;
          qxu -= (s.xf[3][fe] / dx) * dt;
          // N (A of y-face fn)
          hu -= (s.yf[0][fn] / dx) * dt;
          qxu -= (s.yf[1][fn] / dx) * dt;
          qyu -= (s.yf[2][fn] / dx) * dt;
          qyu -= (s.yf[3][fn] / dx) * dt;
          // W (B of x-face fw): flux from this side is the negation
          hu -= (-s.xf[0][fw] / dx) * dt;
          qxu -= (-s.xf[1][fw] / dx) * dt;
          qyu -= (-s.xf[2][fw] / dx) * dt;
          qxu -= (-s.xf[4][fw] / dx) * dt;
          // S (B of y-face fs)
          hu -= (-s.yf[0][fs] / dx) * dt;
          qxu -= (-s.yf[1][fs] / dx) * dt;
          qyu -= (-s.yf[2][fs] / dx) * dt;
          qyu -= (-s.yf[4][fs] / dx) * dt;
        }
        if (bE | bW | bN | bS) {
          double o = 0.0;
          if (bE) o += (double)s.xf[0][fe];
          if (bN) o += (double)s.yf[0][fn];
          if (bW) o -= (double)s.xf[0][fw];
          if (bS) o -= (double)s.yf[0][fs];
          outf += o;
        }
      }
      // rain (HP/SWE_CUDA.py:549 / HC/stationPrecipitation_Kernel.cu:27)
      hu += rain * dt;
      // implicit friction + update (HC/friction_implicit_andUpdate_jh_Kernel.cu:22-146)
      const size_t go = (size_t)(ry + HB_PAD_Y) * P + (rx + HB_PAD_X);
      T h = hc + hu;
      T qx = s.qx[kc], qy = s.qy[kc];
      T sgh = T(0);  // sqrt(g h) in single precision, shared with the CFL speed
      if (h < hs) {
        qx = T(0);
        qy = T(0);
      } else {
        const T n = (T)in.manning[code & 15];
        qx += qxu;
        qy += qyu;
        // the reference takes this square root in single precision
        // (HC/timeControl_Kernel.cu:188); FAST allows the approximate one
        sgh = FAST ? (T)sqrtf((float)(g * h)) : (T)__fsqrt_rn((float)(g * h));
        if constexpr (FAST) {
          if (n > T(0)) {
            const T ih = T(1) / h;
            const T q_norm = sqrtf(qx * qx + qy * qy);
            // a = dt * C_f / h^2 with C_f = g n^2 h^(-1/3)
            const T a = dt * g * n * n * exp2f(-__log2f(h) * (T(1) / T(3))) * ih * ih;
            // (1 - sqrt(1 + 4 a |q|)) / (-2 a |q| / q_c) = q_c * 2 / (1 + sqrt(1 + 4 a |q|))
            const T fct = T(2) / (T(1) + sqrtf(T(1) + T(4) * a * q_norm));
            const T lim = T(5) * h * sgh;
            if (fabsf(qx) > T(1.0e-10)) {
              const T temp = qx * fct;
              if (fabsf(temp) > lim) {
                qx = T(2) * temp - qx;
                if (qx * temp <= T(0)) qx = T(0);
              } else {
                qx = temp;
              }
            }
            if (fabsf(qy) > T(1.0e-10)) {
              const T temp = qy * fct;
              if (fabsf(temp) > lim) {
                qy = T(2) * temp - qy;
                if (qy * temp <= T(0)) qy = T(0);
              } else {
                qy = temp;
              }
            }
          }
        } else {
          const T C_f = g * n * n * pow(h, T(-1.0 / 3.0));
          const T q_norm = sqrt(qx * qx + qy * qy);
          if (n > T(0)) {
            if (fabs(qx) > T(1.0e-10)) {
              T temp = (T(1) - sqrt(T(1) + (T(4) * dt * C_f) / (h * h) * q_norm)) /
                       (T(-2) * dt * C_f / (h * h) * (q_norm / qx));
              if (fabs(temp) > T(5) * h * sqrt(h * g)) {
                qx = T(2) * temp - qx;
                if (qx * temp <= T(0)) qx = T(0);
              } else {
                qx = temp;
              }
            }
            if (fabs(qy) > T(1.0e-10)) {
              T temp = (T(1) - sqrt(T(1) + (T(4) * dt * C_f) / (h * h) * q_norm)) /
                       (T(-2) * dt * C_f / (h * h) * (q_norm / qy));
              if (fabs(temp) > T(5) * h * sqrt(h * g)) {
                qy = T(2) * temp - qy;
                if (qy * temp <= T(0)) qy = T(0);
              } else {
                qy = temp;
              }
            }
          }
        }
      }
      hout[go] = h;
      qxout[go] = qx;
      qyout[go] = qy;
      // timeControl: h_max and the CFL speed (HC/timeControl_Kernel.cu:182-189)
      const T hm = hmax[go];
      hmax[go] = fmax(h, hm);
      if (h > hs) {
        const T sp = sgh + fmax(fabs(qx), fabs(qy)) / h;
        smax = fmax(smax, (double)sp);
      } else {
        any_dry = 1;
      }
      vol += (double)h;
    }

    // --- tile partials
    vol = warp_sum(vol);
    outf = warp_sum(outf);
    smax = warp_max(smax);
    any_dry = __any_sync(0xffffffffu, any_dry);
    const int lane = tid & 31, wid = tid >> 5;
    if (lane == 0) {
      s.red_d[0][wid] = vol;
      s.red_d[1][wid] = outf;
      s.red_s[wid] = smax;
      s.red_i[wid] = any_dry;
    }
    __syncthreads();
    if (tid == 0) {
      TilePartial p;
      p.volume = 0;
      p.outflow = 0;
      p.smax = 0;
      p.any_dry = 0;
      p.pad = 0;
      for (int w = 0; w < kNT / 32; w++) {
        p.volume += s.red_d[0][w];
        p.outflow += s.red_d[1][w];
        p.smax = fmax(p.smax, s.red_s[w]);
        p.any_dry |= s.red_i[w];
      }
      partials[tile] = p;
      const unsigned n_inst_tiles = (unsigned)(in.tiles_x * in.tiles_y);
      // release: this tile's partial is visible before the count moves
      cuda::atomic_ref<unsigned, cuda::thread_scope_device> done(ctrl->tiles_done);
      s.last = (done.fetch_add(1u, cuda::memory_order_acq_rel) == n_inst_tiles - 1);
    }
    __syncthreads();

    if (s.last)
      finalize_instance<T, kNT>(in, ii, partials + in.tile_begin, in.tiles_x * in.tiles_y, bct,
                                s.red_d, s.red_s, s.red_i);
    __syncthreads();
  }
}


// ===========================================================================
// Row-walking kernel over TMA-staged tiles.
//
// A CTA of 4 warps owns a tile of 32 columns x TY rows.  One elected thread
// stages h, qx, qy, z (tile + 2-cell halo, 4 columns each side), the tile's
// h_max and the cell codes into shared memory with 2-D TMA loads completing
// on an mbarrier.  Each warp then walks TY/4 consecutive rows, lane j owning
// column j:
//  * per-cell MUSCL slopes are formed once (x from the row's neighbours, y
//    from a sliding window of the column's rows held in registers) and shared
//    by the cell's two faces along that axis;
//  * the face to the south is evaluated in registers and reused as the next
//    row's north face; the face to the west is evaluated by each lane and
//    handed to the west neighbour as its east face by a warp shuffle;
//  * the cell update (gather, rain, friction, h_max, CFL speed, volume) runs
//    on the same registers and writes the new state with coalesced stores.
// Every face is still evaluated once.
// ===========================================================================
constexpr int kRowsNW = 4;             // warps per CTA
constexpr int kRowsNT = 32 * kRowsNW;  // threads per CTA
constexpr int kTW = 32;                // tile width (one warp)
constexpr int kSWF = kTW + 8;          // staged field row: cols -4..35
constexpr int kSWC = kTW + 32;         // staged code row: cols -16..47
constexpr int kMapsPerInstance = 9;    // h0 h1 qx0 qx1 qy0 qy1 z h_max code

template <typename T, int TY>
struct RowsSmem {
  static constexpr int SH = TY + 4;
  static constexpr int R = TY / kRowsNW;
  T f[4][SH * kSWF];          // h, qx, qy, z
  T hmax[TY * kTW];           // h_max of the tile's cells
  uint8_t code[SH * kSWC];
  alignas(8) unsigned long long bar;
  T xe[TY][4];                // face between cols 31 | 32: fh, fx, fy, sa
  T sxw[TY][4];               // x-slope of col -1: h, z, qx, qy
  double bc[HB_MAX_CLASSES][4];
  int bctype[HB_MAX_CLASSES];
  T manning[HB_MAX_ZONES];
  T ddatum[9];
  double red_d[2][kRowsNW];
  double red_s[kRowsNW];
  int red_i[kRowsNW];
  int last;
  int last2;
  static constexpr unsigned kTxBytes =
      (unsigned)(4 * SH * kSWF * sizeof(T) + TY * kTW * sizeof(T) + SH * kSWC);
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// Bounded wait: false if the phase did not complete within `budget` cycles.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned phase,
                                          long long budget) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, phase)) {
    if (clock64() - t0 > budget) return false;
  }
  return true;
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

template <typename T>
struct Slope {
  T h, z, qx, qy;
};

// minmod slope of cell c between its minus-side neighbour m and plus-side
// neighbour p; a no-data neighbour is replaced by c itself, as the reference
// does with a missing neighbour id (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:416-428).
// The 1st-order scheme uses only the bed's slope
// (HC/fluxCal_jh_modified_surface_Kernel.cu:577-610); its other fields are 0.
template <int ORDER = 2, typename T>
__device__ __forceinline__ Slope<T> slope_of(const Cell<T> &c, const Cell<T> &m, bool vm,
                                             const Cell<T> &p, bool vp) {
  const Cell<T> &mm = vm ? m : c;
  const Cell<T> &pp = vp ? p : c;
  Slope<T> s{T(0), T(0), T(0), T(0)};
  s.z = minmod(c.z - mm.z, pp.z - c.z);
  if constexpr (ORDER == 2) {
    s.h = minmod(c.h - mm.h, pp.h - c.h);
    s.qx = minmod(c.qx - mm.qx, pp.qx - c.qx);
    s.qy = minmod(c.qy - mm.qy, pp.qy - c.qy);
  }
  return s;
}

// Edge state of c on its plus side (sign = +1) or minus side (sign = -1).
template <typename T>
__device__ __forceinline__ Cell<T> edge_of(const Cell<T> &c, const Slope<T> &s, T sign) {
  Cell<T> e;
  e.h = c.h + T(0.5) * (sign * s.h);
  e.z = c.z + T(0.5) * (sign * s.z);
  e.wl = c.wl;
  if (c.h < T(kHSmall)) {
    e.qx = T(0);
    e.qy = T(0);
  } else {
    e.qx = c.qx + T(0.5) * (sign * s.qx);
    e.qy = c.qy + T(0.5) * (sign * s.qy);
  }
  return e;
}

// Face between valid cells A (west/south) and B (east/north) from A's side,
// from the cells and their MUSCL slopes along DIR (0: normal +x, 1: +y).
// ORDER 2: MUSCL edge states and the 2nd-order hydrostatic step
// (HC/flucCal_2ndOrder_jh_improved_Kernel.cu:43-107, 410-485); ORDER 1:
// piecewise-constant states, only the bed gets half its minmod slope, on a
// side whose neighbour across the face is wet, and the 1st-order hydrostatic
// step (HC/fluxCal_jh_modified_surface_Kernel.cu:96-139, 577-610).
// FAST (FP32) evaluates the face with bed elevations measured from A's bed:
// every operation of the scheme is invariant under a common shift of z, and
// in that frame eta = h + z is rounded at the scale of the local relief
// instead of the absolute elevation.
template <typename T, bool FAST, int DIR, int ORDER = 2>
__device__ __forceinline__ FaceOut<T> face_edges(Cell<T> A, Cell<T> B, const Slope<T> &sA,
                                                 const Slope<T> &sB) {
  const T hs = T(kHSmall), g = T(kG);
  FaceOut<T> o{T(0), T(0), T(0), T(0), T(0)};
  if (A.h < hs && B.h < hs) return o;
  if constexpr (FAST) {
    const T zref = A.z;
    A.z = T(0);
    B.z = B.z - zref;
    A.wl = A.h;
    B.wl = B.z + B.h;
  }
  Cell<T> eL, eR;
  if constexpr (ORDER == 1) {
    eL = A;
    eR = B;
    if (B.h > hs) eL.z = A.z + T(0.5) * sA.z;
    if (A.h > hs) eR.z = B.z + T(0.5) * (-sB.z);
  } else {
    eL = edge_of(A, sA, T(1));
    eR = edge_of(B, sB, T(-1));
  }
  T ux_l, uy_l, ux_r, uy_r;
  if constexpr (FAST && ORDER == 1) {
    // 1st order: the edge states are the cells themselves, so a row's two
    // faces share these products; rounded on their own (no contraction into
    // a later add), they come out the same in every build of the kernel
    const T il = eL.h < hs ? T(0) : T(1) / eL.h;
    const T ir = eR.h < hs ? T(0) : T(1) / eR.h;
    ux_l = __fmul_rn(eL.qx, il); uy_l = __fmul_rn(eL.qy, il);
    ux_r = __fmul_rn(eR.qx, ir); uy_r = __fmul_rn(eR.qy, ir);
  } else if constexpr (FAST) {
    const T il = eL.h < hs ? T(0) : T(1) / eL.h;
    const T ir = eR.h < hs ? T(0) : T(1) / eR.h;
    ux_l = eL.qx * il; uy_l = eL.qy * il;
    ux_r = eR.qx * ir; uy_r = eR.qy * ir;
  } else {
    ux_l = eL.h < hs ? T(0) : eL.qx / eL.h;
    uy_l = eL.h < hs ? T(0) : eL.qy / eL.h;
    ux_r = eR.h < hs ? T(0) : eR.qx / eR.h;
    uy_r = eR.h < hs ? T(0) : eR.qy / eR.h;
  }
  if constexpr (ORDER == 1)
    hydro1(A.h, A.z, B.h, B.z, eL, eR);
  else
    hydro2(A.wl, B.wl, eL, eR);
  T Fh, Fn, Ft;
  if (DIR == 0) {
    if (hllc<T, FAST>(eL.h, eR.h, ux_l, ux_r, uy_l, uy_r, Fh, Fn, Ft)) {
      o.fh = Fh; o.fx = Fn; o.fy = Ft;
    }
  } else {
    if (hllc<T, FAST>(eL.h, eR.h, uy_l, uy_r, -ux_l, -ux_r, Fh, Fn, Ft)) {
      o.fh = Fh; o.fx = -Ft; o.fy = Fn;
    }
  }
  o.sa = T(0.5) * g * (A.h + eL.h) * (eL.z - A.z);
  o.sb = T(0.5) * g * (B.h + eR.h) * (eR.z - B.z);
  return o;
}

// Boundary face of valid cell C with outward normal (n0, n1): ghost from
// C's class.  Flux from C's side and C's bed-slope term.
template <typename T, bool FAST, int ORDER = 2>
__device__ __noinline__ void ghost_face(const Cell<T> C, int cls, int type, const double *bcv,
                                        T n0, T n1, T datum, T *out) {
  const T hs = T(kHSmall), g = T(kG);
  out[0] = out[1] = out[2] = out[3] = T(0);
  Cell<T> G;
  const T hb = (T)bcv[0], wlb = (T)(bcv[1] - (double)datum);
  const T qxb = (T)bcv[2], qyb = (T)bcv[3];
  Cell<T> Cl = C;
  T wlbl = wlb;
  if constexpr (FAST) {  // bed measured from C's bed, as for interior faces
    wlbl = wlb - C.z;
    Cl.z = T(0);
    Cl.wl = Cl.h;
  }
  // FALL (type 9) is a ghost of the 1st-order scheme only
  if (!ghost(type, ORDER == 1, Cl, n0, n1, hb, wlbl, qxb, qyb, G)) return;
  (void)cls;
  if (Cl.h < hs && G.h < hs) return;
  Cell<T> eL = Cl, eR = G;
  T ux_l, uy_l, ux_r, uy_r;
  if constexpr (FAST) {
    const T il = eL.h < hs ? T(0) : T(1) / eL.h;
    const T ir = eR.h < hs ? T(0) : T(1) / eR.h;
    ux_l = eL.qx * il; uy_l = eL.qy * il;
    ux_r = eR.qx * ir; uy_r = eR.qy * ir;
  } else {
    ux_l = eL.h < hs ? T(0) : eL.qx / eL.h;
    uy_l = eL.h < hs ? T(0) : eL.qy / eL.h;
    ux_r = eR.h < hs ? T(0) : eR.qx / eR.h;
    uy_r = eR.h < hs ? T(0) : eR.qy / eR.h;
  }
  if constexpr (ORDER == 1)
    hydro1(Cl.h, Cl.z, G.h, G.z, eL, eR);
  else
    hydro2(Cl.wl, G.wl, eL, eR);
  const T u_L = ux_l * n0 + uy_l * n1, u_R = ux_r * n0 + uy_r * n1;
  const T v_L = -ux_l * n1 + uy_l * n0, v_R = -ux_r * n1 + uy_r * n0;
  T Fh, Fn, Ft;
  if (hllc<T, FAST>(eL.h, eR.h, u_L, u_R, v_L, v_R, Fh, Fn, Ft)) {
    out[0] = Fh;
    out[1] = Fn * n0 + Ft * (-n1);
    out[2] = Fn * n1 + Ft * n0;
  }
  out[3] = T(0.5) * g * (Cl.h + eL.h) * (eL.z - Cl.z);
}

template <typename T, int TY>
struct RowsView {
  const RowsSmem<T, TY> &s;
  __device__ __forceinline__ int fi(int i, int j) const { return (i + 2) * kSWF + (j + 4); }
  __device__ __forceinline__ Cell<T> cell(int i, int j) const {
    const int k = fi(i, j);
    Cell<T> c;
    c.h = s.f[0][k];
    c.qx = s.f[1][k];
    c.qy = s.f[2][k];
    c.z = s.f[3][k];
    c.wl = c.z + c.h;  // the reference stores wl = z + h after every update
    return c;
  }
  __device__ __forceinline__ uint8_t code(int i, int j) const {
    return s.code[(i + 2) * kSWC + (j + 16)];
  }
};

// Face between A (minus side) and B (plus side) along DIR, any validity.
// sA / sB: MUSCL slopes of A and B along DIR (used only when both are valid).
// ALLV: both cells are known to be valid (no ghost face can occur).
template <typename T, bool FAST, int DIR, int TY, bool ALLV = false, int ORDER = 2>
__device__ __forceinline__ FaceOut<T> face_any(const RowsSmem<T, TY> &s, const Cell<T> &A,
                                               uint8_t ca, const Cell<T> &B, uint8_t cb,
                                               const Slope<T> &sA, const Slope<T> &sB, T datum) {
  if constexpr (ALLV) return face_edges<T, FAST, DIR, ORDER>(A, B, sA, sB);
  const bool va = is_valid(ca), vb = is_valid(cb);
  if (va && vb) return face_edges<T, FAST, DIR, ORDER>(A, B, sA, sB);
  FaceOut<T> o{T(0), T(0), T(0), T(0), T(0)};
  const T n0 = DIR == 0 ? T(1) : T(0), n1 = DIR == 0 ? T(0) : T(1);
  T out[4];
  if (va) {
    const int cls = ca >> 4;
    ghost_face<T, FAST, ORDER>(A, cls, s.bctype[cls], s.bc[cls], n0, n1, datum, out);
    o.fh = out[0]; o.fx = out[1]; o.fy = out[2]; o.sa = out[3];
  } else if (vb) {
    const int cls = cb >> 4;
    ghost_face<T, FAST, ORDER>(B, cls, s.bctype[cls], s.bc[cls], -n0, -n1, datum, out);
    o.fh = -out[0]; o.fx = -out[1]; o.fy = -out[2]; o.sb = out[3];
  }
  return o;
}

// PATH 0: the general row loop, over the tiles that prepare classified as
// touching no-data cells or the cell-0 rule's cell; PATH 1: the all-valid row
// loop (every validity test a compile-time true), over the other tiles.  The
// two paths are separate kernels so that each gets its own register
// allocation (the general path's ghost faces and selects cost the all-valid
// tiles registers, spills and about 9 % of their time when they share one).
// order[0, counts[0]) are the general tiles, order[counts[0], counts[0] +
// counts[1]) the all-valid ones.
template <typename T, int TY, bool FAST, int MINB, bool SOURCES, int PATH, int ORDER>
__global__ void __launch_bounds__(kRowsNT, MINB)
rows_step_kernel(const hb_instance *__restrict__ insts, const int32_t *__restrict__ tile_inst,
                 const int32_t *__restrict__ order, const int32_t *__restrict__ counts,
                 TilePartial *__restrict__ partials, TilePartial *__restrict__ gparts,
                 unsigned *__restrict__ gcount, BcTable *__restrict__ bct,
                 const CUtensorMap *__restrict__ maps) {
  constexpr bool kAllValid = PATH == 1;
  using S = RowsSmem<T, TY>;
  constexpr int R = S::R;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S &s = *reinterpret_cast<S *>(smem_raw);
  const RowsView<T, TY> V{s};
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const T hs = T(kHSmall), g = T(kG);
  if (tid == 0) {
    mbar_init(&s.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned phase = 0;

  const int n_list = counts[PATH];
  const int32_t *list = order + (kAllValid ? counts[0] : 0);
  for (int k = blockIdx.x; k < n_list; k += gridDim.x) {
    const int tile = list[k];
    const int ii = tile_inst[tile];
    const hb_instance &in = insts[ii];
    hb_ctrl *ctrl = in.ctrl;
    if (ctrl->halted) continue;
    const int lt = tile - in.tile_begin;
    const int tyi = lt / in.tiles_x, txi = lt - tyi * in.tiles_x;
    const int y0 = tyi * TY, x0 = txi * kTW;
    const int cur = ctrl->cur;
    const double t = ctrl->t;
    const T dt = (T)ctrl->dt;
    const T dx = (T)in.dx;
    const T rain = (T)ctrl->rain_rate;
    const bool first = (t == 0.0);
    const int P = in.pitch;
    const CUtensorMap *m = maps + (size_t)ii * kMapsPerInstance;

    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(&s.bar, S::kTxBytes);
      tma_load_2d(s.f[0], m + 0 + cur, x0, y0, &s.bar);
      tma_load_2d(s.f[1], m + 2 + cur, x0, y0, &s.bar);
      tma_load_2d(s.f[2], m + 4 + cur, x0, y0, &s.bar);
      tma_load_2d(s.f[3], m + 6, x0, y0, &s.bar);
      tma_load_2d(s.hmax, m + 7, x0 + HB_PAD_X, y0 + HB_PAD_Y, &s.bar);
      tma_load_2d(s.code, m + 8, x0, y0, &s.bar);
    }
    if (tid < HB_MAX_CLASSES) {
      if constexpr (!kAllValid) {  // ghost faces only
        s.bctype[tid] = in.bc_type[tid];
        for (int q = 0; q < 4; q++) s.bc[tid][q] = bct[ii].v[tid][q];
      }
    } else if (tid >= 64 && tid < 64 + HB_MAX_ZONES) {
      s.manning[tid - 64] = (T)in.manning[tid - 64];
    }
    const int bug_y = in.bug_y, bug_x = in.bug_x;
    T datum_tile = T(0);
    if (in.datum) {
      const int by = y0 / HB_DATUM_BLOCK, bx = x0 / HB_DATUM_BLOCK;
      datum_tile = (T)in.datum[by * in.datum_nx + bx];
      if (tid >= 32 && tid < 41) {
        const int k = tid - 32, dyb = k / 3 - 1, dxb = k % 3 - 1;
        const int yy = min(max(by + dyb, 0), in.datum_ny - 1);
        const int xx = min(max(bx + dxb, 0), in.datum_nx - 1);
        s.ddatum[k] = (T)in.datum[yy * in.datum_nx + xx] - datum_tile;
      }
    }
    const bool arrived = mbar_wait(&s.bar, phase, 4000000000LL);
    if (__syncthreads_or(!arrived)) {
      // the tile's data did not arrive within the budget: flag it, wait once
      // more (bounded) for the copy in flight, and leave without touching the
      // state; the host sees ctrl->status
      if (tid == 0) atomicOr(&ctrl->status, 2);
      mbar_wait(&s.bar, phase, 4000000000LL);
      return;
    }
    phase ^= 1u;
    if (in.datum) {
      __syncthreads();  // ddatum visible
      const int by0 = (y0 / HB_DATUM_BLOCK) * HB_DATUM_BLOCK;
      const int bx0 = (x0 / HB_DATUM_BLOCK) * HB_DATUM_BLOCK;
      // only the halo sides that lie in another datum block
      const DatumHalo dh = datum_halo(y0, x0, by0, bx0, TY, kTW, kSWF, HB_DATUM_BLOCK);
      const int NH = dh.count();
      for (int k = tid; k < NH; k += kRowsNT) {
        int i, j;
        datum_halo_cell(dh, k, TY, kTW, kSWF, i, j);
        const int ry = y0 + i, rx = x0 + j;
        const int dyb = ry < by0 ? 0 : (ry >= by0 + HB_DATUM_BLOCK ? 2 : 1);
        const int dxb = rx < bx0 ? 0 : (rx >= bx0 + HB_DATUM_BLOCK ? 2 : 1);
        if (dyb != 1 || dxb != 1) s.f[3][V.fi(i, j)] += s.ddatum[dyb * 3 + dxb];
      }
    }
    __syncthreads();

    const int r0 = w * R;
    // --- tile edges, all lanes busy: warp 0 evaluates the faces between
    // columns 31 | 32 (the east faces of lane 31), warp 1 the x-slopes of
    // column -1 (needed by lane 0's west faces), for every row of the tile
    if (w == 0) {
      for (int i = lane; i < TY; i += 32) {
        const Cell<T> a = V.cell(i, 31), b = V.cell(i, 32);
        const uint8_t ca = V.code(i, 31), cb = V.code(i, 32);
        const Slope<T> sa = slope_of<ORDER>(a, V.cell(i, 30), is_valid(V.code(i, 30)), b, is_valid(cb));
        const Slope<T> sb = slope_of<ORDER>(b, a, is_valid(ca), V.cell(i, 33), is_valid(V.code(i, 33)));
        const FaceOut<T> f =
            face_any<T, FAST, 0, TY, kAllValid, ORDER>(s, a, ca, b, cb, sa, sb, datum_tile);
        s.xe[i][0] = f.fh;
        s.xe[i][1] = f.fx;
        s.xe[i][2] = f.fy;
        s.xe[i][3] = f.sa;
      }
    } else if (w == 1) {
      for (int i = lane; i < TY; i += 32) {
        const Cell<T> cm2 = V.cell(i, -2), cm1 = V.cell(i, -1), c0 = V.cell(i, 0);
        const Slope<T> sm1 = slope_of<ORDER>(cm1, cm2, is_valid(V.code(i, -2)), c0,
                                      is_valid(V.code(i, 0)));
        s.sxw[i][0] = sm1.h;
        s.sxw[i][1] = sm1.z;
        s.sxw[i][2] = sm1.qx;
        s.sxw[i][3] = sm1.qy;
      }
    }

    // per-thread partial sums over this warp's rows (<= 16 cells) in T; the
    // tile and instance reductions are FP64
    T vol_t = T(0), smax_t = T(0);
    double outf = 0.0;
    int any_dry = 0;
    auto rows = [&](auto allv_tag) {
      constexpr bool ALLV = decltype(allv_tag)::value;
      auto valid = [](uint8_t k) -> bool {
        if constexpr (ALLV) {
          (void)k;
          return true;
        } else {
          return is_valid(k);
        }
      };
      // --- column window: rows r0-2 .. r0+2
      const int j = lane;
      Cell<T> cN = V.cell(r0 - 1, j), cC = V.cell(r0, j), cS = V.cell(r0 + 1, j);
      uint8_t kN = V.code(r0 - 1, j), kC = V.code(r0, j), kS = V.code(r0 + 1, j);
      Slope<T> syC, syS;
      FaceOut<T> nf;
      {
        const Cell<T> cNN = V.cell(r0 - 2, j);
        const uint8_t kNN = V.code(r0 - 2, j);
        const Cell<T> cSS = V.cell(r0 + 2, j);
        const uint8_t kSS = V.code(r0 + 2, j);
        // y-slopes: minus side = south (row + 1), plus side = north (row - 1)
        const Slope<T> syN = slope_of<ORDER>(cN, cC, valid(kC), cNN, valid(kNN));
        syC = slope_of<ORDER>(cC, cS, valid(kS), cN, valid(kN));
        syS = slope_of<ORDER>(cS, cSS, valid(kSS), cC, valid(kC));
        // face between rows r0-1 (north) and r0 (south), from the south side
        nf = face_any<T, FAST, 1, TY, ALLV, ORDER>(s, cC, kC, cN, kN, syC, syN, datum_tile);
      }
      __syncthreads();  // tile-edge faces and slopes ready
      T *hout = (T *)in.h[1 - cur];
      T *qxout = (T *)in.qx[1 - cur];
      T *qyout = (T *)in.qy[1 - cur];
      T *hmaxg = (T *)in.h_max;
      const int rx = x0 + j;
      // read once per tile: the state stores below may alias the record
      // (instances without infiltration or station rain take the SOURCES = false
      // build, in which both branches vanish)
      const bool infil = SOURCES && in.cum != nullptr;
      const bool stations = SOURCES && in.rain_station != nullptr;
      // row strips: does this tile hold rows whose new state also goes to a
      // neighbour strip's halo rows?
      const bool fwd_tile = (y0 < HB_PAD_Y && in.halo_up[0] != nullptr) ||
                            (y0 + TY > in.rows - HB_PAD_Y && in.halo_down[0] != nullptr);

  #pragma unroll 1
      for (int i = r0; i < r0 + R; ++i) {
        const Cell<T> cW = V.cell(i, j - 1), cE = V.cell(i, j + 1);
        const uint8_t kW = V.code(i, j - 1), kE = V.code(i, j + 1);
        const bool vW = valid(kW), vE = valid(kE), vC = valid(kC);
        const Slope<T> sxC = slope_of<ORDER>(cC, cW, vW, cE, vE);
        Slope<T> sxW{T(0), T(0), T(0), T(0)};
        sxW.z = __shfl_up_sync(0xffffffffu, sxC.z, 1);
        if constexpr (ORDER == 2) {
          sxW.h = __shfl_up_sync(0xffffffffu, sxC.h, 1);
          sxW.qx = __shfl_up_sync(0xffffffffu, sxC.qx, 1);
          sxW.qy = __shfl_up_sync(0xffffffffu, sxC.qy, 1);
        }
        if (lane == 0) {
          sxW.z = s.sxw[i][1];
          if constexpr (ORDER == 2) {
            sxW.h = s.sxw[i][0];
            sxW.qx = s.sxw[i][2];
            sxW.qy = s.sxw[i][3];
          }
        }
        // west face (this cell is B) -> the west neighbour's east face
        const FaceOut<T> wf = face_any<T, FAST, 0, TY, ALLV, ORDER>(s, cW, kW, cC, kC, sxW, sxC, datum_tile);
        T ef_h = __shfl_down_sync(0xffffffffu, wf.fh, 1);
        T ef_x = __shfl_down_sync(0xffffffffu, wf.fx, 1);
        T ef_y = __shfl_down_sync(0xffffffffu, wf.fy, 1);
        T ef_a = __shfl_down_sync(0xffffffffu, wf.sa, 1);
        if (lane == 31) {
          ef_h = s.xe[i][0];
          ef_x = s.xe[i][1];
          ef_y = s.xe[i][2];
          ef_a = s.xe[i][3];
        }
        // south face (this cell is B, the row below is A)
        const FaceOut<T> sf = face_any<T, FAST, 1, TY, ALLV, ORDER>(s, cS, kS, cC, kC, syS, syC, datum_tile);
        const int ry = y0 + i;
        if (vC) {
          const T hc = cC.h;
          bool active = first || hc > hs;
          if (!active) {
            if constexpr (ALLV) {
              active = cE.h > hs || cN.h > hs || cW.h > hs || cS.h > hs;
            } else {
              const bool bugE = (ry == bug_y && rx + 1 == bug_x);
              const bool bugW = (ry == bug_y && rx - 1 == bug_x);
              const bool bugN = (ry - 1 == bug_y && rx == bug_x);
              const bool bugS = (ry + 1 == bug_y && rx == bug_x);
              active = (vE && !bugE && cE.h > hs) || (valid(kN) && !bugN && cN.h > hs) ||
                       (vW && !bugW && cW.h > hs) || (valid(kS) && !bugS && cS.h > hs);
            }
          }
          T hu = T(0), qxu = T(0), qyu = T(0);
          if (active) {
            if constexpr (FAST) {
              const T r = dt / dx;
              hu = ((wf.fh + sf.fh) - (ef_h + nf.fh)) * r;
              qxu = ((wf.fx + sf.fx) - (ef_x + nf.fx) - ef_a + wf.sb) * r;
              qyu = ((wf.fy + sf.fy) - (ef_y + nf.fy) - nf.sa + sf.sb) * r;
            } else {
              hu -= (ef_h / dx) * dt;
              qxu -= (ef_x / dx) * dt;
              qyu -= (ef_y / dx) * dt;
              qxu -= (ef_a / dx) * dt;
              hu -= (nf.fh / dx) * dt;
              qxu -= (nf.fx / dx) * dt;
              qyu -= (nf.fy / dx) * dt;
              qyu -= (nf.sa / dx) * dt;
              hu -= (-wf.fh / dx) * dt;
              qxu -= (-wf.fx / dx) * dt;
              qyu -= (-wf.fy / dx) * dt;
              qxu -= (-wf.sb / dx) * dt;
              hu -= (-sf.fh / dx) * dt;
              qxu -= (-sf.fx / dx) * dt;
              qyu -= (-sf.fy / dx) * dt;
              qyu -= (-sf.sb / dx) * dt;
            }
            const bool bE = !vE, bW = !vW, bN = !valid(kN), bS = !valid(kS);
            if (bE | bW | bN | bS) {
              double o = 0.0;
              if (bE) o += (double)ef_h;
              if (bN) o += (double)nf.fh;
              if (bW) o -= (double)wf.fh;
              if (bS) o -= (double)sf.fh;
              outf += o;
            }
          }
          if (stations) {
            // station rain (HC/stationPrecipitation_Kernel.cu:18-29), every valid cell
            const size_t gs = (size_t)(ry + HB_PAD_Y) * P + (rx + HB_PAD_X);
            hu += (T)in.station_rate[in.rain_station[gs]] * dt;
          } else {
            hu += rain * dt;
          }
          if (infil && active) {
            // Green-Ampt infiltration on the flux list, after rain
            // (HC/infiltrationCUDA_Kernel.cu:20-46; order HP/CatchFlood_main.py:164-170)
            T *cum = (T *)in.cum + (size_t)(ry + HB_PAD_Y) * P + (rx + HB_PAD_X);
            const int zc = kC & 15;
            const T K = (T)in.ks[zc], psi = (T)in.psi[zc], dth = (T)in.dtheta[zc];
            const T F0 = *cum;
            const T a = F0 + dt * K;
            const T F1 = T(0.5) * (a + sqrt(a * a + T(4) * dt * K * (psi + hc) * dth));
            const T dF = fmin(hc, F1 - F0);
            *cum = F0 + dF;
            hu -= dF;
          }
          T h = hc + hu;
          T qx = cC.qx, qy = cC.qy;
          T sgh = T(0);
          T ih = T(0);
          if (h < hs) {
            qx = T(0);
            qy = T(0);
          } else {
            const T n = s.manning[kC & 15];
            qx += qxu;
            qy += qyu;
            sgh = FAST ? (T)sqrtf((float)(g * h)) : (T)__fsqrt_rn((float)(g * h));
            if constexpr (FAST) {
              ih = T(1) / h;
              if (n > T(0)) {
                const T q_norm = sqrtf(qx * qx + qy * qy);
                const T a = dt * g * n * n * exp2f(-__log2f(h) * (T(1) / T(3))) * ih * ih;
                const T fct = T(2) / (T(1) + sqrtf(T(1) + T(4) * a * q_norm));
                const T lim = T(5) * h * sgh;
                if (fabsf(qx) > T(1.0e-10)) {
                  const T temp = qx * fct;
                  if (fabsf(temp) > lim) {
                    qx = T(2) * temp - qx;
                    if (qx * temp <= T(0)) qx = T(0);
                  } else {
                    qx = temp;
                  }
                }
                if (fabsf(qy) > T(1.0e-10)) {
                  const T temp = qy * fct;
                  if (fabsf(temp) > lim) {
                    qy = T(2) * temp - qy;
                    if (qy * temp <= T(0)) qy = T(0);
                  } else {
                    qy = temp;
                  }
                }
              }
            } else {
              const T C_f = g * n * n * pow(h, T(-1.0 / 3.0));
              const T q_norm = sqrt(qx * qx + qy * qy);
              if (n > T(0)) {
                if (fabs(qx) > T(1.0e-10)) {
                  T temp = (T(1) - sqrt(T(1) + (T(4) * dt * C_f) / (h * h) * q_norm)) /
                           (T(-2) * dt * C_f / (h * h) * (q_norm / qx));
                  if (fabs(temp) > T(5) * h * sqrt(h * g)) {
                    qx = T(2) * temp - qx;
                    if (qx * temp <= T(0)) qx = T(0);
                  } else {
                    qx = temp;
                  }
                }
                if (fabs(qy) > T(1.0e-10)) {
                  T temp = (T(1) - sqrt(T(1) + (T(4) * dt * C_f) / (h * h) * q_norm)) /
                           (T(-2) * dt * C_f / (h * h) * (q_norm / qy));
                  if (fabs(temp) > T(5) * h * sqrt(h * g)) {
                    qy = T(2) * temp - qy;
                    if (qy * temp <= T(0)) qy = T(0);
                  } else {
                    qy = temp;
                  }
                }
              }
            }
          }
          const size_t go = (size_t)(ry + HB_PAD_Y) * P + (rx + HB_PAD_X);
          hout[go] = h;
          qxout[go] = qx;
          qyout[go] = qy;
          if (fwd_tile) {
            // into the neighbour's halo row of the same output buffer (plain
            // stores; the neighbour's arrays may be on a peer GPU)
            const int ob = 1 - cur;
            auto fwd = [&](void *const *dst, int row) {
              const size_t gh = (size_t)row * P + (rx + HB_PAD_X);
              ((T *)dst[ob])[gh] = h;
              ((T *)dst[2 + ob])[gh] = qx;
              ((T *)dst[4 + ob])[gh] = qy;
            };
            if (ry < HB_PAD_Y && in.halo_up[0] != nullptr)
              fwd(in.halo_up, in.halo_up_rows + HB_PAD_Y + ry);
            if (ry >= in.rows - HB_PAD_Y && in.halo_down[0] != nullptr)
              fwd(in.halo_down, ry - in.rows + HB_PAD_Y);
            // the neighbour may be a peer GPU: order these stores system-wide
            // before this tile's partial, its group count and everything the
            // host orders after the step (the clock all_reduce)
            __threadfence_system();
          }
          hmaxg[go] = fmax(h, s.hmax[i * kTW + j]);
          if (h > hs) {
            // CFL speed (HC/timeControl_Kernel.cu:186-189)
            const T sp = FAST ? sgh + fmax(fabs(qx), fabs(qy)) * ih
                              : sgh + fmax(fabs(qx), fabs(qy)) / h;
            smax_t = fmax(smax_t, sp);
          } else {
            any_dry = 1;
          }
          vol_t += h;
        }
        // slide the column window down one row
        nf = sf;
        cN = cC; kN = kC;
        cC = cS; kC = kS;
        syC = syS;
        if (i + 1 < r0 + R) {
          cS = V.cell(i + 2, j);
          kS = V.code(i + 2, j);
          const Cell<T> cSS = V.cell(i + 3, j);
          const uint8_t kSS = V.code(i + 3, j);
          syS = slope_of<ORDER>(cS, cSS, valid(kSS), cC, valid(kC));
        }
      }

    };
    rows(BoolTag<kAllValid>{});

    // --- tile partials and the instance's last-tile finalize
    double vol = warp_sum((double)vol_t);
    // an all-valid tile has no boundary face, so no outflow to sum; the
    // maximum is exact in T
    if constexpr (!kAllValid) outf = warp_sum(outf);
    const double smax = (double)warp_max(smax_t);
    any_dry = __any_sync(0xffffffffu, any_dry);
    if (lane == 0) {
      s.red_d[0][w] = vol;
      s.red_d[1][w] = outf;
      s.red_s[w] = smax;
      s.red_i[w] = any_dry;
    }
    __syncthreads();
    const int n_inst_tiles = in.tiles_x * in.tiles_y;
    const int grp = lt / kGroupTiles;
    const int gsize = min(kGroupTiles, n_inst_tiles - grp * kGroupTiles);
    const int gbase = in.tile_begin / kGroupTiles + ii;
    if (tid == 0) {
      TilePartial p;
      p.volume = p.outflow = p.smax = 0.0;
      p.any_dry = 0;
      p.pad = 0;
      for (int q = 0; q < kRowsNW; q++) {
        p.volume += s.red_d[0][q];
        p.outflow += s.red_d[1][q];
        p.smax = fmax(p.smax, s.red_s[q]);
        p.any_dry |= s.red_i[q];
      }
      partials[tile] = p;
      // release: this tile's partial is visible before its group's count moves
      cuda::atomic_ref<unsigned, cuda::thread_scope_device> done(gcount[gbase + grp]);
      s.last = (done.fetch_add(1u, cuda::memory_order_acq_rel) == (unsigned)(gsize - 1));
    }
    __syncthreads();
    if (s.last)
      close_group<T, kRowsNT>(in, ii, partials + in.tile_begin + grp * kGroupTiles, gsize,
                              gparts, gcount, gbase + grp, gbase,
                              (n_inst_tiles + kGroupTiles - 1) / kGroupTiles, bct, s.red_d,
                              s.red_s, s.red_i, &s.last2);
    __syncthreads();
  }
}

// The FP32 2nd-order step with two cells per lane (64-wide tiles).
#include "hb_pairs.cuh"

// Prepare: rain rate and boundary values at t, counters; the volume at t is
// summed by prepare_volume_kernel, launched after this one.
template <typename T>
__global__ void __launch_bounds__(kNT)
prepare_kernel(const hb_instance *__restrict__ insts, BcTable *__restrict__ bct) {
  const hb_instance &in = insts[blockIdx.x];
  hb_ctrl *c = in.ctrl;
  if (threadIdx.x == 0) {
    c->volume = 0.0;
    c->volume0 = 0.0;
    c->tiles_done = 0u;
    c->rain_rate = rain_rate_at(in, c, c, c->t);
    bc_values_exact(in, c->t, &bct[blockIdx.x]);
    bc_values_at(in, c, c->t);
  }
  if (in.rain_station) {
    __syncthreads();  // the rain cursor
    station_rates_at(in, c, c->t, threadIdx.x, blockDim.x);
  }
}

// Volume of every instance at t: blockIdx.y is the instance, the x blocks
// share its cells; one FP64 atomic per block into volume and volume0.
template <typename T>
__global__ void __launch_bounds__(kNT)
prepare_volume_kernel(const hb_instance *__restrict__ insts) {
  const hb_instance &in = insts[blockIdx.y];
  hb_ctrl *c = in.ctrl;
  const T *h = (const T *)in.h[c->cur];
  const uint8_t *code = in.code;
  const int64_t n = (int64_t)in.rows * in.cols;
  double v = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / in.cols), cc = (int)(k - (int64_t)r * in.cols);
    const uint8_t cd = code[(size_t)(r + HB_PAD_Y) * in.code_pitch + cc + HB_CODE_PAD_X];
    if ((cd >> 4) != HB_NODATA_CLASS) v += (double)h[(size_t)(r + HB_PAD_Y) * in.pitch + cc + HB_PAD_X];
  }
  __shared__ double red[kNT / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double V = 0;
    for (int w = 0; w < kNT / 32; w++) V += red[w];
    if (V != 0.0) {
      V *= in.dx * in.dx;
      atomicAdd(&c->volume, V);
      atomicAdd(&c->volume0, V);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
// The dynamic shared-memory limit of a kernel, set once per device (the
// attribute belongs to the kernel on the current device).
PerDeviceOnce g_smem_attr;

int set_smem_attr(const void *fn, int bytes) {
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  return g_smem_attr.run(dev, fn, [&]() -> int {
    const cudaError_t a = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               bytes);
    if (a != cudaSuccess)
      return set_error(HB_ERR_CUDA, "fused step setup: %s", cudaGetErrorString(a));
    return (int)HB_OK;
  });
}

template <typename T, int TY, int TX, bool FAST = (sizeof(T) == 4)>
int launch_steps(const hb_fused_batch *b, int nsteps, cudaStream_t st) {
  using S = Smem<T, TY, TX>;
  const void *fn = reinterpret_cast<const void *>(fused_step_kernel<T, TY, TX, FAST>);
  int rc = set_smem_attr(fn, (int)sizeof(S));
  if (rc) return rc;
  int blocks_per_sm = 1;
  const cudaError_t oe =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, fused_step_kernel<T, TY, TX, FAST>,
                                                    kNT, sizeof(S));
  if (oe != cudaSuccess)
    return set_error(HB_ERR_CUDA, "fused step setup: %s", cudaGetErrorString(oe));
  if (blocks_per_sm < 1) blocks_per_sm = 1;
  int grid = b->grid_blocks > 0 ? b->grid_blocks : blocks_per_sm * num_sms();
  if (grid > b->n_tiles) grid = b->n_tiles;
  TilePartial *parts = reinterpret_cast<TilePartial *>(b->workspace);
  BcTable *bct = reinterpret_cast<BcTable *>((char *)b->workspace + ws_bct_offset(b));
  for (int k = 0; k < nsteps; k++) {
    fused_step_kernel<T, TY, TX, FAST><<<grid, kNT, sizeof(S), st>>>(
        b->instances, b->tile_instance, b->n_tiles, parts, bct);
  }
  return check_launch("hb_fused_step");
}

// ---------------------------------------------------------------------------
// Tile classification (at prepare): a tile is all-valid when every staged
// code of rows -2..TY+1, columns -4..35 is a valid cell and the cell-0 rule's
// cell is out of its reach; the rows kernel runs those tiles in its all-valid
// build and the others in its general build.
// ---------------------------------------------------------------------------
template <int TY, int TW>
__global__ void __launch_bounds__(kRowsNT)
classify_tiles_kernel(const hb_instance *__restrict__ insts, const int32_t *__restrict__ tile_inst,
                      int n_tiles, uint8_t *__restrict__ flags) {
  const int tile = blockIdx.x;
  if (tile >= n_tiles) return;
  const hb_instance &in = insts[tile_inst[tile]];
  const int lt = tile - in.tile_begin;
  const int tyi = lt / in.tiles_x, txi = lt - tyi * in.tiles_x;
  const int y0 = tyi * TY, x0 = txi * TW;
  bool ok = !(in.bug_y >= y0 - 2 && in.bug_y <= y0 + TY + 1 && in.bug_x >= x0 - 4 &&
              in.bug_x <= x0 + TW + 3);
  // raster row y is code row y + HB_PAD_Y, raster column x code column
  // x + HB_CODE_PAD_X; the region lies inside the padded code array
  constexpr int W = TW + 8;
  bool own = false;  // a valid cell among the tile's own cells
  for (int k = threadIdx.x; k < (TY + 4) * W; k += kRowsNT) {
    const int y = y0 - 2 + k / W, x = x0 - 4 + k % W;
    const uint8_t c = in.code[(size_t)(y + HB_PAD_Y) * in.code_pitch + (x + HB_CODE_PAD_X)];
    ok = ok && is_valid(c);
    own = own || (is_valid(c) && y >= y0 && y < y0 + TY && x >= x0 && x < x0 + TW);
  }
  ok = __syncthreads_and(ok) != 0;
  own = __syncthreads_or(own) != 0;
  // 2 (64-wide tiles only): no valid cell of its own, nothing to step
  if (threadIdx.x == 0) flags[tile] = ok ? 1 : ((TW == kPW && !own) ? 2 : 0);
}

// Stable partition of the tiles by flag, one block: order = general tiles
// with a valid cell (flag 0) in index order, then all-valid tiles (flag 1) in
// index order, then the tiles without a valid cell (flag 2, 64-wide tiles
// only) in index order, listed as ~tile; counts = {general (flags 0 and 2),
// all-valid, no valid cell}.  The tiles without a valid cell come last so
// that the one-launch step dispatches them at its end, where they take slots
// the last wave of tiles leaves idle.
constexpr int kOrderNT = 1024;
__global__ void __launch_bounds__(kOrderNT)
order_tiles_kernel(const uint8_t *__restrict__ flags, int n, int32_t *__restrict__ order,
                   int32_t *__restrict__ counts) {
  __shared__ int s_c[3][kOrderNT / 32];
  __shared__ int s_total[3], s_base[3];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid < 3) s_total[tid] = 0;
  __syncthreads();
  int c0 = 0, c1 = 0;
  for (int i = tid; i < n; i += kOrderNT) {
    c0 += flags[i] == 0;
    c1 += flags[i] == 1;
  }
  atomicAdd(&s_total[0], c0);
  atomicAdd(&s_total[1], c1);
  __syncthreads();
  if (tid == 0) {
    s_total[2] = n - s_total[0] - s_total[1];
    s_base[0] = 0;
    s_base[1] = s_total[0];
    s_base[2] = s_total[0] + s_total[1];
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
  for (int c = 0; c < n; c += kOrderNT) {
    const int i = c + tid;
    const int f = i < n ? flags[i] : 3;  // past the end: in no list
    unsigned bal[3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      bal[q] = __ballot_sync(0xffffffffu, f == q);
      if (lane == 0) s_c[q][w] = __popc(bal[q]);
    }
    __syncthreads();
    if (f < 3) {
      int o = 0;  // this flag's tiles in the warps before this one
      for (int q = 0; q < w; q++) o += s_c[f][q];
      order[s_base[f] + o + __popc(bal[f] & below)] = f == 2 ? ~i : i;
    }
    __syncthreads();
    if (tid < 3) {
      int t = 0;
      for (int q = 0; q < kOrderNT / 32; q++) t += s_c[tid][q];
      s_base[tid] += t;
    }
    __syncthreads();
  }
  if (tid == 0) {
    counts[0] = s_total[0] + s_total[2];
    counts[1] = s_total[1];
    counts[2] = s_total[2];
  }
}

// The order as TileEntry records (64-wide tiles): entries[k] for order[k].
__global__ void __launch_bounds__(256)
tile_entries_kernel(const int32_t *__restrict__ order, int n,
                    const int32_t *__restrict__ tile_inst, const hb_instance *__restrict__ insts,
                    TileEntry *__restrict__ entries) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int e = order[k];
  const int ii = tile_inst[e < 0 ? ~e : e];
  TileEntry r;
  r.tile = e;
  r.inst = ii;
  r.ctrl = insts[ii].ctrl;
  entries[k] = r;
}

// Per-device side stream (highest priority) and fork/join events for the
// general-tile kernel, created by hb_fused_prepare (outside any capture) and
// kept until exit.  The mutex keeps one fork/join sequence whole when several
// host threads step batches on one device.
constexpr int kMaxSideDevices = 64;
struct SideRes {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
std::mutex g_side_mu;
SideRes g_side[kMaxSideDevices];
// counts of general tiles (with or without a valid cell) and of the tiles
// without a valid cell, per prepared workspace (read back at prepare), so
// that the step launches one CTA per tile; guarded by g_side_mu
struct TileCounts {
  int general = 0, empty = 0;
};
std::unordered_map<const void *, TileCounts> g_general_tiles;

int side_setup() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxSideDevices)
    return set_error(HB_ERR_LIMIT, "hb_fused_prepare: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_side_mu);
  SideRes &r = g_side[dev];
  if (r.stream) return HB_OK;
  int lo = 0, hi = 0;
  e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&r.stream, cudaStreamNonBlocking, hi);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r.join, cudaEventDisableTiming);
  if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "side stream setup: %s", cudaGetErrorString(e));
  return HB_OK;
}

template <typename T, int TY, bool FAST = (sizeof(T) == 4), int MINB = 1, bool SOURCES = false,
          int ORDER = 2>
int launch_rows_impl(const hb_fused_batch *b, int nsteps, cudaStream_t st) {
  using S = RowsSmem<T, TY>;
  // both builds under the same register cap (2048^2 step, all-valid build
  // at 4 / 5 / 6 / 7 CTAs per SM: 130.6 / 121.3 / 129.6 / 139.5 us with
  // steps back to back; 5 and 6 are level, 128.8 / 129.3 us, with L2 flushed
  // between steps)
  constexpr int MINB_A = MINB;
  auto *kg = rows_step_kernel<T, TY, FAST, MINB, SOURCES, 0, ORDER>;
  auto *ka = rows_step_kernel<T, TY, FAST, MINB_A, SOURCES, 1, ORDER>;
  int rc = set_smem_attr(reinterpret_cast<const void *>(kg), (int)sizeof(S));
  if (!rc) rc = set_smem_attr(reinterpret_cast<const void *>(ka), (int)sizeof(S));
  if (rc) return rc;
  // One CTA per tile by default (the block scheduler starts the next tile as
  // soon as a CTA retires, which balances tiles of uneven cost): the general
  // tiles on the side stream, at the highest priority so that the slower
  // tiles start first, the all-valid tiles on the caller's stream; both
  // kernels run at once.  A positive grid_blocks makes every CTA loop over
  // its kernel's tiles.
  std::lock_guard<std::mutex> lock(g_side_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxSideDevices ||
      !g_side[dev].stream)
    return set_error(HB_ERR_ARG, "hb_fused_step: run hb_fused_prepare on this device first");
  const SideRes &sr = g_side[dev];
  const int n = b->n_tiles;
  int n_general = n;  // unknown workspace: CTAs beyond the general count exit at once
  const auto it = g_general_tiles.find(b->workspace);
  if (it != g_general_tiles.end()) n_general = std::max(it->second.general, 1);
  const int grid_a = b->grid_blocks > 0 ? std::min(b->grid_blocks, n) : n;
  const int grid_g = b->grid_blocks > 0 ? std::min(b->grid_blocks, n) : std::min(n_general, n);
  char *ws = reinterpret_cast<char *>(b->workspace);
  TilePartial *parts = reinterpret_cast<TilePartial *>(ws);
  TilePartial *gparts = reinterpret_cast<TilePartial *>(ws + ws_partials_bytes(b->n_tiles));
  unsigned *gcount = reinterpret_cast<unsigned *>(ws + ws_gcount_offset(b));
  const int32_t *order = reinterpret_cast<const int32_t *>(ws + ws_order_offset(b));
  const int32_t *counts = reinterpret_cast<const int32_t *>(ws + ws_counts_offset(b));
  BcTable *bct = reinterpret_cast<BcTable *>(ws + ws_bct_offset(b));
  const CUtensorMap *maps = reinterpret_cast<const CUtensorMap *>(ws + ws_maps_offset(b));
  for (int k = 0; k < nsteps; k++) {
    cudaError_t e = cudaEventRecord(sr.fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sr.stream, sr.fork, 0);
    if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "hb_fused_step fork: %s", cudaGetErrorString(e));
    kg<<<grid_g, kRowsNT, sizeof(S), sr.stream>>>(b->instances, b->tile_instance, order, counts,
                                                  parts, gparts, gcount, bct, maps);
    ka<<<grid_a, kRowsNT, sizeof(S), st>>>(b->instances, b->tile_instance, order, counts, parts,
                                           gparts, gcount, bct, maps);
    e = cudaEventRecord(sr.join, sr.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, sr.join, 0);
    if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "hb_fused_step join: %s", cudaGetErrorString(e));
  }
  return check_launch("hb_fused_step");
}

// The two-cells-per-lane step (64 x TY tiles).  Default (MINB 4, one CTA per
// tile): ONE launch of pairs_mixed_kernel over both tile lists on the
// caller's stream.  Otherwise (MINB 3, or a positive grid_blocks) the
// two builds with the same side-stream scheduling as launch_rows_impl:
// general tiles on the side stream, all-valid tiles on the caller's stream,
// both at once; the general build keeps the register cap of 3 CTAs per SM
// (its ghost-face branches spill under a tighter one) and MINB caps the
// all-valid build.
template <int TY, int MINB, bool SOURCES, int ORDER = 2>
int launch_pairs_impl(const hb_fused_batch *b, int nsteps, cudaStream_t st) {
  using S = PairSmem<TY>;
  const int n = b->n_tiles;
  // the list lengths come from prepare (one read-back there), so that a
  // tile's first load is its own entry
  // entries: general tiles with a valid cell [0, n_live), all-valid tiles
  // [n_live, n_live + n_valid), tiles without a valid cell [.., n)
  int n_general = 0, n_empty = 0;
  {
    std::lock_guard<std::mutex> lock(g_side_mu);
    const auto it = g_general_tiles.find(b->workspace);
    if (it == g_general_tiles.end())
      return set_error(HB_ERR_ARG, "hb_fused_step: run hb_fused_prepare on this workspace first");
    n_general = std::min(std::max(it->second.general, 0), n);
    n_empty = std::min(std::max(it->second.empty, 0), n_general);
  }
  const int n_valid = n - n_general, n_live = n_general - n_empty;
  char *ws = reinterpret_cast<char *>(b->workspace);
  TilePartial *parts = reinterpret_cast<TilePartial *>(ws);
  TilePartial *gparts = reinterpret_cast<TilePartial *>(ws + ws_partials_bytes(b->n_tiles));
  unsigned *gcount = reinterpret_cast<unsigned *>(ws + ws_gcount_offset(b));
  const TileEntry *entries = reinterpret_cast<const TileEntry *>(ws + ws_entries_offset(b));
  BcTable *bct = reinterpret_cast<BcTable *>(ws + ws_bct_offset(b));
  const CUtensorMap *maps = reinterpret_cast<const CUtensorMap *>(ws + ws_maps_offset(b));
  if (MINB == 4 && b->grid_blocks <= 0) {
    auto *km = pairs_mixed_kernel<TY, SOURCES, ORDER>;
    const int rc = set_smem_attr(reinterpret_cast<const void *>(km), (int)sizeof(S));
    if (rc) return rc;
    for (int k = 0; k < nsteps; k++)
      km<<<std::max(n, 1), kRowsNT, sizeof(S), st>>>(b->instances, entries, n_live,
                                                     n_live + n_valid, n, parts, gparts, gcount,
                                                     bct, maps);
    return check_launch("hb_fused_step");
  }
  auto *kg = pairs_step_kernel<TY, 3, SOURCES, 0, ORDER>;
  auto *ka = pairs_step_kernel<TY, MINB, SOURCES, 1, ORDER>;
  int rc = set_smem_attr(reinterpret_cast<const void *>(kg), (int)sizeof(S));
  if (!rc) rc = set_smem_attr(reinterpret_cast<const void *>(ka), (int)sizeof(S));
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(g_side_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxSideDevices ||
      !g_side[dev].stream)
    return set_error(HB_ERR_ARG, "hb_fused_step: run hb_fused_prepare on this device first");
  const SideRes &sr = g_side[dev];
  const int grid_a = std::max(b->grid_blocks > 0 ? std::min(b->grid_blocks, n_valid) : n_valid, 1);
  const int grid_g = std::max(b->grid_blocks > 0 ? std::min(b->grid_blocks, n_general) : n_general,
                              1);
  for (int k = 0; k < nsteps; k++) {
    cudaError_t e = cudaEventRecord(sr.fork, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sr.stream, sr.fork, 0);
    if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "hb_fused_step fork: %s", cudaGetErrorString(e));
    // the general build skips the all-valid entries in the middle of the list
    kg<<<grid_g, kRowsNT, sizeof(S), sr.stream>>>(b->instances, entries, n_general, n_live,
                                                  n_valid, parts, gparts, gcount, bct, maps);
    ka<<<grid_a, kRowsNT, sizeof(S), st>>>(b->instances, entries + n_live, n_valid, n_valid, 0,
                                           parts, gparts, gcount, bct, maps);
    e = cudaEventRecord(sr.join, sr.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, sr.join, 0);
    if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "hb_fused_step join: %s", cudaGetErrorString(e));
  }
  return check_launch("hb_fused_step");
}

int launch_pairs(const hb_fused_batch *b, int nsteps, cudaStream_t st) {
  const int minb = (b->flags >> HB_FLAG_MINB_SHIFT) & 0xF;
  const bool src = (b->flags & HB_FLAG_SOURCES) != 0;
  if (b->order == 1) {  // the 1st-order scheme: the all-valid build at 4 CTAs per SM
    if (minb == 0 || minb == 4) return src ? launch_pairs_impl<32, 4, true, 1>(b, nsteps, st)
                                           : launch_pairs_impl<32, 4, false, 1>(b, nsteps, st);
    return set_error(HB_ERR_ARG, "hb_fused_step: the 1st-order 64-wide tiles are built for "
                                 "4 CTAs per SM (minb 0 or 4), not %d", minb);
  }
  if (minb == 3) return src ? launch_pairs_impl<32, 3, true>(b, nsteps, st)
                            : launch_pairs_impl<32, 3, false>(b, nsteps, st);
  if (minb == 0 || minb == 4) return src ? launch_pairs_impl<32, 4, true>(b, nsteps, st)
                                         : launch_pairs_impl<32, 4, false>(b, nsteps, st);
  return set_error(HB_ERR_ARG, "hb_fused_step: 64-wide tiles are built for 3 or 4 CTAs per SM "
                               "(minb 0, 3 or 4), not %d", minb);
}

// The build with the infiltration / station-rain branches when the batch
// says its instances use them (HB_FLAG_SOURCES).
template <typename T, int TY, bool FAST = (sizeof(T) == 4), int MINB = 1, int ORDER = 2>
int launch_rows(const hb_fused_batch *b, int nsteps, cudaStream_t st) {
  if (b->flags & HB_FLAG_SOURCES)
    return launch_rows_impl<T, TY, FAST, MINB, true, ORDER>(b, nsteps, st);
  return launch_rows_impl<T, TY, FAST, MINB, false, ORDER>(b, nsteps, st);
}

bool uses_rows_kernel(const hb_fused_batch *b) { return !(b->flags & HB_FLAG_TILE_TASKS); }

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

int encode_2d(CUtensorMap *map, CUtensorMapDataType dt, size_t esize, const void *base,
              uint64_t width, uint64_t rows, uint32_t box_w, uint32_t box_h) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return set_error(HB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  if (((uintptr_t)base & 15) != 0)
    return set_error(HB_ERR_ARG, "tensor base address must be 16-byte aligned");
  if ((width * esize) % 16 != 0 || (box_w * esize) % 16 != 0)
    return set_error(HB_ERR_ARG, "tensor row pitch and box width must be multiples of 16 bytes");
  cuuint64_t dims[2] = {width, rows};
  cuuint64_t strides[1] = {width * esize};
  cuuint32_t box[2] = {box_w, box_h};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, dt, 2, const_cast<void *>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(HB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return HB_OK;
}

// Tensor maps of every instance for the rows kernel (box heights depend on
// the tile height), encoded into host_maps and copied to the workspace.
// Host records are read from b->instances_host.
int encode_maps(const hb_fused_batch *b, cudaStream_t st, CUtensorMap *host_maps) {
  if (!b->instances_host) return set_error(HB_ERR_ARG, "hb_fused_prepare: instances_host is null");
  const int TY = b->tile_y;
  const int TW = b->tile_x;  // 32 (rows kernel) or 64 (two cells per lane)
  const size_t es = b->dtype == HB_F64 ? 8 : 4;
  const CUtensorMapDataType dt =
      b->dtype == HB_F64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const size_t n_maps = (size_t)b->n_instances * kMapsPerInstance;
  CUtensorMap *maps = host_maps;
  for (int i = 0; i < b->n_instances; i++) {
    const hb_instance &in = b->instances_host[i];
    const uint64_t rows_s = (uint64_t)((in.rows + 63) / 64 * 64 + 2 * HB_PAD_Y);
    if ((int64_t)in.tiles_y * TY + 4 > (int64_t)rows_s || in.tiles_x * TW + 8 > in.pitch ||
        in.tiles_x * TW + 32 > in.code_pitch)
      return set_error(HB_ERR_ARG, "instance %d: storage smaller than its tiles", i);
    CUtensorMap *m = &maps[(size_t)i * kMapsPerInstance];
    const void *srcs[7] = {in.h[0], in.h[1], in.qx[0], in.qx[1], in.qy[0], in.qy[1], in.z};
    for (int k = 0; k < 7; k++) {
      int rc = encode_2d(&m[k], dt, es, srcs[k], (uint64_t)in.pitch, rows_s, TW + 8, TY + 4);
      if (rc) return rc;
    }
    int rc = encode_2d(&m[7], dt, es, in.h_max, (uint64_t)in.pitch, rows_s, TW, TY);
    if (rc) return rc;
    rc = encode_2d(&m[8], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, in.code, (uint64_t)in.code_pitch,
                   rows_s, TW + 32, TY + 4);
    if (rc) return rc;
  }
  char *dst = reinterpret_cast<char *>(b->workspace) + ws_maps_offset(b);
  cudaError_t e = cudaMemcpyAsync(dst, maps, n_maps * sizeof(CUtensorMap),
                                  cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "tensor maps upload: %s", cudaGetErrorString(e));
  return HB_OK;
}

}  // namespace
}  // namespace hb

using namespace hb;

// the persistent step's counters (3 x uint64), after the tensor maps
inline size_t ws_sync_offset(const hb_fused_batch *b) {
  return align256(ws_maps_offset(b) + (size_t)b->n_instances * kMapsPerInstance * sizeof(CUtensorMap));
}

extern "C" size_t hb_fused_workspace_size(const hb_fused_batch *b) {
  if (!b) return 0;
  return ws_sync_offset(b) + 256;
}

namespace hb {
namespace {

// Prepare with tensor maps staged in host_maps (n_instances * 9 entries), or
// in a temporary vector when host_maps is null.
int prepare_impl(const hb_fused_batch *b, cudaStream_t st, CUtensorMap *host_maps) {
  if (!b || !b->instances || !b->workspace || b->n_instances <= 0)
    return set_error(HB_ERR_ARG, "hb_fused_prepare: bad batch record");
  if (b->dtype != HB_F32 && b->dtype != HB_F64)
    return set_error(HB_ERR_ARG, "hb_fused_prepare: bad dtype %d", b->dtype);
  if (uses_rows_kernel(b)) {
    const bool pairs = b->tile_x == kPW && b->tile_y == 32;
    if (!pairs && (b->tile_x != kTW || (b->tile_y != 32 && b->tile_y != 64)))
      return set_error(HB_ERR_ARG, "hb_fused_prepare: rows kernel tiles are 32 wide, 32 or 64 "
                                   "high, or 64 wide and 32 high");
    if (pairs && (b->dtype != HB_F32 || (b->flags & HB_FLAG_EXACT_FP32)))
      return set_error(HB_ERR_ARG, "hb_fused_prepare: 64-wide tiles (two cells per lane) are "
                                   "built for the FP32 step");
    int rc;
    if (host_maps) {
      rc = encode_maps(b, st, host_maps);
    } else {
      std::vector<CUtensorMap> maps((size_t)b->n_instances * kMapsPerInstance);
      rc = encode_maps(b, st, maps.data());
    }
    if (rc) return rc;
  }
  if (b->instances_host) {
    for (int i = 0; i < b->n_instances; i++) {
      const bool src = b->instances_host[i].cum || b->instances_host[i].rain_station;
      if (src && !uses_rows_kernel(b))
        return set_error(HB_ERR_ARG,
                         "hb_fused_prepare: infiltration and station rain need the rows kernel");
      if (b->instances_host[i].halo_up[0] || b->instances_host[i].halo_down[0]) {
        if (!uses_rows_kernel(b))
          return set_error(HB_ERR_ARG, "hb_fused_prepare: halo forwarding needs the rows kernel");
      }
      if (src && !(b->flags & HB_FLAG_SOURCES))
        return set_error(HB_ERR_ARG, "hb_fused_prepare: instance %d has infiltration or "
                                     "station rain; set HB_FLAG_SOURCES", i);
    }
  }
  BcTable *bct = reinterpret_cast<BcTable *>((char *)b->workspace + ws_bct_offset(b));
  // the rows kernel's group counters start at zero; each group's last tile
  // resets its counter for the next step
  if (b->n_tiles > 0) {
    const cudaError_t e = cudaMemsetAsync((char *)b->workspace + ws_gcount_offset(b), 0,
                                          (size_t)ws_n_groups(b) * sizeof(unsigned), st);
    if (e != cudaSuccess)
      return set_error(HB_ERR_CUDA, "hb_fused_prepare: %s", cudaGetErrorString(e));
  }
  if (uses_rows_kernel(b) && b->n_tiles > 0) {
    // the side stream of the general tiles, and the tile classification
    int rc = side_setup();
    if (rc) return rc;
    char *ws = reinterpret_cast<char *>(b->workspace);
    uint8_t *flags = reinterpret_cast<uint8_t *>(ws + ws_flags_offset(b));
    if (b->tile_x == kPW)
      classify_tiles_kernel<32, kPW><<<b->n_tiles, kRowsNT, 0, st>>>(
          b->instances, b->tile_instance, b->n_tiles, flags);
    else if (b->tile_y == 64)
      classify_tiles_kernel<64, kTW><<<b->n_tiles, kRowsNT, 0, st>>>(
          b->instances, b->tile_instance, b->n_tiles, flags);
    else
      classify_tiles_kernel<32, kTW><<<b->n_tiles, kRowsNT, 0, st>>>(
          b->instances, b->tile_instance, b->n_tiles, flags);
    order_tiles_kernel<<<1, kOrderNT, 0, st>>>(
        flags, b->n_tiles, reinterpret_cast<int32_t *>(ws + ws_order_offset(b)),
        reinterpret_cast<int32_t *>(ws + ws_counts_offset(b)));
    if (b->tile_x == kPW)
      tile_entries_kernel<<<(b->n_tiles + 255) / 256, 256, 0, st>>>(
          reinterpret_cast<const int32_t *>(ws + ws_order_offset(b)), b->n_tiles,
          b->tile_instance, b->instances, reinterpret_cast<TileEntry *>(ws + ws_entries_offset(b)));
    int32_t counts[3] = {0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(counts, ws + ws_counts_offset(b), sizeof(counts),
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
      return set_error(HB_ERR_CUDA, "hb_fused_prepare: tile classes: %s", cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_side_mu);
    g_general_tiles[b->workspace] = TileCounts{counts[0], counts[2]};
  }
  // blocks per instance for the volume sum: about 16 cells per thread of the
  // largest instance (the host copy of the records gives the sizes)
  int64_t most = (int64_t)1 << 22;
  if (b->instances_host) {
    most = 0;
    for (int i = 0; i < b->n_instances; i++)
      most = std::max<int64_t>(most, (int64_t)b->instances_host[i].rows *
                                         b->instances_host[i].cols);
  }
  const int chunks = (int)std::min<int64_t>(std::max<int64_t>((most + 16 * kNT - 1) /
                                                                  (16 * kNT), 1), 1024);
  const dim3 vgrid(chunks, b->n_instances);
  if (b->dtype == HB_F64) {
    prepare_kernel<double><<<b->n_instances, 32, 0, st>>>(b->instances, bct);
    prepare_volume_kernel<double><<<vgrid, kNT, 0, st>>>(b->instances);
  } else {
    prepare_kernel<float><<<b->n_instances, 32, 0, st>>>(b->instances, bct);
    prepare_volume_kernel<float><<<vgrid, kNT, 0, st>>>(b->instances);
  }
  return check_launch("hb_fused_prepare");
}

}  // namespace
}  // namespace hb

extern "C" int hb_fused_prepare(const hb_fused_batch *b, void *stream) {
  return prepare_impl(b, as_stream(stream), nullptr);
}

extern "C" int hb_fused_finish(const hb_fused_batch *b, const double *ext, void *stream) {
  if (!b || !b->instances || !b->workspace || b->n_instances <= 0)
    return set_error(HB_ERR_ARG, "hb_fused_finish: bad batch record");
  BcTable *bct = reinterpret_cast<BcTable *>((char *)b->workspace + ws_bct_offset(b));
  auto st = as_stream(stream);
  if (b->dtype == HB_F64)
    finish_kernel<double><<<b->n_instances, kNT, 0, st>>>(b->instances, bct, ext, b->n_instances);
  else if (b->dtype == HB_F32)
    finish_kernel<float><<<b->n_instances, kNT, 0, st>>>(b->instances, bct, ext, b->n_instances);
  else
    return set_error(HB_ERR_ARG, "hb_fused_finish: bad dtype %d", b->dtype);
  return check_launch("hb_fused_finish");
}

extern "C" int hb_fused_step(const hb_fused_batch *b, int nsteps, void *stream) {
  if (!b || !b->instances || !b->tile_instance || !b->workspace || b->n_tiles <= 0)
    return set_error(HB_ERR_ARG, "hb_fused_step: bad batch record");
  if (nsteps < 0) return set_error(HB_ERR_ARG, "hb_fused_step: negative nsteps");
  if (b->order != 1 && b->order != 2)
    return set_error(HB_ERR_ARG, "hb_fused_step: order %d (1 or 2)", b->order);
  if (b->order == 1 && !uses_rows_kernel(b))
    return set_error(HB_ERR_ARG, "hb_fused_step: the tile-task kernel is 2nd order only");
  if (nsteps == 0) return HB_OK;
  auto st = as_stream(stream);
  const int ty = b->tile_y, tx = b->tile_x;
  const bool exact = (b->flags & HB_FLAG_EXACT_FP32) != 0;
  if (uses_rows_kernel(b) && b->order == 1) {
    // the 1st-order scheme (the coupled server's): FP32 64 x 32 tiles (two
    // cells per lane) or 32 x 32 tiles, FP64 32 x 32 tiles
    if (tx == kPW && ty == 32 && b->dtype == HB_F32 && !exact) return launch_pairs(b, nsteps, st);
    if (tx == kTW && ty == 32 && b->dtype == HB_F32 && !exact) {
      const int minb = (b->flags >> HB_FLAG_MINB_SHIFT) & 0xF;
      if (minb == 0) return launch_rows<float, 32, true, 1, 1>(b, nsteps, st);
      if (minb == 5) return launch_rows<float, 32, true, 5, 1>(b, nsteps, st);
    }
    if (tx == kTW && ty == 32 && b->dtype == HB_F64)
      return launch_rows<double, 32, false, 1, 1>(b, nsteps, st);
    return set_error(HB_ERR_ARG, "hb_fused_step: order 1 is built for FP32 64 x 32 tiles (minb "
                                 "0 or 4) and 32 x 32 tiles (minb 0 or 5), and FP64 32 x 32 tiles");
  }
  if (uses_rows_kernel(b) && tx == kPW) {
    if (ty == 32 && b->dtype == HB_F32 && !exact && b->order == 2) return launch_pairs(b, nsteps, st);
    return set_error(HB_ERR_ARG, "hb_fused_step: 64-wide tiles are built for the FP32 2nd-order "
                                 "step with 32-row tiles");
  }
  if (uses_rows_kernel(b)) {
    if (tx != kTW) return set_error(HB_ERR_ARG, "hb_fused_step: rows kernel tiles are 32 wide");
    if (b->dtype == HB_F32 && exact) {
      if (ty == 32) return launch_rows<float, 32, false>(b, nsteps, st);
    } else if (b->dtype == HB_F32) {
      // register cap by resident CTAs per SM (flags bits 8-11)
      const int minb = (b->flags >> HB_FLAG_MINB_SHIFT) & 0xF;
      if (ty == 32 && minb == 0) return launch_rows<float, 32>(b, nsteps, st);
      if (ty == 32 && minb == 5) return launch_rows<float, 32, true, 5>(b, nsteps, st);
      if (ty == 32 && minb == 6) return launch_rows<float, 32, true, 6>(b, nsteps, st);
      if (ty == 64 && minb == 0) return launch_rows<float, 64>(b, nsteps, st);
      if (ty == 64 && minb == 4) return launch_rows<float, 64, true, 4>(b, nsteps, st);
    } else if (b->dtype == HB_F64) {
      if (ty == 32) return launch_rows<double, 32>(b, nsteps, st);
    }
    return set_error(HB_ERR_ARG, "hb_fused_step: rows kernel %dx%d not built for this dtype", ty, tx);
  }
  if (b->dtype == HB_F32 && exact) {
    if (ty == 32 && tx == 32) return launch_steps<float, 32, 32, false>(b, nsteps, st);
  } else if (b->dtype == HB_F32) {
    if (ty == 32 && tx == 32) return launch_steps<float, 32, 32>(b, nsteps, st);
  } else if (b->dtype == HB_F64) {
    if (ty == 32 && tx == 32) return launch_steps<double, 32, 32>(b, nsteps, st);
  }
  return set_error(HB_ERR_ARG, "hb_fused_step: tile-task kernel %dx%d not built", ty, tx);
}

// ---------------------------------------------------------------------------
// hb_fused_step_noalloc: the fused step with its scratch in this library's
// own fixed device array instead of a caller-allocated workspace.
//
// The scratch (per-tile partial sums, boundary values, TMA descriptors) lives
// in g_noalloc_scratch, kNoAllocScratchBytes per GPU that loads the library,
// held until the process exits.  Host code must not pass g_noalloc_scratch to
// a kernel directly: in host code that name is only a stand-in for the device
// symbol.  Its device address is looked up with cudaGetSymbolAddress on the
// current device by every call with prepare != 0 (so a call after
// cudaDeviceReset that prepares picks up the new address) and kept for the
// calls without prepare.  The first prepare on a device also creates the side
// stream, which is why that call should come before any stream capture.
// The identity of the batch last prepared is kept per device too, so that a
// call without prepare for another batch is refused instead of running on
// that batch's tensor maps, tile order and counts.
// ---------------------------------------------------------------------------
namespace hb {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)4 << 20;  // 4 MiB per GPU
constexpr int kNoAllocMaxInstances = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// What a prepared scratch belongs to: a prepare == 0 call must present the
// same batch.
struct NoAllocOwner {
  bool valid = false;
  const void *instances = nullptr;
  const void *tile_instance = nullptr;
  int32_t n_tiles = 0, n_instances = 0, tile_y = 0, tile_x = 0, dtype = 0, order = 0, flags = 0;
  bool same(const hb_fused_batch *b) const {
    return valid && instances == b->instances && tile_instance == b->tile_instance &&
           n_tiles == b->n_tiles && n_instances == b->n_instances && tile_y == b->tile_y &&
           tile_x == b->tile_x && dtype == b->dtype && order == b->order && flags == b->flags;
  }
  void set(const hb_fused_batch *b) {
    valid = true;
    instances = b->instances;
    tile_instance = b->tile_instance;
    n_tiles = b->n_tiles;
    n_instances = b->n_instances;
    tile_y = b->tile_y;
    tile_x = b->tile_x;
    dtype = b->dtype;
    order = b->order;
    flags = b->flags;
  }
};

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kMaxDevices];
NoAllocOwner g_noalloc_owner[kMaxDevices];
// host staging of the tensor maps (no heap allocation on this path)
CUtensorMap g_noalloc_maps[kNoAllocMaxInstances * kMapsPerInstance];

}  // namespace
}  // namespace hb

extern "C" int hb_fused_step_noalloc(const hb_fused_batch *b, int nsteps, int prepare,
                                     void *stream) {
  if (!b || !b->instances || !b->tile_instance || b->n_tiles <= 0 || b->n_instances <= 0)
    return set_error(HB_ERR_ARG, "hb_fused_step_noalloc: bad batch record");
  hb_fused_batch local = *b;
  local.workspace = nullptr;
  const size_t need = hb_fused_workspace_size(&local);
  if (need > kNoAllocScratchBytes)
    return set_error(HB_ERR_LIMIT,
                     "hb_fused_step_noalloc: this batch needs %zu bytes of scratch; the fixed "
                     "scratch holds %zu bytes (use hb_fused_step with a workspace)",
                     need, kNoAllocScratchBytes);
  if (b->n_instances > kNoAllocMaxInstances)
    return set_error(HB_ERR_LIMIT, "hb_fused_step_noalloc: at most %d instances (got %d)",
                     kNoAllocMaxInstances, b->n_instances);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(HB_ERR_LIMIT, "hb_fused_step_noalloc: device %d out of range", dev);
  NoAllocOwner &owner = g_noalloc_owner[dev];
  if (prepare) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(HB_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
    owner.valid = false;  // the scratch is being rewritten
    local.workspace = p;
    int rc = prepare_impl(&local, as_stream(stream), g_noalloc_maps);
    if (rc) return rc;
    owner.set(b);
  } else if (!owner.same(b)) {
    return set_error(HB_ERR_ARG,
                     owner.valid ? "hb_fused_step_noalloc: the fixed scratch on device %d was "
                                   "last prepared for another batch; call with prepare != 0"
                                 : "hb_fused_step_noalloc: the fixed scratch on device %d has not "
                                   "been prepared; call with prepare != 0 first",
                     dev);
  }
  local.workspace = g_noalloc_ptr[dev];
  return hb_fused_step(&local, nsteps, stream);
}

// ---------------------------------------------------------------------------
// hb_fused_run: nsteps steps of every instance in one persistent cooperative
// launch (FP32 2nd order, 32 x 64 tiles).
// ---------------------------------------------------------------------------
namespace hb {
namespace {

template <bool SOURCES>
int launch_persistent(const hb_fused_batch *b, int nsteps, long long budget, cudaStream_t st) {
  using S = PairSmem<32>;
  auto *kern = pairs_persistent_kernel<32, SOURCES>;
  int rc = set_smem_attr(reinterpret_cast<const void *>(kern), (int)sizeof(S));
  if (rc) return rc;
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kRowsNT, sizeof(S));
  if (e != cudaSuccess || per_sm < 1)
    return set_error(HB_ERR_CUDA, "hb_fused_run: occupancy: %s",
                     e != cudaSuccess ? cudaGetErrorString(e) : "no resident block");
  int grid = per_sm * num_sms();
  if (grid > b->n_tiles) grid = b->n_tiles;
  char *ws = reinterpret_cast<char *>(b->workspace);
  const hb_instance *insts = b->instances;
  const TileEntry *entries = reinterpret_cast<const TileEntry *>(ws + ws_entries_offset(b));
  const int32_t *counts = reinterpret_cast<const int32_t *>(ws + ws_counts_offset(b));
  const uint8_t *allvalid = reinterpret_cast<const uint8_t *>(ws + ws_flags_offset(b));
  TilePartial *parts = reinterpret_cast<TilePartial *>(ws);
  TilePartial *gparts = reinterpret_cast<TilePartial *>(ws + ws_partials_bytes(b->n_tiles));
  unsigned *gcount = reinterpret_cast<unsigned *>(ws + ws_gcount_offset(b));
  BcTable *bct = reinterpret_cast<BcTable *>(ws + ws_bct_offset(b));
  const CUtensorMap *maps = reinterpret_cast<const CUtensorMap *>(ws + ws_maps_offset(b));
  unsigned long long *sync = reinterpret_cast<unsigned long long *>(ws + ws_sync_offset(b));
  int n_instances = b->n_instances;
  e = cudaMemsetAsync(sync, 0, 3 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return set_error(HB_ERR_CUDA, "hb_fused_run: %s", cudaGetErrorString(e));
  void *args[] = {(void *)&insts, (void *)&entries, (void *)&counts, (void *)&allvalid, (void *)&parts, (void *)&gparts, (void *)&gcount,
                  (void *)&bct, (void *)&maps, (void *)&n_instances, (void *)&nsteps,
                  (void *)&sync, (void *)&budget};
  e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(kern), dim3(grid), dim3(kRowsNT),
                                  args, sizeof(S), st);
  if (e != cudaSuccess)
    return set_error(HB_ERR_CUDA, "hb_fused_run: cooperative launch of %d blocks: %s", grid,
                     cudaGetErrorString(e));
  return HB_OK;
}

}  // namespace
}  // namespace hb

extern "C" int hb_fused_run(const hb_fused_batch *b, int nsteps, long long budget_cycles,
                            void *stream) {
  if (!b || !b->instances || !b->tile_instance || !b->workspace || b->n_tiles <= 0)
    return set_error(HB_ERR_ARG, "hb_fused_run: bad batch record");
  if (nsteps < 0) return set_error(HB_ERR_ARG, "hb_fused_run: negative nsteps");
  if (!uses_rows_kernel(b) || b->tile_x != kPW || b->tile_y != 32 || b->dtype != HB_F32 ||
      b->order != 2 || (b->flags & HB_FLAG_EXACT_FP32))
    return set_error(HB_ERR_ARG, "hb_fused_run: the persistent step is built for the FP32 "
                                 "2nd-order step with 32 x 64 tiles");
  if (nsteps == 0) return HB_OK;
  const long long budget = budget_cycles > 0 ? budget_cycles : (1LL << 31);
  auto st = as_stream(stream);
  if (b->flags & HB_FLAG_SOURCES) return launch_persistent<true>(b, nsteps, budget, st);
  return launch_persistent<false>(b, nsteps, budget, st);
}
