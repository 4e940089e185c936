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

#include <mutex>

#include "hb_common.cuh"
#include "hb_physics.cuh"
#include "hipims_b200_fused.h"

namespace hb {
namespace {

constexpr int kNT = 256;  // threads per CTA

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
  const T ux_l = eL.h < hs ? T(0) : eL.qx / eL.h;
  const T uy_l = eL.h < hs ? T(0) : eL.qy / eL.h;
  const T ux_r = eR.h < hs ? T(0) : eR.qx / eR.h;
  const T uy_r = eR.h < hs ? T(0) : eR.qy / eR.h;
  hydro2(C.wl, G.wl, eL, eR);
  const T u_L = ux_l * n0 + uy_l * n1, u_R = ux_r * n0 + uy_r * n1;
  const T v_L = -ux_l * n1 + uy_l * n0, v_R = -ux_r * n1 + uy_r * n0;
  T Fh, Fn, Ft;
  if (hllc<T, false>(eL.h, eR.h, u_L, u_R, v_L, v_R, Fh, Fn, Ft)) {
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
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------------------
// Control-block helpers (single thread)
// ---------------------------------------------------------------------------

// Rain rate at t with the reference's monotone row cursor
// (HP/SWE_CUDA.py:472-495): linear interpolation, zero after the last row.
__device__ double rain_rate_at(const hb_instance &in, hb_ctrl *c, double t) {
  if (!in.rain_tab || in.rain_rows < 2) return 0.0;
  const double *R = in.rain_tab;
  const int C = in.rain_cols;
  if (!(t < R[(int64_t)(in.rain_rows - 1) * C])) return 0.0;
  int idx = min(max(c->rain_index, 0), in.rain_rows - 2);
  while (idx + 2 < in.rain_rows && !(t < R[(int64_t)(idx + 1) * C])) idx++;
  c->rain_index = idx;
  const double *r0 = R + (int64_t)idx * C, *r1 = r0 + C;
  const double per = (t - r0[0]) / (r1[0] - r0[0]);
  return (r0[1] + per * (r1[1] - r0[1])) * c->rain_mult;
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

// Workspace layout: [n_tiles] TilePartial, then [n_instances] BcTable.
inline size_t ws_partials_bytes(int n_tiles) {
  return ((size_t)n_tiles * sizeof(TilePartial) + 255) & ~(size_t)255;
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
  extern __shared__ __align__(16) unsigned char smem_raw[];
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
      __threadfence();
      const unsigned n_inst_tiles = (unsigned)(in.tiles_x * in.tiles_y);
      s.last = (atomicAdd(&ctrl->tiles_done, 1u) == n_inst_tiles - 1);
    }
    __syncthreads();

    if (s.last) {
      // --- finalize this instance: reduce its tiles' partials
      __threadfence();
      const int nt = in.tiles_x * in.tiles_y;
      double v = 0, o = 0, sm = 0;
      int dry = 0;
      for (int k = tid; k < nt; k += kNT) {
        const TilePartial *pp = partials + in.tile_begin + k;
        v += __ldcg(&pp->volume);
        o += __ldcg(&pp->outflow);
        sm = fmax(sm, __ldcg(&pp->smax));
        dry |= __ldcg(&pp->any_dry);
      }
      v = warp_sum(v);
      o = warp_sum(o);
      sm = warp_max(sm);
      dry = __any_sync(0xffffffffu, dry);
      if (lane == 0) {
        s.red_d[0][wid] = v;
        s.red_d[1][wid] = o;
        s.red_s[wid] = sm;
        s.red_i[wid] = dry;
      }
      __syncthreads();
      if (tid == 0) {
        double V = 0, O = 0, SM = 0;
        int D = 0;
        for (int w = 0; w < kNT / 32; w++) {
          V += s.red_d[0][w];
          O += s.red_d[1][w];
          SM = fmax(SM, s.red_s[w]);
          D |= s.red_i[w];
        }
        const double dtn = ctrl->dt, tn = ctrl->t, dxd = in.dx;
        // dt = min over cells of CFL*dx/speed (60 for dry cells); the
        // division is monotone, so dividing once by the max speed is exact.
        double cand = INFINITY;
        if (SM > 0.0) cand = (double)((T)in.cfl * (T)in.dx / (T)SM);
        if (D) cand = fmin(cand, 60.0);
        double dtnew = (cand == INFINITY) ? dtn : cand;
        const double upper = dtn * 10.0;
        if (upper < dtnew) dtnew = upper;  // Python min(self.dt, time_upper)
        const double next_export = (double)(ctrl->export_n + 1) * ctrl->export_step;
        if (ctrl->export_step > 0.0 && dtnew + tn >= next_export) {
          dtnew = next_export - tn;
          ctrl->export_n += 1;
          ctrl->exports += 1;
          if (ctrl->halt_on_export) ctrl->halted = 1;
        }
        if (in.dt_replay && ctrl->step < in.n_replay) dtnew = in.dt_replay[ctrl->step];
        if (!isfinite(dtnew)) ctrl->status = 1;
        ctrl->volume = V * dxd * dxd;
        ctrl->outflow_volume += O * dtn * dxd;
        ctrl->rain_volume += ctrl->rain_rate * dtn * dxd * dxd * (double)in.n_valid;
        const double tnew = tn + dtnew;
        ctrl->dt = dtnew;
        ctrl->t = tnew;
        ctrl->cur = 1 - ctrl->cur;
        ctrl->step += 1;
        if (tnew >= ctrl->t_end) ctrl->halted = 1;
        ctrl->rain_rate = rain_rate_at(in, ctrl, tnew);
        bc_values_exact(in, tnew, &bct[ii]);
        bc_values_at(in, ctrl, tnew);
        __threadfence();
        ctrl->tiles_done = 0u;
      }
    }
    __syncthreads();
  }
}

// Prepare: volume at t, rain rate and boundary values, counters.
template <typename T>
__global__ void __launch_bounds__(kNT)
prepare_kernel(const hb_instance *__restrict__ insts, BcTable *__restrict__ bct) {
  const hb_instance &in = insts[blockIdx.x];
  hb_ctrl *c = in.ctrl;
  const T *h = (const T *)in.h[c->cur];
  const uint8_t *code = in.code;
  double v = 0;
  for (int64_t k = threadIdx.x; k < (int64_t)in.rows * in.cols; k += blockDim.x) {
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
    c->volume = V * in.dx * in.dx;
    c->volume0 = c->volume;
    c->tiles_done = 0u;
    c->rain_rate = rain_rate_at(in, c, c->t);
    bc_values_exact(in, c->t, &bct[blockIdx.x]);
    bc_values_at(in, c, c->t);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename T, int TY, int TX, bool FAST = (sizeof(T) == 4)>
int launch_steps(const hb_fused_batch *b, int nsteps, cudaStream_t st) {
  using S = Smem<T, TY, TX>;
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  static int blocks_per_sm = 1;
  std::call_once(once, [] {
    attr_err = cudaFuncSetAttribute(fused_step_kernel<T, TY, TX, FAST>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(S));
    if (attr_err == cudaSuccess)
      attr_err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &blocks_per_sm, fused_step_kernel<T, TY, TX, FAST>, kNT, sizeof(S));
    if (blocks_per_sm < 1) blocks_per_sm = 1;
  });
  if (attr_err != cudaSuccess)
    return set_error(HB_ERR_CUDA, "fused step setup: %s", cudaGetErrorString(attr_err));
  int grid = b->grid_blocks > 0 ? b->grid_blocks : blocks_per_sm * num_sms();
  if (grid > b->n_tiles) grid = b->n_tiles;
  TilePartial *parts = reinterpret_cast<TilePartial *>(b->workspace);
  BcTable *bct = reinterpret_cast<BcTable *>((char *)b->workspace + ws_partials_bytes(b->n_tiles));
  for (int k = 0; k < nsteps; k++) {
    fused_step_kernel<T, TY, TX, FAST><<<grid, kNT, sizeof(S), st>>>(b->instances, b->tile_instance,
                                                                b->n_tiles, parts, bct);
  }
  return check_launch("hb_fused_step");
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" size_t hb_fused_workspace_size(const hb_fused_batch *b) {
  if (!b) return 0;
  return ws_partials_bytes(b->n_tiles) + (size_t)b->n_instances * sizeof(BcTable);
}

extern "C" int hb_fused_prepare(const hb_fused_batch *b, void *stream) {
  if (!b || !b->instances || !b->workspace || b->n_instances <= 0)
    return set_error(HB_ERR_ARG, "hb_fused_prepare: bad batch record");
  if (b->dtype != HB_F32 && b->dtype != HB_F64)
    return set_error(HB_ERR_ARG, "hb_fused_prepare: bad dtype %d", b->dtype);
  auto st = as_stream(stream);
  BcTable *bct = reinterpret_cast<BcTable *>((char *)b->workspace + ws_partials_bytes(b->n_tiles));
  if (b->dtype == HB_F64)
    prepare_kernel<double><<<b->n_instances, kNT, 0, st>>>(b->instances, bct);
  else
    prepare_kernel<float><<<b->n_instances, kNT, 0, st>>>(b->instances, bct);
  return check_launch("hb_fused_prepare");
}

extern "C" int hb_fused_step(const hb_fused_batch *b, int nsteps, void *stream) {
  if (!b || !b->instances || !b->tile_instance || !b->workspace || b->n_tiles <= 0)
    return set_error(HB_ERR_ARG, "hb_fused_step: bad batch record");
  if (nsteps < 0) return set_error(HB_ERR_ARG, "hb_fused_step: negative nsteps");
  if (b->order != 2) return set_error(HB_ERR_ARG, "hb_fused_step: only order 2 is fused");
  if (nsteps == 0) return HB_OK;
  auto st = as_stream(stream);
  const int ty = b->tile_y, tx = b->tile_x;
  if (b->dtype == HB_F32 && (b->flags & HB_FLAG_EXACT_FP32)) {
    if (ty == 32 && tx == 32) return launch_steps<float, 32, 32, false>(b, nsteps, st);
    return set_error(HB_ERR_ARG, "hb_fused_step: exact FP32 tile %dx%d not built", ty, tx);
  }
  if (b->dtype == HB_F32) {
    if (ty == 32 && tx == 32) return launch_steps<float, 32, 32>(b, nsteps, st);
    if (ty == 16 && tx == 64) return launch_steps<float, 16, 64>(b, nsteps, st);
    if (ty == 16 && tx == 32) return launch_steps<float, 16, 32>(b, nsteps, st);
    if (ty == 8 && tx == 64) return launch_steps<float, 8, 64>(b, nsteps, st);
    return set_error(HB_ERR_ARG, "hb_fused_step: FP32 tile %dx%d not built", ty, tx);
  }
  if (b->dtype == HB_F64) {
    if (ty == 32 && tx == 32) return launch_steps<double, 32, 32>(b, nsteps, st);
    if (ty == 16 && tx == 32) return launch_steps<double, 16, 32>(b, nsteps, st);
    return set_error(HB_ERR_ARG, "hb_fused_step: FP64 tile %dx%d not built", ty, tx);
  }
  return set_error(HB_ERR_ARG, "hb_fused_step: bad dtype %d", b->dtype);
}
