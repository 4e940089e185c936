// hb_physics.cuh -- device functions of the HiPIMS scheme shared by the compat
// kernels and the fused dense-tile step.
//
// With T = double and FAST = false every function performs the reference's
// operations in the reference's order (paths relative to CHANS-HiPIMS/hipims/
// cuda): MUSCL flucCal_2ndOrder_jh_improved_Kernel.cu:83-107, hydrostatic
// reconstruction :43-72 (2nd order) and fluxCal_jh_modified_surface_Kernel.cu
// :96-139 (1st order), HLLC :109-195, ghost states :197-332.  FAST = true
// (FP32 fused path) keeps the same decisions but uses algebraically equal,
// cheaper forms: a* = |(aL + aR)/2 + (uL - uR)/4| instead of sqrt(g * h*),
// one reciprocal of (sR - sL), and approximate division.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace hb {

template <typename T>
struct Cell {
  T h, wl, qx, qy, z;
};

template <typename T>
__device__ __forceinline__ T minmod(T x, T y) {
  if (x * y <= T(0)) return T(0);
  return fabs(x) < fabs(y) ? x : y;
}

template <typename T, bool FAST>
__device__ __forceinline__ T fdiv(T a, T b) {
  if constexpr (FAST && sizeof(T) == 4) return __fdividef(a, b);
  else return a / b;
}

// Edge value of cell c towards r (l is the opposite neighbour).  The edge wl
// is not formed: the hydrostatic step recomputes it from h + z.
template <typename T>
__device__ __forceinline__ void muscl(const Cell<T> &c, const Cell<T> &l,
                                      const Cell<T> &r, Cell<T> &e) {
  e.h = c.h + T(0.5) * minmod(c.h - l.h, r.h - c.h);
  e.wl = c.wl;
  e.z = c.z + T(0.5) * minmod(c.z - l.z, r.z - c.z);
  if (c.h < T(kHSmall)) {
    e.qx = T(0);
    e.qy = T(0);
  } else {
    e.qx = c.qx + T(0.5) * minmod(c.qx - l.qx, r.qx - c.qx);
    e.qy = c.qy + T(0.5) * minmod(c.qy - l.qy, r.qy - c.qy);
  }
}

// Hydrostatic reconstruction, 2nd-order variant.  wl_cl / wl_cr: free-surface
// level of the two cells (the right one may be a ghost).
template <typename T>
__device__ __forceinline__ void hydro2(T wl_cl, T wl_cr, Cell<T> &L, Cell<T> &R) {
  T hi = fmax(wl_cl, wl_cr), lo = fmin(wl_cl, wl_cr);
  L.wl = fmax(fmin(L.h + L.z, hi), lo);
  R.wl = fmax(fmin(R.h + R.z, hi), lo);
  if (wl_cl > wl_cr)
    L.wl = fmax(L.wl, R.wl);
  else
    R.wl = fmax(L.wl, R.wl);
  L.z = L.wl - L.h;
  R.z = R.wl - R.h;
  T zbm = fmax(L.z, R.z);
  L.h = fmax(L.wl - zbm, T(0));
  R.h = fmax(R.wl - zbm, T(0));
  L.z = L.wl - L.h;
  R.z = R.wl - R.h;
}

// Hydrostatic reconstruction, 1st-order variant: eta of the raw cells from
// h + z, averaging the two edge levels when their ordering flips.
template <typename T>
__device__ __forceinline__ void hydro1(T hc, T zc, T hr, T zr, Cell<T> &L,
                                       Cell<T> &R) {
  T ec = hc + zc, er = hr + zr;
  T hi = fmax(ec, er), lo = fmin(ec, er);
  L.wl = fmax(fmin(L.h + L.z, hi), lo);
  R.wl = fmax(fmin(R.h + R.z, hi), lo);
  if ((ec - er) * (L.wl - R.wl) < T(0)) {
    T tmp = (L.wl + R.wl) / T(2);
    L.wl = tmp;
    R.wl = tmp;
  }
  L.z = L.wl - L.h;
  R.z = R.wl - R.h;
  T zbm = fmax(L.z, R.z);
  L.h = fmax(L.wl - zbm, T(0));
  R.h = fmax(R.wl - zbm, T(0));
  L.z = L.wl - L.h;
  R.z = R.wl - R.h;
}

// HLLC flux in the face frame.  hL, hR: depths after the hydrostatic step;
// uL/vL, uR/vR: normal/tangential velocities of the edge states taken before
// it.  Returns false when both sides are dry (no flux).  fh: mass flux,
// fn: normal-momentum flux, ft: tangential-momentum flux.
template <typename T, bool FAST>
__device__ __forceinline__ bool hllc(T hL, T hR, T u_L, T u_R, T v_L, T v_R,
                                     T &fh, T &fn, T &ft) {
  const T hs = T(kHSmall), g = T(kG);
  if (hL < hs && hR < hs) return false;
  T qx_L = u_L * hL, qy_L = v_L * hL;
  T qx_R = u_R * hR, qy_R = v_R * hR;
  T a_L = sqrt(g * hL), a_R = sqrt(g * hR);
  T base = (a_L + a_R) / T(2) + (u_L - u_R) / T(4);
  T u_star = (u_L + u_R) / T(2) + a_L - a_R;
  T a_star;
  if constexpr (FAST) {
    a_star = fabs(base);  // sqrt(g * base^2 / g)
  } else {
    T h_star = (base * base) / g;
    a_star = sqrt(g * h_star);
  }
  T s_L = hL <= hs ? u_R - T(2) * a_R : fmin(u_L - a_L, u_star - a_star);
  T s_R = hR <= hs ? u_L + T(2) * a_L : fmax(u_R + a_R, u_star + a_star);
  T h_flux_L = qx_L;
  T qx_flux_L = u_L * qx_L + T(0.5) * g * hL * hL;
  T qy_flux_L = u_L * qy_L;
  T h_flux_R = qx_R;
  T qx_flux_R = u_R * qx_R + T(0.5) * g * hR * hR;
  T qy_flux_R = u_R * qy_R;
  if constexpr (FAST) {
    // branch-free region selection (same decisions as below; a NaN s_M
    // selects the right state, as the reference's if-chain falls through)
    const T s_M = fdiv<T, FAST>(s_L * hR * (u_R - s_R) - s_R * hL * (u_L - s_L),
                                hR * (u_R - s_R) - hL * (u_L - s_L));
    const T inv = T(1) / (s_R - s_L);
    const T h_flux_M = (s_R * h_flux_L - s_L * h_flux_R + s_L * s_R * (hR - hL)) * inv;
    const T qx_flux_M = (s_R * qx_flux_L - s_L * qx_flux_R + s_L * s_R * (qx_R - qx_L)) * inv;
    const bool left = T(0) <= s_L;
    const bool midL = !left && (s_L < T(0) && T(0) <= s_M);
    const bool midR = !left && !midL && (s_M < T(0) && T(0) <= s_R);
    const bool mid = midL || midR;
    fh = left ? h_flux_L : (mid ? h_flux_M : h_flux_R);
    fn = left ? qx_flux_L : (mid ? qx_flux_M : qx_flux_R);
    ft = left ? qy_flux_L : (midL ? h_flux_M * v_L : (midR ? h_flux_M * v_R : qy_flux_R));
    return true;
  }
  if (T(0) <= s_L) {
    fh = h_flux_L;
    fn = qx_flux_L;
    ft = qy_flux_L;
    return true;
  }
  T s_M = fdiv<T, FAST>(s_L * hR * (u_R - s_R) - s_R * hL * (u_L - s_L),
                        hR * (u_R - s_R) - hL * (u_L - s_L));
  if (s_M < T(0) && !(T(0) <= s_R)) {
    fh = h_flux_R;
    fn = qx_flux_R;
    ft = qy_flux_R;
    return true;
  }
  if (!(s_L < T(0) && T(0) <= s_M) && !(s_M < T(0) && T(0) <= s_R)) {
    // s_M is NaN (degenerate states): the reference falls through to R.
    fh = h_flux_R;
    fn = qx_flux_R;
    ft = qy_flux_R;
    return true;
  }
  T h_flux_M, qx_flux_M;
  if constexpr (FAST) {
    T inv = T(1) / (s_R - s_L);
    h_flux_M = (s_R * h_flux_L - s_L * h_flux_R + s_L * s_R * (hR - hL)) * inv;
    qx_flux_M = (s_R * qx_flux_L - s_L * qx_flux_R + s_L * s_R * (qx_R - qx_L)) * inv;
  } else {
    h_flux_M = (s_R * h_flux_L - s_L * h_flux_R + s_L * s_R * (hR - hL)) / (s_R - s_L);
    qx_flux_M =
        (s_R * qx_flux_L - s_L * qx_flux_R + s_L * s_R * (qx_R - qx_L)) / (s_R - s_L);
  }
  fh = h_flux_M;
  fn = qx_flux_M;
  ft = (T(0) <= s_M) ? h_flux_M * v_L : h_flux_M * v_R;
  return true;
}

// Ghost state of a missing neighbour of cell c with outward normal (n0, n1).
// Types: 3 RIGID, 4 WALL_SLIP, 5 OPEN, 6 H_GIVEN, 7 Q_GIVEN, 8 WL_GIVEN,
// 9 FALL (first order only).  Returns false for a type without a ghost rule.
template <typename T>
__device__ __forceinline__ bool ghost(int type, bool allow_fall, const Cell<T> &c,
                                      T n0, T n1, T hb, T wlb, T qxb, T qyb,
                                      Cell<T> &b) {
  switch (type) {
    case 3:
      b.h = c.h; b.wl = c.wl; b.z = c.z;
      b.qx = (n1 * n1 - n0 * n0) * c.qx;
      b.qy = -(n0 * n0 - n1 * n1) * c.qy;
      return true;
    case 4:
      b.h = c.h; b.wl = c.wl; b.z = c.z;
      b.qx = (n1 * n1 - n0 * n0) * c.qx;
      b.qy = (n0 * n0 - n1 * n1) * c.qy;
      return true;
    case 5:
      b = c;
      return true;
    case 6:
      b.h = hb; b.z = c.z; b.wl = b.z + b.h; b.qx = c.qx; b.qy = c.qy;
      return true;
    case 7:
      b.h = c.h; b.z = c.z; b.wl = b.z + b.h; b.qx = qxb; b.qy = qyb;
      return true;
    case 8:
      b.z = c.z; b.wl = wlb > b.z ? wlb : b.z; b.h = b.wl - b.z;
      b.qx = c.qx; b.qy = c.qy;
      return true;
    case 9:
      if (!allow_fall) return false;
      b.h = T(0); b.wl = c.wl; b.z = c.z; b.qx = T(0); b.qy = T(0);
      return true;
    default:
      return false;
  }
}

// Boundary code decode: leading decimal digit = type, remaining digits = id.
__device__ __forceinline__ void decode_bc(int code, int &type, int &id) {
  int bt = code, p = 1;
  while (bt >= 10) {
    bt /= 10;
    p *= 10;
  }
  type = bt;
  id = code - bt * p;
}

// Row of a boundary table for time t: the first row whose time is not
// below t, clamped to the last row.
template <typename TT>
__device__ __forceinline__ int timelevel(double t, const TT *tab, int rows, int cols) {
  int tl = 0;
  while ((t > (double)tab[(int64_t)tl * cols]) && (tl < rows - 1)) tl++;
  return tl;
}

}  // namespace hb
