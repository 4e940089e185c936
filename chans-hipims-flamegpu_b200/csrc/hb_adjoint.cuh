// hb_adjoint.cuh -- reverse-mode derivatives of the HiPIMS step (FP64).
//
// The forward functions restate, operation for operation, the FP64 path of
// the fused step (hb_fused.cu, itself following the reference kernels
// HC/flucCal_2ndOrder_jh_improved_Kernel.cu:43-506 and
// HC/friction_implicit_andUpdate_jh_Kernel.cu:22-146); the reverse functions
// propagate adjoints back through them with every discrete decision (minmod
// selection, wet/dry thresholds, hydrostatic clamps, HLLC wave region,
// friction limiter) taken as the forward takes it.  The functions are
// __host__ __device__ so that tests can check them against finite
// differences on the CPU.
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define HB_HD __host__ __device__ __forceinline__
#else
#define HB_HD inline
#endif

namespace hb {
namespace adj {

constexpr double kHs = 1.0e-6;
constexpr double kG = 9.81;

struct C3 {  // a cell's prognostic state or its adjoint
  double h, qx, qy;
};
struct Cz {
  double h, qx, qy, z;
};

// ---------------------------------------------------------------- minmod
// r = minmod(x, y); dr/dx, dr/dy in {0, 1}
HB_HD double mm(double x, double y, double &dx, double &dy) {
  if (x * y <= 0.0) {
    dx = dy = 0.0;
    return 0.0;
  }
  if (fabs(x) < fabs(y)) {
    dx = 1.0;
    dy = 0.0;
    return x;
  }
  dx = 0.0;
  dy = 1.0;
  return y;
}

// ------------------------------------------------------------------ face
// Face between A (minus side) and B (plus side) along DIR (0: normal +x,
// 1: normal +y), both cells valid.  L: A's opposite neighbour, RR: B's
// opposite neighbour (used only when valid).  Outputs: fh, fx, fy (fluxes
// in the global frame, from A's side), sa, sb (bed-slope terms of A and B).
struct FaceIn {
  Cz L, A, B, R;
  bool vL, vR;
  bool noslope;  // boundary face: no reconstruction (edges are the cells)
};
struct FaceOut5 {
  double fh, fx, fy, sa, sb;
};

// One slope component: s = minmod(c - m', p' - c) with m' = vm ? m : c.
// Derivatives w.r.t. (m, c, p).
HB_HD double slope1(double m, double c, double p, bool vm, bool vp, double &dm, double &dc,
                    double &dp) {
  const double mm_ = vm ? m : c, pp = vp ? p : c;
  double d1, d2;
  const double s = mm(c - mm_, pp - c, d1, d2);
  // s = d1 * (c - m') + d2 * (p' - c)
  dm = vm ? -d1 : 0.0;
  dp = vp ? d2 : 0.0;
  dc = d1 * (1.0 - (vm ? 0.0 : 1.0)) + d2 * ((vp ? 0.0 : 1.0) - 1.0);
  return s;
}

template <int DIR>
struct FaceTape {
  // slope selections: [field h, qx, qy, z] x [m, c, p] for sA (m=L, c=A, p=B) and sB (m=A, c=B, p=R)
  double dA[4][3], dB[4][3];
  double sA[4], sB[4];
  bool skip;  // both cells dry: no flux, no slope terms
  bool wetA, wetB;
  double eLh, eLz, eLqx, eLqy, eRh, eRz, eRqx, eRqy;
  bool velL, velR;
  double uxl, uyl, uxr, uyr;
  // hydrostatic
  double wlA, wlB, hi, lo;
  bool hiA, loA;  // hi = wlA (else wlB); lo = wlA (else wlB)
  int selL1, selL2, selR1, selR2;  // min/max selections of the clamps
  bool Araise;                      // wlA > wlB: L.wl = max(L, R); else R.wl = max
  bool raiseTookOther;
  double Lw, Rw, Lz, Rz, zbm;
  bool zbmL;
  bool Lpos, Rpos;
  double Lh, Rh;
  // hllc
  bool bothdry;
  double uL, uR, vL, vR;
  double aL, aR, base, ustar, astar, sL, sR;
  int sLcase, sRcase;  // 0: dry formula, 1: first arg of min/max, 2: second
  int region;          // 0 left, 1 midL, 2 midR, 3 right
  double hfL, qfL, tfL, hfR, qfR, tfR, hfM, qfM, inv;
};

template <int DIR>
HB_HD FaceOut5 face_fwd(const FaceIn &in, FaceTape<DIR> &tp) {
  const double hs = kHs, g = kG;
  FaceOut5 o{0, 0, 0, 0, 0};
  const Cz &A = in.A, &B = in.B;
  tp.skip = (A.h < hs && B.h < hs);
  if (tp.skip) return o;
  // slopes (index 0 h, 1 qx, 2 qy, 3 z)
  const double Av[4] = {A.h, A.qx, A.qy, A.z}, Bv[4] = {B.h, B.qx, B.qy, B.z};
  const double Lv[4] = {in.L.h, in.L.qx, in.L.qy, in.L.z};
  const double Rv[4] = {in.R.h, in.R.qx, in.R.qy, in.R.z};
  for (int f = 0; f < 4; f++) {
    if (in.noslope) {
      tp.sA[f] = tp.sB[f] = 0.0;
      tp.dA[f][0] = tp.dA[f][1] = tp.dA[f][2] = 0.0;
      tp.dB[f][0] = tp.dB[f][1] = tp.dB[f][2] = 0.0;
      continue;
    }
    tp.sA[f] = slope1(Lv[f], Av[f], Bv[f], in.vL, true, tp.dA[f][0], tp.dA[f][1], tp.dA[f][2]);
    tp.sB[f] = slope1(Av[f], Bv[f], Rv[f], true, in.vR, tp.dB[f][0], tp.dB[f][1], tp.dB[f][2]);
  }
  // edges
  tp.wetA = !(A.h < hs);
  tp.wetB = !(B.h < hs);
  tp.eLh = A.h + 0.5 * tp.sA[0];
  tp.eLz = A.z + 0.5 * tp.sA[3];
  tp.eLqx = tp.wetA ? A.qx + 0.5 * tp.sA[1] : 0.0;
  tp.eLqy = tp.wetA ? A.qy + 0.5 * tp.sA[2] : 0.0;
  tp.eRh = B.h + 0.5 * (-tp.sB[0]);
  tp.eRz = B.z + 0.5 * (-tp.sB[3]);
  tp.eRqx = tp.wetB ? B.qx + 0.5 * (-tp.sB[1]) : 0.0;
  tp.eRqy = tp.wetB ? B.qy + 0.5 * (-tp.sB[2]) : 0.0;
  // velocities before the hydrostatic step
  tp.velL = !(tp.eLh < hs);
  tp.velR = !(tp.eRh < hs);
  tp.uxl = tp.velL ? tp.eLqx / tp.eLh : 0.0;
  tp.uyl = tp.velL ? tp.eLqy / tp.eLh : 0.0;
  tp.uxr = tp.velR ? tp.eRqx / tp.eRh : 0.0;
  tp.uyr = tp.velR ? tp.eRqy / tp.eRh : 0.0;
  // hydrostatic reconstruction (2nd order)
  tp.wlA = A.z + A.h;
  tp.wlB = B.z + B.h;
  tp.hiA = tp.wlA >= tp.wlB;
  tp.hi = tp.hiA ? tp.wlA : tp.wlB;
  tp.loA = tp.wlA <= tp.wlB;
  tp.lo = tp.loA ? tp.wlA : tp.wlB;
  {
    const double l0 = tp.eLh + tp.eLz;
    const double l1 = l0 <= tp.hi ? l0 : tp.hi;
    tp.selL1 = l0 <= tp.hi ? 0 : 1;
    tp.Lw = l1 >= tp.lo ? l1 : tp.lo;
    tp.selL2 = l1 >= tp.lo ? 0 : 1;
    const double r0 = tp.eRh + tp.eRz;
    const double r1 = r0 <= tp.hi ? r0 : tp.hi;
    tp.selR1 = r0 <= tp.hi ? 0 : 1;
    tp.Rw = r1 >= tp.lo ? r1 : tp.lo;
    tp.selR2 = r1 >= tp.lo ? 0 : 1;
  }
  tp.Araise = tp.wlA > tp.wlB;
  if (tp.Araise) {
    tp.raiseTookOther = tp.Rw > tp.Lw;
    if (tp.raiseTookOther) tp.Lw = tp.Rw;
  } else {
    tp.raiseTookOther = tp.Lw > tp.Rw;
    if (tp.raiseTookOther) tp.Rw = tp.Lw;
  }
  tp.Lz = tp.Lw - tp.eLh;
  tp.Rz = tp.Rw - tp.eRh;
  tp.zbmL = tp.Lz >= tp.Rz;
  tp.zbm = tp.zbmL ? tp.Lz : tp.Rz;
  tp.Lpos = tp.Lw - tp.zbm > 0.0;
  tp.Rpos = tp.Rw - tp.zbm > 0.0;
  tp.Lh = tp.Lpos ? tp.Lw - tp.zbm : 0.0;
  tp.Rh = tp.Rpos ? tp.Rw - tp.zbm : 0.0;
  const double Lz2 = tp.Lw - tp.Lh, Rz2 = tp.Rw - tp.Rh;
  // rotation
  if (DIR == 0) {
    tp.uL = tp.uxl; tp.vL = tp.uyl; tp.uR = tp.uxr; tp.vR = tp.uyr;
  } else {
    tp.uL = tp.uyl; tp.vL = -tp.uxl; tp.uR = tp.uyr; tp.vR = -tp.uxr;
  }
  // HLLC
  const double hL = tp.Lh, hR = tp.Rh;
  tp.bothdry = (hL < hs && hR < hs);
  double Fh = 0, Fn = 0, Ft = 0;
  if (!tp.bothdry) {
    const double uL = tp.uL, uR = tp.uR, vL = tp.vL, vR = tp.vR;
    const double qxL = uL * hL, qyL = vL * hL, qxR = uR * hR, qyR = vR * hR;
    tp.aL = sqrt(g * hL);
    tp.aR = sqrt(g * hR);
    tp.base = (tp.aL + tp.aR) / 2.0 + (uL - uR) / 4.0;
    tp.ustar = (uL + uR) / 2.0 + tp.aL - tp.aR;
    tp.astar = sqrt(g * ((tp.base * tp.base) / g));
    if (hL <= hs) {
      tp.sLcase = 0;
      tp.sL = uR - 2.0 * tp.aR;
    } else {
      const double a1 = uL - tp.aL, a2 = tp.ustar - tp.astar;
      tp.sLcase = a1 <= a2 ? 1 : 2;
      tp.sL = a1 <= a2 ? a1 : a2;
    }
    if (hR <= hs) {
      tp.sRcase = 0;
      tp.sR = uL + 2.0 * tp.aL;
    } else {
      const double b1 = uR + tp.aR, b2 = tp.ustar + tp.astar;
      tp.sRcase = b1 >= b2 ? 1 : 2;
      tp.sR = b1 >= b2 ? b1 : b2;
    }
    const double sL = tp.sL, sR = tp.sR;
    const double sM = (sL * hR * (uR - sR) - sR * hL * (uL - sL)) / (hR * (uR - sR) - hL * (uL - sL));
    tp.hfL = qxL;
    tp.qfL = uL * qxL + 0.5 * g * hL * hL;
    tp.tfL = uL * qyL;
    tp.hfR = qxR;
    tp.qfR = uR * qxR + 0.5 * g * hR * hR;
    tp.tfR = uR * qyR;
    tp.inv = 1.0 / (sR - sL);
    tp.hfM = (sR * tp.hfL - sL * tp.hfR + sL * sR * (hR - hL)) * tp.inv;
    tp.qfM = (sR * tp.qfL - sL * tp.qfR + sL * sR * (qxR - qxL)) * tp.inv;
    if (0.0 <= sL) tp.region = 0;
    else if (sL < 0.0 && 0.0 <= sM) tp.region = 1;
    else if (sM < 0.0 && 0.0 <= sR) tp.region = 2;
    else tp.region = 3;
    switch (tp.region) {
      case 0: Fh = tp.hfL; Fn = tp.qfL; Ft = tp.tfL; break;
      case 1: Fh = tp.hfM; Fn = tp.qfM; Ft = tp.hfM * vL; break;
      case 2: Fh = tp.hfM; Fn = tp.qfM; Ft = tp.hfM * vR; break;
      default: Fh = tp.hfR; Fn = tp.qfR; Ft = tp.tfR; break;
    }
  }
  o.fh = Fh;
  if (DIR == 0) {
    o.fx = Fn;
    o.fy = Ft;
  } else {
    o.fx = -Ft;
    o.fy = Fn;
  }
  o.sa = 0.5 * g * (A.h + tp.Lh) * (Lz2 - A.z);
  o.sb = 0.5 * g * (B.h + tp.Rh) * (Rz2 - B.z);
  return o;
}

struct FaceBar {
  C3 L, A, B, R;
};

// Adjoint of face_fwd: given dJ/dOut, accumulate dJ/d(h, qx, qy) of L, A, B, R.
template <int DIR>
HB_HD void face_rev(const FaceIn &in, const FaceTape<DIR> &tp, const FaceOut5 &ob, FaceBar &xb) {
  const double hs = kHs, g = kG;
  (void)hs;
  if (tp.skip) return;
  const Cz &A = in.A, &B = in.B;
  // outputs -> Fh, Fn, Ft, sa, sb
  double Fh_b = ob.fh, Fn_b, Ft_b;
  if (DIR == 0) {
    Fn_b = ob.fx;
    Ft_b = ob.fy;
  } else {
    Ft_b = -ob.fx;
    Fn_b = ob.fy;
  }
  // slope terms
  const double Lz2 = tp.Lw - tp.Lh, Rz2 = tp.Rw - tp.Rh;
  double Ah_b = 0, Bh_b = 0;
  double Lh_b = 0, Rh_b = 0, Lw_b = 0, Rw_b = 0;
  {
    // sa = 0.5 g (A.h + Lh)(Lz2 - A.z)
    const double f1 = 0.5 * g * (Lz2 - A.z), f2 = 0.5 * g * (A.h + tp.Lh);
    Ah_b += ob.sa * f1;
    Lh_b += ob.sa * f1;
    Lw_b += ob.sa * f2;   // Lz2 = Lw - Lh
    Lh_b -= ob.sa * f2;
    const double g1 = 0.5 * g * (Rz2 - B.z), g2 = 0.5 * g * (B.h + tp.Rh);
    Bh_b += ob.sb * g1;
    Rh_b += ob.sb * g1;
    Rw_b += ob.sb * g2;
    Rh_b -= ob.sb * g2;
  }
  double uL_b = 0, uR_b = 0, vL_b = 0, vR_b = 0;
  if (!tp.bothdry) {
    const double hL = tp.Lh, hR = tp.Rh, uL = tp.uL, uR = tp.uR, vL = tp.vL, vR = tp.vR;
    const double sL = tp.sL, sR = tp.sR;
    double hfL_b = 0, qfL_b = 0, tfL_b = 0, hfR_b = 0, qfR_b = 0, tfR_b = 0, hfM_b = 0,
           qfM_b = 0;
    switch (tp.region) {
      case 0: hfL_b = Fh_b; qfL_b = Fn_b; tfL_b = Ft_b; break;
      case 1: hfM_b = Fh_b + Ft_b * vL; qfM_b = Fn_b; vL_b += Ft_b * tp.hfM; break;
      case 2: hfM_b = Fh_b + Ft_b * vR; qfM_b = Fn_b; vR_b += Ft_b * tp.hfM; break;
      default: hfR_b = Fh_b; qfR_b = Fn_b; tfR_b = Ft_b; break;
    }
    const double qxL = uL * hL, qxR = uR * hR, qyL = vL * hL, qyR = vR * hR;
    double sL_b = 0, sR_b = 0, qxL_b = 0, qxR_b = 0, qyL_b = 0, qyR_b = 0;
    // hfM = (sR hfL - sL hfR + sL sR (hR - hL)) * inv, inv = 1 / (sR - sL)
    if (hfM_b != 0.0) {
      const double num = sR * tp.hfL - sL * tp.hfR + sL * sR * (hR - hL);
      const double inv = tp.inv;
      hfL_b += hfM_b * sR * inv;
      hfR_b -= hfM_b * sL * inv;
      Rh_b += hfM_b * sL * sR * inv;
      Lh_b -= hfM_b * sL * sR * inv;
      sR_b += hfM_b * (tp.hfL + sL * (hR - hL)) * inv;
      sL_b += hfM_b * (-tp.hfR + sR * (hR - hL)) * inv;
      // d inv / d sR = -inv^2, d inv / d sL = +inv^2
      sR_b -= hfM_b * num * inv * inv;
      sL_b += hfM_b * num * inv * inv;
    }
    if (qfM_b != 0.0) {
      const double num = sR * tp.qfL - sL * tp.qfR + sL * sR * (qxR - qxL);
      const double inv = tp.inv;
      qfL_b += qfM_b * sR * inv;
      qfR_b -= qfM_b * sL * inv;
      qxR_b += qfM_b * sL * sR * inv;
      qxL_b -= qfM_b * sL * sR * inv;
      sR_b += qfM_b * (tp.qfL + sL * (qxR - qxL)) * inv;
      sL_b += qfM_b * (-tp.qfR + sR * (qxR - qxL)) * inv;
      sR_b -= qfM_b * num * inv * inv;
      sL_b += qfM_b * num * inv * inv;
    }
    // hfL = qxL; qfL = uL qxL + 0.5 g hL^2; tfL = uL qyL (same for R)
    qxL_b += hfL_b + qfL_b * uL;
    uL_b += qfL_b * qxL + tfL_b * qyL;
    Lh_b += qfL_b * g * hL;
    qyL_b += tfL_b * uL;
    qxR_b += hfR_b + qfR_b * uR;
    uR_b += qfR_b * qxR + tfR_b * qyR;
    Rh_b += qfR_b * g * hR;
    qyR_b += tfR_b * uR;
    // wave speeds
    double aL_b = 0, aR_b = 0, ustar_b = 0, astar_b = 0;
    if (tp.sLcase == 0) {
      uR_b += sL_b;
      aR_b -= 2.0 * sL_b;
    } else if (tp.sLcase == 1) {
      uL_b += sL_b;
      aL_b -= sL_b;
    } else {
      ustar_b += sL_b;
      astar_b -= sL_b;
    }
    if (tp.sRcase == 0) {
      uL_b += sR_b;
      aL_b += 2.0 * sR_b;
    } else if (tp.sRcase == 1) {
      uR_b += sR_b;
      aR_b += sR_b;
    } else {
      ustar_b += sR_b;
      astar_b += sR_b;
    }
    // astar = sqrt(g * base^2 / g) = |base|
    double base_b = astar_b * (tp.base >= 0.0 ? 1.0 : -1.0);
    // ustar = (uL + uR)/2 + aL - aR
    uL_b += 0.5 * ustar_b;
    uR_b += 0.5 * ustar_b;
    aL_b += ustar_b;
    aR_b -= ustar_b;
    // base = (aL + aR)/2 + (uL - uR)/4
    aL_b += 0.5 * base_b;
    aR_b += 0.5 * base_b;
    uL_b += 0.25 * base_b;
    uR_b -= 0.25 * base_b;
    // a = sqrt(g h)
    if (hL > 0.0) Lh_b += aL_b * g / (2.0 * tp.aL);
    if (hR > 0.0) Rh_b += aR_b * g / (2.0 * tp.aR);
    // qxL = uL hL, qyL = vL hL, ...
    uL_b += qxL_b * hL;
    Lh_b += qxL_b * uL + qyL_b * vL;
    vL_b += qyL_b * hL;
    uR_b += qxR_b * hR;
    Rh_b += qxR_b * uR + qyR_b * vR;
    vR_b += qyR_b * hR;
  }
  // rotation back to x/y velocities
  double uxl_b, uyl_b, uxr_b, uyr_b;
  if (DIR == 0) {
    uxl_b = uL_b; uyl_b = vL_b; uxr_b = uR_b; uyr_b = vR_b;
  } else {
    uyl_b = uL_b; uxl_b = -vL_b; uyr_b = uR_b; uxr_b = -vR_b;
  }
  // hydrostatic reconstruction, in reverse
  double eLh_b = 0, eLz_b = 0, eRh_b = 0, eRz_b = 0, wlA_b = 0, wlB_b = 0;
  // Lh = Lpos ? Lw - zbm : 0
  double zbm_b = 0;
  if (tp.Lpos) {
    Lw_b += Lh_b;
    zbm_b -= Lh_b;
  }
  if (tp.Rpos) {
    Rw_b += Rh_b;
    zbm_b -= Rh_b;
  }
  // zbm = max(Lz, Rz)
  double Lz_b = 0, Rz_b = 0;
  if (tp.zbmL) Lz_b += zbm_b; else Rz_b += zbm_b;
  // Lz = Lw - eLh, Rz = Rw - eRh
  Lw_b += Lz_b;
  eLh_b -= Lz_b;
  Rw_b += Rz_b;
  eRh_b -= Rz_b;
  // raise step
  if (tp.Araise) {
    if (tp.raiseTookOther) { Rw_b += Lw_b; Lw_b = 0; }
  } else {
    if (tp.raiseTookOther) { Lw_b += Rw_b; Rw_b = 0; }
  }
  // clamps: Lw = max(min(l0, hi), lo)
  double hi_b = 0, lo_b = 0;
  {
    double l1_b = 0, l0_b = 0;
    if (tp.selL2 == 0) l1_b = Lw_b; else lo_b += Lw_b;
    if (tp.selL1 == 0) l0_b = l1_b; else hi_b += l1_b;
    eLh_b += l0_b;
    eLz_b += l0_b;
    double r1_b = 0, r0_b = 0;
    if (tp.selR2 == 0) r1_b = Rw_b; else lo_b += Rw_b;
    if (tp.selR1 == 0) r0_b = r1_b; else hi_b += r1_b;
    eRh_b += r0_b;
    eRz_b += r0_b;
  }
  if (tp.hiA) wlA_b += hi_b; else wlB_b += hi_b;
  if (tp.loA) wlA_b += lo_b; else wlB_b += lo_b;
  // wlA = A.z + A.h
  Ah_b += wlA_b;
  Bh_b += wlB_b;
  // velocities: u = q / h (when h >= hs)
  double eLqx_b = 0, eLqy_b = 0, eRqx_b = 0, eRqy_b = 0;
  if (tp.velL) {
    eLqx_b += uxl_b / tp.eLh;
    eLqy_b += uyl_b / tp.eLh;
    eLh_b -= (uxl_b * tp.uxl + uyl_b * tp.uyl) / tp.eLh;
  }
  if (tp.velR) {
    eRqx_b += uxr_b / tp.eRh;
    eRqy_b += uyr_b / tp.eRh;
    eRh_b -= (uxr_b * tp.uxr + uyr_b * tp.uyr) / tp.eRh;
  }
  // edges -> cells and slopes (z has no adjoint: the bed is fixed)
  double sA_b[4] = {0, 0, 0, 0}, sB_b[4] = {0, 0, 0, 0};
  Ah_b += eLh_b;
  sA_b[0] += 0.5 * eLh_b;
  (void)eLz_b;  // only enters through z slopes
  double Aqx_b = 0, Aqy_b = 0, Bqx_b = 0, Bqy_b = 0;
  if (tp.wetA) {
    Aqx_b += eLqx_b;
    sA_b[1] += 0.5 * eLqx_b;
    Aqy_b += eLqy_b;
    sA_b[2] += 0.5 * eLqy_b;
  }
  Bh_b += eRh_b;
  sB_b[0] -= 0.5 * eRh_b;
  (void)eRz_b;
  if (tp.wetB) {
    Bqx_b += eRqx_b;
    sB_b[1] -= 0.5 * eRqx_b;
    Bqy_b += eRqy_b;
    sB_b[2] -= 0.5 * eRqy_b;
  }
  // slopes: sA[f] depends on (L, A, B), sB[f] on (A, B, R); z slopes carry no adjoint
  double Lb[3] = {0, 0, 0}, Ab[3] = {Ah_b, Aqx_b, Aqy_b}, Bb[3] = {Bh_b, Bqx_b, Bqy_b},
         Rb[3] = {0, 0, 0};
  for (int f = 0; f < 3; f++) {
    Lb[f] += sA_b[f] * tp.dA[f][0];
    Ab[f] += sA_b[f] * tp.dA[f][1];
    Bb[f] += sA_b[f] * tp.dA[f][2];
    Ab[f] += sB_b[f] * tp.dB[f][0];
    Bb[f] += sB_b[f] * tp.dB[f][1];
    Rb[f] += sB_b[f] * tp.dB[f][2];
  }
  xb.L.h += Lb[0]; xb.L.qx += Lb[1]; xb.L.qy += Lb[2];
  xb.A.h += Ab[0]; xb.A.qx += Ab[1]; xb.A.qy += Ab[2];
  xb.B.h += Bb[0]; xb.B.qx += Bb[1]; xb.B.qy += Bb[2];
  xb.R.h += Rb[0]; xb.R.qx += Rb[1]; xb.R.qy += Rb[2];
}

// ----------------------------------------------------------------- ghost
// Ghost state of a valid cell C across a no-data neighbour, with outward
// normal along `axis` (0: x, 1: y); types as the reference (3 RIGID,
// 4 WALL_SLIP, 5 OPEN, 6 H_GIVEN, 7 Q_GIVEN, 8 WL_GIVEN).  jac: dG/dC per
// component (h, qx, qy), all diagonal.  Returns false without a ghost rule.
HB_HD bool ghost_of(int type, int axis, const Cz &C, double hb, double wlb, double qxb,
                    double qyb, Cz &G, double jac[3]) {
  const double n0s = axis == 0 ? 1.0 : 0.0, n1s = axis == 0 ? 0.0 : 1.0;
  G = C;
  jac[0] = jac[1] = jac[2] = 1.0;
  switch (type) {
    case 3:
      G.qx = (n1s - n0s) * C.qx; jac[1] = n1s - n0s;
      G.qy = -(n0s - n1s) * C.qy; jac[2] = -(n0s - n1s);
      return true;
    case 4:
      G.qx = (n1s - n0s) * C.qx; jac[1] = n1s - n0s;
      G.qy = (n0s - n1s) * C.qy; jac[2] = n0s - n1s;
      return true;
    case 5:
      return true;
    case 6:
      G.h = hb; jac[0] = 0.0;
      return true;
    case 7:
      G.qx = qxb; G.qy = qyb; jac[1] = jac[2] = 0.0;
      return true;
    case 8: {
      const double wl = wlb > C.z ? wlb : C.z;
      G.h = wl - C.z; jac[0] = 0.0;
      return true;
    }
    default:
      return false;
  }
}

// ------------------------------------------------------------------ cell
// Cell update after the fluxes: h1 = h + hu; implicit Manning friction on
// q + qu with the Froude > 5 limiter (reference form and decisions).
struct CellTape {
  double h1, qxa, qya, n, qn, a, S, f, lim;
  bool dry, fric, actx, acty, limx, limy, zerox, zeroy;
  double tempx, tempy;
};

HB_HD C3 cell_fwd(const C3 &u, const C3 &r, double n, double dt, CellTape &tp) {
  const double hs = kHs, g = kG;
  C3 o;
  tp.h1 = u.h + r.h;
  o.h = tp.h1;
  tp.dry = tp.h1 < hs;
  tp.fric = tp.actx = tp.acty = tp.limx = tp.limy = tp.zerox = tp.zeroy = false;
  if (tp.dry) {
    o.qx = o.qy = 0.0;
    return o;
  }
  const double h = tp.h1;
  tp.n = n;
  const double C_f = g * n * n * pow(h, -1.0 / 3.0);
  tp.qxa = u.qx + r.qx;
  tp.qya = u.qy + r.qy;
  tp.qn = sqrt(tp.qxa * tp.qxa + tp.qya * tp.qya);
  o.qx = tp.qxa;
  o.qy = tp.qya;
  if (!(n > 0.0)) return o;
  tp.fric = true;
  tp.a = dt * C_f / (h * h);
  tp.S = sqrt(1.0 + 4.0 * tp.a * tp.qn);
  tp.f = 2.0 / (1.0 + tp.S);
  tp.lim = 5.0 * h * sqrt(h * g);
  if (fabs(tp.qxa) > 1.0e-10) {
    tp.actx = true;
    const double temp = (1.0 - sqrt(1.0 + (4.0 * dt * C_f) / (h * h) * tp.qn)) /
                        (-2.0 * dt * C_f / (h * h) * (tp.qn / tp.qxa));
    tp.tempx = temp;
    if (fabs(temp) > tp.lim) {
      tp.limx = true;
      o.qx = 2.0 * temp - tp.qxa;
      if (o.qx * temp <= 0.0) {
        tp.zerox = true;
        o.qx = 0.0;
      }
    } else {
      o.qx = temp;
    }
  }
  if (fabs(tp.qya) > 1.0e-10) {
    tp.acty = true;
    const double temp = (1.0 - sqrt(1.0 + (4.0 * dt * C_f) / (h * h) * tp.qn)) /
                        (-2.0 * dt * C_f / (h * h) * (tp.qn / tp.qya));
    tp.tempy = temp;
    if (fabs(temp) > tp.lim) {
      tp.limy = true;
      o.qy = 2.0 * temp - tp.qya;
      if (o.qy * temp <= 0.0) {
        tp.zeroy = true;
        o.qy = 0.0;
      }
    } else {
      o.qy = temp;
    }
  }
  return o;
}

// Adjoint of cell_fwd: from dJ/dOut, dJ/du (through the state), dJ/dr (the
// flux + source increments) and dJ/dn.
HB_HD void cell_rev(const CellTape &tp, const C3 &ob, double dt, C3 &ub, C3 &rb, double &nb) {
  double h1_b = ob.h;
  double qxa_b = 0, qya_b = 0;
  nb = 0.0;
  if (!tp.dry) {
    if (!tp.fric) {
      qxa_b = ob.qx;
      qya_b = ob.qy;
    } else {
      // temp_c = qca * f(a, qn), f = 2 / (1 + S), S = sqrt(1 + 4 a qn)
      double tx_b = 0, ty_b = 0;
      if (tp.actx) {
        if (tp.limx) {
          if (!tp.zerox) {
            tx_b += 2.0 * ob.qx;
            qxa_b -= ob.qx;
          }
        } else {
          tx_b += ob.qx;
        }
      } else {
        qxa_b += ob.qx;
      }
      if (tp.acty) {
        if (tp.limy) {
          if (!tp.zeroy) {
            ty_b += 2.0 * ob.qy;
            qya_b -= ob.qy;
          }
        } else {
          ty_b += ob.qy;
        }
      } else {
        qya_b += ob.qy;
      }
      const double f_b = tx_b * tp.qxa + ty_b * tp.qya;
      qxa_b += tx_b * tp.f;
      qya_b += ty_b * tp.f;
      // f = 2/(1+S): df/dS = -2/(1+S)^2; S = sqrt(1 + 4 a qn): dS/d(a qn) = 2/S
      const double x_b = f_b * (-2.0 / ((1.0 + tp.S) * (1.0 + tp.S))) * (2.0 / tp.S);
      const double a_b = x_b * tp.qn;
      const double qn_b = x_b * tp.a;
      if (tp.qn > 0.0) {
        qxa_b += qn_b * tp.qxa / tp.qn;
        qya_b += qn_b * tp.qya / tp.qn;
      }
      // a = dt g n^2 h^(-7/3)
      h1_b += a_b * tp.a * (-7.0 / 3.0) / tp.h1;
      nb += a_b * tp.a * 2.0 / tp.n;
    }
  }
  (void)dt;
  ub.h = h1_b;
  rb.h = h1_b;
  ub.qx = qxa_b;
  rb.qx = qxa_b;
  ub.qy = qya_b;
  rb.qy = qya_b;
}

}  // namespace adj
}  // namespace hb
