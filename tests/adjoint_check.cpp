// Host harness for tests/test_adjoint_math.py: exposes the adjoint header's
// forward and reverse functions (compiled for the CPU) to ctypes.
#include <cmath>
#include <cstring>

#include "hb_adjoint.cuh"

using namespace hb::adj;

static FaceIn make_in(const double *x, int vL, int vR, int noslope) {
  // x: L(h,qx,qy,z) A(...) B(...) R(...)
  FaceIn in;
  in.L = Cz{x[0], x[1], x[2], x[3]};
  in.A = Cz{x[4], x[5], x[6], x[7]};
  in.B = Cz{x[8], x[9], x[10], x[11]};
  in.R = Cz{x[12], x[13], x[14], x[15]};
  in.vL = vL;
  in.vR = vR;
  in.noslope = noslope;
  return in;
}

extern "C" void face_fwd_c(int dir, const double *x, int vL, int vR, int noslope, double *out) {
  FaceIn in = make_in(x, vL, vR, noslope);
  FaceOut5 o;
  if (dir == 0) {
    FaceTape<0> tp;
    o = face_fwd<0>(in, tp);
  } else {
    FaceTape<1> tp;
    o = face_fwd<1>(in, tp);
  }
  out[0] = o.fh; out[1] = o.fx; out[2] = o.fy; out[3] = o.sa; out[4] = o.sb;
}

extern "C" void face_vjp_c(int dir, const double *x, int vL, int vR, int noslope,
                           const double *ob, double *xb /* 12: L,A,B,R x (h,qx,qy) */) {
  FaceIn in = make_in(x, vL, vR, noslope);
  FaceOut5 b{ob[0], ob[1], ob[2], ob[3], ob[4]};
  FaceBar bar{};
  if (dir == 0) {
    FaceTape<0> tp;
    face_fwd<0>(in, tp);
    face_rev<0>(in, tp, b, bar);
  } else {
    FaceTape<1> tp;
    face_fwd<1>(in, tp);
    face_rev<1>(in, tp, b, bar);
  }
  const C3 *c[4] = {&bar.L, &bar.A, &bar.B, &bar.R};
  for (int k = 0; k < 4; k++) {
    xb[3 * k] = c[k]->h;
    xb[3 * k + 1] = c[k]->qx;
    xb[3 * k + 2] = c[k]->qy;
  }
}

extern "C" void cell_fwd_c(const double *u, const double *r, double n, double dt, double *out) {
  CellTape tp;
  C3 o = cell_fwd(C3{u[0], u[1], u[2]}, C3{r[0], r[1], r[2]}, n, dt, tp);
  out[0] = o.h; out[1] = o.qx; out[2] = o.qy;
}

extern "C" void cell_vjp_c(const double *u, const double *r, double n, double dt,
                           const double *ob, double *ub, double *rb, double *nb) {
  CellTape tp;
  cell_fwd(C3{u[0], u[1], u[2]}, C3{r[0], r[1], r[2]}, n, dt, tp);
  C3 U, Rr;
  cell_rev(tp, C3{ob[0], ob[1], ob[2]}, dt, U, Rr, *nb);
  ub[0] = U.h; ub[1] = U.qx; ub[2] = U.qy;
  rb[0] = Rr.h; rb[1] = Rr.qx; rb[2] = Rr.qy;
}
