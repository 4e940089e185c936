// hb_adjoint.cu -- discrete adjoint of the FP64 fused HiPIMS step.
//
// For a loss J of the states, given lambda^{n+1} = dJ/dU^{n+1} it returns
// lambda^n = (dU^{n+1}/dU^n)^T lambda^{n+1} and accumulates
// (dU^{n+1}/dtheta)^T lambda^{n+1} for theta = (Manning n of each zone, rain
// multiplier), with the time step frozen (the forward's dt schedule replayed).
// Two passes per step over the dense raster of one catchment:
//  1. cells: recompute the cell's four faces and its update, reverse the
//     update (friction, rain), write the direct part of lambda^n and mu =
//     dJ/d(flux increments) of active cells;
//  2. faces: every face once, owned by its east / south cell; reverse it with
//     the adjoints of its two cells' increments and scatter the result to its
//     four input cells with FP64 atomics.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "hb_adjoint.cuh"
#include "hb_common.cuh"
#include "hb_physics.cuh"
#include "hipims_b200.h"
#include "hipims_b200_fused.h"

static_assert(sizeof(hb_adjoint_args) == 184, "hb_adjoint_args layout (ctypes mirror)");

namespace hb {
namespace {

using namespace adj;

struct Grid {
  const hb_instance *in;
  int rows, cols, P, CP;
  const double *h, *qx, *qy, *z;
  const uint8_t *code;
  __device__ __forceinline__ size_t off(int r, int c) const {
    return (size_t)(r + HB_PAD_Y) * P + (c + HB_PAD_X);
  }
  __device__ __forceinline__ uint8_t cd(int r, int c) const {
    if (r < 0 || c < 0 || r >= rows || c >= cols) return (uint8_t)(HB_NODATA_CLASS << 4);
    return code[(size_t)(r + HB_PAD_Y) * CP + (c + HB_CODE_PAD_X)];
  }
  __device__ __forceinline__ bool valid(int r, int c) const {
    return (cd(r, c) >> 4) != HB_NODATA_CLASS;
  }
  __device__ __forceinline__ Cz cell(int r, int c) const {
    Cz v{0, 0, 0, 0};
    if (r < -HB_PAD_Y || c < -HB_PAD_X || r >= rows + 2 || c >= cols + 2) return v;
    const size_t k = off(r, c);
    v.h = h[k];
    v.qx = qx[k];
    v.qy = qy[k];
    v.z = z[k];
    return v;
  }
};

struct BcVals {
  double v[HB_MAX_CLASSES][4];
  int type[HB_MAX_CLASSES];
};

__device__ void load_bc(const hb_instance &in, double t, BcVals &bc) {
  const int k = threadIdx.x + threadIdx.y * blockDim.x;
  if (k >= HB_MAX_CLASSES) return;
  const int id = in.bc_id[k];
  double hb = 0, wlb = 0, qxb = 0, qyb = 0;
  if (in.given_depth && id + 1 < in.depth_cols) {
    const int tl = timelevel(t, in.given_depth, in.depth_rows, in.depth_cols);
    hb = in.given_depth[(int64_t)tl * in.depth_cols + id + 1];
  }
  if (in.given_wl && id + 1 < in.wl_cols) {
    const int tl = timelevel(t, in.given_wl, in.wl_rows, in.wl_cols);
    wlb = in.given_wl[(int64_t)tl * in.wl_cols + id + 1];
  }
  if (in.given_q && 2 + 2 * id < in.q_cols) {
    const int tl = timelevel(t, in.given_q, in.q_rows, in.q_cols);
    qxb = in.given_q[(int64_t)tl * in.q_cols + 1 + 2 * id];
    qyb = in.given_q[(int64_t)tl * in.q_cols + 2 + 2 * id];
  }
  bc.v[k][0] = hb;
  bc.v[k][1] = wlb;
  bc.v[k][2] = qxb;
  bc.v[k][3] = qyb;
  bc.type[k] = in.bc_type[k];
}

// Face (A at (ra, ca) minus side, B at (rb, cb) plus side) along DIR, any
// validity.  Forward only when bar == nullptr; otherwise reverse with the
// output adjoint `ob` and scatter into lam (atomics).
template <int DIR>
__device__ FaceOut5 face_at(const Grid &G, const BcVals &bc, int ra, int ca, int rb, int cb,
                            const FaceOut5 *ob, double *lh, double *lqx, double *lqy,
                            double hreg = 0.0) {
  const int dr = rb - ra, dc = cb - ca;  // unit step from A to B
  const bool va = G.valid(ra, ca), vb = G.valid(rb, cb);
  FaceOut5 o{0, 0, 0, 0, 0};
  if (!va && !vb) return o;
  FaceIn fi;
  FaceTape<DIR> tp;
  int rL = ra - dr, cL = ca - dc, rR = rb + dr, cR = cb + dc;
  double jac[3] = {1, 1, 1};
  bool ghostA = false, ghostB = false;
  if (va && vb) {
    fi.A = G.cell(ra, ca);
    fi.B = G.cell(rb, cb);
    fi.L = G.cell(rL, cL);
    fi.R = G.cell(rR, cR);
    fi.vL = G.valid(rL, cL);
    fi.vR = G.valid(rR, cR);
    fi.noslope = false;
  } else {
    // boundary face: the valid cell against its ghost, no reconstruction
    const int rc = va ? ra : rb, cc = va ? ca : cb;
    const Cz C = G.cell(rc, cc);
    const int cls = G.cd(rc, cc) >> 4;
    Cz Gh;
    if (!ghost_of(bc.type[cls], DIR, C, bc.v[cls][0], bc.v[cls][1], bc.v[cls][2],
                  bc.v[cls][3], Gh, jac))
      return o;
    fi.A = va ? C : Gh;
    fi.B = va ? Gh : C;
    fi.L = fi.A;
    fi.R = fi.B;
    fi.vL = fi.vR = false;
    fi.noslope = true;
    ghostA = !va;
    ghostB = !vb;
  }
  o = face_fwd<DIR>(fi, tp);
  if (!ob) return o;
  FaceBar xb{};
  face_rev<DIR>(fi, tp, *ob, xb);
  auto add = [&](int r, int c, const C3 &v) {
    if (!G.valid(r, c)) return;
    const size_t k = G.off(r, c);
    if (G.h[k] < hreg) return;  // masked cell: its state adjoint stays zero
    if (v.h != 0.0) atomicAdd(lh + k, v.h);
    if (v.qx != 0.0) atomicAdd(lqx + k, v.qx);
    if (v.qy != 0.0) atomicAdd(lqy + k, v.qy);
  };
  if (va && vb) {
    add(rL, cL, xb.L);
    add(ra, ca, xb.A);
    add(rb, cb, xb.B);
    add(rR, cR, xb.R);
  } else {
    // only the valid cell receives: directly, and through its ghost
    C3 c = ghostA ? xb.B : xb.A;
    const C3 gb = ghostA ? xb.A : xb.B;
    c.h += gb.h * jac[0];
    c.qx += gb.qx * jac[1];
    c.qy += gb.qy * jac[2];
    add(va ? ra : rb, va ? ca : cb, c);
  }
  return o;
}

// Face values kept by the optional face pass: x-face (r, c-1)|(r, c) and
// y-face (r, c)|(r-1, c) of index r * (cols + 1) + c, fields fh, fx, fy, sa, sb.
__device__ __forceinline__ FaceOut5 load_face(const hb_adjoint_args &a, int dir, int r, int c) {
  const double *f = a.faces + (size_t)dir * 5 * a.face_stride + (size_t)r * (a.cols + 1) + c;
  const int64_t s = a.face_stride;
  return FaceOut5{f[0], f[s], f[2 * s], f[3 * s], f[4 * s]};
}

// Pass 0 (optional): every face once, forward only, into a.faces.
__global__ void __launch_bounds__(128)
adj_facefwd_kernel(hb_adjoint_args a) {
  __shared__ BcVals bc;
  const hb_instance &in = *a.instance;
  Grid G{a.instance, a.rows, a.cols, a.pitch, a.code_pitch, a.h, a.qx, a.qy,
         (const double *)in.z, in.code};
  load_bc(in, a.t, bc);
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (r > a.rows || c > a.cols) return;
  const size_t idx = (size_t)r * (a.cols + 1) + c;
  const int64_t s = a.face_stride;
  FaceOut5 x{0, 0, 0, 0, 0}, y{0, 0, 0, 0, 0};
  if (r < a.rows) x = face_at<0>(G, bc, r, c - 1, r, c, nullptr, nullptr, nullptr, nullptr);
  if (c < a.cols) y = face_at<1>(G, bc, r, c, r - 1, c, nullptr, nullptr, nullptr, nullptr);
  double *fx = a.faces + idx, *fy = a.faces + 5 * s + idx;
  fx[0] = x.fh; fx[s] = x.fx; fx[2 * s] = x.fy; fx[3 * s] = x.sa; fx[4 * s] = x.sb;
  fy[0] = y.fh; fy[s] = y.fx; fy[2 * s] = y.fy; fy[3 * s] = y.sa; fy[4 * s] = y.sb;
}

// Pass 1: per cell.
__global__ void __launch_bounds__(256)
adj_cell_kernel(hb_adjoint_args a) {
  __shared__ BcVals bc;
  __shared__ double red[HB_MAX_ZONES + 1][8];
  const hb_instance &in = *a.instance;
  Grid G{a.instance, a.rows, a.cols, a.pitch, a.code_pitch, a.h, a.qx, a.qy,
         (const double *)in.z, in.code};
  load_bc(in, a.t, bc);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  if (tid < (HB_MAX_ZONES + 1) * 8) (&red[0][0])[tid] = 0.0;
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  double gz = 0.0, gm = 0.0;
  int zone = 0;
  if (r < a.rows && c < a.cols) {
    const size_t k = G.off(r, c);
    double *mu_h = a.mu, *mu_qx = a.mu + a.mu_stride, *mu_qy = a.mu + 2 * a.mu_stride;
    if (!G.valid(r, c)) {
      a.out_h[k] = a.out_qx[k] = a.out_qy[k] = 0.0;
      mu_h[k] = mu_qx[k] = mu_qy[k] = 0.0;
    } else {
      const Cz u = G.cell(r, c);
      const double hs = kHs;
      // fluxMask activity (HC/fluxMaskGenerator_Kernel.cu:19-42, cell 0 ignored)
      bool active = a.first || u.h > hs;
      const int nr[4] = {r, r - 1, r, r + 1}, nc[4] = {c + 1, c, c - 1, c};
      for (int d = 0; d < 4 && !active; d++) {
        const bool bug = (nr[d] == in.bug_y && nc[d] == in.bug_x);
        if (G.valid(nr[d], nc[d]) && !bug && G.cell(nr[d], nc[d]).h > hs) active = true;
      }
      const double kk = a.dt / in.dx;
      C3 rr{0, 0, 0};
      if (active) {
        FaceOut5 fe, fw, fn, fs;
        if (a.faces) {
          fe = load_face(a, 0, r, c + 1);
          fw = load_face(a, 0, r, c);
          fn = load_face(a, 1, r, c);
          fs = load_face(a, 1, r + 1, c);
        } else {
          fe = face_at<0>(G, bc, r, c, r, c + 1, nullptr, nullptr, nullptr, nullptr);
          fw = face_at<0>(G, bc, r, c - 1, r, c, nullptr, nullptr, nullptr, nullptr);
          fn = face_at<1>(G, bc, r, c, r - 1, c, nullptr, nullptr, nullptr, nullptr);
          fs = face_at<1>(G, bc, r + 1, c, r, c, nullptr, nullptr, nullptr, nullptr);
        }
        rr.h = ((fw.fh + fs.fh) - (fe.fh + fn.fh)) * kk;
        rr.qx = ((fw.fx + fs.fx) - (fe.fx + fn.fx) - fe.sa + fw.sb) * kk;
        rr.qy = ((fw.fy + fs.fy) - (fe.fy + fn.fy) - fn.sa + fs.sb) * kk;
      }
      rr.h += a.rain_rate * a.dt;
      zone = G.cd(r, c) & 15;
      const double n = in.manning[zone];
      CellTape tp;
      const C3 uu{u.h, u.qx, u.qy};
      cell_fwd(uu, rr, n, a.dt, tp);
      const C3 ob{a.lam_h[k], a.lam_qx[k], a.lam_qy[k]};
      C3 ub, rb;
      double nb;
      cell_rev(tp, ob, a.dt, ub, rb, nb);
      // Below h_reg the cell's state adjoint is held at zero.  The step never
      // clamps h >= 0 (as the reference); negative depths and films of a few
      // h_small on bumps between deeper cells, with discharges at rounding
      // level, have linearised gains above one per step that the nonlinear
      // step saturates, so the exact adjoint through them grows without bound.
      const bool keep = !(u.h < a.h_reg);
      a.out_h[k] = keep ? ub.h : 0.0;
      a.out_qx[k] = keep ? ub.qx : 0.0;
      a.out_qy[k] = keep ? ub.qy : 0.0;
      mu_h[k] = active ? rb.h : 0.0;
      mu_qx[k] = active ? rb.qx : 0.0;
      mu_qy[k] = active ? rb.qy : 0.0;
      gz = nb;
      gm = rb.h * a.rain_base * a.dt;
    }
  }
  // block reduction of the parameter gradient (zones are few)
  const int lane = tid & 31, wid = tid >> 5;
  for (int zz = 0; zz < HB_MAX_ZONES; zz++) {
    double v = (zone == zz) ? gz : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[zz][wid] = v;
  }
  for (int o = 16; o > 0; o >>= 1) gm += __shfl_xor_sync(0xffffffffu, gm, o);
  if (lane == 0) red[HB_MAX_ZONES][wid] = gm;
  __syncthreads();
  if (tid <= HB_MAX_ZONES) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; w++) v += red[tid][w];
    if (v != 0.0) atomicAdd(a.grad + tid, v);
  }
}

// Pass 2: per face, owned by its east (x) / south (y) cell.
__global__ void __launch_bounds__(128)
adj_face_kernel(hb_adjoint_args a) {
  __shared__ BcVals bc;
  const hb_instance &in = *a.instance;
  Grid G{a.instance, a.rows, a.cols, a.pitch, a.code_pitch, a.h, a.qx, a.qy,
         (const double *)in.z, in.code};
  load_bc(in, a.t, bc);
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (r > a.rows || c > a.cols) return;
  const double kk = a.dt / in.dx;
  const double *mu_h = a.mu, *mu_qx = a.mu + a.mu_stride, *mu_qy = a.mu + 2 * a.mu_stride;
  auto mu = [&](int rr, int cc) {
    C3 m{0, 0, 0};
    if (rr >= 0 && cc >= 0 && rr < a.rows && cc < a.cols && G.valid(rr, cc)) {
      const size_t k = G.off(rr, cc);
      m = C3{mu_h[k], mu_qx[k], mu_qy[k]};
    }
    return m;
  };
  // x-face between (r, c-1) = A and (r, c) = B
  if (r < a.rows) {
    const C3 mA = mu(r, c - 1), mB = mu(r, c);
    const FaceOut5 ob{kk * (mB.h - mA.h), kk * (mB.qx - mA.qx), kk * (mB.qy - mA.qy),
                      -kk * mA.qx, kk * mB.qx};
    if (ob.fh != 0.0 || ob.fx != 0.0 || ob.fy != 0.0 || ob.sa != 0.0 || ob.sb != 0.0)
      face_at<0>(G, bc, r, c - 1, r, c, &ob, a.out_h, a.out_qx, a.out_qy, a.h_reg);
  }
  // y-face between (r, c) = A (south) and (r - 1, c) = B (north)
  if (c < a.cols) {
    const C3 mA = mu(r, c), mB = mu(r - 1, c);
    const FaceOut5 ob{kk * (mB.h - mA.h), kk * (mB.qx - mA.qx), kk * (mB.qy - mA.qy),
                      -kk * mA.qy, kk * mB.qy};
    if (ob.fh != 0.0 || ob.fx != 0.0 || ob.fy != 0.0 || ob.sa != 0.0 || ob.sb != 0.0)
      face_at<1>(G, bc, r, c, r - 1, c, &ob, a.out_h, a.out_qx, a.out_qy, a.h_reg);
  }
}

__global__ void gauge_kernel(int64_t n, const int64_t *off, const double *h, const double *obs,
                             double *lam_h, double w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(lam_h + off[i], 2.0 * w * (h[off[i]] - obs[i]));
}

}  // namespace
}  // namespace hb

using namespace hb;

extern "C" int hb_adjoint_step(const hb_adjoint_args *a, void *stream) {
  if (!a || !a->instance || !a->h || !a->qx || !a->qy || !a->lam_h || !a->lam_qx ||
      !a->lam_qy || !a->out_h || !a->out_qx || !a->out_qy || !a->mu || !a->grad)
    return set_error(HB_ERR_ARG, "hb_adjoint_step: null pointer");
  if (a->rows <= 0 || a->cols <= 0 || a->pitch < a->cols + 8 || a->mu_stride <= 0)
    return set_error(HB_ERR_ARG, "hb_adjoint_step: bad geometry");
  if (a->faces && a->face_stride < (int64_t)(a->rows + 1) * (a->cols + 1))
    return set_error(HB_ERR_ARG, "hb_adjoint_step: face_stride below (rows + 1) * (cols + 1)");
  auto st = as_stream(stream);
  if (a->faces) {
    const dim3 blk0(32, 4);
    const dim3 g0((a->cols + 1 + 31) / 32, (a->rows + 1 + 3) / 4);
    adj_facefwd_kernel<<<g0, blk0, 0, st>>>(*a);
    int rc0 = check_launch("hb_adjoint_step (faces forward)");
    if (rc0) return rc0;
  }
  const dim3 blk(32, 8);
  const dim3 g1((a->cols + 31) / 32, (a->rows + 7) / 8);
  adj_cell_kernel<<<g1, blk, 0, st>>>(*a);
  int rc = check_launch("hb_adjoint_step (cells)");
  if (rc) return rc;
  // 128-thread blocks: the face pass needs ~156 registers a thread, so three
  // blocks (12 warps) fit an SM where one 256-thread block would
  const dim3 blk2(32, 4);
  const dim3 g2((a->cols + 1 + 31) / 32, (a->rows + 1 + 3) / 4);
  adj_face_kernel<<<g2, blk2, 0, st>>>(*a);
  return check_launch("hb_adjoint_step (faces)");
}

extern "C" int hb_adjoint_gauge(int64_t n, const int64_t *offsets, const double *h,
                                const double *obs, double *lam_h, double weight, void *stream) {
  if (n < 0) return set_error(HB_ERR_ARG, "hb_adjoint_gauge: negative n");
  if (n == 0) return HB_OK;
  if (!offsets || !h || !obs || !lam_h) return set_error(HB_ERR_ARG, "hb_adjoint_gauge: null");
  gauge_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(n, offsets, h, obs, lam_h,
                                                                   weight);
  return check_launch("hb_adjoint_gauge");
}
