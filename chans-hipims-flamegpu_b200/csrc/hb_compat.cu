// hb_compat.cu -- the reference's torch-extension op surface as C-ABI entry
// points over caller-owned device arrays, for FP32 and FP64.
//
// Same compacted-cell layout, neighbour table and in-place semantics as the
// reference ops (paths relative to CHANS-HiPIMS/hipims/cuda):
//   hb_flux             fluxCal_2ndOrder_jh_improved.cpp:28-53  (order 2)
//                       fluxCal_jh_modified_surface.cpp:28-53   (order 1)
//   hb_friction_update  friction_implicit_andUpdate_jh_interface.cpp:29-53
//   hb_timestep         timeControl.cpp:27-41
//   hb_rain_station     stationPrecipitation_interface.cpp:26-38
//   hb_flux_mask        fluxMaskGenerator.cpp:22-29
//   hb_euler_update     euler_update.cpp:27-44
//   hb_infiltration     infiltration_interface.cpp (Green-Ampt)
// This file is compiled with -fmad=false so that FP64 results follow the
// reference's operation order without contraction.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "hb_common.cuh"
#include "hb_physics.cuh"

namespace hb {
namespace {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ Cell<T> load_cell(const T *__restrict__ h,
                                             const T *__restrict__ wl,
                                             const T *__restrict__ qx,
                                             const T *__restrict__ qy,
                                             const T *__restrict__ z, int64_t i) {
  Cell<T> c;
  c.h = __ldg(h + i);
  c.wl = __ldg(wl + i);
  c.qx = __ldg(qx + i);
  c.qy = __ldg(qy + i);
  c.z = __ldg(z + i);
  return c;
}

// Per active cell, its four faces E, N, W, S in order; each face is computed
// from this cell's side (the reference's scheme), accumulating -dt/dx * F and
// the bed-slope source into the update arrays.
template <typename T, int ORDER>
__global__ void __launch_bounds__(kThreads)
flux_kernel(int64_t M, int64_t N, const int32_t *__restrict__ wet,
            T *__restrict__ h_flux, T *__restrict__ qx_flux, T *__restrict__ qy_flux,
            const T *__restrict__ h, const T *__restrict__ wl, const T *__restrict__ z,
            const T *__restrict__ qx, const T *__restrict__ qy,
            const int32_t *__restrict__ index, const T *__restrict__ normal,
            const T *__restrict__ gd, int dr, int dc, const T *__restrict__ gw, int wr,
            int wc, const T *__restrict__ gq, int qr, int qc, const T *__restrict__ dxp,
            const T *__restrict__ tp, const T *__restrict__ dtp) {
  int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= M) return;
  const T hs = T(kHSmall), g = T(kG);
  const T dx = dxp[0], dt = dtp[0];
  const double t = (double)tp[0];
  const int tl_d = timelevel(t, gd, dr, dc);
  const int tl_w = timelevel(t, gw, wr, wc);
  const int tl_q = timelevel(t, gq, qr, qc);
  const int32_t i = wet[w];
  const int32_t c_type = index[i];
  T fh = h_flux[i], fqx = qx_flux[i], fqy = qy_flux[i];
  for (int j = 0; j < 4; j++) {
    Cell<T> c = load_cell(h, wl, qx, qy, z, i);
    const T n0 = normal[j * 2], n1 = normal[j * 2 + 1];
    const T t0 = -n1, t1 = n0;
    const int rdir = j + 1;
    const int ldir = (rdir + 2) > 4 ? rdir - 2 : rdir + 2;
    const int32_t l_id = index[(int64_t)ldir * N + i];
    const int32_t r_id = index[(int64_t)rdir * N + i];
    Cell<T> r, eL, eR;
    T c_h = c.h, c_z = c.z;  // raw cell values for the 1st-order scheme
    T r_h = T(0), r_z = T(0);
    if (r_id == -1) {
      int bt, bid;
      decode_bc(c_type, bt, bid);
      // Table columns beyond the given width read as 0 (the reference reads
      // past the row there).
      T hb = bid + 1 < dc ? gd[(int64_t)tl_d * dc + bid + 1] : T(0);
      T wlb = bid + 1 < wc ? gw[(int64_t)tl_w * wc + bid + 1] : T(0);
      T qxb = 2 + 2 * bid < qc ? gq[(int64_t)tl_q * qc + 1 + 2 * bid] : T(0);
      T qyb = 2 + 2 * bid < qc ? gq[(int64_t)tl_q * qc + 2 + 2 * bid] : T(0);
      if (!ghost(bt, ORDER == 1, c, n0, n1, hb, wlb, qxb, qyb, r)) continue;
      r_h = r.h;
      r_z = r.z;
      eL = c;
      eR = r;
    } else if (ORDER == 2) {
      Cell<T> l = (l_id == -1) ? c : load_cell(h, wl, qx, qy, z, l_id);
      const int32_t rr_id = index[(int64_t)rdir * N + r_id];
      r = load_cell(h, wl, qx, qy, z, r_id);
      Cell<T> rr = (rr_id == -1) ? r : load_cell(h, wl, qx, qy, z, rr_id);
      muscl(c, l, r, eL);
      muscl(r, rr, c, eR);
    } else {
      const T l_z = (l_id == -1) ? c.z : __ldg(z + l_id);
      const int32_t rr_id = index[(int64_t)rdir * N + r_id];
      const T rr_z = (rr_id == -1) ? __ldg(z + r_id) : __ldg(z + rr_id);
      r = load_cell(h, wl, qx, qy, z, r_id);
      r_h = r.h;
      r_z = r.z;
      T rb = minmod(c.z - l_z, r.z - c.z);
      if (r.h > hs) c.z += T(0.5) * rb;
      rb = minmod(r.z - rr_z, c_z - r.z);
      if (c.h > hs) r.z += T(0.5) * rb;
      eL = c;
      eR = r;
    }
    if (c.h < hs && r.h < hs) continue;
    // velocities of the edge states before the hydrostatic step
    const T ux_l = eL.h < hs ? T(0) : eL.qx / eL.h;
    const T uy_l = eL.h < hs ? T(0) : eL.qy / eL.h;
    const T ux_r = eR.h < hs ? T(0) : eR.qx / eR.h;
    const T uy_r = eR.h < hs ? T(0) : eR.qy / eR.h;
    if (ORDER == 2)
      hydro2(c.wl, r.wl, eL, eR);
    else
      hydro1(c_h, c_z, r_h, r_z, eL, eR);
    const T u_L = ux_l * n0 + uy_l * n1;
    const T u_R = ux_r * n0 + uy_r * n1;
    const T v_L = -ux_l * n1 + uy_l * n0;
    const T v_R = -ux_r * n1 + uy_r * n0;
    T Fh, Fn, Ft;
    if (hllc<T, false>(eL.h, eR.h, u_L, u_R, v_L, v_R, Fh, Fn, Ft)) {
      fh -= (Fh / dx) * dt;
      fqx -= ((Fn * n0 + Ft * t0) / dx) * dt;
      fqy -= ((Fn * n1 + Ft * t1) / dx) * dt;
    }
    if (ORDER == 2) {
      fqx -= ((T(0.5) * g * (c.h + eL.h) * (eL.z - c.z) * n0) / dx) * dt;
      fqy -= ((T(0.5) * g * (c.h + eL.h) * (eL.z - c.z) * n1) / dx) * dt;
    } else {
      fqx -= ((T(0.5) * g * (eL.h + c_h) * (eL.z - c_z) * n0) / dx) * dt;
      fqy -= ((T(0.5) * g * (eL.h + c_h) * (eL.z - c_z) * n1) / dx) * dt;
    }
  }
  h_flux[i] = fh;
  qx_flux[i] = fqx;
  qy_flux[i] = fqy;
}

// Implicit Manning friction + Euler update, zeroing the accumulators.  The
// reference kernel writes this step with double literals, so its FP32 build
// evaluates C_f and the implicit update in double; D below reproduces those
// promotions (for T = double it changes nothing).
template <typename T>
__global__ void __launch_bounds__(kThreads)
friction_update_kernel(int64_t M, const int32_t *__restrict__ wet, T *__restrict__ hu,
                       T *__restrict__ qxu, T *__restrict__ qyu, T *__restrict__ zu,
                       const uint8_t *__restrict__ landuse, T *__restrict__ hp,
                       T *__restrict__ wlp, T *__restrict__ qxp, T *__restrict__ qyp,
                       T *__restrict__ zp, const T *__restrict__ manning,
                       const T *__restrict__ dtp) {
  using D = double;
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const T hs = T(kHSmall), g = T(kG), dt = dtp[0];
  const int32_t i = wet[j];
  T h = hp[i] + hu[i];
  T qx = qxp[i], qy = qyp[i];
  if (h < hs) {
    qx = T(0);
    qy = T(0);
  } else {
    const T n = manning[landuse[i]];
    const T C_f = (T)((D)(g * n * n) * pow((D)h, -1.0 / 3.0));
    qx += qxu[i];
    qy += qyu[i];
    const T q_norm = sqrt(qx * qx + qy * qy);
    const T h2 = h * h;
    const D lim = 5.0 * (D)h * (D)sqrt(h * g);
    if (n > T(0)) {
      if (fabs(qx) > T(1.0e-10)) {
        const D temp = (1.0 - sqrt(1.0 + (4.0 * (D)dt * (D)C_f) / (D)h2 * (D)q_norm)) /
                       (-2.0 * (D)dt * (D)C_f / (D)h2 * (D)(q_norm / qx));
        if (fabs(temp) > lim) {
          qx = (T)(2.0 * temp - (D)qx);
          if ((D)qx * temp <= 0.0) qx = T(0);
        } else {
          qx = (T)temp;
        }
      }
      if (fabs(qy) > T(1.0e-10)) {
        const D temp = (1.0 - sqrt(1.0 + (4.0 * (D)dt * (D)C_f) / (D)h2 * (D)q_norm)) /
                       (-2.0 * (D)dt * (D)C_f / (D)h2 * (D)(q_norm / qy));
        if (fabs(temp) > lim) {
          qy = (T)(2.0 * temp - (D)qy);
          if ((D)qy * temp <= 0.0) qy = T(0);
        } else {
          qy = (T)temp;
        }
      }
    }
  }
  const T z = zp[i] + zu[i];
  hp[i] = h;
  qxp[i] = qx;
  qyp[i] = qy;
  zp[i] = z;
  wlp[i] = z + h;
  hu[i] = T(0);
  qxu[i] = T(0);
  qyu[i] = T(0);
  zu[i] = T(0);
}

// CFL acceleration per listed cell and running maximum depth.  sqrtf is
// single precision in the reference kernel for both dtypes.
template <typename T>
__global__ void __launch_bounds__(kThreads)
timestep_kernel(int64_t M, const int32_t *__restrict__ wet, T *__restrict__ accel,
                T *__restrict__ h_max, const T *__restrict__ h, const T *__restrict__ qx,
                const T *__restrict__ qy, const T *__restrict__ dxp,
                const T *__restrict__ cflp) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const int32_t j = wet[i];
  const T hj = h[j];
  h_max[j] = fmax(hj, h_max[j]);
  const T g = T(kG);
  accel[i] = hj > T(kHSmall)
                 ? cflp[0] * dxp[0] /
                       ((T)sqrtf((float)(g * hj)) + fmax(fabs(qx[j]), fabs(qy[j])) / hj)
                 : T(60.0);
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
rain_station_kernel(int64_t N, T *__restrict__ hu, const int16_t *__restrict__ mask,
                    const T *__restrict__ data, const T *__restrict__ dtp) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) hu[i] += data[mask[i]] * dtp[0];
}

// Neighbour ids are tested with `> 0` as in the reference, so cell 0 never
// activates its neighbours (HC/fluxMaskGenerator_Kernel.cu:36).
template <typename T>
__global__ void __launch_bounds__(kThreads)
flux_mask_kernel(int64_t N, uint8_t *__restrict__ out, const T *__restrict__ h,
                 const int32_t *__restrict__ index, const T *__restrict__ tp) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (tp[0] == T(0)) {
    out[i] = 1;
    return;
  }
  const T hs = T(kHSmall);
  bool m = h[i] > hs;
#pragma unroll
  for (int nei = 1; nei < 5; nei++) {
    const int32_t k = index[(int64_t)nei * N + i];
    if (k > 0) m = m || (h[k] > hs);
  }
  out[i] = m ? 1 : 0;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
euler_update_kernel(int64_t M, const int32_t *__restrict__ mask,
                    const T *__restrict__ hu, const T *__restrict__ qxu,
                    const T *__restrict__ qyu, const T *__restrict__ zu, T *__restrict__ h,
                    T *__restrict__ wl, T *__restrict__ z, T *__restrict__ qx,
                    T *__restrict__ qy) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const int32_t i = mask[j];
  const T hh = h[i] + hu[i];
  const T zz = z[i] + zu[i];
  h[i] = hh;
  qx[i] = qx[i] + qxu[i];
  qy[i] = qy[i] + qyu[i];
  z[i] = zz;
  wl[i] = hh + zz;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
infiltration_kernel(int64_t M, const int32_t *__restrict__ wet, T *__restrict__ hu,
                    const uint8_t *__restrict__ landuse, const T *__restrict__ hp,
                    const T *__restrict__ ks, const T *__restrict__ psi,
                    const T *__restrict__ dth, T *__restrict__ cum,
                    const T *__restrict__ dtp) {
  int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const int32_t i = wet[j];
  const uint8_t lt = landuse[i];
  const T h = hp[i], dt = dtp[0];
  const T K_s = ks[lt], phi_s = psi[lt], d = dth[lt];
  const T F_0 = cum[i];
  const T total_head = phi_s + h;
  const T F_1 = T(0.5) * (F_0 + dt * K_s +
                          sqrt((F_0 + dt * K_s) * (F_0 + dt * K_s) +
                               T(4) * dt * K_s * total_head * d));
  const T dF = fmin(h, F_1 - F_0);
  cum[i] += dF;
  hu[i] -= dF;
}

// Two-level min: blocks reduce to partials, the last block to finish reduces
// the partials (counter-based, no spinning).
constexpr int kMinThreads = 1024;
constexpr int kMinMaxBlocks = 4096;

template <typename T>
__device__ __forceinline__ T block_min(T v, T *sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : sh[0];
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

template <typename T>
__global__ void __launch_bounds__(kMinThreads)
min_reduce_kernel(int64_t M, const T *__restrict__ x, T *__restrict__ out,
                  T *__restrict__ partial, unsigned int *__restrict__ counter) {
  __shared__ T sh[32];
  __shared__ bool last;
  T v = x[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x)
    v = fmin(v, x[i]);
  v = block_min(v, sh);
  if (gridDim.x == 1) {
    if (threadIdx.x == 0) out[0] = v;
    return;
  }
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = v;
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  T m = partial[0];
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) m = fmin(m, partial[b]);
  __syncthreads();
  m = block_min(m, sh);
  if (threadIdx.x == 0) {
    out[0] = m;
    *counter = 0u;
  }
}

template <typename T>
__global__ void gather_kernel(int64_t n, const int64_t *__restrict__ off,
                              const T *__restrict__ h, const T *__restrict__ qx,
                              const T *__restrict__ qy, T *__restrict__ oh,
                              T *__restrict__ ou, T *__restrict__ ov) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t k = off[i];
  const T hh = h[k];
  if (oh) oh[i] = hh;
  const bool wet = hh > T(kHSmall);
  if (ou) ou[i] = wet ? qx[k] / hh : T(0);
  if (ov) ov[i] = wet ? qy[k] / hh : T(0);
}

// h, qx, qy between the dense arrays and compacted arrays (cell i at dense
// offset off[i]); TO_DENSE: scatter, else gather.
template <typename T, bool TO_DENSE>
__global__ void state_layout_kernel(int64_t n, const int64_t *__restrict__ off, T *h, T *qx,
                                    T *qy, T *ch, T *cqx, T *cqy) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t k = off[i];
  if constexpr (TO_DENSE) {
    h[k] = ch[i];
    qx[k] = cqx[i];
    qy[k] = cqy[i];
  } else {
    ch[i] = h[k];
    cqx[i] = qx[k];
    cqy[i] = qy[k];
  }
}

bool bad_dtype(int dtype) { return dtype != HB_F32 && dtype != HB_F64; }

}  // namespace
}  // namespace hb

using namespace hb;

#define HB_REQUIRE(cond, ...) \
  do {                        \
    if (!(cond)) return set_error(HB_ERR_ARG, __VA_ARGS__); \
  } while (0)

extern "C" int hb_flux_mask(int dtype, int64_t N, uint8_t *flux_mask, const void *h,
                            const int32_t *index, const void *t, void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_flux_mask: bad dtype %d", dtype);
  HB_REQUIRE(N >= 0, "hb_flux_mask: negative N");
  if (N == 0) return HB_OK;
  HB_REQUIRE(flux_mask && h && index && t, "hb_flux_mask: null pointer");
  auto s = as_stream(stream);
  if (dtype == HB_F64)
    flux_mask_kernel<double><<<blocks_for(N, kThreads), kThreads, 0, s>>>(
        N, flux_mask, (const double *)h, index, (const double *)t);
  else
    flux_mask_kernel<float><<<blocks_for(N, kThreads), kThreads, 0, s>>>(
        N, flux_mask, (const float *)h, index, (const float *)t);
  return check_launch("hb_flux_mask");
}

extern "C" int hb_flux(int order, int dtype, int64_t M, int64_t N, const int32_t *wet_mask,
                       void *h_flux, void *qx_flux, void *qy_flux, const void *h,
                       const void *wl, const void *z, const void *qx, const void *qy,
                       const int32_t *index, const void *normal, const void *given_depth,
                       int depth_rows, int depth_cols, const void *given_wl, int wl_rows,
                       int wl_cols, const void *given_q, int q_rows, int q_cols,
                       const void *dx, const void *t, const void *dt, void *stream) {
  HB_REQUIRE(order == 1 || order == 2, "hb_flux: order must be 1 or 2 (got %d)", order);
  HB_REQUIRE(!bad_dtype(dtype), "hb_flux: bad dtype %d", dtype);
  HB_REQUIRE(M >= 0 && N >= 0 && M <= N, "hb_flux: bad sizes M=%lld N=%lld",
             (long long)M, (long long)N);
  if (M == 0) return HB_OK;  // HC/flucCal_2ndOrder_jh_improved_Kernel.cu:537-540
  HB_REQUIRE(wet_mask && h_flux && qx_flux && qy_flux && h && wl && z && qx && qy &&
                 index && normal && given_depth && given_wl && given_q && dx && t && dt,
             "hb_flux: null pointer");
  HB_REQUIRE(depth_rows > 0 && depth_cols > 0 && wl_rows > 0 && wl_cols > 0 &&
                 q_rows > 0 && q_cols > 0,
             "hb_flux: empty boundary table");
  auto s = as_stream(stream);
  const unsigned nb = blocks_for(M, kThreads);
#define HB_FLUX_LAUNCH(T, O)                                                          \
  flux_kernel<T, O><<<nb, kThreads, 0, s>>>(                                          \
      M, N, wet_mask, (T *)h_flux, (T *)qx_flux, (T *)qy_flux, (const T *)h,           \
      (const T *)wl, (const T *)z, (const T *)qx, (const T *)qy, index,               \
      (const T *)normal, (const T *)given_depth, depth_rows, depth_cols,              \
      (const T *)given_wl, wl_rows, wl_cols, (const T *)given_q, q_rows, q_cols,      \
      (const T *)dx, (const T *)t, (const T *)dt)
  if (dtype == HB_F64) {
    if (order == 2) HB_FLUX_LAUNCH(double, 2); else HB_FLUX_LAUNCH(double, 1);
  } else {
    if (order == 2) HB_FLUX_LAUNCH(float, 2); else HB_FLUX_LAUNCH(float, 1);
  }
#undef HB_FLUX_LAUNCH
  return check_launch("hb_flux");
}

extern "C" int hb_friction_update(int dtype, int64_t M, const int32_t *wet_mask,
                                  void *h_update, void *qx_update, void *qy_update,
                                  void *z_update, const uint8_t *landuse, void *h, void *wl,
                                  void *qx, void *qy, void *z, const void *manning,
                                  const void *dt, void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_friction_update: bad dtype %d", dtype);
  HB_REQUIRE(M >= 0, "hb_friction_update: negative M");
  if (M == 0) return HB_OK;
  HB_REQUIRE(wet_mask && h_update && qx_update && qy_update && z_update && landuse && h &&
                 wl && qx && qy && z && manning && dt,
             "hb_friction_update: null pointer");
  auto s = as_stream(stream);
#define HB_FR_LAUNCH(T)                                                                 \
  friction_update_kernel<T><<<blocks_for(M, kThreads), kThreads, 0, s>>>(                \
      M, wet_mask, (T *)h_update, (T *)qx_update, (T *)qy_update, (T *)z_update, landuse, \
      (T *)h, (T *)wl, (T *)qx, (T *)qy, (T *)z, (const T *)manning, (const T *)dt)
  if (dtype == HB_F64) HB_FR_LAUNCH(double); else HB_FR_LAUNCH(float);
#undef HB_FR_LAUNCH
  return check_launch("hb_friction_update");
}

extern "C" int hb_timestep(int dtype, int64_t M, const int32_t *wet_mask, void *accelerator,
                           void *h_max, const void *h, const void *qx, const void *qy,
                           const void *dx, const void *cfl, const void *t, const void *dt,
                           void *stream) {
  (void)t;
  (void)dt;
  HB_REQUIRE(!bad_dtype(dtype), "hb_timestep: bad dtype %d", dtype);
  HB_REQUIRE(M >= 0, "hb_timestep: negative M");
  if (M == 0) return HB_OK;
  HB_REQUIRE(wet_mask && accelerator && h_max && h && qx && qy && dx && cfl,
             "hb_timestep: null pointer");
  auto s = as_stream(stream);
#define HB_TS_LAUNCH(T)                                                             \
  timestep_kernel<T><<<blocks_for(M, kThreads), kThreads, 0, s>>>(                  \
      M, wet_mask, (T *)accelerator, (T *)h_max, (const T *)h, (const T *)qx,       \
      (const T *)qy, (const T *)dx, (const T *)cfl)
  if (dtype == HB_F64) HB_TS_LAUNCH(double); else HB_TS_LAUNCH(float);
#undef HB_TS_LAUNCH
  return check_launch("hb_timestep");
}

extern "C" int hb_rain_station(int dtype, int64_t N, void *h_update, const int16_t *mask,
                               const void *station_data, const void *dt, void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_rain_station: bad dtype %d", dtype);
  HB_REQUIRE(N >= 0, "hb_rain_station: negative N");
  if (N == 0) return HB_OK;
  HB_REQUIRE(h_update && mask && station_data && dt, "hb_rain_station: null pointer");
  auto s = as_stream(stream);
  if (dtype == HB_F64)
    rain_station_kernel<double><<<blocks_for(N, kThreads), kThreads, 0, s>>>(
        N, (double *)h_update, mask, (const double *)station_data, (const double *)dt);
  else
    rain_station_kernel<float><<<blocks_for(N, kThreads), kThreads, 0, s>>>(
        N, (float *)h_update, mask, (const float *)station_data, (const float *)dt);
  return check_launch("hb_rain_station");
}

extern "C" int hb_euler_update(int dtype, int64_t M, const int32_t *update_mask,
                               const void *h_update, const void *qx_update,
                               const void *qy_update, const void *z_update, void *h,
                               void *wl, void *z, void *qx, void *qy, void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_euler_update: bad dtype %d", dtype);
  HB_REQUIRE(M >= 0, "hb_euler_update: negative M");
  if (M == 0) return HB_OK;
  HB_REQUIRE(update_mask && h_update && qx_update && qy_update && z_update && h && wl &&
                 z && qx && qy,
             "hb_euler_update: null pointer");
  auto s = as_stream(stream);
#define HB_EU_LAUNCH(T)                                                                  \
  euler_update_kernel<T><<<blocks_for(M, kThreads), kThreads, 0, s>>>(                   \
      M, update_mask, (const T *)h_update, (const T *)qx_update, (const T *)qy_update,  \
      (const T *)z_update, (T *)h, (T *)wl, (T *)z, (T *)qx, (T *)qy)
  if (dtype == HB_F64) HB_EU_LAUNCH(double); else HB_EU_LAUNCH(float);
#undef HB_EU_LAUNCH
  return check_launch("hb_euler_update");
}

extern "C" int hb_infiltration(int dtype, int64_t M, const int32_t *wet_mask,
                               void *h_update, const uint8_t *landuse, const void *h,
                               const void *ks, const void *psi, const void *dtheta,
                               void *cumulative, const void *dt, void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_infiltration: bad dtype %d", dtype);
  HB_REQUIRE(M >= 0, "hb_infiltration: negative M");
  if (M == 0) return HB_OK;
  HB_REQUIRE(wet_mask && h_update && landuse && h && ks && psi && dtheta && cumulative && dt,
             "hb_infiltration: null pointer");
  auto s = as_stream(stream);
#define HB_IN_LAUNCH(T)                                                                 \
  infiltration_kernel<T><<<blocks_for(M, kThreads), kThreads, 0, s>>>(                  \
      M, wet_mask, (T *)h_update, landuse, (const T *)h, (const T *)ks, (const T *)psi, \
      (const T *)dtheta, (T *)cumulative, (const T *)dt)
  if (dtype == HB_F64) HB_IN_LAUNCH(double); else HB_IN_LAUNCH(float);
#undef HB_IN_LAUNCH
  return check_launch("hb_infiltration");
}

extern "C" size_t hb_min_reduce_workspace_size(int64_t M) {
  int64_t nb = (M + kMinThreads - 1) / kMinThreads;
  if (nb <= 4) return 0;
  if (nb > kMinMaxBlocks) nb = kMinMaxBlocks;
  return (size_t)nb * sizeof(double) + 256;
}

extern "C" int hb_min_reduce(int dtype, int64_t M, const void *x, void *out, void *workspace,
                             void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_min_reduce: bad dtype %d", dtype);
  HB_REQUIRE(M > 0, "hb_min_reduce: M must be positive");
  HB_REQUIRE(x && out, "hb_min_reduce: null pointer");
  int64_t nb = (M + kMinThreads - 1) / kMinThreads;
  if (nb <= 4) nb = 1;
  if (nb > kMinMaxBlocks) nb = kMinMaxBlocks;
  HB_REQUIRE(nb == 1 || workspace, "hb_min_reduce: workspace required for M=%lld",
             (long long)M);
  // the block counter sits at a fixed offset (the first word) so that a
  // workspace reused for inputs of other sizes finds it where the last call
  // left it (zero); the block partials follow at 256 bytes
  unsigned int *counter = nb == 1 ? nullptr : (unsigned int *)workspace;
  void *partial = nb == 1 ? nullptr : (void *)((char *)workspace + 256);
  auto s = as_stream(stream);
  if (dtype == HB_F64)
    min_reduce_kernel<double><<<(unsigned)nb, kMinThreads, 0, s>>>(
        M, (const double *)x, (double *)out, (double *)partial, counter);
  else
    min_reduce_kernel<float><<<(unsigned)nb, kMinThreads, 0, s>>>(
        M, (const float *)x, (float *)out, (float *)partial, counter);
  return check_launch("hb_min_reduce");
}

extern "C" int hb_gather(int dtype, int64_t n, const int64_t *cell_offsets, const void *h,
                         const void *qx, const void *qy, void *out_h, void *out_u,
                         void *out_v, void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_gather: bad dtype %d", dtype);
  HB_REQUIRE(n >= 0, "hb_gather: negative n");
  if (n == 0) return HB_OK;
  HB_REQUIRE(cell_offsets && h, "hb_gather: null pointer");
  HB_REQUIRE(!(out_u || out_v) || (qx && qy), "hb_gather: velocities need qx and qy");
  auto s = as_stream(stream);
  if (dtype == HB_F64)
    gather_kernel<double><<<blocks_for(n, kThreads), kThreads, 0, s>>>(
        n, cell_offsets, (const double *)h, (const double *)qx, (const double *)qy,
        (double *)out_h, (double *)out_u, (double *)out_v);
  else
    gather_kernel<float><<<blocks_for(n, kThreads), kThreads, 0, s>>>(
        n, cell_offsets, (const float *)h, (const float *)qx, (const float *)qy,
        (float *)out_h, (float *)out_u, (float *)out_v);
  return check_launch("hb_gather");
}

extern "C" int hb_state_layout(int dtype, int64_t n, const int64_t *offsets, int to_dense,
                               void *h, void *qx, void *qy, void *ch, void *cqx, void *cqy,
                               void *stream) {
  HB_REQUIRE(!bad_dtype(dtype), "hb_state_layout: bad dtype %d", dtype);
  HB_REQUIRE(n >= 0, "hb_state_layout: negative n");
  if (n == 0) return HB_OK;
  HB_REQUIRE(offsets && h && qx && qy && ch && cqx && cqy, "hb_state_layout: null pointer");
  auto s = as_stream(stream);
  const unsigned nb = blocks_for(n, kThreads);
  if (dtype == HB_F64) {
    auto *a = (double *)h, *b = (double *)qx, *c = (double *)qy;
    auto *d = (double *)ch, *e = (double *)cqx, *f = (double *)cqy;
    if (to_dense)
      state_layout_kernel<double, true><<<nb, kThreads, 0, s>>>(n, offsets, a, b, c, d, e, f);
    else
      state_layout_kernel<double, false><<<nb, kThreads, 0, s>>>(n, offsets, a, b, c, d, e, f);
  } else {
    auto *a = (float *)h, *b = (float *)qx, *c = (float *)qy;
    auto *d = (float *)ch, *e = (float *)cqx, *f = (float *)cqy;
    if (to_dense)
      state_layout_kernel<float, true><<<nb, kThreads, 0, s>>>(n, offsets, a, b, c, d, e, f);
    else
      state_layout_kernel<float, false><<<nb, kThreads, 0, s>>>(n, offsets, a, b, c, d, e, f);
  }
  return check_launch("hb_state_layout");
}
