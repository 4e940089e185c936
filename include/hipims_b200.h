/*
 * hipims_b200.h -- C ABI of libhipims_b200.so, a B200 (sm_100a) implementation
 * of the HiPIMS 2-D shallow-water time step.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative HB_ERR_* code;
 *    hb_last_error() returns a message for the calling thread's last failure.
 *  - Array arguments are DEVICE pointers owned by the caller (plain pointers
 *    and sizes, no framework types).  Scalars the reference passes as
 *    1-element tensors (dx, CFL, t, dt) are device pointers too, so no call
 *    synchronises with the host.
 *  - `stream` is a cudaStream_t passed as void*; NULL is the legacy default
 *    stream.  Work is enqueued asynchronously; errors from the launch are
 *    reported, errors from kernel execution surface at the next sync.
 *  - `dtype` is HB_F32 or HB_F64 and applies to every floating array of a call.
 *
 * Reference paths below are relative to the reference project root
 * (HC = CHANS-HiPIMS/hipims/cuda, HP = CHANS-HiPIMS/hipims/pythonHipims).
 */
#ifndef HIPIMS_B200_H
#define HIPIMS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HB_ABI_VERSION 1

enum hb_dtype { HB_F32 = 0, HB_F64 = 1 };

enum hb_status {
  HB_OK = 0,
  HB_ERR_ARG = -1,     /* invalid argument (null pointer, bad size, bad dtype) */
  HB_ERR_CUDA = -2,    /* CUDA runtime error (message in hb_last_error) */
  HB_ERR_LIMIT = -3,   /* a documented size limit was exceeded */
  HB_ERR_TIMEOUT = -4  /* a bounded device-side wait gave up */
};

/* Library identity and last error of the calling thread. */
int hb_abi_version(void);
const char *hb_last_error(void);
/* sizeof of the records in hipims_b200_fused.h, for FFI layout checks:
 * out[0] = hb_ctrl, out[1] = hb_instance, out[2] = hb_fused_batch. */
void hb_record_sizes(size_t out[3]);

/* ======================================================================
 * Compat ops: the reference's torch-extension op surface, one C entry per op.
 * Same argument meaning, compacted-cell layout and in-place semantics.
 * ==================================================================== */

/* fluxMask.update(fluxMask, h, index, t)  -- HC/fluxMaskGenerator.cpp:22-29,
 * kernel HC/fluxMaskGenerator_Kernel.cu:19-42.  out: uint8 (torch.bool) [N]. */
int hb_flux_mask(int dtype, int64_t N, uint8_t *flux_mask, const void *h,
                 const int32_t *index, const void *t, void *stream);

/* fluxCal_2ndOrder_jh_improved.addFlux (order = 2,
 * HC/fluxCal_2ndOrder_jh_improved.cpp:28-53) and
 * fluxCalculation_jh_modified_surface.addFlux (order = 1,
 * HC/fluxCal_jh_modified_surface.cpp:28-53).  Accumulates into
 * h_flux/qx_flux/qy_flux [N] for the M active cells of wet_mask.
 * Boundary tables are row-major [rows, cols] with time in column 0. */
int hb_flux(int order, int dtype, int64_t M, int64_t N, const int32_t *wet_mask,
            void *h_flux, void *qx_flux, void *qy_flux, const void *h,
            const void *wl, const void *z, const void *qx, const void *qy,
            const int32_t *index, const void *normal, const void *given_depth,
            int depth_rows, int depth_cols, const void *given_wl, int wl_rows,
            int wl_cols, const void *given_q, int q_rows, int q_cols,
            const void *dx, const void *t, const void *dt, void *stream);

/* friction_implicit_andUpdate_jh.addFriction_eulerUpdate --
 * HC/friction_implicit_andUpdate_jh_interface.cpp:29-53, kernel
 * HC/friction_implicit_andUpdate_jh_Kernel.cu:22-146.  landuse: uint8 [N]. */
int hb_friction_update(int dtype, int64_t M, const int32_t *wet_mask,
                       void *h_update, void *qx_update, void *qy_update,
                       void *z_update, const uint8_t *landuse, void *h, void *wl,
                       void *qx, void *qy, void *z, const void *manning,
                       const void *dt, void *stream);

/* timeControl.updateTimestep -- HC/timeControl.cpp:27-41, kernel
 * HC/timeControl_Kernel.cu:164-198.  accelerator [M] out, h_max [N] in/out. */
int hb_timestep(int dtype, int64_t M, const int32_t *wet_mask, void *accelerator,
                void *h_max, const void *h, const void *qx, const void *qy,
                const void *dx, const void *cfl, const void *t, const void *dt,
                void *stream);

/* station_PrecipitationCalculation.addStation_Precipitation --
 * HC/stationPrecipitation_interface.cpp:26-38, kernel
 * HC/stationPrecipitation_Kernel.cu:18-29.  mask: int16 [N]. */
int hb_rain_station(int dtype, int64_t N, void *h_update, const int16_t *mask,
                    const void *station_data, const void *dt, void *stream);

/* euler_update.update -- HC/euler_update.cpp:27-44, kernel
 * HC/euler_update_Kernel.cu:18-36. */
int hb_euler_update(int dtype, int64_t M, const int32_t *update_mask,
                    const void *h_update, const void *qx_update,
                    const void *qy_update, const void *z_update, void *h,
                    void *wl, void *z, void *qx, void *qy, void *stream);

/* infiltrationCalculation.addinfiltration -- HC/infiltration_interface.cpp,
 * kernel HC/infiltrationCUDA_Kernel.cu:20-46 (Green-Ampt). */
int hb_infiltration(int dtype, int64_t M, const int32_t *wet_mask, void *h_update,
                    const uint8_t *landuse, const void *h, const void *ks,
                    const void *psi, const void *dtheta, void *cumulative,
                    const void *dt, void *stream);

/* Device-side minimum of x[0..M) written to out[0] -- replaces the
 * torch.min(accelerator) of HP/SWE_CUDA.py:818-820 without a host sync.
 * workspace: hb_min_reduce_workspace_size(M) bytes, or NULL when M <= 4096;
 * zero-filled before its first use.  Every call leaves it ready for the next
 * (its first word, a block counter, is back at zero), so one workspace of the
 * largest size needed serves calls of any size ordered on one stream. */
size_t hb_min_reduce_workspace_size(int64_t M);
int hb_min_reduce(int dtype, int64_t M, const void *x, void *out, void *workspace,
                  void *stream);

/* ======================================================================
 * Fused dense-tile step (no reference counterpart; replaces the sequence
 * addFlux -> rain -> friction/update -> timeControl -> min of
 * HP/SWE_CUDA.py:339-424, 497-502, 780-831 with one kernel per step).
 * A batch of instances (catchments) advances together; a single run is a
 * batch of one.  Layout and argument records are defined in
 * hipims_b200_fused.h.
 * ==================================================================== */
struct hb_fused_batch; /* host-side launch record, see hipims_b200_fused.h */

/* Bytes of device workspace one step needs (per-tile partial sums). */
size_t hb_fused_workspace_size(const struct hb_fused_batch *batch);
/* Initialise the control blocks: rain rate and boundary values at t, zero
 * counters.  Call once before the first step and after host edits of ctrl. */
int hb_fused_prepare(const struct hb_fused_batch *batch, void *stream);
/* Enqueue `nsteps` fused steps (graph-capturable; no host sync). */
int hb_fused_step(const struct hb_fused_batch *batch, int nsteps, void *stream);
/* The same `nsteps` steps of every instance in ONE persistent cooperative
 * launch (no reference counterpart; the ensemble form of the step): resident
 * blocks take tiles from a counter, the instance's last tile advances its
 * clock, and a grid barrier separates the steps.  Results equal nsteps calls
 * of hb_fused_step bit for bit.  Built for FP32 2nd-order batches with
 * 32 x 64 tiles (not for strips, whose clock needs hb_fused_finish between
 * steps).  Every barrier wait gives up after budget_cycles SM clock cycles
 * (<= 0: 2^31, about a second): the blocks then leave, bit 8 is set in every
 * instance's status and the state is incomplete (re-prepare or restore before
 * stepping on).  Needs hb_fused_prepare first; graph-capturable. */
int hb_fused_run(const struct hb_fused_batch *batch, int nsteps, long long budget_cycles,
                 void *stream);
/* Clock advance of instances stepped with hb_ctrl.external_dt set (no
 * counterpart in the reference; one catchment split into row strips over
 * several instances or GPUs): ext = device [n_instances][2], the largest wave
 * speed and the any-dry flag of each instance's whole catchment (the maximum
 * of hb_ctrl.ext over its strips).  ext = NULL: the batch's instances are
 * all the strips of one catchment, and every instance uses the maximum of
 * hb_ctrl.ext over the batch.  Applies HP/SWE_CUDA.py:818-831 (CFL dt,
 * 10x cap, export clip, t += dt) and sets the next step's rain rate and
 * boundary values.  One step, then this, per time step. */
int hb_fused_finish(const struct hb_fused_batch *batch, const double *ext, void *stream);

/* Allocation-free variant of hb_fused_step (no counterpart in the reference).
 * For callers that must not allocate device memory: host programs that own a
 * fixed device-memory budget and manage it themselves (the FLAMEGPU agent
 * runtime preallocates its buffers), and threads that cannot afford the
 * device-wide synchronisation cudaMalloc/cudaFree can cause while other
 * kernels, such as the agent model's, are running.  It allocates nothing: the
 * step's scratch (per-tile partial sums, boundary values, TMA descriptors)
 * lives in one fixed 4 MiB device array inside this library, present on every
 * GPU that loads it until the process exits; b->workspace is ignored.
 *  - prepare != 0 (re)initialises that scratch for this batch (as
 *    hb_fused_prepare does for a workspace), then runs nsteps steps; pass it
 *    on the first call and whenever the batch or its control blocks change.
 *  - Limits: hb_fused_workspace_size(b) <= 4 MiB (about 110,000 tiles, e.g.
 *    110 M cells with 32 x 32 tiles; about 100,000 with 256 instances; with
 *    64-wide tiles, which keep a 16-byte entry per tile, about 78,000, i.e.
 *    160 M cells, and 70,000) and at most 256 instances; larger batches get
 *    HB_ERR_LIMIT with a message.
 *  - Every call with prepare != 0 looks up the array's device address on the
 *    current device, and the first such call on a device creates the
 *    library's side stream and two events for that device (kept until exit;
 *    no device memory is allocated for them by this library); make that
 *    first call before any stream capture.  After cudaDeviceReset the array
 *    has a new address: the next call on that device must pass prepare != 0.
 *  - The library remembers, per device, which batch the array was last
 *    prepared for (its instance records, tile and instance counts, tile
 *    shape, dtype, order and flags).  A call with prepare == 0 for any other
 *    batch, or before any prepare on that device, returns HB_ERR_ARG instead
 *    of running with another batch's scratch.  Two batches used in turn each
 *    need prepare != 0 when their turn comes.
 *  - Every call on a device shares the one array and leaves its contents
 *    behind: calls that overlap on the GPU (other streams, other threads)
 *    race with each other. */
int hb_fused_step_noalloc(const struct hb_fused_batch *batch, int nsteps, int prepare,
                          void *stream);

/* ======================================================================
 * Discrete adjoint of the FP64 fused step (no reference counterpart).
 * Given lambda^{n+1} = dJ/dU^{n+1} (U = h, qx, qy on the dense layout of
 * one instance) and the forward state U^n, writes lambda^n = (dU^{n+1}/dU^n)^T
 * lambda^{n+1} and adds (dU^{n+1}/dtheta)^T lambda^{n+1} to grad, theta =
 * (Manning n of zones 0..15, rain multiplier).  dt is frozen (the forward's
 * schedule); every discrete decision is the forward's.
 * ==================================================================== */
typedef struct hb_adjoint_args {
  const struct hb_instance *instance; /* device record of the instance (FP64) */
  int32_t rows, cols, pitch, code_pitch;
  const double *h, *qx, *qy;          /* U^n, dense */
  const double *lam_h, *lam_qx, *lam_qy; /* lambda^{n+1} */
  double *out_h, *out_qx, *out_qy;    /* lambda^n (overwritten) */
  double *mu;                         /* scratch: 3 * mu_stride doubles */
  int64_t mu_stride;                  /* >= elements of one dense array */
  double *grad;                       /* [17]: d/dn_zone (16), d/d rain multiplier */
  double t, dt;                       /* time and time step of step n */
  double rain_rate;                   /* rain rate used by step n (m/s) */
  double rain_base;                   /* the same without the multiplier */
  double h_reg;                       /* cells with h^n < h_reg get no state adjoint
                                         (films of a few h_small between deeper cells
                                         have unstable linearisations; 0 masks only
                                         negative depths) */
  int32_t first;                      /* step n starts at t == 0 */
  int32_t pad;
  double *faces;                      /* optional scratch, 10 * face_stride doubles: the
                                         forward face values of step n, computed once
                                         instead of twice per face; NULL: recomputed */
  int64_t face_stride;                /* >= (rows + 1) * (cols + 1) */
} hb_adjoint_args;
int hb_adjoint_step(const hb_adjoint_args *args, void *stream);
/* lam_h[offsets[i]] += 2 * weight * (h[offsets[i]] - obs[i]): the gradient of
 * a sum of squared gauge misfits, added at a sampled step. */
int hb_adjoint_gauge(int64_t n, const int64_t *offsets, const double *h, const double *obs,
                     double *lam_h, double weight, void *stream);

/* ======================================================================
 * Coupling gather (no reference counterpart; replaces the
 * h[idx_target_ABM1] gather of CHANS-HiPIMS/CHANS-HiPIMS_server.py:255-256).
 * Gathers depth (and optionally velocities u = qx/h, v = qy/h, 0 when dry)
 * at n agent cells given as flat raster offsets (row * pitch + col of the
 * dense arrays).  out: float [n] per requested field.
 * ==================================================================== */
int hb_gather(int dtype, int64_t n, const int64_t *cell_offsets, const void *h,
              const void *qx, const void *qy, void *out_h, void *out_u,
              void *out_v, void *stream);

/* ======================================================================
 * State layout (no reference counterpart: the reference holds h, qx, qy
 * compacted, the valid cells in row-major order, h[mask > 0] of
 * HP/SWE_CUDA.py:62-227).  Copies the three state fields between the dense
 * arrays of the fused step and compacted arrays of n cells, cell i at dense
 * element offset offsets[i] (row * pitch + col of the dense layout).
 *   to_dense != 0: h[offsets[i]] = ch[i] (and qx, qy); 0: ch[i] = h[offsets[i]].
 * Lets a host that keeps the reference's compacted state feed the fused step
 * (a per-step host copy then moves n cells per field instead of the padded
 * raster).
 * ==================================================================== */
int hb_state_layout(int dtype, int64_t n, const int64_t *offsets, int to_dense, void *h,
                    void *qx, void *qy, void *ch, void *cqx, void *cqy, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* HIPIMS_B200_H */
