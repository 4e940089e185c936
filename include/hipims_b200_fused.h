/*
 * hipims_b200_fused.h -- records of the fused dense-tile step (hb_fused_*).
 *
 * Dense layout (one instance = one catchment raster of rows x cols cells):
 *  - State arrays (h, qx, qy, z, h_max) are row-major with `pitch` elements
 *    per row.  Raster cell (r, c) lives at element (r + 2) * pitch + (c + 4):
 *    two halo rows above, four columns on the left so that every tile load,
 *    halo included, starts on a 16-byte boundary.  Storage has at least
 *    round_up(rows, 64) + 4 rows and pitch >= round_up(cols, 64) + 8.
 *  - The cell code array (uint8) has `code_pitch` bytes per row, raster
 *    cell (r, c) at (r + 2) * code_pitch + (c + 16).  Low nibble = Manning
 *    zone, high nibble = boundary class; class 15 = no-data.  Padding is
 *    no-data (0xF0).
 *  - In FP32 mode z is stored relative to a datum per 64 x 64 block of the
 *    raster (datum[by * datum_nx + bx], integer-valued floats), so that
 *    eta = h + z keeps sub-millimetre resolution on high terrain.  FP64 mode
 *    stores z absolute with a zero datum.
 *  - State buffers ping-pong: ctrl->cur names the one holding the latest
 *    state; a step reads cur and writes 1 - cur.
 */
#ifndef HIPIMS_B200_FUSED_H
#define HIPIMS_B200_FUSED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HB_MAX_CLASSES 16
#define HB_NODATA_CLASS 15
#define HB_MAX_ZONES 16
#define HB_DATUM_BLOCK 64
#define HB_PAD_Y 2
#define HB_PAD_X 4
#define HB_CODE_PAD_X 16
/* hb_fused_batch.flags: FP32 with the reference's operation forms (no
 * approximate division/square root, no algebraic shortcuts). */
#define HB_FLAG_EXACT_FP32 1
/* hb_fused_batch.flags: use the face-task kernel (any 32x32 tile, staged by
 * plain loads) instead of the row-walking kernel (32-wide tiles staged by TMA). */
#define HB_FLAG_TILE_TASKS 2
/* hb_fused_batch.flags: some instance has infiltration or station rain (the
 * rows kernel build with those source terms; hb_fused_prepare checks it). */
#define HB_FLAG_SOURCES 4
/* hb_fused_batch.flags bits 8-11: register cap of the rows kernel expressed
 * as resident CTAs per SM (0 = compiler default; 5, 6 for 32-row tiles; 4 for
 * 64-row tiles).  The autotuner picks it. */
#define HB_FLAG_MINB_SHIFT 8

/* Per-instance control block, device memory.  Written by hb_fused_prepare
 * and by the last tile of every step; read by the host between launches. */
typedef struct hb_ctrl {
  double t;              /* simulated time of the next step (HP/SWE_CUDA.py self.t) */
  double dt;             /* time step of the next step (self.dt) */
  double export_step;    /* Export_timeStep; dt is clipped to its multiples */
  double t_end;          /* the step that reaches t >= t_end halts the instance */
  double volume;         /* FP64 sum of h * dx^2 over valid cells, after the last step */
  double volume0;        /* volume at prepare */
  double rain_volume;    /* FP64 accumulated rain input (m^3) */
  double outflow_volume; /* FP64 accumulated boundary outflow (m^3) */
  double rain_rate;      /* uniform rain rate (m/s) used by the next step */
  double rain_mult;      /* multiplier applied to the rain table */
  int64_t step;          /* steps taken */
  int32_t export_n;      /* export counter (self._export_n) */
  int32_t cur;           /* state buffer holding the latest state */
  int32_t halted;        /* nonzero: steps are no-ops */
  int32_t halt_on_export;/* nonzero: halt after a step that hits an export time */
  int32_t exports;       /* export clips taken */
  int32_t rain_index;    /* monotone cursor into the rain table */
  uint32_t tiles_done;   /* internal last-tile-done counter */
  int32_t status;        /* bits: 1 non-finite dt, 2 a tile's data did not arrive
                            (TMA wait timed out), 4 non-finite depth (FP64 volume),
                            8 a grid barrier of hb_fused_run gave up (budget) */
  float bc_vals[HB_MAX_CLASSES][4]; /* given h, wl, qx, qy per class at t */
  /* Deferred time step (strips of one catchment on several instances or
   * GPUs): with external_dt set, a step leaves dt, t, the step counter and
   * the next step's rain rate and boundary values alone and writes its
   * largest wave speed and whether any valid cell was dry to ext[0], ext[1];
   * hb_fused_finish then advances the clock from values reduced over all
   * strips (max of each). */
  int32_t external_dt;
  int32_t pad1;
  double ext[2];
} hb_ctrl;

/* One catchment.  Pointers are device pointers. */
typedef struct hb_instance {
  int32_t rows, cols;        /* raster size */
  int32_t tiles_x, tiles_y;  /* tile grid over the raster */
  int32_t tile_begin;        /* first flat tile index of this instance */
  int32_t pitch;             /* elements per row of the state arrays */
  int32_t code_pitch;        /* bytes per row of the code array */
  int32_t datum_nx, datum_ny;/* datum blocks */
  int32_t bug_y, bug_x;      /* raster cell whose compacted id is 0, or -1 */
  int32_t rain_rows, rain_cols;
  int32_t depth_rows, depth_cols, wl_rows, wl_cols, q_rows, q_cols;
  int32_t pad0;
  void *h[2], *qx[2], *qy[2];/* ping-pong state */
  void *z;                   /* bed elevation (datum-relative in FP32 mode) */
  void *h_max;               /* running maximum depth */
  const uint8_t *code;       /* zone | class << 4 */
  const float *datum;        /* [datum_ny * datum_nx] */
  hb_ctrl *ctrl;
  const double *rain_tab;    /* [rain_rows, rain_cols]: time, rate (m/s) */
  const double *given_depth; /* boundary tables, HP/SWE_CUDA.py:102-110 layout */
  const double *given_wl;
  const double *given_q;
  double dx, cfl;
  double manning[HB_MAX_ZONES];
  int32_t bc_type[HB_MAX_CLASSES]; /* 1 interior, 3..8 ghost types */
  int32_t bc_id[HB_MAX_CLASSES];
  int64_t n_valid;           /* valid cells */
  const double *dt_replay;   /* optional: dt of step k+1 is dt_replay[k] for k < n_replay */
  int64_t n_replay;          /* (frozen time-step schedule; 0 = adaptive CFL step) */
  /* optional Green-Ampt infiltration (HC/infiltrationCUDA_Kernel.cu:20-46), applied
   * to the active cells after rain as HP/CatchFlood_main.py:164-170 orders it;
   * cum = NULL disables it.  Rows kernel only. */
  void *cum;                 /* cumulative infiltrated depth, dense like h (in place) */
  double ks[HB_MAX_ZONES];   /* saturated hydraulic conductivity per zone (m/s) */
  double psi[HB_MAX_ZONES];  /* capillary head per zone (m) */
  double dtheta[HB_MAX_ZONES]; /* water-content difference per zone */
  /* optional station rain (HC/stationPrecipitation_Kernel.cu:18-29 with the
   * station interpolation of HP/SWE_CUDA.py:472-502): rain_tab holds one rate
   * column per station, rain_station the station of every cell (dense like h);
   * NULL rain_station: uniform rain from column 1.  Rows kernel only. */
  const uint16_t *rain_station;
  double *station_rate;      /* [n_stations] rates at t, kept by the library */
  const double *station_cells; /* [n_stations] valid cells per station */
  int32_t n_stations;
  int32_t pad2;
  /* optional halo forwarding between row strips of one catchment (no
   * reference counterpart; replaces the halo exchange of
   * HP/Parallel_SWE_CUDA.py).  The new h, qx, qy of this strip's first
   * HB_PAD_Y rows are also stored into the bottom halo rows of the strip
   * above (halo_up), and those of its last HB_PAD_Y rows into the top halo
   * rows of the strip below (halo_down), in the output buffer of the step.
   * Each side lists [h0, h1, qx0, qx1, qy0, qy1] of the neighbour (same
   * columns and pitch as this strip); NULL halo_*[0]: no neighbour on that
   * side.  The neighbour's arrays may be a peer GPU's memory (plain stores).
   * Rows kernel only. */
  void *halo_up[6];
  void *halo_down[6];
  int32_t halo_up_rows;      /* rows of the strip above */
  int32_t pad3;
} hb_instance;

/* Launch record (host memory). */
typedef struct hb_fused_batch {
  int32_t dtype;             /* HB_F32 or HB_F64 */
  int32_t n_instances;
  int32_t n_tiles;           /* sum of tiles_x * tiles_y */
  int32_t tile_y, tile_x;    /* tile shape: 32 wide, 32 or 64 high */
  int32_t grid_blocks;       /* 0: one block per tile (rows kernel), one wave of resident
                                blocks (tile-task kernel); > 0: that many blocks, each
                                looping over tiles */
  int32_t order;             /* 2 (MUSCL); 1 (bed-only minmod) */
  int32_t flags;             /* HB_FLAG_* bits */
  const hb_instance *instances;  /* device [n_instances] */
  const int32_t *tile_instance;  /* device [n_tiles] */
  void *workspace;               /* device, hb_fused_workspace_size() bytes */
  const hb_instance *instances_host; /* host copy of instances (hb_fused_prepare) */
} hb_fused_batch;

#ifdef __cplusplus
}
#endif

#endif /* HIPIMS_B200_FUSED_H */
