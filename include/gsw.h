/*
 * gsw.h -- C ABI of libgsw.so, the B200 (sm_100a) finite-volume step of GeoSWE.
 *
 * The reference launches its step kernels from Python as CuPy RawKernels with raw
 * device pointers and scalars on CuPy's current stream, and checks nothing on the
 * device side (geoswe/solver.py:2271-2290, geoswe/compressed_solver.py:880-905).
 * Each entry point below replaces one of those launches, or one of the host-side
 * loop pieces the reference keeps in Python, with a C function that
 *   - takes plain device pointers (the caller owns every buffer: torch tensors,
 *     cudaMalloc, anything) and an explicit cudaStream_t,
 *   - never allocates on the step path,
 *   - returns 0 on success or a negative GSW_ERR_* code, with a message in
 *     gsw_last_error() (thread-local).
 * Every argument struct starts with `abi_version`; pass GSW_ABI_VERSION.
 *
 * Layouts
 *   Dense fields are the reference's padded (nx+2*ngh, ny+2*ngh) C-order arrays,
 *   with an explicit row pitch (elements between rows, >= nyp) so rows can be
 *   128-byte aligned. The pointer addresses padded cell (0, 0).
 *   Flat (compressed-mesh) fields live in brick storage: bricks of
 *   GSW_BRICK_W x brick_h cells, each stored as brick_h rows of
 *   GSW_BRICK_PITCH elements, bricks ordered along a Hilbert curve. The canonical
 *   row-major flat order of the reference (geoswe/compressed_mesh.py:135-160) maps
 *   to brick slots through the permutation gsw_mesh_build returns.
 */
#ifndef GSW_H
#define GSW_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GSW_API __attribute__((visibility("default")))
#else
#define GSW_API
#endif

#define GSW_ABI_VERSION 4u

/* return codes */
#define GSW_OK               0
#define GSW_ERR_INVALID     -1   /* bad argument (shape, null pointer, range) */
#define GSW_ERR_CUDA        -2   /* a CUDA runtime call failed */
#define GSW_ERR_ABI         -3   /* abi_version mismatch */
#define GSW_ERR_NONFINITE   -4   /* non-finite wave speed (NaN/Inf in the state) */
#define GSW_ERR_RANGE       -5   /* table/delta out of the representable range */
#define GSW_ERR_TIMEOUT     -6   /* a bounded device wait gave up */

/* element types */
#define GSW_F32 0
#define GSW_F64 1

/* boundary kinds per face (geoswe/bc.py:50-172) */
#define GSW_BC_EXTRAPOLATE 0
#define GSW_BC_WALL        1
#define GSW_BC_FALL        2
#define GSW_BC_PERIODIC    3
#define GSW_BC_NONE        4   /* leave this face's ghosts alone */

/* rain kinds */
#define GSW_RAIN_NONE     0
#define GSW_RAIN_UNIFORM  1    /* rain[frame] is one rate (m/s) */
#define GSW_RAIN_GRIDDED  2    /* rain + frame*nx*ny is an interior (nx, ny) frame (m/s) */
#define GSW_RAIN_LOOKUP   3    /* flat: rate_table[frame*ncol + lookup[cell]] */

/* step arithmetic (the `arith` field of the step argument structs)
 *   EXACT:    separately rounded IEEE operations in the reference kernel's operand order,
 *             and Manning's h^(-4/3) by CUDA's powf(h, -4.0f/3.0f) as the reference
 *             kernel text evaluates it (geoswe/rhs_cuda.py:1830,
 *             geoswe/compressed_rhs.py:730); bit-identical to the reference kernel text
 *             compiled without FMA contraction, friction included.
 *   FAST:     binary32 only; FMA contraction, flush-to-zero, approximate square root and
 *             division. Held to a depth tolerance against EXACT (stated by the tests and
 *             the benchmark), not to bit equality.
 *   PORTABLE: EXACT with h^(-4/3) by a Newton iteration of IEEE +, -, *, / only (within
 *             1.85 ulp of the exact power), so that any IEEE host reproduces every bit of
 *             a friction run (the CPU oracle restates it). Binary64 steps always use the
 *             iteration (the reference's friction is binary32 only). */
#define GSW_ARITH_EXACT    0
#define GSW_ARITH_FAST     1
#define GSW_ARITH_PORTABLE 2

/* friction kinds */
#define GSW_FRICTION_NONE  0
#define GSW_FRICTION_TABLE 1   /* n = n_tab[n_cls[cell]] */
#define GSW_FRICTION_FIELD 2   /* n = n_field[cell] */

/* CFL velocity norms */
#define GSW_NORM_LINF 0        /* max(|u|,|v|): geoswe/solver.py:152-205 */
#define GSW_NORM_L2   1        /* sqrt(u^2+v^2): geoswe/compressed_solver.py:209-244 */

/* compressed-mesh brick geometry */
#define GSW_BRICK_W      30
#define GSW_BRICK_PITCH  32

/* ------------------------------------------------------------------------- */
/* Device-resident loop control.                                              */
/* One per solver, in device memory, written only by the library's kernels.  */
/* ------------------------------------------------------------------------- */
typedef struct GswLoopState {
    double   t;          /* simulated time (s), accumulated in fp64 as the reference host loop does */
    double   dt;         /* this step's time step (s) */
    double   t_new;      /* t + dt, committed by the next gsw_dt_finalize / gsw_loop_commit */
    int64_t  steps;      /* steps taken */
    uint64_t lam_bits;   /* max wave speed of the current state as IEEE double bits (atomicMax target) */
    double   lam_used;   /* wave speed the last dt came from (diagnostic) */
    float    dt_f32;     /* (float)dt, the value fp32 kernels read */
    int32_t  rain_idx;   /* rain frame of the current step */
    int32_t  done;       /* 1: loop condition false, step cap reached, or error */
    int32_t  error;      /* 0 or a GSW_ERR_* code raised on the device */
    int32_t  pending;    /* 1: t_new/steps not committed yet */
    int32_t  reserved[3];
} GswLoopState;

/* Time-step rule (replaces the host arithmetic of Solver2D.run / cfl_dt /
 * _rain_step_limit, geoswe/solver.py:2569-2693, 2975-3027, and of the flat loop,
 * geoswe/compressed_solver.py:713-748, 2133-2235). All in fp64:
 *   lam = max((double)lam_f32, lam_floor)
 *   dt  = cfl_dmin / (lam + 1e-12)
 *   dt  = min(dt, rain_lim[rain_idx])   when rain_lim != NULL and rain_lim[idx] > 0
 *   dt  = min(dt, dt_max)               when dt_max > 0
 *   dt  = t_end - t                     when t + dt > t_end   (dense form)
 *   dt  = min(dt, t_end - t)            (flat form, same value)
 * The loop stops (done = 1) when !(t < t_end - eps_end) or steps >= max_steps. */
typedef struct GswDtParams {
    uint32_t abi_version;
    int32_t  mode;        /* 0: CFL rule above; 1: fixed dt (fixed_dt); 2: dt_table[steps] */
    double   cfl_dmin;    /* cfl * min(dx, dy), computed by the caller in fp64 */
    double   lam_floor;   /* sqrt(g * h_floor), computed by the caller */
    double   t_end;
    double   eps_end;     /* 1e-12 (dense loop) or 1e-9 (flat loop) */
    double   dt_max;      /* <= 0: none */
    double   fixed_dt;
    int64_t  max_steps;
    const double* rain_t;   /* device, n_rain knot times (bisect_right - 1, clamped) or NULL */
    const double* rain_lim; /* device, per-frame rain step limit (<= 0: none) or NULL */
    int32_t  n_rain;
    int32_t  clip_flat;     /* 0: dense clip (t + dt > t_end -> t_end - t); 1: flat dt = min(dt, t_end - t) */
    const double* dt_table; /* mode 2: dt = dt_table[steps] (a recorded schedule, replayed exactly) */
    double*  dt_log;        /* non-NULL: dt_log[steps] = the dt this step takes */
} GswDtParams;

/* ------------------------------------------------------------------------- */
/* Dense fused step.                                                          */
/* ------------------------------------------------------------------------- */
typedef struct GswDenseArgs {
    uint32_t abi_version;
    int32_t  dtype;            /* GSW_F32 or GSW_F64 */
    int32_t  nxp, nyp, ngh;    /* padded extents; ngh >= 2 */
    int64_t  pitch;            /* row pitch of every float field, elements */
    const void* q0; const void* q1; const void* q2;   /* state in */
    void* qn0; void* qn1; void* qn2;                  /* state out (step) / residual (rhs) */
    const void* bed;
    const uint8_t* inside_mask; /* padded, pitch `mask_pitch`; NULL: every cell inside */
    int64_t  mask_pitch;
    double   inv_dx, inv_dy, g, h_min;
    /* step only */
    const GswLoopState* state; /* dt, rain frame and done flag are read from here */
    uint64_t* lam_target;     /* atomicMax target (double bits) of the new state's wave speed, or NULL */
    int32_t  rain_kind;        /* GSW_RAIN_NONE / UNIFORM / GRIDDED */
    const void* rain;          /* uniform: rates[n_frames]; gridded: frames[n_frames][nx][ny] */
    int32_t  friction_kind;    /* GSW_FRICTION_* */
    const uint8_t* n_cls; int64_t n_cls_pitch;
    const void* n_tab; int32_t n_tab_len;
    const void* n_field;       /* pitch = pitch */
    double   vcap;             /* velocity cap (inf disables) */
    int32_t  quadratic;        /* 1: quadratic alpha (default), 0: linearised */
    int32_t  keep_h;           /* 1: dry cells keep max(h,0) (default), 0: h = 0 */
    void*    max_h;            /* running max depth, pitch = pitch, or NULL */
    const uint8_t* cfl_skip;   /* interior (nx, ny) C-order: 1 = excluded from the wave speed */
    double   h_cfl;            /* wave-speed wet threshold (and divisor), > 0; h_min > 0 too */
    int32_t  tile_rows;        /* rows per warp strip; 0: the largest of 32, 16, 8, 4 that gives at least
                                  twice the warps the GPU runs at once */
    int32_t  warps;            /* warps per block (0: default 4) */
    int32_t  min_blocks;       /* register cap: 0 (compiler's choice), 3 (80 regs), 4 (64 regs) or 5 (48 regs) */
    int32_t  arith;            /* GSW_ARITH_EXACT (default), GSW_ARITH_PORTABLE, or GSW_ARITH_FAST (GSW_F32 step only) */
    /* Window of the cells computed: rows [row_lo, row_hi) x columns [col_lo, col_hi) of
     * the padded grid, inside the usual range (rows and columns [ngh, n - ngh) for the
     * step, [2, n - 2) for the residual). 0 in both ends of an axis: that whole range.
     * A run split over ranks steps the cells whose stencil reads no seam ghost while the
     * halo is in flight, then the bands next to the seams (the reference's interior /
     * band overlap, geoswe/solver.py:1750-1790). No cell's value depends on the window. */
    int32_t  row_lo, row_hi, col_lo, col_hi;
} GswDenseArgs;

/* One fused step over the interior: SRM-HLLC residual, rain, forward Euler,
 * wet/dry floor, point-implicit Manning, running max and the new state's wave
 * speed. Replaces the fused-step launch (geoswe/rhs_cuda.py:1738-1796, 2095-2192;
 * geoswe/solver.py:2166-2322) and the split path it equals (solver.py:2735-2771). */
GSW_API int gsw_dense_step(const GswDenseArgs* a, void* stream);

/* Residual only, written to qn0..qn2 (rhs0..rhs2) on cells [2, n-3]^2 with the
 * inside mask honoured; other cells are set to 0. Replaces
 * fused_rhs_linear2_lf_2d(recon="wb_srm", flux="hllc") (geoswe/rhs_cuda.py:2411-2556). */
GSW_API int gsw_dense_rhs(const GswDenseArgs* a, void* stream);

/* Wave speed of the current dense state into *lam_bits (atomicMax; caller zeroes it):
 * max over interior cells of max(|u|,|v|) + sqrt(g h), cells with h < h_cfl or
 * cfl_skip set skipped, non-finite -> +Inf. Replaces lammax_fp32_lean
 * (geoswe/solver.py:152-205). */
GSW_API int gsw_dense_lammax(const GswDenseArgs* a, uint64_t* lam_bits, void* stream);

/* Ghost fill of one dense state. kinds[4] = x-, x+, y-, y+ (GSW_BC_*).
 * Writes every ghost cell; corners come out as apply_bc_2d's x-then-y passes leave them.
 * Replaces apply_bc_2d / apply_bc_2d_face (geoswe/bc.py:50-172). */
typedef struct GswBcArgs {
    uint32_t abi_version;
    int32_t  dtype;
    int32_t  nxp, nyp, ngh;
    int64_t  pitch;
    void* q0; void* q1; void* q2;
    int32_t  kinds[4];
    const GswLoopState* state;   /* skip when state->done; may be NULL */
} GswBcArgs;
GSW_API int gsw_bc_fill(const GswBcArgs* a, void* stream);

/* Stage (Dirichlet eta) boundary applied after the step: eta(t_new) by linear
 * interpolation of (time_s, stage_m) clamped at the ends, h = max(eta - bed, 0),
 * hu = hv = 0 on the listed cells; the wave speed of those cells is folded into
 * lam_target. Replaces StageBoundary.apply (geoswe/forcing.py:315-377). */
typedef struct GswStageArgs {
    uint32_t abi_version;
    int32_t  dtype;
    int64_t  pitch;
    void* q0; void* q1; void* q2;
    const int64_t* cell_off;   /* n_cells element offsets (i*pitch + j) */
    const double*  bed64;      /* n_cells bed values (fp64 copy) */
    int32_t  bed_is_f32;       /* 1: eta - bed evaluated in fp32 (bed given as float32) */
    int32_t  n_cells;
    const double* time_s; const double* stage_m; int32_t n_knots;
    const GswLoopState* state; /* eta is taken at state->t_new */
    uint64_t* lam_target;      /* NULL: no wave-speed fold */
    const uint8_t* cfl_ghost;  /* per stage cell: 1 = excluded from the wave speed, or NULL */
    double g, h_cfl;
} GswStageArgs;
GSW_API int gsw_stage_apply(const GswStageArgs* a, void* stream);
/* Fold the wave speed of the listed cells (cell_off, n_cells; cfl_ghost excludes) into
 * lam_target, after several stage boundaries have written overlapping cells. Only the
 * q*, cell_off, n_cells, cfl_ghost, state, lam_target, g and h_cfl fields are read. */
GSW_API int gsw_lam_cells(const GswStageArgs* a, void* stream);

/* Discharge inflow through ghost cells (one inlet): Q(t) = interp(t, knots),
 * depth-weighted split w = h/sum(h) with numpy's pairwise float32 sum, dry
 * inlet seeded from the bed relief or the critical depth. Replaces
 * Solver2D._fill_inflow_ghosts / apply_inflow_discharge
 * (geoswe/solver.py:1944-1971, geoswe/bc.py:175-235). */
typedef struct GswInflowArgs {
    uint32_t abi_version;
    int32_t  dtype;
    int64_t  pitch;
    void* q0; void* q1; void* q2;
    const void* bed;
    const int64_t* inlet_off;   /* n element offsets of the inlet cells */
    int32_t  n;
    int32_t  ngh;
    int64_t  step_off;          /* offset of one cell outward along the inward normal (-(si*pitch + sj)) */
    double   nx_n, ny_n, ds, dry_frac;
    const double* t_knots; const double* q_knots; int32_t n_knots;
    const GswLoopState* state;  /* Q is taken at state->t (pre-step) */
    const double* hsum;         /* device; NULL: the depth sum of the cells above. Non-NULL: the inlet's
                                   depth sum over every rank of a split run (the per-rank sums of
                                   gsw_inflow_depth_sum added by an all-reduce), as the reference's
                                   hsum argument (geoswe/solver.py:1956-1966, geoswe/bc.py:207); the
                                   dry-inlet seed still uses this rank's cells, as there */
} GswInflowArgs;
GSW_API int gsw_inflow_apply(const GswInflowArgs* a, void* stream);
/* *out = this rank's depth sum over the inlet's cells (the pairwise float sum of
 * gsw_inflow_apply, widened to double; 0 for no cells), on the device. A split run adds
 * these over the ranks and passes the total as hsum. Replaces the per-rank sum the
 * reference's split loop feeds its Allreduce (geoswe/solver.py:1958-1963). */
GSW_API int gsw_inflow_depth_sum(const GswInflowArgs* a, double* out, void* stream);

/* ------------------------------------------------------------------------- */
/* Compressed (flat) mesh.                                                    */
/* ------------------------------------------------------------------------- */
/* Slot flags of the brick storage */
#define GSW_SLOT_STORED 1u
#define GSW_SLOT_ACTIVE 2u

typedef struct GswFlatArgs {
    uint32_t abi_version;
    int32_t  dtype;            /* GSW_F32 or GSW_F64: q*, qn*, bed, rain, n_tab and max_h */
    int32_t  brick_h;          /* rows per brick (>= 2) */
    int32_t  warps;            /* warps per block (0: 4) */
    int32_t  min_blocks;       /* fp32 step register cap: 0 (compiler's choice), 3 (80 regs), 4 (64 regs) or 5 (48 regs) */
    int32_t  arith;            /* GSW_ARITH_EXACT (default), GSW_ARITH_PORTABLE, or GSW_ARITH_FAST (GSW_F32 step only) */
    int64_t  n_bricks;         /* brick n_bricks is the all-zero brick (a missing neighbour) */
    const int32_t* brick_ij;   /* (n_bricks, 2) brick row, brick column */
    const int32_t* brick_nbr;  /* (n_bricks, 4) up, down, left, right */
    const uint8_t* flags;      /* per slot: GSW_SLOT_STORED | GSW_SLOT_ACTIVE */
    const void* q0; const void* q1; const void* q2;   /* state in, slot-indexed */
    void* qn0; void* qn1; void* qn2;                  /* state out (step) / residual (rhs) */
    const void* bed;
    double   inv_dx, inv_dy, g, h_min, h_min_cfl;     /* rounded to dtype by the kernels; h_min and
                                                         h_min_cfl (divisor floors) > 0 */
    int32_t  linf;             /* 1: CFL norm max(|u|,|v|); 0: sqrt(u^2+v^2) */
    /* step only */
    int32_t  rain_kind;        /* GSW_RAIN_NONE / UNIFORM / GRIDDED / LOOKUP */
    const GswLoopState* state;
    uint64_t* lam_target;
    const void* rain;          /* uniform: rates[n_frames]; gridded: frames[n_frames][nx][ny];
                                  lookup: rows[n_frames][rain_ncol] (the reference's cached table) */
    int32_t  ngh, nx, ny;      /* dense padding and interior extents (gridded rain index) */
    int32_t  n_tab_len;
    const uint8_t* n_cls; const void* n_tab;
    double   vcap;
    int32_t  quadratic, keep_h;
    void*    max_h;            /* slot-indexed, or NULL */
    const int32_t* rain_lookup;/* GSW_RAIN_LOOKUP: per slot, the column of rain[frame * rain_ncol + col] */
    int32_t  rain_ncol;
    int32_t  segments;         /* warps per brick: 1 (one warp walks the brick's rows), 2 or 4 (each walks
                                  brick_h / segments rows: shorter per-warp latency for small meshes),
                                  0 (chosen from the brick count against the warps the GPU runs at once) */
    int64_t  brick_lo, brick_hi; /* step: update bricks [brick_lo, brick_hi) only (a split run steps the
                                  bricks that read no seam ghost cell while the seam exchange is in flight,
                                  then the rest); 0, 0: every brick. Ignored by the wave-speed pass. */
} GswFlatArgs;

/* Discharge inlet of the compressed mesh: one ghost (ring) slot per inlet cell, next to
 * its active neighbour. Per step, at state->t: Q = np.interp(t, t_knots, q_knots);
 * wet inlet (sum of the neighbours' depths > 0): ghost h = neighbour h, unit discharge
 * (float)(Q/ds) * h/sum; dry inlet: depth seeded from the bed relief of the neighbours
 * (10 %), plus the critical depth where that relief is flat, flow in the lowest cells.
 * Ghost hu, hv = unit discharge * inward normal. Replaces the flat loop's inlet block
 * and its dry seed (geoswe/compressed_solver.py:2144-2167, 1559-1594). The depth sum
 * is taken in NumPy's pairwise order (bitwise with a NumPy sum; the reference's CuPy
 * reduction may order a multi-cell sum differently, so results can differ there in
 * the last bit of the weights). */
typedef struct GswFlatInflowArgs {
    uint32_t abi_version;
    int32_t  dtype;               /* GSW_F32 or GSW_F64 */
    void* q0; void* q1; void* q2; /* brick storage, written at the ghost slots */
    const void* bed;
    const int64_t* ghost_slot;    /* n ghost slots */
    const int64_t* nbr_slot;      /* n active neighbour slots */
    int32_t  n;
    int32_t  n_knots;
    double   nx_n, ny_n, ds;      /* inward unit normal (axis-aligned) and cell width */
    const double* t_knots; const double* q_knots;
    const GswLoopState* state;    /* Q is taken at state->t; nothing is written when done */
    const double* hsum;           /* device; NULL: the neighbours' depth sum above. Non-NULL: the inlet's
                                     depth sum over every rank of a split run (the per-rank sums of
                                     gsw_flat_inflow_depth_sum added by an all-reduce), as the
                                     reference's split loop does (geoswe/compressed_solver.py:2145-2153) */
    const double* dry;            /* device; NULL: the dry-inlet seed's bed range and counts come from the
                                     cells above. Non-NULL: 4 doubles {zmin, zmax, nlow, hmax} over every
                                     rank's cells of the inlet (bed minimum and maximum, cells at the
                                     minimum, largest seed depth), as the reference reduces them once over
                                     the ranks (geoswe/compressed_solver.py:1559-1594) */
} GswFlatInflowArgs;
GSW_API int gsw_flat_inflow_apply(const GswFlatInflowArgs* a, void* stream);
/* *out = this rank's depth sum over the inlet's active neighbours (the pairwise float sum
 * of gsw_flat_inflow_apply, widened to double; 0 for none), on the device. Replaces the
 * per-rank sum of the reference's split flat loop (geoswe/compressed_solver.py:2147). */
GSW_API int gsw_flat_inflow_depth_sum(const GswFlatInflowArgs* a, double* out, void* stream);

/* Stage on ghost-ring cells of the compressed mesh, applied after the step at the
 * step's start time state->t: per gauge g the stage is interpolated in the (NG, n_t)
 * table at ti = clamp(searchsorted_left(t_common, t) - 1, 0, n_t - 2) with weight
 * wt = clamp((t - t_common[ti]) / (t_common[ti+1] - t_common[ti] + 1e-12), 0, 1) as
 * stage[g][ti]*(1-wt) + stage[g][ti+1]*wt in the array type; per ring cell k,
 * eta = sum_g wg[k][g] * stage_g, h = max(0, eta - bed[k]), hu = hv = 0. Replaces
 * ring_bc_flat and its on-device interpolation (geoswe/compressed_solver.py:287-307,
 * 1622-1634, 2338-2350). Nothing is written when state->done. */
typedef struct GswFlatRingArgs {
    uint32_t abi_version;
    int32_t  dtype;              /* GSW_F32 or GSW_F64 */
    void* q0; void* q1; void* q2;/* brick storage */
    const int64_t* slots;        /* n ring slots (-1: not stored, skipped) */
    const void* bed;             /* n ring-cell beds */
    const void* wg;              /* (n, NG) gauge weights */
    int32_t  n, NG;
    const double* t_common;      /* n_t >= 2 increasing times */
    int32_t  n_t;
    int32_t  reserved0;
    const void* stage_all;       /* (NG, n_t) gauge stages (m) */
    const GswLoopState* state;
} GswFlatRingArgs;
GSW_API int gsw_flat_ring_stage(const GswFlatRingArgs* a, void* stream);

/* Per-step forcings of the flat loop, applied after the step in the reference's order
 * (geoswe/compressed_solver.py:2330-2366): phase 0 = landcover infiltration
 * (infiltrate_flat, :143-158), then the open-boundary sponge band (sponge_band,
 * :1320-1328); the ring stage (gsw_flat_ring_stage) comes between; phase 1 = Green-Ampt
 * infiltration with the linear-reservoir drain (ga_drain_flat / ga_flat / drain_tau_flat,
 * :313-420), the stage clamp (stage_clamp_flat, :422-437), then the karst drain cap
 * (drain_cap, :268-283). Each part is skipped when its pointers are NULL. dt is the
 * step's state->dt_f32; nothing runs when state->done. fp32 only, as the reference. */
typedef struct GswFlatForcingArgs {
    uint32_t abi_version;
    int32_t  phase;                 /* 0 or 1 (above) */
    float* q0; float* q1; float* q2;/* brick storage */
    const uint8_t* flags;           /* slot flags; forcings over all slots touch active slots only */
    int64_t  nslots;
    float    h_min;
    int32_t  reserved0;
    const GswLoopState* state;
    /* landcover infiltration: rate infil_tab[n_cls[slot]] (m/s) */
    const uint8_t* n_cls; const float* infil_tab;
    /* sponge band: q0 = q0*keep + amb, q1, q2 *= keep on the listed slots */
    const int64_t* sp_slots; const float* sp_keep; const float* sp_amb; int32_t sp_n;
    /* Green-Ampt / drain: 1 fused, 2 Green-Ampt only, 3 drain only (0 off); per-slot
       class, cumulative infiltration F (state, updated), cap Fmax, drain rate inv_tau */
    int32_t  ga_mode;
    const uint8_t* ga_cls; const float* Ks_t; const float* psi_t; const float* dth_t;
    float* F; const float* Fmax; const float* inv_tau;
    /* stage clamp: h <= h_max on the listed slots, momentum scaled */
    const int64_t* cl_slots; const float* cl_hmax; int32_t cl_n;
    /* karst drain cap: h <= h_tgt on the listed slots, momentum scaled */
    int32_t  dr_n;
    const int64_t* dr_slots; const float* dr_htgt;
} GswFlatForcingArgs;
GSW_API int gsw_flat_forcings(const GswFlatForcingArgs* a, void* stream);

/* Fused step on the compressed mesh: active cells get the SRM-HLLC residual, rain,
 * Euler, wet/dry and Manning (table); stored ring cells are carried unchanged.
 * Replaces the flat fused step + CFL launch (geoswe/compressed_rhs.py:673-865, 990-1118;
 * geoswe/compressed_solver.py:819-905). Residuals of active cells are bit-identical to
 * the dense kernel's at the same state. */
GSW_API int gsw_flat_step(const GswFlatArgs* a, void* stream);
/* Residual of active cells into qn0..qn2 (0 at ring cells and empty slots). Replaces
 * CompressedSWE.run_rhs / CompressedStepper.rhs (geoswe/compressed_rhs.py:355-369). */
GSW_API int gsw_flat_rhs(const GswFlatArgs* a, void* stream);
/* Wave speed of active cells of the current state into *lam_bits (atomicMax).
 * Replaces cfl_lammax_flat_blk[_ns] (geoswe/compressed_solver.py:209-244). */
GSW_API int gsw_flat_lammax(const GswFlatArgs* a, uint64_t* lam_bits, void* stream);

/* Host-side compressed-mesh construction (gsw_mesh.cpp). */
GSW_API int gsw_mesh_count(const uint8_t* inside, int nxp, int nyp, int ring,
                           int64_t* n_stored, int64_t* n_active);
GSW_API int gsw_mesh_build(const uint8_t* inside, int nxp, int nyp, int ring, int32_t* ij,
                           int16_t* nbr16, uint8_t* is_active, int32_t* active_id, int32_t* covered);
GSW_API int gsw_bricks_build(const uint8_t* stored, int nxp, int nyp, int brick_h,
                             int64_t* n_bricks, int32_t* brick_ij, int32_t* brick_nbr);
/* Canonical cell k (padded row, column ij[2k], ij[2k+1], as gsw_mesh_build returns
 * them) -> its slot in brick storage, for bricks from gsw_bricks_build. A host that
 * keeps the reference's canonical flat arrays uses it to scatter them into brick
 * storage and gather results back. No counterpart in the reference (its kernels read
 * the canonical arrays directly). */
GSW_API int gsw_bricks_slot_of(const int32_t* ij, int64_t n_cells, const int32_t* brick_ij, int64_t n_bricks,
                               int brick_h, int nxp, int nyp, int64_t* slot_of);

/* ------------------------------------------------------------------------- */
/* Adjoint of the compressed-mesh step. No counterpart in the reference, which */
/* has no derivatives; it reverses gsw_flat_step (+ gsw_flat_inflow_apply)     */
/* for calibration of Manning's n, the rain scale and inlet hydrographs.       */
/* ------------------------------------------------------------------------- */
typedef struct GswFlatAdjArgs {
    uint32_t abi_version;
    int32_t  min_blocks;  /* register cap of the binary32 reverse kernels: 0 (compiler's), 6 (80), 8 (64 regs) */
    GswFlatArgs f;     /* the step being reversed: q* = the state it read (inlet ghosts written),
                          state = its dt, rain frame and step index (steps); qn*, max_h unused */
    const void* lam_in0; const void* lam_in1; const void* lam_in2;   /* adjoint of the new state */
    void* lam_out0; void* lam_out1; void* lam_out2;                   /* adjoint of the old state (written) */
    void* rbar0; void* rbar1; void* rbar2;   /* scratch of the residual adjoints, slot-indexed; must be
                                                zero on every slot that is not stored (and the zero brick) */
    double*  n_bar;    /* += dL/dn per Manning class (f.n_tab_len <= 256) */
    double*  rate_bar; /* uniform rain: rate_bar[state->steps] += dL/d(rate of this step), or NULL */
} GswFlatAdjArgs;
/* lam_out = (d step / d q)^T lam_in with dt, the rain frame and every branch of the
 * forward step held fixed; n_bar and rate_bar accumulate. Two launches. */
GSW_API int gsw_adj_flat_step(const GswFlatAdjArgs* a, void* stream);
/* Reverse of gsw_flat_inflow_apply for the same state and time: the ghost slots'
 * adjoint (lam*) moves to the inlet's active cells and to q_bar[state->steps]
 * (dL/dQ of this step); the ghost slots' adjoint is then zeroed. */
GSW_API int gsw_adj_flat_inflow(const GswFlatInflowArgs* a, void* lam0, void* lam1, void* lam2,
                                double* q_bar, void* stream);

/* Gauge series: depth at n slots, recorded per step, and the adjoint of a squared misfit. */
typedef struct GswGaugeArgs {
    uint32_t abi_version;
    int32_t  dtype;
    const void* q0;          /* depth, slot-indexed */
    const int64_t* slots;
    int32_t  n;
    int32_t  offset;         /* row = state->steps + offset - first (state NULL: steps = 0) */
    int64_t  first, count;   /* rows [0, count) are kept */
    double*  series;         /* record: (count, n) */
    const double* target;    /* adjoint: (count, n) */
    double   weight;         /* adjoint: lam0[slot] += weight * 2 * (depth - target) */
    void*    lam0;
    const GswLoopState* state;
} GswGaugeArgs;
GSW_API int gsw_gauge_record(const GswGaugeArgs* a, void* stream);
GSW_API int gsw_gauge_adjoint(const GswGaugeArgs* a, void* stream);

/* ------------------------------------------------------------------------- */
/* Batched ensemble: many compressed meshes advanced by one kernel per step.  */
/* No counterpart in the reference, which runs scenarios one after another    */
/* (a Python loop over CompressedSolver.run, geoswe/compressed_solver.py:     */
/* 3359); each member follows that solver's flat loop exactly.                */
/* ------------------------------------------------------------------------- */
/* Physics and time-step rule of one member. */
typedef struct GswMember {
    GswDtParams dt;          /* the member's flat time-step rule (rain limit folded into dt_max) */
    float    inv_dx, g, h_min, h_min_cfl, vcap;    /* h_min, h_min_cfl > 0 (divisor floors) */
    int32_t  linf, quadratic, keep_h;
    int32_t  rain_kind;      /* GSW_RAIN_NONE or GSW_RAIN_UNIFORM */
    float    g_recip;        /* gsw_div_const_recip(g), or 0 (the star depth's h / g divides) */
    const float* rain;       /* uniform rate (m/s) per rain frame */
    const float* n_tab;      /* the member's Manning class table */
} GswMember;

typedef struct GswEnsembleArgs {
    uint32_t abi_version;
    int32_t  brick_h;
    int64_t  n_bricks;           /* bricks of all members; brick n_bricks is the zero brick */
    int32_t  n_members;
    int32_t  warps;              /* warps per block (0: 4) */
    int32_t  grid;               /* persistent blocks (0: 2 per SM) */
    int32_t  min_blocks;         /* register cap: 0 (compiler's choice), 3 (80 regs), 4 (64 regs) or 5 (48 regs) */
    int32_t  arith;              /* GSW_ARITH_EXACT (default), GSW_ARITH_PORTABLE or GSW_ARITH_FAST */
    int32_t  segments;           /* warps per brick: 1, 2 or 4 (as GswFlatArgs.segments), or 0: chosen per
                                    launch from the running members' bricks against the grid's warps */
    const int32_t* brick_ij;     /* (n_bricks, 2) */
    const int32_t* brick_nbr;    /* (n_bricks, 4) global brick ids */
    const int32_t* brick_member; /* (n_bricks) */
    const uint8_t* flags;        /* per slot */
    const uint8_t* n_cls;        /* per slot, or NULL (class 0) */
    const float* q0; const float* q1; const float* q2;
    float* qn0; float* qn1; float* qn2;
    const float* bed;
    float*   max_h;              /* per slot, or NULL */
    const GswMember* members;    /* device, n_members */
    GswLoopState* states;        /* device, n_members */
    uint32_t* scratch;           /* device, GSW_ENS_SCRATCH_WORDS (2) words, zero before the first step: the
                                    block ticket and the work-item counter. Read by gsw_ensemble_step only
                                    (gsw_ensemble_finalize zeroes it when non-NULL); may be NULL for
                                    gsw_ensemble_lammax, gsw_ensemble_finalize and gsw_ensemble_step_static */
    int32_t* all_done;           /* device int: 1 once every member is done */
    /* Running-member brick list (optional; NULL: every launch scans all bricks and skips
       finished members brick by brick). member_brick_off: device, n_members + 1, member
       k's bricks are [off[k], off[k+1]). run: device, 2 * n_members + 2 words, written by
       gsw_ensemble_finalize and rebuilt by the step when a member finishes: run[0] = the
       running count R, run[1 .. R+1] = their brick-count prefix, run[n_members + 2 + i]
       = the i-th running member. A launch then visits running members' bricks only. */
    const int64_t* member_brick_off;
    int64_t* run;
    int32_t  lean;               /* 1: every member has quadratic = 1, keep_h = 1 and linf = 0 (the production
                                    configuration), which the step then compiles in (bit-identical results); a
                                    member that has not is stopped with states[m].error = GSW_ERR_INVALID.
                                    0: the general step. */
} GswEnsembleArgs;

/* Wave speed of every member's current state into states[m].lam_bits (atomicMax). */
GSW_API int gsw_ensemble_lammax(const GswEnsembleArgs* a, void* stream);
/* Each member's dt / rain frame / done from states[m].lam_bits (the flat loop's rule);
 * sets *all_done. */
GSW_API int gsw_ensemble_finalize(const GswEnsembleArgs* a, void* stream);
/* One step of every member that is not done, in one persistent launch: warps take
 * bricks from the whole ensemble, each with its member's dt, rain and Manning table,
 * and reduce the member's new wave speed; the last block to finish computes every
 * member's next dt (no grid barrier). A member's trajectory equals its CompressedSolver
 * run bit for bit. */
GSW_API int gsw_ensemble_step(const GswEnsembleArgs* a, void* stream);

/* gsw_ensemble_step without caller scratch. No counterpart in the reference (its
 * scenarios run one after another, with no device scratch).
 * The step's scratch is its block ticket counter and its work-item counter:
 * GSW_ENS_SCRATCH_WORDS uint32 words, zero before a launch and left at zero by it. This entry point keeps those words in a
 * static, 256-byte aligned device array of the library (GSW_ENS_STATIC_SCRATCH_WORDS
 * words per device) and ignores a->scratch; a requirement above that size is refused
 * with GSW_ERR_RANGE. It allocates nothing: on the first call on a device it looks the
 * array up (cudaGetSymbolAddress) and zeroes it on `stream`, so make that first call
 * outside any stream capture. With gsw_ensemble_lammax and gsw_ensemble_finalize, which
 * accept a->scratch == NULL, a whole ensemble loop runs on caller state and fields alone.
 * When the step returns an error, the words are zeroed again on `stream`. The address is
 * looked up once per device and process: a cudaDeviceReset after the first call is not
 * supported. The array is shared by all callers on a device: calls whose launches
 * overlap in time (other streams, other threads) race on the ticket counter and must be
 * serialised by the caller. */
#define GSW_ENS_SCRATCH_WORDS        2
#define GSW_ENS_STATIC_SCRATCH_WORDS 64
GSW_API int gsw_ensemble_step_static(const GswEnsembleArgs* a, void* stream);

/* ------------------------------------------------------------------------- */
/* Loop control.                                                              */
/* ------------------------------------------------------------------------- */
/* Commit the pending t/steps, test the loop condition, and compute this step's dt
 * and rain frame from state->lam_bits (then zeroed for the step's reduction). */
GSW_API int gsw_dt_finalize(const GswDtParams* p, GswLoopState* state, void* stream);
/* Device-resident parameters, for loops captured once in a CUDA graph and replayed
 * for any t_end / dt_max / max_steps: gsw_dt_params_upload validates *p on the host
 * and copies it to `dev` (device memory, sizeof(GswDtParams) bytes) on `stream`;
 * gsw_dt_finalize_dev is gsw_dt_finalize reading the parameters from `dev` when it
 * runs. Replaces the same host-side dt computation as gsw_dt_finalize. */
GSW_API int gsw_dt_params_upload(const GswDtParams* p, GswDtParams* dev, void* stream);
GSW_API int gsw_dt_finalize_dev(const GswDtParams* dev, GswLoopState* state, void* stream);
/* Commit a pending t_new/steps (call once after the last step). */
GSW_API int gsw_loop_commit(GswLoopState* state, void* stream);

/* ------------------------------------------------------------------------- */
/* Launch-shape search (no counterpart in the reference: its launch shapes are */
/* fixed). Times the fused step at every shape of the search space with CUDA   */
/* events on `stream` and the caller's buffers, and returns the fastest:       */
/*   dense: tile_rows {0 (automatic), 4, 8, 16, 32, 64} x warps {2, 4, 8} x     */
/*          register cap min_blocks {0, 3, 4, 5}                               */
/*   flat:  warps {2, 4, 8} x min_blocks {0, 3, 4, 5} x segments {0, 1, 2, 4}   */
/* The step's outputs (qn*) are overwritten; lam_target and max_h are not      */
/* touched; the loop state is read (it must not be done). Results are cached   */
/* per device, kernel family, arithmetic, dtype and size class (< 2^20,        */
/* < 2^24, larger) behind a mutex; use_cache = 1 returns a cached result       */
/* without launching.                                                          */
/* ------------------------------------------------------------------------- */
typedef struct GswTuneResult {
    uint32_t abi_version;      /* GSW_ABI_VERSION, set by the caller (the rest is written by the library) */
    int32_t  tile_rows;        /* dense */
    int32_t  warps;
    int32_t  min_blocks;
    int32_t  segments;         /* flat */
    int32_t  n_tried;          /* shapes timed */
    float    ms;               /* mean launch time of the winner */
    int32_t  reserved;
} GswTuneResult;
GSW_API int gsw_dense_autotune(const GswDenseArgs* a, int32_t reps, int32_t use_cache, GswTuneResult* out,
                               void* stream);
GSW_API int gsw_flat_autotune(const GswFlatArgs* a, int32_t reps, int32_t use_cache, GswTuneResult* out,
                              void* stream);

/* ------------------------------------------------------------------------- */
/* Split runs                                                                 */
/* ------------------------------------------------------------------------- */
/* Seam exchange of a compressed mesh split over ranks: the pack and unpack of the
 * reference's CompressedHalo (geoswe/compressed_solver.py:1069-1132, its per-face
 * gathers into and scatters out of a dense (3, ngh, P) face buffer), on brick slots.
 *   scatter = 0: dense[c * stride + pos[k]] = q_c[slot[k]]      (gather, before sending)
 *   scatter = 1: q_c[slot[k]] = dense[c * stride + pos[k]]      (after receiving)
 * for k < n and c = 0, 1, 2. An entry with slot outside [0, nslots) or pos outside
 * [0, stride) is skipped (the caller validates both lists once, when it builds them). */
typedef struct GswSeamArgs {
    uint32_t abi_version;
    int32_t  dtype;          /* GSW_F32 or GSW_F64 */
    void* q0; void* q1; void* q2;
    int64_t  nslots;
    const int64_t* slot;     /* n brick slots */
    const int64_t* pos;      /* n dense positions */
    int64_t  n;
    void*    dense;          /* 3 * stride elements */
    int64_t  stride;
    int32_t  scatter;
    int32_t  reserved;
} GswSeamArgs;
GSW_API int gsw_seam_copy(const GswSeamArgs* a, void* stream);

/* ------------------------------------------------------------------------- */
/* Library                                                                    */
/* ------------------------------------------------------------------------- */
/* RN(1/g) when the reciprocal-and-remainder sequence the step uses for the HLLC star
 * depth's h / g reproduces the IEEE quotient for every binary32 significand of h (an
 * exhaustive check, once per g per process), else 0. The dense and flat steps apply it
 * themselves; an ensemble caller passes it in GswMember.g_recip. */
GSW_API float gsw_div_const_recip(float g);
GSW_API const char* gsw_last_error(void);
GSW_API uint32_t    gsw_abi_version(void);
/* Number of this library's kernels launched since load (all entry points). */
GSW_API uint64_t    gsw_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* GSW_H */
