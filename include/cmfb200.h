/*
 * cmfb200.h -- C ABI of libcmfb200.so, the B200 (sm_100a) river-routing core.
 *
 * This library replaces the per-sub-step routing path of CaMa-Flood-GPU: the
 * native launchers in cmfgpu/phys/cuda/*.cu (bound there through hydroforge's
 * CudaExtensionGroup, cmfgpu/phys/cuda/__init__.py:68-166).  Instead of one
 * at::Tensor launcher per physics phase, a caller describes all model tensors
 * once in a CmfView (plain device pointers + sizes), creates a plan, and then
 * advances whole forcing intervals.  Per-phase entry points remain for parity
 * work.  No torch type crosses this boundary.
 *
 * Ownership: every buffer in CmfView is owned by the caller.  The library never
 * allocates device memory on the step path; cmf_plan_create allocates only the
 * plan object (host) and, lazily, its CUDA graph.  Scratch lives in the
 * caller-provided workspace (size from cmf_workspace_size).
 *
 * Errors: every entry point returns an int status (CMF_OK == 0).  Kernels
 * report numeric trouble through the device status word (CmfView.status).
 * Nothing aborts the process.
 *
 * Threading: one host thread per plan.  All work is enqueued on the caller's
 * stream.
 */
#ifndef CMFB200_H
#define CMFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMF_ABI_VERSION 1

/* ---- return codes ------------------------------------------------------- */
#define CMF_OK 0
#define CMF_ERR_ARG 1         /* invalid argument / inconsistent view       */
#define CMF_ERR_CUDA 2        /* a CUDA runtime call failed                  */
#define CMF_ERR_TIMEOUT 3     /* a bounded device wait gave up               */
#define CMF_ERR_NUMERIC 4     /* device status word reported a bad value     */
#define CMF_ERR_UNSUPPORTED 5 /* feature combination not compiled            */

/* ---- device status word bits (CmfView.status[0]) ------------------------- */
#define CMF_STATUS_NONFINITE 1   /* NaN/Inf storage or discharge produced     */
#define CMF_STATUS_SUBSTEP_CAP 2 /* CFL asked for more sub-steps than allowed */
#define CMF_STATUS_SYNC_TIMEOUT 8 /* a grid barrier of the persistent interval kernel gave up */

/* ---- feature bits (CmfView.features) ------------------------------------- */
#define CMF_FEAT_BIFURCATION 1 /* bifurcation module open                    */
#define CMF_FEAT_LEVEE 2       /* levee module open                          */
#define CMF_FEAT_RESERVOIR 4   /* reservoir module open                      */
#define CMF_FEAT_ADAPTIVE 8    /* adaptive_time module open (CFL sub-steps)  */
#define CMF_FEAT_BUDGET 16     /* accumulate the fp64 water budget           */
#define CMF_FEAT_FP64 32       /* REAL fields are double (else float)        */
#define CMF_FEAT_GRAPH 64      /* run intervals through a CUDA graph         */

/* ---- per-catchment flag bits (CmfView.cell_flags) ------------------------ */
#define CMF_CELL_MOUTH 1
#define CMF_CELL_LEVEE 2
#define CMF_CELL_RESERVOIR 4
#define CMF_CELL_DAM_UPSTREAM 8
#define CMF_CELL_DAM_RELATED 16
#define CMF_CELL_BIFURCATION 32

/* ---- member-batched parameter bits (CmfView.batched_mask) ---------------- */
/* A set bit means the parameter is stored [N, M] member-innermost instead of
 * shared [N].  State fields are always [N, M]. */
#define CMF_BATCH_RUNOFF 1
#define CMF_BATCH_RIVER_MANNING 2
#define CMF_BATCH_FLOOD_MANNING 4
#define CMF_BATCH_RIVER_WIDTH 8
#define CMF_BATCH_RIVER_HEIGHT 16
#define CMF_BATCH_RIVER_LENGTH 32

/* ---- fp64 water budget terms (CmfView.budget) ----------------------------- */
#define CMF_BUDGET_STORAGE_START 0 /* sum of storage at interval start (m3)  */
#define CMF_BUDGET_STORAGE_END 1   /* sum of storage at interval end (m3)    */
#define CMF_BUDGET_RUNOFF_IN 2     /* runoff volume added (m3)               */
#define CMF_BUDGET_MOUTH_OUT 3     /* volume leaving through mouths (m3)     */
#define CMF_BUDGET_CLIP_GAIN 4     /* volume created by clipping at zero     */
#define CMF_BUDGET_SUBSTEPS 5      /* sub-steps accumulated                  */
#define CMF_BUDGET_TERMS 6

/*
 * CmfView: every tensor of the model, by the reference's field names.
 * REAL pointers are float* unless CMF_FEAT_FP64 is set; STO pointers are
 * always double* (the reference "hpfloat" storage dtype).  Catchment-indexed
 * arrays are in the plan's catchment order, which MUST be the basin-major
 * breadth-first order produced by cmf_topo_bfs_order: the upstream cells of p
 * are [upstream_ptr[p], upstream_ptr[p+1] - m), m = 1 when p+1 is a mouth
 * and 0 otherwise.  With M > 1 members every state
 * field is [N, M] with the member index innermost.
 * Field order is part of the ABI; cmf_view_field_offsets() reports it.
 */
typedef struct CmfView {
    int32_t abi_version;
    int32_t features;
    int64_t num_catchments;          /* N */
    int32_t num_members;             /* M, 1 for the plain model */
    int32_t num_flood_levels;        /* K, columns of flood_depth_table */
    int64_t num_bifurcation_paths;   /* P */
    int32_t num_bifurcation_levels;  /* L */
    int32_t batched_mask;            /* CMF_BATCH_* bits */
    int64_t num_levees;
    int64_t num_reservoirs;
    double gravity;                  /* base.gravity (9.8) */
    double min_kinematic_slope;      /* base.min_kinematic_slope (1e-5) */
    double adaptive_time_factor;     /* adaptive_time.adaptive_time_factor */
    double max_sub_step_seconds;     /* optional dt cap, 0 = none */
    int32_t max_sub_steps_cap;       /* reject intervals needing more; 0 = none */
    int32_t block_size;              /* threads per CTA (autotuned), 0 = default */

    /* topology (device, int32 / uint8) */
    const int32_t* downstream_idx;   /* [N], self at mouths */
    const int32_t* upstream_ptr;     /* [N+1] */
    const uint8_t* cell_flags;       /* [N] CMF_CELL_* */
    const int32_t* levee_slot;       /* [N] levee index or -1 */
    const int32_t* reservoir_slot;   /* [N] reservoir index or -1 */
    const int32_t* bif_cell_ptr;     /* [N+1] incident-path CSR */
    const int32_t* bif_cell_paths;   /* [2P] 2*path + (cell is downstream end) */

    /* base parameters (REAL, [N] or [N,M] by batched_mask) */
    const void* river_width;
    const void* river_length;
    const void* river_height;
    const void* catchment_elevation;
    const void* catchment_area;
    const void* downstream_distance;
    const void* river_manning;
    const void* flood_manning;
    const void* flood_depth_table;   /* [N, K] row-major */
    const void* runoff;              /* m3/s */

    /* base state (REAL) */
    void* river_outflow;
    void* flood_outflow;
    void* river_depth;
    void* flood_depth;
    void* protected_depth;
    void* river_cross_section_depth;
    void* flood_cross_section_depth;
    void* flood_cross_section_area;
    void* flood_fraction;
    /* base state (STO = double) */
    double* river_storage;
    double* flood_storage;
    double* protected_storage;

    /* diagnostics written on the last sub-step of an interval (optional) */
    double* river_inflow;
    double* flood_inflow;
    double* outgoing_storage;
    double* total_storage;
    double* global_bifurcation_outflow;
    void* limit_rate;
    void* water_surface_elevation;
    void* protected_water_surface_elevation;

    /* bifurcation module */
    const int32_t* bifurcation_catchment_idx;   /* [P] */
    const int32_t* bifurcation_downstream_idx;  /* [P] */
    const void* bifurcation_manning;            /* [P, L] */
    const void* bifurcation_width;              /* [P, L] */
    const void* bifurcation_length;             /* [P] */
    const void* bifurcation_elevation;          /* [P, L] */
    void* bifurcation_outflow;                  /* [P, L] (x M) */
    void* bifurcation_cross_section_depth;      /* [P, L] (x M) */

    /* levee module (per levee, [Lv]) */
    const int32_t* levee_catchment_idx;
    const void* levee_crown_height;
    const void* levee_fraction;
    const void* levee_base_height;

    /* reservoir module (per reservoir, [R]) */
    const int32_t* reservoir_catchment_idx;
    const void* conservation_volume;
    const void* emergency_volume;
    const void* adjustment_volume;
    const void* effective_normal_outflow;
    const void* adjustment_outflow;
    const void* flood_control_outflow;
    double* reservoir_total_inflow;             /* [N] (x M) */

    /* time control (device) */
    void* time_step;                 /* [M] REAL sub-step length */
    void* outer_time_step;           /* [1] REAL forcing interval */
    int32_t* max_sub_steps;          /* [M] sub-step count of the interval */
    int32_t* current_step;           /* [1] */

    /* fp64 water budget, accumulated (optional, CMF_BUDGET_TERMS x M) */
    double* budget;
    /* device status word (CMF_STATUS_* bits), [1] */
    int32_t* status;

    /* caller-provided scratch */
    void* workspace;
    size_t workspace_bytes;
} CmfView;

typedef struct CmfPlan CmfPlan;

/* ---- library / ABI introspection ----------------------------------------- */
int cmf_abi_version(void);
const char* cmf_status_string(int code);
/* Byte offsets of every CmfView field in declaration order; returns the
 * number of fields (writes at most cap entries). */
int cmf_view_field_offsets(int64_t* offsets, int cap);
size_t cmf_view_size(void);

/* ---- plan lifecycle ------------------------------------------------------ */
/* Bytes of scratch the view needs (Qu fluxes, path sums, budget partials,
 * levee-indexed copies of the levee cells' static fields and marks). */
int cmf_workspace_size(const CmfView* view, size_t* bytes);
/* Validate the view and bind a plan to its pointers (cmfgpu phys dispatch:
 * BackendRegistry(...).selected binding by parameter name,
 * cmfgpu/phys/outflow.py:51-60).  With levees, the plan copies each levee
 * cell's floodplain row and (when not member-batched) river height, width
 * and length into the workspace once, synchronously, and with that shared
 * geometry computes each levee's marks: the storages at which its regimes
 * change (profile filled to the base and to the crown, the river-side wedge)
 * and its layer geometry.  A caller that changes those parameters afterwards
 * creates a new plan. */
int cmf_plan_create(const CmfView* view, CmfPlan** plan);
void cmf_plan_destroy(CmfPlan* plan);
/* Persistent interval kernel (no counterpart in the reference; it replaces
 * the per-sub-step launch loop of cmfgpu/models/cama_flood_model.py:134-162
 * for small networks).  enable != 0: cmf_step_interval runs every sub-step of
 * an interval in one cooperative launch whose blocks meet at a grid-wide
 * barrier after each phase, instead of the interval graph.  Results are the
 * same.  One member only, no budget and no output statistics
 * (CMF_ERR_UNSUPPORTED otherwise, and cmf_stats_attach refuses while it is
 * on); the grid is the device's resident CTAs, or fewer when the network
 * needs fewer.  A barrier wait that outlasts 1 s raises
 * CMF_STATUS_SYNC_TIMEOUT and ends the interval.  enable == 0 returns to the
 * interval graph. */
int cmf_plan_set_persistent(CmfPlan* plan, int enable);
/* Test of the persistent kernel's failure path (no counterpart in the
 * reference): launches, cooperatively, two blocks that meet at a grid barrier
 * waiting for one arrival more than they make, so each wait gives up after
 * timeout_us (1 .. 1,000,000), sets CMF_STATUS_SYNC_TIMEOUT in *status and
 * the abort word in control[6], and returns; nothing hangs.  control: 16
 * device int32 words, zeroed by the caller, 8-byte aligned. */
int cmf_probe_barrier_timeout(void* stream, int32_t* control, int32_t* status, int32_t timeout_us);
/* Member-tile width of the member-batched kernels (no counterpart in the
 * reference): each thread handles `width` consecutive members of one
 * catchment, so the catchment's shared fields are loaded once from HBM and
 * then from L1.  width divides num_members (1 for one member); the default is
 * 1, and the interval graph is rebuilt on the next step.  The autotuner picks
 * it with the block size. */
int cmf_plan_set_member_tile(CmfPlan* plan, int32_t width);

/* ---- the step path ------------------------------------------------------- */
/* Advance one forcing interval of `outer_seconds`.  Replaces the body of
 * CaMaFlood.step_advance (cmfgpu/models/cama_flood_model.py:104-173):
 * adaptive sub-step count on the device (no host sync), dt = T / n, then n
 * sub-steps of momentum -> limiter/inflow/stage.  fixed_sub_steps > 0 skips
 * the CFL and uses that count (the reference's fixed mode). */
int cmf_step_interval(CmfPlan* plan, void* stream, double outer_seconds,
                      int32_t fixed_sub_steps);

/* ---- per-phase entry points (parity / debugging) ------------------------- */
/* Momentum phase of one sub-step.  Replaces, fused:
 *   launch_outflow            cmfgpu/phys/cuda/outflow.cu:272-367
 *   launch_reservoir_outflow  cmfgpu/phys/cuda/reservoir.cu:327-363
 *   launch_bif_outflow        cmfgpu/phys/cuda/bifurcation.cu:158-199
 *   launch_levee_bif_outflow  cmfgpu/phys/cuda/levee.cu:424-466
 * Writes the unlimited fluxes to the workspace and the cross-section state in
 * place.  diag != 0 also writes water_surface_elevation,
 * protected_water_surface_elevation and total_storage. */
int cmf_phase_momentum(CmfPlan* plan, void* stream, int diag);
/* Limiter + inflow + storage/stage phase of one sub-step.  Replaces, fused:
 *   launch_inflow             cmfgpu/phys/cuda/outflow.cu:389-422
 *   launch_bif_inflow         cmfgpu/phys/cuda/bifurcation.cu:201-231
 *   launch_flood_stage(_log)  cmfgpu/phys/cuda/storage.cu:318-445
 *   launch_levee_stage(_log)  cmfgpu/phys/cuda/levee.cu:343-422
 * The upstream inflow is a deterministic gather over upstream_ptr instead of
 * fp64 atomics.  diag != 0 also writes river_inflow, flood_inflow,
 * limit_rate, global_bifurcation_outflow and protected_depth of non-levee
 * cells. */
int cmf_phase_stage(CmfPlan* plan, void* stream, int diag);
/* Adaptive sub-step count and dt for an interval of outer_seconds.  Replaces
 *   launch_adaptive_time      cmfgpu/phys/cuda/adaptive_time.cu:50-77
 * Writes max_sub_steps[m], time_step[m] and outer_time_step. */
int cmf_phase_cfl(CmfPlan* plan, void* stream, double outer_seconds);
/* Set time_step[m] = outer/n and max_sub_steps[m] = n for a fixed count. */
int cmf_phase_fixed_dt(CmfPlan* plan, void* stream, double outer_seconds,
                       int32_t n);
/* One kernel of sub-step k of the current interval (after cmf_phase_cfl or
 * cmf_phase_fixed_dt), launched directly on `stream` so a caller can time it
 * with events: part = CMF_PART_MOMENTUM, CMF_PART_LIMIT (the per-cell limit
 * rate), CMF_PART_STAGE, CMF_PART_LEVEE (the levee re-partition, a no-op
 * without levees) or CMF_PART_END (the interval epilogue, after the last
 * sub-step).  Running MOMENTUM, LIMIT, STAGE and LEVEE for k = 0..n-1 then
 * END is exactly cmf_step_interval without the graph. */
#define CMF_PART_MOMENTUM 1
#define CMF_PART_STAGE 2
#define CMF_PART_END 4
#define CMF_PART_LIMIT 8
#define CMF_PART_LEVEE 16
int cmf_launch_substep(CmfPlan* plan, void* stream, int32_t k, int part);
/* One sub-step (momentum, limit rate, stage) of a single-member view that
 * allocates nothing.  No counterpart in the reference.  It is for callers that
 * own all device memory and cannot call cudaMalloc -- code running inside a
 * stream capture, or a host whose memory pool hands out only the model
 * tensors -- so they cannot supply a workspace or create a plan.  The scratch
 * lives in a static device array of this library (3 MiB on every GPU that
 * loads it, held until exit), which limits the view to at most 65,536
 * catchments, 8,192 bifurcation paths and one member; larger views return
 * CMF_ERR_ARG.  view.workspace is ignored; view.time_step[0] must hold the
 * sub-step length.  diag != 0 writes the diagnostic fields as
 * cmf_phase_stage does.  `stream` must belong to the current device (a
 * stream of another device returns CMF_ERR_ARG): the call uses the current
 * device's copy of the array.  The first call on a device looks up the
 * array's device address (with that device current), so make it before any
 * stream capture.  Every call shares the one array: calls that overlap on the GPU
 * (two streams, two host threads) race and must be serialised by the caller. */
int cmf_substep_noalloc(const CmfView* view, void* stream, int diag);
/* Reduce the per-CTA budget partials into view.budget and clear them. */
int cmf_budget_flush(CmfPlan* plan, void* stream);

/* ---- output statistics accumulated on the device -------------------------
 * The reference's `variables_to_save` (scripts/run_daily_bin.py:28, e.g.
 * {"mean": ["total_outflow"], "last": ["river_depth"]}) aggregated by its
 * output layer outside the step.  Here the aggregation is one kernel appended
 * to the sub-step inside the interval graph, so a whole output period runs
 * without a device-to-host copy.  Conventions:
 *   MEAN  sum over sub-steps of value * dt, divided at finalize by the sum
 *         of dt of the member (a time average over the output period);
 *   MAX / MIN  over the values after every sub-step (NaN sticks);
 *   LAST  the value at finalize time.
 * Products and sums are rounded separately (no fused multiply-add), in the
 * order of the sub-steps, so a host replay with separate fp64 ops matches
 * bit for bit.  Accumulators are caller-owned fp64 arrays of N x M elements
 * in the state layout; `weight` is a caller-owned fp64 array of M elements. */
#define CMF_VAR_RIVER_OUTFLOW 0
#define CMF_VAR_FLOOD_OUTFLOW 1
#define CMF_VAR_TOTAL_OUTFLOW 2 /* river + flood outflow (base.py:412-419)  */
#define CMF_VAR_RIVER_DEPTH 3
#define CMF_VAR_FLOOD_DEPTH 4
#define CMF_VAR_FLOOD_FRACTION 5
#define CMF_VAR_PROTECTED_DEPTH 6
#define CMF_VAR_RIVER_STORAGE 7
#define CMF_VAR_FLOOD_STORAGE 8
#define CMF_VAR_PROTECTED_STORAGE 9
#define CMF_VAR_COUNT 10

#define CMF_STAT_MEAN 0
#define CMF_STAT_MAX 1
#define CMF_STAT_MIN 2
#define CMF_STAT_LAST 3

#define CMF_MAX_STATISTICS 16

typedef struct CmfStatistic {
    int32_t variable; /* CMF_VAR_*  */
    int32_t op;       /* CMF_STAT_* */
    double* out;      /* [N * M] device accumulator / result */
} CmfStatistic;

/* Attach `count` statistics to the plan (count == 0 detaches).  The interval
 * graph is rebuilt on the next cmf_step_interval.  Protected fields need the
 * levee module. */
int cmf_stats_attach(CmfPlan* plan, int count, const CmfStatistic* stats,
                     double* weight);
/* Start an output period: MEAN -> 0, MAX -> -inf, MIN -> +inf, weight -> 0. */
int cmf_stats_reset(CmfPlan* plan, void* stream);
/* Fold the sub-step that the per-phase entry points just finished (host step
 * index k, as in cmf_launch_substep) into the statistics. */
int cmf_stats_accumulate(CmfPlan* plan, void* stream, int32_t k);
/* End an output period: MEAN /= weight, LAST := the current value. */
int cmf_stats_finalize(CmfPlan* plan, void* stream);

/* ---- runoff forcing map: gridded runoff -> catchments --------------------
 * Replaces the forcing step before the routing path: hydroforge's
 * `dataset.build_local_mapping(mapping_file, desired_catchment_ids, device)`
 * and `dataset.shard_forcing(chunk, local_mapping)`
 * (scripts/run_daily_bin.py:98-118).  The mapping is the reference's runoff
 * mapping table (`.npz`: catchment_ids, sparse_data, sparse_indices,
 * sparse_indptr, matrix_shape; read in cmfgpu/params/export_bin.py:955-983)
 * restricted to the model's catchments, rows in model order, columns the
 * flattened runoff grid index iy * nx + ix (export_bin.py:1071-1075),
 * weights in m^2.  For every catchment row r, step t and member m:
 *   out[t, r, m] = (sum_k w_k * grid[t, m, col_k]) * (1 / unit_factor)
 * summed in entry order in fp64 with products and sums rounded separately;
 * the reciprocal of unit_factor is rounded once on the host.
 * CMF_FORCING_SKIP_MISSING leaves out entries whose grid value is NaN or
 * equals missing_value (compared in the grid's dtype);
 * CMF_FORCING_CLAMP_NEGATIVE sets negative sums to zero.  A column outside
 * [0, num_cols) is skipped and sets CMF_STATUS_BAD_INDEX in *status (when
 * status is not NULL). */
#define CMF_DTYPE_F32 0
#define CMF_DTYPE_F64 1
#define CMF_FORCING_SKIP_MISSING 1
#define CMF_FORCING_CLAMP_NEGATIVE 2
#define CMF_STATUS_BAD_INDEX 4

typedef struct CmfForcingMap {
    int64_t num_rows;       /* catchments (model order)                */
    int64_t num_cols;       /* runoff grid cells (ny * nx)             */
    const int64_t* row_ptr; /* [num_rows + 1] device                   */
    const int32_t* col;     /* [nnz] device                            */
    const double* weight;   /* [nnz] device, m^2                       */
} CmfForcingMap;

/* grid: element (t, m, c) at grid[t * grid_step_stride + m * grid_member_stride
 * + c]; out: element (t, r, m) at out[t * out_step_strides + m *
 * out_member_stride + r * out_row_stride] (strides in elements). */
int cmf_forcing_apply(const CmfForcingMap* map, void* stream, const void* grid,
                      int grid_dtype, int32_t steps, int32_t members,
                      int64_t grid_step_stride, int64_t grid_member_stride,
                      void* out, int out_dtype, int64_t out_step_stride,
                      int64_t out_member_stride, int64_t out_row_stride,
                      double unit_factor, double missing_value, int flags,
                      int* status);

/* ---- adjoint of the sub-step (no counterpart in the reference) -----------
 * Reverse mode of the routing sub-step in fp64, every physics module, for
 * gradients of a loss on discharge with respect to the Manning coefficients,
 * river height, river width, runoff and the initial state.  It differentiates
 * the forward of cmfgpu/phys/cuda/outflow.cu, reservoir.cu, bifurcation.cu,
 * storage.cu and levee.cu in the step order of
 * cmfgpu/models/cama_flood_model.py:134-162.
 *
 * Layout (N = catchments, P = bifurcation paths, L = levels; doubles):
 *   state   [12][N] river storage, flood storage, river outflow, flood
 *                   outflow, river depth, flood depth, river cross-section
 *                   depth, flood cross-section depth, flood cross-section
 *                   area, protected storage, protected depth, reservoir
 *                   total inflow; then [2][P*L] bifurcation outflow and
 *                   cross-section depth
 *   slot    a state's cell fields plus the sub-step's river/flood flux and
 *           limit rate ([15][N]), then the path state and the limited path
 *           fluxes ([3][P*L] + [2][P]), then the flood-stage result of the
 *           levee cells before their re-partition ([4][NLV]); its length
 *           comes from cmf_adj_sizes
 *   lambda  adjoint of a state (state layout)
 *   grad    [4][N] river Manning, flood Manning, river height, river width
 *   scratch reverse-sweep intermediates; zero it before a sweep
 *
 * The view must have CMF_FEAT_FP64 and one member (else
 * CMF_ERR_UNSUPPORTED).  The plan keeps the view's topology and parameter
 * pointers; the differentiated parameters are read through river_manning,
 * flood_manning, river_height and river_width.  cmf_adj_plan_create copies
 * the cell flags to the host once to list the dam cells (a small device
 * array owned by the plan); every other entry queues its work on `stream`
 * and allocates nothing. */
typedef struct CmfAdjPlan CmfAdjPlan;
int cmf_adj_plan_create(const CmfView* view, CmfAdjPlan** out);
void cmf_adj_plan_destroy(CmfAdjPlan* plan);
/* Lengths (doubles) of a state, a tape slot and the scratch, and the number
 * of gradient fields, for this plan. */
int cmf_adj_sizes(const CmfAdjPlan* plan, int64_t* state_len, int64_t* slot_len,
                  int64_t* scratch_len, int* grad_fields);
/* CFL sub-step count of the state in `slot` for one forcing interval
 * (adaptive_time.cu:19-48) into *n_device (a device int). */
int cmf_adj_sub_steps(CmfAdjPlan* plan, void* stream, const double* slot,
                      double outer_seconds, int* n_device);
/* num_sub_steps forward sub-steps of length dt with forcing `runoff` [N].
 * keep_tape != 0: slots[k] (k = 0..n, stride slot_len) receives X_k and the
 * sub-step's fluxes; the caller fills the state of slots[0].  keep_tape == 0:
 * two slots ping-pong and the final state is in slots[n & 1]. */
int cmf_adj_forward(CmfAdjPlan* plan, void* stream, double* slots,
                    int num_sub_steps, int keep_tape, const double* runoff,
                    double dt);
/* Reverse sweep over a tape written by cmf_adj_forward(keep_tape = 1) with the
 * same runoff and dt: lambda holds the adjoint of X_n on entry and of X_0 on
 * exit (except the pending river-depth terms, see cmf_adj_finalize); grad and
 * grad_runoff [N] are accumulated. */
int cmf_adj_reverse(CmfAdjPlan* plan, void* stream, const double* tape,
                    int num_sub_steps, const double* runoff, double dt,
                    double* lambda, double* grad_params, double* grad_runoff,
                    double* scratch);
/* Add the pending terms of the last reversed sub-step (downstream depth read
 * by momentum, end states read by the paths) to lambda and grad (river
 * height); call once after the sweep. */
int cmf_adj_finalize(CmfAdjPlan* plan, void* stream, double* lambda,
                     double* grad_params, double* scratch);

/* ---- host topology helpers (bit-exact with the reference preprocessing) -- */
/* cmfgpu/params/utils.py:83-138 */
int cmf_topo_topological_sort(int64_t n, const int64_t* catchment_id,
                              const int64_t* downstream_id, int32_t* order_out);
/* cmfgpu/params/utils.py:160-206 */
int cmf_topo_upstream_csr(int64_t n, const int32_t* dn, int32_t* indptr,
                          int32_t* indices);
/* basin-major breadth-first order from the mouths (no reference counterpart) */
int cmf_topo_bfs_order(int64_t n, const int32_t* dn, int32_t* order_out,
                       int32_t* up_ptr_out);
/* cmfgpu/params/utils.py:140-157 */
int cmf_topo_init_river_depth(int64_t n, const float* catchment_elevation,
                              const float* river_height, const int32_t* dn,
                              const int32_t* visit, float* river_depth);
int cmf_topo_accumulate_upstream(int64_t n, const int32_t* dn,
                                 const double* vals, double* out);
int cmf_topo_accumulate_downstream(int64_t n, const int32_t* dn,
                                   const double* vals, double* out);

#ifdef __cplusplus
}
#endif

#endif /* CMFB200_H */
