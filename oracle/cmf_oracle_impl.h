/*
 * CPU restatement of the reference CaMa-Flood-GPU sub-step -- TEST
 * INFRASTRUCTURE ONLY.  This file is the oracle: only tests/, the smoke check
 * and the CPU-baseline leg of bench.py may load it.  The product (libcmfb200)
 * never links or calls it.
 *
 * Included twice by cmf_oracle.c with REAL = float / double and ORC_SFX = the
 * symbol suffix.  STO (the reference "hpfloat") is always double.
 *
 * Each function restates one reference CUDA kernel, keeping its expression
 * order so that float rounding follows the reference:
 *   orc_outflow          cmfgpu/phys/cuda/outflow.cu:21-175
 *   orc_inflow           cmfgpu/phys/cuda/outflow.cu:180-222
 *   orc_flood_stage      cmfgpu/phys/cuda/storage.cu:22-226 (non-LOG path)
 *   orc_adaptive_time    cmfgpu/phys/cuda/adaptive_time.cu:19-48
 *   orc_bif_outflow      cmfgpu/phys/cuda/bifurcation.cu:21-129
 *   orc_bif_inflow       cmfgpu/phys/cuda/bifurcation.cu:131-156
 *   orc_reservoir        cmfgpu/phys/cuda/reservoir.cu:18-94
 *   orc_levee_stage      cmfgpu/phys/cuda/levee.cu:29-261 (non-LOG path)
 *   orc_levee_bif        cmfgpu/phys/cuda/levee.cu:263-341
 *   orc_substep          phase order of cmfgpu/models/cama_flood_model.py:134-162
 *   orc_step_advance     cmfgpu/models/cama_flood_model.py:104-173
 * Scatters are the reference's atomicAdd, done with `omp atomic` so that the
 * OpenMP build keeps the reference's race-free (but order-dependent) sums; run
 * with one thread for a deterministic checker.
 */

#define ORC_CAT2(a, b) a##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define ORC(name) ORC_CAT(name, ORC_SFX)
#define OrcModelT ORC(OrcModel)

#define R(x) ((REAL)(x))

typedef struct OrcModelT {
    int64_t n;            /* catchments */
    int64_t n_paths;      /* bifurcation paths */
    int64_t n_levees;
    int64_t n_res;
    int32_t n_flood_levels;
    int32_t n_bif_levels;
    int32_t has_bif, has_levee, has_res;
    int32_t has_total_storage, has_wse, has_pwse;
    double gravity, min_kinematic_slope, adaptive_time_factor;
    REAL time_step;        /* base.time_step[0] */
    REAL outer_time_step;  /* base.outer_time_step[0] */
    /* topology */
    const int32_t* downstream_idx;
    const uint8_t* is_levee;
    const uint8_t* is_reservoir;
    const uint8_t* is_dam_upstream;
    const uint8_t* is_dam_related;
    /* base params */
    const REAL *river_width, *river_length, *river_height, *catchment_elevation,
        *catchment_area, *downstream_distance, *river_manning, *flood_manning,
        *flood_depth_table, *runoff;
    /* base state */
    REAL *river_outflow, *flood_outflow, *river_depth, *flood_depth, *protected_depth,
        *river_cross_section_depth, *flood_cross_section_depth, *flood_cross_section_area,
        *flood_fraction;
    double *river_storage, *flood_storage, *protected_storage;
    /* scratch state */
    double *river_inflow, *flood_inflow, *outgoing_storage, *total_storage,
        *global_bifurcation_outflow;
    REAL *limit_rate, *water_surface_elevation, *protected_water_surface_elevation;
    /* bifurcation */
    const int32_t *bif_catchment_idx, *bif_downstream_idx;
    const REAL *bif_manning, *bif_width, *bif_length, *bif_elevation;
    REAL *bif_outflow, *bif_cross_section_depth;
    /* levee */
    const int32_t* levee_catchment_idx;
    const REAL *levee_crown_height, *levee_fraction, *levee_base_height;
    /* reservoir */
    const int32_t* reservoir_catchment_idx;
    const REAL *conservation_volume, *emergency_volume, *adjustment_volume,
        *effective_normal_outflow, *adjustment_outflow, *flood_control_outflow;
    double* reservoir_total_inflow;
} OrcModelT;

static inline REAL ORC(fmaxr)(REAL a, REAL b) { return sizeof(REAL) == 4 ? (REAL)fmaxf((float)a, (float)b) : (REAL)fmax((double)a, (double)b); }
static inline REAL ORC(fminr)(REAL a, REAL b) { return sizeof(REAL) == 4 ? (REAL)fminf((float)a, (float)b) : (REAL)fmin((double)a, (double)b); }
static inline REAL ORC(sqrtr)(REAL a) { return sizeof(REAL) == 4 ? (REAL)sqrtf((float)a) : (REAL)sqrt((double)a); }
static inline REAL ORC(cbrtr)(REAL a) { return sizeof(REAL) == 4 ? (REAL)cbrtf((float)a) : (REAL)cbrt((double)a); }
static inline REAL ORC(fabsr)(REAL a) { return a < 0 ? -a : a; }
static inline REAL ORC(expr_)(REAL a) { return sizeof(REAL) == 4 ? (REAL)expf((float)a) : (REAL)exp((double)a); }
static inline REAL ORC(logr)(REAL a) { return sizeof(REAL) == 4 ? (REAL)logf((float)a) : (REAL)log((double)a); }
static inline REAL ORC(floorr)(REAL a) { return sizeof(REAL) == 4 ? (REAL)floorf((float)a) : (REAL)floor((double)a); }
#define FMAX ORC(fmaxr)
#define FMIN ORC(fminr)
#define SQRT ORC(sqrtr)
#define CBRT ORC(cbrtr)
#define FABS ORC(fabsr)
#define EXP ORC(expr_)
#define LOG ORC(logr)
#define FLOOR ORC(floorr)

static inline void ORC(atomic_add)(double* p, double v)
{
#pragma omp atomic
    *p += v;
}
#define AADD ORC(atomic_add)

/* outflow.cu:21-175 (sea level and BASE_ONLY specialisation folded: the
 * reservoir block runs when has_res). */
void ORC(orc_outflow)(OrcModelT* m)
{
    const REAL gravity = R(m->gravity);
    const REAL time_step = m->time_step;
    const REAL min_kin = R(m->min_kinematic_slope);
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < m->n; ++t) {
        int dn = m->downstream_idx[t];
        int mouth = (dn == (int)t);
        REAL r_out = m->river_outflow[t];
        REAL r_man = m->river_manning[t];
        REAL r_dep = m->river_depth[t];
        REAL r_wid = m->river_width[t];
        REAL r_len = m->river_length[t];
        REAL r_hgt = m->river_height[t];
        REAL f_out = m->flood_outflow[t];
        REAL f_man = m->flood_manning[t];
        REAL f_dep = m->flood_depth[t];
        REAL p_dep = m->protected_depth[t];
        REAL c_elv = m->catchment_elevation[t];
        REAL dn_dist = m->downstream_distance[t];
        REAL r_cs_dep = m->river_cross_section_depth[t];
        REAL f_cs_dep = m->flood_cross_section_depth[t];
        REAL f_cs_area = m->flood_cross_section_area[t];
        REAL rs = (REAL)m->river_storage[t];
        REAL fs = (REAL)m->flood_storage[t];
        REAL ps = (REAL)m->protected_storage[t];

        REAL river_elevation = c_elv - r_hgt;
        REAL wse = r_dep + river_elevation;
        REAL pwse = (m->has_levee && m->is_levee[t]) ? FMIN(c_elv + p_dep, wse) : wse;
        REAL total_storage_f = rs + fs + ps;

        REAL r_dep_dn = m->river_depth[dn];
        REAL r_hgt_dn = m->river_height[dn];
        REAL c_elv_dn = m->catchment_elevation[dn];
        REAL river_elevation_dn = c_elv_dn - r_hgt_dn;
        REAL wse_dn = r_dep_dn + river_elevation_dn;
        if (mouth) wse_dn = c_elv;
        REAL max_wse = FMAX(wse, wse_dn);

        REAL river_slope = (wse - wse_dn) / dn_dist;
        REAL flood_slope = FMIN(FMAX(river_slope, R(-0.005)), R(0.005));

        REAL upd_r_cs_dep = mouth ? r_dep : max_wse - river_elevation;
        REAL r_sifd = FMAX(SQRT(upd_r_cs_dep * r_cs_dep), R(1e-6));
        REAL flood_surface = mouth ? wse : max_wse;
        REAL upd_f_cs_dep = FMAX(flood_surface - c_elv, R(0.0));
        REAL f_sifd = FMAX(SQRT(upd_f_cs_dep * f_cs_dep), R(1e-6));
        REAL upd_f_cs_area = FMAX(fs / r_len - f_dep * r_wid, R(0.0));

        REAL r_cs_area = upd_r_cs_dep * r_wid;
        int river_condition = (r_sifd > R(1e-5)) && (r_cs_area > R(1e-5));
        REAL unit_r_out = r_out / r_wid;
        REAL num_r = r_wid * (unit_r_out + gravity * time_step * r_sifd * river_slope);
        REAL den_r = R(1.0) + gravity * time_step * (r_man * r_man) * FABS(unit_r_out)
                     * (R(1.0) / (r_sifd * r_sifd * CBRT(r_sifd)));
        REAL upd_r_out = num_r / den_r;
        upd_r_out = river_condition ? upd_r_out : R(0.0);

        int flood_condition = (f_sifd > R(1e-5)) && (upd_f_cs_area > R(1e-5));
        REAL upd_f_out = R(0.0);
        if (flood_condition) {
            REAL f_imp_area = FMAX(SQRT(upd_f_cs_area * FMAX(f_cs_area, R(1e-6))), R(1e-6));
            REAL num_f = f_out + gravity * time_step * f_imp_area * flood_slope;
            REAL den_f = R(1.0) + gravity * time_step * (f_man * f_man) * FABS(f_out)
                         * (R(1.0) / (f_sifd * CBRT(f_sifd))) / f_imp_area;
            upd_f_out = num_f / den_f;
        }

        int opposite = (upd_r_out * upd_f_out) < R(0.0);
        if (opposite) upd_f_out = R(0.0);
        int negative = (upd_r_out < R(0.0)) && !mouth;
        REAL total_negative_flow = negative ? (-upd_r_out - upd_f_out) * time_step : R(1.0);
        REAL limit_rate = FMIN(negative ? R(0.05) * total_storage_f / total_negative_flow : R(1.0), R(1.0));
        if (negative) { upd_r_out *= limit_rate; upd_f_out *= limit_rate; }

        if (m->has_res) {
            int is_dam_up = m->is_dam_upstream && m->is_dam_upstream[t];
            REAL bed_slope = (c_elv - c_elv_dn) / dn_dist;
            bed_slope = FMAX(bed_slope, min_kin);
            REAL kin_riv_vel = (R(1.0) / r_man) * SQRT(bed_slope) * CBRT(r_dep * r_dep);
            REAL kin_riv = r_wid * r_dep * kin_riv_vel;
            kin_riv = FMIN(kin_riv, rs / time_step);
            kin_riv = FMAX(kin_riv, R(0.0));
            REAL bed_slope_f = FMIN(bed_slope, R(0.005));
            REAL kin_fld_vel = (R(1.0) / f_man) * SQRT(bed_slope_f) * CBRT(f_dep * f_dep);
            REAL kin_fld_area = FMAX(fs / r_len - f_dep * r_wid, R(0.0));
            REAL kin_fld = kin_fld_area * kin_fld_vel;
            kin_fld = FMIN(kin_fld, fs / time_step);
            kin_fld = FMAX(kin_fld, R(0.0));
            if (is_dam_up) { upd_r_out = kin_riv; upd_f_out = kin_fld; }
        }

        m->river_outflow[t] = upd_r_out;
        m->flood_outflow[t] = upd_f_out;
        if (m->has_wse) m->water_surface_elevation[t] = wse;
        if (m->has_pwse) m->protected_water_surface_elevation[t] = pwse;
        m->river_cross_section_depth[t] = upd_r_cs_dep;
        m->flood_cross_section_depth[t] = upd_f_cs_dep;
        m->flood_cross_section_area[t] = upd_f_cs_area;
        if (m->has_total_storage) m->total_storage[t] = (double)total_storage_f;
        m->river_inflow[t] = 0.0;
        m->flood_inflow[t] = 0.0;
        if (m->has_bif) m->global_bifurcation_outflow[t] = 0.0;

        REAL pos = FMAX(upd_r_out, R(0.0)) + FMAX(upd_f_out, R(0.0));
        REAL neg = FMIN(upd_r_out, R(0.0)) + FMIN(upd_f_out, R(0.0));
        AADD(m->outgoing_storage + t, (double)(pos * time_step));
        REAL to_add = mouth ? R(0.0) : -neg * time_step;
        AADD(m->outgoing_storage + dn, (double)to_add);
    }
}

/* outflow.cu:180-222 */
void ORC(orc_inflow)(OrcModelT* m)
{
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < m->n; ++t) {
        REAL r_out = m->river_outflow[t];
        REAL f_out = m->flood_outflow[t];
        REAL outgoing = (REAL)m->outgoing_storage[t];
        REAL rate_storage = (REAL)(m->river_storage[t] + m->flood_storage[t]);
        REAL limit_rate = (outgoing > R(1e-8)) ? FMIN(rate_storage / outgoing, R(1.0)) : R(1.0);
        int dn = m->downstream_idx[t];
        REAL outgoing_dn = (REAL)m->outgoing_storage[dn];
        REAL rate_storage_dn = (REAL)(m->river_storage[dn] + m->flood_storage[dn]);
        REAL limit_rate_dn = (outgoing_dn > R(1e-8)) ? FMIN(rate_storage_dn / outgoing_dn, R(1.0)) : R(1.0);
        REAL upd_r_out = (r_out >= R(0.0)) ? r_out * limit_rate : r_out * limit_rate_dn;
        REAL upd_f_out = (f_out >= R(0.0)) ? f_out * limit_rate : f_out * limit_rate_dn;
        m->river_outflow[t] = upd_r_out;
        m->flood_outflow[t] = upd_f_out;
        if (m->has_bif) m->limit_rate[t] = limit_rate;
        if (dn != (int)t) {
            AADD(m->river_inflow + dn, (double)upd_r_out);
            AADD(m->flood_inflow + dn, (double)upd_f_out);
            if (m->has_res && m->is_reservoir && m->is_reservoir[dn])
                AADD(m->reservoir_total_inflow + dn, (double)(upd_r_out + upd_f_out));
        }
    }
}

/* storage.cu:22-226 with LOG=false (the fp64 budget is checked separately). */
void ORC(orc_flood_stage)(OrcModelT* m)
{
    const int nl = m->n_flood_levels;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < m->n; ++t) {
        REAL ts = m->time_step;
        double rsto = m->river_storage[t];
        double fsto = m->flood_storage[t];
        double prot = m->protected_storage[t];
        REAL rinf = (REAL)m->river_inflow[t];
        REAL finf = (REAL)m->flood_inflow[t];
        REAL gbif = m->has_bif ? (REAL)m->global_bifurcation_outflow[t] : R(0);
        REAL rout = m->river_outflow[t];
        REAL fout = m->flood_outflow[t];
        REAL ro = m->runoff[t];
        REAL prescribed_inflow = R(0);

        REAL river_delta = (rinf - rout) * ts;
        double river_su = rsto + (double)river_delta;
        REAL flood_delta = (finf - fout - gbif) * ts;
        double flood_su = fsto + (river_su < 0.0 ? river_su : 0.0) + (double)flood_delta;
        river_su = river_su > 0.0 ? river_su : 0.0;
        if (flood_su < 0.0) {
            double tt = river_su + flood_su;
            river_su = tt > 0.0 ? tt : 0.0;
        }
        flood_su = flood_su > 0.0 ? flood_su : 0.0;
        REAL external_delta = (ro + prescribed_inflow) * ts;
        double total_next = river_su + flood_su + prot + (double)external_delta;
        double total_s = total_next > 0.0 ? total_next : 0.0;
        REAL total_storage = (REAL)total_s;

        REAL rh = m->river_height[t];
        REAL rw = m->river_width[t];
        REAL rl = m->river_length[t];
        REAL river_max_storage = rl * rw * rh;

        if (total_storage <= river_max_storage) {
            REAL river_depth_dry = total_storage / (rl * rw);
            m->outgoing_storage[t] = 0.0;
            m->river_storage[t] = total_s;
            m->flood_storage[t] = 0.0;
            m->protected_storage[t] = 0.0;
            m->river_depth[t] = river_depth_dry;
            m->flood_depth[t] = R(0);
            m->protected_depth[t] = R(0);
            m->flood_fraction[t] = R(0);
            continue;
        }
        REAL ca = m->catchment_area[t];
        REAL catchment_width = ca / rl;
        REAL width_increment = catchment_width / (REAL)nl;
        int level = 0;
        REAL S_accum = river_max_storage;
        REAL prev_H = R(0);
        REAL prev_W = rw;
        REAL prev_total_storage = river_max_storage;
        REAL prev_flood_depth = R(0);
        REAL next_flood_depth = R(0);
        for (int i = 0; i < nl; ++i) {
            REAL H_curr = m->flood_depth_table[t * nl + i];
            REAL W_curr = rw + (REAL)(i + 1) * width_increment;
            REAL dS = rl * R(0.5) * (prev_W + W_curr) * (H_curr - prev_H);
            REAL S_curr = S_accum + dS;
            next_flood_depth = H_curr;
            if (total_storage > S_curr) {
                level += 1;
                prev_total_storage = S_curr;
                prev_flood_depth = H_curr;
                S_accum = S_curr;
                prev_H = H_curr;
                prev_W = W_curr;
            } else {
                break;
            }
        }
        REAL prev_total_width = rw + (REAL)level * width_increment;
        REAL diff_width = R(0);
        REAL fdep;
        if (level == nl) {
            fdep = prev_flood_depth + (total_storage - prev_total_storage) / (prev_total_width * rl);
        } else {
            REAL flood_grad = (next_flood_depth - prev_flood_depth) / width_increment;
            diff_width = SQRT(prev_total_width * prev_total_width
                              + R(2) * (total_storage - prev_total_storage) / (flood_grad * rl))
                         - prev_total_width;
            fdep = prev_flood_depth + diff_width * flood_grad;
        }
        REAL cap = river_max_storage + rl * rw * fdep;
        double cap_s = (double)cap;
        double river_storage_final = cap_s < total_s ? cap_s : total_s;
        REAL rdep = (REAL)river_storage_final / (rl * rw);
        REAL ff_mid = (prev_total_width + diff_width - rw) * rl / ca;
        ff_mid = ff_mid < R(0) ? R(0) : (ff_mid > R(1) ? R(1) : ff_mid);
        REAL ffr = (level == nl) ? R(1) : ff_mid;
        double flood_storage_final = total_s - river_storage_final;
        if (flood_storage_final < 0.0) flood_storage_final = 0.0;

        m->outgoing_storage[t] = 0.0;
        m->river_storage[t] = river_storage_final;
        m->flood_storage[t] = flood_storage_final;
        m->protected_storage[t] = 0.0;
        m->river_depth[t] = rdep;
        m->flood_depth[t] = fdep;
        m->protected_depth[t] = fdep;
        m->flood_fraction[t] = ffr;
    }
}

/* adaptive_time.cu:19-48, the block/atomic max folded into a serial max.
 * max_dt > 0 adds the optional dt cap (not in the reference). */
int ORC(orc_adaptive_time)(const OrcModelT* m, double max_dt)
{
    int result = 0;
    const REAL factor = R(m->adaptive_time_factor);
    const REAL gravity = R(m->gravity);
#pragma omp parallel for schedule(static) reduction(max : result)
    for (int64_t t = 0; t < m->n; ++t) {
        int n_steps = 1;
        int skip = m->has_res && m->is_dam_related && m->is_dam_related[t];
        if (!skip) {
            REAL dist = m->downstream_distance[t];
            REAL raw_depth = m->river_depth[t];
            REAL depth = FMAX(raw_depth, R(0.01));
            REAL dt = factor * dist / SQRT(gravity * depth);
            if (max_dt > 0) dt = FMIN(dt, R(max_dt));
            REAL outer_dt = m->outer_time_step;
            REAL dt_clamped = FMIN(dt, outer_dt);
            n_steps = (int)(FLOOR(outer_dt / dt_clamped - R(0.01)) + R(1.0));
        }
        if (n_steps > result) result = n_steps;
    }
    return result > 0 ? result : 0;
}

static inline REAL ORC(pow73)(REAL x) { return x * x * CBRT(x); }

/* bifurcation.cu:21-129 (generic level loop; the register fast path of the
 * reference computes the same values). */
void ORC(orc_bif_outflow)(OrcModelT* m)
{
    const REAL gravity = R(m->gravity);
    const REAL time_step = m->time_step;
    const int L = m->n_bif_levels;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < m->n_paths; ++t) {
        int ci = m->bif_catchment_idx[t];
        int di = m->bif_downstream_idx[t];
        REAL blen = m->bif_length[t];
        REAL wse_c = m->water_surface_elevation[ci];
        REAL wse_d = m->water_surface_elevation[di];
        REAL max_wse = FMAX(wse_c, wse_d);
        REAL slope = (wse_c - wse_d) / blen;
        slope = FMIN(FMAX(slope, R(-0.005)), R(0.005));
        REAL ts_c = (REAL)m->total_storage[ci];
        REAL ts_d = (REAL)m->total_storage[di];
        REAL sum_out = R(0);
        for (int lv = 0; lv < L; ++lv) {
            int64_t li = t * L + lv;
            REAL man = m->bif_manning[li];
            REAL csd = m->bif_cross_section_depth[li];
            REAL elv = m->bif_elevation[li];
            REAL upd_csd = FMAX(max_wse - elv, R(0));
            REAL sifd = FMAX(SQRT(upd_csd * csd), SQRT(upd_csd * R(0.01)));
            REAL upd_o = R(0);
            if (sifd > R(1e-5)) {
                REAL w = m->bif_width[li];
                REAL o = m->bif_outflow[li];
                REAL unit_o = o / w;
                REAL num = w * (unit_o + gravity * time_step * sifd * slope);
                REAL den = R(1) + gravity * time_step * (man * man) * FABS(unit_o)
                           * (R(1) / ORC(pow73)(sifd));
                upd_o = num / den;
            }
            sum_out += upd_o;
            m->bif_cross_section_depth[li] = upd_csd;
            m->bif_outflow[li] = upd_o;
        }
        REAL limit_rate = FMIN(R(0.05) * FMIN(ts_c, ts_d) / (FABS(sum_out) * time_step), R(1));
        sum_out *= limit_rate;
        for (int lv = 0; lv < L; ++lv) {
            int64_t li = t * L + lv;
            m->bif_outflow[li] = m->bif_outflow[li] * limit_rate;
        }
        REAL pos = FMAX(sum_out, R(0));
        REAL neg = FMIN(sum_out, R(0));
        AADD(m->outgoing_storage + ci, (double)(pos * time_step));
        AADD(m->outgoing_storage + di, (double)(-neg * time_step));
    }
}

/* levee.cu:263-341 */
void ORC(orc_levee_bif)(OrcModelT* m)
{
    const REAL gravity = R(m->gravity);
    const REAL time_step = m->time_step;
    const int L = m->n_bif_levels;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < m->n_paths; ++t) {
        int ci = m->bif_catchment_idx[t];
        int di = m->bif_downstream_idx[t];
        REAL blen = m->bif_length[t];
        REAL wse_c = m->water_surface_elevation[ci];
        REAL wse_d = m->water_surface_elevation[di];
        REAL max_wse = FMAX(wse_c, wse_d);
        REAL pwse_c = m->protected_water_surface_elevation[ci];
        REAL pwse_d = m->protected_water_surface_elevation[di];
        REAL max_pwse = FMAX(pwse_c, pwse_d);
        REAL slope = (wse_c - wse_d) / blen;
        slope = FMIN(FMAX(slope, R(-0.005)), R(0.005));
        REAL ts_c = (REAL)m->total_storage[ci];
        REAL ts_d = (REAL)m->total_storage[di];
        REAL sum_out = R(0);
        for (int lv = 0; lv < L; ++lv) {
            int64_t li = t * L + lv;
            REAL current_max_wse = (lv == 0) ? max_wse : max_pwse;
            REAL elv = m->bif_elevation[li];
            REAL upd_csd = FMAX(current_max_wse - elv, R(0));
            REAL semi_depth;
            if (lv == 0) {
                REAL old_csd = m->bif_cross_section_depth[li];
                semi_depth = SQRT(upd_csd * old_csd);
                if (semi_depth <= R(0)) semi_depth = upd_csd;
            } else {
                semi_depth = upd_csd;
            }
            REAL upd_out = R(0);
            if (semi_depth > R(1e-5)) {
                REAL man = m->bif_manning[li];
                REAL w = m->bif_width[li];
                REAL o = m->bif_outflow[li];
                REAL unit_o = o / w;
                REAL num = w * (unit_o + gravity * time_step * semi_depth * slope);
                REAL den = R(1) + gravity * time_step * (man * man) * FABS(unit_o)
                           * (R(1) / ORC(pow73)(semi_depth));
                upd_out = num / den;
            }
            sum_out += upd_out;
            m->bif_cross_section_depth[li] = upd_csd;
            m->bif_outflow[li] = upd_out;
        }
        REAL limit_rate = FMIN(R(0.05) * FMIN(ts_c, ts_d) / (FABS(sum_out) * time_step), R(1));
        sum_out *= limit_rate;
        for (int lv = 0; lv < L; ++lv) {
            int64_t li = t * L + lv;
            m->bif_outflow[li] = m->bif_outflow[li] * limit_rate;
        }
        REAL pos = FMAX(sum_out, R(0));
        REAL neg = FMIN(sum_out, R(0));
        AADD(m->outgoing_storage + ci, (double)(pos * time_step));
        AADD(m->outgoing_storage + di, (double)(-neg * time_step));
    }
}

/* bifurcation.cu:131-156 */
void ORC(orc_bif_inflow)(OrcModelT* m)
{
    const int L = m->n_bif_levels;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < m->n_paths; ++t) {
        int ci = m->bif_catchment_idx[t];
        int di = m->bif_downstream_idx[t];
        REAL lr_c = m->limit_rate[ci];
        REAL lr_d = m->limit_rate[di];
        REAL raw_sum = R(0);
        for (int lv = 0; lv < L; ++lv) {
            int64_t li = t * L + lv;
            REAL o = m->bif_outflow[li];
            raw_sum += o;
            m->bif_outflow[li] = (o >= R(0)) ? o * lr_c : o * lr_d;
        }
        REAL net = (raw_sum >= R(0)) ? raw_sum * lr_c : raw_sum * lr_d;
        AADD(m->global_bifurcation_outflow + ci, (double)net);
        AADD(m->global_bifurcation_outflow + di, (double)(-net));
    }
}

/* reservoir.cu:18-94 */
void ORC(orc_reservoir)(OrcModelT* m)
{
    const REAL time_step = m->time_step;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < m->n_res; ++t) {
        int ci = m->reservoir_catchment_idx[t];
        int di = m->downstream_idx[ci];
        int mouth = (di == ci);
        REAL old_r = m->river_outflow[ci];
        REAL old_f = m->flood_outflow[ci];
        REAL old_pos = FMAX(old_r, R(0)) + FMAX(old_f, R(0));
        REAL old_neg = FMIN(old_r, R(0)) + FMIN(old_f, R(0));
        AADD(m->outgoing_storage + ci, (double)(-(old_pos * time_step)));
        double undo_dn = mouth ? 0.0 : (double)(old_neg * time_step);
        AADD(m->outgoing_storage + di, undo_dn);

        REAL rs = (REAL)m->river_storage[ci];
        REAL fs = (REAL)m->flood_storage[ci];
        REAL total = rs + fs;
        REAL total_inflow = (REAL)m->reservoir_total_inflow[ci];
        m->reservoir_total_inflow[ci] = 0.0;
        REAL runoff_v = m->runoff[ci];
        REAL inflow = total_inflow + runoff_v;
        REAL cons = m->conservation_volume[t];
        REAL emerg = m->emergency_volume[t];
        REAL adj = m->adjustment_volume[t];
        REAL n_out = m->effective_normal_outflow[t];
        REAL a_out = m->adjustment_outflow[t];
        REAL fc_out = m->flood_control_outflow[t];
        REAL ro;
        if (total <= cons) {
            ro = n_out * SQRT(total / cons);
        } else if (total <= adj) {
            REAL frac2 = (total - cons) / (adj - cons);
            ro = n_out + EXP(R(3.0) * LOG(frac2)) * (a_out - n_out);
        } else if (total <= emerg) {
            REAL frac3 = (total - adj) / (emerg - adj);
            REAL tmp = a_out + EXP(R(0.1) * LOG(frac3)) * (fc_out - a_out);
            if (inflow >= fc_out) {
                REAL flood = n_out + ((total - cons) / (emerg - cons)) * (inflow - n_out);
                ro = FMAX(flood, tmp);
            } else {
                ro = tmp;
            }
        } else {
            ro = (inflow >= fc_out) ? inflow : fc_out;
        }
        ro = FMAX(ro, R(0));
        ro = FMIN(ro, total / time_step);
        m->river_outflow[ci] = ro;
        m->flood_outflow[ci] = R(0);
        m->total_storage[ci] = (double)total;
        REAL new_pos = FMAX(ro, R(0));
        AADD(m->outgoing_storage + ci, (double)(new_pos * time_step));
        REAL new_neg = FMIN(ro, R(0));
        double to_add = mouth ? 0.0 : (double)(-(new_neg * time_step));
        AADD(m->outgoing_storage + di, to_add);
    }
}

static inline REAL ORC(clamp01)(REAL x) { return FMIN(FMAX(x, R(0)), R(1)); }

/* levee.cu:29-261 with LOG=false */
void ORC(orc_levee_stage)(OrcModelT* m)
{
    const int nl = m->n_flood_levels;
#pragma omp parallel for schedule(static)
    for (int64_t li = 0; li < m->n_levees; ++li) {
        int ci = m->levee_catchment_idx[li];
        REAL rl = m->river_length[ci];
        REAL rw = m->river_width[ci];
        REAL rh = m->river_height[ci];
        REAL ca = m->catchment_area[ci];
        REAL l_crown = m->levee_crown_height[li];
        REAL l_frac = m->levee_fraction[li];
        REAL l_base_h = m->levee_base_height[li];
        double riv_sto_curr_hp = m->river_storage[ci];
        double fld_sto_curr_hp = m->flood_storage[ci];
        double total_sto_hp = riv_sto_curr_hp + fld_sto_curr_hp;
        REAL riv_sto_curr = (REAL)riv_sto_curr_hp;
        REAL fld_sto_curr = (REAL)fld_sto_curr_hp;
        REAL fld_depth_curr = m->flood_depth[ci];
        REAL total_sto = (REAL)total_sto_hp;
        REAL riv_max_sto = rl * rw * rh;
        if (!(total_sto >= riv_max_sto)) {
            m->river_storage[ci] = riv_sto_curr_hp;
            m->flood_storage[ci] = fld_sto_curr_hp;
            m->protected_storage[ci] = 0.0;
            m->protected_depth[ci] = R(0);
            continue;
        }
        REAL dwth_inc = (ca / rl) / (REAL)nl;
        REAL levee_dist = l_frac * (ca / rl);
        REAL s_curr = riv_max_sto;
        REAL dhgt_pre = R(0);
        REAL dwth_pre = rw;
        REAL levee_base_sto = riv_max_sto;
        REAL levee_fill_sto = riv_max_sto;
        int found_base = 0, found_fill = 0;
        int ilev = (int)(l_frac * (REAL)nl);
        REAL dsto_fil_B = R(0), dwth_fil_B = R(0), ddph_fil_B = R(0), gradient_B = R(0);
        int found_B = 0;
        int scan_needed = 1;
        for (int i = 0; i < nl; ++i) {
            if (!scan_needed) break;
            REAL depth_val = m->flood_depth_table[(int64_t)ci * nl + i];
            REAL dhgt_seg = FMAX(depth_val - dhgt_pre, R(1e-6));
            REAL dwth_mid = dwth_pre + R(0.5) * dwth_inc;
            REAL dsto_seg = rl * dwth_mid * dhgt_seg;
            REAL s_next = s_curr + dsto_seg;
            REAL gradient = dhgt_seg / dwth_inc;

            int cond_base = (l_base_h > dhgt_pre) && (l_base_h <= depth_val);
            REAL ratio_base = (l_base_h - dhgt_pre) / dhgt_seg;
            REAL dsto_base_p = rl * (dwth_pre + R(0.5) * ratio_base * dwth_inc) * (ratio_base * dhgt_seg);
            if (cond_base && !found_base) levee_base_sto = s_curr + dsto_base_p;
            found_base = found_base || cond_base;

            int cond_fill = (l_crown > dhgt_pre) && (l_crown <= depth_val);
            REAL ratio_fill = (l_crown - dhgt_pre) / dhgt_seg;
            REAL dsto_fill_p = rl * (dwth_pre + R(0.5) * ratio_fill * dwth_inc) * (ratio_fill * dhgt_seg);
            if (cond_fill && !found_fill) levee_fill_sto = s_curr + dsto_fill_p;
            found_fill = found_fill || cond_fill;

            REAL dhgt_dif_loop = l_crown - l_base_h;
            REAL s_top_loop = levee_base_sto + (levee_dist + rw) * dhgt_dif_loop * rl;
            REAL dsto_add_wedge = (levee_dist + rw) * (l_crown - depth_val) * rl;
            REAL threshold = s_next + dsto_add_wedge;

            int cond_check = (i >= ilev) && !found_B;
            int cond_found = cond_check && (total_sto < threshold);
            REAL current_lb = (i == ilev) ? s_top_loop : dsto_fil_B;
            if (cond_check && !cond_found) {
                dsto_fil_B = threshold;
                dwth_fil_B = dwth_inc * (REAL)(i + 1) - levee_dist;
                ddph_fil_B = depth_val - l_base_h;
            } else {
                dsto_fil_B = current_lb;
            }
            if (cond_found) gradient_B = gradient;
            found_B = found_B || cond_found;

            s_curr = s_next;
            dhgt_pre = depth_val;
            dwth_pre += dwth_inc;
            scan_needed = !(found_base && found_fill && found_B);
        }
        REAL s_base_extra = s_curr + rl * dwth_pre * (l_base_h - dhgt_pre);
        if (!found_base) levee_base_sto = (l_base_h > dhgt_pre) ? s_base_extra : riv_max_sto;
        REAL s_fill_extra = s_curr + rl * dwth_pre * (l_crown - dhgt_pre);
        if (!found_fill) levee_fill_sto = (l_crown > dhgt_pre) ? s_fill_extra : riv_max_sto;

        REAL dhgt_dif = l_crown - l_base_h;
        REAL s_top = levee_base_sto + (levee_dist + rw) * dhgt_dif * rl;
        int is_case4 = total_sto >= levee_fill_sto;
        int is_case3 = (!is_case4) && (total_sto >= s_top);
        int is_case2 = (!is_case4) && (!is_case3) && (total_sto >= levee_base_sto);

        REAL dsto_add_c2 = total_sto - levee_base_sto;
        REAL dwth_add_c2 = levee_dist + rw;
        REAL f_dph_c2 = l_base_h + dsto_add_c2 / dwth_add_c2 / rl;
        REAL r_sto_c2 = riv_max_sto + rl * rw * f_dph_c2;
        REAL r_dph_c2 = r_sto_c2 / rl / rw;
        REAL f_sto_c2 = FMAX(total_sto - r_sto_c2, R(0));
        REAL f_frc_c2 = l_frac;

        REAL dsto_add_B = total_sto - dsto_fil_B;
        REAL term_B = dwth_fil_B * dwth_fil_B + R(2.0) * dsto_add_B / rl / (gradient_B + R(1e-9));
        REAL dwth_add_B = -dwth_fil_B + SQRT(FMAX(term_B, R(0)));
        REAL ddph_add_B = dwth_add_B * gradient_B;
        REAL p_dph_B_found = l_base_h + ddph_fil_B + ddph_add_B;
        REAL f_frc_B_found = (dwth_fil_B + levee_dist) / (dwth_inc * (REAL)nl);
        REAL ddph_add_B_extra = dsto_add_B / (dwth_fil_B * rl + R(1e-9));
        REAL p_dph_B_extra = l_base_h + ddph_fil_B + ddph_add_B_extra;
        REAL p_dph_B = found_B ? p_dph_B_found : p_dph_B_extra;
        REAL f_frc_B = found_B ? f_frc_B_found : R(1.0);

        REAL f_dph_c3 = l_crown;
        REAL r_sto_c3 = riv_max_sto + rl * rw * f_dph_c3;
        REAL r_dph_c3 = r_sto_c3 / rl / rw;
        REAL f_sto_c3 = FMAX(s_top - r_sto_c3, R(0));
        REAL p_dph_c3 = p_dph_B;
        REAL f_frc_c3 = ORC(clamp01)(f_frc_B);

        REAL f_dph_c4 = fld_depth_curr;
        REAL r_sto_c4 = riv_sto_curr;
        REAL dsto_add_c4 = (f_dph_c4 - l_crown) * (levee_dist + rw) * rl;
        REAL f_sto_c4 = FMAX(s_top + dsto_add_c4 - r_sto_c4, R(0));
        REAL p_dph_c4 = f_dph_c4;

        REAL r_dph_curr = m->river_depth[ci];
        REAL f_frc_curr = m->flood_fraction[ci];

        REAL r_sto_candidate = is_case2 ? r_sto_c2 : (is_case3 ? r_sto_c3 : (is_case4 ? r_sto_c4 : riv_sto_curr));
        REAL f_sto_candidate = is_case2 ? f_sto_c2 : (is_case3 ? f_sto_c3 : (is_case4 ? f_sto_c4 : fld_sto_curr));
        int no_levee_partition = !is_case2 && !is_case3 && !is_case4;
        double r_sto;
        if (is_case4 || no_levee_partition) {
            r_sto = riv_sto_curr_hp;
        } else {
            double c = (double)r_sto_candidate;
            r_sto = fmin(c, total_sto_hp);
        }
        double remaining_sto = total_sto_hp - r_sto;
        remaining_sto = remaining_sto > 0.0 ? remaining_sto : 0.0;
        double f_sto_candidate_hp = (double)f_sto_candidate;
        double f_sto = fmin(f_sto_candidate_hp > 0.0 ? f_sto_candidate_hp : 0.0, remaining_sto);
        if (is_case2) f_sto = remaining_sto;
        if (no_levee_partition) f_sto = fld_sto_curr_hp;
        double p_sto = remaining_sto - f_sto;
        p_sto = p_sto > 0.0 ? p_sto : 0.0;
        REAL r_dph = is_case2 ? r_dph_c2 : (is_case3 ? r_dph_c3 : r_dph_curr);
        REAL f_dph = is_case2 ? f_dph_c2 : (is_case3 ? f_dph_c3 : fld_depth_curr);
        REAL p_dph = is_case2 ? R(0) : (is_case3 ? p_dph_c3 : (is_case4 ? p_dph_c4 : R(0)));
        REAL f_frc = is_case2 ? f_frc_c2 : (is_case3 ? f_frc_c3 : f_frc_curr);

        m->river_storage[ci] = r_sto;
        m->flood_storage[ci] = f_sto;
        m->protected_storage[ci] = p_sto;
        m->river_depth[ci] = r_dph;
        m->flood_depth[ci] = f_dph;
        m->protected_depth[ci] = p_dph;
        m->flood_fraction[ci] = f_frc;
    }
}

/* One sub-step in the reference phase order, cama_flood_model.py:134-162. */
void ORC(orc_substep)(OrcModelT* m)
{
    ORC(orc_outflow)(m);
    if (m->has_res) ORC(orc_reservoir)(m);
    if (m->has_bif) {
        if (m->has_levee) ORC(orc_levee_bif)(m);
        else ORC(orc_bif_outflow)(m);
    }
    ORC(orc_inflow)(m);
    if (m->has_bif) ORC(orc_bif_inflow)(m);
    ORC(orc_flood_stage)(m);
    if (m->has_levee) ORC(orc_levee_stage)(m);
}

/* One forcing interval, cama_flood_model.py:104-173.  adaptive != 0 runs the
 * CFL count (optionally capped at max_dt seconds per sub-step), otherwise
 * fixed_n sub-steps.  dt is the fp32/fp64 rounding of the double quotient
 * outer/n, as base.time_step.fill_() stores it.  Returns the sub-step count. */
int ORC(orc_step_advance)(OrcModelT* m, double outer_seconds, int adaptive,
                          int fixed_n, double max_dt)
{
    m->outer_time_step = (REAL)outer_seconds;
    int n = fixed_n;
    if (adaptive) n = ORC(orc_adaptive_time)(m, max_dt);
    if (n < 1) n = 1;
    m->time_step = (REAL)(outer_seconds / (double)n);
    for (int k = 0; k < n; ++k) ORC(orc_substep)(m);
    return n;
}

#undef FMAX
#undef FMIN
#undef SQRT
#undef CBRT
#undef FABS
#undef EXP
#undef LOG
#undef FLOOR
#undef AADD
#undef R
#undef OrcModelT
