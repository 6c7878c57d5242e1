// Device kernels of the B200 routing core.
//
// One sub-step of CaMa-Flood routing is four HBM-bound kernels:
//
//   k_momentum  per catchment (x member): local-inertial river + floodplain
//               momentum, negative-flow limiter, dam-upstream kinematic flow
//               and reservoir release; per bifurcation path (x member): the
//               multi-level path flux and its path limiter.  Writes the
//               unlimited fluxes ("qu") to scratch and the cross-section state
//               in place.
//   k_limit     per catchment (x member): the storage-based outflow limit
//               rate from the unlimited fluxes of the cell, its upstream range
//               and its bifurcation ends.
//   k_stage     per catchment (x member): limited fluxes, upstream inflow as a
//               deterministic gather over the catchment's contiguous upstream
//               range, bifurcation net flux, fp64 storage update, flood-stage
//               diagnosis over the floodplain table and the fp64 water budget;
//               per path: the limit-rate scaling of the level fluxes.
//   k_levee     per levee (x member): the levee re-partition of the levee
//               cells' flood-stage result.
//
// After them, with output statistics attached, k_stats_accumulate folds the
// sub-step into the statistics.
//
// With several members the state is member-innermost ([N][M]) and a thread
// of the per-catchment, per-path and per-levee parts walks W elements of that
// order (the member tile, see tile_elem); W = 1 for one member.
//
// Catchments are stored breadth-first from the mouths, so the upstream cells
// of p are [up[p], up[p+1]) and no upstream index array exists.  Every float
// expression keeps the operand order of the reference kernels it replaces so
// that float rounding matches (cmfgpu/phys/cuda: outflow.cu, reservoir.cu,
// bifurcation.cu, storage.cu, levee.cu, adaptive_time.cu).  Storage is fp64
// ("STO") and ping-pongs between two buffers inside an interval so the
// limiter can read pre-update storage of neighbours while cells update their
// own.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "cmfb200.h"

// minimum resident 256-thread CTAs per SM (register caps) of the sub-step kernels;
// k_stage: 4 (64 registers, no spills)
#ifndef CMF_STAGE_MIN_BLOCKS
#define CMF_STAGE_MIN_BLOCKS 4
#endif
// k_momentum: 8 CTAs (32 registers) for one fp32 member, where the few bytes
// it spills cost less than the occupancy they buy (182 -> 161 us per 6M
// sub-step); fp64 and member-batched variants would spill hundreds of bytes
#ifndef CMF_MOMENTUM_MIN_BLOCKS
#define CMF_MOMENTUM_MIN_BLOCKS(REAL, ONE) ((sizeof(REAL) == 4 && (ONE)) ? 8 : 1)
#endif

namespace cmf {

constexpr int kMaxBifLevels = 8;
constexpr int kRowRegs = 10;         // floodplain levels held in registers (the CaMa layout)
constexpr int kChildUnroll = 4;      // upstream cells gathered with independent loads
constexpr int kMaxBlock = 256;       // threads per CTA (kernels use __launch_bounds__(256))
constexpr int kBudgetTerms = CMF_BUDGET_TERMS;
// control words (Dev::ctl)
constexpr int kCtlStep = 0;       // current sub-step index k
constexpr int kCtlMaxSteps = 1;   // max over members of the sub-step count
constexpr int kCtlBlocksDone = 2; // last-block-done counter of k_stage
constexpr int kHardSubStepCap = 100000;  // bound of the device-side sub-step loop

template <typename REAL>
struct Dev {
    long N;
    int M;
    int mshift;   // log2(M) when M is a power of two, else -1
    int mtile;    // member-tile width: consecutive members of a cell per thread (divides M)
    int K;
    long P;
    int L;
    int batched;
    int features;
    REAL g, min_kin, cfl_alpha, max_dt;
    int max_sub_cap;
    int cell_blocks;
    int path_blocks;
    // topology
    const int* dn;
    const int* up;
    const uint8_t* flags;
    const int* lslot;
    const int* rslot;
    const int* bptr;
    const int* bpaths;
    // parameters
    const REAL *rw, *rl, *rh, *celv, *ca, *dnd, *rman, *fman, *tbl, *runoff;
    // state
    REAL *rout, *fout, *rdep, *fdep, *pdep, *rcsd, *fcsd, *fcsa, *ffr;
    double *rs0, *fs0, *rs1, *fs1, *ps;
    // diagnostics
    double *rinf, *finf, *tsto, *gbif;
    REAL *lr, *wse, *pwse;
    // bifurcation
    const int *bci, *bdi;
    const REAL *bman, *bwid, *blen, *belv;
    REAL *bout, *bcsd, *bsum, *braw;
    // levee
    long NLV;
    const int* lci;
    const REAL *lcrown, *lfrac, *lbase;
    // reservoir
    const REAL *rcons, *remerg, *radj, *rnout, *raout, *rfcout;
    double* rti;
    // time / control
    REAL* dt;
    REAL* outer;
    int* nsub;
    int* cur;
    int* ctl;
    double* tsec;  // outer interval in seconds (double)
    double* budget;
    double* bpart;  // [kBudgetTerms][cell_blocks]
    int* status;
    // scratch fluxes
    REAL *qur, *quf;
    REAL* lrs;  // limit rate of the current sub-step, per cell x member
    // Levee-indexed copies, packed once per plan (null where the plan keeps
    // none): each levee cell's catchment area [NLV], floodplain row [NLV][K]
    // and, when members share them, river height, width, length [3][NLV].
    REAL* lpk_ca;
    REAL* lpk_tbl;
    REAL* lpk_geo;
};

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
template <bool ONE>
__device__ __forceinline__ long ix(long i, int m, int M) { return ONE ? i : i * (long)M + m; }

// Member-tile width of the batched kernels (1 for one member).  Warp g owns
// the 32 * W consecutive elements [32 W g, 32 W (g + 1)) of the member-
// innermost order and walks them in W warp-wide rows: lane l of the warp
// takes elements 32 W g + 32 w + l, w = 0 .. W-1.  Every row is a coalesced
// run of 32 members, and with 32 W <= M all W rows of a warp belong to one
// cell, whose topology and static fields the warp then reads once per row
// from L1.  Elements grow with w, so past the end in one row means past the
// end in all later rows.
template <typename REAL, bool ONE>
__device__ __forceinline__ int mtile_of(const Dev<REAL>& v) { return ONE ? 1 : v.mtile; }

__device__ __forceinline__ long tile_elem(long t0, int w, int W)
{
    return ((t0 >> 5) * W + w) * 32 + (t0 & 31);
}

// (item, member) of flat thread index t over [items, M]: a shift and a mask
// when M is a power of two, a division otherwise.
template <bool ONE, typename REAL>
__device__ __forceinline__ long split_member(const Dev<REAL>& v, long t, int& m)
{
    if (ONE) {
        m = 0;
        return t;
    }
    if (v.mshift >= 0) {
        m = (int)(t & ((1L << v.mshift) - 1));
        return t >> v.mshift;
    }
    const long i = t / v.M;
    m = (int)(t - i * v.M);
    return i;
}

template <bool ONE, typename REAL>
__device__ __forceinline__ REAL par(const REAL* p, int bit, int batched, long i, int m, int M)
{
    return p[(ONE || !(batched & bit)) ? i : i * (long)M + m];
}

template <typename REAL>
__device__ __forceinline__ REAL pow73(REAL x) { return x * x * cbrt(x); }

// End of the upstream range of cell x.  In the basin-major breadth-first
// order a basin's mouth sits right before its own upstream cells, so when
// x + 1 is a mouth the range of x ends one position earlier.
template <typename REAL>
__device__ __forceinline__ int upstream_end(const Dev<REAL>& v, long x)
{
    const int e = v.up[x + 1];
    return (x + 1 < v.N && (v.flags[x + 1] & CMF_CELL_MOUTH)) ? e - 1 : e;
}

// Member-active test and the per-member last-sub-step flag.
//   kh >= 0: a host-chosen step index (per-phase entry points);
//   kh == -1: read the interval's step counter from the device;
//   kh == -2: every member active, diag only when force_diag == 1.
// force_diag: 0 = last sub-step of the member, 1 = always, 2 = never.
__device__ __forceinline__ bool member_step(const int* ctl, const int* nsub, int kh, int m,
                                            int force_diag, bool& diag)
{
    if (kh == -2) { diag = force_diag == 1; return true; }
    int k = kh >= 0 ? kh : ctl[kCtlStep];
    int nm = nsub[m];
    diag = (force_diag == 1) || (force_diag == 0 && k == nm - 1);
    return k < nm;
}

__device__ __forceinline__ int step_index(const int* ctl, int kh)
{
    return kh >= 0 ? kh : (kh == -1 ? ctl[kCtlStep] : 0);
}

// Step index, activity and last-sub-step flag of member m (see member_step).
// With a single member the interval loop only runs k < n, so activity needs
// no load and nothing waits on the sub-step count except the diag flag.
struct StepInfo {
    int k;
    bool active;
    bool diag;
};

template <bool ONE>
__device__ __forceinline__ StepInfo step_info(const int* ctl, const int* nsub, int kh, int m,
                                              int force_diag)
{
    StepInfo s;
    if (kh == -2) {
        s.k = 0;
        s.active = true;
        s.diag = force_diag == 1;
        return s;
    }
    s.k = kh >= 0 ? kh : ctl[kCtlStep];
    const int nm = nsub[m];
    s.diag = (force_diag == 1) || (force_diag == 0 && s.k == nm - 1);
    s.active = ONE || s.k < nm;
    return s;
}

// ---------------------------------------------------------------------------
// k_momentum: cell part (outflow.cu:21-175, reservoir.cu:18-94)
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF>
__device__ __forceinline__ void momentum_cell(const Dev<REAL>& v, long i, int m, int kh,
                                              int force_diag)
{
    const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, force_diag);
    if (!st.active) return;
    const bool diag = st.diag;
    const int k = st.k;
    const double* __restrict__ rsrc = (k & 1) ? v.rs1 : v.rs0;
    const double* __restrict__ fsrc = (k & 1) ? v.fs1 : v.fs0;
    const int M = v.M;
    const long im = ix<ONE>(i, m, M);
    const REAL time_step = v.dt[m];
    const REAL gravity = v.g;
    const uint8_t fl = v.flags[i];
    const bool mouth = fl & CMF_CELL_MOUTH;
    const int dn = v.dn[i];

    REAL r_out = v.rout[im];
    REAL r_man = par<ONE>(v.rman, CMF_BATCH_RIVER_MANNING, v.batched, i, m, M);
    REAL r_dep = v.rdep[im];
    REAL r_wid = par<ONE>(v.rw, CMF_BATCH_RIVER_WIDTH, v.batched, i, m, M);
    REAL r_len = par<ONE>(v.rl, CMF_BATCH_RIVER_LENGTH, v.batched, i, m, M);
    REAL r_hgt = par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, i, m, M);
    REAL f_out = v.fout[im];
    REAL f_man = par<ONE>(v.fman, CMF_BATCH_FLOOD_MANNING, v.batched, i, m, M);
    REAL f_dep = v.fdep[im];
    REAL c_elv = v.celv[i];
    REAL dn_dist = v.dnd[i];
    REAL r_cs_dep = v.rcsd[im];
    REAL f_cs_dep = v.fcsd[im];
    REAL f_cs_area = v.fcsa[im];
    REAL fs = (REAL)fsrc[im];

    REAL river_elevation = c_elv - r_hgt;
    REAL wse = r_dep + river_elevation;

    const long dm = ix<ONE>(dn, m, M);
    REAL r_dep_dn = v.rdep[dm];
    REAL r_hgt_dn = par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, dn, m, M);
    REAL c_elv_dn = v.celv[dn];
    REAL river_elevation_dn = c_elv_dn - r_hgt_dn;
    REAL wse_dn = r_dep_dn + river_elevation_dn;
    if (mouth) wse_dn = c_elv;
    REAL max_wse = fmax(wse, wse_dn);

    REAL river_slope = (wse - wse_dn) / dn_dist;
    REAL flood_slope = fmin(fmax(river_slope, (REAL)-0.005), (REAL)0.005);

    REAL upd_r_cs_dep = mouth ? r_dep : max_wse - river_elevation;
    REAL r_sifd = fmax(sqrt(upd_r_cs_dep * r_cs_dep), (REAL)1e-6);
    REAL flood_surface = mouth ? wse : max_wse;
    REAL upd_f_cs_dep = fmax(flood_surface - c_elv, (REAL)0.0);
    REAL f_sifd = fmax(sqrt(upd_f_cs_dep * f_cs_dep), (REAL)1e-6);
    REAL upd_f_cs_area = fmax(fs / r_len - f_dep * r_wid, (REAL)0.0);

    REAL r_cs_area = upd_r_cs_dep * r_wid;
    bool river_condition = (r_sifd > (REAL)1e-5) && (r_cs_area > (REAL)1e-5);
    REAL unit_r_out = r_out / r_wid;
    REAL num_r = r_wid * (unit_r_out + gravity * time_step * r_sifd * river_slope);
    REAL den_r = (REAL)1.0 + gravity * time_step * (r_man * r_man) * fabs(unit_r_out)
                 * ((REAL)1.0 / (r_sifd * r_sifd * cbrt(r_sifd)));
    REAL upd_r_out = num_r / den_r;
    upd_r_out = river_condition ? upd_r_out : (REAL)0.0;

    bool flood_condition = (f_sifd > (REAL)1e-5) && (upd_f_cs_area > (REAL)1e-5);
    REAL upd_f_out = (REAL)0.0;
    if (flood_condition) {
        REAL f_imp_area = fmax(sqrt(upd_f_cs_area * fmax(f_cs_area, (REAL)1e-6)), (REAL)1e-6);
        REAL num_f = f_out + gravity * time_step * f_imp_area * flood_slope;
        REAL den_f = (REAL)1.0 + gravity * time_step * (f_man * f_man) * fabs(f_out)
                     * ((REAL)1.0 / (f_sifd * cbrt(f_sifd))) / f_imp_area;
        upd_f_out = num_f / den_f;
    }

    if ((upd_r_out * upd_f_out) < (REAL)0.0) upd_f_out = (REAL)0.0;
    const bool lev_cell = LEV && (fl & CMF_CELL_LEVEE);
    bool is_negative_flow = (upd_r_out < (REAL)0.0) && !mouth;
    REAL rs = (REAL)0;
    bool rs_loaded = false;
    if (is_negative_flow) {
        rs = (REAL)rsrc[im];
        rs_loaded = true;
        REAL ps = lev_cell ? (REAL)v.ps[im] : (REAL)0;
        REAL total_storage_f = rs + fs + ps;
        REAL total_negative_flow = (-upd_r_out - upd_f_out) * time_step;
        REAL limit_rate = fmin((REAL)0.05 * total_storage_f / total_negative_flow, (REAL)1.0);
        upd_r_out *= limit_rate;
        upd_f_out *= limit_rate;
    }

    if (RES && (fl & CMF_CELL_DAM_UPSTREAM)) {
        if (!rs_loaded) { rs = (REAL)rsrc[im]; rs_loaded = true; }
        REAL bed_slope = (c_elv - c_elv_dn) / dn_dist;
        bed_slope = fmax(bed_slope, v.min_kin);
        REAL kin_riv_vel = ((REAL)1.0 / r_man) * sqrt(bed_slope) * cbrt(r_dep * r_dep);
        REAL kin_riv = r_wid * r_dep * kin_riv_vel;
        kin_riv = fmin(kin_riv, rs / time_step);
        kin_riv = fmax(kin_riv, (REAL)0.0);
        REAL bed_slope_f = fmin(bed_slope, (REAL)0.005);
        REAL kin_fld_vel = ((REAL)1.0 / f_man) * sqrt(bed_slope_f) * cbrt(f_dep * f_dep);
        REAL kin_fld_area = fmax(fs / r_len - f_dep * r_wid, (REAL)0.0);
        REAL kin_fld = kin_fld_area * kin_fld_vel;
        kin_fld = fmin(kin_fld, fs / time_step);
        kin_fld = fmax(kin_fld, (REAL)0.0);
        upd_r_out = kin_riv;
        upd_f_out = kin_fld;
    }

    REAL res_total = (REAL)0;
    const bool res_cell = RES && (fl & CMF_CELL_RESERVOIR);
    if (res_cell) {
        // reservoir.cu:18-94: the release replaces the local-inertial flux;
        // undo/redo of the outgoing scatter is implicit because the limiter
        // gathers qu directly.
        if (!rs_loaded) { rs = (REAL)rsrc[im]; rs_loaded = true; }
        const int slot = v.rslot[i];
        REAL total = rs + fs;
        res_total = total;
        REAL total_inflow = (REAL)v.rti[im];
        REAL runoff_v = par<ONE>(v.runoff, CMF_BATCH_RUNOFF, v.batched, i, m, M);
        REAL inflow = total_inflow + runoff_v;
        REAL cons = v.rcons[slot];
        REAL emerg = v.remerg[slot];
        REAL adj = v.radj[slot];
        REAL n_out = v.rnout[slot];
        REAL a_out = v.raout[slot];
        REAL fc_out = v.rfcout[slot];
        REAL ro;
        if (total <= cons) {
            ro = n_out * sqrt(total / cons);
        } else if (total <= adj) {
            REAL frac2 = (total - cons) / (adj - cons);
            ro = n_out + exp((REAL)3.0 * log(frac2)) * (a_out - n_out);
        } else if (total <= emerg) {
            REAL frac3 = (total - adj) / (emerg - adj);
            REAL tmp = a_out + exp((REAL)0.1 * log(frac3)) * (fc_out - a_out);
            if (inflow >= fc_out) {
                REAL flood = n_out + ((total - cons) / (emerg - cons)) * (inflow - n_out);
                ro = fmax(flood, tmp);
            } else {
                ro = tmp;
            }
        } else {
            ro = (inflow >= fc_out) ? inflow : fc_out;
        }
        ro = fmax(ro, (REAL)0.0);
        ro = fmin(ro, total / time_step);
        upd_r_out = ro;
        upd_f_out = (REAL)0.0;
    }

    v.qur[im] = upd_r_out;
    v.quf[im] = upd_f_out;
    v.rcsd[im] = upd_r_cs_dep;
    v.fcsd[im] = upd_f_cs_dep;
    v.fcsa[im] = upd_f_cs_area;

    if (diag) {
        if (v.wse) v.wse[im] = wse;
        if (v.pwse) {
            REAL pwse = wse;
            if (lev_cell) pwse = fmin(c_elv + v.pdep[im], wse);
            v.pwse[im] = pwse;
        }
        if (v.tsto) {
            REAL tot;
            if (res_cell) {
                tot = res_total;
            } else {
                if (!rs_loaded) rs = (REAL)rsrc[im];
                REAL ps = lev_cell ? (REAL)v.ps[im] : (REAL)0;
                tot = rs + fs + ps;
            }
            v.tsto[im] = (double)tot;
        }
    }
}

// Water-surface elevation, protected WSE and total storage of a path end
// (the values outflow.cu/reservoir.cu leave in the scratch fields).
template <typename REAL, bool ONE, bool RES, bool LEV>
__device__ __forceinline__ void path_end_state(const Dev<REAL>& v, const double* rsrc,
                                               const double* fsrc, int c, int m, REAL& wse,
                                               REAL& pwse, REAL& tot)
{
    const long cm = ix<ONE>(c, m, v.M);
    const uint8_t fl = v.flags[c];
    REAL r_dep = v.rdep[cm];
    REAL r_hgt = par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, c, m, v.M);
    REAL c_elv = v.celv[c];
    wse = r_dep + (c_elv - r_hgt);
    pwse = wse;
    const bool lev_cell = LEV && (fl & CMF_CELL_LEVEE);
    if (lev_cell) pwse = fmin(c_elv + v.pdep[cm], wse);
    REAL rs = (REAL)rsrc[cm];
    REAL fs = (REAL)fsrc[cm];
    if (RES && (fl & CMF_CELL_RESERVOIR)) {
        tot = rs + fs;
    } else {
        REAL ps = lev_cell ? (REAL)v.ps[cm] : (REAL)0;
        tot = rs + fs + ps;
    }
}

// ---------------------------------------------------------------------------
// k_momentum: path part (bifurcation.cu:21-129, levee.cu:263-341)
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE, bool RES, bool LEV>
__device__ __forceinline__ void momentum_path(const Dev<REAL>& v, long p, int m, int kh)
{
    const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, 2);
    if (!st.active) return;
    const int k = st.k;
    const double* rsrc = (k & 1) ? v.rs1 : v.rs0;
    const double* fsrc = (k & 1) ? v.fs1 : v.fs0;
    const int M = v.M;
    const int L = v.L;
    const REAL time_step = v.dt[m];
    const REAL gravity = v.g;
    const int ci = v.bci[p];
    const int di = v.bdi[p];
    const REAL blen = v.blen[p];
    REAL wse_c, pwse_c, ts_c, wse_d, pwse_d, ts_d;
    path_end_state<REAL, ONE, RES, LEV>(v, rsrc, fsrc, ci, m, wse_c, pwse_c, ts_c);
    path_end_state<REAL, ONE, RES, LEV>(v, rsrc, fsrc, di, m, wse_d, pwse_d, ts_d);
    REAL max_wse = fmax(wse_c, wse_d);
    REAL max_pwse = fmax(pwse_c, pwse_d);
    REAL slope = (wse_c - wse_d) / blen;
    slope = fmin(fmax(slope, (REAL)-0.005), (REAL)0.005);

    REAL upd[kMaxBifLevels];
    REAL sum_out = (REAL)0;
#pragma unroll
    for (int lv = 0; lv < kMaxBifLevels; ++lv) {
        REAL upd_o = (REAL)0;
        if (lv < L) {
            const long lp = p * (long)L + lv;      // parameter index
            const long ls = ix<ONE>(lp, m, M);     // state index
            REAL elv = v.belv[lp];
            REAL upd_csd;
            REAL sifd;
            if (LEV) {
                REAL current_max_wse = (lv == 0) ? max_wse : max_pwse;
                upd_csd = fmax(current_max_wse - elv, (REAL)0.0);
                if (lv == 0) {
                    REAL old_csd = v.bcsd[ls];
                    sifd = sqrt(upd_csd * old_csd);
                    if (sifd <= (REAL)0.0) sifd = upd_csd;
                } else {
                    sifd = upd_csd;
                }
            } else {
                REAL csd = v.bcsd[ls];
                upd_csd = fmax(max_wse - elv, (REAL)0);
                sifd = fmax(sqrt(upd_csd * csd), sqrt(upd_csd * (REAL)0.01));
            }
            if (sifd > (REAL)1e-5) {
                REAL man = v.bman[lp];
                REAL w = v.bwid[lp];
                REAL o = v.bout[ls];
                REAL unit_o = o / w;
                REAL num = w * (unit_o + gravity * time_step * sifd * slope);
                REAL den = (REAL)1 + gravity * time_step * (man * man) * fabs(unit_o)
                           * ((REAL)1 / pow73(sifd));
                upd_o = num / den;
            }
            sum_out += upd_o;
            v.bcsd[ls] = upd_csd;
        }
        upd[lv] = upd_o;
    }
    REAL limit_rate = fmin((REAL)0.05 * fmin(ts_c, ts_d) / (fabs(sum_out) * time_step), (REAL)1);
    sum_out *= limit_rate;
    REAL raw = (REAL)0;
#pragma unroll
    for (int lv = 0; lv < kMaxBifLevels; ++lv) {
        if (lv < L) {
            REAL o = upd[lv] * limit_rate;
            v.bout[ix<ONE>(p * (long)L + lv, m, M)] = o;
            raw += o;
        }
    }
    const long pm = ix<ONE>(p, m, M);
    v.bsum[pm] = sum_out;
    v.braw[pm] = raw;
}

template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF>
__global__ void __launch_bounds__(256, CMF_MOMENTUM_MIN_BLOCKS(REAL, ONE)) k_momentum(const Dev<REAL> v, int kh, int force_diag)
{
    const int W = mtile_of<REAL, ONE>(v);
    if (BIF && (int)blockIdx.x >= v.cell_blocks) {
        const long t0 = (long)(blockIdx.x - v.cell_blocks) * blockDim.x + threadIdx.x;
        for (int w = 0; w < W; ++w) {
            const long t = tile_elem(t0, w, W);
            if (t >= v.P * (long)v.M) return;
            int m;
            long p = split_member<ONE>(v, t, m);
            momentum_path<REAL, ONE, RES, LEV>(v, p, m, kh);
        }
        return;
    }
    const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int w = 0; w < W; ++w) {
        const long t = tile_elem(t0, w, W);
        if (t >= v.N * (long)v.M) return;
        int m;
        long i = split_member<ONE>(v, t, m);
        momentum_cell<REAL, ONE, RES, LEV, BIF>(v, i, m, kh, force_diag);
    }
}

// ---------------------------------------------------------------------------
// Limit rate of one catchment (outflow.cu:196-203 with the outgoing storage of
// outflow.cu:170-174, reservoir.cu:273-277/320-324, bifurcation.cu:125-128
// gathered instead of scattered).
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE, bool BIF>
__device__ __forceinline__ REAL outgoing_of(const Dev<REAL>& v, long x, int m, REAL ts,
                                            REAL qr, REAL qf)
{
    const int M = v.M;
    REAL pos = fmax(qr, (REAL)0.0) + fmax(qf, (REAL)0.0);
    double og = (double)(pos * ts);
    const int c0 = v.up[x], c1 = upstream_end(v, x);
    for (int cb = c0; cb < c1; cb += kChildUnroll) {
        REAL nr[kChildUnroll], nf[kChildUnroll];
#pragma unroll
        for (int j = 0; j < kChildUnroll; ++j) {
            if (cb + j < c1) {
                const long cm = ix<ONE>(cb + j, m, M);
                nr[j] = v.qur[cm];
                nf[j] = v.quf[cm];
            }
        }
#pragma unroll
        for (int j = 0; j < kChildUnroll; ++j) {
            if (cb + j < c1) {
                REAL neg = fmin(nr[j], (REAL)0.0) + fmin(nf[j], (REAL)0.0);
                og += (double)(-neg * ts);
            }
        }
    }
    if (BIF && (v.flags[x] & CMF_CELL_BIFURCATION)) {
        const int b0 = v.bptr[x], b1 = v.bptr[x + 1];
        for (int b = b0; b < b1; ++b) {
            const int e = v.bpaths[b];
            REAL s = v.bsum[ix<ONE>(e >> 1, m, M)];
            if (e & 1) og += (double)(-fmin(s, (REAL)0) * ts);
            else og += (double)(fmax(s, (REAL)0) * ts);
        }
    }
    return (REAL)og;
}

template <typename REAL, bool ONE, bool BIF>
__device__ __forceinline__ REAL limit_rate_of(const Dev<REAL>& v, const double* rsrc,
                                              const double* fsrc, long x, int m, REAL ts)
{
    const long xm = ix<ONE>(x, m, v.M);
    REAL outgoing = outgoing_of<REAL, ONE, BIF>(v, x, m, ts, v.qur[xm], v.quf[xm]);
    REAL rate_storage = (REAL)(rsrc[xm] + fsrc[xm]);
    return (outgoing > (REAL)1e-8) ? fmin(rate_storage / outgoing, (REAL)1.0) : (REAL)1.0;
}

// ---------------------------------------------------------------------------
// Flood stage (storage.cu:118-211) on a known total storage.  Writes river /
// flood storage split, depths and fraction into the out-parameters.
// ---------------------------------------------------------------------------
template <typename REAL>
struct StageOut {
    double rs, fs;
    REAL rdep, fdep, ffr;
};

// A floodplain-table row held in registers (the CaMa layout has exactly
// kRowRegs levels; other level counts scan the row from memory) together with
// the catchment area, both needed only by flooded cells.
template <typename REAL>
struct TableRow {
    REAL H[kRowRegs];
    REAL ca;
    bool valid;
};

// Issue the row loads (independent 8-byte loads for fp32) and the area load.
template <typename REAL>
__device__ __forceinline__ void load_row(const Dev<REAL>& v, long i, TableRow<REAL>& r)
{
    const REAL* __restrict__ row = v.tbl + i * (long)kRowRegs;
    if (sizeof(REAL) == 4 && ((uintptr_t)row & 7) == 0) {
        const float2* r2 = reinterpret_cast<const float2*>(row);
#pragma unroll
        for (int q = 0; q < kRowRegs / 2; ++q) {
            float2 x = __ldg(r2 + q);
            r.H[2 * q] = (REAL)x.x;
            r.H[2 * q + 1] = (REAL)x.y;
        }
    } else {
#pragma unroll
        for (int l = 0; l < kRowRegs; ++l) r.H[l] = __ldg(row + l);
    }
    r.ca = v.ca[i];
    r.valid = true;
}

template <typename REAL, bool ONE>
__device__ __forceinline__ void flood_stage(const Dev<REAL>& v, long i, int m, double total_s,
                                            REAL rh, REAL rw, REAL rl, TableRow<REAL>& row,
                                            StageOut<REAL>& o)
{
    REAL total_storage = (REAL)total_s;
    REAL river_max_storage = rl * rw * rh;
    if (total_storage <= river_max_storage) {
        o.rs = total_s;
        o.fs = 0.0;
        o.rdep = total_storage / (rl * rw);
        o.fdep = (REAL)0;
        o.ffr = (REAL)0;
        return;
    }
    const int nl = v.K;
    const bool in_regs = nl == kRowRegs;
    if (in_regs && !row.valid) load_row(v, i, row);
    REAL ca = in_regs ? row.ca : v.ca[i];
    REAL catchment_width = ca / rl;
    REAL width_increment = catchment_width / (REAL)nl;
    int level = 0;
    REAL S_accum = river_max_storage;
    REAL prev_H = (REAL)0;
    REAL prev_W = rw;
    REAL prev_total_storage = river_max_storage;
    REAL prev_flood_depth = (REAL)0;
    REAL next_flood_depth = (REAL)0;
    // The scan stops at the first level the storage does not exceed, exactly
    // as the reference's `break`.
    auto level_step = [&](int l, REAL H_curr) -> bool {
        REAL W_curr = rw + (REAL)(l + 1) * width_increment;
        REAL dS = rl * (REAL)0.5 * (prev_W + W_curr) * (H_curr - prev_H);
        REAL S_curr = S_accum + dS;
        next_flood_depth = H_curr;
        if (total_storage > S_curr) {
            level += 1;
            prev_total_storage = S_curr;
            prev_flood_depth = H_curr;
            S_accum = S_curr;
            prev_H = H_curr;
            prev_W = W_curr;
            return true;
        }
        return false;
    };
    if (in_regs) {
        // row loaded up front (independent loads, one memory latency)
        bool scanning = true;
#pragma unroll
        for (int l = 0; l < kRowRegs; ++l)
            if (scanning) scanning = level_step(l, row.H[l]);
    } else {
        const REAL* trow = v.tbl + i * (long)nl;
        for (int l = 0; l < nl; ++l)
            if (!level_step(l, __ldg(trow + l))) break;
    }
    REAL prev_total_width = rw + (REAL)level * width_increment;
    REAL diff_width = (REAL)0;
    REAL fdep;
    if (level == nl) {
        fdep = prev_flood_depth + (total_storage - prev_total_storage) / (prev_total_width * rl);
    } else {
        REAL flood_grad = (next_flood_depth - prev_flood_depth) / width_increment;
        diff_width = sqrt(prev_total_width * prev_total_width
                          + (REAL)2 * (total_storage - prev_total_storage) / (flood_grad * rl))
                     - prev_total_width;
        fdep = prev_flood_depth + diff_width * flood_grad;
    }
    REAL cap = river_max_storage + rl * rw * fdep;
    double cap_s = (double)cap;
    double river_storage_final = cap_s < total_s ? cap_s : total_s;
    REAL rdep = (REAL)river_storage_final / (rl * rw);
    REAL ff_mid = (prev_total_width + diff_width - rw) * rl / ca;
    ff_mid = ff_mid < (REAL)0 ? (REAL)0 : (ff_mid > (REAL)1 ? (REAL)1 : ff_mid);
    REAL ffr = (level == nl) ? (REAL)1 : ff_mid;
    double flood_storage_final = total_s - river_storage_final;
    if (flood_storage_final < 0.0) flood_storage_final = 0.0;
    o.rs = river_storage_final;
    o.fs = flood_storage_final;
    o.rdep = rdep;
    o.fdep = fdep;
    o.ffr = ffr;
}

// ---------------------------------------------------------------------------
// Levee re-partition (levee.cu:29-261) of one levee cell after its flood
// stage.  In: storages/depths/fraction from flood_stage.  Out: the same plus
// protected storage/depth.
// ---------------------------------------------------------------------------
template <typename REAL>
__device__ __forceinline__ REAL clamp01(REAL x) { return fmin(fmax(x, (REAL)0), (REAL)1); }

template <typename REAL, bool ONE>
__device__ __forceinline__ void levee_stage(const Dev<REAL>& v, const REAL* row, REAL l_crown,
                                            REAL l_frac, REAL l_base_h, REAL ca, REAL rh,
                                            REAL rw, REAL rl, StageOut<REAL>& s, double& p_out,
                                            REAL& pdep_out)
{
    const int nl = v.K;
    double riv_sto_curr_hp = s.rs;
    double fld_sto_curr_hp = s.fs;
    double total_sto_hp = riv_sto_curr_hp + fld_sto_curr_hp;
    REAL riv_sto_curr = (REAL)riv_sto_curr_hp;
    REAL fld_sto_curr = (REAL)fld_sto_curr_hp;
    REAL fld_depth_curr = s.fdep;
    REAL total_sto = (REAL)total_sto_hp;
    REAL riv_max_sto = rl * rw * rh;
    if (!(total_sto >= riv_max_sto)) {
        p_out = 0.0;
        pdep_out = (REAL)0.0;
        return;
    }
    REAL dwth_inc = (ca / rl) / (REAL)nl;
    REAL levee_dist = l_frac * (ca / rl);
    REAL s_curr = riv_max_sto;
    REAL dhgt_pre = (REAL)0.0;
    REAL dwth_pre = rw;
    REAL levee_base_sto = riv_max_sto;
    REAL levee_fill_sto = riv_max_sto;
    bool found_base = false, found_fill = false;
    int ilev = (int)(l_frac * (REAL)nl);
    REAL dsto_fil_B = (REAL)0.0, dwth_fil_B = (REAL)0.0, ddph_fil_B = (REAL)0.0,
         gradient_B = (REAL)0.0;
    bool found_B = false;
    bool scan_needed = true;
    for (int l = 0; l < nl; ++l) {
        if (!scan_needed) break;
        REAL depth_val = row[l];
        REAL dhgt_seg = fmax(depth_val - dhgt_pre, (REAL)1e-6);
        REAL dwth_mid = dwth_pre + (REAL)0.5 * dwth_inc;
        REAL dsto_seg = rl * dwth_mid * dhgt_seg;
        REAL s_next = s_curr + dsto_seg;
        REAL gradient = dhgt_seg / dwth_inc;

        bool cond_base = (l_base_h > dhgt_pre) && (l_base_h <= depth_val);
        REAL ratio_base = (l_base_h - dhgt_pre) / dhgt_seg;
        REAL dsto_base_p = rl * (dwth_pre + (REAL)0.5 * ratio_base * dwth_inc) * (ratio_base * dhgt_seg);
        if (cond_base && !found_base) levee_base_sto = s_curr + dsto_base_p;
        found_base = found_base || cond_base;

        bool cond_fill = (l_crown > dhgt_pre) && (l_crown <= depth_val);
        REAL ratio_fill = (l_crown - dhgt_pre) / dhgt_seg;
        REAL dsto_fill_p = rl * (dwth_pre + (REAL)0.5 * ratio_fill * dwth_inc) * (ratio_fill * dhgt_seg);
        if (cond_fill && !found_fill) levee_fill_sto = s_curr + dsto_fill_p;
        found_fill = found_fill || cond_fill;

        REAL dhgt_dif_loop = l_crown - l_base_h;
        REAL s_top_loop = levee_base_sto + (levee_dist + rw) * dhgt_dif_loop * rl;
        REAL dsto_add_wedge = (levee_dist + rw) * (l_crown - depth_val) * rl;
        REAL threshold = s_next + dsto_add_wedge;

        bool cond_check = (l >= ilev) && !found_B;
        bool cond_found = cond_check && (total_sto < threshold);
        REAL current_lb = (l == ilev) ? s_top_loop : dsto_fil_B;
        if (cond_check && !cond_found) {
            dsto_fil_B = threshold;
            dwth_fil_B = dwth_inc * (REAL)(l + 1) - levee_dist;
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
    bool is_case4 = total_sto >= levee_fill_sto;
    bool is_case3 = (!is_case4) && (total_sto >= s_top);
    bool is_case2 = (!is_case4) && (!is_case3) && (total_sto >= levee_base_sto);

    REAL dsto_add_c2 = total_sto - levee_base_sto;
    REAL dwth_add_c2 = levee_dist + rw;
    REAL f_dph_c2 = l_base_h + dsto_add_c2 / dwth_add_c2 / rl;
    REAL r_sto_c2 = riv_max_sto + rl * rw * f_dph_c2;
    REAL r_dph_c2 = r_sto_c2 / rl / rw;
    REAL f_sto_c2 = fmax(total_sto - r_sto_c2, (REAL)0.0);
    REAL f_frc_c2 = l_frac;

    REAL dsto_add_B = total_sto - dsto_fil_B;
    REAL term_B = dwth_fil_B * dwth_fil_B + (REAL)2.0 * dsto_add_B / rl / (gradient_B + (REAL)1e-9);
    REAL dwth_add_B = -dwth_fil_B + sqrt(fmax(term_B, (REAL)0.0));
    REAL ddph_add_B = dwth_add_B * gradient_B;
    REAL p_dph_B_found = l_base_h + ddph_fil_B + ddph_add_B;
    REAL f_frc_B_found = (dwth_fil_B + levee_dist) / (dwth_inc * (REAL)nl);
    REAL ddph_add_B_extra = dsto_add_B / (dwth_fil_B * rl + (REAL)1e-9);
    REAL p_dph_B_extra = l_base_h + ddph_fil_B + ddph_add_B_extra;
    REAL p_dph_B = found_B ? p_dph_B_found : p_dph_B_extra;
    REAL f_frc_B = found_B ? f_frc_B_found : (REAL)1.0;

    REAL f_dph_c3 = l_crown;
    REAL r_sto_c3 = riv_max_sto + rl * rw * f_dph_c3;
    REAL r_dph_c3 = r_sto_c3 / rl / rw;
    REAL f_sto_c3 = fmax(s_top - r_sto_c3, (REAL)0.0);
    REAL p_dph_c3 = p_dph_B;
    REAL f_frc_c3 = clamp01(f_frc_B);

    REAL f_dph_c4 = fld_depth_curr;
    REAL r_sto_c4 = riv_sto_curr;
    REAL dsto_add_c4 = (f_dph_c4 - l_crown) * (levee_dist + rw) * rl;
    REAL f_sto_c4 = fmax(s_top + dsto_add_c4 - r_sto_c4, (REAL)0.0);
    REAL p_dph_c4 = f_dph_c4;

    REAL r_sto_candidate = is_case2 ? r_sto_c2 : (is_case3 ? r_sto_c3 : (is_case4 ? r_sto_c4 : riv_sto_curr));
    REAL f_sto_candidate = is_case2 ? f_sto_c2 : (is_case3 ? f_sto_c3 : (is_case4 ? f_sto_c4 : fld_sto_curr));
    bool no_levee_partition = !is_case2 && !is_case3 && !is_case4;
    double r_sto = (is_case4 || no_levee_partition) ? riv_sto_curr_hp
                                                     : fmin((double)r_sto_candidate, total_sto_hp);
    double remaining_sto = total_sto_hp - r_sto;
    remaining_sto = remaining_sto > 0.0 ? remaining_sto : 0.0;
    double f_sto_candidate_hp = (double)f_sto_candidate;
    double f_sto = fmin(f_sto_candidate_hp > 0.0 ? f_sto_candidate_hp : 0.0, remaining_sto);
    if (is_case2) f_sto = remaining_sto;
    if (no_levee_partition) f_sto = fld_sto_curr_hp;
    double p_sto = remaining_sto - f_sto;
    p_sto = p_sto > 0.0 ? p_sto : 0.0;
    REAL r_dph = is_case2 ? r_dph_c2 : (is_case3 ? r_dph_c3 : s.rdep);
    REAL f_dph = is_case2 ? f_dph_c2 : (is_case3 ? f_dph_c3 : fld_depth_curr);
    REAL p_dph = is_case2 ? (REAL)0.0 : (is_case3 ? p_dph_c3 : (is_case4 ? p_dph_c4 : (REAL)0.0));
    REAL f_frc = is_case2 ? f_frc_c2 : (is_case3 ? f_frc_c3 : s.ffr);
    s.rs = r_sto;
    s.fs = f_sto;
    s.rdep = r_dph;
    s.fdep = f_dph;
    s.ffr = f_frc;
    p_out = p_sto;
    pdep_out = p_dph;
}

// ---------------------------------------------------------------------------
// Deterministic block sum of kBudgetTerms fp64 values into bpart[term][block]
// (fixed shuffle tree + fixed smem order; partials are accumulated across the
// sub-steps of an interval, each block always owning the same cells).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void block_budget(double (&val)[kBudgetTerms], double* bpart,
                                             int nblocks)
{
    __shared__ double part[kBudgetTerms][32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int t = 0; t < kBudgetTerms; ++t) {
        double x = val[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) part[t][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < kBudgetTerms; ++t) {
            double x = lane < nwarps ? part[t][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) bpart[(long)t * nblocks + blockIdx.x] += x;
        }
    }
}

// ---------------------------------------------------------------------------
// k_stage: cell part
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF, bool BUDGET>
__device__ __forceinline__ void stage_cell(const Dev<REAL>& v, long i, int m, int kh,
                                           int force_diag, double (&bud)[kBudgetTerms])
{
    // Every load of this cell is issued before anything waits on another
    // load's value: the activity test of a single member is static (the
    // interval loop only runs k < n), and the upstream gather is unrolled into
    // independent predicated loads.
    const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, force_diag);
    if (!st.active) return;
    const int k = st.k;
    const double* __restrict__ rsrc = (k & 1) ? v.rs1 : v.rs0;
    const double* __restrict__ fsrc = (k & 1) ? v.fs1 : v.fs0;
    double* __restrict__ rdst = (k & 1) ? v.rs0 : v.rs1;
    double* __restrict__ fdst = (k & 1) ? v.fs0 : v.fs1;
    const int M = v.M;
    const long im = ix<ONE>(i, m, M);
    const REAL ts = v.dt[m];
    const uint8_t fl = v.flags[i];
    const bool mouth = fl & CMF_CELL_MOUTH;
    const bool lev_cell = LEV && (fl & CMF_CELL_LEVEE);
    const bool res_cell = RES && (fl & CMF_CELL_RESERVOIR);

    const double rsto = rsrc[im];
    const double fsto = fsrc[im];
    const REAL qr = v.qur[im], qf = v.quf[im];
    const REAL ro = par<ONE>(v.runoff, CMF_BATCH_RUNOFF, v.batched, i, m, M);
    const REAL rh = par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, i, m, M);
    const REAL rw = par<ONE>(v.rw, CMF_BATCH_RIVER_WIDTH, v.batched, i, m, M);
    const REAL rl = par<ONE>(v.rl, CMF_BATCH_RIVER_LENGTH, v.batched, i, m, M);
    // limit rates of this sub-step were computed once per cell by k_limit
    const REAL lr_i = v.lrs[im];
    const int c0 = v.up[i], c1 = upstream_end(v, i);
    const double prot = lev_cell ? v.ps[im] : 0.0;

    // A cell flooded in the previous sub-step will almost surely need its
    // floodplain row: start those loads now, alongside the upstream gather.
    TableRow<REAL> row;
    row.valid = false;
    if (v.K == kRowRegs && fsto > 0.0) load_row(v, i, row);

    // upstream inflow: gather the limited fluxes of the upstream cells, in
    // range order, kChildUnroll independent loads at a time
    double rin = 0.0, fin = 0.0, rti = 0.0;
    for (int cb = c0; cb < c1; cb += kChildUnroll) {
        REAL cr[kChildUnroll], cf[kChildUnroll], cl[kChildUnroll];
#pragma unroll
        for (int j = 0; j < kChildUnroll; ++j) {
            if (cb + j < c1) {
                const long cm = ix<ONE>(cb + j, m, M);
                cr[j] = v.qur[cm];
                cf[j] = v.quf[cm];
                cl[j] = v.lrs[cm];
            }
        }
#pragma unroll
        for (int j = 0; j < kChildUnroll; ++j) {
            if (cb + j < c1) {
                const REAL ur = (cr[j] >= (REAL)0.0) ? cr[j] * cl[j] : cr[j] * lr_i;
                const REAL uf = (cf[j] >= (REAL)0.0) ? cf[j] * cl[j] : cf[j] * lr_i;
                rin += (double)ur;
                fin += (double)uf;
                if (res_cell) rti += (double)(ur + uf);
            }
        }
    }

    // own limited flux (the downstream rate is needed only for negative flux)
    REAL lr_dn = lr_i;
    if (!mouth && (qr < (REAL)0.0 || qf < (REAL)0.0))
        lr_dn = v.lrs[ix<ONE>(v.dn[i], m, M)];
    const REAL rout = (qr >= (REAL)0.0) ? qr * lr_i : qr * lr_dn;
    const REAL fout = (qf >= (REAL)0.0) ? qf * lr_i : qf * lr_dn;

    // bifurcation net flux of this cell (bifurcation.cu:131-156 gathered)
    double gb = 0.0;
    if (BIF && (fl & CMF_CELL_BIFURCATION)) {
        const int b0 = v.bptr[i], b1 = v.bptr[i + 1];
        for (int b = b0; b < b1; ++b) {
            const int e = v.bpaths[b];
            const int p = e >> 1;
            const REAL raw = v.braw[ix<ONE>(p, m, M)];
            const int other = (e & 1) ? v.bci[p] : v.bdi[p];
            const REAL lr_o = v.lrs[ix<ONE>(other, m, M)];
            const REAL lr_c = (e & 1) ? lr_o : lr_i;
            const REAL lr_d = (e & 1) ? lr_i : lr_o;
            const REAL net = (raw >= (REAL)0) ? raw * lr_c : raw * lr_d;
            gb += (e & 1) ? (double)(-net) : (double)net;
        }
    }

    // storage update (storage.cu:67-116)
    const REAL rinf = (REAL)rin;
    const REAL finf = (REAL)fin;
    const REAL gbif = BIF ? (REAL)gb : (REAL)0;
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
    REAL external_delta = ro * ts;
    double total_next = river_su + flood_su + prot + (double)external_delta;
    double total_s = total_next > 0.0 ? total_next : 0.0;

    StageOut<REAL> s;
    flood_stage<REAL, ONE>(v, i, m, total_s, rh, rw, rl, row, s);
    // Levee cells are re-partitioned afterwards by k_levee; the partition
    // conserves r + f + p, so the budget's end storage is taken here.
    const double p_new = 0.0;

    if (BUDGET) {
        const double pre = rsto + fsto + prot;
        const double raw_next = rsto + (double)river_delta + fsto + (double)flood_delta + prot
                                + (double)external_delta;
        bud[CMF_BUDGET_RUNOFF_IN] += (double)external_delta;
        bud[CMF_BUDGET_CLIP_GAIN] += total_s - raw_next;
        if (mouth) bud[CMF_BUDGET_MOUTH_OUT] += ((double)rout + (double)fout) * (double)ts;
        if (k == 0 || kh == -2) bud[CMF_BUDGET_STORAGE_START] += pre;
        if (st.diag) bud[CMF_BUDGET_STORAGE_END] += s.rs + s.fs + p_new;
    }

    v.rout[im] = rout;
    v.fout[im] = fout;
    rdst[im] = s.rs;
    fdst[im] = s.fs;
    v.rdep[im] = s.rdep;
    v.fdep[im] = s.fdep;
    v.ffr[im] = s.ffr;

    if (!lev_cell && st.diag) v.pdep[im] = s.fdep;
    if (res_cell) v.rti[im] = rti;
    if (st.diag) {
        if (v.rinf) v.rinf[im] = rin;
        if (v.finf) v.finf[im] = fin;
        if (v.lr) v.lr[im] = lr_i;
        if (v.gbif) v.gbif[im] = gb;
    }
    if (!isfinite(s.rs) || !isfinite(s.fs) || !isfinite(rout) || !isfinite(fout))
        atomicOr(v.status, CMF_STATUS_NONFINITE);
}

// k_stage: path part (bifurcation.cu:131-156, level fluxes only)
template <typename REAL, bool ONE, bool BIF>
__device__ __forceinline__ void stage_path(const Dev<REAL>& v, long p, int m, int kh)
{
    bool diag;
    if (!member_step(v.ctl, v.nsub, kh, m, 2, diag)) return;
    const int ci = v.bci[p], di = v.bdi[p];
    const REAL lr_c = v.lrs[ix<ONE>(ci, m, v.M)];
    const REAL lr_d = v.lrs[ix<ONE>(di, m, v.M)];
    for (int lv = 0; lv < v.L; ++lv) {
        const long ls = ix<ONE>(p * (long)v.L + lv, m, v.M);
        REAL o = v.bout[ls];
        v.bout[ls] = (o >= (REAL)0) ? o * lr_c : o * lr_d;
    }
}

// ---------------------------------------------------------------------------
// k_limit: the storage-based outflow limiter rate of every catchment
// (outflow.cu:196-203) from this sub-step's unlimited fluxes, computed once
// per cell; k_stage reads it for the cell, its upstream cells, its downstream
// cell and its bifurcation partners.
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE, bool BIF>
__global__ void __launch_bounds__(256, (sizeof(REAL) == 4 ? 8 : 4)) k_limit(const Dev<REAL> v, int kh)
{
    const int W = mtile_of<REAL, ONE>(v);
    const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int w = 0; w < W; ++w) {
        const long t = tile_elem(t0, w, W);
        if (t >= v.N * (long)v.M) return;
        int m;
        long i = split_member<ONE>(v, t, m);
        const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, 2);
        if (!st.active) continue;
        const int k = st.k;
        const double* rsrc = (k & 1) ? v.rs1 : v.rs0;
        const double* fsrc = (k & 1) ? v.fs1 : v.fs0;
        v.lrs[ix<ONE>(i, m, v.M)] = limit_rate_of<REAL, ONE, BIF>(v, rsrc, fsrc, i, m, v.dt[m]);
    }
}

// Interval loop control, run by the last kernel of a sub-step: the last
// block to finish advances the step counter (every block has read it by
// then) and, inside the interval graph, sets the while-condition.
__device__ __forceinline__ void advance_step(int* ctl, cudaGraphConditionalHandle h, int set_cond)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        int done = atomicAdd(&ctl[kCtlBlocksDone], 1);
        if (done == (int)gridDim.x - 1) {
            ctl[kCtlBlocksDone] = 0;
            const int next = ctl[kCtlStep] + 1;
            ctl[kCtlStep] = next;
            __threadfence();
            if (set_cond) cudaGraphSetConditional(h, next < ctl[kCtlMaxSteps] ? 1u : 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// k_levee: levee re-partition (levee.cu:29-261) over the compact levee list,
// after k_stage wrote the sub-step's flood-stage result.  A kernel of its own:
// levee cells are a scattered minority, and running their long scan inside
// k_stage would stretch every CTA of the much larger catchment grid.
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE>
__global__ void __launch_bounds__(256) k_levee(const Dev<REAL> v, int kh, int force_diag,
                                               cudaGraphConditionalHandle h, int advance)
{
    const int W = mtile_of<REAL, ONE>(v);
    const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int w = 0; w < W; ++w) {
        const long t = tile_elem(t0, w, W);
        if (t >= v.NLV * (long)v.M) break;
        int m;
        const long li = split_member<ONE>(v, t, m);
        const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, force_diag);
        if (st.active) {
            const int k = st.k;
            double* rdst = (k & 1) ? v.rs0 : v.rs1;
            double* fdst = (k & 1) ? v.fs0 : v.fs1;
            const long ci = v.lci[li];
            const long cm = ix<ONE>(ci, m, v.M);
            const REAL l_crown = v.lcrown[li], l_frac = v.lfrac[li], l_base = v.lbase[li];
            REAL rh, rw, rl, ca;
            const REAL* row;
            StageOut<REAL> s;
            s.rs = rdst[cm];
            s.fs = fdst[cm];
            s.rdep = v.rdep[cm];
            s.fdep = v.fdep[cm];
            s.ffr = v.ffr[cm];
            // static fields from the levee-indexed copies where the plan keeps
            // them (coalesced over the levee list), else from the cells
            if (v.lpk_ca) {
                ca = v.lpk_ca[li];
                row = v.lpk_tbl + li * (long)v.K;
            } else {
                ca = v.ca[ci];
                row = v.tbl + ci * (long)v.K;
            }
            if (v.lpk_geo) {
                rh = v.lpk_geo[li];
                rw = v.lpk_geo[v.NLV + li];
                rl = v.lpk_geo[2 * v.NLV + li];
            } else {
                rh = par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, ci, m, v.M);
                rw = par<ONE>(v.rw, CMF_BATCH_RIVER_WIDTH, v.batched, ci, m, v.M);
                rl = par<ONE>(v.rl, CMF_BATCH_RIVER_LENGTH, v.batched, ci, m, v.M);
            }
            double p_new;
            REAL pdep_new;
            levee_stage<REAL, ONE>(v, row, l_crown, l_frac, l_base, ca, rh, rw, rl, s, p_new,
                                   pdep_new);
            rdst[cm] = s.rs;
            fdst[cm] = s.fs;
            v.ps[cm] = p_new;
            v.rdep[cm] = s.rdep;
            v.fdep[cm] = s.fdep;
            v.pdep[cm] = pdep_new;
            v.ffr[cm] = s.ffr;
        }
    }
    if (kh == -1 && advance) advance_step(v.ctl, h, 1);
}

template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF, bool BUDGET>
__global__ void __launch_bounds__(256, CMF_STAGE_MIN_BLOCKS) k_stage(const Dev<REAL> v, int kh, int force_diag,
                                               cudaGraphConditionalHandle h, int set_cond)
{
    const int W = mtile_of<REAL, ONE>(v);
    if (BIF && (int)blockIdx.x >= v.cell_blocks) {
        const long t0 = (long)(blockIdx.x - v.cell_blocks) * blockDim.x + threadIdx.x;
        for (int w = 0; w < W; ++w) {
            const long t = tile_elem(t0, w, W);
            if (t >= v.P * (long)v.M) break;
            int m;
            long p = split_member<ONE>(v, t, m);
            stage_path<REAL, ONE, BIF>(v, p, m, kh);
        }
    } else {
        double bud[kBudgetTerms];
#pragma unroll
        for (int q = 0; q < kBudgetTerms; ++q) bud[q] = 0.0;
        const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x;
        for (int w = 0; w < W; ++w) {
            const long t = tile_elem(t0, w, W);
            if (t >= v.N * (long)v.M) break;
            int m;
            long i = split_member<ONE>(v, t, m);
            stage_cell<REAL, ONE, RES, LEV, BIF, BUDGET>(v, i, m, kh, force_diag, bud);
        }
        if (BUDGET) block_budget(bud, v.bpart, v.cell_blocks);
    }
    // With levees, k_levee is the last kernel of the sub-step and advances.
    if (!LEV && kh == -1) advance_step(v.ctl, h, set_cond);
}

// ---------------------------------------------------------------------------
// CFL sub-step count (adaptive_time.cu:19-48), per member.
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE, bool RES>
__global__ void __launch_bounds__(256) k_cfl(const Dev<REAL> v)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int n_steps = 1;
    int m = 0;
    if (t < v.N * (long)v.M) {
        long i = split_member<ONE>(v, t, m);
        bool skip = RES && (v.flags[i] & CMF_CELL_DAM_RELATED);
        if (!skip) {
            REAL dist = v.dnd[i];
            REAL raw_depth = v.rdep[ix<ONE>(i, m, v.M)];
            REAL depth = fmax(raw_depth, (REAL)0.01);
            REAL dt = v.cfl_alpha * dist / sqrt(v.g * depth);
            if (v.max_dt > (REAL)0) dt = fmin(dt, v.max_dt);
            REAL outer_dt = v.outer[0];
            REAL dt_clamped = fmin(dt, outer_dt);
            n_steps = (int)(floor(outer_dt / dt_clamped - (REAL)0.01) + (REAL)1.0);
        }
    }
    if (ONE) {
        // warp then block max, one atomic per block (max is order-free)
        for (int o = 16; o > 0; o >>= 1) n_steps = max(n_steps, __shfl_down_sync(0xffffffffu, n_steps, o));
        __shared__ int part[32];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) part[warp] = n_steps;
        __syncthreads();
        if (warp == 0) {
            int x = lane < (int)((blockDim.x + 31) >> 5) ? part[lane] : 0;
            for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_down_sync(0xffffffffu, x, o));
            if (lane == 0 && x > 0) atomicMax(&v.nsub[0], x);
        }
    } else if (v.M <= (int)blockDim.x) {
        // per-member maximum inside the block (shared-memory atomics), then
        // one global atomic per member and block
        __shared__ int smax[kMaxBlock];
        if ((int)threadIdx.x < v.M) smax[threadIdx.x] = 0;
        __syncthreads();
        if (t < v.N * (long)v.M) atomicMax(&smax[m], n_steps);
        __syncthreads();
        if ((int)threadIdx.x < v.M && smax[threadIdx.x] > 0)
            atomicMax(&v.nsub[threadIdx.x], smax[threadIdx.x]);
    } else {
        if (t < v.N * (long)v.M) atomicMax(&v.nsub[m], n_steps);
    }
}

// Interval prologue: outer step, clear counters.
template <typename REAL>
__global__ void k_interval_begin(const Dev<REAL> v, double outer_seconds, int adaptive)
{
    const int m = threadIdx.x;
    if (m == 0) {
        v.tsec[0] = outer_seconds;
        v.outer[0] = (REAL)outer_seconds;
        v.ctl[kCtlStep] = 0;
        v.ctl[kCtlBlocksDone] = 0;
    }
    for (int q = m; q < v.M; q += blockDim.x)
        if (adaptive) v.nsub[q] = 0;
}

// After the CFL: dt = T / n per member, loop bound, while-condition.
template <typename REAL>
__global__ void k_interval_plan(const Dev<REAL> v, int fixed_n, cudaGraphConditionalHandle h,
                                int set_cond)
{
    __shared__ int smax;
    if (threadIdx.x == 0) smax = 0;
    __syncthreads();
    const double T = v.tsec[0];
    for (int m = threadIdx.x; m < v.M; m += blockDim.x) {
        int n = fixed_n > 0 ? fixed_n : v.nsub[m];
        if (n < 1) n = 1;
        // A non-finite depth makes the CFL count meaningless (NaN -> int is
        // undefined); the hard cap keeps the device-side loop bounded.
        const int cap = v.max_sub_cap > 0 ? v.max_sub_cap : kHardSubStepCap;
        if (n > cap) {
            atomicOr(v.status, CMF_STATUS_SUBSTEP_CAP);
            n = cap;
        }
        v.nsub[m] = n;
        v.dt[m] = (REAL)(T / (double)n);
        atomicMax(&smax, n);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        v.ctl[kCtlMaxSteps] = smax;
        v.ctl[kCtlStep] = 0;
        if (set_cond) cudaGraphSetConditional(h, smax > 0 ? 1u : 0u);
    }
}

// Interval epilogue: storage buffers whose member ran an odd number of
// sub-steps hold the state in the second buffer; copy it back.
template <typename REAL, bool ONE>
__global__ void __launch_bounds__(256) k_interval_end(const Dev<REAL> v)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.N * (long)v.M) return;
    int m;
    split_member<ONE>(v, t, m);
    if (v.nsub[m] & 1) {
        v.rs0[t] = v.rs1[t];
        v.fs0[t] = v.fs1[t];
    }
    if (t == 0) v.cur[0] = v.ctl[kCtlMaxSteps] - 1;
}

template <typename REAL, bool ONE>
__global__ void __launch_bounds__(256) k_copy_back(const Dev<REAL> v)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.N * (long)v.M) return;
    v.rs0[t] = v.rs1[t];
    v.fs0[t] = v.fs1[t];
}

// Levee-indexed copies of the static fields k_levee reads (once per plan).
template <typename REAL>
__global__ void __launch_bounds__(256) k_levee_pack(const Dev<REAL> v)
{
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= v.NLV) return;
    const long ci = v.lci[l];
    v.lpk_ca[l] = v.ca[ci];
    for (int k = 0; k < v.K; ++k) v.lpk_tbl[l * (long)v.K + k] = v.tbl[ci * (long)v.K + k];
    if (v.lpk_geo) {
        v.lpk_geo[l] = v.rh[ci];
        v.lpk_geo[v.NLV + l] = v.rw[ci];
        v.lpk_geo[2 * v.NLV + l] = v.rl[ci];
    }
}

// Budget partials -> budget (fixed order), then clear partials.
__global__ void k_budget_flush(double* bpart, int nblocks, double* budget, const int* ctl,
                               int count_steps)
{
    __shared__ double red[256];
    for (int t = 0; t < kBudgetTerms; ++t) {
        double x = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
            x += bpart[(long)t * nblocks + b];
            bpart[(long)t * nblocks + b] = 0.0;
        }
        red[threadIdx.x] = x;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) budget[t] += red[0];
        __syncthreads();
    }
    if (threadIdx.x == 0 && count_steps) budget[CMF_BUDGET_SUBSTEPS] += (double)ctl[kCtlMaxSteps];
}

// ---------------------------------------------------------------------------
// Output statistics (the reference's variables_to_save), folded in after each
// sub-step by one elementwise kernel at the end of the sub-step.
// ---------------------------------------------------------------------------
struct StatsArgs {
    int count;
    int need_weight;
    int var[CMF_MAX_STATISTICS];
    int op[CMF_MAX_STATISTICS];
    double* out[CMF_MAX_STATISTICS];
    double* weight;
};

// Value of a statistics variable at element t.  `after` selects the storage
// buffer: the state after sub-step k (k >= 0, the ping-pong destination of
// k) or the interval state (k < 0, after k_interval_end).  Cells without a
// levee carry protected depth == flood depth (k_stage writes that only on the
// member's last sub-step, so it is taken from the flood depth here).
template <typename REAL>
__device__ __forceinline__ double stat_value(const Dev<REAL>& v, int var, long t, long i, int k)
{
    const bool second = k >= 0 && !(k & 1);
    switch (var) {
    case CMF_VAR_RIVER_OUTFLOW: return (double)v.rout[t];
    case CMF_VAR_FLOOD_OUTFLOW: return (double)v.fout[t];
    case CMF_VAR_TOTAL_OUTFLOW: return __dadd_rn((double)v.rout[t], (double)v.fout[t]);
    case CMF_VAR_RIVER_DEPTH: return (double)v.rdep[t];
    case CMF_VAR_FLOOD_DEPTH: return (double)v.fdep[t];
    case CMF_VAR_FLOOD_FRACTION: return (double)v.ffr[t];
    case CMF_VAR_PROTECTED_DEPTH:
        return (v.flags[i] & CMF_CELL_LEVEE) ? (double)v.pdep[t] : (double)v.fdep[t];
    case CMF_VAR_RIVER_STORAGE: return second ? v.rs1[t] : v.rs0[t];
    case CMF_VAR_FLOOD_STORAGE: return second ? v.fs1[t] : v.fs0[t];
    case CMF_VAR_PROTECTED_STORAGE: return (v.flags[i] & CMF_CELL_LEVEE) ? v.ps[t] : 0.0;
    default: return 0.0;
    }
}

// kh >= 0: host step index; kh == -1: the step that the last kernel of the
// sub-step just finished (the device counter was advanced by it).
template <typename REAL, bool ONE>
__global__ void __launch_bounds__(256) k_stats_accumulate(const Dev<REAL> v, const StatsArgs a, int kh)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.N * (long)v.M) return;
    int m;
    const long i = split_member<ONE>(v, t, m);
    const int k = kh >= 0 ? kh : v.ctl[kCtlStep] - 1;
    if (k >= v.nsub[m]) return;  // member idle in this sub-step
    const double dt = (double)v.dt[m];
    if (a.need_weight && i == 0) a.weight[m] = __dadd_rn(a.weight[m], dt);
#pragma unroll 1
    for (int q = 0; q < a.count; ++q) {
        const int op = a.op[q];
        if (op == CMF_STAT_LAST) continue;
        const double x = stat_value(v, a.var[q], t, i, k);
        double* o = a.out[q] + t;
        const double acc = *o;
        if (op == CMF_STAT_MEAN) *o = __dadd_rn(acc, __dmul_rn(x, dt));
        else if (op == CMF_STAT_MAX) *o = (x > acc || x != x) ? x : acc;
        else *o = (x < acc || x != x) ? x : acc;
    }
}

template <typename REAL, bool ONE>
__global__ void __launch_bounds__(256) k_stats_reset(const Dev<REAL> v, const StatsArgs a)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < v.M && a.weight) a.weight[t] = 0.0;
    if (t >= v.N * (long)v.M) return;
    for (int q = 0; q < a.count; ++q) {
        const int op = a.op[q];
        a.out[q][t] = op == CMF_STAT_MAX ? -INFINITY : (op == CMF_STAT_MIN ? INFINITY : 0.0);
    }
}

template <typename REAL, bool ONE>
__global__ void __launch_bounds__(256) k_stats_finalize(const Dev<REAL> v, const StatsArgs a)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.N * (long)v.M) return;
    int m;
    const long i = split_member<ONE>(v, t, m);
    for (int q = 0; q < a.count; ++q) {
        const int op = a.op[q];
        if (op == CMF_STAT_MEAN) a.out[q][t] = a.out[q][t] / a.weight[m];
        else if (op == CMF_STAT_LAST) a.out[q][t] = stat_value(v, a.var[q], t, i, -1);
    }
}

}  // namespace cmf
