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
// of p are [up[p], up[p+1]) and no upstream index array exists.  This file
// holds the kernels' data movement (layout, gathers, member tiles, step
// control); the per-element physics is cmf_physics.cuh, whose rounded
// operation sequences are those of the reference kernels (cmfgpu/phys/cuda),
// so results match them bit for bit.  Storage is fp64 ("STO") and
// ping-pongs between two buffers inside an interval so the limiter can read
// pre-update storage of neighbours while cells update their own.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "cmfb200.h"
#include "cmf_physics.cuh"

// minimum resident 256-thread CTAs per SM (register caps) of the sub-step kernels;
// k_stage: 4 (64 registers, no spills)
// minimum resident 256-thread CTAs per SM of the persistent interval kernel
// (64 registers, the budget of k_stage, which it inlines)
#ifndef CMF_PERSIST_MIN_BLOCKS
#define CMF_PERSIST_MIN_BLOCKS 4
#endif
// k_stage: 5 CTAs (48 registers) for one fp32 member, which walks the
// floodplain row from memory (L1) instead of holding it in registers (234 ->
// 223 us per 6M sub-step); 4 CTAs (64 registers, the row in registers) for
// fp64 and for member-batched runs
#ifndef CMF_STAGE_MIN_BLOCKS
#define CMF_STAGE_MIN_BLOCKS(REAL, ONE) ((sizeof(REAL) == 4 && (ONE)) ? 5 : 4)
#endif
// whether a k_stage instantiation holds the floodplain row in registers
template <typename REAL, bool ONE>
__host__ __device__ constexpr bool stage_row_in_regs() { return !(sizeof(REAL) == 4 && ONE); }
// k_momentum: 8 CTAs (32 registers) for one fp32 member, where the few bytes
// it spills cost less than the occupancy they buy (182 -> 161 us per 6M
// sub-step); fp64 and member-batched variants would spill hundreds of bytes
#ifndef CMF_MOMENTUM_MIN_BLOCKS
#define CMF_MOMENTUM_MIN_BLOCKS(REAL, ONE) ((sizeof(REAL) == 4 && (ONE)) ? 8 : 1)
#endif

namespace cmf {

constexpr int kMaxBifLevels = 8;
constexpr int kRowRegs = 10;         // floodplain levels held in registers (the CaMa layout)
// Upstream cells gathered with independent loads per loop trip: 4 for one
// member, whose lanes hold different cells with different upstream counts;
// 1 with members, where the lanes of a warp row share the cell and a
// predicated-off trip would only cost issue slots.
#ifndef CMF_CHILD_UNROLL_BATCHED
#define CMF_CHILD_UNROLL_BATCHED 1
#endif
constexpr int kChildUnroll = 4;
template <bool ONE>
__host__ __device__ constexpr int child_unroll() { return ONE ? kChildUnroll : CMF_CHILD_UNROLL_BATCHED; }
constexpr int kMaxBlock = 256;       // threads per CTA (kernels use __launch_bounds__(256))
constexpr int kBudgetTerms = CMF_BUDGET_TERMS;
// control words (Dev::ctl)
constexpr int kCtlStep = 0;       // current sub-step index k
constexpr int kCtlMaxSteps = 1;   // max over members of the sub-step count
constexpr int kCtlBlocksDone = 2; // last-block-done counter of k_stage
constexpr int kCtlBarrier = 4;    // [4..5]: arrival counter (u64) of the persistent kernel's grid barrier
constexpr int kCtlAbort = 6;      // set when a grid barrier gave up: every block leaves the interval
constexpr int kHardSubStepCap = 100000;  // bound of the device-side sub-step loop

// Two fluxes of one element stored together (river, floodplain): one 8-byte
// (fp32) or 16-byte (fp64) access instead of two.
template <typename REAL> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };
template <typename REAL> using pair_t = typename Pair<REAL>::type;

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
    pair_t<REAL>* qu;  // unlimited (river, floodplain) fluxes
    REAL* lrs;  // limit rate of the current sub-step, per cell x member
    // Levee-indexed copies, packed once per plan (null where the plan keeps
    // none): each levee cell's floodplain row [NLV][K] and, when members
    // share the river geometry, its river height, width, length [3][NLV] and
    // the levee's marks (LeveeMarks) [6][NLV]: base, crown, top and
    // first-layer storages, layer width step, levee distance.
    REAL* lpk_tbl;
    REAL* lpk_geo;
    REAL* lmk;
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
// k_momentum, cell part: a catchment's outflow over the sub-step
// (outflow.cu:21-175, reservoir.cu:18-94), from the physics of
// cmf_physics.cuh.  Writes the unlimited river and floodplain fluxes and the
// new interface state (flow depths, floodplain flow area).
// ---------------------------------------------------------------------------
template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF>
__device__ __forceinline__ void momentum_cell(const Dev<REAL>& v, long i, int m, int kh,
                                              int force_diag)
{
    const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, force_diag);
    if (!st.active) return;
    const double* __restrict__ rsrc = (st.k & 1) ? v.rs1 : v.rs0;
    const double* __restrict__ fsrc = (st.k & 1) ? v.fs1 : v.fs0;
    const int M = v.M;
    const long im = ix<ONE>(i, m, M);
    const REAL dt = v.dt[m];
    const REAL gdt = v.g * dt;
    const uint8_t fl = v.flags[i];
    const bool mouth = fl & CMF_CELL_MOUTH;
    const bool lev_cell = LEV && (fl & CMF_CELL_LEVEE);
    const bool res_cell = RES && (fl & CMF_CELL_RESERVOIR);
    const int dn = v.dn[i];
    const long dm = ix<ONE>(dn, m, M);

    const REAL width = par<ONE>(v.rw, CMF_BATCH_RIVER_WIDTH, v.batched, i, m, M);
    const REAL len = par<ONE>(v.rl, CMF_BATCH_RIVER_LENGTH, v.batched, i, m, M);
    const REAL bank_h = par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, i, m, M);
    const REAL n_riv = par<ONE>(v.rman, CMF_BATCH_RIVER_MANNING, v.batched, i, m, M);
    const REAL n_fld = par<ONE>(v.fman, CMF_BATCH_FLOOD_MANNING, v.batched, i, m, M);
    const REAL elev = v.celv[i];
    const REAL dx = v.dnd[i];
    const REAL q_riv_old = v.rout[im];
    const REAL q_fld_old = v.fout[im];
    const REAL h_riv = v.rdep[im];
    const REAL h_fld = v.fdep[im];
    const REAL hr_before = v.rcsd[im];
    const REAL hf_before = v.fcsd[im];
    const REAL af_before = v.fcsa[im];
    const REAL s_fld = (REAL)fsrc[im];

    // water surfaces: this cell's over its river bed; downstream the next
    // cell's, or the sea at this catchment's elevation for a mouth
    const REAL bed = elev - bank_h;
    const REAL eta = h_riv + bed;
    const REAL elev_dn = v.celv[dn];
    const REAL eta_dn = mouth ? elev
                              : v.rdep[dm] + (elev_dn - par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT,
                                                                 v.batched, dn, m, M));
    const REAL eta_top = smax(eta, eta_dn);
    const REAL slope = (eta - eta_dn) / dx;

    // interface state: river flow depth (the own depth at a mouth, whose sea
    // level sets the slope only), floodplain flow depth and flow area
    const REAL hr_now = mouth ? h_riv : eta_top - bed;
    const REAL hf_now = smax((mouth ? eta : eta_top) - elev, REAL(0));
    const REAL af_now = smax(s_fld / len - h_fld * width, REAL(0));
    const REAL hr_si = implicit_mean(hr_now, hr_before, REAL(1e-6));
    const REAL hf_si = implicit_mean(hf_now, hf_before, REAL(1e-6));

    REAL q_riv = REAL(0);
    if (hr_si > REAL(1e-5) && hr_now * width > REAL(1e-5))
        q_riv = channel_discharge(q_riv_old, width, n_riv, hr_si, slope, gdt);
    REAL q_fld = REAL(0);
    if (hf_si > REAL(1e-5) && af_now > REAL(1e-5)) {
        const REAL af_si = implicit_mean(af_now, smax(af_before, REAL(1e-6)), REAL(1e-6));
        q_fld = plain_discharge(q_fld_old, af_si, n_fld, hf_si, capped_slope(slope, REAL(0.005)), gdt);
    }
    // the floodplain never flows against the river
    if (q_riv * q_fld < REAL(0)) q_fld = REAL(0);

    // river storage, read only where a rule below needs it
    REAL s_riv = REAL(0);
    bool have_s_riv = false;
    auto river_store = [&]() -> REAL {
        if (!have_s_riv) {
            s_riv = (REAL)rsrc[im];
            have_s_riv = true;
        }
        return s_riv;
    };
    // backwater into the cell draws at most 5 % of what it holds per sub-step
    if (q_riv < REAL(0) && !mouth) {
        const REAL held = river_store() + s_fld + (lev_cell ? (REAL)v.ps[im] : REAL(0));
        const REAL rate = smin(REAL(0.05) * held / ((-q_riv - q_fld) * dt), REAL(1));
        q_riv *= rate;
        q_fld *= rate;
    }
    if (RES && (fl & CMF_CELL_DAM_UPSTREAM)) {
        const REAL bed_slope = smax((elev - elev_dn) / dx, v.min_kin);
        kinematic_outflow(bed_slope, len, h_riv, h_fld, river_store(), s_fld, width, n_riv, n_fld,
                          dt, q_riv, q_fld);
    }
    if (res_cell) {
        // the release replaces the routed flux; the limiter gathers fluxes,
        // so nothing scattered before needs undoing
        const int slot = v.rslot[i];
        const DamRule<REAL> rule{v.rcons[slot], v.radj[slot], v.remerg[slot],
                                 v.rnout[slot], v.raout[slot], v.rfcout[slot]};
        const REAL inflow = (REAL)v.rti[im] + par<ONE>(v.runoff, CMF_BATCH_RUNOFF, v.batched, i, m, M);
        q_riv = dam_release(rule, river_store() + s_fld, inflow, dt);
        q_fld = REAL(0);
    }

    v.qu[im] = {q_riv, q_fld};
    v.rcsd[im] = hr_now;
    v.fcsd[im] = hf_now;
    v.fcsa[im] = af_now;

    if (st.diag) {
        if (v.wse) v.wse[im] = eta;
        if (v.pwse) v.pwse[im] = lev_cell ? smin(elev + v.pdep[im], eta) : eta;
        if (v.tsto) {
            const REAL held = res_cell ? river_store() + s_fld
                                       : river_store() + s_fld + (lev_cell ? (REAL)v.ps[im] : REAL(0));
            v.tsto[im] = (double)held;
        }
    }
}

// ---------------------------------------------------------------------------
// k_momentum, path part: the level fluxes of a bifurcation path and its
// limiter (bifurcation.cu:21-129, levee.cu:263-341), from cmf_physics.cuh.
// ---------------------------------------------------------------------------

// The end-cell quantities a path reads: water-surface elevation, protected
// water surface (the levee's crown side, capped by the river surface) and
// total storage -- what the reference's outflow and reservoir kernels leave
// in its scratch fields.
template <typename REAL, bool ONE, bool RES, bool LEV>
__device__ __forceinline__ void path_end_state(const Dev<REAL>& v, const double* rsrc,
                                               const double* fsrc, int c, int m, REAL& eta,
                                               REAL& peta, REAL& store)
{
    const long cm = ix<ONE>(c, m, v.M);
    const uint8_t fl = v.flags[c];
    const REAL elev = v.celv[c];
    eta = v.rdep[cm] + (elev - par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, c, m, v.M));
    const bool lev_cell = LEV && (fl & CMF_CELL_LEVEE);
    peta = lev_cell ? smin(elev + v.pdep[cm], eta) : eta;
    const REAL held = (REAL)rsrc[cm] + (REAL)fsrc[cm];
    store = (RES && (fl & CMF_CELL_RESERVOIR)) ? held
                                               : held + (lev_cell ? (REAL)v.ps[cm] : REAL(0));
}

// Level fields of path p for member m, loaded on first use.
template <typename REAL, bool ONE>
struct PathLevelFields {
    const Dev<REAL>& v;
    long p;
    int m;
    __device__ long par_at(int l) const { return p * (long)v.L + l; }
    __device__ long state_at(int l) const { return ix<ONE>(par_at(l), m, v.M); }
    __device__ REAL sill(int l) const { return v.belv[par_at(l)]; }
    __device__ REAL width(int l) const { return v.bwid[par_at(l)]; }
    __device__ REAL manning(int l) const { return v.bman[par_at(l)]; }
    __device__ REAL flux(int l) const { return v.bout[state_at(l)]; }
    __device__ REAL depth(int l) const { return v.bcsd[state_at(l)]; }
    __device__ void new_depth(int l, REAL h) const { v.bcsd[state_at(l)] = h; }
};

template <typename REAL, bool ONE, bool RES, bool LEV>
__device__ __forceinline__ void momentum_path(const Dev<REAL>& v, long p, int m, int kh)
{
    const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, 2);
    if (!st.active) return;
    const double* rsrc = (st.k & 1) ? v.rs1 : v.rs0;
    const double* fsrc = (st.k & 1) ? v.fs1 : v.fs0;
    const REAL dt = v.dt[m];
    PathEnds<REAL> ends;
    path_end_state<REAL, ONE, RES, LEV>(v, rsrc, fsrc, v.bci[p], m, ends.eta_a, ends.peta_a,
                                        ends.store_a);
    path_end_state<REAL, ONE, RES, LEV>(v, rsrc, fsrc, v.bdi[p], m, ends.eta_b, ends.peta_b,
                                        ends.store_b);
    const PathLevelFields<REAL, ONE> lv{v, p, m};
    REAL flux[kMaxBifLevels];
    const REAL sum = path_level_fluxes<LEV>(lv, v.L, ends, v.blen[p], v.g * dt, flux);
    const REAL rate = path_rate(sum, ends.store_a, ends.store_b, dt);
    REAL moved = REAL(0);
#pragma unroll
    for (int l = 0; l < kMaxBifLevels; ++l) {
        if (l < v.L) {
            const REAL q = flux[l] * rate;
            v.bout[lv.state_at(l)] = q;
            moved += q;
        }
    }
    const long pm = ix<ONE>(p, m, v.M);
    v.bsum[pm] = sum * rate;
    v.braw[pm] = moved;
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
    constexpr int U = child_unroll<ONE>();
    for (int cb = c0; cb < c1; cb += U) {
        REAL nr[U], nf[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            if (cb + j < c1) {
                const long cm = ix<ONE>(cb + j, m, M);
                const pair_t<REAL> q = v.qu[cm];
                nr[j] = q.x;
                nf[j] = q.y;
            }
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
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
    const pair_t<REAL> q = v.qu[xm];
    REAL outgoing = outgoing_of<REAL, ONE, BIF>(v, x, m, ts, q.x, q.y);
    REAL rate_storage = (REAL)(rsrc[xm] + fsrc[xm]);
    return (outgoing > (REAL)1e-8) ? fmin(rate_storage / outgoing, (REAL)1.0) : (REAL)1.0;
}

// ---------------------------------------------------------------------------
// A catchment's floodplain profile for the flood stage: the catchment area
// and the table row, needed only by cells above their banks.  With REGS and
// the CaMa layout (kRowRegs levels) the row is held in registers and
// stage_cell starts its loads early for cells that were flooded before the
// sub-step; otherwise the walk reads the row from memory (L1) level by level,
// which leaves the single-member fp32 stage room for more resident CTAs.
// ---------------------------------------------------------------------------
template <typename REAL, bool REGS = true>
struct CellProfile {
    // REGS: the CaMa row (kRowRegs levels) is held in registers; otherwise
    // every level count walks the row in memory
    static constexpr bool kRegs = REGS;
    const Dev<REAL>* v;
    long i;
    REAL D[kRowRegs];
    REAL ca;
    bool loaded;

    __device__ void load()
    {
        const REAL* __restrict__ row = v->tbl + i * (long)kRowRegs;
        if (sizeof(REAL) == 4 && ((uintptr_t)row & 7) == 0) {
            const float2* r2 = reinterpret_cast<const float2*>(row);
#pragma unroll
            for (int q = 0; q < kRowRegs / 2; ++q) {
                const float2 x = __ldg(r2 + q);
                D[2 * q] = (REAL)x.x;
                D[2 * q + 1] = (REAL)x.y;
            }
        } else {
#pragma unroll
            for (int l = 0; l < kRowRegs; ++l) D[l] = __ldg(row + l);
        }
        ca = v->ca[i];
        loaded = true;
    }
    __device__ bool in_regs() const { return REGS && v->K == kRowRegs; }
    __device__ REAL area()
    {
        if (!in_regs()) return v->ca[i];
        if (!loaded) load();
        return ca;
    }
    __device__ FillLevel<REAL> walk(REAL S, REAL bank, REAL width, REAL len, REAL dw)
    {
        if (in_regs()) return fill_level_regs(D, S, bank, width, len, dw);
        return fill_level_mem(v->tbl + i * (long)v->K, v->K, S, bank, width, len, dw);
    }
};

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
    const pair_t<REAL> q_own = v.qu[im];
    const REAL qr = q_own.x, qf = q_own.y;
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
    CellProfile<REAL, stage_row_in_regs<REAL, ONE>()> prof;
    prof.v = &v;
    prof.i = i;
    prof.loaded = false;
    if (prof.in_regs() && fsto > 0.0) prof.load();

    // upstream inflow: gather the limited fluxes of the upstream cells, in
    // range order, child_unroll independent loads at a time
    double rin = 0.0, fin = 0.0, rti = 0.0;
    constexpr int U = child_unroll<ONE>();
    for (int cb = c0; cb < c1; cb += U) {
        REAL cr[U], cf[U], cl[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            if (cb + j < c1) {
                const long cm = ix<ONE>(cb + j, m, M);
                const pair_t<REAL> q = v.qu[cm];
                cr[j] = q.x;
                cf[j] = q.y;
                cl[j] = v.lrs[cm];
            }
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
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

    // continuity and flood stage; levee cells are re-partitioned afterwards
    // by k_levee, which conserves river + flood + protected storage, so the
    // budget's end storage is taken here
    const Continuity<double, REAL> c =
        continuity<double, REAL>(rsto, fsto, prot, (REAL)rin, rout, (REAL)fin, fout,
                                 BIF ? (REAL)gb : REAL(0), ro, ts);
    const StageOut<double, REAL> s = flood_stage_of(c.total, rw, rl, rh, v.K, prof);

    if (BUDGET) {
        const double pre = rsto + fsto + prot;
        const double raw_next = rsto + (double)c.d_river + fsto + (double)c.d_flood + prot
                                + (double)c.d_runoff;
        bud[CMF_BUDGET_RUNOFF_IN] += (double)c.d_runoff;
        bud[CMF_BUDGET_CLIP_GAIN] += c.total - raw_next;
        if (mouth) bud[CMF_BUDGET_MOUTH_OUT] += ((double)rout + (double)fout) * (double)ts;
        if (st.k == 0 || kh == -2) bud[CMF_BUDGET_STORAGE_START] += pre;
        if (st.diag) bud[CMF_BUDGET_STORAGE_END] += s.rs + s.fs;
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
__device__ __forceinline__ void limit_cell(const Dev<REAL>& v, long i, int m, int kh)
{
    const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, 2);
    if (!st.active) return;
    const int k = st.k;
    const double* rsrc = (k & 1) ? v.rs1 : v.rs0;
    const double* fsrc = (k & 1) ? v.fs1 : v.fs0;
    v.lrs[ix<ONE>(i, m, v.M)] = limit_rate_of<REAL, ONE, BIF>(v, rsrc, fsrc, i, m, v.dt[m]);
}

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
        limit_cell<REAL, ONE, BIF>(v, i, m, kh);
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
// One levee (list index li) of member m: re-partition of its cell's
// flood-stage result, as k_levee and the persistent interval kernel run it.
template <typename REAL, bool ONE>
__device__ __forceinline__ void levee_cell(const Dev<REAL>& v, long li, int m, int kh, int force_diag)
{
    const StepInfo st = step_info<ONE>(v.ctl, v.nsub, kh, m, force_diag);
    if (!st.active) return;
    const int k = st.k;
    double* rdst = (k & 1) ? v.rs0 : v.rs1;
    double* fdst = (k & 1) ? v.fs0 : v.fs1;
    const long ci = v.lci[li];
    const long cm = ix<ONE>(ci, m, v.M);
    // The cell's river and flood storage decide the regime; its depths and
    // flooded fraction are read only where a regime uses them (the flood
    // depth when overtopped) and written only where a regime changes them:
    // the scattered levee cells cost a sector per field touched.
    LeveeState<double, REAL> lst;
    lst.rs = rdst[cm];
    lst.fs = fdst[cm];
    lst.rdep = REAL(0);
    lst.fdep = REAL(0);
    lst.ffr = REAL(0);
    // static fields from the levee-indexed copies where the plan keeps
    // them (coalesced over the levee list), else from the cells
    const REAL* row = v.lpk_tbl ? v.lpk_tbl + li * (long)v.K : v.tbl + ci * (long)v.K;
    auto depth = [row](int l) { return row[l]; };
    REAL rh, rw, rl;
    if (v.lpk_geo) {
        rh = v.lpk_geo[li];
        rw = v.lpk_geo[v.NLV + li];
        rl = v.lpk_geo[2 * v.NLV + li];
    } else {
        rh = par<ONE>(v.rh, CMF_BATCH_RIVER_HEIGHT, v.batched, ci, m, v.M);
        rw = par<ONE>(v.rw, CMF_BATCH_RIVER_WIDTH, v.batched, ci, m, v.M);
        rl = par<ONE>(v.rl, CMF_BATCH_RIVER_LENGTH, v.batched, ci, m, v.M);
    }
    const REAL crown = v.lcrown[li], frac = v.lfrac[li], base = v.lbase[li];
    int regime;
    if (v.lmk) {
        // the plan's marks: the row is read only while the protected
        // side fills
        const long n = v.NLV;
        LeveeMarks<REAL, REAL> mk;
        mk.s_base = v.lmk[li];
        mk.s_crown = v.lmk[n + li];
        mk.s_top = v.lmk[2 * n + li];
        mk.s_first = v.lmk[3 * n + li];
        mk.dw = v.lmk[4 * n + li];
        mk.dist = v.lmk[5 * n + li];
        // the overtopped test of levee_apply, to fetch the flood depth it reads
        const REAL total = narrow<REAL>(lst.rs + lst.fs);
        const REAL bank = xmul(xmul(rl, rw), rh);
        if (total >= bank && total >= mk.s_crown) lst.fdep = v.fdep[cm];
        regime = levee_apply<0>(lst, mk, rw, rh, rl, crown, frac, base, v.K, depth);
    } else {
        lst.fdep = v.fdep[cm];
        regime = levee_partition<0>(lst, rw, rh, rl, v.ca[ci], crown, frac, base, v.K, depth);
    }
    v.ps[cm] = lst.ps;
    v.pdep[cm] = lst.pdep;
    if (regime == kLeveeOvertopped) {
        fdst[cm] = lst.fs;
    } else if (regime == kLeveeFilling || regime == kLeveeWedge) {
        rdst[cm] = lst.rs;
        fdst[cm] = lst.fs;
        v.rdep[cm] = lst.rdep;
        v.fdep[cm] = lst.fdep;
        v.ffr[cm] = lst.ffr;
    }
}

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
        levee_cell<REAL, ONE>(v, li, m, kh, force_diag);
    }
    if (kh == -1 && advance) advance_step(v.ctl, h, 1);
}

template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF, bool BUDGET>
__global__ void __launch_bounds__(256, CMF_STAGE_MIN_BLOCKS(REAL, ONE)) k_stage(const Dev<REAL> v, int kh, int force_diag,
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
// Persistent interval kernel (one member, no budget or statistics): every
// sub-step of a forcing interval in one cooperative launch.  The blocks walk
// the catchments, paths and levees in grid-stride loops and meet at a
// grid-wide barrier after each phase (momentum, limit rate, stage, levee),
// where the interval graph has a kernel boundary; the per-element work is
// the same device functions the four sub-step kernels call, with the step
// index passed explicitly.  On small networks the sub-step is a few
// microseconds of work, and a barrier costs less than a graph's kernel
// boundary.
//
// The barrier counts arrivals on a monotone 64-bit counter (reset by
// k_interval_plan): the b-th barrier of the launch completes when the counter
// reaches (b + 1) x gridDim.x.  All blocks are co-resident (cooperative
// launch), so every wait ends; each is still bounded in time, after which the
// block raises CMF_STATUS_SYNC_TIMEOUT and the abort flag, and every block
// leaves the interval at its next barrier.
// ---------------------------------------------------------------------------
constexpr unsigned long long kBarrierTimeoutNs = 1000000000ull;  // 1 s

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long load_acquire_u64(const unsigned long long* p)
{
    unsigned long long x;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(x) : "l"(p) : "memory");
    return x;
}

// false: the interval was abandoned (a barrier gave up); the caller returns.
__device__ __forceinline__ bool grid_barrier(int* ctl, int* status, unsigned long long& target,
                                             unsigned long long timeout_ns = kBarrierTimeoutNs,
                                             unsigned arrivals = 0)
{
    __shared__ int go_on;
    __syncthreads();
    target += arrivals ? arrivals : gridDim.x;
    if (threadIdx.x == 0) {
        unsigned long long* count = reinterpret_cast<unsigned long long*>(ctl + kCtlBarrier);
        volatile int* abort_flag = ctl + kCtlAbort;
        __threadfence();
        atomicAdd(count, 1ull);
        int ok = 1;
        const unsigned long long t0 = global_ns();
        while (load_acquire_u64(count) < target) {
            if (*abort_flag) { ok = 0; break; }
            if (global_ns() - t0 > timeout_ns) {
                atomicOr(status, CMF_STATUS_SYNC_TIMEOUT);
                atomicExch(ctl + kCtlAbort, 1);
                ok = 0;
                break;
            }
            __nanosleep(100);
        }
        __threadfence();
        go_on = ok;
    }
    __syncthreads();
    return go_on != 0;
}

template <typename REAL, bool RES, bool LEV, bool BIF>
__global__ void __launch_bounds__(256, CMF_PERSIST_MIN_BLOCKS) k_persistent(const Dev<REAL> v)
{
    const int n = v.ctl[kCtlMaxSteps];
    const long first = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long stride = (long)gridDim.x * blockDim.x;
    unsigned long long target = 0;
    double bud[kBudgetTerms];
    for (int k = 0; k < n; ++k) {
        for (long i = first; i < v.N; i += stride)
            momentum_cell<REAL, true, RES, LEV, BIF>(v, i, 0, k, 0);
        if (BIF)
            for (long p = first; p < v.P; p += stride) momentum_path<REAL, true, RES, LEV>(v, p, 0, k);
        if (!grid_barrier(v.ctl, v.status, target)) return;
        for (long i = first; i < v.N; i += stride) limit_cell<REAL, true, BIF>(v, i, 0, k);
        if (!grid_barrier(v.ctl, v.status, target)) return;
        for (long i = first; i < v.N; i += stride)
            stage_cell<REAL, true, RES, LEV, BIF, false>(v, i, 0, k, 0, bud);
        if (BIF)
            for (long p = first; p < v.P; p += stride) stage_path<REAL, true, BIF>(v, p, 0, k);
        if (!grid_barrier(v.ctl, v.status, target)) return;
        if (LEV) {
            for (long l = first; l < v.NLV; l += stride) levee_cell<REAL, true>(v, l, 0, k, 0);
            if (!grid_barrier(v.ctl, v.status, target)) return;
        }
    }
    if (first == 0) v.ctl[kCtlStep] = n;
}

// The barrier's give-up path, for a test: every block arrives once at a
// barrier that waits for one arrival more than the grid has, so each wait
// runs out after timeout_ns, raises CMF_STATUS_SYNC_TIMEOUT and the abort
// flag, and the kernel returns.
__global__ void k_barrier_timeout_probe(int* ctl, int* status, unsigned long long timeout_ns)
{
    unsigned long long target = 0;
    grid_barrier(ctl, status, target, timeout_ns, gridDim.x + 1);
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
        *reinterpret_cast<unsigned long long*>(v.ctl + kCtlBarrier) = 0ull;
        v.ctl[kCtlAbort] = 0;
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

// Levee-indexed copies of the static fields k_levee reads, and with a shared
// river geometry the levees' marks (levee_marks_of on the cell's row), once
// per plan.
template <typename REAL>
__global__ void __launch_bounds__(256) k_levee_pack(const Dev<REAL> v)
{
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= v.NLV) return;
    const long ci = v.lci[l];
    const REAL* row = v.tbl + ci * (long)v.K;
    for (int k = 0; k < v.K; ++k) v.lpk_tbl[l * (long)v.K + k] = row[k];
    if (v.lpk_geo) {
        v.lpk_geo[l] = v.rh[ci];
        v.lpk_geo[v.NLV + l] = v.rw[ci];
        v.lpk_geo[2 * v.NLV + l] = v.rl[ci];
    }
    if (v.lmk) {
        const LeveeMarks<REAL, REAL> mk =
            levee_marks_of<0>(v.rw[ci], v.rh[ci], v.rl[ci], v.ca[ci], v.lcrown[l], v.lfrac[l],
                              v.lbase[l], v.K, [row](int k) { return row[k]; });
        const long n = v.NLV;
        v.lmk[l] = mk.s_base;
        v.lmk[n + l] = mk.s_crown;
        v.lmk[2 * n + l] = mk.s_top;
        v.lmk[3 * n + l] = mk.s_first;
        v.lmk[4 * n + l] = mk.dw;
        v.lmk[5 * n + l] = mk.dist;
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
