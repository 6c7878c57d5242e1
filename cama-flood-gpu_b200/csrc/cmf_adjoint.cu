// Reverse-mode adjoint of the routing sub-step, fp64, all physics modules.
//
// The reference has no adjoint; this is the differentiable routing core the
// calibration path needs.  A forward sub-step k maps the state
//
//   X_k = (river/flood storage, river/flood outflow, river/flood depth,
//          river/flood cross-section depth, flood cross-section area,
//          protected storage, protected depth, reservoir total inflow;
//          per bifurcation path and level: outflow, cross-section depth)
//
// to X_{k+1} through phases that read neighbours (momentum reads the
// downstream depth; a path reads both end cells; the limiter and the stage
// read the upstream fluxes, the path sums and the limit rates).  The primal
// kernels here restate the product forward (cmf_device.cuh, REAL = double)
// with every intermediate kept, and a tape slot stores X_k with the
// sub-step's fluxes, limit rates and limited path fluxes.
//
// The reverse of one sub-step is up to eight kernels, each a gather: every scatter of
// the forward (inflow into the downstream cell, outgoing storage of the
// downstream cell, the downstream depth read by momentum, path fluxes into
// their end cells, reservoir inflow) becomes a gather over the contiguous
// upstream range of the breadth-first order or over the per-cell path CSR, so
// the adjoint is deterministic and atomic-free like the forward:
//
//   kr_levee       levee re-partition reversed over the levee list, one
//                  thread per levee and input direction;
//   kr_stage       flood stage and storage update reversed per cell, after
//                  the pending depth/storage adjoints that the later
//                  sub-step's momentum and path kernels left behind;
//   kr_stage_path  path inflow (net flux, level-flux scaling) reversed;
//   kr_limit       limit-rate and outgoing-storage adjoints;
//   kr_momentum    local-inertial momentum reversed per cell;
//   kr_dam         reservoir release and the dam-upstream kinematic flow
//                  reversed for the dam cells (trailing blocks of the
//                  kr_momentum launch, applied one sub-step later);
//   kr_path        path momentum reversed, one thread per path and input
//                  direction (trailing blocks of the kr_momentum launch).
//
// The long scalar branches -- reservoir release, dam-upstream kinematic flow,
// path momentum with its limiter, levee re-partition -- are templates on the
// scalar type.  The primal evaluates them on double; the reverse evaluates
// them on a forward-mode dual number, one input direction at a time, and
// contracts the Jacobian columns with the output adjoints.  The local-inertial
// momentum and the flood stage are reversed by hand.
//
// Subgradient convention (that of the PyTorch transcription used as the
// autograd oracle): clamp passes the gradient on its bounds, a two-operand
// max of the momentum splits it at a tie, a ternary routes it to the taken
// branch, max(sqrt(p), f) is differentiable only where p > f*f; in the
// templated branches fmax/fmin take the first operand on a tie and sqrt/cbrt
// have derivative 0 at 0.

#include "cmfb200.h"
#include "cmf_physics.cuh"

#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

// Minimum resident 256-thread CTAs per SM of the long primal and reverse
// kernels: 4 caps them at 64 registers.  They spill (kr_momentum most, ~0.4 KB
// to L1), but the extra occupancy hides more gather latency: over a 3-day
// window on the 250k full-physics network the reverse sub-step went from 299
// to 242 us and the forward from 70 to 67 us.  5 CTAs (48 registers) slowed
// both.
#ifndef CMF_ADJ_MIN_BLOCKS
#define CMF_ADJ_MIN_BLOCKS 4
#endif

// Programmatic dependent launch, for the reverse sweep (the forward chain
// measured slower with it: 67 -> 69.6 us per sub-step, against 236 -> 223 us
// for the reverse).  The sweep is a chain of dependent, latency-bound
// launches whose last wave is partly empty.  Each kernel lets
// the next one launch as soon as all of its own blocks are resident, so the
// next grid's blocks are scheduled during this one's tail; they then wait in
// hardware until this grid has completed and its writes are visible.  The
// dependents launch only after every block of the running grid has started,
// so they never hold back its blocks.  Kernels launched without the
// attribute (or after a kernel that does not trigger) just start after it.
#ifndef CMF_ADJ_PDL
#define CMF_ADJ_PDL 1
#endif
__device__ __forceinline__ void pdl_begin()
{
#if CMF_ADJ_PDL
    cudaTriggerProgrammaticLaunchCompletion();
    cudaGridDependencySynchronize();
#endif
}
#include <cuda_runtime.h>

namespace {

using namespace cmf;

// ---------------------------------------------------------------------------
// layout
// ---------------------------------------------------------------------------
enum CellField { F_RS = 0, F_FS, F_ROUT, F_FOUT, F_RDEP, F_FDEP, F_RCSD, F_FCSD, F_FCSA, F_PS,
                 F_PDEP, F_RTI, kCellState };
enum SlotExtra { F_QR = kCellState, F_QF, F_LR, kSlotCell };
// path area of a slot: [BOUT | BCSD | BLIM] x P*L, then [BSUM | BRAW] x P
enum PathField { PF_BOUT = 0, PF_BCSD, PF_BLIM };
// cell scratch of the reverse sweep
enum Scratch { S_RINB = 0, S_FINB, S_ROB, S_FOB, S_OGB, S_QRB, S_QFB, S_WDNB, S_GBB, S_RTIB,
               kCellScratch };
// path scratch: [LRCB | LRDB] x P, BLIMB x P*L, PEB x 6P
enum Grad { G_RMAN = 0, G_FMAN, G_RH, G_RW, kGradFields };

constexpr int kBlock = 256;
constexpr int kMaxLevels = 8;
constexpr int kDamDirs = 7;  // input directions of the dam-upstream kinematic flow
constexpr int kMaxFloodLevels = 16;
constexpr double kFloor = 1e-6;
constexpr double kFloor2 = 1e-6 * 1e-6;

// Dual numbers, the scalar operations and the per-element physics are shared
// with the forward kernels (cmf_scalar.cuh, cmf_physics.cuh).
template <typename T>
__device__ __forceinline__ T cnst(double x) { return T(x); }

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct Ctx {
    long N, P;
    int K, L;
    bool lev, res, bif;
    double g, alpha, max_dt, min_kin;
    const int* dn;
    const int* up;
    const uint8_t* flags;
    const double *rw, *rl, *rh, *celv, *ca, *dnd, *rman, *fman, *tbl;
    // levee (slot per cell, cell per slot)
    long NLV, R;
    const int* lslot;
    const int* lci;
    const int* rci;
    const double *lcrown, *lfrac, *lbase;
    // reservoir (slot per cell)
    const int* rslot;
    const double *rcons, *remerg, *radj, *rnout, *raout, *rfcout;
    // bifurcation
    const int *bptr, *bpaths, *bci, *bdi;
    const double *bman, *bwid, *blen, *belv;
    // dam cells (reservoir or dam-upstream), compact, and each cell's index
    // in that list (-1 elsewhere)
    long ND;
    const int* dam;
    const int* dam_slot;
    // slot geometry (doubles); lev_off: the pre-levee stage of the levee
    // cells [4][NLV] (river/flood storage, river/flood depth) that ka_levee
    // records in the slot of its sub-step for kr_levee
    long slot_len, path_off, lev_off;
    int grid_cells, grid_paths;
};

__device__ __forceinline__ int up_end(const Ctx& c, long x)
{
    const int e = c.up[x + 1];
    return (x + 1 < c.N && (c.flags[x + 1] & CMF_CELL_MOUTH)) ? e - 1 : e;
}

__device__ __forceinline__ double sgn(double x) { return (double)((x > 0.0) - (x < 0.0)); }

// path-area accessors of a slot
__device__ __forceinline__ double* pth(const Ctx& c, double* X, int f) { return X + c.path_off + (long)f * c.P * c.L; }
__device__ __forceinline__ const double* pth(const Ctx& c, const double* X, int f) { return X + c.path_off + (long)f * c.P * c.L; }
__device__ __forceinline__ double* bsum_of(const Ctx& c, double* X) { return X + c.path_off + 3L * c.P * c.L; }
__device__ __forceinline__ const double* bsum_of(const Ctx& c, const double* X) { return X + c.path_off + 3L * c.P * c.L; }
__device__ __forceinline__ double* braw_of(const Ctx& c, double* X) { return bsum_of(c, X) + c.P; }
__device__ __forceinline__ const double* braw_of(const Ctx& c, const double* X) { return bsum_of(c, X) + c.P; }

// ---------------------------------------------------------------------------
// templated scalar branches
// ---------------------------------------------------------------------------

// Reservoir release of a dam cell (dam_release, reservoir.cu:18-94).
template <typename T>
__device__ __forceinline__ T release(const Ctx& c, int slot, T rs, T fs, T total_inflow, T runoff_v,
                                     double time_step)
{
    const DamRule<double> rule{c.rcons[slot], c.radj[slot], c.remerg[slot],
                               c.rnout[slot], c.raout[slot], c.rfcout[slot]};
    return dam_release(rule, rs + fs, total_inflow + runoff_v, time_step);
}

// Kinematic flow of a cell right upstream of a dam (kinematic_outflow,
// outflow.cu:137-153); the bed slope depends on the geometry alone.
template <typename T>
__device__ __forceinline__ void kinematic(const Ctx& c, long i, T r_dep, T f_dep, T rs, T fs, T r_wid,
                                          T r_man, T f_man, double time_step, T& kin_riv, T& kin_fld)
{
    const int dn = c.dn[i];
    const double bed_slope = fmax((c.celv[i] - c.celv[dn]) / c.dnd[i], c.min_kin);
    kinematic_outflow(bed_slope, c.rl[i], r_dep, f_dep, rs, fs, r_wid, r_man, f_man, time_step,
                      kin_riv, kin_fld);
}

// Level fields of path p: the parameters from the plan, the previous flux
// and depth from the input vector of path_flux.
template <typename T>
struct InputPathLevels {
    const Ctx& c;
    long p;
    const T* in;
    T* depth_out;
    __device__ double sill(int l) const { return c.belv[p * c.L + l]; }
    __device__ double width(int l) const { return c.bwid[p * c.L + l]; }
    __device__ double manning(int l) const { return c.bman[p * c.L + l]; }
    __device__ T flux(int l) const { return in[6 + l]; }
    __device__ T depth(int l) const { return in[6 + c.L + l]; }
    __device__ void new_depth(int l, T h) const { depth_out[l] = h; }
};

// Path momentum with the path limiter (path_level_fluxes and path_rate,
// bifurcation.cu:21-129, levee.cu:263-341): in = (wse_c, wse_d, pwse_c,
// pwse_d, tot_c, tot_d, outflow[L], cross-section depth[L]); out = limited
// level fluxes, their limited sum and the new cross-section depths.
template <typename T>
__device__ __forceinline__ void path_flux(const Ctx& c, long p, const T* in, double time_step,
                                          T* blim, T& bsum, T* bcsd_new)
{
    const PathEnds<T> ends{in[0], in[1], in[2], in[3], in[4], in[5]};
    const InputPathLevels<T> lv{c, p, in, bcsd_new};
    T flux[kMaxLevels];
    const double gdt = c.g * time_step;
    const T sum = c.lev ? path_level_fluxes<true>(lv, c.L, ends, c.blen[p], gdt, flux)
                        : path_level_fluxes<false>(lv, c.L, ends, c.blen[p], gdt, flux);
    const T rate = path_rate(sum, ends.store_a, ends.store_b, time_step);
    bsum = sum * rate;
    for (int l = 0; l < c.L; ++l) blim[l] = flux[l] * rate;
}

// Levee re-partition of a levee cell after its flood stage (levee_partition,
// levee.cu:29-261).  in = (river storage, flood storage, river depth, flood
// depth), geometry = (river width, river height); out = (river, flood,
// protected storage, river, flood, protected depth); the flooded fraction
// passes through `ffr` (value only).  T is the scalar of everything the
// state reaches, G that of what depends on the geometry alone (the profile
// walks): a reverse pass along a state direction runs them on plain doubles.
template <typename T, typename G>
__device__ __forceinline__ void levee_part(const Ctx& c, long ci, const T* in, G rw, G rh,
                                           double& ffr, T* out)
{
    const int slot = c.lslot[ci];
    LeveeState<T, T> st;
    st.rs = in[0];
    st.fs = in[1];
    st.ps = T(0);
    st.rdep = in[2];
    st.fdep = in[3];
    st.pdep = T(0);
    st.ffr = T(ffr);
    const double* row = c.tbl + ci * (long)c.K;
    levee_partition<0>(st, rw, rh, c.rl[ci], c.ca[ci], c.lcrown[slot], c.lfrac[slot], c.lbase[slot],
                    c.K, [row](int l) { return row[l]; });
    out[0] = st.rs;
    out[1] = st.fs;
    out[2] = st.ps;
    out[3] = st.rdep;
    out[4] = st.fdep;
    out[5] = st.pdep;
    ffr = val(st.ffr);
}

// Contract the Jacobian of a templated branch with output adjoints:
// in_bar[j] += sum_o out_bar[o] * d out[o] / d in[j], one dual pass per input.
template <int NI, int NO, typename F>
__device__ __forceinline__ double vjp_column(const double* in, const double* out_bar, int j, F f)
{
    Dual x[NI];
    for (int q = 0; q < NI; ++q) x[q] = {in[q], q == j ? 1.0 : 0.0};
    Dual y[NO];
    f(x, y);
    double s = 0.0;
    for (int o = 0; o < NO; ++o) s += out_bar[o] * y[o].d;
    return s;
}

template <int NI, int NO, typename F>
__device__ __forceinline__ void vjp(const double* in, const double* out_bar, double* in_bar, F f)
{
    for (int j = 0; j < NI; ++j) in_bar[j] += vjp_column<NI, NO>(in, out_bar, j, f);
}

// ---------------------------------------------------------------------------
// Momentum primal with its intermediates (outflow.cu:21-135; the same
// operation order as momentum_cell with REAL = double).
// ---------------------------------------------------------------------------
struct Mom {
    bool mouth, rc, fc, zero_f, neg;
    int dn;
    double rw, rman, fman, rl, rout, fout, fdep, rcsd, fcsd, fcsa;
    double wse, wse_dn, slope, hr_now, P1, s1, hf_raw, hf_now, P2, s2, af_raw, af_now;
    double hr_si, hf_si, q, num, den, qr0_val, fc6, P3, s3, af_si, numf, denf, qf0_val;
    double qr0, qf0, qf1, tnf, lrn_raw, lrn, qr, qf;
};

__device__ __forceinline__ void mom_eval(const Ctx& c, const double* X, long i, double dt, Mom& m)
{
    const long N = c.N;
    m.mouth = c.flags[i] & CMF_CELL_MOUTH;
    m.dn = c.dn[i];
    m.rout = X[F_ROUT * N + i];
    m.rman = c.rman[i];
    const double r_dep = X[F_RDEP * N + i];
    m.rw = c.rw[i];
    m.rl = c.rl[i];
    const double r_hgt = c.rh[i];
    m.fout = X[F_FOUT * N + i];
    m.fman = c.fman[i];
    m.fdep = X[F_FDEP * N + i];
    const double c_elv = c.celv[i];
    const double dn_dist = c.dnd[i];
    m.rcsd = X[F_RCSD * N + i];
    m.fcsd = X[F_FCSD * N + i];
    m.fcsa = X[F_FCSA * N + i];
    const double fs = X[F_FS * N + i];

    // surfaces and interface state as momentum_cell forms them
    const double bed = c_elv - r_hgt;
    m.wse = r_dep + bed;
    m.wse_dn = m.mouth ? c_elv : X[F_RDEP * N + m.dn] + (c.celv[m.dn] - c.rh[m.dn]);
    const double top = fmax(m.wse, m.wse_dn);
    m.slope = (m.wse - m.wse_dn) / dn_dist;
    const double fslope = capped_slope(m.slope, 0.005);

    m.hr_now = m.mouth ? r_dep : top - bed;
    m.P1 = m.hr_now * m.rcsd;
    m.s1 = sqrt(m.P1);
    m.hr_si = fmax(m.s1, kFloor);
    m.hf_raw = (m.mouth ? m.wse : top) - c_elv;
    m.hf_now = fmax(m.hf_raw, 0.0);
    m.P2 = m.hf_now * m.fcsd;
    m.s2 = sqrt(m.P2);
    m.hf_si = fmax(m.s2, kFloor);
    m.af_raw = fs / m.rl - m.fdep * m.rw;
    m.af_now = fmax(m.af_raw, 0.0);

    // river channel: channel_discharge with its terms kept for the reverse
    m.rc = (m.hr_si > 1e-5) && (m.hr_now * m.rw > 1e-5);
    m.q = m.rout / m.rw;
    m.num = m.rw * (m.q + c.g * dt * m.hr_si * m.slope);
    m.den = 1.0 + c.g * dt * (m.rman * m.rman) * fabs(m.q)
            * (1.0 / (m.hr_si * m.hr_si * cbrt(m.hr_si)));
    m.qr0_val = m.num / m.den;
    m.qr0 = m.rc ? m.qr0_val : 0.0;

    m.fc = (m.hf_si > 1e-5) && (m.af_now > 1e-5);
    m.qf0 = 0.0;
    m.fc6 = fmax(m.fcsa, kFloor);
    m.P3 = m.af_now * m.fc6;
    m.s3 = sqrt(m.P3);
    m.af_si = fmax(m.s3, kFloor);
    m.numf = m.fout + c.g * dt * m.af_si * fslope;
    m.denf = 1.0 + c.g * dt * (m.fman * m.fman) * fabs(m.fout)
             * (1.0 / (m.hf_si * cbrt(m.hf_si))) / m.af_si;
    m.qf0_val = m.numf / m.denf;
    if (m.fc) m.qf0 = m.qf0_val;

    m.zero_f = (m.qr0 * m.qf0) < 0.0;
    m.qf1 = m.zero_f ? 0.0 : m.qf0;
    m.neg = (m.qr0 < 0.0) && !m.mouth;
    m.qr = m.qr0;
    m.qf = m.qf1;
    m.lrn = 1.0;
    m.lrn_raw = 1.0;
    m.tnf = 1.0;
    if (m.neg) {
        const double rs = X[F_RS * N + i];
        const double ps = X[F_PS * N + i];
        const double held = rs + fs + ps;
        m.tnf = (-m.qr0 - m.qf1) * dt;
        m.lrn_raw = 0.05 * held / m.tnf;
        m.lrn = fmin(m.lrn_raw, 1.0);
        m.qr = m.qr0 * m.lrn;
        m.qf = m.qf1 * m.lrn;
    }
}

// Final fluxes of a cell: momentum, then the dam-upstream and reservoir overrides.
__device__ __forceinline__ void cell_flux(const Ctx& c, const double* X, const double* runoff, long i,
                                          double dt, const Mom& m, double& qr, double& qf)
{
    const long N = c.N;
    qr = m.qr;
    qf = m.qf;
    if (!c.res) return;
    const uint8_t fl = c.flags[i];
    if (fl & CMF_CELL_DAM_UPSTREAM) {
        kinematic<double>(c, i, X[F_RDEP * N + i], X[F_FDEP * N + i], X[F_RS * N + i],
                          X[F_FS * N + i], c.rw[i], c.rman[i], c.fman[i], dt, qr, qf);
    }
    if (fl & CMF_CELL_RESERVOIR) {
        qr = release<double>(c, c.rslot[i], X[F_RS * N + i], X[F_FS * N + i], X[F_RTI * N + i],
                             runoff[i], dt);
        qf = 0.0;
    }
}

// End state of a path end cell: water-surface elevation, protected WSE and
// total storage (path_end_state of the product).
__device__ __forceinline__ void end_state(const Ctx& c, const double* X, int ci, double& wse,
                                          double& pwse, double& tot)
{
    const long N = c.N;
    const uint8_t fl = c.flags[ci];
    wse = X[F_RDEP * N + ci] + (c.celv[ci] - c.rh[ci]);
    pwse = wse;
    if (c.lev && (fl & CMF_CELL_LEVEE)) pwse = fmin(c.celv[ci] + X[F_PDEP * N + ci], wse);
    const double rs = X[F_RS * N + ci], fs = X[F_FS * N + ci];
    if (c.res && (fl & CMF_CELL_RESERVOIR)) tot = rs + fs;
    else tot = rs + fs + X[F_PS * N + ci];
}

__device__ __forceinline__ int path_inputs(const Ctx& c, const double* X, long p, double* in)
{
    const int ci = c.bci[p], di = c.bdi[p];
    end_state(c, X, ci, in[0], in[2], in[4]);
    end_state(c, X, di, in[1], in[3], in[5]);
    const int L = c.L;
    const double* bout = pth(c, X, PF_BOUT);
    const double* bcsd = pth(c, X, PF_BCSD);
    for (int lv = 0; lv < L; ++lv) {
        in[6 + lv] = bout[p * L + lv];
        in[6 + L + lv] = bcsd[p * L + lv];
    }
    return 6 + 2 * L;
}

// ---------------------------------------------------------------------------
// Flood stage primal (storage.cu:118-211) with the quantities its reverse needs.
// ---------------------------------------------------------------------------
struct Stage {
    bool flooded, top, cap_taken;
    int level;
    double rmax, winc, S_prev, D_prev, grad, W_tot, excess, arg, sq, diff_w, fdep, cap;
    double rs, fs, rdep, ffr;
};

__device__ __forceinline__ void stage_eval(const Ctx& c, long i, double total_s, double rh,
                                           double rw, double rl, Stage& s)
{
    s.rmax = rl * rw * rh;
    s.flooded = !(total_s <= s.rmax);
    s.top = false;
    s.cap_taken = false;
    s.level = 0;
    if (!s.flooded) {
        s.rs = total_s;
        s.fs = 0.0;
        s.rdep = total_s / (rl * rw);
        s.fdep = 0.0;
        s.ffr = 0.0;
        return;
    }
    const int K = c.K;
    const double ca = c.ca[i];
    s.winc = ca / rl / (double)K;
    // where the storage lies on the floodplain profile (fill_level_mem,
    // flood_surface), with the quantities the reverse needs kept
    const FillLevel<double> f = fill_level_mem(c.tbl + i * (long)K, K, total_s, s.rmax, rw, rl, s.winc);
    const FloodSurface<double> surf = flood_surface(f, K, total_s, rw, rl, s.winc);
    s.level = f.full;
    s.top = f.full == K;
    s.S_prev = f.s_top;
    s.D_prev = f.d_top;
    s.W_tot = surf.width_top;
    s.excess = total_s - f.s_top;
    s.diff_w = surf.extra_width;
    s.fdep = surf.depth;
    if (!s.top) {
        s.grad = (f.d_next - f.d_top) / s.winc;
        s.arg = s.W_tot * s.W_tot + 2.0 * s.excess / (s.grad * rl);
        s.sq = sqrt(s.arg);
    }
    s.cap = s.rmax + rl * rw * s.fdep;
    s.cap_taken = s.cap < total_s;
    const double river = s.cap_taken ? s.cap : total_s;
    s.rdep = river / (rl * rw);
    double ff = (s.W_tot + s.diff_w - rw) * rl / ca;
    ff = ff < 0.0 ? 0.0 : (ff > 1.0 ? 1.0 : ff);
    s.ffr = s.top ? 1.0 : ff;
    const double flood = total_s - river;
    s.rs = river;
    s.fs = flood < 0.0 ? 0.0 : flood;
}

// Reverse of stage_eval: output adjoints (river/flood storage, river/flood
// depth) -> total-storage adjoint, plus the river width/height gradients.
__device__ __forceinline__ double stage_reverse(const Stage& s, double tot, double rw, double rh,
                                                double rl, double L_rs, double L_fs, double L_rdep,
                                                double L_fdep, double& g_rw, double& g_rh)
{
    double tot_bar = 0.0;
    const double rlrw = rl * rw;
    const double rs_out_bar = L_rs + L_rdep / rlrw;       // rdep' = rs' / (rl rw)
    g_rw += -L_rdep * s.rdep / rw;
    if (!s.flooded) return tot_bar + rs_out_bar;
    double river_bar = rs_out_bar;
    if (!(tot - s.rs < 0.0)) {          // flood' = tot - river where that is >= 0
        tot_bar += L_fs;
        river_bar -= L_fs;
    }
    double cap_bar = 0.0;
    if (s.cap_taken) cap_bar = river_bar;
    else tot_bar += river_bar;
    double rmax_bar = cap_bar;
    g_rw += cap_bar * rl * s.fdep;
    const double fdep_bar = L_fdep + cap_bar * rlrw;
    double excess_bar, W_bar;
    if (s.top) {
        const double wr = s.W_tot * rl;
        excess_bar = fdep_bar / wr;
        W_bar = -fdep_bar * s.excess / (s.W_tot * wr);
    } else {
        const double dw_bar = fdep_bar * s.grad;
        const double arg_bar = dw_bar / (2.0 * s.sq);
        W_bar = arg_bar * 2.0 * s.W_tot - dw_bar;
        excess_bar = arg_bar * 2.0 / (s.grad * rl);
    }
    tot_bar += excess_bar;
    const double Sp_bar = -excess_bar;
    g_rw += W_bar;
    // S_prev = rmax + sum_{l < level} rl (W_{l-1} + W_l)/2 (H_l - H_{l-1}); the
    // river-width derivative of the layer sum telescopes to rl * H_{level-1}
    rmax_bar += Sp_bar;
    if (s.level > 0) g_rw += Sp_bar * rl * s.D_prev;
    g_rw += rmax_bar * rl * rh;
    g_rh += rmax_bar * rlrw;
    return tot_bar;
}

// Storage update (storage.cu:67-116) with its branch record.
struct Store {
    double rsu1, fsu1, rsu2, tt, total_next;
    double rin, fin, rti, gb, ur, uf;
};

// Inflow gather, own limited flux, reservoir inflow and bifurcation net flux.
__device__ __forceinline__ void gather_inflow(const Ctx& c, const double* X, long i, Store& t)
{
    const long N = c.N;
    const double lr_i = X[F_LR * N + i];
    const double qr = X[F_QR * N + i], qf = X[F_QF * N + i];
    const uint8_t fl = c.flags[i];
    const bool res_cell = c.res && (fl & CMF_CELL_RESERVOIR);
    double rin = 0.0, fin = 0.0, rti = 0.0;
    const int c0 = c.up[i], c1 = up_end(c, i);
    for (int u = c0; u < c1; ++u) {
        const double cr = X[F_QR * N + u], cf = X[F_QF * N + u], cl = X[F_LR * N + u];
        const double ur = (cr >= 0.0) ? cr * cl : cr * lr_i;
        const double uf = (cf >= 0.0) ? cf * cl : cf * lr_i;
        rin += ur;
        fin += uf;
        if (res_cell) rti += ur + uf;
    }
    const bool mouth = fl & CMF_CELL_MOUTH;
    const double lr_dn = mouth ? lr_i : X[F_LR * N + c.dn[i]];
    t.rin = rin;
    t.fin = fin;
    t.rti = rti;
    t.ur = (qr >= 0.0) ? qr * lr_i : qr * lr_dn;
    t.uf = (qf >= 0.0) ? qf * lr_i : qf * lr_dn;
    double gb = 0.0;
    if (c.bif && (fl & CMF_CELL_BIFURCATION)) {
        const double* braw = braw_of(c, X);
        for (int b = c.bptr[i]; b < c.bptr[i + 1]; ++b) {
            const int e = c.bpaths[b];
            const int p = e >> 1;
            const double raw = braw[p];
            const int other = (e & 1) ? c.bci[p] : c.bdi[p];
            const double lr_o = X[F_LR * N + other];
            const double lr_c = (e & 1) ? lr_o : lr_i;
            const double lr_d = (e & 1) ? lr_i : lr_o;
            const double net = (raw >= 0.0) ? raw * lr_c : raw * lr_d;
            gb += (e & 1) ? -net : net;
        }
    }
    t.gb = gb;
}

__device__ __forceinline__ double store_eval(double rsto, double fsto, double prot, double ro,
                                             double dt, Store& t)
{
    const double river_delta = (t.rin - t.ur) * dt;
    t.rsu1 = rsto + river_delta;
    const double flood_delta = (t.fin - t.uf - t.gb) * dt;
    t.fsu1 = fsto + (t.rsu1 < 0.0 ? t.rsu1 : 0.0) + flood_delta;
    t.rsu2 = t.rsu1 > 0.0 ? t.rsu1 : 0.0;
    double river_su = t.rsu2;
    t.tt = river_su + t.fsu1;
    if (t.fsu1 < 0.0) river_su = t.tt > 0.0 ? t.tt : 0.0;
    const double flood_su = t.fsu1 > 0.0 ? t.fsu1 : 0.0;
    const double external_delta = ro * dt;
    t.total_next = river_su + flood_su + prot + external_delta;
    return t.total_next > 0.0 ? t.total_next : 0.0;
}

// ---------------------------------------------------------------------------
// forward kernels (tape)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock, CMF_ADJ_MIN_BLOCKS) ka_momentum(const Ctx c, double* X, double* Y,
                                                      const double* runoff, double dt)
{
    if ((int)blockIdx.x >= c.grid_cells) {
        const long p = (long)(blockIdx.x - c.grid_cells) * blockDim.x + threadIdx.x;
        if (p >= c.P) return;
        double in[6 + 2 * kMaxLevels], blim[kMaxLevels], bcsd_new[kMaxLevels], bsum;
        path_inputs(c, X, p, in);
        path_flux<double>(c, p, in, dt, blim, bsum, bcsd_new);
        double* lim = pth(c, X, PF_BLIM);
        double* ncsd = pth(c, Y, PF_BCSD);
        double raw = 0.0;
        for (int lv = 0; lv < c.L; ++lv) {
            lim[p * c.L + lv] = blim[lv];
            ncsd[p * c.L + lv] = bcsd_new[lv];
            raw += blim[lv];
        }
        bsum_of(c, X)[p] = bsum;
        braw_of(c, X)[p] = raw;
        return;
    }
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    Mom m;
    mom_eval(c, X, i, dt, m);
    double qr, qf;
    cell_flux(c, X, runoff, i, dt, m, qr, qf);
    const long N = c.N;
    X[F_QR * N + i] = qr;
    X[F_QF * N + i] = qf;
    Y[F_RCSD * N + i] = m.hr_now;
    Y[F_FCSD * N + i] = m.hf_now;
    Y[F_FCSA * N + i] = m.af_now;
}

__device__ __forceinline__ double outgoing(const Ctx& c, const double* X, long i, double dt)
{
    const long N = c.N;
    const double qr = X[F_QR * N + i], qf = X[F_QF * N + i];
    double og = (fmax(qr, 0.0) + fmax(qf, 0.0)) * dt;
    const int c0 = c.up[i], c1 = up_end(c, i);
    for (int u = c0; u < c1; ++u) {
        const double neg = fmin(X[F_QR * N + u], 0.0) + fmin(X[F_QF * N + u], 0.0);
        og += -neg * dt;
    }
    if (c.bif && (c.flags[i] & CMF_CELL_BIFURCATION)) {
        const double* bsum = bsum_of(c, X);
        for (int b = c.bptr[i]; b < c.bptr[i + 1]; ++b) {
            const int e = c.bpaths[b];
            const double s = bsum[e >> 1];
            if (e & 1) og += -fmin(s, 0.0) * dt;
            else og += fmax(s, 0.0) * dt;
        }
    }
    return og;
}

__global__ void __launch_bounds__(kBlock) ka_limit(const Ctx c, double* X, double dt)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const long N = c.N;
    const double og = outgoing(c, X, i, dt);
    const double store = X[F_RS * N + i] + X[F_FS * N + i];
    X[F_LR * N + i] = (og > 1e-8) ? fmin(store / og, 1.0) : 1.0;
}

__global__ void __launch_bounds__(kBlock) ka_stage(const Ctx c, const double* X, double* Y,
                                                   const double* runoff, double dt)
{
    const long N = c.N;
    if ((int)blockIdx.x >= c.grid_cells) {
        const long p = (long)(blockIdx.x - c.grid_cells) * blockDim.x + threadIdx.x;
        if (p >= c.P) return;
        const double lr_c = X[F_LR * N + c.bci[p]], lr_d = X[F_LR * N + c.bdi[p]];
        const double* lim = pth(c, X, PF_BLIM);
        double* out = pth(c, Y, PF_BOUT);
        for (int lv = 0; lv < c.L; ++lv) {
            const double o = lim[p * c.L + lv];
            out[p * c.L + lv] = (o >= 0.0) ? o * lr_c : o * lr_d;
        }
        return;
    }
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const uint8_t fl = c.flags[i];
    Store t;
    gather_inflow(c, X, i, t);
    const double tot = store_eval(X[F_RS * N + i], X[F_FS * N + i], X[F_PS * N + i], runoff[i], dt, t);
    Stage s;
    stage_eval(c, i, tot, c.rh[i], c.rw[i], c.rl[i], s);
    // levee cells are re-partitioned afterwards by ka_levee
    Y[F_RS * N + i] = s.rs;
    Y[F_FS * N + i] = s.fs;
    Y[F_PS * N + i] = 0.0;
    Y[F_RDEP * N + i] = s.rdep;
    Y[F_FDEP * N + i] = s.fdep;
    Y[F_PDEP * N + i] = s.fdep;
    Y[F_ROUT * N + i] = t.ur;
    Y[F_FOUT * N + i] = t.uf;
    Y[F_RTI * N + i] = (c.res && (fl & CMF_CELL_RESERVOIR)) ? t.rti : 0.0;
}

// Levee re-partition of the levee cells (levee.cu:29-261) on the flood-stage
// result ka_stage left in Y, over the compact levee list.
__global__ void __launch_bounds__(kBlock, CMF_ADJ_MIN_BLOCKS) ka_levee(const Ctx c, double* X, double* Y)
{
    const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= c.NLV) return;
    const long N = c.N;
    const long i = c.lci[l];
    const double in[6] = {Y[F_RS * N + i], Y[F_FS * N + i], Y[F_RDEP * N + i], Y[F_FDEP * N + i],
                          c.rw[i], c.rh[i]};
    double* rec = X + c.lev_off;
#pragma unroll
    for (int k = 0; k < 4; ++k) rec[k * c.NLV + l] = in[k];
    double out[6], ffr = 0.0;
    levee_part<double, double>(c, i, in, in[4], in[5], ffr, out);
    Y[F_RS * N + i] = out[0];
    Y[F_FS * N + i] = out[1];
    Y[F_PS * N + i] = out[2];
    Y[F_RDEP * N + i] = out[3];
    Y[F_FDEP * N + i] = out[4];
    Y[F_PDEP * N + i] = out[5];
}

__global__ void __launch_bounds__(kBlock) ka_cfl(const Ctx c, const double* X, double outer,
                                                 int* n_out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int n_steps = 1;
    if (i < c.N && !(c.res && (c.flags[i] & CMF_CELL_DAM_RELATED))) {
        const double dist = c.dnd[i];
        const double depth = fmax(X[F_RDEP * c.N + i], 0.01);
        double dt = c.alpha * dist / sqrt(c.g * depth);
        if (c.max_dt > 0.0) dt = fmin(dt, c.max_dt);
        const double dt_clamped = fmin(dt, outer);
        n_steps = (int)(floor(outer / dt_clamped - 0.01) + 1.0);
    }
    for (int o = 16; o > 0; o >>= 1) n_steps = max(n_steps, __shfl_down_sync(0xffffffffu, n_steps, o));
    if ((threadIdx.x & 31) == 0) atomicMax(n_out, n_steps);
}

// ---------------------------------------------------------------------------
// reverse kernels
// ---------------------------------------------------------------------------
struct Adj {
    double* lam;      // adjoint of a state (cell fields, then path fields)
    double* grad;     // [kGradFields][N]
    double* groff;    // [N] runoff gradient of the current interval
    double* scr;      // cell scratch [kCellScratch][N], then path scratch
};

__device__ __forceinline__ double* lam_path(const Ctx& c, double* lam, int f)
{
    return lam + (long)kCellState * c.N + (long)f * c.P * c.L;
}
__device__ __forceinline__ double* pscr(const Ctx& c, double* scr) { return scr + (long)kCellScratch * c.N; }
// path scratch: LRCB [P], LRDB [P], BLIMB [P*L], BCSDB [P*L], PEB [8P];
// levee scratch: LEVB [6*NLV]
__device__ __forceinline__ double* lrcb(const Ctx& c, double* scr) { return pscr(c, scr); }
__device__ __forceinline__ double* lrdb(const Ctx& c, double* scr) { return pscr(c, scr) + c.P; }
__device__ __forceinline__ double* blimb(const Ctx& c, double* scr) { return pscr(c, scr) + 2 * c.P; }
__device__ __forceinline__ double* bcsdb(const Ctx& c, double* scr) { return pscr(c, scr) + 2 * c.P + c.P * c.L; }
__device__ __forceinline__ double* peb(const Ctx& c, double* scr) { return pscr(c, scr) + 2 * c.P + 2 * c.P * c.L; }
__device__ __forceinline__ double* levb(const Ctx& c, double* scr) { return peb(c, scr) + 8 * c.P; }
// dam scratch: the deferred dam adjoints, DAMB [ND][kDamDirs]
__device__ __forceinline__ double* damb(const Ctx& c, double* scr) { return levb(c, scr) + 6 * c.NLV; }

// Apply the adjoints the later sub-step's momentum (downstream depth) and path
// kernels (end states) left for cell i; returns nothing, updates lam / grad.
// The pending depth / end-state adjoints of cell i gathered from what the
// later sub-step's momentum and path reverses left in the scratch.
__device__ __forceinline__ void pending_sums(const Ctx& c, long i, const Adj& a, double& rdep_bar,
                                             double& pdep_bar, double& tot_bar)
{
    const long N = c.N;
    double wsum = 0.0;
    const int c0 = c.up[i], c1 = up_end(c, i);
    for (int u = c0; u < c1; ++u) wsum += a.scr[S_WDNB * N + u];
    rdep_bar = wsum;
    pdep_bar = 0.0;
    tot_bar = 0.0;
    const uint8_t fl = c.flags[i];
    if (c.bif && (fl & CMF_CELL_BIFURCATION)) {
        const double* pe = peb(c, a.scr);
        for (int b = c.bptr[i]; b < c.bptr[i + 1]; ++b) {
            const int e = c.bpaths[b];
            const double* q = pe + 8L * (e >> 1) + ((e & 1) ? 4 : 0);
            rdep_bar += q[0] + q[1];
            pdep_bar += q[2];
            tot_bar += q[3];
        }
    }
}

__device__ __forceinline__ void apply_pending(const Ctx& c, long i, const Adj& a)
{
    const long N = c.N;
    double* lam = a.lam;
    const uint8_t fl = c.flags[i];
    double rdep_bar, pdep_bar, tot_bar;
    pending_sums(c, i, a, rdep_bar, pdep_bar, tot_bar);
    lam[F_RDEP * N + i] += rdep_bar;
    a.grad[G_RH * N + i] -= rdep_bar;
    if (c.ND > 0 && (fl & (CMF_CELL_RESERVOIR | CMF_CELL_DAM_UPSTREAM))) {
        // what the later sub-step's dam reverse left for this cell
        const double* db = damb(c, a.scr) + (long)kDamDirs * c.dam_slot[i];
        if (fl & CMF_CELL_RESERVOIR) {
            lam[F_RS * N + i] += db[0];
            lam[F_FS * N + i] += db[1];
            lam[F_RTI * N + i] += db[2];
        } else {
            lam[F_RDEP * N + i] += db[0];
            lam[F_FDEP * N + i] += db[1];
            lam[F_RS * N + i] += db[2];
            lam[F_FS * N + i] += db[3];
            a.grad[G_RW * N + i] += db[4];
            a.grad[G_RMAN * N + i] += db[5];
            a.grad[G_FMAN * N + i] += db[6];
        }
    }
    if (pdep_bar != 0.0) lam[F_PDEP * N + i] += pdep_bar;
    if (tot_bar != 0.0) {
        lam[F_RS * N + i] += tot_bar;
        lam[F_FS * N + i] += tot_bar;
        if (!(c.res && (fl & CMF_CELL_RESERVOIR))) lam[F_PS * N + i] += tot_bar;
    }
}

// lambda_{k+1} of cell i's river/flood/protected storage and river/flood/
// protected depth with its pending terms added, in apply_pending's order,
// without writing them (kr_stage applies them).
__device__ __forceinline__ void pending_view(const Ctx& c, long i, const Adj& a, double (&q)[6])
{
    const long N = c.N;
    const double* lam = a.lam;
    const uint8_t fl = c.flags[i];
    double rdep_bar, pdep_bar, tot_bar;
    pending_sums(c, i, a, rdep_bar, pdep_bar, tot_bar);
    double rs = lam[F_RS * N + i], fs = lam[F_FS * N + i], ps = lam[F_PS * N + i];
    double rdep = lam[F_RDEP * N + i], fdep = lam[F_FDEP * N + i], pdep = lam[F_PDEP * N + i];
    rdep += rdep_bar;
    if (c.ND > 0 && (fl & (CMF_CELL_RESERVOIR | CMF_CELL_DAM_UPSTREAM))) {
        const double* db = damb(c, a.scr) + (long)kDamDirs * c.dam_slot[i];
        if (fl & CMF_CELL_RESERVOIR) {
            rs += db[0];
            fs += db[1];
        } else {
            rdep += db[0];
            fdep += db[1];
            rs += db[2];
            fs += db[3];
        }
    }
    if (pdep_bar != 0.0) pdep += pdep_bar;
    if (tot_bar != 0.0) {
        rs += tot_bar;
        fs += tot_bar;
        if (!(c.res && (fl & CMF_CELL_RESERVOIR))) ps += tot_bar;
    }
    q[0] = rs;
    q[1] = fs;
    q[2] = ps;
    q[3] = rdep;
    q[4] = fdep;
    q[5] = pdep;
}

// Levee re-partition reversed, over the levee list, before kr_stage: one dual
// pass per levee and input direction, on the flood-stage result from the tape
// and lambda_{k+1} of the outputs (with the pending terms, which kr_stage then
// applies), leaving the adjoints of the flood-stage outputs (and of river
// width/height) for kr_stage.  A compact kernel keeps the long dual passes
// out of the per-cell stage kernel.
__global__ void __launch_bounds__(kBlock, CMF_ADJ_MIN_BLOCKS) kr_levee(const Ctx c, const double* X, Adj a)
{
    pdl_begin();
    // threads [0, 4 NLV): the four state directions of each levee; then
    // [4 NLV, 6 NLV): the two geometry directions -- so that a warp runs one
    // instantiation of levee_part
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long nlv = c.NLV;
    if (t >= nlv * 6L) return;
    long l;
    int j;
    if (t < 4 * nlv) {
        l = t >> 2;
        j = (int)(t & 3);
    } else {
        const long u = t - 4 * nlv;
        l = u >> 1;
        j = 4 + (int)(u & 1);
    }
    const long i = c.lci[l];
    // the flood-stage result the levee re-partitioned (recorded by ka_levee)
    // and lambda_{k+1} of the outputs with their pending terms
    const double* rec = X + c.lev_off;
    double lb[6];
    pending_view(c, i, a, lb);
    Dual x[4], y[6];
    for (int k = 0; k < 4; ++k) x[k] = {rec[k * nlv + l], k == j ? 1.0 : 0.0};
    double ffr = 0.0;
    if (j < 4) {
        levee_part<Dual, double>(c, i, x, c.rw[i], c.rh[i], ffr, y);
    } else {
        const Dual rw = {c.rw[i], j == 4 ? 1.0 : 0.0}, rh = {c.rh[i], j == 5 ? 1.0 : 0.0};
        levee_part<Dual, Dual>(c, i, x, rw, rh, ffr, y);
    }
    double v = 0.0;
    for (int o = 0; o < 6; ++o) v += lb[o] * y[o].d;
    levb(c, a.scr)[6 * l + j] = v;
}

// Stage, levee and storage update reversed (kr_stage).
__global__ void __launch_bounds__(kBlock, CMF_ADJ_MIN_BLOCKS) kr_stage(const Ctx c, const double* X,
                                                   const double* runoff, double dt, Adj a)
{
    pdl_begin();
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const long N = c.N;
    double* lam = a.lam;
    double* scr = a.scr;
    const double rw = c.rw[i], rl = c.rl[i], rh = c.rh[i];
    const uint8_t fl = c.flags[i];
    const bool lev_cell = c.lev && (fl & CMF_CELL_LEVEE);
    const bool res_cell = c.res && (fl & CMF_CELL_RESERVOIR);

    apply_pending(c, i, a);
    double L_rs = lam[F_RS * N + i], L_fs = lam[F_FS * N + i];
    const double L_rout = lam[F_ROUT * N + i], L_fout = lam[F_FOUT * N + i];
    double L_rdep = lam[F_RDEP * N + i], L_fdep = lam[F_FDEP * N + i];
    const double L_pdep = lam[F_PDEP * N + i];   // protected storage' is 0 off levees
    const double L_rti = lam[F_RTI * N + i];
    double g_rh = 0.0, g_rw = 0.0;

    Store t;
    gather_inflow(c, X, i, t);
    const double rsto = X[F_RS * N + i], fsto = X[F_FS * N + i], prot = X[F_PS * N + i];
    const double tot = store_eval(rsto, fsto, prot, runoff[i], dt, t);
    Stage s;
    stage_eval(c, i, tot, rh, rw, rl, s);

    // ---- levee re-partition reverse (outputs -> flood-stage outputs), from kr_levee
    if (lev_cell) {
        const double* ib = levb(c, scr) + 6L * c.lslot[i];
        L_rs = ib[0];
        L_fs = ib[1];
        L_rdep = ib[2];
        L_fdep = ib[3];
        g_rw += ib[4];
        g_rh += ib[5];
    } else {
        L_fdep += L_pdep;   // protected depth = flood depth outside levees
    }

    // ---- flood stage reverse
    const double tot_bar = stage_reverse(s, tot, rw, rh, rl, L_rs, L_fs, L_rdep, L_fdep, g_rw, g_rh);

    // ---- storage update reverse
    const double tn_bar = t.total_next > 0.0 ? tot_bar : 0.0;
    const double rsu3_bar = tn_bar, fsu2_bar = tn_bar;
    a.groff[i] += tn_bar * dt;
    double fsu1_bar = t.fsu1 > 0.0 ? fsu2_bar : 0.0;
    double rsu2_bar = 0.0;
    if (t.fsu1 < 0.0) {
        if (t.tt > 0.0) {
            rsu2_bar += rsu3_bar;
            fsu1_bar += rsu3_bar;
        }
    } else {
        rsu2_bar += rsu3_bar;
    }
    double rsu1_bar = t.rsu1 > 0.0 ? rsu2_bar : 0.0;
    if (t.rsu1 < 0.0) rsu1_bar += fsu1_bar;

    lam[F_RS * N + i] = rsu1_bar;
    lam[F_FS * N + i] = fsu1_bar;
    lam[F_PS * N + i] = tn_bar;
    lam[F_PDEP * N + i] = 0.0;
    lam[F_RTI * N + i] = 0.0;
    scr[S_RINB * N + i] = rsu1_bar * dt;
    scr[S_FINB * N + i] = fsu1_bar * dt;
    scr[S_ROB * N + i] = L_rout - rsu1_bar * dt;
    scr[S_FOB * N + i] = L_fout - fsu1_bar * dt;
    scr[S_GBB * N + i] = -fsu1_bar * dt;
    scr[S_RTIB * N + i] = res_cell ? L_rti : 0.0;
    a.grad[G_RH * N + i] += g_rh;
    a.grad[G_RW * N + i] += g_rw;
}

// Path inflow reversed (kr_stage_path): net flux into the end cells and the
// limit-rate scaling of the level fluxes.
__global__ void __launch_bounds__(kBlock) kr_stage_path(const Ctx c, const double* X, Adj a)
{
    pdl_begin();
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= c.P) return;
    const long N = c.N;
    const int L = c.L;
    const int ci = c.bci[p], di = c.bdi[p];
    const double lr_c = X[F_LR * N + ci], lr_d = X[F_LR * N + di];
    const double raw = braw_of(c, X)[p];
    const double net_bar = a.scr[S_GBB * N + ci] - a.scr[S_GBB * N + di];
    double lrc_bar = 0.0, lrd_bar = 0.0;
    double raw_bar;
    if (raw >= 0.0) {
        raw_bar = net_bar * lr_c;
        lrc_bar += net_bar * raw;
    } else {
        raw_bar = net_bar * lr_d;
        lrd_bar += net_bar * raw;
    }
    const double* lim = pth(c, X, PF_BLIM);
    double* lb = lam_path(c, a.lam, PF_BOUT);
    double* bb = blimb(c, a.scr);
    for (int lv = 0; lv < L; ++lv) {
        const double o = lim[p * L + lv];
        const double lam_o = lb[p * L + lv];
        double ob = raw_bar;
        if (o >= 0.0) {
            ob += lam_o * lr_c;
            lrc_bar += lam_o * o;
        } else {
            ob += lam_o * lr_d;
            lrd_bar += lam_o * o;
        }
        bb[p * L + lv] = ob;
    }
    lrcb(c, a.scr)[p] = lrc_bar;
    lrdb(c, a.scr)[p] = lrd_bar;
    // lambda_{k+1} of the path cross-section depths, read by every direction
    // thread of kr_path while some of them write lambda_k in place
    const double* lc = lam_path(c, a.lam, PF_BCSD);
    double* cb = bcsdb(c, a.scr);
    for (int lv = 0; lv < L; ++lv) cb[p * L + lv] = lc[p * L + lv];
}

// Limit-rate adjoint (kr_limit).  u_j = q_j * (q_j >= 0 ? lr_j : lr_dn(j))
// enters the cell's own update (-u dt), its downstream inflow (+u dt) and, for
// a reservoir downstream, that reservoir's inflow record; lr_j collects the
// positive own fluxes, the negative fluxes of the upstream cells and the path
// terms of its bifurcation ends.
__global__ void __launch_bounds__(kBlock) kr_limit(const Ctx c, const double* X, double dt, Adj a)
{
    pdl_begin();
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= c.N) return;
    const long N = c.N;
    const double* scr = a.scr;
    const uint8_t fl = c.flags[j];
    const bool mouth = fl & CMF_CELL_MOUTH;
    const int dn = c.dn[j];
    const double qr = X[F_QR * N + j], qf = X[F_QF * N + j], lr = X[F_LR * N + j];
    const double lr_dn = mouth ? lr : X[F_LR * N + dn];
    const double rinb = scr[S_RINB * N + j], finb = scr[S_FINB * N + j];
    const double rtib = scr[S_RTIB * N + j];
    const double dn_r = mouth ? 0.0 : scr[S_RINB * N + dn] + scr[S_RTIB * N + dn];
    const double dn_f = mouth ? 0.0 : scr[S_FINB * N + dn] + scr[S_RTIB * N + dn];
    const double a_r = scr[S_ROB * N + j] + dn_r;
    const double a_f = scr[S_FOB * N + j] + dn_f;

    double lr_bar = 0.0;
    if (qr >= 0.0 || mouth) lr_bar += a_r * qr;
    if (qf >= 0.0 || mouth) lr_bar += a_f * qf;
    double qr_bar = a_r * ((qr >= 0.0) ? lr : lr_dn);
    double qf_bar = a_f * ((qf >= 0.0) ? lr : lr_dn);

    double og = (fmax(qr, 0.0) + fmax(qf, 0.0)) * dt;
    const int c0 = c.up[j], c1 = up_end(c, j);
    for (int u = c0; u < c1; ++u) {
        const double cr = X[F_QR * N + u], cf = X[F_QF * N + u];
        if (cr < 0.0) lr_bar += (scr[S_ROB * N + u] + rinb + rtib) * cr;
        if (cf < 0.0) lr_bar += (scr[S_FOB * N + u] + finb + rtib) * cf;
        og += -(fmin(cr, 0.0) + fmin(cf, 0.0)) * dt;
    }
    if (c.bif && (fl & CMF_CELL_BIFURCATION)) {
        const double* bsum = bsum_of(c, X);
        double* ps_ = a.scr + (long)kCellScratch * N;
        for (int b = c.bptr[j]; b < c.bptr[j + 1]; ++b) {
            const int e = c.bpaths[b];
            const int p = e >> 1;
            lr_bar += (e & 1) ? ps_[c.P + p] : ps_[p];
            const double s = bsum[p];
            if (e & 1) og += -fmin(s, 0.0) * dt;
            else og += fmax(s, 0.0) * dt;
        }
    }

    double og_bar = 0.0;
    if (og > 1e-8) {
        const double store = X[F_RS * N + j] + X[F_FS * N + j];
        const double ratio = store / og;
        if (ratio <= 1.0) {
            const double s_bar = lr_bar / og;
            og_bar = -lr_bar * ratio / og;
            a.lam[F_RS * N + j] += s_bar;
            a.lam[F_FS * N + j] += s_bar;
        }
    }
    if (qr >= 0.0) qr_bar += og_bar * dt;
    if (qf >= 0.0) qf_bar += og_bar * dt;
    a.scr[S_OGB * N + j] = og_bar;
    a.scr[S_QRB * N + j] = qr_bar;
    a.scr[S_QFB * N + j] = qf_bar;
}

// Path momentum reversed on dual numbers (the form built with
// CMF_ADJ_PATH_HAND=0, kept as the cross-check of path_reverse_hand): each
// thread takes kPathLanes of the
// path's input directions (6 end-state inputs and two per level) and
// evaluates the path flux once on DualN<kPathLanes> numbers seeded with
// them, so the primal part of the evaluation (roots, divisions, branches)
// runs once per kPathLanes directions; it writes each direction's adjoint:
// lambda_k of the path state, or an end-state adjoint left for the end cell.
// Runs as the trailing blocks of the kr_momentum launch: it reads the tape,
// the outgoing-storage adjoint of kr_limit and the path buffers of
// kr_stage_path, and writes only the path lambdas and the path-end buffer,
// none of which the momentum or dam reverse touches.  Two lanes: wider
// numbers spill under the launch's 64-register cap (measured on the 250k
// full-physics window, forward plus adjoint per sub-step: 247 us at 2 lanes,
// 253 at 4, 293 at 8, 265 with one direction per thread).
#ifndef CMF_ADJ_PATH_LANES
#define CMF_ADJ_PATH_LANES 2
#endif
constexpr int kPathLanes = CMF_ADJ_PATH_LANES;

__host__ __device__ constexpr int path_threads(int L) { return (6 + 2 * L + kPathLanes - 1) / kPathLanes; }

__device__ __forceinline__ void path_reverse(const Ctx& c, const double* X, double dt, const Adj& a,
                                             long t)
{
    const int L = c.L;
    const int NI = 6 + 2 * L;
    const int G = path_threads(L);
    if (t >= c.P * (long)G) return;
    const long p = t / G;
    const int j0 = (int)(t - p * G) * kPathLanes;
    const long N = c.N;
    const int ci = c.bci[p], di = c.bdi[p];
    using D = DualN<kPathLanes>;
    double in[6 + 2 * kMaxLevels];
    path_inputs(c, X, p, in);
    D x[6 + 2 * kMaxLevels];
    for (int q = 0; q < NI; ++q) {
        x[q] = D(in[q]);
        if (q >= j0 && q < j0 + kPathLanes) x[q].d[q - j0] = 1.0;
    }
    D blim[kMaxLevels], bcsd_new[kMaxLevels], bs;
    path_flux<D>(c, p, x, dt, blim, bs, bcsd_new);
    const double bsum = bsum_of(c, X)[p];
    double sb = 0.0;
    if (bsum >= 0.0) sb += a.scr[S_OGB * N + ci] * dt;
    if (bsum <= 0.0) sb -= a.scr[S_OGB * N + di] * dt;
    const double* bb = blimb(c, a.scr);
    const double* cb = bcsdb(c, a.scr);
#pragma unroll
    for (int k = 0; k < kPathLanes; ++k) {
        const int j = j0 + k;
        if (j >= NI) break;
        double v = sb * bs.d[k];
        for (int lv = 0; lv < L; ++lv)
            v += bb[p * L + lv] * blim[lv].d[k] + cb[p * L + lv] * bcsd_new[lv].d[k];
        if (j >= 6 + L) {
            lam_path(c, a.lam, PF_BCSD)[p * L + (j - 6 - L)] = v;
        } else if (j >= 6) {
            lam_path(c, a.lam, PF_BOUT)[p * L + (j - 6)] = v;
        } else {
            // end state: [wse, protected-WSE part on the WSE, protected depth, total storage]
            const int end = j & 1;
            double* q = peb(c, a.scr) + 8L * p + 4 * end;
            if (j < 2) {
                q[0] = v;
            } else if (j < 4) {
                const int e = end ? di : ci;
                bool to_pdep = false;
                if (c.lev && (c.flags[e] & CMF_CELL_LEVEE)) {
                    const double wse = X[F_RDEP * N + e] + (c.celv[e] - c.rh[e]);
                    to_pdep = c.celv[e] + X[F_PDEP * N + e] <= wse;
                }
                q[1] = to_pdep ? 0.0 : v;
                q[2] = to_pdep ? v : 0.0;
            } else {
                q[3] = v;
            }
        }
    }
}

// Path momentum reversed by hand (kr_path, one thread per path): the path
// flux of path_flux evaluated once on doubles with the quantities its
// reverse needs, then swept backwards.  It gives every input's adjoint in one
// pass, where the dual-number form needs one evaluation per kPathLanes
// directions.  Every branch is taken on the primal values exactly as the
// dual evaluation takes it, with the same subgradients: smax/smin pass the
// derivative of the first operand on a tie, square roots have derivative 0
// at 0, |x| has derivative sign(x), and a level whose semi-implicit depth is
// at most 1e-5 carries a constant zero flux.
#ifndef CMF_ADJ_PATH_HAND
#define CMF_ADJ_PATH_HAND 1
#endif

__device__ __forceinline__ void path_reverse_hand(const Ctx& c, const double* X, double dt,
                                                  const Adj& a, long p)
{
    if (p >= c.P) return;
    const int L = c.L;
    const long N = c.N;
    const int ci = c.bci[p], di = c.bdi[p];
    double in[6 + 2 * kMaxLevels];
    path_inputs(c, X, p, in);
    const double eta_a = in[0], eta_b = in[1], peta_a = in[2], peta_b = in[3];
    const double st_a = in[4], st_b = in[5];
    const double len = c.blen[p];
    const double gdt = c.g * dt;
    const double cap = 0.005;

    // forward, keeping what the reverse needs
    const bool top_a = eta_a >= eta_b;
    const double top = top_a ? eta_a : eta_b;
    const bool ptop_a = peta_a >= peta_b;
    const double ptop = c.lev ? (ptop_a ? peta_a : peta_b) : top;
    const double raw = (eta_a - eta_b) / len;
    const double t1 = raw >= -cap ? raw : -cap;
    const double slope = t1 <= cap ? t1 : cap;
    const bool slope_free = raw >= -cap && t1 <= cap;
    double q[kMaxLevels], h[kMaxLevels], hs[kMaxLevels];
    bool live[kMaxLevels], hpos[kMaxLevels];
    double sum = 0.0;
    for (int l = 0; l < L; ++l) {
        const double surface = (c.lev && l > 0) ? ptop : top;
        const double hraw = surface - c.belv[p * L + l];
        hpos[l] = hraw >= 0.0;
        h[l] = hpos[l] ? hraw : 0.0;
        double h_si;
        if (c.lev) {
            h_si = h[l];
            if (l == 0) {
                const double r = sqrt(h[l] * in[6 + L]);
                if (r > 0.0) h_si = r;
            }
        } else {
            const double r1 = sqrt(h[l] * in[6 + L + l]), r2 = sqrt(h[l] * 0.01);
            h_si = r1 >= r2 ? r1 : r2;
        }
        hs[l] = h_si;
        live[l] = h_si > 1e-5;
        q[l] = 0.0;
        if (live[l]) {
            const double B = c.bwid[p * L + l], n = c.bman[p * L + l];
            const double qq = in[6 + l] / B;
            const double drive = qq + gdt * h_si * slope;
            const double drag = 1.0 + gdt * (n * n) * fabs(qq) * (1.0 / (h_si * h_si * cbrt(h_si)));
            q[l] = B * drive / drag;
        }
        sum = sum + q[l];
    }
    const double moved = fabs(sum) * dt;
    const bool limited = moved > 0.0;
    const bool st_first = st_a <= st_b;
    const double smin_st = st_first ? st_a : st_b;
    double r0 = 1.0, rate = 1.0;
    if (limited) {
        r0 = 0.05 * smin_st / moved;
        rate = r0 <= 1.0 ? r0 : 1.0;
    }

    // output adjoints: the limited sum (through the end cells' outgoing
    // storage), each limited level flux and each new depth
    const double bsum_tape = bsum_of(c, X)[p];
    double g_sum = 0.0;
    if (bsum_tape >= 0.0) g_sum += a.scr[S_OGB * N + ci] * dt;
    if (bsum_tape <= 0.0) g_sum -= a.scr[S_OGB * N + di] * dt;
    const double* bb = blimb(c, a.scr);
    const double* cb = bcsdb(c, a.scr);

    // rate and sum
    double rate_bar = g_sum * sum;
    for (int l = 0; l < L; ++l) rate_bar += bb[p * L + l] * q[l];
    double sum_bar = g_sum * rate;
    double st_a_bar = 0.0, st_b_bar = 0.0;
    if (limited && r0 <= 1.0) {
        const double smin_bar = rate_bar * 0.05 / moved;
        const double moved_bar = -rate_bar * r0 / moved;
        if (st_first) st_a_bar += smin_bar;
        else st_b_bar += smin_bar;
        sum_bar += moved_bar * dt * (double)((sum > 0.0) - (sum < 0.0));
    }

    // levels
    double top_bar = 0.0, ptop_bar = 0.0, slope_bar = 0.0;
    double flux_bar[kMaxLevels], depth_bar[kMaxLevels];
    for (int l = 0; l < L; ++l) {
        flux_bar[l] = 0.0;
        depth_bar[l] = 0.0;
        double h_bar = cb[p * L + l];
        if (live[l]) {
            const double q_bar = bb[p * L + l] * rate + sum_bar;
            const double B = c.bwid[p * L + l], n = c.bman[p * L + l];
            const double h_si = hs[l];
            const double qq = in[6 + l] / B;
            const double inv = 1.0 / (h_si * h_si * cbrt(h_si));
            const double drive = qq + gdt * h_si * slope;
            const double drag = 1.0 + gdt * (n * n) * fabs(qq) * inv;
            const double out = B * drive / drag;
            const double drive_bar = q_bar / drag * B;
            const double drag_bar = -q_bar * out / drag;
            double qq_bar = drive_bar + drag_bar * gdt * (n * n) * (double)((qq > 0.0) - (qq < 0.0)) * inv;
            const double inv_bar = drag_bar * gdt * (n * n) * fabs(qq);
            double hsi_bar = drive_bar * gdt * slope + inv_bar * (-(7.0 / 3.0) * inv / h_si);
            slope_bar += drive_bar * gdt * h_si;
            flux_bar[l] = qq_bar / B;
            // semi-implicit depth
            if (c.lev) {
                if (l == 0) {
                    const double d0 = in[6 + L];
                    const double r = sqrt(h[l] * d0);
                    if (r > 0.0) {
                        const double arg_bar = hsi_bar / (2.0 * r);
                        h_bar += arg_bar * d0;
                        depth_bar[0] += arg_bar * h[l];
                    } else {
                        h_bar += hsi_bar;
                    }
                } else {
                    h_bar += hsi_bar;
                }
            } else {
                const double d = in[6 + L + l];
                const double r1 = sqrt(h[l] * d), r2 = sqrt(h[l] * 0.01);
                if (r1 >= r2) {
                    if (h[l] * d > 0.0) {
                        const double arg_bar = hsi_bar / (2.0 * r1);
                        h_bar += arg_bar * d;
                        depth_bar[l] += arg_bar * h[l];
                    }
                } else if (h[l] * 0.01 > 0.0) {
                    h_bar += hsi_bar / (2.0 * r2) * 0.01;
                }
            }
        }
        if (hpos[l]) {
            if (c.lev && l > 0) ptop_bar += h_bar;
            else top_bar += h_bar;
        }
    }

    // end states
    double in_bar[6] = {0.0, 0.0, 0.0, 0.0, st_a_bar, st_b_bar};
    if (top_a) in_bar[0] += top_bar;
    else in_bar[1] += top_bar;
    if (c.lev) {
        if (ptop_a) in_bar[2] += ptop_bar;
        else in_bar[3] += ptop_bar;
    } else {
        if (top_a) in_bar[0] += ptop_bar;
        else in_bar[1] += ptop_bar;
    }
    if (slope_free) {
        in_bar[0] += slope_bar / len;
        in_bar[1] -= slope_bar / len;
    }

    // write, as the dual-number form does
    for (int l = 0; l < L; ++l) {
        lam_path(c, a.lam, PF_BOUT)[p * L + l] = flux_bar[l];
        lam_path(c, a.lam, PF_BCSD)[p * L + l] = depth_bar[l];
    }
    for (int end = 0; end < 2; ++end) {
        double* qe = peb(c, a.scr) + 8L * p + 4 * end;
        qe[0] = in_bar[end];
        const double v = in_bar[2 + end];
        const int e = end ? di : ci;
        bool to_pdep = false;
        if (c.lev && (c.flags[e] & CMF_CELL_LEVEE)) {
            const double wse = X[F_RDEP * N + e] + (c.celv[e] - c.rh[e]);
            to_pdep = c.celv[e] + X[F_PDEP * N + e] <= wse;
        }
        qe[1] = to_pdep ? 0.0 : v;
        qe[2] = to_pdep ? v : 0.0;
        qe[3] = in_bar[4 + end];
    }
}

__host__ __device__ constexpr int path_reverse_threads(long, int L)
{
    return CMF_ADJ_PATH_HAND ? 1 : path_threads(L);
}

// Momentum reversed (kr_momentum): lambda_k of the cell, the downstream-depth
// adjoint left for the downstream cell, parameter gradients.
__device__ __forceinline__ void dam_reverse(const Ctx& c, const double* X, const double* runoff,
                                            double dt, const Adj& a, long t);

__global__ void __launch_bounds__(kBlock, CMF_ADJ_MIN_BLOCKS) kr_momentum(const Ctx c, const double* X,
                                                      const double* runoff, double dt, Adj a)
{
    pdl_begin();
    if ((int)blockIdx.x >= c.grid_cells) {
        // trailing blocks: path direction threads, then dam direction threads
        const long b = (long)blockIdx.x - c.grid_cells;
        const long pb = c.bif ? (c.P * path_reverse_threads(c.P, c.L) + kBlock - 1) / kBlock : 0;
        if (b < pb) {
            if (CMF_ADJ_PATH_HAND) path_reverse_hand(c, X, dt, a, b * blockDim.x + threadIdx.x);
            else path_reverse(c, X, dt, a, b * blockDim.x + threadIdx.x);
        }
        else dam_reverse(c, X, runoff, dt, a, (b - pb) * blockDim.x + threadIdx.x);
        return;
    }
    const long N = c.N;
    double* lam = a.lam;
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    Mom m;
    mom_eval(c, X, i, dt, m);
    const double Dg = c.g * dt;
    const uint8_t fl = c.flags[i];

    double qr_bar = a.scr[S_QRB * N + i];
    double qf_bar = a.scr[S_QFB * N + i];
    double qr_final, qf_final;
    cell_flux(c, X, runoff, i, dt, m, qr_final, qf_final);
    if (!m.mouth) {
        const double ogb_dn = a.scr[S_OGB * N + m.dn];
        if (qr_final <= 0.0) qr_bar += -ogb_dn * dt;
        if (qf_final <= 0.0) qf_bar += -ogb_dn * dt;
    }
    double hr_now_bar = lam[F_RCSD * N + i];
    double hf_now_bar = lam[F_FCSD * N + i];
    double af_now_bar = lam[F_FCSA * N + i];

    double rs_bar = 0.0, fs_bar = 0.0, ps_bar = 0.0, rout_bar = 0.0, fout_bar = 0.0, rdep_bar = 0.0;
    double fdep_bar = 0.0, rcsd_bar = 0.0, fcsd_bar = 0.0, fcsa_bar = 0.0;
    double g_rman = 0.0, g_fman = 0.0, g_rw = 0.0, relev_bar = 0.0;

    // the dam-upstream kinematic flow and the reservoir release replace the
    // flux of those cells; kr_dam reverses them
    if (c.res && (fl & (CMF_CELL_RESERVOIR | CMF_CELL_DAM_UPSTREAM))) {
        qr_bar = 0.0;
        qf_bar = 0.0;
    }

    // negative-flow limiter
    double qr0_bar = qr_bar, qf1_bar = qf_bar;
    if (m.neg) {
        qr0_bar = qr_bar * m.lrn;
        qf1_bar = qf_bar * m.lrn;
        const double lrn_bar = qr_bar * m.qr0 + qf_bar * m.qf1;
        if (m.lrn_raw <= 1.0) {
            const double tsf_bar = lrn_bar * 0.05 / m.tnf;
            const double tnf_bar = -lrn_bar * m.lrn_raw / m.tnf;
            rs_bar += tsf_bar;
            fs_bar += tsf_bar;
            ps_bar += tsf_bar;
            qr0_bar += -tnf_bar * dt;
            qf1_bar += -tnf_bar * dt;
        }
    }
    const double qf0_bar = m.zero_f ? 0.0 : qf1_bar;

    double slope_bar = 0.0, fslope_bar = 0.0, hr_si_bar = 0.0, hf_si_bar = 0.0;
    if (m.fc) {
        const double numf_bar = qf0_bar / m.denf;
        const double denf_bar = -qf0_bar * m.qf0_val / m.denf;
        fout_bar += numf_bar;
        double af_si_bar = numf_bar * Dg * fmin(fmax(m.slope, -0.005), 0.005);
        fslope_bar += numf_bar * Dg * m.af_si;
        const double af = fabs(m.fout);
        const double B = 1.0 / (m.hf_si * cbrt(m.hf_si));
        const double nf2 = m.fman * m.fman;
        const double T = Dg * nf2 * af * B / m.af_si;
        g_fman += denf_bar * Dg * 2.0 * m.fman * af * B / m.af_si;
        fout_bar += denf_bar * Dg * nf2 * B / m.af_si * sgn(m.fout);
        hf_si_bar += denf_bar * Dg * nf2 * af / m.af_si * (-(4.0 / 3.0) * B / m.hf_si);
        af_si_bar += denf_bar * (-T / m.af_si);
        if (m.P3 > kFloor2) {
            const double P3_bar = af_si_bar / (2.0 * m.s3);
            af_now_bar += P3_bar * m.fc6;
            if (m.fcsa >= kFloor) fcsa_bar += P3_bar * m.af_now;
        }
    }
    if (m.rc) {
        const double num_bar = qr0_bar / m.den;
        const double den_bar = -qr0_bar * m.qr0_val / m.den;
        g_rw += num_bar * (m.q + Dg * m.hr_si * m.slope);
        const double inner_bar = num_bar * m.rw;
        double q_bar = inner_bar;
        hr_si_bar += inner_bar * Dg * m.slope;
        slope_bar += inner_bar * Dg * m.hr_si;
        const double aq = fabs(m.q);
        const double Br = 1.0 / (m.hr_si * m.hr_si * cbrt(m.hr_si));
        const double n2 = m.rman * m.rman;
        g_rman += den_bar * Dg * 2.0 * m.rman * aq * Br;
        q_bar += den_bar * Dg * n2 * Br * sgn(m.q);
        hr_si_bar += den_bar * Dg * n2 * aq * (-(7.0 / 3.0) * Br / m.hr_si);
        rout_bar += q_bar / m.rw;
        g_rw += -q_bar * m.q / m.rw;
    }
    if (m.slope >= -0.005 && m.slope <= 0.005) slope_bar += fslope_bar;
    if (m.af_raw >= 0.0) {
        fs_bar += af_now_bar / m.rl;
        fdep_bar += -af_now_bar * m.rw;
        g_rw += -af_now_bar * m.fdep;
    }
    if (m.P2 > kFloor2) {
        const double P2_bar = hf_si_bar / (2.0 * m.s2);
        hf_now_bar += P2_bar * m.fcsd;
        fcsd_bar += P2_bar * m.hf_now;
    }
    double fsurf_bar = (m.hf_raw >= 0.0) ? hf_now_bar : 0.0;
    if (m.P1 > kFloor2) {
        const double P1_bar = hr_si_bar / (2.0 * m.s1);
        hr_now_bar += P1_bar * m.rcsd;
        rcsd_bar += P1_bar * m.hr_now;
    }
    double wse_bar = 0.0, wse_dn_bar = 0.0, mw_bar = 0.0;
    if (m.mouth) {
        rdep_bar += hr_now_bar;
        wse_bar += fsurf_bar;
    } else {
        mw_bar += hr_now_bar;
        relev_bar -= hr_now_bar;
        mw_bar += fsurf_bar;
    }
    wse_bar += slope_bar / c.dnd[i];
    wse_dn_bar -= slope_bar / c.dnd[i];
    if (m.wse > m.wse_dn) wse_bar += mw_bar;
    else if (m.wse < m.wse_dn) wse_dn_bar += mw_bar;
    else { wse_bar += 0.5 * mw_bar; wse_dn_bar += 0.5 * mw_bar; }
    rdep_bar += wse_bar;
    relev_bar += wse_bar;

    lam[F_RS * N + i] += rs_bar;
    lam[F_FS * N + i] += fs_bar;
    lam[F_PS * N + i] += ps_bar;
    lam[F_ROUT * N + i] = rout_bar;
    lam[F_FOUT * N + i] = fout_bar;
    lam[F_RDEP * N + i] = rdep_bar;
    lam[F_FDEP * N + i] = fdep_bar;
    lam[F_RCSD * N + i] = rcsd_bar;
    lam[F_FCSD * N + i] = fcsd_bar;
    lam[F_FCSA * N + i] = fcsa_bar;
    a.scr[S_WDNB * N + i] = m.mouth ? 0.0 : wse_dn_bar;
    a.grad[G_RMAN * N + i] += g_rman;
    a.grad[G_FMAN * N + i] += g_fman;
    a.grad[G_RH * N + i] += -relev_bar;
    a.grad[G_RW * N + i] += g_rw;
}

// Flux adjoints of a cell after kr_limit: the stage/limiter part plus the
// outgoing storage of its downstream cell.
__device__ __forceinline__ void flux_bars(const Ctx& c, const double* X, const Adj& a, long i,
                                          double dt, double& qr_bar, double& qf_bar)
{
    const long N = c.N;
    qr_bar = a.scr[S_QRB * N + i];
    qf_bar = a.scr[S_QFB * N + i];
    if (!(c.flags[i] & CMF_CELL_MOUTH)) {
        const double ogb_dn = a.scr[S_OGB * N + c.dn[i]];
        if (X[F_QR * N + i] <= 0.0) qr_bar += -ogb_dn * dt;
        if (X[F_QF * N + i] <= 0.0) qf_bar += -ogb_dn * dt;
    }
}

// Reservoir release and dam-upstream kinematic flow reversed (kr_dam), one
// thread per dam cell and input direction (one dual pass each), as trailing
// blocks of the kr_momentum launch.  kr_momentum writes the same cells'
// lambdas, so these adjoints go to the dam scratch instead and apply_pending
// adds them at the start of the earlier sub-step (before anything reads those
// lambdas); the runoff gradient, which kr_momentum never writes and which
// belongs to this sub-step's interval, is added at once.
__device__ __forceinline__ void dam_reverse(const Ctx& c, const double* X, const double* runoff,
                                            double dt, const Adj& a, long t)
{
    if (t >= c.ND * (long)kDamDirs) return;
    const long d = t / kDamDirs;
    const int j = (int)(t - d * kDamDirs);
    const long i = c.dam[d];
    const uint8_t fl = c.flags[i];
    const long N = c.N;
    double qr_bar, qf_bar;
    flux_bars(c, X, a, i, dt, qr_bar, qf_bar);
    double* db = damb(c, a.scr) + (long)kDamDirs * d;
    if (fl & CMF_CELL_RESERVOIR) {
        if (j >= 4) return;
        const double in[4] = {X[F_RS * N + i], X[F_FS * N + i], X[F_RTI * N + i], runoff[i]};
        const double ob[1] = {qr_bar};
        const int slot = c.rslot[i];
        const double ib = 0.0 + vjp_column<4, 1>(in, ob, j, [&](const Dual* x, Dual* y) {
            y[0] = release<Dual>(c, slot, x[0], x[1], x[2], x[3], dt);
        });
        if (j == 3) a.groff[i] += ib;
        else db[j] = ib;
    } else {
        const double in[7] = {X[F_RDEP * N + i], X[F_FDEP * N + i], X[F_RS * N + i],
                              X[F_FS * N + i], c.rw[i], c.rman[i], c.fman[i]};
        const double ob[2] = {qr_bar, qf_bar};
        db[j] = 0.0 + vjp_column<7, 2>(in, ob, j, [&](const Dual* x, Dual* y) {
            kinematic<Dual>(c, i, x[0], x[1], x[2], x[3], x[4], x[5], x[6], dt, y[0], y[1]);
        });
    }
}

// Apply the pending adjoints of the last reversed sub-step (end of the sweep).
__global__ void __launch_bounds__(kBlock) kr_finalize(const Ctx c, Adj a)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    apply_pending(c, i, a);
}

}  // namespace

namespace {
template <typename... KArgs, typename... Args>
void launch_dep(void (*kernel)(KArgs...), int grid, cudaStream_t s, Args... args)
{
    if (grid <= 0) return;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBlock);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = CMF_ADJ_PDL;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
}  // namespace

struct CmfAdjPlan {
    Ctx ctx;
    int grid;
    int* dam_list;  // device, ctx.ND entries
    int* dam_slot;  // device, N entries
};

namespace {

int launch_status()
{
    return cudaGetLastError() == cudaSuccess ? CMF_OK : CMF_ERR_CUDA;
}

long scratch_len(const Ctx& c)
{
    return (long)kCellScratch * c.N + 2 * c.P + 2 * c.P * c.L + 8 * c.P + 6 * c.NLV + kDamDirs * c.ND;
}

}  // namespace

extern "C" {

int cmf_adj_sizes(const CmfAdjPlan* plan, int64_t* state_len, int64_t* slot_len,
                  int64_t* scratch_doubles, int* grad_fields)
{
    if (!plan) return CMF_ERR_ARG;
    const Ctx& c = plan->ctx;
    if (state_len) *state_len = (int64_t)kCellState * c.N + 2 * c.P * c.L;
    if (slot_len) *slot_len = c.slot_len;
    if (scratch_doubles) *scratch_doubles = scratch_len(c);
    if (grad_fields) *grad_fields = kGradFields;
    return CMF_OK;
}

int cmf_adj_plan_create(const CmfView* v, CmfAdjPlan** out)
{
    if (!v || !out) return CMF_ERR_ARG;
    *out = nullptr;
    if (v->abi_version != CMF_ABI_VERSION) return CMF_ERR_ARG;
    if (!(v->features & CMF_FEAT_FP64)) return CMF_ERR_UNSUPPORTED;
    if (v->num_members != 1 || v->batched_mask != 0) return CMF_ERR_UNSUPPORTED;
    if (v->num_catchments < 1 || v->num_catchments > (1L << 31) - 2 || v->num_flood_levels < 1 ||
        v->num_flood_levels > kMaxFloodLevels)
        return CMF_ERR_ARG;
    const void* need[] = {v->downstream_idx, v->upstream_ptr, v->cell_flags, v->river_width,
                          v->river_length, v->river_height, v->catchment_elevation,
                          v->catchment_area, v->downstream_distance, v->river_manning,
                          v->flood_manning, v->flood_depth_table};
    for (const void* p : need)
        if (!p) return CMF_ERR_ARG;
    const bool lev = v->features & CMF_FEAT_LEVEE;
    const bool res = v->features & CMF_FEAT_RESERVOIR;
    const bool bif = v->features & CMF_FEAT_BIFURCATION;
    if (lev && (!v->levee_slot || !v->levee_catchment_idx || !v->levee_crown_height || !v->levee_fraction ||
                !v->levee_base_height))
        return CMF_ERR_ARG;
    if (res && (!v->reservoir_slot || !v->reservoir_catchment_idx || !v->conservation_volume || !v->emergency_volume ||
                !v->adjustment_volume || !v->effective_normal_outflow ||
                !v->adjustment_outflow || !v->flood_control_outflow))
        return CMF_ERR_ARG;
    if (bif && (!v->bif_cell_ptr || !v->bif_cell_paths || !v->bifurcation_catchment_idx ||
                !v->bifurcation_downstream_idx || !v->bifurcation_manning ||
                !v->bifurcation_width || !v->bifurcation_length || !v->bifurcation_elevation ||
                v->num_bifurcation_levels < 1 || v->num_bifurcation_levels > kMaxLevels))
        return CMF_ERR_ARG;
    CmfAdjPlan* p = new (std::nothrow) CmfAdjPlan;
    if (!p) return CMF_ERR_ARG;
    std::memset(p, 0, sizeof(CmfAdjPlan));
    Ctx& c = p->ctx;
    c.N = v->num_catchments;
    c.K = v->num_flood_levels;
    c.lev = lev;
    c.res = res;
    c.bif = bif;
    c.P = bif ? v->num_bifurcation_paths : 0;
    c.L = bif ? v->num_bifurcation_levels : 0;
    c.g = v->gravity;
    c.alpha = v->adaptive_time_factor;
    c.max_dt = v->max_sub_step_seconds;
    c.min_kin = v->min_kinematic_slope;
    c.dn = static_cast<const int*>(v->downstream_idx);
    c.up = static_cast<const int*>(v->upstream_ptr);
    c.flags = static_cast<const uint8_t*>(v->cell_flags);
    c.rw = static_cast<const double*>(v->river_width);
    c.rl = static_cast<const double*>(v->river_length);
    c.rh = static_cast<const double*>(v->river_height);
    c.celv = static_cast<const double*>(v->catchment_elevation);
    c.ca = static_cast<const double*>(v->catchment_area);
    c.dnd = static_cast<const double*>(v->downstream_distance);
    c.rman = static_cast<const double*>(v->river_manning);
    c.fman = static_cast<const double*>(v->flood_manning);
    c.tbl = static_cast<const double*>(v->flood_depth_table);
    if (lev) {
        c.NLV = v->num_levees;
        c.lci = v->levee_catchment_idx;
        c.lslot = v->levee_slot;
        c.lcrown = static_cast<const double*>(v->levee_crown_height);
        c.lfrac = static_cast<const double*>(v->levee_fraction);
        c.lbase = static_cast<const double*>(v->levee_base_height);
    }
    if (res) {
        c.R = v->num_reservoirs;
        c.rci = v->reservoir_catchment_idx;
        c.rslot = v->reservoir_slot;
        c.rcons = static_cast<const double*>(v->conservation_volume);
        c.remerg = static_cast<const double*>(v->emergency_volume);
        c.radj = static_cast<const double*>(v->adjustment_volume);
        c.rnout = static_cast<const double*>(v->effective_normal_outflow);
        c.raout = static_cast<const double*>(v->adjustment_outflow);
        c.rfcout = static_cast<const double*>(v->flood_control_outflow);
    }
    if (bif) {
        c.bptr = v->bif_cell_ptr;
        c.bpaths = v->bif_cell_paths;
        c.bci = v->bifurcation_catchment_idx;
        c.bdi = v->bifurcation_downstream_idx;
        c.bman = static_cast<const double*>(v->bifurcation_manning);
        c.bwid = static_cast<const double*>(v->bifurcation_width);
        c.blen = static_cast<const double*>(v->bifurcation_length);
        c.belv = static_cast<const double*>(v->bifurcation_elevation);
    }
    c.path_off = (long)kSlotCell * c.N;
    c.lev_off = c.path_off + 3L * c.P * c.L + 2 * c.P;
    c.slot_len = c.lev_off + 4L * c.NLV;
    if (res) {
        // compact list of the dam cells, from the cell flags (one copy per plan)
        std::vector<uint8_t> fl((size_t)c.N);
        if (cudaMemcpy(fl.data(), c.flags, (size_t)c.N, cudaMemcpyDeviceToHost) != cudaSuccess) {
            delete p;
            return CMF_ERR_CUDA;
        }
        std::vector<int> dam;
        for (long i = 0; i < c.N; ++i)
            if (fl[(size_t)i] & (CMF_CELL_RESERVOIR | CMF_CELL_DAM_UPSTREAM)) dam.push_back((int)i);
        c.ND = (long)dam.size();
        if (c.ND > 0) {
            std::vector<int> slot((size_t)c.N, -1);
            for (size_t d = 0; d < dam.size(); ++d) slot[(size_t)dam[d]] = (int)d;
            bool ok = cudaMalloc(&p->dam_list, dam.size() * sizeof(int)) == cudaSuccess &&
                      cudaMalloc(&p->dam_slot, slot.size() * sizeof(int)) == cudaSuccess &&
                      cudaMemcpy(p->dam_list, dam.data(), dam.size() * sizeof(int),
                                 cudaMemcpyHostToDevice) == cudaSuccess &&
                      cudaMemcpy(p->dam_slot, slot.data(), slot.size() * sizeof(int),
                                 cudaMemcpyHostToDevice) == cudaSuccess;
            if (!ok) {
                if (p->dam_list) cudaFree(p->dam_list);
                if (p->dam_slot) cudaFree(p->dam_slot);
                delete p;
                return CMF_ERR_CUDA;
            }
        }
        c.dam = p->dam_list;
        c.dam_slot = p->dam_slot;
    }
    c.grid_cells = (int)((c.N + kBlock - 1) / kBlock);
    c.grid_paths = (int)((c.P + kBlock - 1) / kBlock);
    p->grid = c.grid_cells;
    *out = p;
    return CMF_OK;
}

void cmf_adj_plan_destroy(CmfAdjPlan* plan)
{
    if (!plan) return;
    if (plan->dam_list) cudaFree(plan->dam_list);
    if (plan->dam_slot) cudaFree(plan->dam_slot);
    delete plan;
}

int cmf_adj_sub_steps(CmfAdjPlan* plan, void* stream, const double* slot, double outer_seconds,
                      int* n_device)
{
    if (!plan || !slot || !n_device || !(outer_seconds > 0.0)) return CMF_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(n_device, 0, sizeof(int), s) != cudaSuccess) return CMF_ERR_CUDA;
    ka_cfl<<<plan->grid, kBlock, 0, s>>>(plan->ctx, slot, outer_seconds, n_device);
    return launch_status();
}

int cmf_adj_forward(CmfAdjPlan* plan, void* stream, double* slots, int num_sub_steps,
                    int keep_tape, const double* runoff, double dt)
{
    if (!plan || !slots || !runoff || num_sub_steps < 0 || !(dt > 0.0)) return CMF_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Ctx& c = plan->ctx;
    const long stride = c.slot_len;
    const int grid_all = c.grid_cells + (c.bif ? c.grid_paths : 0);
    for (int k = 0; k < num_sub_steps; ++k) {
        double* X = slots + (keep_tape ? (long)k : (long)(k & 1)) * stride;
        double* Y = slots + (keep_tape ? (long)(k + 1) : (long)((k + 1) & 1)) * stride;
        ka_momentum<<<grid_all, kBlock, 0, s>>>(c, X, Y, runoff, dt);
        ka_limit<<<c.grid_cells, kBlock, 0, s>>>(c, X, dt);
        ka_stage<<<grid_all, kBlock, 0, s>>>(c, X, Y, runoff, dt);
        if (c.lev && c.NLV > 0)
            ka_levee<<<(int)((c.NLV + kBlock - 1) / kBlock), kBlock, 0, s>>>(c, X, Y);
    }
    return launch_status();
}

int cmf_adj_reverse(CmfAdjPlan* plan, void* stream, const double* tape, int num_sub_steps,
                    const double* runoff, double dt, double* lambda, double* grad_params,
                    double* grad_runoff, double* scratch)
{
    if (!plan || !tape || !runoff || !lambda || !grad_params || !grad_runoff || !scratch ||
        num_sub_steps < 0 || !(dt > 0.0))
        return CMF_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const Ctx& c = plan->ctx;
    const long stride = c.slot_len;
    Adj a{lambda, grad_params, grad_runoff, scratch};
    for (int k = num_sub_steps - 1; k >= 0; --k) {
        const double* X = tape + (long)k * stride;
        if (c.lev && c.NLV > 0) {
            launch_dep(kr_levee, (int)((c.NLV * 6 + kBlock - 1) / kBlock), s, c, X, a);
        }
        launch_dep(kr_stage, c.grid_cells, s, c, X, runoff, dt, a);
        if (c.bif) launch_dep(kr_stage_path, c.grid_paths, s, c, X, a);
        launch_dep(kr_limit, c.grid_cells, s, c, X, dt, a);
        // cells, then the path and dam direction threads in trailing blocks
        const int path_blocks = c.bif ? (int)((c.P * path_reverse_threads(c.P, c.L) + kBlock - 1) / kBlock) : 0;
        const int dam_blocks = (c.res && c.ND > 0) ? (int)((c.ND * kDamDirs + kBlock - 1) / kBlock) : 0;
        launch_dep(kr_momentum, c.grid_cells + path_blocks + dam_blocks, s, c, X, runoff, dt, a);
    }
    return launch_status();
}

int cmf_adj_finalize(CmfAdjPlan* plan, void* stream, double* lambda, double* grad_params,
                     double* scratch)
{
    if (!plan || !lambda || !grad_params || !scratch) return CMF_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Adj a{lambda, grad_params, nullptr, scratch};
    kr_finalize<<<plan->grid, kBlock, 0, s>>>(plan->ctx, a);
    return launch_status();
}

}  // extern "C"
