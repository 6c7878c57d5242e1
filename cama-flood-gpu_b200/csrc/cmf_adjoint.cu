// Reverse-mode adjoint of the base-physics sub-step, fp64.
//
// The reference has no adjoint; this is the differentiable routing core the
// calibration path needs.  A forward sub-step k maps the state
//
//   X_k = (river/flood storage, river/flood outflow, river/flood depth,
//          river/flood cross-section depth, flood cross-section area)
//
// to X_{k+1} through three phases that each read neighbours (momentum reads
// the downstream depth; the limiter and the stage read the upstream fluxes
// and limit rates).  The primal phases here restate the product forward
// (cmf_device.cuh, REAL = double, base physics) with every intermediate kept,
// and a "tape" slot stores X_k plus the sub-step's fluxes and limit rates:
//
//   slot k = [X_k (9 fields) | qr, qf, lr of sub-step k] x N doubles.
//
// The reverse of one sub-step is three per-cell kernels; every scatter of the
// forward (inflow into the downstream cell, outgoing storage of the downstream
// cell, the downstream depth read by momentum) becomes a gather over the
// contiguous upstream range of the breadth-first order, so the adjoint is
// deterministic and atomic-free like the forward:
//
//   kr_stage     flood stage and storage update reversed per cell (plus the
//                pending downstream-depth adjoints of the upstream cells);
//   kr_limit     limit-rate adjoint gathered over the cell, its upstream cells
//                and its downstream cell; outgoing-storage adjoint;
//   kr_momentum  local-inertial momentum reversed per cell; writes lambda_k
//                and accumulates the parameter gradients.
//
// The subgradient convention is that of the PyTorch transcription used as
// the autograd oracle: clamp passes the gradient on its bounds, a two-operand
// max splits it at a tie, a ternary routes it to the taken branch, and
// max(sqrt(p), f) is differentiable only where p > f*f.

#include "cmfb200.h"

#include <cstdint>
#include <cstring>
#include <new>
#include <cuda_runtime.h>

namespace {

enum StateField { F_RS = 0, F_FS, F_ROUT, F_FOUT, F_RDEP, F_FDEP, F_RCSD, F_FCSD, F_FCSA,
                  kStateFields };
enum SlotExtra { F_QR = kStateFields, F_QF, F_LR, kSlotFields };
enum Scratch { S_RINB = 0, S_FINB, S_ROB, S_FOB, S_OGB, S_QRB, S_QFB, S_WDNB, kScratchFields };
enum Grad { G_RMAN = 0, G_FMAN, G_RH, G_RW, kGradFields };

constexpr int kBlock = 256;
constexpr double kFloor = 1e-6;
constexpr double kFloor2 = 1e-6 * 1e-6;

struct Ctx {
    long N;
    int K;
    double g, alpha, max_dt;
    const int* dn;
    const int* up;
    const uint8_t* flags;
    const double *rw, *rl, *rh, *celv, *ca, *dnd, *rman, *fman, *tbl;
};

__device__ __forceinline__ int up_end(const Ctx& c, long x)
{
    const int e = c.up[x + 1];
    return (x + 1 < c.N && (c.flags[x + 1] & CMF_CELL_MOUTH)) ? e - 1 : e;
}

__device__ __forceinline__ double sgn(double x) { return (double)((x > 0.0) - (x < 0.0)); }

// ---------------------------------------------------------------------------
// Momentum primal with its intermediates (outflow.cu:21-135, base physics; the
// same operation order as momentum_cell with REAL = double).
// ---------------------------------------------------------------------------
struct Mom {
    bool mouth, rc, fc, zero_f, neg;
    int dn;
    double rw, rman, fman, rl, rout, fout, fdep, rcsd, fcsd, fcsa;
    double wse, wse_dn, slope, ucsd, P1, s1, fsurf_m, ufcsd, P2, s2, ufcsa_raw, ufcsa;
    double r_sifd, f_sifd, q, num, den, qr0_val, fc6, P3, s3, fimp, numf, denf, qf0_val;
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

    const double river_elevation = c_elv - r_hgt;
    m.wse = r_dep + river_elevation;
    const double r_dep_dn = X[F_RDEP * N + m.dn];
    const double river_elevation_dn = c.celv[m.dn] - c.rh[m.dn];
    m.wse_dn = m.mouth ? c_elv : r_dep_dn + river_elevation_dn;
    const double max_wse = fmax(m.wse, m.wse_dn);
    m.slope = (m.wse - m.wse_dn) / dn_dist;
    const double fslope = fmin(fmax(m.slope, -0.005), 0.005);

    m.ucsd = m.mouth ? r_dep : max_wse - river_elevation;
    m.P1 = m.ucsd * m.rcsd;
    m.s1 = sqrt(m.P1);
    m.r_sifd = fmax(m.s1, kFloor);
    const double flood_surface = m.mouth ? m.wse : max_wse;
    m.fsurf_m = flood_surface - c_elv;
    m.ufcsd = fmax(m.fsurf_m, 0.0);
    m.P2 = m.ufcsd * m.fcsd;
    m.s2 = sqrt(m.P2);
    m.f_sifd = fmax(m.s2, kFloor);
    m.ufcsa_raw = fs / m.rl - m.fdep * m.rw;
    m.ufcsa = fmax(m.ufcsa_raw, 0.0);

    const double r_cs_area = m.ucsd * m.rw;
    m.rc = (m.r_sifd > 1e-5) && (r_cs_area > 1e-5);
    m.q = m.rout / m.rw;
    m.num = m.rw * (m.q + c.g * dt * m.r_sifd * m.slope);
    m.den = 1.0 + c.g * dt * (m.rman * m.rman) * fabs(m.q)
            * (1.0 / (m.r_sifd * m.r_sifd * cbrt(m.r_sifd)));
    m.qr0_val = m.num / m.den;
    m.qr0 = m.rc ? m.qr0_val : 0.0;

    m.fc = (m.f_sifd > 1e-5) && (m.ufcsa > 1e-5);
    m.qf0 = 0.0;
    m.fc6 = fmax(m.fcsa, kFloor);
    m.P3 = m.ufcsa * m.fc6;
    m.s3 = sqrt(m.P3);
    m.fimp = fmax(m.s3, kFloor);
    m.numf = m.fout + c.g * dt * m.fimp * fslope;
    m.denf = 1.0 + c.g * dt * (m.fman * m.fman) * fabs(m.fout)
             * (1.0 / (m.f_sifd * cbrt(m.f_sifd))) / m.fimp;
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
        const double total_storage_f = rs + fs;
        m.tnf = (-m.qr0 - m.qf1) * dt;
        m.lrn_raw = 0.05 * total_storage_f / m.tnf;
        m.lrn = fmin(m.lrn_raw, 1.0);
        m.qr = m.qr0 * m.lrn;
        m.qf = m.qf1 * m.lrn;
    }
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
    const double total_storage = total_s;
    s.rmax = rl * rw * rh;
    s.flooded = !(total_storage <= s.rmax);
    s.top = false;
    s.cap_taken = false;
    s.level = 0;
    if (!s.flooded) {
        s.rs = total_s;
        s.fs = 0.0;
        s.rdep = total_storage / (rl * rw);
        s.fdep = 0.0;
        s.ffr = 0.0;
        return;
    }
    const int nl = c.K;
    const double ca = c.ca[i];
    const double catchment_width = ca / rl;
    s.winc = catchment_width / (double)nl;
    double S_accum = s.rmax, prev_H = 0.0, prev_W = rw;
    double prev_total_storage = s.rmax, prev_flood_depth = 0.0, next_flood_depth = 0.0;
    const double* row = c.tbl + i * (long)nl;
    for (int l = 0; l < nl; ++l) {
        const double H_curr = __ldg(row + l);
        const double W_curr = rw + (double)(l + 1) * s.winc;
        const double dS = rl * 0.5 * (prev_W + W_curr) * (H_curr - prev_H);
        const double S_curr = S_accum + dS;
        next_flood_depth = H_curr;
        if (total_storage > S_curr) {
            s.level += 1;
            prev_total_storage = S_curr;
            prev_flood_depth = H_curr;
            S_accum = S_curr;
            prev_H = H_curr;
            prev_W = W_curr;
        } else {
            break;
        }
    }
    s.top = s.level == nl;
    s.S_prev = prev_total_storage;
    s.D_prev = prev_flood_depth;
    s.W_tot = rw + (double)s.level * s.winc;
    s.excess = total_storage - prev_total_storage;
    s.diff_w = 0.0;
    if (s.top) {
        s.fdep = prev_flood_depth + s.excess / (s.W_tot * rl);
    } else {
        s.grad = (next_flood_depth - prev_flood_depth) / s.winc;
        s.arg = s.W_tot * s.W_tot + 2.0 * s.excess / (s.grad * rl);
        s.sq = sqrt(s.arg);
        s.diff_w = s.sq - s.W_tot;
        s.fdep = prev_flood_depth + s.diff_w * s.grad;
    }
    s.cap = s.rmax + rl * rw * s.fdep;
    s.cap_taken = s.cap < total_s;
    const double river = s.cap_taken ? s.cap : total_s;
    s.rdep = river / (rl * rw);
    double ff = (s.W_tot + s.diff_w - rw) * rl / ca;
    ff = ff < 0.0 ? 0.0 : (ff > 1.0 ? 1.0 : ff);
    s.ffr = s.top ? 1.0 : ff;
    double flood = total_s - river;
    if (flood < 0.0) flood = 0.0;
    s.rs = river;
    s.fs = flood;
}

// Storage update (storage.cu:67-116) with its branch record.
struct Store {
    double rsu1, fsu1, rsu2, tt, total_next;
    double rin, fin, ur, uf;
};

// Inflow gather and own limited flux of cell i.
__device__ __forceinline__ void gather_inflow(const Ctx& c, const double* X, long i, Store& t)
{
    const long N = c.N;
    const double lr_i = X[F_LR * N + i];
    const double qr = X[F_QR * N + i], qf = X[F_QF * N + i];
    double rin = 0.0, fin = 0.0;
    const int c0 = c.up[i], c1 = up_end(c, i);
    for (int u = c0; u < c1; ++u) {
        const double cr = X[F_QR * N + u], cf = X[F_QF * N + u], cl = X[F_LR * N + u];
        rin += (cr >= 0.0) ? cr * cl : cr * lr_i;
        fin += (cf >= 0.0) ? cf * cl : cf * lr_i;
    }
    const bool mouth = c.flags[i] & CMF_CELL_MOUTH;
    const double lr_dn = mouth ? lr_i : X[F_LR * N + c.dn[i]];
    t.rin = rin;
    t.fin = fin;
    t.ur = (qr >= 0.0) ? qr * lr_i : qr * lr_dn;
    t.uf = (qf >= 0.0) ? qf * lr_i : qf * lr_dn;
}

__device__ __forceinline__ double store_eval(const double rsto, const double fsto,
                                             const double ro, double dt, Store& t)
{
    const double river_delta = (t.rin - t.ur) * dt;
    t.rsu1 = rsto + river_delta;
    const double flood_delta = (t.fin - t.uf - 0.0) * dt;
    t.fsu1 = fsto + (t.rsu1 < 0.0 ? t.rsu1 : 0.0) + flood_delta;
    t.rsu2 = t.rsu1 > 0.0 ? t.rsu1 : 0.0;
    double river_su = t.rsu2;
    t.tt = river_su + t.fsu1;
    if (t.fsu1 < 0.0) river_su = t.tt > 0.0 ? t.tt : 0.0;
    const double flood_su = t.fsu1 > 0.0 ? t.fsu1 : 0.0;
    const double external_delta = ro * dt;
    t.total_next = river_su + flood_su + 0.0 + external_delta;
    return t.total_next > 0.0 ? t.total_next : 0.0;
}

// ---------------------------------------------------------------------------
// forward kernels (tape)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) ka_momentum(const Ctx c, double* X, double* Y, double dt)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    Mom m;
    mom_eval(c, X, i, dt, m);
    const long N = c.N;
    X[F_QR * N + i] = m.qr;
    X[F_QF * N + i] = m.qf;
    Y[F_RCSD * N + i] = m.ucsd;
    Y[F_FCSD * N + i] = m.ufcsd;
    Y[F_FCSA * N + i] = m.ufcsa;
}

__global__ void __launch_bounds__(kBlock) ka_limit(const Ctx c, double* X, double dt)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const long N = c.N;
    const double qr = X[F_QR * N + i], qf = X[F_QF * N + i];
    const double pos = fmax(qr, 0.0) + fmax(qf, 0.0);
    double og = pos * dt;
    const int c0 = c.up[i], c1 = up_end(c, i);
    for (int u = c0; u < c1; ++u) {
        const double neg = fmin(X[F_QR * N + u], 0.0) + fmin(X[F_QF * N + u], 0.0);
        og += -neg * dt;
    }
    const double store = X[F_RS * N + i] + X[F_FS * N + i];
    X[F_LR * N + i] = (og > 1e-8) ? fmin(store / og, 1.0) : 1.0;
}

__global__ void __launch_bounds__(kBlock) ka_stage(const Ctx c, const double* X, double* Y,
                                                   const double* runoff, double dt)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const long N = c.N;
    Store t;
    gather_inflow(c, X, i, t);
    const double tot = store_eval(X[F_RS * N + i], X[F_FS * N + i], runoff[i], dt, t);
    Stage s;
    stage_eval(c, i, tot, c.rh[i], c.rw[i], c.rl[i], s);
    Y[F_RS * N + i] = s.rs;
    Y[F_FS * N + i] = s.fs;
    Y[F_ROUT * N + i] = t.ur;
    Y[F_FOUT * N + i] = t.uf;
    Y[F_RDEP * N + i] = s.rdep;
    Y[F_FDEP * N + i] = s.fdep;
}

__global__ void __launch_bounds__(kBlock) ka_cfl(const Ctx c, const double* X, double outer,
                                                 int* n_out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int n_steps = 1;
    if (i < c.N) {
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
    double* lam;      // [kStateFields][N], lambda_{k+1} on entry of a sub-step, lambda_k on exit
    double* grad;     // [kGradFields][N]
    double* groff;    // [N] runoff gradient of the current interval
    double* scr;      // [kScratchFields][N]
};

// Stage and storage update reversed (kr_stage).
__global__ void __launch_bounds__(kBlock) kr_stage(const Ctx c, const double* X,
                                                   const double* runoff, double dt, Adj a)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const long N = c.N;
    double* lam = a.lam;
    double* scr = a.scr;
    const double rw = c.rw[i], rl = c.rl[i], rh = c.rh[i];

    // lambda_{k+1} of the river depth: own part plus the pending downstream-
    // depth adjoints of the upstream cells (their momentum read this depth).
    double wsum = 0.0;
    const int c0 = c.up[i], c1 = up_end(c, i);
    for (int u = c0; u < c1; ++u) wsum += scr[S_WDNB * N + u];
    const double L_rdep = lam[F_RDEP * N + i] + wsum;
    double g_rh = -wsum, g_rw = 0.0;

    const double L_rs = lam[F_RS * N + i], L_fs = lam[F_FS * N + i];
    const double L_rout = lam[F_ROUT * N + i], L_fout = lam[F_FOUT * N + i];
    const double L_fdep = lam[F_FDEP * N + i];

    Store t;
    gather_inflow(c, X, i, t);
    const double rsto = X[F_RS * N + i], fsto = X[F_FS * N + i];
    const double tot = store_eval(rsto, fsto, runoff[i], dt, t);
    Stage s;
    stage_eval(c, i, tot, rh, rw, rl, s);

    // ---- flood stage reverse -> tot_bar, rw, rh
    double tot_bar = 0.0;
    const double rlrw = rl * rw;
    double rs_out_bar = L_rs + L_rdep / rlrw;       // rs' and rdep' = rs' / (rl rw)
    g_rw += -L_rdep * s.rdep / rw;
    if (!s.flooded) {
        tot_bar = rs_out_bar;
    } else {
        double river_bar = rs_out_bar;
        const double d = tot - s.rs;
        if (!(d < 0.0)) {            // flood' = d where d >= 0
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
        // S_prev = rmax + sum_{l < level} rl (W_{l-1} + W_l)/2 (H_l - H_{l-1});
        // d/d rw of the layer sum telescopes to rl * H_{level-1}
        rmax_bar += Sp_bar;
        if (s.level > 0) g_rw += Sp_bar * rl * s.D_prev;
        g_rw += rmax_bar * rl * rh;
        g_rh += rmax_bar * rlrw;
    }

    // ---- storage update reverse
    double tn_bar = t.total_next > 0.0 ? tot_bar : 0.0;
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
    const double fs_bar = fsu1_bar;
    if (t.rsu1 < 0.0) rsu1_bar += fsu1_bar;
    const double fin_bar = fsu1_bar * dt;
    const double uf_own = -fsu1_bar * dt;
    const double rs_bar = rsu1_bar;
    const double rin_bar = rsu1_bar * dt;
    const double ur_own = -rsu1_bar * dt;

    lam[F_RS * N + i] = rs_bar;
    lam[F_FS * N + i] = fs_bar;
    scr[S_RINB * N + i] = rin_bar;
    scr[S_FINB * N + i] = fin_bar;
    scr[S_ROB * N + i] = L_rout + ur_own;
    scr[S_FOB * N + i] = L_fout + uf_own;
    a.grad[G_RH * N + i] += g_rh;
    a.grad[G_RW * N + i] += g_rw;
}

// Limit-rate adjoint (kr_limit).  u_j = q_j * (q_j >= 0 ? lr_j : lr_dn(j))
// enters the cell's own update (-u dt) and its downstream inflow (+u dt), so
// its adjoint is rob_j + rinb_dn(j); lr_j collects the positive own fluxes and
// the negative fluxes of the upstream cells.
__global__ void __launch_bounds__(kBlock) kr_limit(const Ctx c, const double* X, double dt, Adj a)
{
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= c.N) return;
    const long N = c.N;
    const double* scr = a.scr;
    const bool mouth = c.flags[j] & CMF_CELL_MOUTH;
    const int dn = c.dn[j];
    const double qr = X[F_QR * N + j], qf = X[F_QF * N + j], lr = X[F_LR * N + j];
    const double lr_dn = mouth ? lr : X[F_LR * N + dn];
    const double rinb = scr[S_RINB * N + j], finb = scr[S_FINB * N + j];
    const double a_r = scr[S_ROB * N + j] + (mouth ? 0.0 : scr[S_RINB * N + dn]);
    const double a_f = scr[S_FOB * N + j] + (mouth ? 0.0 : scr[S_FINB * N + dn]);

    double lr_bar = 0.0;
    if (qr >= 0.0 || mouth) lr_bar += a_r * qr;
    if (qf >= 0.0 || mouth) lr_bar += a_f * qf;
    double qr_bar = a_r * ((qr >= 0.0) ? lr : lr_dn);
    double qf_bar = a_f * ((qf >= 0.0) ? lr : lr_dn);

    double og = (fmax(qr, 0.0) + fmax(qf, 0.0)) * dt;
    const int c0 = c.up[j], c1 = up_end(c, j);
    for (int u = c0; u < c1; ++u) {
        const double cr = X[F_QR * N + u], cf = X[F_QF * N + u];
        if (cr < 0.0) lr_bar += (scr[S_ROB * N + u] + rinb) * cr;
        if (cf < 0.0) lr_bar += (scr[S_FOB * N + u] + finb) * cf;
        og += -(fmin(cr, 0.0) + fmin(cf, 0.0)) * dt;
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

// Momentum reversed (kr_momentum): lambda_k of the cell, the downstream-depth
// adjoint left for the downstream cell's next kr_stage, parameter gradients.
__global__ void __launch_bounds__(kBlock) kr_momentum(const Ctx c, const double* X, double dt, Adj a)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const long N = c.N;
    double* lam = a.lam;
    Mom m;
    mom_eval(c, X, i, dt, m);
    const double D = c.g * dt;

    // adjoints of the final fluxes: stage/limiter part, plus the outgoing
    // storage of the downstream cell (negative fluxes leave through it)
    double qr_bar = a.scr[S_QRB * N + i];
    double qf_bar = a.scr[S_QFB * N + i];
    if (!m.mouth) {
        const double ogb_dn = a.scr[S_OGB * N + m.dn];
        if (m.qr <= 0.0) qr_bar += -ogb_dn * dt;
        if (m.qf <= 0.0) qf_bar += -ogb_dn * dt;
    }
    double ucsd_bar = lam[F_RCSD * N + i];
    double ufcsd_bar = lam[F_FCSD * N + i];
    double ufcsa_bar = lam[F_FCSA * N + i];

    double rs_bar = 0.0, fs_bar = 0.0, rout_bar = 0.0, fout_bar = 0.0, rdep_bar = 0.0;
    double fdep_bar = 0.0, rcsd_bar = 0.0, fcsd_bar = 0.0, fcsa_bar = 0.0;
    double g_rman = 0.0, g_fman = 0.0, g_rw = 0.0, relev_bar = 0.0;

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
            qr0_bar += -tnf_bar * dt;
            qf1_bar += -tnf_bar * dt;
        }
    }
    const double qf0_bar = m.zero_f ? 0.0 : qf1_bar;

    double slope_bar = 0.0, fslope_bar = 0.0, r_sifd_bar = 0.0, f_sifd_bar = 0.0;
    // floodplain flux
    if (m.fc) {
        const double numf_bar = qf0_bar / m.denf;
        const double denf_bar = -qf0_bar * m.qf0_val / m.denf;
        fout_bar += numf_bar;
        double fimp_bar = numf_bar * D * fmin(fmax(m.slope, -0.005), 0.005);
        fslope_bar += numf_bar * D * m.fimp;
        const double af = fabs(m.fout);
        const double B = 1.0 / (m.f_sifd * cbrt(m.f_sifd));
        const double nf2 = m.fman * m.fman;
        const double T = D * nf2 * af * B / m.fimp;
        g_fman += denf_bar * D * 2.0 * m.fman * af * B / m.fimp;
        fout_bar += denf_bar * D * nf2 * B / m.fimp * sgn(m.fout);
        f_sifd_bar += denf_bar * D * nf2 * af / m.fimp * (-(4.0 / 3.0) * B / m.f_sifd);
        fimp_bar += denf_bar * (-T / m.fimp);
        if (m.P3 > kFloor2) {
            const double P3_bar = fimp_bar / (2.0 * m.s3);
            ufcsa_bar += P3_bar * m.fc6;
            if (m.fcsa >= kFloor) fcsa_bar += P3_bar * m.ufcsa;
        }
    }
    // river flux
    if (m.rc) {
        const double num_bar = qr0_bar / m.den;
        const double den_bar = -qr0_bar * m.qr0_val / m.den;
        g_rw += num_bar * (m.q + D * m.r_sifd * m.slope);
        const double inner_bar = num_bar * m.rw;
        double q_bar = inner_bar;
        r_sifd_bar += inner_bar * D * m.slope;
        slope_bar += inner_bar * D * m.r_sifd;
        const double aq = fabs(m.q);
        const double Br = 1.0 / (m.r_sifd * m.r_sifd * cbrt(m.r_sifd));
        const double n2 = m.rman * m.rman;
        g_rman += den_bar * D * 2.0 * m.rman * aq * Br;
        q_bar += den_bar * D * n2 * Br * sgn(m.q);
        r_sifd_bar += den_bar * D * n2 * aq * (-(7.0 / 3.0) * Br / m.r_sifd);
        rout_bar += q_bar / m.rw;
        g_rw += -q_bar * m.q / m.rw;
    }
    if (m.slope >= -0.005 && m.slope <= 0.005) slope_bar += fslope_bar;
    // flood cross-section area
    if (m.ufcsa_raw >= 0.0) {
        fs_bar += ufcsa_bar / m.rl;
        fdep_bar += -ufcsa_bar * m.rw;
        g_rw += -ufcsa_bar * m.fdep;
    }
    // flood cross-section depth
    if (m.P2 > kFloor2) {
        const double P2_bar = f_sifd_bar / (2.0 * m.s2);
        ufcsd_bar += P2_bar * m.fcsd;
        fcsd_bar += P2_bar * m.ufcsd;
    }
    double fsurf_bar = (m.fsurf_m >= 0.0) ? ufcsd_bar : 0.0;
    // river cross-section depth
    if (m.P1 > kFloor2) {
        const double P1_bar = r_sifd_bar / (2.0 * m.s1);
        ucsd_bar += P1_bar * m.rcsd;
        rcsd_bar += P1_bar * m.ucsd;
    }
    double wse_bar = 0.0, wse_dn_bar = 0.0, mw_bar = 0.0;
    if (m.mouth) {
        rdep_bar += ucsd_bar;
        wse_bar += fsurf_bar;
    } else {
        mw_bar += ucsd_bar;
        relev_bar -= ucsd_bar;
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

// Apply the pending downstream-depth adjoints (end of the reverse sweep).
__global__ void __launch_bounds__(kBlock) kr_finalize(const Ctx c, Adj a)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.N) return;
    const long N = c.N;
    double wsum = 0.0;
    const int c0 = c.up[i], c1 = up_end(c, i);
    for (int u = c0; u < c1; ++u) wsum += a.scr[S_WDNB * N + u];
    a.lam[F_RDEP * N + i] += wsum;
    a.grad[G_RH * N + i] -= wsum;
}

}  // namespace

struct CmfAdjPlan {
    Ctx ctx;
    int grid;
};

namespace {

int launch_status()
{
    return cudaGetLastError() == cudaSuccess ? CMF_OK : CMF_ERR_CUDA;
}

}  // namespace

extern "C" {

int cmf_adj_layout(int* state_fields, int* slot_fields, int* scratch_fields, int* grad_fields)
{
    if (state_fields) *state_fields = kStateFields;
    if (slot_fields) *slot_fields = kSlotFields;
    if (scratch_fields) *scratch_fields = kScratchFields;
    if (grad_fields) *grad_fields = kGradFields;
    return CMF_OK;
}

int cmf_adj_plan_create(const CmfView* v, CmfAdjPlan** out)
{
    if (!v || !out) return CMF_ERR_ARG;
    *out = nullptr;
    if (v->abi_version != CMF_ABI_VERSION) return CMF_ERR_ARG;
    if (!(v->features & CMF_FEAT_FP64)) return CMF_ERR_UNSUPPORTED;
    if (v->features & (CMF_FEAT_BIFURCATION | CMF_FEAT_LEVEE | CMF_FEAT_RESERVOIR))
        return CMF_ERR_UNSUPPORTED;
    if (v->num_members != 1 || v->batched_mask != 0) return CMF_ERR_UNSUPPORTED;
    if (v->num_catchments < 1 || v->num_catchments > (1L << 31) - 2 || v->num_flood_levels < 1)
        return CMF_ERR_ARG;
    const void* need[] = {v->downstream_idx, v->upstream_ptr, v->cell_flags, v->river_width,
                          v->river_length, v->river_height, v->catchment_elevation,
                          v->catchment_area, v->downstream_distance, v->river_manning,
                          v->flood_manning, v->flood_depth_table};
    for (const void* p : need)
        if (!p) return CMF_ERR_ARG;
    CmfAdjPlan* p = new (std::nothrow) CmfAdjPlan;
    if (!p) return CMF_ERR_ARG;
    Ctx& c = p->ctx;
    c.N = v->num_catchments;
    c.K = v->num_flood_levels;
    c.g = v->gravity;
    c.alpha = v->adaptive_time_factor;
    c.max_dt = v->max_sub_step_seconds;
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
    p->grid = (int)((c.N + kBlock - 1) / kBlock);
    *out = p;
    return CMF_OK;
}

void cmf_adj_plan_destroy(CmfAdjPlan* plan) { delete plan; }

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
    const long stride = (long)kSlotFields * c.N;
    for (int k = 0; k < num_sub_steps; ++k) {
        double* X = slots + (keep_tape ? (long)k : (long)(k & 1)) * stride;
        double* Y = slots + (keep_tape ? (long)(k + 1) : (long)((k + 1) & 1)) * stride;
        ka_momentum<<<plan->grid, kBlock, 0, s>>>(c, X, Y, dt);
        ka_limit<<<plan->grid, kBlock, 0, s>>>(c, X, dt);
        ka_stage<<<plan->grid, kBlock, 0, s>>>(c, X, Y, runoff, dt);
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
    const long stride = (long)kSlotFields * c.N;
    Adj a{lambda, grad_params, grad_runoff, scratch};
    for (int k = num_sub_steps - 1; k >= 0; --k) {
        const double* X = tape + (long)k * stride;
        kr_stage<<<plan->grid, kBlock, 0, s>>>(c, X, runoff, dt, a);
        kr_limit<<<plan->grid, kBlock, 0, s>>>(c, X, dt, a);
        kr_momentum<<<plan->grid, kBlock, 0, s>>>(c, X, dt, a);
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
