// Per-element routing physics of CaMa-Flood, written from its equations and
// shared by the forward kernels (cmf_device.cuh: float or double) and the
// adjoint (cmf_adjoint.cu: double and forward-mode dual numbers).
//
// Nothing here touches memory layouts: callers load the element's fields,
// call these functions and store the results.  Every floating-point
// expression is the rounded-operation sequence of the reference kernel that
// computes the same quantity (cmfgpu/phys/cuda/*.cu), cited per function, so
// the forward stays bit-identical to those kernels; names and control flow
// are this project's own.  Constants are typed by the caller's scalar (P(x))
// so that a float instantiation never widens to double.
#pragma once

#include "cmf_scalar.cuh"

namespace cmf {

// ---------------------------------------------------------------------------
// Momentum
// ---------------------------------------------------------------------------

// Local-inertial discharge of a channel of width B after one sub-step
// (Bates et al. 2010, in CaMa-Flood's per-unit-width form):
//     Q' = B (q + g dt h S) / (1 + g dt n^2 |q| h^(-7/3)),   q = Q / B,
// h the semi-implicit flow depth, S the water-surface slope, gdt = g dt.
// River channels (outflow.cu:107-115) and bifurcation levels
// (bifurcation.cu:72-77) use it alike.
template <typename T, typename B, typename N, typename P>
__device__ __forceinline__ T channel_discharge(T Q, B width, N manning, T h, T slope, P gdt)
{
    const T q = Q / width;
    const T drive = q + gdt * h * slope;
    const T drag = P(1) + gdt * (manning * manning) * sabs(q) * (P(1) / (h * h * scbrt(h)));
    return width * drive / drag;
}

// The floodplain form, per flow area A (outflow.cu:119-127):
//     Q' = (Q + g dt A S) / (1 + g dt n^2 |Q| h^(-4/3) / A).
template <typename T, typename N, typename P>
__device__ __forceinline__ T plain_discharge(T Q, T area, N manning, T h, T slope, P gdt)
{
    const T drive = Q + gdt * area * slope;
    const T drag = P(1) + gdt * (manning * manning) * sabs(Q) * (P(1) / (h * scbrt(h))) / area;
    return drive / drag;
}

// Semi-implicit depth (or area) of the friction term: the geometric mean of
// the new and the previous value, floored.
template <typename T, typename P>
__device__ __forceinline__ T implicit_mean(T now, T before, P floor)
{
    return smax(ssqrt(now * before), T(floor));
}

// Surface slope limited for the floodplain and the bifurcation paths.
template <typename T, typename P>
__device__ __forceinline__ T capped_slope(T slope, P cap)
{
    return smin(smax(slope, T(-cap)), T(cap));
}

// Kinematic-wave outflow of a catchment right upstream of a dam, which the
// local-inertial form cannot resolve (outflow.cu:137-153): Manning velocity
// with the hydraulic radius taken as the depth, v = S^(1/2) h^(2/3) / n,
// on the bed slope (floored by the caller; the floodplain uses at most
// 0.005), each flux clamped to [0, storage / dt].
template <typename T, typename P>
__device__ __forceinline__ void kinematic_outflow(P bed_slope, P length, T h_riv, T h_fld,
                                                  T s_riv, T s_fld, T width, T n_riv, T n_fld,
                                                  P dt, T& q_riv, T& q_fld)
{
    const T v_riv = (P(1) / n_riv) * ssqrt(bed_slope) * scbrt(h_riv * h_riv);
    q_riv = smax(smin(width * h_riv * v_riv, s_riv / dt), T(0));
    const P fld_slope = smin(bed_slope, P(0.005));
    const T v_fld = (P(1) / n_fld) * ssqrt(fld_slope) * scbrt(h_fld * h_fld);
    const T area = smax(s_fld / length - h_fld * width, T(0));
    q_fld = smax(smin(area * v_fld, s_fld / dt), T(0));
}

// ---------------------------------------------------------------------------
// Reservoir operation: the default release rule of CaMa-Flood's dam scheme
// (reservoir.cu:62-84).  Storage regimes, by volume:
//   up to the conservation volume   normal release x sqrt(fill fraction)
//   up to the adjustment volume     cubic ramp from normal to adjustment release
//   up to the emergency volume      0.1-power ramp to the flood-control
//                                   release, raised by the inflow-proportional
//                                   rule while the inflow exceeds it
//   above                           pass the inflow, at least the flood release
// The release is clamped to [0, storage / dt].
// ---------------------------------------------------------------------------
template <typename P>
struct DamRule {
    P v_cons, v_adj, v_emerg;  // conservation, adjustment, emergency volumes
    P q_norm, q_adj, q_flood;  // effective normal, adjustment, flood-control release
};

template <typename T, typename P>
__device__ __forceinline__ T dam_release(const DamRule<P>& r, T storage, T inflow, P dt)
{
    T q;
    if (val(storage) <= r.v_cons) {
        q = r.q_norm * ssqrt(storage / r.v_cons);
    } else if (val(storage) <= r.v_adj) {
        const T fill = (storage - r.v_cons) / (r.v_adj - r.v_cons);
        q = r.q_norm + sexp(P(3) * slog(fill)) * (r.q_adj - r.q_norm);
    } else if (val(storage) <= r.v_emerg) {
        const T fill = (storage - r.v_adj) / (r.v_emerg - r.v_adj);
        const T ramp = r.q_adj + sexp(P(0.1) * slog(fill)) * (r.q_flood - r.q_adj);
        if (val(inflow) >= r.q_flood) {
            const T share = r.q_norm + ((storage - r.v_cons) / (r.v_emerg - r.v_cons))
                                           * (inflow - r.q_norm);
            q = smax(share, ramp);
        } else {
            q = ramp;
        }
    } else {
        q = (val(inflow) >= r.q_flood) ? inflow : T(r.q_flood);
    }
    return smin(smax(q, T(0)), storage / dt);
}

// ---------------------------------------------------------------------------
// Bifurcation paths (bifurcation.cu:21-129; with levees levee.cu:263-341)
// ---------------------------------------------------------------------------
template <typename T>
struct PathEnds {
    T eta_a, eta_b;    // water-surface elevation of the path's two end cells
    T peta_a, peta_b;  // protected-side water surface (levee variant)
    T store_a, store_b;  // total storage of the end cells
};

// Unlimited per-level fluxes of one path.  Level l carries water above its
// sill elevation; with levees, level 0 sees the river surfaces and the higher
// levels the protected-side surfaces, and the semi-implicit depth falls back
// to the new depth where the geometric mean vanishes; without levees the
// previous depth is floored at 0.01 m.  `lv` supplies the level's sill
// elevation, width, Manning coefficient, previous flux and previous depth,
// loaded only when used, and receives each level's new depth
// (lv.new_depth).  Writes the unlimited fluxes; returns their sum.
template <bool LEVEE, int LMAX, typename T, typename P, typename Levels>
__device__ __forceinline__ T path_level_fluxes(const Levels& lv, int L, const PathEnds<T>& e,
                                               P length, P gdt, T (&flux)[LMAX])
{
    const T top = smax(e.eta_a, e.eta_b);
    const T ptop = LEVEE ? smax(e.peta_a, e.peta_b) : top;
    const T slope = capped_slope((e.eta_a - e.eta_b) / length, P(0.005));
    T sum = T(0);
#pragma unroll
    for (int l = 0; l < LMAX; ++l) {
        T q = T(0);
        if (l < L) {
            const T surface = (LEVEE && l > 0) ? ptop : top;
            const T h = smax(surface - lv.sill(l), T(0));
            T h_si;
            if (LEVEE) {
                h_si = h;
                if (l == 0) {
                    h_si = ssqrt(h * lv.depth(0));
                    if (val(h_si) <= P(0)) h_si = h;
                }
            } else {
                h_si = smax(ssqrt(h * lv.depth(l)), ssqrt(h * P(0.01)));
            }
            if (val(h_si) > P(1e-5))
                q = channel_discharge(lv.flux(l), lv.width(l), lv.manning(l), h_si, slope, gdt);
            sum = sum + q;
            lv.new_depth(l, h);
        }
        flux[l] = q;
    }
    return sum;
}

// Path limiter: the summed path flux may move at most 5 % of the smaller end
// storage in one sub-step.  A path without flow keeps rate 1 (the reference's
// division by zero yields the same).
template <typename T, typename P>
__device__ __forceinline__ T path_rate(T sum, T store_a, T store_b, P dt)
{
    const T moved = sabs(sum) * dt;
    if (!(val(moved) > P(0))) return T(1);
    return smin(P(0.05) * smin(store_a, store_b) / moved, T(1));
}

// ---------------------------------------------------------------------------
// Flood stage: inversion of the floodplain profile (storage.cu:118-211)
//
// The floodplain of a catchment of length L, river width B and area A is K
// layers: layer l spans the widths B + l dW .. B + (l+1) dW, dW = A / (L K),
// between the table depths D_(l-1) and D_l (D_(-1) = 0), so the storage below
// its top is S_l = S_bank + sum of L (w_lo + w_hi) / 2 (D_l - D_(l-1)).
// ---------------------------------------------------------------------------
template <typename R>
struct FillLevel {
    int full;  // layers the storage fills completely
    R s_top;   // storage at the top of the last full layer (bank storage if none)
    R d_top;   // depth at that top (0 if none)
    R d_next;  // table depth at the top of the next layer (last one read)
};

// Adds layer l (top depth d_hi) to the walk; false when the storage does not
// exceed the layer's top, which ends the walk.
template <typename R>
__device__ __forceinline__ bool fill_layer(FillLevel<R>& f, R& w_lo, int l, R d_hi, R S, R width,
                                           R len, R dw)
{
    const R w_hi = width + R(l + 1) * dw;
    const R s_hi = f.s_top + len * R(0.5) * (w_lo + w_hi) * (d_hi - f.d_top);
    f.d_next = d_hi;
    if (!(val(S) > val(s_hi))) return false;
    f.full = l + 1;
    f.s_top = s_hi;
    f.d_top = d_hi;
    w_lo = w_hi;
    return true;
}

// Walk over a table row held in registers (KR levels, fully unrolled).
template <int KR, typename R>
__device__ __forceinline__ FillLevel<R> fill_level_regs(const R (&D)[KR], R S, R bank, R width,
                                                        R len, R dw)
{
    FillLevel<R> f{0, bank, R(0), R(0)};
    R w_lo = width;
    bool rising = true;
#pragma unroll
    for (int l = 0; l < KR; ++l)
        if (rising) rising = fill_layer(f, w_lo, l, D[l], S, width, len, dw);
    return f;
}

// Walk over a table row in memory (any number of levels).
template <typename R>
__device__ __forceinline__ FillLevel<R> fill_level_mem(const R* D, int K, R S, R bank, R width,
                                                       R len, R dw)
{
    FillLevel<R> f{0, bank, R(0), R(0)};
    R w_lo = width;
    for (int l = 0; l < K; ++l)
        if (!fill_layer(f, w_lo, l, __ldg(D + l), S, width, len, dw)) break;
    return f;
}

// Depth above the bank and the flooded width beyond the last full layer.
// Inside a partly filled layer the flooded width w grows linearly with depth
// at the layer's gradient g, so L (w_top x + g x^2 / 2) = S - s_top for the
// extra width x; above the table the walls are vertical.
template <typename R>
struct FloodSurface {
    R depth;        // flood depth above the bank
    R width_top;    // width at the top of the last full layer
    R extra_width;  // flooded width beyond it (0 above the table)
};

template <typename R>
__device__ __forceinline__ FloodSurface<R> flood_surface(const FillLevel<R>& f, int K, R S,
                                                         R width, R len, R dw)
{
    FloodSurface<R> o;
    o.width_top = width + R(f.full) * dw;
    if (f.full == K) {
        o.extra_width = R(0);
        o.depth = f.d_top + (S - f.s_top) / (o.width_top * len);
    } else {
        const R grad = (f.d_next - f.d_top) / dw;
        o.extra_width = ssqrt(o.width_top * o.width_top + R(2) * (S - f.s_top) / (grad * len))
                        - o.width_top;
        o.depth = f.d_top + o.extra_width * grad;
    }
    return o;
}

// Partition of a cell's total storage between river and floodplain.
template <typename S, typename R>
struct StageOut {
    S rs, fs;         // river / flood storage
    R rdep, fdep;     // river / flood depth
    R ffr;            // flooded fraction of the catchment
};

// Continuity over one sub-step (storage.cu:89-116): the river gains its net
// channel flux, the floodplain its net floodplain flux less the bifurcation
// outflow; a river deficit is taken from the floodplain and a floodplain
// deficit from the river, each store clipped at zero; the runoff then joins
// the total.  Volume changes are formed on the flux type and added on the
// storage type.
template <typename S, typename R>
struct Continuity {
    S river, flood;  // the two stores after the exchange, before the runoff
    S total;         // new total storage (clipped at zero), runoff included
    R d_river, d_flood, d_runoff;  // the sub-step's volume changes
};

template <typename S, typename R>
__device__ __forceinline__ Continuity<S, R> continuity(S s_riv, S s_fld, S s_prot, R in_riv,
                                                       R out_riv, R in_fld, R out_fld, R out_bif,
                                                       R runoff, R dt)
{
    Continuity<S, R> c;
    c.d_river = (in_riv - out_riv) * dt;
    c.d_flood = (in_fld - out_fld - out_bif) * dt;
    c.d_runoff = runoff * dt;
    S river = s_riv + static_cast<S>(c.d_river);
    S flood = s_fld + (val(river) < 0 ? river : S(0)) + static_cast<S>(c.d_flood);
    river = pos_part(river);
    if (val(flood) < 0) river = pos_part(river + flood);
    flood = pos_part(flood);
    c.river = river;
    c.flood = flood;
    c.total = pos_part(river + flood + s_prot + static_cast<S>(c.d_runoff));
    return c;
}

// Flood stage of total storage S_tot (storage type S; the profile arithmetic
// runs on its flux-type value).  A storage within the banks is all river;
// above them the flood depth comes from the profile, the river holds its
// bankfull storage plus a column of that depth (at most the total), the
// floodplain the rest, and the flooded fraction is the flooded width over
// the catchment width (1 above the table).  `prof` supplies the catchment
// area and the profile walk; both are asked for only above the banks.
template <typename S, typename R, typename Profile>
__device__ __forceinline__ StageOut<S, R> flood_stage_of(S S_tot, R width, R len, R height, int K,
                                                         Profile& prof)
{
    StageOut<S, R> o;
    const R total = narrow<R>(S_tot);
    const R bank = len * width * height;
    if (val(total) <= val(bank)) {
        o.rs = S_tot;
        o.fs = S(0);
        o.rdep = total / (len * width);
        o.fdep = R(0);
        o.ffr = R(0);
        return o;
    }
    const R area = prof.area();
    const R dw = area / len / R(K);
    const FillLevel<R> f = prof.walk(total, bank, width, len, dw);
    const FloodSurface<R> s = flood_surface(f, K, total, width, len, dw);
    const S column = static_cast<S>(bank + len * width * s.depth);
    const S river = val(column) < val(S_tot) ? column : S_tot;
    o.rs = river;
    o.rdep = narrow<R>(river) / (len * width);
    R frac = (s.width_top + s.extra_width - width) * len / area;
    frac = val(frac) < 0 ? R(0) : (val(frac) > 1 ? R(1) : frac);
    o.ffr = (f.full == K) ? R(1) : frac;
    const S rest = S_tot - river;
    o.fs = val(rest) < 0 ? S(0) : rest;
    o.fdep = s.depth;
    return o;
}

// ---------------------------------------------------------------------------
// Levee stage (levee.cu:29-261): re-partition of a levee cell's flood-stage
// result between the river side, the floodplain outside the levee and the
// protected side behind it.
//
// The levee stands at distance d = frac x A / L from the bank, with base
// height H_b (the profile height there) and crown H_c.  On the profile walk
// of the levee scheme (layers summed from the bank with the running width
// plus half a width step, layer heights floored at 1e-6 m) three storages
// mark the regimes:
//   S_base   the profile filled up to the base height,
//   S_top    S_base plus the river-side wedge (d + B) (H_c - H_b) L up to the
//            crown,
//   S_crown  the profile filled up to the crown height;
// and the total storage S selects
//   S >= S_crown             overtopped: the flood stage stands, the
//                            protected side takes what exceeds the wedge;
//   S_top <= S < S_crown     river side at the crown, the protected side
//                            filling (its surface from a second walk);
//   S_base <= S < S_top      water rising in the wedge between river and
//                            levee, nothing behind it;
//   otherwise                no levee effect.
// Only the selected regime's formulas are evaluated.
//
// Scalar types: S storage, R state-derived quantities, G what depends on
// the river geometry (width, height), P static inputs (length, area, levee
// parameters, table depths).
// ---------------------------------------------------------------------------
// Which regime a levee partition took; a caller that keeps the cell's fields
// in memory stores only what that regime changed (river storage, depths and
// flooded fraction pass through unchanged below the banks, below the levee
// base and when overtopped; the flood storage also below the base).
enum LeveeRegime : int {
    kLeveeBelowBank = 0,  // sets ps, pdep
    kLeveeOvertopped,     // sets fs, ps, pdep (reads rs, fs, fdep)
    kLeveeFilling,        // sets every field
    kLeveeWedge,          // sets every field
    kLeveeNoEffect,       // sets ps, pdep
};

template <typename S, typename R>
struct LeveeState {
    S rs, fs, ps;            // river / flood / protected storage
    R rdep, fdep, pdep, ffr; // river / flood / protected depth, flooded fraction
};

// The levee arithmetic is written with contraction-fixed operations (xfma,
// xmul, xadd, xsub, xdiv): its storages pass through several case branches,
// and fixing each rounding keeps the results independent of how the compiler
// arranges them.  Each xfma stands where the reference kernel's compiled
// code fuses the product into the sum; the protected depth above the fill
// point is a separately rounded product and sum (levee.cu:196-202), which the
// bit-exact parity runs against the reference kernels pin down.

// Profile storage up to height z inside the layer [d_lo, d_lo + dh] that
// starts at storage s_lo and width w_lo: the trapezoid of the partial layer,
// its width grown linearly with height.
template <typename G, typename P>
__device__ __forceinline__ G levee_partial_storage(G s_lo, G w_lo, P d_lo, P dh, P dw, P len, P z)
{
    const P r = xdiv(xsub(z, d_lo), dh);
    const G w_mid = xfma(G(xmul(P(0.5), r)), G(dw), w_lo);
    return xfma(xmul(G(len), w_mid), G(xmul(r, dh)), s_lo);
}

// One layer of the levee scheme's walk: storage at its top and the running
// width after it.
template <typename G, typename P>
__device__ __forceinline__ G levee_layer_top(G s_lo, G w_lo, P dh, P dw, P len)
{
    return xfma(xmul(G(len), xfma(G(P(0.5)), G(dw), w_lo)), G(dh), s_lo);
}

// Storage that fills the wedge between river and levee from storage s up to
// the crown, over a surface at height z: s + (d + B) (H_c - z) L.
template <typename G, typename P>
__device__ __forceinline__ G wedge_fill(G s, G wedge, P crown, P z, P len)
{
    return xfma(xmul(wedge, G(xsub(crown, z))), G(len), s);
}

// Runs fn(l) for the floodplain layers l = 0, 1, ... until fn returns false
// or the K layers are done.  KR > 0: a row of exactly KR layers held in
// registers, walked fully unrolled (so that fn may index a register array by
// l); KR == 0: any K, a plain loop.
template <int KR, typename Fn>
__device__ __forceinline__ void for_layers(int K, Fn&& fn)
{
    if constexpr (KR > 0) {
#pragma unroll
        for (int l = 0; l < KR; ++l)
            if (!fn(l)) return;
    } else {
        for (int l = 0; l < K; ++l)
            if (!fn(l)) return;
    }
}

// What the levee partition needs beyond a cell's flood-stage result: the
// regime storages of its levee and the layer geometry.  They depend on the
// river geometry, the floodplain row and the levee alone, so a plan whose
// geometry is shared by all members computes them once (levee_marks_of) and
// every sub-step reads them.
template <typename G, typename P>
struct LeveeMarks {
    G s_base;   // profile filled up to the levee base
    G s_crown;  // profile filled up to the crown
    G s_top;    // S_base plus the river-side wedge up to the crown
    G s_first;  // the wedge over the base as the protected-side walk sees it
                // at its first layer (the base storage once the base layer
                // is reached, the bank storage before)
    P dw;       // width step of a layer
    P dist;     // levee distance from the bank
};

template <int KR, typename G, typename P, typename Depth>
__device__ __forceinline__ LeveeMarks<G, P> levee_marks_of(G width, G height, P len, P area,
                                                           P crown, P frac, P base, int K,
                                                           Depth depth_at)
{
    LeveeMarks<G, P> m;
    const G bank = xmul(xmul(G(len), width), height);
    const P span = xdiv(area, len);
    m.dw = xdiv(span, P(K));
    m.dist = xmul(frac, span);
    int base_layer = K;
    bool have_base = false, have_crown = false;
    G s = bank, w = width;
    P d = P(0);
    for_layers<KR>(K, [&](int l) -> bool {
        if (have_base && have_crown) return false;
        const P top = depth_at(l);
        const P dh = smax(xsub(top, d), P(1e-6));
        if (!have_base && base > d && base <= top) {
            m.s_base = levee_partial_storage(s, w, d, dh, m.dw, len, base);
            base_layer = l;
            have_base = true;
        }
        if (!have_crown && crown > d && crown <= top) {
            m.s_crown = levee_partial_storage(s, w, d, dh, m.dw, len, crown);
            have_crown = true;
        }
        s = levee_layer_top(s, w, dh, m.dw, len);
        d = top;
        w = xadd(w, G(m.dw));
        return true;
    });
    // heights above the table extend the top layer's width vertically; a
    // height at or below the bank marks the bank
    if (!have_base) m.s_base = (base > d) ? xfma(xmul(G(len), w), G(xsub(base, d)), s) : bank;
    if (!have_crown) m.s_crown = (crown > d) ? xfma(xmul(G(len), w), G(xsub(crown, d)), s) : bank;
    const G wedge = xadd(G(m.dist), width);
    m.s_top = wedge_fill(m.s_base, wedge, crown, base, len);
    const int first = (int)xmul(frac, P(K));
    m.s_first = wedge_fill(base_layer <= first ? m.s_base : bank, wedge, crown, base, len);
    return m;
}

// Protected side while the river side stands at the crown.  From layer
// `first` = floor(frac K) on, the storage that raises the protected surface to
// the top of layer l is the profile storage there plus the river-side wedge
// above it up to the crown; the first layer whose threshold exceeds the total
// storage holds the protected surface; the fill point below it is the
// previous layer's threshold (at `first` itself: s_first).
template <typename G, typename P>
struct ProtectedFill {
    bool inside;  // the surface lies inside the table
    G s_fill;     // storage at the fill point
    P w_fill;     // protected width at the fill point, from the levee
    P d_fill;     // protected depth at the fill point, above the base
    P grad;       // depth gradient of the layer holding the surface
};

template <int KR, typename G, typename P, typename V, typename Depth>
__device__ __forceinline__ ProtectedFill<G, P> protected_fill(V total, G bank, G width, P len,
                                                              P dw, int K, int first, P crown,
                                                              P base, P dist, G s_first,
                                                              Depth depth_at)
{
    ProtectedFill<G, P> f{false, G(0), P(0), P(0), P(0)};
    if (first >= K) return f;
    f.s_fill = s_first;
    const G wedge = xadd(G(dist), width);
    G s = bank, w = width;
    P d = P(0);
    for_layers<KR>(K, [&](int l) -> bool {
        const P top = depth_at(l);
        const P dh = smax(xsub(top, d), P(1e-6));
        s = levee_layer_top(s, w, dh, dw, len);
        if (l >= first) {
            const G threshold = wedge_fill(s, wedge, crown, top, len);
            if (val(total) < val(threshold)) {
                f.inside = true;
                f.grad = xdiv(dh, dw);
                return false;
            }
            f.s_fill = threshold;
            f.w_fill = xfma(dw, P(l + 1), -dist);
            f.d_fill = xsub(top, base);
        }
        d = top;
        w = xadd(w, G(dw));
        return true;
    });
    return f;
}

// The partition itself, on the levee's marks; the floodplain row is read
// only when the protected side is filling.
template <int KR, typename S, typename R, typename G, typename P, typename Depth>
__device__ __forceinline__ int levee_apply(LeveeState<S, R>& st, const LeveeMarks<G, P>& mk,
                                            G width, G height, P len, P crown, P frac, P base,
                                            int K, Depth depth_at)
{
    const S total_s = st.rs + st.fs;
    const R total = narrow<R>(total_s);
    const G len_w = xmul(G(len), width);
    const G bank = xmul(len_w, height);
    if (!(val(total) >= val(bank))) {
        st.ps = S(0);
        st.pdep = R(0);
        return kLeveeBelowBank;
    }
    const G wedge = xadd(G(mk.dist), width);
    if (val(total) >= val(mk.s_crown)) {
        // overtopped: river and flood stage stand; the protected side takes
        // what the floodplain holds beyond the wedge at the flood depth
        const S remaining = pos_part(total_s - st.rs);
        const R at_depth = xfma(xmul(R(xsub(st.fdep, R(crown))), R(wedge)), R(len), R(mk.s_top));
        const R outside = smax(xsub(at_depth, narrow<R>(st.rs)), R(0));
        const S fs = smin(pos_part(static_cast<S>(outside)), remaining);
        st.ps = pos_part(remaining - fs);
        st.fs = fs;
        st.pdep = st.fdep;
        return kLeveeOvertopped;
    }
    if (val(total) >= val(mk.s_top)) {
        // river side at the crown, the protected side filling
        const G column = xfma(len_w, G(crown), bank);
        const S rs = smin(static_cast<S>(column), total_s);
        const S remaining = pos_part(total_s - rs);
        const G outside = smax(xsub(mk.s_top, column), G(0));
        const S fs = smin(pos_part(static_cast<S>(outside)), remaining);
        const int first = (int)xmul(frac, P(K));
        const ProtectedFill<G, P> pf = protected_fill<KR>(total, bank, width, len, mk.dw, K, first,
                                                          crown, base, mk.dist, mk.s_first,
                                                          depth_at);
        const R extra = xsub(total, R(pf.s_fill));
        const P raised = xadd(base, pf.d_fill);
        R pdep, pfrac;
        if (pf.inside) {
            const R q = xfma(R(pf.w_fill), R(pf.w_fill),
                             xdiv(xdiv(xmul(R(P(2)), extra), R(len)), R(xadd(pf.grad, P(1e-9)))));
            const R w_add = xadd(R(-pf.w_fill), ssqrt(smax(q, R(0))));
            pdep = xadd(R(raised), xmul(w_add, R(pf.grad)));
            pfrac = R(xdiv(xadd(pf.w_fill, mk.dist), xmul(mk.dw, P(K))));
        } else {
            pdep = xadd(R(raised), xdiv(extra, R(xfma(pf.w_fill, len, P(1e-9)))));
            pfrac = R(1);
        }
        st.rs = rs;
        st.fs = fs;
        st.ps = pos_part(remaining - fs);
        st.rdep = R(xdiv(xdiv(column, G(len)), width));
        st.fdep = R(crown);
        st.pdep = pdep;
        st.ffr = smin(smax(pfrac, R(0)), R(1));
        return kLeveeFilling;
    }
    if (val(total) >= val(mk.s_base)) {
        // water rising in the wedge between the river and the levee
        const R fdep = xadd(R(base), xdiv(xdiv(xsub(total, R(mk.s_base)), R(wedge)), R(len)));
        const R column = xfma(R(len_w), fdep, R(bank));
        const S rs = smin(static_cast<S>(column), total_s);
        const S remaining = pos_part(total_s - rs);
        st.rs = rs;
        st.fs = remaining;
        st.ps = pos_part(remaining - remaining);
        st.rdep = xdiv(xdiv(column, R(len)), R(width));
        st.fdep = fdep;
        st.pdep = R(0);
        st.ffr = R(frac);
        return kLeveeWedge;
    }
    // below the levee base: no levee effect
    const S remaining = pos_part(total_s - st.rs);
    st.ps = pos_part(remaining - st.fs);
    st.pdep = R(0);
    return kLeveeNoEffect;
}

// Marks and partition in one call (geometry that varies by member, the
// adjoint).  A cell below its banks needs neither.
template <int KR, typename S, typename R, typename G, typename P, typename Depth>
__device__ __forceinline__ int levee_partition(LeveeState<S, R>& st, G width, G height, P len,
                                                P area, P crown, P frac, P base, int K,
                                                Depth depth_at)
{
    const R total = narrow<R>(st.rs + st.fs);
    const G bank = xmul(xmul(G(len), width), height);
    if (!(val(total) >= val(bank))) {
        st.ps = S(0);
        st.pdep = R(0);
        return kLeveeBelowBank;
    }
    const LeveeMarks<G, P> mk =
        levee_marks_of<KR>(width, height, len, area, crown, frac, base, K, depth_at);
    return levee_apply<KR>(st, mk, width, height, len, crown, frac, base, K, depth_at);
}

}  // namespace cmf
