// Host side of the C ABI (include/cmfb200.h): view validation, plan binding,
// workspace layout, kernel dispatch and the per-interval CUDA graph.
//
// The interval graph replaces the Python sub-step loop of
// CaMaFlood.step_advance (cmfgpu/models/cama_flood_model.py:104-173) and its
// device->host `.item()` of the sub-step count (:122):
//
//   begin -> [cfl] -> plan (n, dt per member, while-condition)
//         -> WHILE(cond) { momentum -> limit -> stage -> [levee]
//                          (last block of the last of them: k += 1, cond = k < n)
//                          -> [statistics] }
//         -> end (storage copy-back for odd counts, current_step)
//         -> [budget flush]
//
// so a whole forcing interval is one cudaGraphLaunch with the sub-step count
// decided on the device.

#include "cmfb200.h"
#include "cmf_device.cuh"

#include <cstdint>
#include <cstring>
#include <cstddef>
#include <mutex>
#include <new>

using namespace cmf;

namespace {

constexpr int kDefaultBlock = 256;

struct KernelSet {
    const void* momentum;
    const void* stage;
    const void* cfl;
    const void* begin;
    const void* plan;
    const void* end;
    const void* copy_back;
    const void* limit;
    const void* levee;
    const void* stats_acc;
    const void* stats_reset;
    const void* stats_fin;
    const void* persist;  // persistent interval kernel (one member, no budget), else null
};

template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF, bool BUD>
KernelSet make_set()
{
    KernelSet k;
    k.momentum = (const void*)k_momentum<REAL, ONE, RES, LEV, BIF>;
    k.stage = (const void*)k_stage<REAL, ONE, RES, LEV, BIF, BUD>;
    k.cfl = (const void*)k_cfl<REAL, ONE, RES>;
    k.begin = (const void*)k_interval_begin<REAL>;
    k.plan = (const void*)k_interval_plan<REAL>;
    k.end = (const void*)k_interval_end<REAL, ONE>;
    k.copy_back = (const void*)k_copy_back<REAL, ONE>;
    k.limit = (const void*)k_limit<REAL, ONE, BIF>;
    k.levee = (const void*)k_levee<REAL, ONE>;
    k.stats_acc = (const void*)k_stats_accumulate<REAL, ONE>;
    k.stats_reset = (const void*)k_stats_reset<REAL, ONE>;
    k.stats_fin = (const void*)k_stats_finalize<REAL, ONE>;
    if constexpr (ONE && !BUD) k.persist = (const void*)k_persistent<REAL, RES, LEV, BIF>;
    else k.persist = nullptr;
    return k;
}

template <typename REAL, bool ONE, bool RES, bool LEV, bool BIF>
KernelSet pick_bud(bool bud)
{
    return bud ? make_set<REAL, ONE, RES, LEV, BIF, true>() : make_set<REAL, ONE, RES, LEV, BIF, false>();
}
template <typename REAL, bool ONE, bool RES, bool LEV>
KernelSet pick_bif(bool bif, bool bud)
{
    return bif ? pick_bud<REAL, ONE, RES, LEV, true>(bud) : pick_bud<REAL, ONE, RES, LEV, false>(bud);
}
template <typename REAL, bool ONE, bool RES>
KernelSet pick_lev(bool lev, bool bif, bool bud)
{
    return lev ? pick_bif<REAL, ONE, RES, true>(bif, bud) : pick_bif<REAL, ONE, RES, false>(bif, bud);
}
template <typename REAL, bool ONE>
KernelSet pick_res(bool res, bool lev, bool bif, bool bud)
{
    return res ? pick_lev<REAL, ONE, true>(lev, bif, bud) : pick_lev<REAL, ONE, false>(lev, bif, bud);
}
template <typename REAL>
KernelSet pick_one(bool one, bool res, bool lev, bool bif, bool bud)
{
    return one ? pick_res<REAL, true>(res, lev, bif, bud) : pick_res<REAL, false>(res, lev, bif, bud);
}

inline size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
    size_t qu, lrs, bsum, braw, rs1, fs1, bpart, ctl, tsec;
    size_t base_total;  // the regions every caller needs
    // levee-indexed copies that plans keep (after base_total; none without levees)
    size_t lpk_tbl, lpk_geo, lmk;
    size_t total;
};

Layout layout_of(const CmfView* v, int cell_blocks)
{
    const size_t real = (v->features & CMF_FEAT_FP64) ? 8 : 4;
    const size_t nm = (size_t)v->num_catchments * (size_t)v->num_members;
    const size_t pm = (size_t)v->num_bifurcation_paths * (size_t)v->num_members;
    Layout L;
    size_t o = 0;
    L.qu = o; o = align_up(o + 2 * nm * real);
    L.lrs = o; o = align_up(o + nm * real);
    L.bsum = o; o = align_up(o + pm * real);
    L.braw = o; o = align_up(o + pm * real);
    L.rs1 = o; o = align_up(o + nm * 8);
    L.fs1 = o; o = align_up(o + nm * 8);
    L.bpart = o; o = align_up(o + (size_t)kBudgetTerms * (size_t)cell_blocks * 8);
    L.ctl = o; o = align_up(o + 16 * sizeof(int));
    L.tsec = o; o = align_up(o + 8);
    L.base_total = o;
    const size_t nlv = (v->features & CMF_FEAT_LEVEE) ? (size_t)v->num_levees : 0;
    L.lpk_tbl = o; o = align_up(o + nlv * (size_t)v->num_flood_levels * real);
    L.lpk_geo = o; o = align_up(o + 3 * nlv * real);
    L.lmk = o; o = align_up(o + 6 * nlv * real);
    L.total = o;
    return L;
}

int block_of(const CmfView* v)
{
    int b = v->block_size > 0 ? v->block_size : kDefaultBlock;
    if (b > 256) b = 256;  // kernels are compiled with __launch_bounds__(256)
    if (b < 32) b = 32;
    return (b / 32) * 32;
}

int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace

struct CmfPlan {
    CmfView view;
    bool fp64;
    bool one;
    bool adaptive;
    bool graph_enabled;
    KernelSet ks;
    alignas(16) unsigned char dev[sizeof(Dev<double>)];
    int tpb;
    int cell_blocks;
    int path_blocks;
    int levee_blocks;
    int layout_blocks;  // cell_blocks the workspace layout was made with (member tile 1)
    int mtile;          // member-tile width of the batched kernels
    // graph
    bool graph_ready;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    cudaGraphNode_t begin_node;
    cudaGraphNode_t plan_node;
    cudaGraphConditionalHandle cond;
    double graph_T;
    int graph_fixed;
    // output statistics folded in after every sub-step (count == 0: none)
    StatsArgs stats;
    // persistent interval kernel instead of the interval graph
    bool persistent;
    int persist_grid;
};

namespace {

// packed: bind the levee-indexed copies (plans); the allocation-free entry
// leaves them null, and k_levee then reads the cell-indexed fields.
template <typename REAL>
void fill_dev(CmfPlan* p, const Layout& L, bool packed)
{
    const CmfView& v = p->view;
    Dev<REAL> d;
    std::memset(&d, 0, sizeof(d));
    char* ws = (char*)v.workspace;
    d.N = (long)v.num_catchments;
    d.M = v.num_members;
    d.mshift = -1;
    d.mtile = p->mtile > 0 ? p->mtile : 1;
    for (int b = 0; b < 31; ++b)
        if (v.num_members == (1 << b)) d.mshift = b;
    d.K = v.num_flood_levels;
    d.P = (long)v.num_bifurcation_paths;
    d.L = v.num_bifurcation_levels;
    d.batched = v.batched_mask;
    d.features = v.features;
    d.g = (REAL)v.gravity;
    d.min_kin = (REAL)v.min_kinematic_slope;
    d.cfl_alpha = (REAL)v.adaptive_time_factor;
    d.max_dt = (REAL)v.max_sub_step_seconds;
    d.max_sub_cap = v.max_sub_steps_cap;
    d.cell_blocks = p->cell_blocks;
    d.path_blocks = p->path_blocks;
    d.dn = v.downstream_idx;
    d.up = v.upstream_ptr;
    d.flags = v.cell_flags;
    d.lslot = v.levee_slot;
    d.rslot = v.reservoir_slot;
    d.bptr = v.bif_cell_ptr;
    d.bpaths = v.bif_cell_paths;
    d.rw = (const REAL*)v.river_width;
    d.rl = (const REAL*)v.river_length;
    d.rh = (const REAL*)v.river_height;
    d.celv = (const REAL*)v.catchment_elevation;
    d.ca = (const REAL*)v.catchment_area;
    d.dnd = (const REAL*)v.downstream_distance;
    d.rman = (const REAL*)v.river_manning;
    d.fman = (const REAL*)v.flood_manning;
    d.tbl = (const REAL*)v.flood_depth_table;
    d.runoff = (const REAL*)v.runoff;
    d.rout = (REAL*)v.river_outflow;
    d.fout = (REAL*)v.flood_outflow;
    d.rdep = (REAL*)v.river_depth;
    d.fdep = (REAL*)v.flood_depth;
    d.pdep = (REAL*)v.protected_depth;
    d.rcsd = (REAL*)v.river_cross_section_depth;
    d.fcsd = (REAL*)v.flood_cross_section_depth;
    d.fcsa = (REAL*)v.flood_cross_section_area;
    d.ffr = (REAL*)v.flood_fraction;
    d.rs0 = v.river_storage;
    d.fs0 = v.flood_storage;
    d.rs1 = (double*)(ws + L.rs1);
    d.fs1 = (double*)(ws + L.fs1);
    d.ps = v.protected_storage;
    d.rinf = v.river_inflow;
    d.finf = v.flood_inflow;
    d.tsto = v.total_storage;
    d.gbif = v.global_bifurcation_outflow;
    d.lr = (REAL*)v.limit_rate;
    d.wse = (REAL*)v.water_surface_elevation;
    d.pwse = (REAL*)v.protected_water_surface_elevation;
    d.bci = v.bifurcation_catchment_idx;
    d.bdi = v.bifurcation_downstream_idx;
    d.bman = (const REAL*)v.bifurcation_manning;
    d.bwid = (const REAL*)v.bifurcation_width;
    d.blen = (const REAL*)v.bifurcation_length;
    d.belv = (const REAL*)v.bifurcation_elevation;
    d.bout = (REAL*)v.bifurcation_outflow;
    d.bcsd = (REAL*)v.bifurcation_cross_section_depth;
    d.bsum = (REAL*)(ws + L.bsum);
    d.braw = (REAL*)(ws + L.braw);
    d.NLV = (v.features & CMF_FEAT_LEVEE) ? (long)v.num_levees : 0;
    d.lci = v.levee_catchment_idx;
    d.lcrown = (const REAL*)v.levee_crown_height;
    d.lfrac = (const REAL*)v.levee_fraction;
    d.lbase = (const REAL*)v.levee_base_height;
    d.rcons = (const REAL*)v.conservation_volume;
    d.remerg = (const REAL*)v.emergency_volume;
    d.radj = (const REAL*)v.adjustment_volume;
    d.rnout = (const REAL*)v.effective_normal_outflow;
    d.raout = (const REAL*)v.adjustment_outflow;
    d.rfcout = (const REAL*)v.flood_control_outflow;
    d.rti = v.reservoir_total_inflow;
    d.dt = (REAL*)v.time_step;
    d.outer = (REAL*)v.outer_time_step;
    d.nsub = v.max_sub_steps;
    d.cur = v.current_step;
    d.ctl = (int*)(ws + L.ctl);
    d.tsec = (double*)(ws + L.tsec);
    d.budget = v.budget;
    d.bpart = (double*)(ws + L.bpart);
    d.status = v.status;
    d.qu = (pair_t<REAL>*)(ws + L.qu);
    d.lrs = (REAL*)(ws + L.lrs);
    if (packed && d.NLV > 0) {
        d.lpk_tbl = (REAL*)(ws + L.lpk_tbl);
        const int geo = CMF_BATCH_RIVER_HEIGHT | CMF_BATCH_RIVER_WIDTH | CMF_BATCH_RIVER_LENGTH;
        if (!(v.batched_mask & geo)) {
            d.lpk_geo = (REAL*)(ws + L.lpk_geo);
            d.lmk = (REAL*)(ws + L.lmk);
        }
    }
    std::memcpy(p->dev, &d, sizeof(d));
}

int check_cuda(cudaError_t e) { return e == cudaSuccess ? CMF_OK : CMF_ERR_CUDA; }

int launch(const void* fn, int grid, int block, void** args, cudaStream_t s)
{
    if (grid <= 0) return CMF_OK;
    return check_cuda(cudaLaunchKernel(fn, dim3(grid), dim3(block), args, 0, s));
}

int validate(const CmfView* v)
{
    if (!v) return CMF_ERR_ARG;
    if (v->abi_version != CMF_ABI_VERSION) return CMF_ERR_ARG;
    if (v->num_catchments <= 0 || v->num_members <= 0 || v->num_flood_levels <= 0)
        return CMF_ERR_ARG;
    if ((long double)v->num_catchments * v->num_members >= (long double)INT32_MAX * 64)
        return CMF_ERR_ARG;
    if (!v->downstream_idx || !v->upstream_ptr || !v->cell_flags) return CMF_ERR_ARG;
    const void* base[] = {v->river_width, v->river_length, v->river_height,
                          v->catchment_elevation, v->catchment_area, v->downstream_distance,
                          v->river_manning, v->flood_manning, v->flood_depth_table, v->runoff,
                          v->river_outflow, v->flood_outflow, v->river_depth, v->flood_depth,
                          v->protected_depth, v->river_cross_section_depth,
                          v->flood_cross_section_depth, v->flood_cross_section_area,
                          v->flood_fraction, v->river_storage, v->flood_storage,
                          v->protected_storage, v->time_step, v->outer_time_step,
                          v->max_sub_steps, v->current_step, v->status, v->workspace};
    for (const void* q : base)
        if (!q) return CMF_ERR_ARG;
    if (v->features & CMF_FEAT_BIFURCATION) {
        if (v->num_bifurcation_paths <= 0 || v->num_bifurcation_levels <= 0) return CMF_ERR_ARG;
        if (v->num_bifurcation_levels > kMaxBifLevels) return CMF_ERR_UNSUPPORTED;
        const void* b[] = {v->bif_cell_ptr, v->bif_cell_paths, v->bifurcation_catchment_idx,
                           v->bifurcation_downstream_idx, v->bifurcation_manning,
                           v->bifurcation_width, v->bifurcation_length,
                           v->bifurcation_elevation, v->bifurcation_outflow,
                           v->bifurcation_cross_section_depth};
        for (const void* q : b)
            if (!q) return CMF_ERR_ARG;
    }
    if (v->features & CMF_FEAT_LEVEE) {
        if (!v->levee_slot || !v->levee_crown_height || !v->levee_fraction ||
            !v->levee_base_height || !v->levee_catchment_idx || v->num_levees < 0)
            return CMF_ERR_ARG;
    }
    if (v->features & CMF_FEAT_RESERVOIR) {
        const void* r[] = {v->reservoir_slot, v->conservation_volume, v->emergency_volume,
                           v->adjustment_volume, v->effective_normal_outflow,
                           v->adjustment_outflow, v->flood_control_outflow,
                           v->reservoir_total_inflow};
        for (const void* q : r)
            if (!q) return CMF_ERR_ARG;
    }
    if ((v->features & CMF_FEAT_BUDGET) && !v->budget) return CMF_ERR_ARG;
    return CMF_OK;
}

int add_kernel(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps,
               const void* fn, int grid, int block, void** args)
{
    cudaKernelNodeParams kp;
    std::memset(&kp, 0, sizeof(kp));
    kp.func = (void*)fn;
    kp.gridDim = dim3(grid > 0 ? grid : 1);
    kp.blockDim = dim3(block);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    kp.extra = nullptr;
    return check_cuda(cudaGraphAddKernelNode(node, g, deps, ndeps, &kp));
}

// Dependency edge between two sub-step kernels of the interval graph.
int add_edge(cudaGraph_t g, cudaGraphNode_t from, cudaGraphNode_t to)
{
    return check_cuda(cudaGraphAddDependencies(g, &from, &to, 1));
}

int build_graph(CmfPlan* p, double T, int fixed_n)
{
    const CmfView& v = p->view;
    int rc;
    cudaGraph_t g;
    if ((rc = check_cuda(cudaGraphCreate(&g, 0))) != CMF_OK) return rc;
    cudaGraphConditionalHandle h;
    if ((rc = check_cuda(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault))) != CMF_OK) {
        cudaGraphDestroy(g);
        return rc;
    }
    const int adaptive = (fixed_n <= 0) ? 1 : 0;
    cudaGraphNode_t nbegin, ncfl, nplan, nwhile, nend, nflush;
    {
        int a = adaptive;
        void* args[] = {p->dev, &T, &a};
        if ((rc = add_kernel(&nbegin, g, nullptr, 0, p->ks.begin, 1, 32, args)) != CMF_OK) goto fail;
    }
    cudaGraphNode_t prev;
    prev = nbegin;
    if (adaptive) {
        const int cfl_blocks = ceil_div((long)v.num_catchments * v.num_members, p->tpb);
        void* args[] = {p->dev};
        if ((rc = add_kernel(&ncfl, g, &prev, 1, p->ks.cfl, cfl_blocks, p->tpb, args)) != CMF_OK) goto fail;
        prev = ncfl;
    }
    {
        int f = fixed_n;
        int set = 1;
        void* args[] = {p->dev, &f, &h, &set};
        if ((rc = add_kernel(&nplan, g, &prev, 1, p->ks.plan, 1, 256, args)) != CMF_OK) goto fail;
    }
    {
        // cudaGraphNodeParams has no default constructor (it holds a union);
        // zero-initialise raw storage instead.
        alignas(cudaGraphNodeParams) unsigned char cp_raw[sizeof(cudaGraphNodeParams)];
        std::memset(cp_raw, 0, sizeof(cp_raw));
        cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_raw);
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        if ((rc = check_cuda(cudaGraphAddNode(&nwhile, g, &nplan, 1, &cp))) != CMF_OK) goto fail;
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        const int grid = p->cell_blocks + p->path_blocks;
        cudaGraphNode_t b1, bl, b2;
        int kh = -1, fd = 0;
        void* a1[] = {p->dev, &kh, &fd};
        if ((rc = add_kernel(&b1, body, nullptr, 0, p->ks.momentum, grid, p->tpb, a1)) != CMF_OK) goto fail;
        void* al[] = {p->dev, &kh};
        if ((rc = add_kernel(&bl, body, nullptr, 0, p->ks.limit, p->cell_blocks, p->tpb, al)) != CMF_OK)
            goto fail;
        if ((rc = add_edge(body, b1, bl)) != CMF_OK) goto fail;
        int set = 1;
        void* a2[] = {p->dev, &kh, &fd, &h, &set};
        if ((rc = add_kernel(&b2, body, nullptr, 0, p->ks.stage, grid, p->tpb, a2)) != CMF_OK) goto fail;
        if ((rc = add_edge(body, bl, b2)) != CMF_OK) goto fail;
        cudaGraphNode_t last = b2;
        if (p->levee_blocks > 0) {
            cudaGraphNode_t b3;
            int adv = 1;
            void* a3[] = {p->dev, &kh, &fd, &h, &adv};
            if ((rc = add_kernel(&b3, body, nullptr, 0, p->ks.levee, p->levee_blocks, p->tpb, a3)) != CMF_OK)
                goto fail;
            if ((rc = add_edge(body, b2, b3)) != CMF_OK) goto fail;
            last = b3;
        }
        if (p->stats.count > 0) {
            // after the advancing kernel: reads step counter - 1
            cudaGraphNode_t b4;
            void* a4[] = {p->dev, &p->stats, &kh};
            const int sb = ceil_div((long)v.num_catchments * v.num_members, 256);
            if ((rc = add_kernel(&b4, body, &last, 1, p->ks.stats_acc, sb, 256, a4)) != CMF_OK) goto fail;
        }
    }
    {
        const int eb = ceil_div((long)v.num_catchments * v.num_members, 256);
        void* args[] = {p->dev};
        if ((rc = add_kernel(&nend, g, &nwhile, 1, p->ks.end, eb, 256, args)) != CMF_OK) goto fail;
    }
    if (v.features & CMF_FEAT_BUDGET) {
        Layout L = layout_of(&v, p->layout_blocks);
        double* bpart = (double*)((char*)v.workspace + L.bpart);
        int* ctl = (int*)((char*)v.workspace + L.ctl);
        double* budget = v.budget;
        int nb = p->cell_blocks;
        int cs = 1;
        void* args[] = {&bpart, &nb, &budget, &ctl, &cs};
        if ((rc = add_kernel(&nflush, g, &nend, 1, (const void*)k_budget_flush, 1, 256, args)) != CMF_OK) goto fail;
    }
    cudaGraphExec_t exec;
    if ((rc = check_cuda(cudaGraphInstantiate(&exec, g, 0))) != CMF_OK) goto fail;
    p->graph = g;
    p->exec = exec;
    p->begin_node = nbegin;
    p->plan_node = nplan;
    p->cond = h;
    p->graph_T = T;
    p->graph_fixed = fixed_n;
    p->graph_ready = true;
    return CMF_OK;
fail:
    cudaGraphDestroy(g);
    return rc;
}

void destroy_graph(CmfPlan* p)
{
    if (!p->graph_ready) return;
    cudaGraphExecDestroy(p->exec);
    cudaGraphDestroy(p->graph);
    p->graph_ready = false;
}

int interval_direct(CmfPlan* p, cudaStream_t s, double T, int fixed_n)
{
    const CmfView& v = p->view;
    int rc;
    const int adaptive = fixed_n <= 0 ? 1 : 0;
    {
        int a = adaptive;
        void* args[] = {p->dev, &T, &a};
        if ((rc = launch(p->ks.begin, 1, 32, args, s)) != CMF_OK) return rc;
    }
    if (adaptive) {
        void* args[] = {p->dev};
        const int cfl_blocks = ceil_div((long)v.num_catchments * v.num_members, p->tpb);
        if ((rc = launch(p->ks.cfl, cfl_blocks, p->tpb, args, s)) != CMF_OK) return rc;
    }
    {
        int f = fixed_n;
        cudaGraphConditionalHandle h = 0;
        int set = 0;
        void* args[] = {p->dev, &f, &h, &set};
        if ((rc = launch(p->ks.plan, 1, 256, args, s)) != CMF_OK) return rc;
    }
    Layout L = layout_of(&v, p->layout_blocks);
    int* ctl = (int*)((char*)v.workspace + L.ctl);
    int nmax = 0;
    if ((rc = check_cuda(cudaMemcpyAsync(&nmax, ctl + kCtlMaxSteps, sizeof(int),
                                         cudaMemcpyDeviceToHost, s))) != CMF_OK)
        return rc;
    if ((rc = check_cuda(cudaStreamSynchronize(s))) != CMF_OK) return rc;
    if (nmax < 0 || nmax > kHardSubStepCap) return CMF_ERR_NUMERIC;
    const int grid = p->cell_blocks + p->path_blocks;
    for (int k = 0; k < nmax; ++k) {
        int kh = k, fd = 0;
        void* a1[] = {p->dev, &kh, &fd};
        if ((rc = launch(p->ks.momentum, grid, p->tpb, a1, s)) != CMF_OK) return rc;
        void* al[] = {p->dev, &kh};
        if ((rc = launch(p->ks.limit, p->cell_blocks, p->tpb, al, s)) != CMF_OK) return rc;
        cudaGraphConditionalHandle h = 0;
        int set = 0;
        void* a2[] = {p->dev, &kh, &fd, &h, &set};
        if ((rc = launch(p->ks.stage, grid, p->tpb, a2, s)) != CMF_OK) return rc;
        if (p->levee_blocks > 0) {
            if ((rc = launch(p->ks.levee, p->levee_blocks, p->tpb, a2, s)) != CMF_OK) return rc;
        }
        if (p->stats.count > 0) {
            void* a4[] = {p->dev, &p->stats, &kh};
            const int sb = ceil_div((long)v.num_catchments * v.num_members, 256);
            if ((rc = launch(p->ks.stats_acc, sb, 256, a4, s)) != CMF_OK) return rc;
        }
    }
    {
        void* args[] = {p->dev};
        const int eb = ceil_div((long)v.num_catchments * v.num_members, 256);
        if ((rc = launch(p->ks.end, eb, 256, args, s)) != CMF_OK) return rc;
    }
    if (v.features & CMF_FEAT_BUDGET) {
        double* bpart = (double*)((char*)v.workspace + L.bpart);
        double* budget = v.budget;
        int nb = p->cell_blocks;
        int cs = 1;
        void* args[] = {&bpart, &nb, &budget, &ctl, &cs};
        if ((rc = launch((const void*)k_budget_flush, 1, 256, args, s)) != CMF_OK) return rc;
    }
    return CMF_OK;
}

// One interval through the persistent kernel: the prologue kernels, then
// every sub-step in one cooperative launch, then the epilogue.
int interval_persistent(CmfPlan* p, cudaStream_t s, double T, int fixed_n)
{
    const CmfView& v = p->view;
    int rc;
    const int adaptive = fixed_n <= 0 ? 1 : 0;
    {
        int a = adaptive;
        void* args[] = {p->dev, &T, &a};
        if ((rc = launch(p->ks.begin, 1, 32, args, s)) != CMF_OK) return rc;
    }
    if (adaptive) {
        void* args[] = {p->dev};
        const int cfl_blocks = ceil_div((long)v.num_catchments * v.num_members, p->tpb);
        if ((rc = launch(p->ks.cfl, cfl_blocks, p->tpb, args, s)) != CMF_OK) return rc;
    }
    {
        int f = fixed_n;
        cudaGraphConditionalHandle h = 0;
        int set = 0;
        void* args[] = {p->dev, &f, &h, &set};
        if ((rc = launch(p->ks.plan, 1, 256, args, s)) != CMF_OK) return rc;
    }
    {
        void* args[] = {p->dev};
        if ((rc = check_cuda(cudaLaunchCooperativeKernel(p->ks.persist, dim3(p->persist_grid),
                                                          dim3(p->tpb), args, 0, s))) != CMF_OK)
            return rc;
    }
    void* args[] = {p->dev};
    const int eb = ceil_div((long)v.num_catchments * v.num_members, 256);
    return launch(p->ks.end, eb, 256, args, s);
}

}  // namespace

extern "C" {

int cmf_abi_version(void) { return CMF_ABI_VERSION; }

const char* cmf_status_string(int code)
{
    switch (code) {
        case CMF_OK: return "ok";
        case CMF_ERR_ARG: return "invalid argument";
        case CMF_ERR_CUDA: return "CUDA runtime error";
        case CMF_ERR_TIMEOUT: return "device wait timed out";
        case CMF_ERR_NUMERIC: return "non-finite value produced";
        case CMF_ERR_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

size_t cmf_view_size(void) { return sizeof(CmfView); }

int cmf_view_field_offsets(int64_t* out, int cap)
{
#define OFF(f) offsetof(CmfView, f)
    const size_t offs[] = {
        OFF(abi_version), OFF(features), OFF(num_catchments), OFF(num_members),
        OFF(num_flood_levels), OFF(num_bifurcation_paths), OFF(num_bifurcation_levels),
        OFF(batched_mask), OFF(num_levees), OFF(num_reservoirs), OFF(gravity),
        OFF(min_kinematic_slope), OFF(adaptive_time_factor), OFF(max_sub_step_seconds),
        OFF(max_sub_steps_cap), OFF(block_size), OFF(downstream_idx), OFF(upstream_ptr),
        OFF(cell_flags), OFF(levee_slot), OFF(reservoir_slot), OFF(bif_cell_ptr),
        OFF(bif_cell_paths), OFF(river_width), OFF(river_length), OFF(river_height),
        OFF(catchment_elevation), OFF(catchment_area), OFF(downstream_distance),
        OFF(river_manning), OFF(flood_manning), OFF(flood_depth_table), OFF(runoff),
        OFF(river_outflow), OFF(flood_outflow), OFF(river_depth), OFF(flood_depth),
        OFF(protected_depth), OFF(river_cross_section_depth), OFF(flood_cross_section_depth),
        OFF(flood_cross_section_area), OFF(flood_fraction), OFF(river_storage),
        OFF(flood_storage), OFF(protected_storage), OFF(river_inflow), OFF(flood_inflow),
        OFF(outgoing_storage), OFF(total_storage), OFF(global_bifurcation_outflow),
        OFF(limit_rate), OFF(water_surface_elevation), OFF(protected_water_surface_elevation),
        OFF(bifurcation_catchment_idx), OFF(bifurcation_downstream_idx),
        OFF(bifurcation_manning), OFF(bifurcation_width), OFF(bifurcation_length),
        OFF(bifurcation_elevation), OFF(bifurcation_outflow),
        OFF(bifurcation_cross_section_depth), OFF(levee_catchment_idx),
        OFF(levee_crown_height), OFF(levee_fraction), OFF(levee_base_height),
        OFF(reservoir_catchment_idx), OFF(conservation_volume), OFF(emergency_volume),
        OFF(adjustment_volume), OFF(effective_normal_outflow), OFF(adjustment_outflow),
        OFF(flood_control_outflow), OFF(reservoir_total_inflow), OFF(time_step),
        OFF(outer_time_step), OFF(max_sub_steps), OFF(current_step), OFF(budget),
        OFF(status), OFF(workspace), OFF(workspace_bytes)};
#undef OFF
    const int n = (int)(sizeof(offs) / sizeof(offs[0]));
    for (int q = 0; q < n && q < cap; ++q) out[q] = (int64_t)offs[q];
    return n;
}

int cmf_workspace_size(const CmfView* v, size_t* bytes)
{
    if (!v || !bytes) return CMF_ERR_ARG;
    if (v->num_catchments <= 0 || v->num_members <= 0) return CMF_ERR_ARG;
    const int tpb = block_of(v);
    const int cb = ceil_div((long)v->num_catchments * v->num_members, tpb);
    *bytes = layout_of(v, cb).total;
    return CMF_OK;
}

int cmf_plan_create(const CmfView* view, CmfPlan** out)
{
    if (!out) return CMF_ERR_ARG;
    *out = nullptr;
    int rc = validate(view);
    if (rc != CMF_OK) return rc;
    size_t need = 0;
    cmf_workspace_size(view, &need);
    if (view->workspace_bytes < need) return CMF_ERR_ARG;
    CmfPlan* p = new (std::nothrow) CmfPlan;
    if (!p) return CMF_ERR_ARG;
    std::memset((void*)p, 0, sizeof(CmfPlan));
    p->view = *view;
    const int f = view->features;
    p->fp64 = f & CMF_FEAT_FP64;
    p->one = view->num_members == 1;
    p->adaptive = f & CMF_FEAT_ADAPTIVE;
    p->graph_enabled = f & CMF_FEAT_GRAPH;
    p->tpb = block_of(view);
    p->mtile = 1;
    p->cell_blocks = ceil_div((long)view->num_catchments * view->num_members, p->tpb);
    p->layout_blocks = p->cell_blocks;
    p->path_blocks = (f & CMF_FEAT_BIFURCATION)
                         ? ceil_div((long)view->num_bifurcation_paths * view->num_members, p->tpb)
                         : 0;
    p->levee_blocks = (f & CMF_FEAT_LEVEE)
                          ? ceil_div((long)view->num_levees * view->num_members, p->tpb)
                          : 0;
    const bool res = f & CMF_FEAT_RESERVOIR, lev = f & CMF_FEAT_LEVEE,
               bif = f & CMF_FEAT_BIFURCATION, bud = f & CMF_FEAT_BUDGET;
    Layout L = layout_of(view, p->layout_blocks);
    if (p->fp64) {
        p->ks = pick_one<double>(p->one, res, lev, bif, bud);
        fill_dev<double>(p, L, true);
    } else {
        p->ks = pick_one<float>(p->one, res, lev, bif, bud);
        fill_dev<float>(p, L, true);
    }
    // clear the control words and budget partials once
    char* ws = (char*)view->workspace;
    if ((rc = check_cuda(cudaMemset(ws + L.bpart, 0, L.tsec + 8 - L.bpart))) != CMF_OK) {
        delete p;
        return rc;
    }
    if (p->levee_blocks > 0) {
        // levee-indexed copies of the static fields k_levee reads and, with a
        // shared river geometry, the levees' marks
        void* args[] = {p->dev};
        const void* fn = p->fp64 ? (const void*)k_levee_pack<double> : (const void*)k_levee_pack<float>;
        rc = launch(fn, ceil_div((long)view->num_levees, 256), 256, args, 0);
        if (rc == CMF_OK) rc = check_cuda(cudaDeviceSynchronize());
        if (rc != CMF_OK) {
            delete p;
            return rc;
        }
    }
    *out = p;
    return CMF_OK;
}

void cmf_plan_destroy(CmfPlan* p)
{
    if (!p) return;
    destroy_graph(p);
    delete p;
}

int cmf_step_interval(CmfPlan* p, void* stream, double outer_seconds, int32_t fixed_sub_steps)
{
    if (!p || !(outer_seconds > 0)) return CMF_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int fixed = p->adaptive ? (fixed_sub_steps > 0 ? fixed_sub_steps : 0)
                            : (fixed_sub_steps > 0 ? fixed_sub_steps : -1);
    if (fixed < 0) return CMF_ERR_ARG;  // fixed mode needs a sub-step count
    if (p->persistent) return interval_persistent(p, s, outer_seconds, fixed);
    if (!p->graph_enabled) return interval_direct(p, s, outer_seconds, fixed);
    int rc;
    const bool adaptive_now = fixed == 0;
    if (p->graph_ready) {
        const bool was_adaptive = p->graph_fixed == 0;
        if (was_adaptive != adaptive_now) destroy_graph(p);
    }
    if (!p->graph_ready) {
        if ((rc = build_graph(p, outer_seconds, fixed)) != CMF_OK) return rc;
    } else {
        if (p->graph_T != outer_seconds) {
            int a = adaptive_now ? 1 : 0;
            double T = outer_seconds;
            void* args[] = {p->dev, &T, &a};
            cudaKernelNodeParams kp;
            std::memset(&kp, 0, sizeof(kp));
            kp.func = (void*)p->ks.begin;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(32);
            kp.kernelParams = args;
            if ((rc = check_cuda(cudaGraphExecKernelNodeSetParams(p->exec, p->begin_node, &kp))) != CMF_OK)
                return rc;
            p->graph_T = outer_seconds;
        }
        if (p->graph_fixed != fixed) {
            int fx = fixed;
            cudaGraphConditionalHandle h = p->cond;
            int set = 1;
            void* args[] = {p->dev, &fx, &h, &set};
            cudaKernelNodeParams kp;
            std::memset(&kp, 0, sizeof(kp));
            kp.func = (void*)p->ks.plan;
            kp.gridDim = dim3(1);
            kp.blockDim = dim3(256);
            kp.kernelParams = args;
            if ((rc = check_cuda(cudaGraphExecKernelNodeSetParams(p->exec, p->plan_node, &kp))) != CMF_OK)
                return rc;
            p->graph_fixed = fixed;
        }
    }
    return check_cuda(cudaGraphLaunch(p->exec, s));
}

int cmf_phase_momentum(CmfPlan* p, void* stream, int diag)
{
    if (!p) return CMF_ERR_ARG;
    int kh = -2, fd = diag ? 1 : 2;
    void* args[] = {p->dev, &kh, &fd};
    return launch(p->ks.momentum, p->cell_blocks + p->path_blocks, p->tpb, args,
                  (cudaStream_t)stream);
}

int cmf_phase_stage(CmfPlan* p, void* stream, int diag)
{
    if (!p) return CMF_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int kh = -2, fd = diag ? 1 : 2;
    cudaGraphConditionalHandle h = 0;
    int set = 0;
    void* al[] = {p->dev, &kh};
    int rc = launch(p->ks.limit, p->cell_blocks, p->tpb, al, s);
    if (rc != CMF_OK) return rc;
    void* args[] = {p->dev, &kh, &fd, &h, &set};
    rc = launch(p->ks.stage, p->cell_blocks + p->path_blocks, p->tpb, args, s);
    if (rc != CMF_OK) return rc;
    if (p->levee_blocks > 0) {
        rc = launch(p->ks.levee, p->levee_blocks, p->tpb, args, s);
        if (rc != CMF_OK) return rc;
    }
    void* a2[] = {p->dev};
    return launch(p->ks.copy_back,
                  ceil_div((long)p->view.num_catchments * p->view.num_members, 256), 256, a2, s);
}

int cmf_phase_cfl(CmfPlan* p, void* stream, double outer_seconds)
{
    if (!p || !(outer_seconds > 0)) return CMF_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    {
        int a = 1;
        void* args[] = {p->dev, &outer_seconds, &a};
        if ((rc = launch(p->ks.begin, 1, 32, args, s)) != CMF_OK) return rc;
    }
    {
        void* args[] = {p->dev};
        if ((rc = launch(p->ks.cfl, ceil_div((long)p->view.num_catchments * p->view.num_members, p->tpb),
                         p->tpb, args, s)) != CMF_OK)
            return rc;
    }
    int f = 0;
    cudaGraphConditionalHandle h = 0;
    int set = 0;
    void* args[] = {p->dev, &f, &h, &set};
    return launch(p->ks.plan, 1, 256, args, s);
}

int cmf_phase_fixed_dt(CmfPlan* p, void* stream, double outer_seconds, int32_t n)
{
    if (!p || !(outer_seconds > 0) || n <= 0) return CMF_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    {
        int a = 0;
        void* args[] = {p->dev, &outer_seconds, &a};
        if ((rc = launch(p->ks.begin, 1, 32, args, s)) != CMF_OK) return rc;
    }
    int f = n;
    cudaGraphConditionalHandle h = 0;
    int set = 0;
    void* args[] = {p->dev, &f, &h, &set};
    return launch(p->ks.plan, 1, 256, args, s);
}

int cmf_launch_substep(CmfPlan* p, void* stream, int32_t k, int part)
{
    if (!p || k < 0) return CMF_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = p->cell_blocks + p->path_blocks;
    int kh = k, fd = 0;
    if (part == CMF_PART_MOMENTUM) {
        void* a1[] = {p->dev, &kh, &fd};
        return launch(p->ks.momentum, grid, p->tpb, a1, s);
    }
    if (part == CMF_PART_LIMIT) {
        void* al[] = {p->dev, &kh};
        return launch(p->ks.limit, p->cell_blocks, p->tpb, al, s);
    }
    if (part == CMF_PART_STAGE) {
        cudaGraphConditionalHandle h = 0;
        int set = 0;
        void* a2[] = {p->dev, &kh, &fd, &h, &set};
        return launch(p->ks.stage, grid, p->tpb, a2, s);
    }
    if (part == CMF_PART_LEVEE) {
        if (p->levee_blocks == 0) return CMF_OK;
        cudaGraphConditionalHandle h = 0;
        int set = 0;
        void* a3[] = {p->dev, &kh, &fd, &h, &set};
        return launch(p->ks.levee, p->levee_blocks, p->tpb, a3, s);
    }
    if (part == CMF_PART_END) {
        void* args[] = {p->dev};
        return launch(p->ks.end, ceil_div((long)p->view.num_catchments * p->view.num_members, 256),
                      256, args, s);
    }
    return CMF_ERR_ARG;
}

int cmf_budget_flush(CmfPlan* p, void* stream)
{
    if (!p) return CMF_ERR_ARG;
    if (!(p->view.features & CMF_FEAT_BUDGET)) return CMF_OK;
    Layout L = layout_of(&p->view, p->layout_blocks);
    double* bpart = (double*)((char*)p->view.workspace + L.bpart);
    int* ctl = (int*)((char*)p->view.workspace + L.ctl);
    double* budget = p->view.budget;
    int nb = p->cell_blocks;
    int cs = 0;
    void* args[] = {&bpart, &nb, &budget, &ctl, &cs};
    return launch((const void*)k_budget_flush, 1, 256, args, (cudaStream_t)stream);
}

int cmf_plan_set_persistent(CmfPlan* p, int enable)
{
    if (!p) return CMF_ERR_ARG;
    if (!enable) {
        p->persistent = false;
        return CMF_OK;
    }
    if (!p->ks.persist || p->stats.count > 0) return CMF_ERR_UNSUPPORTED;
    int dev = 0, coop = 0, sms = 0, per_sm = 0;
    int rc;
    if ((rc = check_cuda(cudaGetDevice(&dev))) != CMF_OK) return rc;
    if ((rc = check_cuda(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev))) != CMF_OK) return rc;
    if ((rc = check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) != CMF_OK) return rc;
    if ((rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, p->ks.persist, p->tpb, 0)))
        != CMF_OK)
        return rc;
    if (!coop || per_sm < 1) return CMF_ERR_UNSUPPORTED;
    const CmfView& v = p->view;
    long work = v.num_catchments;
    if (p->path_blocks > 0 && v.num_bifurcation_paths > work) work = v.num_bifurcation_paths;
    if (p->levee_blocks > 0 && v.num_levees > work) work = v.num_levees;
    const int need = ceil_div(work, p->tpb);
    const int resident = per_sm * sms;
    p->persist_grid = need < resident ? (need > 0 ? need : 1) : resident;
    p->persistent = true;
    return CMF_OK;
}

int cmf_probe_barrier_timeout(void* stream, int32_t* control, int32_t* status, int32_t timeout_us)
{
    if (!control || !status || timeout_us <= 0 || timeout_us > 1000000) return CMF_ERR_ARG;
    if (((uintptr_t)control & 7) != 0) return CMF_ERR_ARG;
    int* ctl = control;
    int* st = status;
    unsigned long long ns = (unsigned long long)timeout_us * 1000ull;
    void* args[] = {&ctl, &st, &ns};
    return check_cuda(cudaLaunchCooperativeKernel((const void*)k_barrier_timeout_probe, dim3(2), dim3(32),
                                                  args, 0, (cudaStream_t)stream));
}

int cmf_plan_set_member_tile(CmfPlan* p, int32_t width)
{
    if (!p || width < 1) return CMF_ERR_ARG;
    const int M = p->view.num_members;
    if (M % width != 0 || (M == 1 && width != 1)) return CMF_ERR_ARG;
    if (width == p->mtile) return CMF_OK;
    if (p->graph_ready) {  // the graph's grids change: drop it once no launch is in flight
        const int rc = check_cuda(cudaDeviceSynchronize());
        if (rc != CMF_OK) return rc;
    }
    destroy_graph(p);
    const CmfView& v = p->view;
    const long per_block = (long)p->tpb * width;
    p->mtile = width;
    p->cell_blocks = ceil_div((long)v.num_catchments * M, per_block);
    p->path_blocks = (v.features & CMF_FEAT_BIFURCATION)
                         ? ceil_div((long)v.num_bifurcation_paths * M, per_block) : 0;
    p->levee_blocks = (v.features & CMF_FEAT_LEVEE) ? ceil_div((long)v.num_levees * M, per_block) : 0;
    Layout L = layout_of(&v, p->layout_blocks);
    if (p->fp64) fill_dev<double>(p, L, true);
    else fill_dev<float>(p, L, true);
    return CMF_OK;
}

int cmf_stats_attach(CmfPlan* p, int count, const CmfStatistic* stats, double* weight)
{
    if (!p || count < 0 || count > CMF_MAX_STATISTICS) return CMF_ERR_ARG;
    if (count > 0 && !stats) return CMF_ERR_ARG;
    if (count > 0 && p->persistent) return CMF_ERR_UNSUPPORTED;  // the persistent kernel folds none in
    StatsArgs a;
    std::memset(&a, 0, sizeof(a));
    const bool lev = p->view.features & CMF_FEAT_LEVEE;
    for (int q = 0; q < count; ++q) {
        const int var = stats[q].variable, op = stats[q].op;
        if (var < 0 || var >= CMF_VAR_COUNT || op < CMF_STAT_MEAN || op > CMF_STAT_LAST) return CMF_ERR_ARG;
        if (!stats[q].out) return CMF_ERR_ARG;
        if ((var == CMF_VAR_PROTECTED_DEPTH || var == CMF_VAR_PROTECTED_STORAGE) && !lev)
            return CMF_ERR_ARG;
        a.var[q] = var;
        a.op[q] = op;
        a.out[q] = stats[q].out;
        if (op == CMF_STAT_MEAN) a.need_weight = 1;
    }
    if (a.need_weight && !weight) return CMF_ERR_ARG;
    a.count = count;
    a.weight = weight;
    // the sub-step body changes: drop the graph once no launch of it is in flight
    if (p->graph_ready) {
        const int rc = check_cuda(cudaDeviceSynchronize());
        if (rc != CMF_OK) return rc;
    }
    destroy_graph(p);
    p->stats = a;
    return CMF_OK;
}

int cmf_stats_reset(CmfPlan* p, void* stream)
{
    if (!p) return CMF_ERR_ARG;
    if (p->stats.count == 0) return CMF_OK;
    void* args[] = {p->dev, &p->stats};
    return launch(p->ks.stats_reset, ceil_div((long)p->view.num_catchments * p->view.num_members, 256),
                  256, args, (cudaStream_t)stream);
}

int cmf_stats_accumulate(CmfPlan* p, void* stream, int32_t k)
{
    if (!p || k < 0) return CMF_ERR_ARG;
    if (p->stats.count == 0) return CMF_OK;
    int kh = k;
    void* args[] = {p->dev, &p->stats, &kh};
    return launch(p->ks.stats_acc, ceil_div((long)p->view.num_catchments * p->view.num_members, 256),
                  256, args, (cudaStream_t)stream);
}

int cmf_stats_finalize(CmfPlan* p, void* stream)
{
    if (!p) return CMF_ERR_ARG;
    if (p->stats.count == 0) return CMF_OK;
    void* args[] = {p->dev, &p->stats};
    return launch(p->ks.stats_fin, ceil_div((long)p->view.num_catchments * p->view.num_members, 256),
                  256, args, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free sub-step.
//
// For callers that own all device memory and may not allocate any: code that
// runs inside a stream capture, a host framework whose memory pool hands out
// only the model tensors, or an embedded runtime without cudaMalloc.  The
// scratch that cmf_plan_create would take from a caller workspace lives in a
// fixed static device array instead, sized for at most
// kNoAllocMaxCatchments catchments, kNoAllocMaxPaths bifurcation paths and
// one member (3 MiB, held by every GPU that loads this library until exit).
// ---------------------------------------------------------------------------
namespace {
constexpr long kNoAllocMaxCatchments = 65536;
constexpr long kNoAllocMaxPaths = 8192;
constexpr size_t kNoAllocScratchBytes = 3u << 20;
constexpr int kNoAllocMaxDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
// Device address of g_noalloc_scratch per device (host code may not use the
// symbol itself as a device pointer).  Looked up once per device, with that
// device current, on its first call.
void* g_noalloc_addr[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

int noalloc_scratch(void* stream, void** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return CMF_ERR_CUDA;
    // the kernels run on the stream's device and must get that device's
    // copy of the array: a stream of another device is an argument error
    if (stream) {
        int sdev = -1;
        if (cudaStreamGetDevice((cudaStream_t)stream, &sdev) != cudaSuccess) return CMF_ERR_ARG;
        if (sdev != dev) return CMF_ERR_ARG;
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) return CMF_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void* addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr)
            return CMF_ERR_CUDA;
        g_noalloc_addr[dev] = addr;
    }
    *out = g_noalloc_addr[dev];
    return CMF_OK;
}
}  // namespace

extern "C" int cmf_substep_noalloc(const CmfView* view, void* stream, int diag)
{
    if (!view) return CMF_ERR_ARG;
    if (view->num_members != 1 || view->num_catchments > kNoAllocMaxCatchments) return CMF_ERR_ARG;
    if ((view->features & CMF_FEAT_BIFURCATION) && view->num_bifurcation_paths > kNoAllocMaxPaths)
        return CMF_ERR_ARG;
    void* scratch = nullptr;
    int rc = noalloc_scratch(stream, &scratch);
    if (rc != CMF_OK) return rc;
    CmfView v = *view;
    v.workspace = scratch;
    v.workspace_bytes = kNoAllocScratchBytes;
    if ((rc = validate(&v)) != CMF_OK) return rc;
    // no levee-indexed copies here: only the regions every caller needs
    const size_t need = layout_of(&v, ceil_div((long)v.num_catchments, block_of(&v))).base_total;
    if (need > kNoAllocScratchBytes) return CMF_ERR_ARG;

    // A plan on the stack: kernel set and device view, no graph.
    CmfPlan p;
    std::memset((void*)&p, 0, sizeof(CmfPlan));
    p.view = v;
    const int f = v.features;
    p.fp64 = f & CMF_FEAT_FP64;
    p.one = true;
    p.tpb = block_of(&v);
    p.cell_blocks = ceil_div((long)v.num_catchments, p.tpb);
    p.layout_blocks = p.cell_blocks;
    p.path_blocks = (f & CMF_FEAT_BIFURCATION) ? ceil_div((long)v.num_bifurcation_paths, p.tpb) : 0;
    p.levee_blocks = (f & CMF_FEAT_LEVEE) ? ceil_div((long)v.num_levees, p.tpb) : 0;
    const bool res = f & CMF_FEAT_RESERVOIR, lev = f & CMF_FEAT_LEVEE,
               bif = f & CMF_FEAT_BIFURCATION, bud = f & CMF_FEAT_BUDGET;
    Layout L = layout_of(&v, p.cell_blocks);
    if (p.fp64) {
        p.ks = pick_one<double>(true, res, lev, bif, bud);
        fill_dev<double>(&p, L, false);
    } else {
        p.ks = pick_one<float>(true, res, lev, bif, bud);
        fill_dev<float>(&p, L, false);
    }
    // The array keeps the previous call's contents: clear the control words
    // and the budget partials, which are accumulated rather than overwritten.
    char* ws = (char*)scratch;
    if (cudaMemsetAsync(ws + L.bpart, 0, L.tsec + 8 - L.bpart, (cudaStream_t)stream) != cudaSuccess)
        return CMF_ERR_CUDA;
    if ((rc = cmf_phase_momentum(&p, stream, diag)) != CMF_OK) return rc;
    if ((rc = cmf_phase_stage(&p, stream, diag)) != CMF_OK) return rc;
    if (bud) rc = cmf_budget_flush(&p, stream);
    return rc;
}
