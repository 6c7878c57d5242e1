// Runoff forcing map: gridded runoff -> catchment runoff, on the device.
//
// Replaces the forcing step in front of the routing path: hydroforge's
// `dataset.shard_forcing(runoff_chunk.to(device), local_mapping)` driven by
// scripts/run_daily_bin.py:98-118, with the local mapping built from the
// reference's runoff mapping table (cmfgpu/params/export_bin.py:955-983).
//
// The mapping is a CSR matrix over the model's catchments (rows in model
// order) whose columns are flattened runoff-grid cells and whose weights are
// areas.  One thread owns one catchment row and every series (forcing step x
// member) of the chunk, kSeriesTile series at a time: for each entry of the
// row it issues the tile's grid loads together (one base pointer plus
// compile-time multiples of the step stride), then folds them into one fp64
// accumulator per series in entry order.  The row's entries come from HBM on
// the first tile and from L1 after it.  Output rows are consecutive threads,
// so every store of a series is coalesced; catchments are stored basin by
// basin, so neighbouring threads gather nearby grid cells (L2 hits).
//
// Bytes per launch: row pointers 8 (rows + 1), entries 12 nnz, grid reads of
// the distinct mapped cells per series, one output element per row and
// series.  Bound: HBM on paper; in practice the per-thread chain
// row pointer -> entry -> grid load (one L2 round trip per entry and tile)
// limits it.  No tensor-core work exists in an SpMM with ~2 entries per row.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "cmfb200.h"

namespace {

#ifndef CMF_FORCING_TILE
#define CMF_FORCING_TILE 8
#endif
#ifndef CMF_FORCING_MIN_BLOCKS
#define CMF_FORCING_MIN_BLOCKS 1
#endif
constexpr int kSeriesTile = CMF_FORCING_TILE;  // series (step x member) per register tile
constexpr int kBlock = 256;

struct ForcingArgs {
    long rows;
    long cols;
    const int64_t* row_ptr;
    const int32_t* col;
    const double* weight;
    const void* grid;
    long steps;
    int members;
    long gs_step, gs_member;
    void* out;
    long os_step, os_member, os_row;
    double scale;  // 1 / unit_factor, rounded once on the host
    double missing;
    int* status;
};

template <typename XT>
__device__ __forceinline__ bool is_missing(XT x, XT missing)
{
    return x != x || x == missing;
}

// Offsets of series s -> s + 1 for several members, by additions only:
// (t, m) -> (t, m + 1) or (t + 1, 0).
__device__ __forceinline__ void next_series(const ForcingArgs& a, long& xo, long& oo, int& m)
{
    xo += a.gs_member;
    oo += a.os_member;
    if (++m == a.members) {
        m = 0;
        xo += a.gs_step - (long)a.members * a.gs_member;
        oo += a.os_step - (long)a.members * a.os_member;
    }
}

template <typename XT, bool SKIP>
__device__ __forceinline__ void fold(double& acc, XT x, double w, XT missing)
{
    if (SKIP && is_missing(x, missing)) return;
    acc = __dadd_rn(acc, __dmul_rn((double)x, w));
}

template <typename OT, bool CLAMP>
__device__ __forceinline__ OT finish(double acc, double scale)
{
    double y = __dmul_rn(acc, scale);
    if (CLAMP) y = y < 0.0 ? 0.0 : y;
    return (OT)y;
}

// ONE: a single member, and the host has checked that kSeriesTile forcing
// steps of grid and of output fit 32-bit offsets, so a tile is one 64-bit base
// pointer plus compile-time multiples of the step strides.
template <typename XT, typename OT, bool SKIP, bool CLAMP, bool ONE>
__global__ void __launch_bounds__(kBlock, CMF_FORCING_MIN_BLOCKS) k_forcing_map(const ForcingArgs a)
{
    const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.rows) return;
    const long b = a.row_ptr[r], e = a.row_ptr[r + 1];
    const XT* __restrict__ grid = (const XT*)a.grid;
    OT* __restrict__ out = (OT*)a.out;
    const XT missing = (XT)a.missing;
    bool bad = false;
    if (ONE) {
        const int gs = (int)a.gs_step, os = (int)a.os_step;
        for (long t0 = 0; t0 < a.steps; t0 += kSeriesTile) {
            const XT* __restrict__ g0 = grid + t0 * a.gs_step;
            OT* __restrict__ o0 = out + t0 * a.os_step + r * a.os_row;
            const int nt = a.steps - t0 < kSeriesTile ? (int)(a.steps - t0) : kSeriesTile;
            double acc[kSeriesTile];
#pragma unroll
            for (int j = 0; j < kSeriesTile; ++j) acc[j] = 0.0;
            for (long q = b; q < e; ++q) {
                const int c = a.col[q];
                if (c < 0 || (long)c >= a.cols) {
                    bad = true;
                    continue;
                }
                const double w = a.weight[q];
                const XT* __restrict__ p = g0 + c;
                XT x[kSeriesTile];
#pragma unroll
                for (int j = 0; j < kSeriesTile; ++j) x[j] = j < nt ? p[j * gs] : (XT)0;
#pragma unroll
                for (int j = 0; j < kSeriesTile; ++j) fold<XT, SKIP>(acc[j], x[j], w, missing);
            }
#pragma unroll
            for (int j = 0; j < kSeriesTile; ++j)
                if (j < nt) o0[j * os] = finish<OT, CLAMP>(acc[j], a.scale);
        }
    } else {
        const long S = a.steps * (long)a.members;
        long xo = 0, oo = r * a.os_row;  // offsets of the tile's first series
        int m = 0;
        for (long s0 = 0; s0 < S; s0 += kSeriesTile) {
            long xs[kSeriesTile], os[kSeriesTile];
            double acc[kSeriesTile];
#pragma unroll
            for (int j = 0; j < kSeriesTile; ++j) {
                const bool live = s0 + j < S;
                xs[j] = live ? xo : 0;
                os[j] = live ? oo : -1;
                acc[j] = 0.0;
                next_series(a, xo, oo, m);
            }
            for (long q = b; q < e; ++q) {
                const int c = a.col[q];
                if (c < 0 || (long)c >= a.cols) {
                    bad = true;
                    continue;
                }
                const double w = a.weight[q];
                XT x[kSeriesTile];
#pragma unroll
                for (int j = 0; j < kSeriesTile; ++j) x[j] = grid[xs[j] + c];
#pragma unroll
                for (int j = 0; j < kSeriesTile; ++j) fold<XT, SKIP>(acc[j], x[j], w, missing);
            }
#pragma unroll
            for (int j = 0; j < kSeriesTile; ++j)
                if (os[j] >= 0) out[os[j]] = finish<OT, CLAMP>(acc[j], a.scale);
        }
    }
    if (bad && a.status) atomicOr(a.status, CMF_STATUS_BAD_INDEX);
}

template <typename XT, typename OT, bool ONE>
const void* pick_flags(int flags)
{
    const bool skip = flags & CMF_FORCING_SKIP_MISSING, clamp = flags & CMF_FORCING_CLAMP_NEGATIVE;
    if (skip) return clamp ? (const void*)k_forcing_map<XT, OT, true, true, ONE>
                           : (const void*)k_forcing_map<XT, OT, true, false, ONE>;
    return clamp ? (const void*)k_forcing_map<XT, OT, false, true, ONE>
                 : (const void*)k_forcing_map<XT, OT, false, false, ONE>;
}

template <typename XT, typename OT>
const void* pick_members(int flags, bool one)
{
    return one ? pick_flags<XT, OT, true>(flags) : pick_flags<XT, OT, false>(flags);
}

}  // namespace

extern "C" int cmf_forcing_apply(const CmfForcingMap* map, void* stream, const void* grid,
                                 int grid_dtype, int32_t steps, int32_t members,
                                 int64_t grid_step_stride, int64_t grid_member_stride, void* out,
                                 int out_dtype, int64_t out_step_stride, int64_t out_member_stride,
                                 int64_t out_row_stride, double unit_factor, double missing_value,
                                 int flags, int* status)
{
    if (!map || map->num_rows < 0 || map->num_cols < 0 || steps < 0 || members < 1) return CMF_ERR_ARG;
    if (grid_dtype != CMF_DTYPE_F32 && grid_dtype != CMF_DTYPE_F64) return CMF_ERR_ARG;
    if (out_dtype != CMF_DTYPE_F32 && out_dtype != CMF_DTYPE_F64) return CMF_ERR_ARG;
    if (flags & ~(CMF_FORCING_SKIP_MISSING | CMF_FORCING_CLAMP_NEGATIVE)) return CMF_ERR_ARG;
    if (!(unit_factor != 0.0) || !std::isfinite(unit_factor)) return CMF_ERR_ARG;
    if (map->num_cols > INT32_MAX) return CMF_ERR_ARG;  // columns are int32
    if (map->num_rows == 0 || steps == 0) return CMF_OK;
    if (!map->row_ptr || !map->col || !map->weight || !grid || !out) return CMF_ERR_ARG;
    ForcingArgs a;
    a.rows = map->num_rows;
    a.cols = map->num_cols;
    a.row_ptr = map->row_ptr;
    a.col = map->col;
    a.weight = map->weight;
    a.grid = grid;
    a.steps = steps;
    a.members = members;
    a.gs_step = grid_step_stride;
    a.gs_member = grid_member_stride;
    a.out = out;
    a.os_step = out_step_stride;
    a.os_member = out_member_stride;
    a.os_row = out_row_stride;
    a.scale = 1.0 / unit_factor;
    a.missing = missing_value;
    a.status = status;
    const void* fn;
    // the single-member kernel keeps a tile's step offsets in 32 bits
    const bool one = members == 1 && grid_step_stride >= 0 && out_step_stride >= 0 &&
                     grid_step_stride * (int64_t)kSeriesTile < INT32_MAX &&
                     out_step_stride * (int64_t)kSeriesTile < INT32_MAX;
    if (grid_dtype == CMF_DTYPE_F32)
        fn = out_dtype == CMF_DTYPE_F32 ? pick_members<float, float>(flags, one)
                                        : pick_members<float, double>(flags, one);
    else
        fn = out_dtype == CMF_DTYPE_F32 ? pick_members<double, float>(flags, one)
                                        : pick_members<double, double>(flags, one);
    const long blocks = (map->num_rows + kBlock - 1) / kBlock;
    if (blocks > INT32_MAX) return CMF_ERR_ARG;
    void* args[] = {&a};
    cudaError_t e = cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(kBlock), args, 0, (cudaStream_t)stream);
    return e == cudaSuccess ? CMF_OK : CMF_ERR_CUDA;
}
