// Host-side topology and index construction for the river network.
//
// Everything here runs once at model construction, on the host, and is
// integer/index work that must be bit-exact with the reference's numba
// preprocessing:
//   * topological sort          -> cmfgpu/params/utils.py:83-138
//   * upstream CSR adjacency     -> cmfgpu/params/utils.py:160-206
//   * initial river depth        -> cmfgpu/params/utils.py:140-157
// plus the breadth-first "children are contiguous" catchment order that the
// device kernels are laid out in (no reference counterpart; see cmf_bfs_order).
//
// All functions are plain C ABI, take caller-owned buffers and never allocate
// memory that outlives the call.

#include "cmfb200.h"

#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

extern "C" {

// Kahn topological sort over (catchment_id, downstream_id) pairs.
// Follows cmfgpu/params/utils.py:83-138: a dense id->index table, indegree
// counting over valid downstream ids, a FIFO seeded with zero-indegree nodes in
// index order.  Returns CMF_ERR_ARG when a cycle prevents a full ordering.
int cmf_topo_topological_sort(int64_t n, const int64_t* catchment_id,
                              const int64_t* downstream_id, int32_t* order_out)
{
    if (n < 0 || (n > 0 && (!catchment_id || !downstream_id || !order_out)))
        return CMF_ERR_ARG;
    int64_t max_id = 0;
    for (int64_t i = 0; i < n; ++i)
        if (catchment_id[i] > max_id) max_id = catchment_id[i];
    const int64_t total = max_id + 1;
    std::vector<int64_t> grid_to_idx((size_t)total, -1);
    for (int64_t i = 0; i < n; ++i) {
        if (catchment_id[i] < 0) return CMF_ERR_ARG;
        grid_to_idx[(size_t)catchment_id[i]] = i;
    }
    std::vector<int32_t> indeg((size_t)n, 0);
    for (int64_t i = 0; i < n; ++i) {
        int64_t d = downstream_id[i];
        if (d >= 0 && d < total) {
            int64_t di = grid_to_idx[(size_t)d];
            if (di >= 0) indeg[(size_t)di] += 1;
        }
    }
    std::vector<int32_t> q((size_t)n);
    int64_t front = 0, back = 0, count = 0;
    for (int64_t i = 0; i < n; ++i)
        if (indeg[(size_t)i] == 0) q[(size_t)back++] = (int32_t)i;
    while (front < back) {
        int32_t u = q[(size_t)front++];
        order_out[count++] = u;
        int64_t d = downstream_id[u];
        if (d >= 0 && d < total) {
            int64_t di = grid_to_idx[(size_t)d];
            if (di >= 0) {
                if (--indeg[(size_t)di] == 0) q[(size_t)back++] = (int32_t)di;
            }
        }
    }
    return count == n ? CMF_OK : CMF_ERR_ARG;
}

// Upstream CSR in index space from downstream indices (dn[i] == i marks a
// mouth, dn[i] < 0 is treated the same way).  Semantics of
// cmfgpu/params/utils.py:160-206: self-loops are excluded and, for every node,
// its upstream neighbours are listed in increasing index order.
// indptr has n+1 entries; indices has indptr[n] entries (<= n).
int cmf_topo_upstream_csr(int64_t n, const int32_t* dn, int32_t* indptr,
                          int32_t* indices)
{
    if (n < 0 || (n > 0 && (!dn || !indptr || !indices))) return CMF_ERR_ARG;
    std::vector<int32_t> count((size_t)n, 0);
    for (int64_t i = 0; i < n; ++i) {
        int32_t d = dn[i];
        if (d >= n) return CMF_ERR_ARG;
        if (d >= 0 && d != i) count[(size_t)d] += 1;
    }
    indptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) indptr[i + 1] = indptr[i] + count[(size_t)i];
    std::vector<int32_t> fill((size_t)n, 0);
    for (int64_t i = 0; i < n; ++i) {
        int32_t d = dn[i];
        if (d >= 0 && d != i) indices[indptr[d] + fill[(size_t)d]++] = (int32_t)i;
    }
    return CMF_OK;
}

// Basin-major breadth-first catchment order.
//
// order_out[new] = old index.  Mouths are taken in old index order; each
// mouth's basin is emitted breadth-first (every node's upstream cells appended
// in old index order) before the next mouth.  Consequences used by the device
// kernels:
//   * the upstream cells of new node p are exactly the new indices
//     [up_ptr[p], up_ptr[p+1] - m) with m = 1 when p+1 is a mouth (a basin's
//     mouth sits just before its own upstream cells) and 0 otherwise -- no
//     index array is needed; up_ptr[n] = n;
//   * parents precede their upstream cells and the downstream index is
//     non-decreasing along a basin level, so downstream and upstream gathers
//     of a warp touch short monotone ranges close to the warp's own cells.
// up_ptr_out has n+1 entries and is expressed in the NEW order.
// Returns CMF_ERR_ARG when some node is not connected to a mouth (cycle).
int cmf_topo_bfs_order(int64_t n, const int32_t* dn, int32_t* order_out,
                       int32_t* up_ptr_out)
{
    if (n < 0 || (n > 0 && (!dn || !order_out || !up_ptr_out))) return CMF_ERR_ARG;
    std::vector<int32_t> ptr((size_t)n + 1), idx((size_t)n);
    int rc = cmf_topo_upstream_csr(n, dn, ptr.data(), idx.data());
    if (rc != CMF_OK) return rc;
    // Basin-major: each basin (the tree of one mouth) is laid out completely,
    // breadth-first, before the next one starts.  Upstream ranges stay
    // contiguous and monotone, and parent/child distances are bounded by the
    // width of one basin's level instead of the whole network's.
    int64_t back = 0, front = 0;
    for (int64_t r = 0; r < n; ++r) {
        if (!(dn[r] == r || dn[r] < 0)) continue;
        order_out[back++] = (int32_t)r;
        while (front < back) {
            int32_t u = order_out[front];
            int32_t c0 = ptr[(size_t)u], c1 = ptr[(size_t)u + 1];
            up_ptr_out[front] = (int32_t)back;
            for (int32_t k = c0; k < c1; ++k) order_out[back++] = idx[(size_t)k];
            ++front;
        }
    }
    up_ptr_out[n] = (int32_t)back;
    return back == n ? CMF_OK : CMF_ERR_ARG;
}

// Initial river depth: cmfgpu/params/utils.py:140-157, in float32 exactly as
// the numba function computes it.  The reference loops i from n-1 down to 0 and
// relies on dn[i] > i; here any order in which a node's downstream cell comes
// earlier is accepted through `visit` (visit == NULL means n-1 .. 0).
int cmf_topo_init_river_depth(int64_t n, const float* catchment_elevation,
                              const float* river_height, const int32_t* dn,
                              const int32_t* visit, float* river_depth)
{
    if (n < 0 || (n > 0 && (!catchment_elevation || !river_height || !dn || !river_depth)))
        return CMF_ERR_ARG;
    for (int64_t k = 0; k < n; ++k) {
        int64_t i = visit ? visit[k] : (n - 1 - k);
        int32_t j = dn[i];
        float re_i = catchment_elevation[i] - river_height[i];
        float d;
        if (i == j || j < 0) {
            d = river_height[i];
        } else {
            float re_j = catchment_elevation[j] - river_height[j];
            float v = (river_depth[j] + re_j) - re_i;
            d = v > 0.0f ? v : 0.0f;
        }
        river_depth[i] = d < river_height[i] ? d : river_height[i];
    }
    return CMF_OK;
}

// out[i] = vals[i] + sum over upstream u of out[u]  (requires dn[i] > i for
// non-mouths, i.e. topological order).  Used for upstream-area accumulation.
int cmf_topo_accumulate_upstream(int64_t n, const int32_t* dn, const double* vals,
                                 double* out)
{
    if (n < 0 || (n > 0 && (!dn || !vals || !out))) return CMF_ERR_ARG;
    for (int64_t i = 0; i < n; ++i) out[i] = vals[i];
    for (int64_t i = 0; i < n; ++i) {
        int32_t d = dn[i];
        if (d < 0 || d == i) continue;
        if (d < i) return CMF_ERR_ARG;
        out[d] += out[i];
    }
    return CMF_OK;
}

// out[i] = vals[i] + out[dn[i]] (out[mouth] = vals[mouth]); requires
// topological order.  Used to integrate bed drops into elevations.
int cmf_topo_accumulate_downstream(int64_t n, const int32_t* dn, const double* vals,
                                   double* out)
{
    if (n < 0 || (n > 0 && (!dn || !vals || !out))) return CMF_ERR_ARG;
    for (int64_t i = n - 1; i >= 0; --i) {
        int32_t d = dn[i];
        if (d < 0 || d == i) { out[i] = vals[i]; continue; }
        if (d < i) return CMF_ERR_ARG;
        out[i] = vals[i] + out[d];
    }
    return CMF_OK;
}

}  // extern "C"
