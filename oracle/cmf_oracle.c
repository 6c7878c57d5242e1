/*
 * CPU oracle for the CaMa-Flood-GPU sub-step -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates the reference CUDA kernels (the .cu files of cmfgpu/phys/cuda) on the host, in
 * the reference phase order, for two precisions:
 *   *_f32  REAL = float,  STO = double  (the reference "mixed" mode)
 *   *_f64  REAL = double, STO = double
 * It is loaded only by tests/, the smoke check and bench.py's CPU-baseline leg,
 * through oracle/oracle.py.  Built with -ffp-contract=off so that every float
 * operation rounds exactly once.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <omp.h>

#define REAL float
#define ORC_SFX _f32
#include "cmf_oracle_impl.h"
#undef REAL
#undef ORC_SFX

#define REAL double
#define ORC_SFX _f64
#include "cmf_oracle_impl.h"
#undef REAL
#undef ORC_SFX

size_t orc_model_size_f32(void) { return sizeof(OrcModel_f32); }
size_t orc_model_size_f64(void) { return sizeof(OrcModel_f64); }

void orc_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int orc_max_threads(void) { return omp_get_max_threads(); }

/*
 * Host restatements of the three network-generation helpers, so that a run
 * which must not load the product library (the reference arm of the
 * benchmark) can still build the synthetic networks bit for bit:
 *   orc_accumulate_upstream    a cell's value plus everything upstream of it
 *                              (upstream area); cells in topological order
 *   orc_accumulate_downstream  a cell's value plus its downstream cell's sum
 *                              (bed drops integrated into elevations)
 *   orc_init_river_depth       cold-start river depth,
 *                              cmfgpu/params/utils.py:140-157
 * Each returns 0, or 1 when the order is not topological.
 */
int orc_accumulate_upstream(int64_t n, const int32_t* dn, const double* vals, double* out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = vals[i];
    for (int64_t i = 0; i < n; ++i) {
        const int64_t d = dn[i];
        if (d < 0 || d == i) continue;
        if (d < i) return 1;
        out[d] += out[i];
    }
    return 0;
}

int orc_accumulate_downstream(int64_t n, const int32_t* dn, const double* vals, double* out)
{
    for (int64_t i = n - 1; i >= 0; --i) {
        const int64_t d = dn[i];
        if (d < 0 || d == i) {
            out[i] = vals[i];
        } else {
            if (d < i) return 1;
            out[i] = vals[i] + out[d];
        }
    }
    return 0;
}

int orc_init_river_depth(int64_t n, const float* elevation, const float* height,
                         const int32_t* dn, float* depth)
{
    /* numba loop of the reference: from the last cell to the first, each
       cell's depth follows its downstream cell's water surface */
    for (int64_t i = n - 1; i >= 0; --i) {
        const int64_t j = dn[i];
        float d;
        if (j == i || j < 0) {
            d = height[i];
        } else {
            if (j < i) return 1;
            const float bed_j = elevation[j] - height[j];
            const float bed_i = elevation[i] - height[i];
            const float surf = (depth[j] + bed_j) - bed_i;
            d = surf > 0.0f ? surf : 0.0f;
        }
        depth[i] = d < height[i] ? d : height[i];
    }
    return 0;
}
