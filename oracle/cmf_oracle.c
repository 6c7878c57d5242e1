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
