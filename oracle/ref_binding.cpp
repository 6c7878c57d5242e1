// pybind11 binding of the reference CaMa-Flood-GPU CUDA launchers -- TEST
// INFRASTRUCTURE ONLY (the GPU parity oracle).
//
// The launchers are compiled unmodified from the reference sources where they
// lie (cmfgpu/phys/cuda/*.cu, see oracle/build_ref.py); this file only
// declares their signatures (cmfgpu/phys/cuda/outflow.cu:272,389;
// storage.cu:318; adaptive_time.cu:50; bifurcation.cu:158,201;
// reservoir.cu:327; levee.cu:343,424) and exposes them to Python.  In the
// reference the same functions are bound by hydroforge's CudaExtensionGroup
// (cmfgpu/phys/cuda/__init__.py:29-166), which is not available here.
#include <torch/extension.h>

using OptT = c10::optional<at::Tensor>;
using T = at::Tensor;

void launch_outflow(T, T, T, T, T, T, T, T, T, T, T, T, T, T, OptT, T, T, T, T, T, T, T, OptT,
                    OptT, T, OptT, OptT, double, T, long, bool, bool, bool, bool, bool, OptT, bool,
                    double, OptT, OptT, bool, long, long);
void launch_inflow(T, T, T, T, T, T, T, T, OptT, OptT, OptT, long, bool, bool, long);
void launch_flood_stage(T, T, T, T, OptT, T, OptT, OptT, T, T, T, T, T, T, T, T, T, T, T, T, T, T,
                        long, int, int, bool, bool, long);
void launch_adaptive_time(T, T, OptT, T, T, double, double, long, bool, long);
void launch_bif_outflow(T, T, T, T, T, T, T, T, T, T, T, double, T, long, long, int, long);
void launch_bif_inflow(T, T, T, T, T, long, long, int, long);
void launch_reservoir_outflow(T, T, T, T, T, T, T, T, T, T, T, T, T, T, T, T, T, long, long, long);
void launch_levee_stage(T, T, T, T, T, T, T, T, T, T, T, T, T, T, T, T, long, long, int, long);
void launch_levee_bif_outflow(T, T, T, T, T, T, T, T, T, T, T, T, double, T, long, long, int, long);

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    m.def("launch_outflow", &launch_outflow);
    m.def("launch_inflow", &launch_inflow);
    m.def("launch_flood_stage", &launch_flood_stage);
    m.def("launch_adaptive_time", &launch_adaptive_time);
    m.def("launch_bif_outflow", &launch_bif_outflow);
    m.def("launch_bif_inflow", &launch_bif_inflow);
    m.def("launch_reservoir_outflow", &launch_reservoir_outflow);
    m.def("launch_levee_stage", &launch_levee_stage);
    m.def("launch_levee_bif_outflow", &launch_levee_bif_outflow);
}
