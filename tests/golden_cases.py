"""Network cases of the reference-CUDA golden fixtures (tests/golden/ref_*.npz).

The fixtures store only states and the sub-step count/length; parameters are
regenerated from these seeded specs, which must therefore not change."""
from cmfb200 import synthetic as syn

CASES = {
    "plain": syn.NetworkSpec(1500, seed=101),
    "bif": syn.NetworkSpec(1500, seed=102, bifurcation_paths=80),
    "levee": syn.NetworkSpec(1500, seed=103, levee_fraction=0.25),
    "res": syn.NetworkSpec(1500, seed=104, reservoirs=12),
    "full": syn.NetworkSpec(1500, seed=105, bifurcation_paths=80, levee_fraction=0.25,
                            reservoirs=12),
}

CELL = ("river_outflow", "flood_outflow", "river_depth", "flood_depth", "protected_depth",
        "river_cross_section_depth", "flood_cross_section_depth", "flood_cross_section_area",
        "flood_fraction", "river_storage", "flood_storage", "protected_storage")


def state_fields(modules):
    out = list(CELL)
    if "bifurcation" in modules:
        out += ["bifurcation_outflow", "bifurcation_cross_section_depth"]
    if "reservoir" in modules:
        out += ["reservoir_total_inflow"]
    return out


def diag_fields(modules):
    out = ["river_inflow", "flood_inflow"]
    if "bifurcation" in modules:
        out += ["limit_rate", "global_bifurcation_outflow", "water_surface_elevation"]
    if "bifurcation" in modules or "reservoir" in modules:
        out += ["total_storage"]
    if "bifurcation" in modules and "levee" in modules:
        out += ["protected_water_surface_elevation"]
    return out
