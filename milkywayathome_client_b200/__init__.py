"""B200 (sm_100a) Barnes-Hut step of the Milkyway@Home N-body client.

The step -- bounding box, octree build, mass/quadrupole moments, opening-criterion walk and
kick-drift-kick under the Milky Way potential -- runs in libnbody_b200.so (CUDA kernels for
sm_100a, C ABI in include/nbody_b200.h).  `nbody` mirrors the reference's step interface
(NBodyCtx, Potential, NBodyState.create / step) on top of it; `models` holds the set-up
formulas and a synthetic dwarf sampler.
"""
from .nbody import (Disk, Dwarf, Halo, NBodyBatch, NBodyCtx, NBodyError, NBodyState, Potential,
                    Spherical, emd, ext_acceleration, kernel_launches, milky_way_potential,
                    mixed_dwarf_particle_masses, mixed_dwarf_struct)
from ._lib import status_is_fatal, status_names
from .histogram import (DataHistogram, HistogramParams, data_from_counts, read_histogram,
                        write_histogram)

__all__ = ["Disk", "Dwarf", "Halo", "NBodyBatch", "NBodyCtx", "NBodyError", "NBodyState", "Potential",
           "Spherical",
           "emd", "ext_acceleration", "kernel_launches", "milky_way_potential", "status_is_fatal",
           "status_names", "DataHistogram", "HistogramParams", "data_from_counts", "write_histogram",
           "read_histogram", "mixed_dwarf_struct", "mixed_dwarf_particle_masses"]
