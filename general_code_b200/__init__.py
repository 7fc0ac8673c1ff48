"""general_code_b200: APE/HYP smearing and on-axis Wilson loops W(R,T) for
SU(2)/SU(3) lattice gauge configurations on NVIDIA B200 (sm_100a).

The compute path is libgc_b200.so (hand-written CUDA kernels behind the C ABI
in include/gc_lattice.h); this package is a thin ctypes host layer over it.
"""
from .lattice import (GCError, Lattice, LatticeData, fma_peak, generate_config, job_device_bytes,
                      launches_per_job,
                      link_size, plaket, plaket_space, plaket_time, polyakov_average_directions,
                      polyakov_loop, polyakov_loop_correlator_color_average,
                      polyakov_loop_correlator_singlet, probe_config, read_data_convert,
                      smearing_APE, smearing_HYP, unit_config, volume, wilson_gevp_adjoint_indexed,
                      wilson_gevp_indexed, wilson_loop, wilson_loop_adjoint, wilson_offaxis,
                      wilson_offaxis_adjoint, wilson_offaxis_adjoint_result,
                      wilson_offaxis_result, wilson_spatial_3d_indexed)

__all__ = ["GCError", "Lattice", "LatticeData", "fma_peak", "generate_config", "job_device_bytes",
           "launches_per_job",
           "link_size", "plaket", "plaket_space", "plaket_time", "polyakov_average_directions",
           "polyakov_loop", "polyakov_loop_correlator_color_average",
           "polyakov_loop_correlator_singlet", "probe_config", "read_data_convert",
           "smearing_APE", "smearing_HYP", "unit_config", "volume",
           "wilson_gevp_adjoint_indexed", "wilson_gevp_indexed", "wilson_loop",
           "wilson_loop_adjoint", "wilson_offaxis", "wilson_offaxis_adjoint",
           "wilson_offaxis_adjoint_result", "wilson_offaxis_result",
           "wilson_spatial_3d_indexed"]
