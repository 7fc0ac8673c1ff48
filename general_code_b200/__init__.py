"""general_code_b200: APE/HYP smearing and on-axis Wilson loops W(R,T) for
SU(2)/SU(3) lattice gauge configurations on NVIDIA B200 (sm_100a).

The compute path is libgc_b200.so (hand-written CUDA kernels behind the C ABI
in include/gc_lattice.h); this package is a thin ctypes host layer over it.
"""
from .lattice import (GCError, Lattice, LatticeData, generate_config, job_device_bytes,
                      link_size, plaket, probe_config, read_data_convert, smearing_APE,
                      smearing_HYP, unit_config, volume, wilson_loop)

__all__ = ["GCError", "Lattice", "LatticeData", "generate_config", "job_device_bytes",
           "link_size", "plaket", "probe_config", "read_data_convert", "smearing_APE",
           "smearing_HYP", "unit_config", "volume", "wilson_loop"]
