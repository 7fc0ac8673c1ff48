"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own CPU
code (oracle/_ref/libref_parity.so: lib/cpu smearing_HYP, smearing_APE,
wilson_loop, wilson_loop_adjoint and plaket_site compiled from the reference sources with -O2 and
no fast-math by oracle/Makefile).

Each case: a seeded synthetic configuration (the product's generator,
gc_generate_host), one HYP step, then APE steps, then a W(R,T) table, with
the plaquette of the input and of the result. The fixture stores the input
links, the links after HYP, the links after HYP+APE, the W table and the
plaquettes, so the tests do not depend on the generator staying unchanged.
Also from the reference, on the same links: the adjoint W table; the
two-configuration (GEVP) tables of (HYP+APE, HYP) (wilson_gevp_indexed and
wilson_gevp_adjoint_indexed); the time and space plaquettes after HYP+APE;
the Polyakov loop and both correlator tables (D_max = 2) after HYP, with the
reference's distance averages of the tables; the merged off-axis loops
(wilson_offaxis_result, and wilson_offaxis_adjoint_result for SU(3)) after
HYP+APE for R in [1, 2], T in [1, 2]; two smearing_APE_2d steps of the
(x, z) links after HYP; the spatial loops (wilson_spatial_3d_indexed) after
HYP for R, T in [1, 2], alpha 0.5, smearing 1..3 measured every step.

Run here (needs the reference sources and oracle/_ref):
    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from general_code_b200 import generate_config  # noqa: E402
from oracle import py_oracle  # noqa: E402

OUT = Path(__file__).resolve().parent

# name, nc, dims, eps, seed, cfg, (a1, a2, a3), ape_steps, ape_alpha, (rmin, rmax, tmin, tmax)
CASES = [
    ("su2_4x4x4x6", 2, (4, 4, 4, 6), 0.3, 20261203, 0, (1.0, 0.75, 0.6), 3, 0.5, (1, 2, 1, 3)),
    ("su3_4x4x4x4", 3, (4, 4, 4, 4), 0.25, 20261203, 1, (1.0, 0.75, 0.6), 3, 0.5, (1, 2, 1, 2)),
    # odd, unequal extents; the reference script's HYP alphas (1,1,0.5); t_min > 1
    ("su2_6x4x5x8", 2, (6, 4, 5, 8), 0.3, 7, 2, (1.0, 1.0, 0.5), 2, 0.45, (1, 3, 2, 4)),
    # every site is a boundary site
    ("su3_3x3x3x4", 3, (3, 3, 3, 4), 0.25, 11, 3, (1.0, 0.75, 0.6), 2, 0.5, (1, 1, 1, 2)),
    # r_min > 1 and a W range reaching half the extent
    ("su3_4x3x4x8", 3, (4, 3, 4, 8), 0.25, 5, 4, (1.0, 0.75, 0.6), 1, 0.5, (2, 2, 1, 4)),
]


def main() -> None:
    ref = py_oracle.ref("parity")
    index = {}
    for name, nc, dims, eps, seed, cfg, (a1, a2, a3), n_ape, alpha, (r0, r1, t0, t1) in CASES:
        links0 = generate_config(dims, nc, eps, seed, cfg, gauge=True)
        plaq0 = ref.plaquette(nc, dims, links0)
        links_hyp = links0.copy()
        ref.hyp(nc, dims, links_hyp, a1, a2, a3, 1)
        links_ape = links_hyp.copy()
        ref.ape(nc, dims, links_ape, alpha, n_ape)
        w = ref.wilson(nc, dims, links_ape, r0, r1, t0, t1)
        wa = ref.wilson_adjoint(nc, dims, links_ape, r0, r1, t0, t1)
        plaq1 = ref.plaquette(nc, dims, links_ape)
        gevp = ref.wilson_gevp(nc, dims, links_ape, links_hyp, r0, r1, t0, t1, False)
        gevp_adj = ref.wilson_gevp(nc, dims, links_ape, links_hyp, r0, r1, t0, t1, True)
        plaq_t = ref.plaquette_time(nc, dims, links_ape)
        plaq_s = ref.plaquette_space(nc, dims, links_ape)
        poly = ref.polyakov_loop(nc, dims, links_hyp)
        d_max = 2
        corr_s = ref.polyakov_correlator(nc, dims, links_hyp, d_max, True)
        corr_c = ref.polyakov_correlator(nc, dims, links_hyp, d_max, False)
        avg_s = ref.polyakov_average_directions(corr_s, d_max)
        avg_c = ref.polyakov_average_directions(corr_c, d_max)
        links_plane = links_hyp.copy()
        ref.ape_plane(nc, dims, links_plane, 0, 2, 0.5, 2)
        spatial = ref.wilson_spatial_3d(nc, dims, links_hyp, 1, 2, 1, 2, 0.5, 1, 3, 1)
        off = ref.wilson_offaxis_result(nc, dims, links_ape, 1.0, 2.0, 1, 2)
        off_adj = (ref.wilson_offaxis_result(nc, dims, links_ape, 1.0, 2.0, 1, 2, True)
                   if nc == 3 else {})
        np.savez_compressed(OUT / f"{name}.npz", links0=links0, links_hyp=links_hyp,
                            links_ape=links_ape, wilson=w, wilson_adjoint=wa,
                            plaquettes=np.array([plaq0, plaq1]), gevp=gevp,
                            gevp_adjoint=gevp_adj, plaquettes_time_space=np.array([plaq_t, plaq_s]),
                            polyakov_loop=np.array([poly]), polyakov_singlet=corr_s,
                            polyakov_color_average=corr_c, links_ape_plane=links_plane)
        index[name] = {"nc": nc, "dims": list(dims), "eps": eps, "seed": seed,
                       "config_index": cfg, "hyp_alpha": [a1, a2, a3], "ape_steps": n_ape,
                       "ape_alpha": alpha, "r_min": r0, "r_max": r1, "time_min": t0,
                       "time_max": t1, "plaquette_in": plaq0, "plaquette_out": plaq1,
                       "wilson": w.tolist(), "wilson_adjoint": wa.tolist(),
                       "gevp": gevp.tolist(), "gevp_adjoint": gevp_adj.tolist(),
                       "plaquette_time": plaq_t, "plaquette_space": plaq_s,
                       "polyakov_loop": poly, "polyakov_d_max": d_max,
                       "polyakov_singlet_by_distance": [[k, v] for k, v in avg_s.items()],
                       "polyakov_color_average_by_distance": [[k, v] for k, v in avg_c.items()],
                       "offaxis_range": [1.0, 2.0, 1, 2],
                       "offaxis": [[t, size, w] for (t, size), w in off.items()],
                       "offaxis_adjoint": [[t, size, w] for (t, size), w in off_adj.items()],
                       "ape_plane": [0, 2, 0.5, 2],
                       "spatial_args": [1, 2, 1, 2, 0.5, 1, 3, 1],
                       "spatial": [[sm, t, r, w] for (sm, t, r), w in spatial.items()]}
        print(name, "plaq", plaq0, "->", plaq1, "W[0,0]", w[0, 0])
    meta = {"generated_by": "tests/golden/make_golden.py",
            "reference_code": "oracle/_ref/libref_parity.so (lib/cpu smearing_HYP, "
                              "smearing_APE, wilson_loop, wilson_loop_adjoint, "
                              "wilson_gevp_indexed, wilson_gevp_adjoint_indexed, plaket_site, "
                              "plaket_site_time, plaket_site_space, get_polyakov_loop, "
                              "polyakov_loop_correlator_singlet, "
                              "polyakov_loop_correlator_color_average, "
                              "polyakov_average_directions, wilson_offaxis_result, "
                              "wilson_offaxis_adjoint_result, smearing_APE_2d, "
                              "wilson_spatial_3d_indexed; -O2 -fno-fast-math)",
            "link_layout": "4*V links, link index 4*site+mu, row-major (get_data order)",
            "cases": index}
    (OUT / "index.json").write_text(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
