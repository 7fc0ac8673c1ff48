"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own CPU
code (oracle/_ref/libref_parity.so: lib/cpu smearing_HYP, smearing_APE,
wilson_loop, wilson_loop_adjoint and plaket_site compiled from the reference sources with -O2 and
no fast-math by oracle/Makefile).

Each case: a seeded synthetic configuration (the product's generator,
gc_generate_host), one HYP step, then APE steps, then a W(R,T) table, with
the plaquette of the input and of the result. The fixture stores the input
links, the links after HYP, the links after HYP+APE, the W table and the
plaquettes, so the tests do not depend on the generator staying unchanged.

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
        np.savez_compressed(OUT / f"{name}.npz", links0=links0, links_hyp=links_hyp,
                            links_ape=links_ape, wilson=w, wilson_adjoint=wa,
                            plaquettes=np.array([plaq0, plaq1]))
        index[name] = {"nc": nc, "dims": list(dims), "eps": eps, "seed": seed,
                       "config_index": cfg, "hyp_alpha": [a1, a2, a3], "ape_steps": n_ape,
                       "ape_alpha": alpha, "r_min": r0, "r_max": r1, "time_min": t0,
                       "time_max": t1, "plaquette_in": plaq0, "plaquette_out": plaq1,
                       "wilson": w.tolist(), "wilson_adjoint": wa.tolist()}
        print(name, "plaq", plaq0, "->", plaq1, "W[0,0]", w[0, 0])
    meta = {"generated_by": "tests/golden/make_golden.py",
            "reference_code": "oracle/_ref/libref_parity.so (lib/cpu smearing_HYP, "
                              "smearing_APE, wilson_loop, wilson_loop_adjoint, plaket_site; "
                              "-O2 -fno-fast-math)",
            "link_layout": "4*V links, link index 4*site+mu, row-major (get_data order)",
            "cases": index}
    (OUT / "index.json").write_text(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
