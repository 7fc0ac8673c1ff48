"""Generates tests/golden/fullsize.json: W(R,T) tables of the benchmark's
large configurations computed by the REFERENCE's own CPU code
(oracle/_ref/libref_parity.so: lib/cpu smearing_HYP, smearing_APE and
wilson_loop compiled from the reference sources with -O2 and no fast-math by
oracle/Makefile), too slow to recompute inside a test.

Cases (seeded synthetic configurations; the input is regenerated from the
seed by the tests, so only its SHA-256 and a few moments are stored):
  su3_32  SU(3) 32^4, eps 0.25, HYP x1 (1, 0.75, 0.6) + APE x40 (0.5),
          W for R,T = 1..16
  su2_48  SU(2) 48^4, eps 0.3,  HYP x1 (1, 0.75, 0.6) + APE x10 (0.5),
          W for R,T = 1..24

The input comes from the oracle-side copy of the generator
(oracle/libgen.so), the same source the product library builds; a test that
regenerates it with the product's generator checks the SHA-256 first.

Run here (needs the reference sources and oracle/_ref; a few minutes):
    make -C oracle ref gen && python tests/golden/make_golden_fullsize.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import py_oracle  # noqa: E402

OUT = Path(__file__).resolve().parent / "fullsize.json"
SEED = 20261203
HYP = (1.0, 0.75, 0.6)

# name, nc, dims, eps, config index, ape steps, ape alpha, (rmin, rmax, tmin, tmax)
CASES = [
    ("su3_32", 3, (32, 32, 32, 32), 0.25, 0, 40, 0.5, (1, 16, 1, 16)),
    ("su2_48", 2, (48, 48, 48, 48), 0.3, 0, 10, 0.5, (1, 24, 1, 24)),
]


def digest(links: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(links).tobytes()).hexdigest()


def main(names=None) -> None:
    ref = py_oracle.ref("parity")
    ref.set_threads(os.cpu_count() or 1)
    gen = py_oracle.generator()
    cases = json.loads(OUT.read_text())["cases"] if OUT.exists() else {}
    for name, nc, dims, eps, cfg, n_ape, alpha, (r0, r1, t0, t1) in CASES:
        if names and name not in names:
            continue
        links = gen.generate(dims, nc, eps, SEED, cfg)
        sha = digest(links)
        plaq0 = ref.plaquette(nc, dims, links)
        t = time.time()
        w, times = ref.job(nc, dims, links, 1, *HYP, n_ape, alpha, r0, r1, t0, t1)
        wall = time.time() - t
        plaq1 = ref.plaquette(nc, dims, links)
        cases[name] = {"nc": nc, "dims": list(dims), "eps": eps, "seed": SEED,
                       "config_index": cfg, "hyp_alpha": list(HYP), "hyp_steps": 1,
                       "ape_steps": n_ape, "ape_alpha": alpha, "r_min": r0, "r_max": r1,
                       "time_min": t0, "time_max": t1, "input_sha256": sha,
                       "plaquette_in": plaq0, "plaquette_out": plaq1,
                       "wilson": w.tolist(),
                       "reference_seconds": {"hyp": times[0], "ape": times[1],
                                             "wilson": times[2], "threads": ref.num_threads()}}
        print(name, f"{wall:.1f} s", "plaq", plaq0, "->", plaq1, "W[0,0]", w[0, 0],
              "W[-1,-1]", w[-1, -1], flush=True)
    meta = {"generated_by": "tests/golden/make_golden_fullsize.py",
            "reference_code": "oracle/_ref/libref_parity.so (lib/cpu smearing_HYP, "
                              "smearing_APE, wilson_loop, plaket_site; -O2 -fno-fast-math)",
            "wilson_layout": "rows T = time_min.., columns R = r_min..",
            "cases": cases}
    OUT.write_text(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main(sys.argv[1:])
