"""Freezes known answers of the reference's own hot-path sources (built by
oracle/Makefile into oracle/_ref/librhref.so from the reference tree) as
small fixtures, so that the oracle can be checked where the reference tree is
absent.

    python tests/golden/make_golden.py

Each fixture holds the state after N steps of a small configuration: every
grid array, the particles (cell counts and records) of every species, and
the counters, all exactly as the reference computed them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from harness import closed_box_config, run  # noqa: E402
from oracle import oracle  # noqa: E402
from rhybrid_b200 import config as cf  # noqa: E402

CASES = {
    "periodic_6cubed_5steps": (lambda: cf.config_empty_box(6, 6, 6, ppc=3.0), 5),
    "closed_box_7x6x5_4steps": (lambda: closed_box_config(nx=7, ny=6, nz=5, ppc=3.0), 4),
}


def save(name, st):
    out = {f"a_{k}": v for k, v in st["arrays"].items()}
    for s, (cnt, p) in enumerate(st["particles"]):
        out[f"p{s}_counts"] = cnt
        out[f"p{s}_records"] = p
    keys = sorted(st["counters"])
    out["counter_names"] = np.array(keys)
    out["counter_values"] = np.array([st["counters"][k] for k in keys], dtype=np.float64)
    out["time"] = np.array([st["time"][0], st["time"][1]], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def main():
    oracle.build(reference=True)
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("the reference build (oracle/_ref) is not available")
    for name, (make, steps) in CASES.items():
        save(name, run(ref, make(), steps))
        print("wrote", name)


if __name__ == "__main__":
    main()
