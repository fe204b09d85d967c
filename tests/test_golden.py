"""The oracle and the GPU library against known answers of the reference's
own sources frozen by tests/golden/make_golden.py (bit for bit; the GPU's
atomically accumulated escape/impact sums to 1e-12 relative)."""
import os

import numpy as np
import pytest

from rhybrid_b200 import abi

from harness import SUM_COUNTERS, STATE_ARRAYS, run

import golden.make_golden as mg

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    st = {"arrays": {n: z[f"a_{n}"] for n in STATE_ARRAYS}, "particles": [], "counters": {}}
    s = 0
    while f"p{s}_counts" in z:
        st["particles"].append((z[f"p{s}_counts"], z[f"p{s}_records"]))
        s += 1
    for k, v in zip(z["counter_names"], z["counter_values"]):
        st["counters"][str(k)] = float(v)
    st["time"] = (float(z["time"][0]), int(z["time"][1]))
    return st


def check(got, want, what, sum_rtol=0.0):
    for n in STATE_ARRAYS:
        a, b = np.asarray(got["arrays"][n]).reshape(-1), np.asarray(want["arrays"][n]).reshape(-1)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), f"{what}: {n} differs"
    assert len(got["particles"]) == len(want["particles"])
    for s, ((ca, pa), (cb, pb)) in enumerate(zip(got["particles"], want["particles"])):
        assert np.array_equal(ca, cb), f"{what}: species {s} counts differ"
        assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64)), f"{what}: species {s} particles differ"
    for k, w in want["counters"].items():
        v = got["counters"][k]
        if sum_rtol and k.split("[")[0] in SUM_COUNTERS:
            assert abs(v - w) <= sum_rtol * max(abs(w), 1e-300), f"{what}: {k}: {v} vs {w}"
        else:
            assert v == w, f"{what}: {k}: {v} != {w}"
    assert got["time"][1] == want["time"][1] and got["time"][0] == want["time"][0]


@pytest.mark.parametrize("name", sorted(mg.CASES))
def test_oracle_matches_golden(port_lib, name):
    make, steps = mg.CASES[name]
    check(run(port_lib, make(), steps), load_fixture(name), name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(mg.CASES))
def test_gpu_exact_path_matches_golden(name):
    make, steps = mg.CASES[name]
    check(run(abi.gpu_library(), make(), steps, fast=False), load_fixture(name), name, sum_rtol=1e-12)
