"""Pins the CPU oracle to the reference's own outputs (no GPU needed).

tests/golden/*.npz were produced by tests/golden/make_golden.py running the
reference's CUDA kernels (oracle/_ref harness builds of its sources) on a
B200.  The FP32 and FP64 oracles must reproduce them: bit-exact after the
first step from the reference's initial state, and within 1e-5 relative
L-infinity (rho, |u|, phi; see helpers.field_errors) at the last dump.
"""
import os

import numpy as np
import pytest

from helpers import FIELDS, field_errors, harness_params
from oracle.oracle import Oracle, seeded_macros
from golden.make_golden import GOLDEN

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", sorted(GOLDEN))
@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_reproduces_reference(name, precision):
    spec = GOLDEN[name]
    d = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    p = harness_params(spec["case"], periodic_y=spec["periodic_y"])
    o = Oracle(p, precision)
    if spec["seed"] is not None:
        o.init_macros(*seeded_macros((p.nz, p.ny, p.nx), seed=spec["seed"]))
    else:
        o.init_jets()
    done = 0
    for s in spec["at"]:
        o.step(s - done)
        done = s
        ref = {k: d[f"{k}_{s}"] for k in FIELDS}
        got = {k: o.get(k) for k in FIELDS}
        errs = field_errors(got, ref)
        if s == 1 and spec["seed"] is None:
            assert max(errs.values()) == 0.0, errs
        tol = 2e-6 if s == 1 else 1e-5
        assert max(errs.values()) <= tol, (s, errs)


def test_golden_files_cover_both_velocity_sets_and_face_kinds():
    cases = {GOLDEN[n]["case"] for n in GOLDEN}
    assert cases == {"q19_s", "q27_s"}
    assert {GOLDEN[n]["periodic_y"] for n in GOLDEN} == {False, True}
