"""Pins the oracle (oracle/lbm_oracle.c) to the reference itself.

The fixtures in tests/golden were produced by the reference's own CPU solver
(CPU/Inamuro.cpp, compiled unmodified, see tests/golden/make_golden.py).  The
restatement must reproduce them bit for bit: same per-step sweep counts and
identical FP64 fields.
"""
import numpy as np
import pytest

from oracle import pyoracle
from tests.helpers import fixture, fields_dict, oracle_params, params_from_text, sha

STEP_CASES = ["step_single_tanh", "step_two_sharp", "step_example_16x32x32", "step_laplace_32"]


@pytest.mark.parametrize("name", STEP_CASES)
def test_oracle_matches_reference_bitwise(name):
    fx = fixture(name)
    p = params_from_text(fx["params_text"])
    o = pyoracle.Oracle(p.shape, oracle_params(p), fields_dict(fx["init"]))
    nsteps = len(fx["sweeps"])
    for s in range(nsteps):
        info = o.step()
        assert info["sweeps"] == fx["sweeps"][s], f"step {s + 1} sweep count"
        got = o.fields()
        for i, k in enumerate(("phi", "rho", "u", "v", "w", "p")):
            if "fields" in fx.files:
                assert np.array_equal(got[k], fx["fields"][s, i]), f"{k} step {s + 1}"
            assert sha(got[k]) == fx["digests"][s, i], f"{k} digest step {s + 1}"
        # fixture mass is numpy's pairwise sum, the oracle's a serial x-outer sum
        assert abs(info["mass"] - fx["mass"][s]) <= 1e-11 * abs(fx["mass"][s])


def test_oracle_replay_matches_natural_counts():
    """Forcing the reference's own sweep counts reproduces the natural run."""
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    a = pyoracle.Oracle(p.shape, oracle_params(p), fields_dict(fx["init"]))
    b = pyoracle.Oracle(p.shape, oracle_params(p), fields_dict(fx["init"]))
    for s in range(len(fx["sweeps"])):
        ia = a.step()
        ib = b.step(replay=int(fx["sweeps"][s]))
        assert ia["sweeps"] == ib["sweeps"]
        fa, fb = a.fields(), b.fields()
        for k in fa:
            assert np.array_equal(fa[k], fb[k])


def test_oracle_dual_residual_is_stricter():
    """The dual exit (GPU/InamuroCUDA.cu:2126-2129) never stops earlier than the
    relative-change exit alone, and reports a finite fixed-point residual."""
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    a = pyoracle.Oracle(p.shape, oracle_params(p), fields_dict(fx["init"]))
    b = pyoracle.Oracle(p.shape, oracle_params(p), fields_dict(fx["init"]), dual=True)
    for _ in range(2):
        ia, ib = a.step(), b.step()
        assert ib["sweeps"] >= ia["sweeps"]
        assert np.isfinite(ib["fp_rel"]) and ib["fp_rel"] < 1e-3
        assert ib["relative_error"] < 1e-3


def test_oracle_budget_and_nonfinite():
    # moving drops: a non-zero Poisson source from the first step on
    fx = fixture("step_two_sharp")
    p = params_from_text(fx["params_text"])
    f = fields_dict(fx["init"])
    o = pyoracle.Oracle(p.shape, oracle_params(p), f, max_sweeps=100, tol=1e-12)
    with pytest.raises(pyoracle.OracleError) as e:
        o.step()
    assert e.value.code == 3
    bad = {k: v.copy() for k, v in f.items()}
    bad["u"][0, 0, 0] = np.nan
    o2 = pyoracle.Oracle(p.shape, oracle_params(p), bad)
    with pytest.raises(pyoracle.OracleError) as e2:
        o2.step()
    assert e2.value.code == 2
