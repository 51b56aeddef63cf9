"""The oracle's restatement of the reference's one-pass Poisson form and its
accelerators (poisson_onepass in oracle/lbm_oracle.c; GPU/InamuroCUDA.cu:
780-844, 931-1013, 1198-1328): each variant converges to the fixed point of
the production split form, so at a tight tolerance p agrees with the split
solve; with unit relaxation and no accelerator the one-pass iterate is the
split iterate (h_old + (T h - h_old) reproduces T h here)."""
import numpy as np
import pytest

from oracle import pyoracle
from tests.helpers import laplace_case, oracle_params, rel_err

SH = (16, 12, 10)


def case():
    p, f = laplace_case(SH, DD=6.0, noise=1e-4, seed=3)
    f["w"] = 0.01 * np.sin(2 * np.pi * np.arange(SH[2]) / SH[2])[:, None, None] * np.ones_like(f["w"])
    return p, f


@pytest.mark.parametrize("periodic", [False, True])
def test_onepass_variants_reach_the_split_fixed_point(periodic):
    p, f = case()
    ref = pyoracle.Oracle(SH, oracle_params(p), f, tol=1e-12, max_sweeps=2000000, periodic_x=periodic)
    r = ref.step()
    pr = ref.fields()["p"]
    plain = pyoracle.Oracle(SH, oracle_params(p), f, tol=1e-12, max_sweeps=2000000, periodic_x=periodic,
                            poisson_form=2)
    assert plain.step()["sweeps"] == r["sweeps"]
    assert np.array_equal(plain.fields()["p"], pr)
    for acc in ({"fixed_point_relax": 0.8}, {"anderson_m1": 1}, {"two_grid": 1}):
        o = pyoracle.Oracle(SH, oracle_params(p), f, tol=1e-12, max_sweeps=2000000, periodic_x=periodic,
                            poisson_form=2, accel=acc)
        o.step()
        assert rel_err(o.fields()["p"], pr) <= 1e-11, acc


def test_anderson_cuts_sweeps():
    """Anderson-m1 needs fewer sweeps than the plain one-pass iteration here."""
    p, f = case()
    counts = {}
    for name, acc in (("plain", {}), ("anderson", {"anderson_m1": 1})):
        o = pyoracle.Oracle(SH, oracle_params(p), f, tol=1e-12, max_sweeps=2000000, poisson_form=2, accel=acc)
        counts[name] = o.step()["sweeps"]
    assert counts["anderson"] < counts["plain"], counts
