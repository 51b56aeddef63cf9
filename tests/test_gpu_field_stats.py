"""Device field statistics (lbm_field_statistics) against numpy on the
downloaded field, with the NaN/Inf rules of Inamuro::updateFieldStatistics
(CPU/Inamuro.cpp:1050-1092)."""
import numpy as np
import pytest

import lbm_b200 as L
from tests.helpers import laplace_case

pytestmark = pytest.mark.gpu


def host_stats(a):
    a = a.ravel()
    fin = np.isfinite(a)
    v = a[fin]
    out = {"nan_count": int(np.isnan(a).sum()), "inf_count": int(np.isinf(a).sum()),
           "valid_count": int(fin.sum())}
    if v.size:
        out.update(min=float(v.min()), max=float(v.max()), abs_max=float(np.abs(v).max()),
                   sum=float(v.sum()), mean=float(v.sum() / v.size), abs_sum=float(np.abs(v).sum()))
    return out


def check(dev, host):
    for k in ("nan_count", "inf_count", "valid_count"):
        assert dev[k] == host[k], k
    if host["valid_count"] == 0:
        assert np.isnan(dev["min"]) and np.isnan(dev["mean"])
        return
    for k in ("min", "max", "abs_max"):
        assert dev[k] == host[k], k
    # summation order differs: bound by the conditioning sum|x|, not |sum x|
    assert abs(dev["sum"] - host["sum"]) <= 1e-12 * host["abs_sum"], "sum"
    assert abs(dev["mean"] - host["mean"]) <= 1e-12 * host["abs_sum"] / host["valid_count"], "mean"


def test_field_statistics_after_steps():
    p, f = laplace_case((40, 36, 30), DD=12.0, noise=1e-4)
    g = L.InamuroCUDA(p, f)
    g.set_poisson(max_sweeps=60000, fail_on_limit=True)
    st = g.step(2)
    for k in L.FIELDS:
        check(g.field_statistics(k), host_stats(g.download(k)))
    # the step's mass is the same reduction of phi
    assert abs(g.field_statistics("phi")["sum"] - st[-1]["mass"]) <= 1e-12 * abs(st[-1]["mass"])
    a = g.field_statistics("p")
    b = g.field_statistics("p")
    assert a == b


def test_field_statistics_nan_inf_and_empty():
    p, f = laplace_case((33, 7, 5), DD=3.0)
    bad = {k: v.copy() for k, v in f.items()}
    bad["u"][0, 0, 0] = np.nan
    bad["u"][1, 2, 3] = np.inf
    bad["u"][4, 6, 32] = -np.inf
    bad["v"][:] = np.nan
    g = L.InamuroCUDA(p, bad)
    su = g.field_statistics("u")
    assert su["nan_count"] == 1 and su["inf_count"] == 2
    check(su, host_stats(bad["u"]))
    sv = g.field_statistics("v")
    assert sv["valid_count"] == 0 and sv["nan_count"] == bad["v"].size
    check(sv, host_stats(bad["v"]))
