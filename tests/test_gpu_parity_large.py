"""Parity at the scale of the 256^3 head-on collision: the same workload
(two R = 32 drops 96 cells apart approaching at +-0.02, rho_L/rho_G = 100,
seeded phi noise) on a 128^3 box, both x boundaries (the reference's slip
walls and the periodic box), two steps replayed at 100 and 200 sweeps, against
the FP64 oracle on the same inputs.

Bars: FP64 <= 1e-10 and mixed <= 1e-5 norm-wise relative error
(max|gpu - oracle| / max|oracle|) in phi, rho, u, v, w and p after each step;
the velocity components are held against the velocity scale (one component
can stay near zero); the periodic box keeps sum(phi) to 1e-12 of the loaded
phi's sum in both precisions."""
import numpy as np
import pytest

import bench
import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import oracle_params

pytestmark = pytest.mark.gpu
N = 128
PLAN = (100, 200)
TOL = {"fp64": 1e-10, "mixed": 1e-5}


@pytest.fixture(scope="module", params=[0, 1], ids=["slip_x", "periodic_x"])
def oracle_run(request):
    p = bench.workload_params(N)
    p.periodic_x = request.param
    f = bench.workload_fields(p)
    o = pyoracle.Oracle(p.shape, oracle_params(p), f, max_sweeps=10 ** 6, periodic_x=bool(request.param))
    out = []
    for k in PLAN:
        info = o.step(k)
        assert info["sweeps"] == k
        out.append((info, o.fields()))
    o.close()
    return p, f, out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_headon_128_against_oracle(oracle_run, precision):
    p, f, ref = oracle_run
    g = L.InamuroCUDA(p, f, precision=precision)
    g.set_poisson(max_sweeps=10 ** 6, fail_on_limit=True)
    m0 = float(np.sum(f["phi"]))
    for k, (info, want) in zip(PLAN, ref):
        st = g.step_replay([k])[0]
        assert st["iterations"] == k
        got = g.download_fields()
        vscale = max(float(np.max(np.abs(want[c]))) for c in ("u", "v", "w"))
        for c in L.FIELDS:
            scale = vscale if c in ("u", "v", "w") else float(np.max(np.abs(want[c])))
            err = float(np.max(np.abs(got[c] - want[c]))) / scale
            assert err <= TOL[precision], f"{precision} after {k} sweeps: {c} {err:.3e}"
        if p.periodic_x:
            assert abs(st["mass"] - m0) <= 1e-12 * abs(m0), (st["mass"], m0)
            assert abs(info["mass"] - m0) <= 1e-12 * abs(m0)
    g.close()
