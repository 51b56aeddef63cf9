"""The batched droplet-oscillation workload (bench.batch_workload): seeded,
inside the stated ranges, one centred ellipsoidal drop per box."""
import numpy as np

import bench


def test_batch_workload_ranges_and_seed():
    params, fields = bench.batch_workload(12, seed=7)
    again, _ = bench.batch_workload(12, seed=7)
    assert [(p.lx, p.ly, p.lz, p.rho_L, p.k_f) for p in params] == \
        [(p.lx, p.ly, p.lz, p.rho_L, p.k_f) for p in again]
    for p, f in zip(params, fields):
        assert {p.lx, p.ly, p.lz} <= set(bench.BATCH_SIDES) and p.periodic_x == 1
        assert 10.0 <= p.rho_L / p.rho_G <= 1000.0
        assert 0.03 <= p.k_f <= 0.1
        R = p.DD / 2.0
        assert 6.0 <= R <= min(p.lx, p.ly, p.lz) / 4.0
        assert f["phi"].shape == (p.lz, p.ly, p.lx)
        # liquid at the centre, gas at the corners, drop longer in x than in z
        phi = f["phi"]
        mid = (p.lz // 2, p.ly // 2, p.lx // 2)
        assert phi[mid] > 0.9 * p.fei_max and phi[0, 0, 0] < p.fei_min + 1e-3
        liquid = phi > 0.5 * (p.fei_max + p.fei_min)
        ext_x = liquid.any(axis=(0, 1)).sum()
        ext_z = liquid.any(axis=(1, 2)).sum()
        assert ext_x > ext_z
        assert np.all(f["u"] == 0.0) and np.all(f["p"] == 0.0)
