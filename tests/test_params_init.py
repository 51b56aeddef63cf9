"""params.in parser and droplet initial condition of the library's C ABI
(lbm_params_load, lbm_init_droplets; host-only entry points, no GPU) against
the reference GPU-tree Inamuro constructor (fixtures from oracle/_ref)."""
import os
import tempfile

import numpy as np
import pytest

import lbm_b200 as L
from oracle import pyoracle
from tests.helpers import fixture, params_from_text

INIT_CASES = ["init_two_sharp", "init_single_tanh", "init_two_tanh_offset", "init_mixed_styles"]
PARSED_KEYS = ("lx", "ly", "lz", "rho_L", "rho_G", "mu_L", "mu_G", "tauf", "taug", "k_f", "k_g",
               "T", "a", "b", "fei_L", "fei_G")


@pytest.mark.parametrize("name", INIT_CASES)
def test_params_and_init_match_reference(name):
    fx = fixture(name)
    p = params_from_text(fx["params_text"])
    for i, k in enumerate(PARSED_KEYS):
        assert getattr(p, k) == fx["parsed"][i], k
    f = L.init_droplets(p)
    for i, k in enumerate(L.FIELDS):
        assert np.array_equal(f[k], fx["fields"][i]), k


@pytest.mark.parametrize("name", INIT_CASES)
def test_oracle_init_matches_reference(name):
    """The oracle's restated init agrees with the reference too."""
    fx = fixture(name)
    p = params_from_text(fx["params_text"])
    f = pyoracle.init_droplets(p.shape, p.DD, p.fei_max, p.fei_min, p.rho_L, p.rho_G,
                               single=bool(p.init_single_droplet), tanh=bool(p.init_tanh),
                               velocity=p.init_velocity, width=p.interface_width,
                               center=(p.init_center_x, p.init_center_y, p.init_center_z),
                               separation=p.init_separation, offset_x=p.init_offset_x)
    for i, k in enumerate(L.FIELDS):
        assert np.array_equal(f[k], fx["fields"][i]), k


def test_params_defaults_match_reference_struct():
    p = L.params_default()
    assert (p.lx, p.ly, p.lz) == (48, 96, 128)
    assert (p.rho_L, p.rho_G, p.mu_L, p.mu_G) == (50.0, 1.0, 0.008, 0.00016)
    assert (p.k_f, p.k_g, p.fei_L, p.fei_G, p.fei_max, p.fei_min) == (0.5, 0.0005, 0.092, 0.015,
                                                                        0.09714, 0.01134)
    assert (p.T, p.a, p.b, p.DD, p.init_velocity, p.interface_width) == (0.035, 1.0, 6.7, 32.0,
                                                                          0.035, 2.0)


def test_params_errors():
    with pytest.raises(L.LBMError) as e:
        L.params_load("/nonexistent/params.in")
    assert e.value.status == 6
    with tempfile.NamedTemporaryFile("w", suffix=".in", delete=False) as f:
        f.write("16 32\n1\n")
        path = f.name
    try:
        with pytest.raises(L.LBMError) as e2:
            L.params_load(path)
        assert e2.value.status == 4
    finally:
        os.unlink(path)


def test_init_mode_fallbacks():
    """Unknown init_mode / init_profile fall back to two_droplets / sharp."""
    base = fixture("init_two_sharp")["params_text"].item()
    p1 = params_from_text(base + "init_mode=bogus init_profile=bogus\n")
    p0 = params_from_text(base)
    assert p1.init_single_droplet == 0 and p1.init_tanh == 0
    for k in L.FIELDS:
        assert np.array_equal(L.init_droplets(p1)[k], L.init_droplets(p0)[k])


def test_boundary_x_token():
    """boundary_x=periodic|slip (not a reference key) sets lbm_params.periodic_x;
    the reference's slip walls stay the default; other values are rejected."""
    base = fixture("init_two_sharp")["params_text"].item()
    assert params_from_text(base).periodic_x == 0
    assert params_from_text(base + "boundary_x=periodic\n").periodic_x == 1
    assert params_from_text(base + "boundary_x=slip\n").periodic_x == 0
    with pytest.raises(L.LBMError) as e:
        params_from_text(base + "boundary_x=open\n")
    assert e.value.status == 4
