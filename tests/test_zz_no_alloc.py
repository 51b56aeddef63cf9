"""lbm_field_statistics_noalloc: the allocation-free variant of the device
field-statistics reduction, for callers that cannot allocate device memory
(a host application that owns all device memory through its own pool, a
latency-critical loop that must not call cudaMalloc, a plugin given device
pointers but no allocator).  Checked through the C ABI against
lbm_field_statistics on two calls in a row.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

import lbm_b200 as L
from tests.helpers import laplace_case

pytestmark = pytest.mark.gpu


def close(a, b):
    for k in ("nan_count", "inf_count", "valid_count"):
        assert a[k] == b[k], k
    for k in ("min", "max", "mean", "abs_max", "sum"):
        assert abs(a[k] - b[k]) <= 1e-10 * max(abs(b[k]), 1e-300), (k, a[k], b[k])


def test_noalloc_matches_handle_statistics_two_calls():
    p, f = laplace_case((40, 36, 30), DD=12.0, noise=1e-4)
    g = L.InamuroCUDA(p, f)
    g.set_poisson(max_sweeps=60000, fail_on_limit=True)
    g.step(1)
    n = p.lx * p.ly * p.lz
    lib = L.load_library()
    for name in ("phi", "p"):          # two calls in a row on the shared scratch
        out = L.FieldStats()
        st = lib.lbm_field_statistics_noalloc(g.device_ptr(name), n, None, C.byref(out))
        assert st == 0
        close(out.as_dict(), g.field_statistics(name))
        host = g.download(name)
        assert out.valid_count == host.size
        assert abs(out.sum - host.sum()) <= 1e-12 * np.abs(host).sum()
    g.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = L.load_library()
    out = L.FieldStats()
    assert lib.lbm_field_statistics_noalloc(C.c_void_p(1), L.NOALLOC_MAX_CELLS + 1, None, C.byref(out)) == 4
    assert lib.lbm_field_statistics_noalloc(None, 10, None, C.byref(out)) == 4
    with pytest.raises(L.LBMError):
        L.field_statistics_noalloc(1, L.NOALLOC_MAX_CELLS + 1)
