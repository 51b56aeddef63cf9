"""All-or-nothing allocation of a handle's lazily allocated buffer sets (the
Krylov work vectors, the Anderson-m1 history): a host test with a failing
fake allocator, no GPU involved.  A failed set leaves every pointer null, so
the handle's "set allocated" test stays false and a retried step allocates
again instead of launching on null buffers."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_alloc_set_all_or_nothing(tmp_path):
    exe = tmp_path / "alloc_set_test"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror",
                    os.path.join(ROOT, "tests", "cpp", "alloc_set_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and "alloc_set ok" in r.stdout, (r.returncode, r.stdout, r.stderr)


def test_lazy_buffer_sets_use_alloc_set():
    """The Krylov and Anderson-m1 buffer sets go through alloc_set (no
    one-by-one cudaMalloc of a set whose first pointer is its flag)."""
    src = open(os.path.join(ROOT, "lbm_b200", "csrc", "lbm_capi.cu")).read()
    assert "Krylov work vectors: device allocation failed" in src
    assert "Anderson-m1 buffers: device allocation failed" in src
    assert "cudaMalloc(&h->kb." not in src and "cudaMalloc(&h->and_" not in src
