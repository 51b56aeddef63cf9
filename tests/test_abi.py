"""The C ABI library loads and exports every function include/lbm_b200.h
declares (no GPU needed; no compute calls)."""
import ctypes
import os
import subprocess

import lbm_b200 as L


def test_library_exports_every_declared_symbol():
    lib = L.load_library()
    names = L.header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_nm_lists_exports_as_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for n in L.header_functions():
        assert n in exported, n


def test_status_strings_and_version():
    lib = L.load_library()
    assert lib.lbm_abi_version() == L.ABI_VERSION == 6
    for s in range(9):
        assert lib.lbm_status_string(s)


def test_struct_sizes_match_header():
    # lbm_params: 6 ints + 16 doubles + 2 ints + 7 doubles (natural alignment)
    assert ctypes.sizeof(L.Params) == 6 * 4 + 16 * 8 + 2 * 4 + 7 * 8 + 8   # periodic_x + tail padding
    assert ctypes.sizeof(L.PoissonCfg) == 40
    assert ctypes.sizeof(L.StepStats) == 8 + 16 * 8 + 6 * 4 + 8
    assert ctypes.sizeof(L.Timing) == 5 * 8 + 5 * 8


def test_create_without_gpu_fails_loudly():
    """On a machine without an sm_100 GPU the solver refuses to start (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        return
    p = L.make_params(lx=8, ly=8, lz=8)
    try:
        L.InamuroCUDA(p)
    except L.LBMError as e:
        assert e.status == 7
    else:
        raise AssertionError("expected LBM_ERR_NO_DEVICE")


def test_header_compiles_as_c():
    src = "#include \"lbm_b200.h\"\nint main(void){lbm_params p; lbm_params_default(&p); return p.lx != 48;}\n"
    inc = os.path.join(os.path.dirname(L.HEADER_PATH))
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", inc, "-x", "c", "-"],
                       input=src, text=True, capture_output=True)
    assert r.returncode == 0, r.stderr


def test_python_structs_match_the_header_layout(tmp_path):
    """Every structure the Python bindings mirror has the header's size and
    field offsets (a C program built from the Python field lists prints them;
    a field name the header lacks fails to compile)."""
    pairs = [("lbm_params", L.Params), ("lbm_poisson_cfg", L.PoissonCfg), ("lbm_step_stats", L.StepStats),
             ("lbm_timing", L.Timing), ("lbm_field_stats", L.FieldStats), ("lbm_diagnostics", L.Diagnostics),
             ("lbm_batch_tuning", L.BatchTuning), ("lbm_poisson_accel", L.PoissonAccel),
             ("lbm_adjoint_cfg", L.AdjointCfg), ("lbm_adjoint_stats", L.AdjointStats)]
    lines = ["#include <stddef.h>", "#include <stdio.h>", "#include \"lbm_b200.h\"", "int main(void) {"]
    for cname, cls in pairs:
        lines.append(f'    printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'    printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    inc = os.path.dirname(L.HEADER_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", inc, str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for cname, cls in pairs:
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(cls, f).offset, (cname, f)


def test_python_poisson_form_names_match_the_header_enum():
    """Every lbm_poisson_form value the header declares has its Python name
    with the same value (and no Python name has a value the header lacks)."""
    import re
    hdr = open(os.path.join(os.path.dirname(L.LIB_PATH), "..", "include", "lbm_b200.h")).read()
    body = hdr[hdr.index("LBM_POISSON_KINETIC"):hdr.index("} lbm_poisson_form;")]
    values = {int(v) for v in re.findall(r"LBM_POISSON_[A-Z_]+\s*=\s*(\d+)", body)}
    assert values == set(L.InamuroCUDA.POISSON_FORMS.values()), (values, L.InamuroCUDA.POISSON_FORMS)
    assert L.InamuroCUDA.POISSON_FORMS["refine"] == 6
