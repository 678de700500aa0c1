"""C ABI checks that need no GPU: the library loads, exports every symbol
include/*.h declares, validates its arguments before touching CUDA, and the
product never reaches the oracle."""
import ctypes
import glob
import os
import re

import pytest

from cfd_cavity_b200 import _lib as L

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(cav\w*)\s*\(", text, flags=re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(L.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 25, syms
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_default_params_are_the_reference_cli_defaults():
    """src/cli.rs:94-130."""
    lib = L.load()
    p = L.CavParams()
    assert lib.cav_default_params(ctypes.byref(p)) == 0
    assert (p.nx, p.ny) == (64, 256)
    assert (p.ra, p.pr, p.cs, p.pr_t, p.utarget, p.seed) == (1e6, 0.71, 0.10, 0.9, 0.02, 42)
    assert (p.alpha_mult, p.nu_start_mult, p.has_nu_override) == (1.0, 1.0, 0)
    assert p.noise_amp == 1e-3 and p.init_mode == L.CAV_INIT_LINEAR and p.geq_order == 2


def _create(**kw):
    lib = L.load()
    p = L.CavParams()
    lib.cav_default_params(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    h = ctypes.c_void_p()
    rc = lib.cav_create(ctypes.byref(p), ctypes.byref(h))
    if rc == 0:
        lib.cav_destroy(h)
    return rc, lib.cav_last_error(None).decode()


@pytest.mark.parametrize("kw,code", [
    (dict(nx=2), L.CAV_ERR_ARG),
    (dict(ny=3), L.CAV_ERR_ARG),
    (dict(precision=9), L.CAV_ERR_ARG),
    (dict(geq_order=3), L.CAV_ERR_ARG),
    (dict(init_mode=5), L.CAV_ERR_ARG),
    (dict(has_nu_override=1, nu_override=-1.0), L.CAV_ERR_ARG),
    (dict(has_nu_override=1, nu_override=1e-5), L.CAV_ERR_TAU),
    (dict(alpha_mult=1e-3), L.CAV_ERR_TAU),
])
def test_create_rejects_bad_arguments_before_cuda(kw, code):
    """The reference asserts (src/uniform/solver.rs:130-132, 152-154); the ABI
    returns a status and a message instead."""
    rc, msg = _create(**kw)
    assert rc == code, (rc, msg)
    assert msg


def test_null_handle_is_an_error():
    lib = L.load()
    assert lib.cav_step(None, 1) == L.CAV_ERR_ARG
    assert lib.cav_destroy(None) == L.CAV_ERR_ARG


def test_product_sources_never_reach_the_oracle():
    pkg = os.path.join(ROOT, "cfd_cavity_b200")
    for path in glob.glob(os.path.join(pkg, "**", "*"), recursive=True):
        if not path.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
            continue
        text = open(path).read()
        assert not re.search(r"^\s*(from|import)\s+oracle\b", text, flags=re.M), path
        assert "cavity_oracle" not in text, path


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError):
        L._lib_saved = L._lib
        try:
            L._lib = None
            L.load(str(tmp_path / "nope.so"))
        finally:
            L._lib = L._lib_saved


def test_batch_rejects_bad_arguments_before_cuda():
    lib = L.load()
    h = ctypes.c_void_p()
    ps = (L.CavParams * 2)()
    for p in ps:
        lib.cav_default_params(ctypes.byref(p))
    assert lib.cav_batch_create(ps, 0, ctypes.byref(h)) == L.CAV_ERR_ARG
    ps[1].precision = L.CAV_PREC_F32
    assert lib.cav_batch_create(ps, 2, ctypes.byref(h)) == L.CAV_ERR_ARG
    assert lib.cav_batch_last_error(None)
    assert lib.cav_batch_step(None, 1) == L.CAV_ERR_ARG


def test_sweep_configs_follow_the_benchmark_ranges():
    from cfd_cavity_b200 import sweep_configs

    cfg = sweep_configs(64, seed=2024)
    assert len(cfg) == 64
    assert {(c["nx"], c["ny"]) for c in cfg} == {(64, 256), (96, 384), (128, 512)}
    assert all(1e6 <= c["ra"] <= 1e8 and 0.08 <= c["cs"] <= 0.12 for c in cfg)
    assert cfg == sweep_configs(64, seed=2024)


def test_octree_default_params_and_argument_checks():
    """cav_octree_*: defaults (256x1024 base, the reference CLI's octree
    options, src/cli.rs:94-130) and CavitySolver::new's assertions
    (src/octree/solver.rs:298-303) as CAV_ERR_ARG before any CUDA call."""
    lib = L.load()
    p = L.CavOctreeParams()
    assert lib.cav_octree_default_params(ctypes.byref(p)) == 0
    assert (p.nx0, p.ny0, p.bl_width, p.levels, p.odd_exact) == (256, 1024, 16, 2, 0)
    assert (p.ra, p.pr, p.utarget, p.seed, p.nu_start_mult) == (1e6, 0.71, 0.02, 42, 1.0)
    assert (p.cs, p.pr_t, p.precision) == (0.0, 0.9, L.CAV_OCT_F64)
    for field, bad in (("bl_width", 1), ("bl_width", 128), ("levels", 4), ("precision", 9), ("ny0", 3)):
        q = L.CavOctreeParams()
        lib.cav_octree_default_params(ctypes.byref(q))
        setattr(q, field, bad)
        h = ctypes.c_void_p()
        assert lib.cav_octree_create(ctypes.byref(q), ctypes.byref(h)) == L.CAV_ERR_ARG, field
        assert not h.value
        assert lib.cav_octree_last_error(None)


# ---- struct layouts: the Python mirror of every public struct ----------------
STRUCTS = [
    ("cav_params", "CavParams"), ("cav_info", "CavInfo"), ("cav_diag_out", "CavDiag"),
    ("cav_batch_tuning", "CavBatchTuning"), ("cav_adjoint_spec", "CavAdjointSpec"),
    ("cav_adjoint_result", "CavAdjointResult"), ("cav_octree_params", "CavOctreeParams"),
    ("cav_octree_info", "CavOctreeInfo"), ("cav_octree_diag_out", "CavOctreeDiag"),
]


def test_struct_layouts_match_the_header(tmp_path):
    """sizeof and every field's offset of the header's structs (compiled by
    the C compiler) equal those of the ctypes mirrors in _lib.py."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cavity.h"', "int main(void) {"]
    for c_name, py_name in STRUCTS:
        py = getattr(L, py_name)
        lines.append(f'printf("{py_name} size %zu\\n", sizeof({c_name}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{py_name} {f} %zu\\n", offsetof({c_name}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, out):
        py_name, field, value = line.split()
        py = getattr(L, py_name)
        got = ctypes.sizeof(py) if field == "size" else getattr(py, field).offset
        assert got == int(value), (py_name, field, got, value)
