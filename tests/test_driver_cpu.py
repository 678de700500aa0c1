"""The driver binary ``cavity_les`` on the CPU: its command line (parse_args,
src/cli.rs:185-384: flags, aliases, checks and exit codes) and its Rust float
formats (rustfmt.h) against an independent restatement of Rust's core::fmt
(tests/driver_expect.py).  Runs that need the GPU are in test_gpu_driver.py.
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from driver_expect import rust_display, rust_exp, rust_exp_short, rust_fixed

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
BIN = os.path.join(ROOT, "cfd_cavity_b200", "_build", "cavity_les")


@pytest.fixture(scope="module")
def driver():
    if not os.path.exists(BIN):
        from cfd_cavity_b200 import build
        build.build()
    return BIN


def run(args, **kw):
    return subprocess.run([BIN, *args], capture_output=True, text=True, timeout=60, **kw)


def test_help_exits_zero(driver):
    r = run(["--help"])
    assert r.returncode == 0
    for flag in ("--mode", "--nx", "--bl-width", "--levels", "--odd-exact", "--dynamic-smag",
                 "--snapshot-every", "--restart", "--precision"):
        assert flag in r.stderr


@pytest.mark.parametrize("args,needle", [
    (["--nx", "4"], "nx and ny must be >= 8"),
    (["--nx", "64", "--ny", "64"], "ny must be > nx"),
    (["--ra", "-1"], "ra and pr must be > 0"),
    (["--sample-every", "0"], "sample-every must be >= 1"),
    (["--jobs", "0"], "jobs must be >= 1"),
    (["--alpha-mult", "0"], "alpha-mult"),
    (["--nu-start-mult", "0.5"], "nu-start-mult"),
    (["--smag-alpha", "2"], "smag-alpha"),
    (["--eta-test", "0.5"], "eta-test"),
    (["--nu", "0.01"], "0.002"),
    (["--nu", "-1"], "--nu must be > 0"),
    (["--mode", "sphere"], "--mode"),
    (["--nx", "abc"], "--nx: integer expected"),
    (["--ra", "x1"], "--ra: number expected"),
    (["--bogus", "1"], "unknown option '--bogus'"),
    (["--steps"], "missing value for --steps"),
    (["--dynamic-smag=maybe"], "boolean expected"),
    (["--mode", "octree", "--levels", "4"], "levels must be 2 or 3"),
    (["--mode", "octree", "--nx0", "8"], "nx0 and ny0 must be >= 16"),
    (["--mode", "octree", "--bl-width", "40"], "bl-width"),
    (["--progress-every", "0"], "progress-every"),
])
def test_argument_errors_exit_one(driver, args, needle):
    r = run(args)
    assert r.returncode == 1, (args, r.stdout, r.stderr)
    assert needle in r.stderr, r.stderr


def test_aliases_and_inline_values_parse(driver):
    """--key=value, the underscore aliases and the boolean forms parse; the
    run then stops at the precision check (exit 1) before any device call."""
    r = run(["--nx=24", "--ny", "96", "--pr_t=0.8", "--prt", "0.8", "--sample_every=5", "--j", "1",
             "--dynamic_smag=false", "--odd-exact=1", "--precision", "nope"])
    assert r.returncode == 1 and "unknown --precision 'nope'" in r.stderr
    assert "Grille : 24×96 (Az = 4.13) | Ra = 1.000e6 | Pr = 0.71 | Cs = 0.1 | Pr_t = 0.8" in r.stdout


def _check_values(vals):
    src = os.path.join(ROOT, "tests", "native", "rustfmt_check.cpp")
    exe = os.path.join(ROOT, "tests", "native", "_rustfmt_check")
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    subprocess.run([gxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "cfd_cavity_b200", "csrc"), src, "-o",
                    exe], check=True, timeout=120)
    inp = "".join(f"{struct.unpack('<Q', struct.pack('<d', v))[0]:016x}\n" for v in vals)
    out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.splitlines()
    os.remove(exe)
    assert len(out) == len(vals)
    for v, line in zip(vals, out):
        want = "|".join([rust_fixed(v, 4), rust_fixed(v, 6), rust_exp(v, 3), rust_exp(v, 8), rust_exp_short(v),
                         rust_display(v)])
        assert line == want, (v, line, want)


def test_rust_formats_known_answers():
    """Known outputs of Rust's formatter for the driver's formats."""
    assert rust_exp(1.5e-5, 8) == "1.50000000e-5"
    assert rust_exp(-2.5e10, 3) == "-2.500e10"
    assert rust_exp(0.0, 3) == "0.000e0"
    assert rust_exp_short(1.0e6) == "1e6" and rust_exp_short(1.5e8) == "1.5e8"
    assert rust_exp_short(1.0e-7) == "1e-7"
    assert rust_display(0.71) == "0.71" and rust_display(1.0) == "1" and rust_display(100.0) == "100"
    assert rust_display(1e-7) == "0.0000001" and rust_display(-0.1) == "-0.1"
    assert rust_display(2.3585) == "2.3585" and rust_display(-0.0) == "-0"
    assert rust_fixed(float("nan"), 4) == "NaN" and rust_exp(float("inf"), 3) == "inf"
    assert rust_fixed(-1e-9, 4) == "-0.0000"


def test_driver_formats_match_restatement():
    rng = np.random.default_rng(7)
    vals = [0.71, 1.0, 1e-7, 1e21, -0.1, 2.3585, 100.0, 0.0, -0.0, 1e6, 1.5e8, 12345.0, 0.1 + 0.2,
            5e-324, 1.7976931348623157e308, float("nan"), float("inf"), -float("inf"), 0.5, 2.5, 1e-300,
            123456789.0, 9.999999999e-5, 0.99999995]
    vals += list(rng.normal(size=200) * 10.0 ** rng.integers(-12, 12, size=200))
    vals += list(rng.random(100))
    _check_values([float(v) for v in vals])
