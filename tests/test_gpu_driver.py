"""The driver binary ``cavity_les`` end to end on the GPU.

FP64 runs are compared with the reference driver's loop restated on the FP64
oracle (tests/driver_expect.py: run_uniform / run_octree of src/main.rs and
Rust's float formats): progress.log, fields_mean.csv, profiles_w.csv,
snapshot.vti, snapshot.bin and summary.json must be the same bytes.  The
only values not computed in the reference's order are device reductions
printed at 3-6 digits (mass, Nusselt sums, y+), which agree at that
precision.  Also: the exit codes of the reference (2 guard, 3 no samples),
--snapshot-every + --restart with regridding, the dynamic model's extra
outputs and a reduced-precision run.
"""
import json
import os
import subprocess

import pytest

from driver_expect import octree_progress, rust_display, rust_exp, rust_fixed, uniform_run

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
BIN = os.path.join(ROOT, "cfd_cavity_b200", "_build", "cavity_les")


def run(args, timeout=600):
    return subprocess.run([BIN, *[str(a) for a in args]], capture_output=True, text=True, timeout=timeout)


def read(path, binary=False):
    with open(path, "rb" if binary else "r", encoding=None if binary else "utf-8") as f:
        return f.read()


def test_uniform_fp64_outputs_match_reference_loop(tmp_path):
    nx, ny, ra, steps, ss, se, pe = 24, 96, 1.0e5, 301, 100, 50, 100
    out = tmp_path / "u"
    r = run(["--nx", nx, "--ny", ny, "--ra", "1e5", "--steps", steps, "--sample-start", ss, "--sample-every", se,
             "--progress-every", pe, "--out", out])
    assert r.returncode == 0, r.stderr
    exp = uniform_run(nx, ny, ra, steps, ss, se, pe)
    assert "Moyennage sur 5 échantillons." in r.stdout and exp["n_samples"] == 5
    for name in ("progress.log", "fields_mean.csv", "profiles_w.csv", "snapshot.vti", "summary.json"):
        got = read(out / name)
        assert got == exp[name], name
    assert read(out / "snapshot.bin", binary=True) == exp["snapshot.bin"]
    json.loads(read(out / "summary.json"))
    s = exp["summary"]
    assert f"Nuc = {rust_fixed(s['nuc'], 4)} | Nuf = {rust_fixed(s['nuf'], 4)}" in r.stdout
    assert f"y+ (paroi chaude) = {rust_fixed(s['yplus'], 3)}" in r.stdout


def test_octree_fp64_progress_matches_reference_loop(tmp_path):
    args = dict(nx0=32, ny0=128, bl_width=4, ra=1.0e6, steps=61, sample_start=20, sample_every=10,
                progress_every=20, levels=3)
    out = tmp_path / "o"
    r = run(["--mode", "octree", "--nx0", 32, "--ny0", 128, "--bl-width", 4, "--levels", 3, "--ra", "1e6",
             "--steps", 61, "--sample-start", 20, "--sample-every", 10, "--progress-every", 20, "--out", out])
    assert r.returncode == 0, r.stderr
    log, means, cnt, nmax, imax = octree_progress(**args)
    nuc, nuf, nucl0, nufine = means
    ecart = abs((nuc - 2.3585) / 2.3585) * 100.0
    summary = (f"--- Bilan (moyenné sur {cnt} échantillons, fenêtre 20→61) ---\n"
               f"Nuc (2ᵉ liaison) = {rust_fixed(nuc, 4)} | écart like-for-like vs {rust_display(2.3585)} = "
               f"{rust_fixed(ecart, 1)} %\n"
               f"Nuc_link0 (1ʳᵉ liaison) = {rust_fixed(nucl0, 4)} | Nuf = {rust_fixed(nuf, 4)} | "
               f"Nu_fin (bloc chaud) = {rust_fixed(nufine, 4)}\n"
               f"Références uniforme Ra=1e6 : 2ᵉ liaison = 2.3585 | 1ʳᵉ liaison = 1.366\n"
               f"Bruit acoustique (max sur la run) : max|ρ−ρ̄| = {rust_exp(nmax, 3)} | interfaces = "
               f"{rust_exp(imax, 3)}\n"
               f"PORTE V2 (écart Nuc ≤ 5 %) : {'PASS' if ecart <= 5.0 else 'FAIL'}")
    assert read(out / "progress.log") == "\n".join(log + [summary]) + "\n"


def test_snapshot_every_and_restart_with_regrid(tmp_path):
    a, b = tmp_path / "a", tmp_path / "b"
    r = run(["--nx", 24, "--ny", 96, "--steps", 200, "--sample-start", 100, "--sample-every", 50,
             "--progress-every", 100, "--snapshot-every", 100, "--out", a])
    assert r.returncode == 0, r.stderr
    assert "snapshot exporté au pas 99" in r.stdout and "snapshot exporté au pas 199" in r.stdout
    assert read(a / "snapshot.bin", binary=True)[:8] == b"CAVSNAP1"
    r = run(["--nx", 32, "--ny", 128, "--steps", 20, "--sample-start", 0, "--sample-every", 10,
             "--progress-every", 10, "--restart", a / "snapshot.bin", "--out", b])
    assert r.returncode == 0, r.stderr
    assert f"Restart depuis {a / 'snapshot.bin'} : snapshot 24×96 → grille 32×128 (interpolation bilinéaire)" \
        in r.stdout
    r = run(["--nx", 32, "--ny", 128, "--steps", 5, "--restart", tmp_path / "missing.bin", "--out", b])
    assert r.returncode == 6


def test_octree_snapshot_every_and_restart(tmp_path):
    a = tmp_path / "oa"
    common = ["--mode", "octree", "--nx0", 32, "--ny0", 128, "--bl-width", 4, "--sample-start", 0,
              "--sample-every", 5, "--progress-every", 10]
    r = run(common + ["--steps", 20, "--snapshot-every", 10, "--out", a])
    assert r.returncode == 0, r.stderr
    assert "snapshot final exporté au pas 19" in r.stdout
    assert read(a / "snapshot.bin", binary=True)[:8] == b"OCTSNAP1"
    r = run(common + ["--steps", 10, "--restart", a / "snapshot.bin", "--out", tmp_path / "ob"])
    assert r.returncode == 0, r.stderr
    assert "snapshot levels=2 (3 grilles), pas 20" in r.stdout


def test_no_samples_exits_three(tmp_path):
    r = run(["--nx", 24, "--ny", 96, "--steps", 50, "--sample-start", 100, "--out", tmp_path / "n"])
    assert r.returncode == 3 and "Aucun échantillon moyenné" in r.stderr
    r = run(["--mode", "octree", "--nx0", 32, "--ny0", 128, "--bl-width", 4, "--steps", 10, "--sample-start",
             100, "--out", tmp_path / "m"])
    assert r.returncode == 3


def test_guard_exits_two_and_keeps_log(tmp_path):
    """A buoyancy far beyond the lattice's range (Ra = 1e14 on 16 x 64 with
    nu forced to 1.9e-3, beta_eff ~ 2e3) trips the guard at the first
    progress check; a forced nu whose tau_t falls under the reference's 0.505
    floor is refused at creation."""
    out = tmp_path / "g"
    r = run(["--nx", 16, "--ny", 64, "--ra", "1e14", "--nu", "0.0005", "--out", out])
    assert r.returncode == 101 and "tau_t too close to 0.5" in r.stderr
    r = run(["--nx", 16, "--ny", 64, "--ra", "1e14", "--nu", "0.0019", "--cs", 0, "--steps", 500,
             "--progress-every", 10, "--out", out])
    assert r.returncode == 2, (r.stdout, r.stderr)
    assert "AVORT : max_u" in r.stderr or "DIVERGENCE détectée" in r.stderr
    if "AVORT" in r.stderr:
        assert read(out / "progress.log").splitlines()[-1].startswith("AVORT : max_u = ")


def test_dynamic_model_outputs(tmp_path):
    out = tmp_path / "d"
    r = run(["--nx", 24, "--ny", 96, "--steps", 60, "--sample-start", 20, "--sample-every", 20,
             "--progress-every", 20, "--dynamic-smag", "--out", out])
    assert r.returncode == 0, r.stderr
    assert "cs_dyn_mean = " in read(out / "progress.log")
    d = json.loads(read(out / "dynamic_sgs.json"))
    assert d["dynamic_smag"] is True and 0.0 <= d["cs_dyn_max"] <= 0.04
    r = run(["--mode", "octree", "--nx0", 32, "--ny0", 128, "--bl-width", 4, "--levels", 3, "--steps", 20,
             "--sample-start", 0, "--sample-every", 10, "--progress-every", 10, "--dynamic-smag",
             "--out", tmp_path / "do"])
    assert r.returncode == 0, r.stderr
    assert "cs_dyn = " in read(tmp_path / "do" / "progress.log")


@pytest.mark.parametrize("mode,prec", [("uniform", "f16sr"), ("octree", "f32_f16")])
def test_reduced_precision_runs(tmp_path, mode, prec):
    geo = ["--nx", 32, "--ny", 128] if mode == "uniform" else ["--nx0", 32, "--ny0", 128, "--bl-width", 4]
    r = run(["--mode", mode, *geo, "--precision", prec, "--steps", 100, "--sample-start", 50, "--sample-every",
             10, "--progress-every", 50, "--out", tmp_path / prec])
    assert r.returncode == 0, r.stderr
    assert os.path.exists(tmp_path / prec / "progress.log")
