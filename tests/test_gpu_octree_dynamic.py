"""The octree's dynamic mixed-scale SGS model on the GPU
(cav_octree_set_dynamic_sgs; src/octree/smag.rs and the dynamic branch of
step_cavity, src/octree/solver.rs:647-947) against the FP64 oracle.

FP64: the model's a^alpha powers (CUDA's pow against the host's, within 2
ulp) and the means behind xi A / xi B (a fixed-order tree against the
reference's sequential sum) are the only operations that are not bit-exact,
so the GPU and the oracle agree to rounding level, not bit for bit;
tolerances are stated in each test.  The reference's tests of the path
(src/octree/tests.rs:594-784) run on the GPU solver too.
"""
import numpy as np
import pytest

import oracle
from cfd_cavity_b200 import _lib as L
from cfd_cavity_b200.octree import OctreeSolver

pytestmark = pytest.mark.gpu

ARGS = (32, 64, 4, 1.0e6, 0.71, 0.02, 42)


def pair(levels=3, args=ARGS, **kw):
    g = OctreeSolver(*args, levels=levels, precision="f64", **kw)
    o = oracle.OracleOctree(*args, levels=levels, **kw)
    g.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    o.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    return g, o


def max_rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("levels", [2, 3])
def test_fp64_first_step_model_matches_oracle(levels):
    """One coarse step: nu_t / alpha_t of every level within 1e-12 of the
    largest value (relative) and every field within 1e-13."""
    g, o = pair(levels)
    g.step_cavity(1)
    o.step_cavity(1)
    for lvl in range(3 if levels == 2 else 5):
        for a, b in zip(g.nu_t(lvl), o.nu_t(lvl)):
            assert max_rel(a, b) <= 1e-12, lvl
        lg, lo = g.level(lvl, pops=True), o.level(lvl, pops=True)
        for k in ("rho", "ux", "uy", "temp", "f", "g"):
            assert np.max(np.abs(lg[k] - lo[k])) <= 1e-13, (lvl, k)


@pytest.mark.parametrize("nu_start_mult", [2.5, 1.0])
def test_fp64_many_steps_close_to_oracle(nu_start_mult):
    """40 coarse steps, 3 levels, with the viscosity ramp (host-launched
    steps) and without it (graphs of 16 steps): fields within 1e-11,
    coefficient statistics within 1e-9 (relative), rescaling factors within
    1e-12.  Measured on a B200: bit-identical fields."""
    args = (48, 96, 6, 1.0e7, 0.71, 0.03, 7)
    g, o = pair(3, args, nu_start_mult=nu_start_mult)
    g.step_cavity(1)
    n0 = g.launch_count()
    g.step_cavity(39)
    o.step_cavity(40)
    per_step = (g.launch_count() - n0) / 39
    # L0: 3 model kernels + statistics + 2 for xi A + collide + step; c2f;
    # L1: 3 + collide + step; 2 for xi B; c2f; 2 x L2 (3 + collide + step);
    # f2c; L1 again (5); f2c; step counter
    assert per_step == 35, per_step
    for lvl in range(5):
        lg, lo = g.level(lvl), o.level(lvl)
        for k in ("rho", "ux", "uy", "temp"):
            assert np.max(np.abs(lg[k] - lo[k])) <= 1e-11, (lvl, k)
    dg, do = g.dynamic_stats(), o.dynamic_stats()
    for k in ("cs_dyn_mean", "cs_dyn_max", "kappa_dyn_mean", "kappa_dyn_max", "nu_t_max"):
        assert abs(dg[k] - do[k]) <= 1e-9 * max(abs(do[k]), 1e-30), k
    for k in dg:
        if k.startswith("xi"):
            assert abs(dg[k] - do[k]) <= 1e-12, k
    assert g.time_step == 40


def test_fp64_toggle_on_off_matches_oracle():
    """3 dynamic steps, then 3 molecular ones (the molecular path resumes from
    the REF state), against the oracle doing the same."""
    g, o = pair(3)
    g.step_cavity(3)
    o.step_cavity(3)
    g.set_dynamic_sgs(False, 0.5, -0.1, 2.0)
    o.set_dynamic_sgs(False, 0.5, -0.1, 2.0)
    g.step_cavity(20)
    o.step_cavity(20)
    for lvl in range(5):
        lg, lo = g.level(lvl, pops=True), o.level(lvl, pops=True)
        for k in ("rho", "ux", "uy", "temp", "f", "g"):
            assert np.max(np.abs(lg[k] - lo[k])) <= 1e-12, (lvl, k)


def test_off_leaves_path_bit_identical():
    """dynamic_smag_off_matches_fixed_cs_nu_t (src/octree/tests.rs:601-620)."""
    a = OctreeSolver(*ARGS, levels=3, precision="f64")
    a.set_dynamic_sgs(False, 0.5, -0.1, 2.0)
    b = OctreeSolver(*ARGS, levels=3, precision="f64")
    a.step_cavity(5)
    b.step_cavity(5)
    for lvl in range(5):
        la, lb = a.level(lvl, pops=True), b.level(lvl, pops=True)
        for k in ("f", "g"):
            np.testing.assert_array_equal(la[k], lb[k])


@pytest.mark.parametrize("prec", ["f64", "f32", "f32_f16"])
def test_on_runs_sane_and_reports_coefficients(prec):
    """dynamic_smag_on_runs_sane_and_reports_coefficients
    (src/octree/tests.rs:627-676)."""
    sim = OctreeSolver(*ARGS, levels=3, precision=prec)
    sim.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    for _ in range(5):
        sim.step_cavity(1)
        d = sim.dynamic_stats()
        assert np.isfinite(d["cs_dyn_mean"]) and np.isfinite(d["cs_dyn_max"])
        assert 0.0 <= d["cs_dyn_max"] <= 0.04
        assert d["cs_dyn_mean"] <= d["cs_dyn_max"] + 1e-12
        assert 0.0 <= d["kappa_dyn_max"] <= 0.04
        for lvl in (0, 1):
            l = sim.level(lvl)
            for k in ("rho", "ux", "uy", "temp"):
                assert np.all(np.isfinite(l[k]))
            for v in sim.nu_t(lvl):
                assert np.all(np.isfinite(v))
        assert sim.check_guards() == 0
    for v in sim.nu_t(3):
        assert np.all(np.isfinite(v))


def test_xi_recomputed_from_effective_taus():
    """dynamic_smag_xi_recomputed_from_effective_taus
    (src/octree/tests.rs:687-784) on the GPU solver."""
    off = OctreeSolver(*ARGS, levels=3, precision="f64")
    d0 = off.dynamic_stats()
    i0 = off.info()
    off.step_cavity(5)
    assert off.dynamic_stats() == d0                   # flag off: never rewritten
    sim = OctreeSolver(*ARGS, levels=3, precision="f64")
    sim.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    assert sim.dynamic_stats()["xi_even"] == d0["xi_even"]
    sim.step_cavity(5)
    d = sim.dynamic_stats()
    assert d["nu_t_max"] > 0.0
    assert d["xi_even"] != d0["xi_even"] and d["xi_th"] != d0["xi_th"]
    assert 0.0 < d["xi_even"] and abs(d["xi_even"] - d0["xi_even"]) / d0["xi_even"] < 0.1
    assert d["xi_b_hot_even"] != d0["xi_b_hot_even"]
    bis = OctreeSolver(*ARGS, levels=3, precision="f64")
    bis.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    bis.step_cavity(5)
    assert bis.dynamic_stats() == d                    # deterministic reductions
    assert i0["time_step"] == 0


@pytest.mark.parametrize("prec,tol_t", [("f32", 1e-4), ("f32_f16", 3e-3)])
def test_reduced_precision_dynamic_against_fp64(prec, tol_t):
    """64 x 256 base, bl_width 8, 3 levels, Ra = 1e7, 300 dynamic coarse
    steps: max |T - T_64| over every level <= tol_t."""
    args = (64, 256, 8, 1.0e7, 0.71, 0.02, 42)
    ref = OctreeSolver(*args, levels=3, precision="f64")
    red = OctreeSolver(*args, levels=3, precision=prec)
    for s in (ref, red):
        s.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
        s.step_cavity(300)
    for lvl in range(5):
        a, b = ref.level(lvl), red.level(lvl)
        assert np.max(np.abs(a["temp"] - b["temp"])) <= tol_t, lvl
    dr, dd = ref.dynamic_stats(), red.dynamic_stats()
    assert abs(dd["xi_even"] - dr["xi_even"]) <= 1e-5
    assert red.diag()["finite"] == 1.0


def test_dynamic_argument_checks():
    s = OctreeSolver(*ARGS, levels=2, precision="f64", cs=0.1)
    with pytest.raises(L.CavError) as e:
        s.set_dynamic_sgs(True)
    assert e.value.code == L.CAV_ERR_ARG
    t = OctreeSolver(*ARGS, levels=2, precision="f64")
    with pytest.raises(L.CavError) as e:
        t.nu_t(0)
    assert e.value.code == L.CAV_ERR_STATE
    for bad in ({"smag_alpha": 1.5}, {"eta_test": 0.5}, {"nu_sm_min": float("nan")}):
        with pytest.raises(L.CavError) as e:
            t.set_dynamic_sgs(True, **bad)
        assert e.value.code == L.CAV_ERR_ARG
    with pytest.raises(L.CavError):
        t.nu_t(3)
