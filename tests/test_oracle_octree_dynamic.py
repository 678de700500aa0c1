"""The oracle's octree dynamic mixed-scale SGS path (src/octree/smag.rs and the
dynamic branch of step_cavity, src/octree/solver.rs:647-947), checked with the
reference's own tests of that path (src/octree/tests.rs:594-784), restated on
the FP64 oracle:

  * dynamic_smag_off_matches_fixed_cs_nu_t: the flag off leaves the path
    untouched, bit for bit;
  * dynamic_smag_on_runs_sane_and_reports_coefficients: Lilly coefficients in
    [0, 0.04], finite fields and nu_t / alpha_t on every level;
  * dynamic_smag_xi_recomputed_from_effective_taus: the molecular factors at
    step 0, recomputed factors within 10 % of them afterwards (xi A and xi
    B), unchanged factors with the flag off, determinism.
The per-grid model itself is shared with the uniform path (dynamic_sgs_grid),
whose checks live in test_oracle_dynamic.py.
"""
import numpy as np

import oracle

ARGS = (32, 64, 4, 1.0e6, 0.71, 0.02, 42)


def mol_xi(ra):
    """rescaling_factors_multilevel of the molecular taus (tests.rs:695-708)."""
    utarget, pr, lz = 0.02, 0.71, 63.0
    nu = (utarget * np.sqrt(pr) * lz / (1.7 * np.sqrt(ra))) ** (2.0 / 3.0)
    alpha = nu / pr

    def tau(n, a):
        tp = 0.5 + 3.0 * n
        return tp, 0.5 + (3.0 / 16.0) / (tp - 0.5), 0.5 + 3.0 * a

    def xi(c, f):
        return 0.5 * f[0] / c[0], 0.5, 0.5 * f[2] / c[2]

    tc, tf, ts = tau(nu, alpha), tau(2 * nu, 2 * alpha), tau(4 * nu, 4 * alpha)
    return xi(tc, tf), xi(tf, ts)


def test_off_matches_untouched_path():
    a = oracle.OracleOctree(*ARGS, levels=3)
    a.set_dynamic_sgs(False, 0.5, -0.1, 2.0)
    b = oracle.OracleOctree(*ARGS, levels=3)
    a.step_cavity(5)
    b.step_cavity(5)
    for lvl in range(5):
        la, lb = a.level(lvl, pops=True), b.level(lvl, pops=True)
        for k in ("f", "g", "rho", "ux", "uy", "temp"):
            np.testing.assert_array_equal(la[k], lb[k], err_msg=f"{lvl} {k}")


def test_on_runs_sane_and_reports_coefficients():
    sim = oracle.OracleOctree(*ARGS, levels=3)
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
                assert np.all(np.isfinite(l[k])), (lvl, k)
        for lvl in (0, 1):
            nt, at = sim.nu_t(lvl)
            assert np.all(np.isfinite(nt)) and np.all(np.isfinite(at))
        dg = sim.diag()
        assert dg["max_u"] <= 0.10 and dg["finite"] == 1.0
    nt, at = sim.nu_t(3)
    assert np.all(np.isfinite(nt)) and np.all(np.isfinite(at))
    # the TRT floor of the model (smag.rs:380-396): tau+ and tau_t stay >= 0.505
    info = sim.info()
    for lvl, mult in ((0, 1.0), (1, 2.0), (3, 4.0)):
        nt, at = sim.nu_t(lvl)
        assert np.all(0.5 + 3.0 * (mult * info["nu"] + nt) >= 0.505 - 1e-15)
        assert np.all(0.5 + 3.0 * (mult * info["alpha"] + at) >= 0.505 - 1e-15)


def test_xi_recomputed_from_effective_taus():
    xa_mol, xb_mol = mol_xi(1.0e6)
    sim0 = oracle.OracleOctree(*ARGS, levels=2)
    i0 = sim0.info()
    assert i0["xi_even"] == xa_mol[0] and i0["xi_thermal"] == xa_mol[2]

    sim = oracle.OracleOctree(*ARGS, levels=3)
    sim.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    d0 = sim.dynamic_stats()
    assert (d0["xi_even"], d0["xi_odd"], d0["xi_th"]) == xa_mol
    sim.step_cavity(5)
    d = sim.dynamic_stats()
    assert d["nu_t_max"] > 0.0
    assert d["xi_even"] != xa_mol[0] and d["xi_th"] != xa_mol[2]
    assert d["xi_even"] > 0.0
    assert abs(d["xi_even"] - xa_mol[0]) / xa_mol[0] < 0.1
    assert d["xi_b_hot_even"] != xb_mol[0]
    assert d["xi_b_hot_even"] != d["xi_b_cold_even"]   # one xi B per strip

    off = oracle.OracleOctree(*ARGS, levels=3)
    off.step_cavity(5)
    doff = off.dynamic_stats()
    assert (doff["xi_even"], doff["xi_odd"], doff["xi_th"]) == xa_mol
    assert (doff["xi_b_hot_even"], doff["xi_b_hot_odd"], doff["xi_b_hot_th"]) == xb_mol

    bis = oracle.OracleOctree(*ARGS, levels=3)
    bis.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    bis.step_cavity(5)
    assert bis.dynamic_stats() == d
