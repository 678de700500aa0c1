"""The octree reference tests (src/octree/tests.rs) on the FP64 oracle.

The oracle restates src/octree/{grid,interface,lbm,cavity,solver}.rs; these
are the reference's own checks of that code, on the same configuration
(CavitySolver::new(32, 64, 4, 1e6, 0.71, 0.02, 42, 1, false, levels, 1.0,
None)) and with the same tolerances, plus the relaxation-time and rescaling
identities of v1_xi_matches_relaxation_time_ratio.
"""
import pytest

import oracle

LAMBDA = 3.0 / 16.0


def small(levels=2):
    return oracle.OracleOctree(32, 64, 4, 1.0e6, 0.71, 0.02, 42, levels=levels)


def test_v2_cavity_mass_conserved_with_guo_force():
    """src/octree/tests.rs:397-407: |mean rho - 1| < 1e-6 over 10 steps."""
    sim = small()
    for _ in range(10):
        sim.step_cavity()
        assert abs(sim.diag()["mass"] - 1.0) < 1e-6


def test_v2_noise_stats_bounded_and_covers_both_levels():
    """src/octree/tests.rs:419-448."""
    sim = small()
    for step in range(20):
        sim.step_cavity()
        d = sim.diag()
        assert d["max_rho_dev"] >= d["max_rho_dev_ifaces"]
        if step >= 5:
            assert d["max_rho_dev_ifaces"] < 1.0


def test_v2_nusselt_conductive_initial():
    """src/octree/tests.rs:450-476: Nu (2nd link, Lx scale) ~ 1 at step 0."""
    d = small().diag()
    assert abs(d["nu_hot"] - 1.0) < 0.05
    assert abs(d["nu_cold"] - 1.0) < 0.05
    # the fine-field estimator is exactly conductive on the interpolated field
    assert abs(d["nu_hot_fine"] - 1.0) < 0.05


def tau_plus(nu):
    return 0.5 + 3.0 * nu


def test_v6_multilevel_mapping_structure():
    """src/octree/tests.rs:478-547: nx2 = 7, tau+ of L2 from 4 nu, xi_even of
    the L1/L2 interface = tau+_L2 / tau+_L1 / 2."""
    sim = small(levels=3)
    i = sim.info()
    nu0 = i["nu"]
    assert sim.level_dims(3) == (7, sim.level_dims(1)[1] * 2 - 3)
    assert sim.level_dims(4)[0] == 7
    tp2 = 0.5 + 3.0 * (4.0 * nu0)
    assert abs(i["tau_plus_l2"] - tp2) < 1e-15
    assert abs(i["xi_even_sub"] - 0.5 * tp2 / i["tau_plus_l1"]) < 1e-15
    assert abs(i["tau_plus_l1"] - (0.5 + 3.0 * 2.0 * nu0)) < 1e-15


def test_v6_cavity_3levels_stable_short():
    """src/octree/tests.rs:549-580."""
    sim = small(levels=3)
    for _ in range(10):
        sim.step_cavity()
        d = sim.diag()
        assert abs(d["mass"] - 1.0) < 1e-6
        assert d["max_rho_dev"] >= d["max_rho_dev_ifaces"]
        assert d["max_rho_dev_ifaces"] < 1.0
        assert d["max_u"] <= 0.10 and d["finite"] == 1.0


@pytest.mark.parametrize("odd_exact", [False, True])
def test_v1_xi_matches_relaxation_time_ratio(odd_exact):
    """src/octree/tests.rs:322-390 (relaxation-time identities), on the
    factors the octree derives in CavitySolver::new."""
    sim = oracle.OracleOctree(32, 64, 4, 1.0e6, 0.71, 0.02, 42, odd_exact=odd_exact)
    i = sim.info()
    nu, al = i["nu"], i["alpha"]
    tpc, tpf = tau_plus(nu), tau_plus(2 * nu)
    assert abs(tpf - 0.5 - 2.0 * (tpc - 0.5)) < 1e-15
    assert i["xi_even"] == 0.5 * tpf / tpc
    assert i["xi_thermal"] == 0.5 * (0.5 + 3.0 * 2 * al) / (0.5 + 3.0 * al)
    if odd_exact:
        tmc = 0.5 + LAMBDA / (tpc - 0.5)
        tmf = 0.5 + LAMBDA / (tpf - 0.5)
        assert i["xi_odd"] == 0.5 * tmf / tmc
    else:
        assert i["xi_odd"] == 0.5


def test_grid_tables_counts():
    """OctreeGrid::build (src/octree/grid.rs:103-204) on the cavity blocks:
    ghost ring 2 (nx1 + ny1) - 4 per block; coincident nodes exclude the
    domain boundary (hot block loses column 0)."""
    sim = small()
    nx1, ny1 = sim.level_dims(1)
    assert (nx1, ny1) == (2 * 4 + 3, 2 * 63 + 3)
    i = sim.info()
    assert i["n_ghosts"] == 2 * (2 * (nx1 + ny1) - 4)
    # hot: cx in 1..3, cold: cx in 27..30; cy in 1..62
    assert i["n_coincident"] == (3 + 4) * 62
