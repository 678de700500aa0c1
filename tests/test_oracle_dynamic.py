"""The dynamic mixed-scale subgrid model (--dynamic-smag) on the FP64 oracle:
the reference's own tests (src/uniform/tests.rs:515-578) on its restatement
of compute_dynamic_sgs (src/uniform/solver.rs:562-828)."""
import numpy as np

import oracle


def small():
    # small_solver(), src/uniform/tests.rs:11-13
    return oracle.OracleSolver(16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42)


def test_lilly_coefficient_clamps_on_zero_denominator_and_bounds():
    """src/uniform/tests.rs:517-529."""
    L = oracle.lilly_coefficient
    assert L(1.0, 0.0) == 0.0
    assert L(1.0, -1e-12) == 0.0
    assert L(float("nan"), 1.0) == 0.0
    assert abs(L(0.02, 1.0) - 0.01) < 1e-12
    assert L(100.0, 1.0) == 0.04
    assert L(-100.0, 1.0) == 0.0


def test_mixed_factor_alpha_half_is_geometric_mean():
    """src/uniform/tests.rs:531-541."""
    a, b = 4.0, 9.0
    assert abs(oracle.mixed_factor(a, b, 0.5) - (a * b) ** 0.5) < 1e-12
    assert abs(oracle.mixed_factor(a, b, 0.0) - b) < 1e-12
    assert abs(oracle.mixed_factor(a, b, 1.0) - a) < 1e-12


def test_dynamic_smag_off_matches_fixed_cs_nu_t():
    """src/uniform/tests.rs:543-559."""
    s, r = small(), small()
    s.set_dynamic_sgs(False, 0.5, -0.1, 2.0)
    s.step(30)
    r.step(30)
    np.testing.assert_array_equal(s.fields()["nu_t"], r.fields()["nu_t"])
    st = s.dynamic_stats()
    assert np.isnan(st[4]).all()  # no per-node buffers in the off mode


def test_dynamic_smag_on_runs_sane_and_reports_coefficients():
    """src/uniform/tests.rs:561-578."""
    s = small()
    s.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    s.step(5)
    mean, mx, kmean, kmx, nut_pre, at_pre = s.dynamic_stats()
    assert np.isfinite([mean, mx, kmean, kmx]).all()
    assert 0.0 <= mx <= 0.04
    assert mean <= mx + 1e-12
    assert np.isfinite(s.fields()["nu_t"]).all()
    np.testing.assert_array_equal(s.fields()["nu_t"], nut_pre)  # the collision used nu_t_pre
