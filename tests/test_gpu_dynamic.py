"""The dynamic mixed-scale subgrid model on the GPU (cav_set_dynamic_sgs).

Against the FP64 oracle (its restatement of compute_dynamic_sgs,
src/uniform/solver.rs:562-828): every quantity of the model is evaluated in
the reference's order except the a^alpha powers (CUDA's pow, within 2 ulp of
the C library's), so the FP64 fields agree to a relative 1e-12 after one
step and 1e-9 after 300 (tolerances in each test).  Plus the reference's
own dynamic-model tests (src/uniform/tests.rs:543-578) on the GPU path.
"""
import numpy as np
import pytest

import oracle
from cfd_cavity_b200 import CavitySolver
from cfd_cavity_b200 import _lib as L

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("args,steps,tol", [
    ((16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42), 1, 1e-12),
    ((16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42), 40, 1e-10),
    ((64, 256, 1.0e7, 0.71, 0.1, 0.9, 0.02, 7), 300, 1e-9),
])
def test_fp64_dynamic_model_matches_oracle(args, steps, tol):
    g = CavitySolver(*args, precision="f64")
    o = oracle.OracleSolver(*args)
    g.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    o.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    g.step(steps)
    o.step(steps)
    fg, fo = g.fields(), o.fields()
    for k in ("rho", "ux", "uy", "temperature", "nu_t"):
        assert rel(fg[k], fo[k]) <= tol, (k, rel(fg[k], fo[k]))
    sg = g.dynamic_stats()
    so = o.dynamic_stats()
    assert abs(sg["cs_dyn_max"] - so[1]) <= 1e-9 * max(so[1], 1e-30)
    assert abs(sg["cs_dyn_mean"] - so[0]) <= 1e-9 * max(so[0], 1e-30)
    assert abs(sg["kappa_dyn_max"] - so[3]) <= 1e-9 * max(so[3], 1e-30)


def test_dynamic_smag_off_matches_fixed_cs_nu_t():
    """src/uniform/tests.rs:543-559 on the GPU: the switch off leaves the step
    bit-identical."""
    a = CavitySolver(16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42, precision="f64")
    b = CavitySolver(16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42, precision="f64")
    a.set_dynamic_sgs(False, 0.5, -0.1, 2.0)
    a.step(30)
    b.step(30)
    np.testing.assert_array_equal(a.fields()["nu_t"], b.fields()["nu_t"])
    assert a.dynamic_stats()["cs_dyn_max"] == 0.0


@pytest.mark.parametrize("precision", ["f64", "f32", "f16sr"])
def test_dynamic_smag_on_runs_sane_and_reports_coefficients(precision):
    """src/uniform/tests.rs:561-578 on the GPU path, every storage format."""
    s = CavitySolver(16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42, precision=precision)
    s.set_dynamic_sgs(True, 0.5, -0.1, 2.0)
    s.step(5)
    st = s.dynamic_stats()
    assert all(np.isfinite(v) for v in st.values())
    assert 0.0 <= st["cs_dyn_max"] <= 0.04
    assert st["cs_dyn_mean"] <= st["cs_dyn_max"] + 1e-12
    assert np.isfinite(s.fields()["nu_t"]).all()


def test_fp32_dynamic_against_fp64():
    """FP32 storage with the dynamic model vs FP64, 64x256 Ra = 1e7, 300
    steps: max |T - T_64| <= 1e-5 (temperatures are O(0.5))."""
    args = (64, 256, 1.0e7, 0.71, 0.1, 0.9, 0.02, 7)
    a = CavitySolver(*args, precision="f64")
    b = CavitySolver(*args, precision="f32")
    for s in (a, b):
        s.set_dynamic_sgs(True)
        s.step(300)
    assert np.max(np.abs(a.fields()["temperature"] - b.fields()["temperature"])) <= 1e-5


def test_dynamic_model_argument_checks_and_adjoint_refusal():
    s = CavitySolver(16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42, precision="f64")
    with pytest.raises(L.CavError) as e:
        s.set_dynamic_sgs(True, 1.5, -0.1, 2.0)
    assert e.value.code == L.CAV_ERR_ARG
    with pytest.raises(L.CavError):
        s.set_dynamic_sgs(True, 0.5, -0.1, 0.5)
    s.set_dynamic_sgs(True)
    with pytest.raises(L.CavError) as e:
        s.adjoint_nusselt(100, 50, 10)
    assert e.value.code == L.CAV_ERR_STATE
