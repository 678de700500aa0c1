"""Known-answer tests of the reference, written once for any solver object.

Each function restates one test of ``src/uniform/tests.rs`` (line ranges
cited) against an object with the ``CavitySolver`` interface: the oracle
(``oracle.OracleSolver``, CPU) or the CUDA path
(``cfd_cavity_b200.CavitySolver``).  ``make(nx, ny, ra, pr, cs, pr_t,
utarget, seed, jobs, alpha_mult, nu_start_mult, nu_override)`` builds one.
``tol`` scales the absolute tolerances for reduced-precision storage.
"""
from __future__ import annotations

import numpy as np

T_HOT, T_COLD, DELTA_T = 0.5, -0.5, 1.0
EPS = 1e-10


def small(make):
    """``small_solver``, src/uniform/tests.rs:11-13."""
    return make(16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42, 1, 1.0, 1.0, None)


def init_temperature_linear_and_bounded(make, tol=1.0):
    """src/uniform/tests.rs:138-149."""
    s = small(make)
    f = s.fields()
    nx = s.nx()
    assert abs(f["temperature"][s.idx(0, 10)] - T_HOT) < 2e-3
    assert abs(f["temperature"][s.idx(nx - 1, 10)] - T_COLD) < 2e-3
    assert np.all(np.abs(f["ux"]) < EPS)
    assert np.all(np.abs(f["uy"]) < EPS)


def mass_conserved_per_phase(make, tol=1.0):
    """src/uniform/tests.rs:154-169 (each phase within 1e-8)."""
    s = small(make)
    m0 = s.total_f_mass()
    s.collide(100)
    m1 = s.total_f_mass()
    s.stream()
    m2 = s.total_f_mass()
    s.apply_bounce_back()
    m3 = s.total_f_mass()
    s.apply_thermal_boundary_conditions()
    m4 = s.total_f_mass()
    for m in (m1, m2, m3, m4):
        assert abs(m - m0) < 1e-8 * tol, (m0, m1, m2, m3, m4)


def guo_forcing_preserves_mass_and_upward_sign(make, tol=1.0):
    """src/uniform/tests.rs:174-222: mass after 210 steps (rel 1e-9) and
    u_y = (sum c_y f)/rho + 0.5 fy/rho at every interior node (1e-12)."""
    s = small(make)
    m0 = s.total_f_mass()
    s.step(210)
    m1 = s.total_f_mass()
    assert abs(m1 - m0) / abs(m0) < 1e-9 * tol, (m0, m1)
    f, _ = s.populations()
    fl = s.fields()
    nx, ny = s.nx(), s.ny()
    cy = np.array([0, 0, 1, 1, 1, 0, -1, -1, -1], dtype=np.float64)
    worst = 0.0
    for iy in range(1, ny - 1):
        for ix in range(1, nx - 1):
            k = s.idx(ix, iy)
            mom_y = 0.0
            for j in range(9):
                mom_y += cy[j] * f[k, j]
            uy_expected = mom_y / fl["rho"][k]
            uy_expected += 0.5 * fl["fy_node"][k] / fl["rho"][k]
            worst = max(worst, abs(fl["uy"][k] - uy_expected))
    assert worst < 1e-12 * tol, worst


def hot_fluid_pushed_upward(make, tol=1.0):
    """src/uniform/tests.rs:381-401."""
    s = make(16, 40, 1.0e5, 0.71, 0.1, 0.9, 0.02, 42, 1, 1.0, 1.0, None)
    s.step(200)
    uy = s.fields()["uy"]
    nx, ny = s.nx(), s.ny()
    vals = [uy[s.idx(ix, iy)] for iy in range(ny // 2, ny - 2) for ix in range(1, 4)]
    assert np.mean(vals) > 0.0


def isothermal_walls_fixed(make, tol=1.0):
    """src/uniform/tests.rs:406-425 (1e-9)."""
    s = small(make)
    s.step(50)
    t = s.fields()["temperature"]
    nx, ny = s.nx(), s.ny()
    for iy in range(ny):
        assert abs(t[s.idx(0, iy)] - T_HOT) < 1e-9 * tol
        assert abs(t[s.idx(nx - 1, iy)] - T_COLD) < 1e-9 * tol


def adiabatic_walls_zero_gradient(make, tol=1.0):
    """src/uniform/tests.rs:428-452 (1e-9)."""
    s = small(make)
    s.step(50)
    t = s.fields()["temperature"]
    nx, ny = s.nx(), s.ny()
    for ix in range(nx):
        assert abs(t[s.idx(ix, 0)] - t[s.idx(ix, 1)]) < 1e-9 * tol
        assert abs(t[s.idx(ix, ny - 1)] - t[s.idx(ix, ny - 2)]) < 1e-9 * tol


def no_slip_walls(make, tol=1.0):
    """src/uniform/tests.rs:457-476 (1e-12)."""
    s = small(make)
    s.step(50)
    fl = s.fields()
    nx, ny = s.nx(), s.ny()
    for iy in range(ny):
        for ix in (0, nx - 1):
            k = s.idx(ix, iy)
            assert abs(fl["ux"][k]) < 1e-12 and abs(fl["uy"][k]) < 1e-12
    for iy in (0, ny - 1):
        for ix in range(nx):
            k = s.idx(ix, iy)
            assert abs(fl["ux"][k]) < 1e-12 and abs(fl["uy"][k]) < 1e-12


def nusselt_conduction_limit(make, tol=1.0):
    """src/uniform/tests.rs:481-506: linear T gives Nu_hot = Az (height scale)."""
    s = small(make)
    nx, ny = s.nx(), s.ny()
    t = np.empty(nx * ny)
    for iy in range(ny):
        for ix in range(nx):
            xf = ix / (nx - 1)
            t[s.idx(ix, iy)] = T_HOT + (T_COLD - T_HOT) * xf
    s.set_fields(temperature=t)
    nuc = s.diag()["nusselt_hot"]
    az = (ny - 1) / (nx - 1)
    assert abs(nuc - az) < 0.05, nuc


def thermal_wall_link_conductance(make, tol=1.0):
    """src/uniform/tests.rs:602-643: pure diffusion 21x21, nu = 0.00169,
    20 000 steps; first-link / interior jump ratio 0.5 +- 0.05 on both walls."""
    s = make(21, 21, 1.0, 1.0, 0.0, 1.0, 0.02, 42, 1, 1.0, 1.0, 0.00169)
    s.step(20_000)
    t = s.fields()["temperature"]
    nx, ny = s.nx(), s.ny()
    hot1 = hot2 = cold1 = cold2 = 0.0
    cnt = 0
    for iy in range(1, ny - 1):
        t0, t1, t2 = (t[s.idx(i, iy)] for i in (0, 1, 2))
        hot1 += abs(t0 - t1)
        hot2 += abs(t1 - t2)
        tn1, tn2, tn3 = (t[s.idx(nx - i, iy)] for i in (1, 2, 3))
        cold1 += abs(tn1 - tn2)
        cold2 += abs(tn2 - tn3)
        cnt += 1
    r_hot = (hot1 / cnt) / (hot2 / cnt)
    r_cold = (cold1 / cnt) / (cold2 / cnt)
    assert abs(r_hot - 0.5) < 0.05 and abs(r_cold - 0.5) < 0.05, (r_hot, r_cold)


ALL = [
    init_temperature_linear_and_bounded,
    mass_conserved_per_phase,
    guo_forcing_preserves_mass_and_upward_sign,
    hot_fluid_pushed_upward,
    isothermal_walls_fixed,
    adiabatic_walls_zero_gradient,
    no_slip_walls,
    nusselt_conduction_limit,
    thermal_wall_link_conductance,
]
