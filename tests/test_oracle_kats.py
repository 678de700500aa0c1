"""The reference's own known-answer tests (src/uniform/tests.rs) run against
the FP64 oracle on the CPU.  These pin the oracle before it is trusted as the
checker of the CUDA path."""
import math

import numpy as np
import pytest

import oracle
from tests import kats


def make(*args):
    return oracle.OracleSolver(*args)


@pytest.mark.parametrize("kat", kats.ALL, ids=lambda f: f.__name__)
def test_reference_kat_on_oracle(kat):
    kat(make)


def test_feq_sum_equals_rho():
    """src/uniform/tests.rs:116-120."""
    rho = 1.3
    s = sum(oracle.feq(i, rho, 0.07, -0.03) for i in range(9))
    assert abs(s - rho) < 1e-12


@pytest.mark.parametrize("order", [1, 2])
def test_geq_sum_equals_temperature(order):
    """src/uniform/tests.rs:123-127 (both geq forms; only the sum is pinned)."""
    t = 0.37
    s = sum(oracle.geq(i, t, 0.05, 0.02, order) for i in range(9))
    assert abs(s - t) < 1e-12


def test_weights_sum_to_one():
    """src/uniform/tests.rs:130-133."""
    assert abs(sum(oracle.weights()) - 1.0) < 1e-12


def test_opposites_map_one_to_four_onto_five_to_eight():
    """swap_opposite (src/uniform/solver.rs:938-946) loops i in 1..4 and swaps
    with opp(i); the lattice order has c_{i+4} = -c_i."""
    c = oracle.velocities()
    for i in range(1, 5):
        assert c[i + 4] == (-c[i][0], -c[i][1])
    assert c[0] == (0, 0)


def test_delta_t_is_one():
    """src/uniform/tests.rs:511-514."""
    assert abs(oracle.DELTA_T - 1.0) < 1e-10


def test_feq_matches_poiseuille_restatement():
    """feq of the oracle equals the form the reference restates in its
    Poiseuille test (src/uniform/tests.rs:314-316)."""
    w = oracle.weights()
    c = oracle.velocities()
    rng = np.random.default_rng(3)
    for _ in range(20):
        rho, ux, uy = 1 + 0.1 * rng.standard_normal(), 0.05 * rng.standard_normal(), 0.05 * rng.standard_normal()
        for i in range(9):
            eu = c[i][0] * ux + c[i][1] * uy
            u2 = ux * ux + uy * uy
            cs2 = 1.0 / 3.0
            ref = w[i] * rho * (1.0 + eu / cs2 + eu * eu / (2.0 * cs2 * cs2) - u2 / (2.0 * cs2))
            assert oracle.feq(i, rho, ux, uy) == ref


def test_guo_forcing_exact_momentum_poiseuille():
    """src/uniform/tests.rs:246-376: TRT (Lambda = 3/16) + Guo forcing with the
    per-mode lattice-effect factors, periodic channel 30x21 with mid-link
    bounce-back walls, 15 000 steps, u_max within 10 % of the first-mode
    transient.  The test restates its own collision (the reference test does
    not call the solver); this is that restatement, vectorised."""
    nx, ny = 30, 21
    h = float(ny)
    nu, fx = 0.01, 1.0e-6
    tau_p = 0.5 + 3.0 * nu
    tau_m = 0.5 + (3.0 / 16.0) / (tau_p - 0.5)
    u_steady = fx * h * h / (8.0 * nu)
    a_f = 0.5 * (1.0 / tau_p + 1.0 / tau_m)
    b_f = 0.5 * (1.0 / tau_p - 1.0 / tau_m)
    nsteps = 15_000
    conv = 1.0 - math.exp(-nsteps * nu * math.pi ** 2 / (h * h))
    u_expected = u_steady * conv
    w = np.array(oracle.weights())
    c = np.array(oracle.velocities(), dtype=np.float64)
    opp = np.array([0, 5, 6, 7, 8, 1, 2, 3, 4])
    cs2 = 1.0 / 3.0
    f = np.tile(w, (ny, nx, 1))  # [y, x, i]
    for _ in range(nsteps):
        rho = f.sum(-1)
        ux = (f * c[:, 0]).sum(-1) / rho
        uy = (f * c[:, 1]).sum(-1) / rho
        fn = fx * rho
        u_x = ux + 0.5 * fn / rho
        eu = c[:, 0] * u_x[..., None] + c[:, 1] * uy[..., None]
        u2 = (u_x * u_x + uy * uy)[..., None]
        feq = w * rho[..., None] * (1.0 + eu / cs2 + eu * eu / (2 * cs2 * cs2) - u2 / (2 * cs2))
        d = f - feq
        s_i = w * ((c[:, 0] - u_x[..., None]) / cs2 + eu * c[:, 0] / (cs2 * cs2)) * fn[..., None]
        s_m = w * (c[:, 0] / cs2) * fn[..., None]
        s_p = s_i - s_m
        fp = f + (-a_f * d - b_f * d[..., opp] + (1 - 0.5 / tau_m) * s_m + (1 - 0.5 / tau_p) * s_p)
        new = np.empty_like(fp)
        for i in range(9):
            cx, cy = int(c[i, 0]), int(c[i, 1])
            shifted = np.roll(fp[..., i], cx, axis=1)  # periodic in x
            if cy == 0:
                new[..., i] = shifted
            elif cy == 1:
                new[1:, :, i] = shifted[:-1]
                new[0, :, i] = fp[0, :, opp[i]]
            else:
                new[:-1, :, i] = shifted[1:]
                new[-1, :, i] = fp[-1, :, opp[i]]
        f = new
    rho = f.sum(-1)
    ux = (f * c[:, 0]).sum(-1) / rho + 0.5 * fx
    u_max = ux.max()
    assert abs(u_max - u_expected) / u_steady < 0.10, (u_max, u_expected)


def test_oracle_threads_bitwise_identical():
    """The row-band threading is deterministic (README.md:250-256: --jobs N
    gives results bitwise equal to --jobs 1)."""
    a = oracle.OracleSolver(24, 60, 1e6, 0.71, 0.1, 0.9, 0.02, 7, 1)
    b = oracle.OracleSolver(24, 60, 1e6, 0.71, 0.1, 0.9, 0.02, 7, 4)
    a.step(150)
    b.step(150)
    fa, fb = a.fields(), b.fields()
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), k


def test_oracle_rng_matches_xorshift64star():
    """Initial noise: xorshift64* (src/uniform/rng.rs:5-31), seed|1, U = (x>>11)/2^53,
    pert = 1e-3 (2U - 1) on the linear profile (src/uniform/solver.rs:159-176)."""
    nx, ny, seed = 8, 6, 42
    s = oracle.OracleSolver(nx, ny, 1e5, 0.71, 0.1, 0.9, 0.02, seed, 1)
    t = s.fields()["temperature"]
    state = seed | 1
    mask = (1 << 64) - 1
    for iy in range(ny):
        for ix in range(nx):
            x = state
            x ^= x >> 12
            x ^= (x << 25) & mask
            x ^= x >> 27
            state = x
            u = ((x * 0x2545F4914F6CDD1D) & mask) >> 11
            uf = u / float(1 << 53)
            exp = 0.5 + (-0.5 - 0.5) * (ix / (nx - 1)) + 1.0e-3 * (2.0 * uf - 1.0)
            assert t[iy * nx + ix] == exp


def test_lattice_units_of_new():
    """CavitySolver::new calibration (src/uniform/solver.rs:123-154): the
    64x256 Ra=1e6 run the reference validated has nu ~ 0.0186."""
    s = oracle.OracleSolver(64, 256, 1e6, 0.71, 0.1, 0.9, 0.02, 42, 1)
    i = s.info()
    assert abs(i["nu"] - 0.0186) < 5e-4
    assert i["tau"] == 0.5 + 3.0 * i["nu"]
    assert i["spin_up_steps"] == 200
    assert abs(i["beta_eff"] - 1e6 * i["nu"] * i["alpha_phys"] / 255.0 ** 3) < 1e-18


def test_tau_assertion_is_an_error():
    """solver.rs:152-154: tau too close to 1/2 is refused."""
    with pytest.raises(oracle.OracleError):
        oracle.OracleSolver(16, 40, 1e5, 0.71, 0.1, 0.9, 0.02, 42, 1, 1.0, 1.0, 1e-5)
