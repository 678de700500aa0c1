"""The reference's known-answer tests (src/uniform/tests.rs) on the CUDA path,
through the C ABI.  FP64 storage must pass them at the reference's own
tolerances; FP32 at the tolerances of FP32 arithmetic (stated per test)."""
import pytest

from cfd_cavity_b200 import CavitySolver
from tests import kats

pytestmark = pytest.mark.gpu


def maker(precision):
    def make(*args):
        return CavitySolver(*args, precision=precision)
    return make


@pytest.mark.parametrize("kat", kats.ALL, ids=lambda f: f.__name__)
def test_reference_kat_fp64(kat):
    kat(maker("f64"))


# FP32 arithmetic on f_i - w_i: the tolerances of the FP64 tests scale by the
# ratio of the unit roundoffs (2^-24 / 2^-53 ~ 5e8), capped where a test
# compares against a physical bound instead.
FP32_TOL = {
    "mass_conserved_per_phase": 1e4,                     # 1e-8 -> 1e-4 absolute on sum f (640 nodes)
    "guo_forcing_preserves_mass_and_upward_sign": 1e5,   # 1e-9 rel -> 1e-4; 1e-12 abs -> 1e-7
    "isothermal_walls_fixed": 1e3,                       # 1e-9 -> 1e-6
    "adiabatic_walls_zero_gradient": 1e3,
}


@pytest.mark.parametrize("kat", [k for k in kats.ALL if k.__name__ != "no_slip_walls"],
                         ids=lambda f: f.__name__)
def test_reference_kat_fp32(kat):
    kat(maker("f32"), tol=FP32_TOL.get(kat.__name__, 1.0))


def test_no_slip_walls_fp32():
    """No-slip holds exactly in every precision (the wall velocity is set, not computed)."""
    kats.no_slip_walls(maker("f32"))


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_guo_forcing_exact_momentum_poiseuille_on_the_fused_kernel(precision):
    """src/uniform/tests.rs:246-376 on the production kernel: the fused step's
    channel variant (CAV_PHASE_CHANNEL: periodic in y, bounce-back walls at
    x = 0 and nx - 1, TRT Lambda = 3/16 with Guo forcing, body force
    rho * beta_eff along +y) is the reference's 30 x 21 channel turned by 90
    degrees: width H = 21, period 30, nu = 0.01, force 1e-6, 15 000 steps.
    The reference's check: u_max within 10 % of u_steady of the first-mode
    transient u_steady (1 - exp(-N nu pi^2 / H^2)).  Tighter, within 1 % of
    u_steady: the transient with the centre-line mode amplitude 32 / pi^3 and
    the solver's 200-step linear force ramp (a 100-step delay), which the
    reference's own first-mode estimate leaves out (~0.3 %)."""
    import math

    import numpy as np

    from cfd_cavity_b200 import _lib as L

    nx, ny, nu, fx, pr = 21, 30, 0.01, 1.0e-6, 0.71
    lz = ny - 1
    ra = fx * lz ** 3 / (nu * (nu / pr))   # beta_eff = Ra nu alpha_phys / Lz^3 = fx
    s = CavitySolver(nx, ny, ra, pr, 0.0, 0.9, 0.02, 1, 1, 1.0, 1.0, nu, precision=precision)
    info = s.info()
    assert abs(info["beta_eff"] - fx) <= 1e-15 and info["spin_up_steps"] == 200
    n = nx * ny
    s.init_from_fields(np.ones(n), np.zeros(n), np.zeros(n), np.ones(n))
    nsteps = 15_000
    s._ck(L.load().cav_debug_phase(s._h, L.CAV_PHASE_CHANNEL, nsteps))
    u_max = float(np.max(s.fields()["uy"]))
    h = float(nx)
    u_steady = fx * h * h / (8.0 * nu)
    conv = 1.0 - math.exp(-nsteps * nu * math.pi ** 2 / (h * h))
    assert abs(u_max - u_steady * conv) / u_steady < 0.10, (u_max, u_steady * conv)
    conv_c = 1.0 - 32.0 / math.pi ** 3 * math.exp(-(nsteps - 100) * nu * math.pi ** 2 / (h * h))
    assert abs(u_max - u_steady * conv_c) / u_steady < 0.01, (u_max, u_steady * conv_c)
    # the profile across the channel is the symmetric parabola of Poiseuille flow
    uy = s.fields()["uy"].reshape(ny, nx)[ny // 2]
    assert np.allclose(uy, uy[::-1], rtol=0, atol=1e-6 * u_steady)
