"""Adjoint of the cavity step (cav_adjoint_run): gradients of the time-averaged
hot-wall Nusselt number w.r.t. the hot-wall theta profile and Cs.

Checks (tolerances stated here):
  * against the FP64 tangent-linear oracle (oracle/tangent.cpp) on a small
    cavity: FP64 adjoint dJ.v within 1e-8 relative, FP32 within 1e-3;
  * against central finite differences (h = 1e-4) of FP64 forward runs on the
    96x384, Ra = 1e7 configuration (J = mean Nu over steps 40 001-60 000,
    checkpoints every 500 steps): FP32 adjoint within 1e-3 relative.
"""
import numpy as np
import pytest

import oracle
from cfd_cavity_b200 import CavitySolver
from cfd_cavity_b200 import _lib as L
from cfd_cavity_b200.batch import Xorshift64Star

pytestmark = pytest.mark.gpu


def profile(ny, seed=7, amp=0.01):
    rng = Xorshift64Star(seed)
    return np.array([0.5 + amp * (2.0 * rng.next_f64() - 1.0) for _ in range(ny)])


SMALL = dict(nx=16, ny=40, ra=1e5, cs=0.1, n=600, ws=301, ck=100)


@pytest.mark.parametrize("precision,tol,n,ck", [
    ("f64", 1e-8, 600, 100),   # odd partial last segment, graph-replayed full segments
    ("f32", 1e-3, 600, 100),
    ("f64", 1e-8, 601, 100),   # no partial segment
    ("f64", 1e-8, 600, 99),    # odd checkpoint interval: direct launches only
])
def test_adjoint_matches_tangent_linear_oracle(precision, tol, n, ck):
    c = dict(SMALL, n=n, ck=ck)
    th = profile(c["ny"])
    s = CavitySolver(c["nx"], c["ny"], c["ra"], 0.71, c["cs"], 0.9, 0.02, 42, precision=precision,
                     t_hot_profile=th)
    J, gth, gcs, info = s.adjoint_nusselt(c["n"], c["ws"], c["ck"])
    assert info["checkpoints"] == -(-(n - 1) // ck)
    assert s.info()["time_step"] == c["n"]
    assert gth[0] == 0.0 and gth[-1] == 0.0
    rng = np.random.default_rng(3)
    for trial in range(3):
        v = rng.standard_normal(c["ny"])
        dcs = float(rng.standard_normal())
        Jo, dJo = oracle.tangent_nusselt(c["nx"], c["ny"], c["ra"], 0.71, c["cs"], 0.9, 0.02, 42,
                                         c["n"], c["ws"], dtheta=v, dcs=dcs, t_hot_profile=th, jobs=4)
        adj = float(np.dot(gth, v) + gcs * dcs)
        assert abs(J - Jo) <= (1e-12 if precision == "f64" else 1e-5) * abs(Jo)
        assert abs(adj - dJo) <= tol * abs(dJo), (trial, adj, dJo)


def test_adjoint_state_checks():
    s = CavitySolver(16, 40, 1e5, 0.71, 0.1, 0.9, 0.02, 42, precision="f32")
    s.step(3)
    with pytest.raises(L.CavError) as e:
        s.adjoint_nusselt(100, 50, 10)
    assert e.value.code == L.CAV_ERR_STATE
    h = CavitySolver(16, 40, 1e5, 0.71, 0.1, 0.9, 0.02, 42, precision="f16sr")
    with pytest.raises(L.CavError) as e:
        h.adjoint_nusselt(100, 50, 10)
    assert e.value.code == L.CAV_ERR_ARG


MID = dict(nx=64, ny=256, ra=1e7, cs=0.1, n=5000, ws=2501, ck=500)


@pytest.mark.parametrize("precision,tol", [("f64", 1e-8), ("f32", 1e-3)])
def test_adjoint_mid_size_matches_tangent_linear_oracle(precision, tol):
    """A mid-size case against the FP64 tangent-linear oracle: 64x256,
    Ra = 1e7, theta = 0 + 1e-4 noise (the benchmark initial field), 5000
    steps, J over steps 2501-5000, checkpoints every 500 (ten segments); a
    random direction in (theta profile, Cs).  FP64 adjoint within 1e-8
    relative, FP32 within 1e-3 (J itself: 1e-12 / 1e-4)."""
    import os

    c = MID
    th = profile(c["ny"], seed=11)
    kw = dict(init_mode=L.CAV_INIT_ZERO, noise_amp=1e-4, t_hot_profile=th)
    s = CavitySolver(c["nx"], c["ny"], c["ra"], 0.71, c["cs"], 0.9, 0.02, 42, precision=precision, **kw)
    J, gth, gcs, info = s.adjoint_nusselt(c["n"], c["ws"], c["ck"])
    assert info["checkpoints"] == -(-(c["n"] - 1) // c["ck"])
    rng = np.random.default_rng(5)
    v = rng.standard_normal(c["ny"])
    dcs = float(rng.standard_normal())
    Jo, dJo = oracle.tangent_nusselt(c["nx"], c["ny"], c["ra"], 0.71, c["cs"], 0.9, 0.02, 42, c["n"], c["ws"],
                                     dtheta=v, dcs=dcs, jobs=max(1, os.cpu_count() or 1), **kw)
    adj = float(np.dot(gth, v) + gcs * dcs)
    # J: FP64 to 1e-12; FP32 arithmetic over 5000 steps at Ra = 1e7 to 1e-4
    assert abs(J - Jo) <= (1e-12 if precision == "f64" else 1e-4) * abs(Jo), (J, Jo)
    assert abs(adj - dJo) <= tol * abs(dJo), (adj, dJo)


C4 = dict(nx=96, ny=384, ra=1e7, cs=0.1, n=60_000, ws=40_001, ck=500)


def test_adjoint_c4_fp32_gradient_matches_fp64_adjoint_in_every_component():
    """The C4 gradient (96x384, Ra = 1e7, 60 000 steps, J over 40 001-60 000,
    checkpoints every 500) of the FP32 adjoint against the FP64 adjoint (the
    one that matches the tangent-linear oracle to 1e-8) in all 385
    components: the 384 hot-wall theta values and Cs.  Tolerances: 1e-3
    relative on the gradient's norm and on dJ/dCs; per theta component
    1e-3 of its own size plus 1e-4 of the gradient's RMS (components that
    are almost zero, the wall rows, are compared on the RMS scale)."""
    c = C4
    th = profile(c["ny"])
    out = {}
    for prec in ("f64", "f32"):
        s = CavitySolver(c["nx"], c["ny"], c["ra"], 0.71, c["cs"], 0.9, 0.02, 42, precision=prec,
                         t_hot_profile=th, init_mode=L.CAV_INIT_ZERO, noise_amp=1e-4)
        out[prec] = s.adjoint_nusselt(c["n"], c["ws"], c["ck"])
        s.close()
    J64, g64, cs64, _ = out["f64"]
    J32, g32, cs32, _ = out["f32"]
    rms = float(np.sqrt(np.mean(g64 ** 2)))
    err = np.abs(g32 - g64)
    print(f"C4 FP32 vs FP64 adjoint: |dg|/|g| {np.linalg.norm(g32 - g64) / np.linalg.norm(g64):.3e}, "
          f"max component error / (|g_i| + 0.1 rms) {np.max(err / (np.abs(g64) + 0.1 * rms)):.3e}, "
          f"dJ/dCs {cs32:.6e} vs {cs64:.6e}")
    assert abs(J32 - J64) <= 1e-4 * abs(J64)
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)
    assert np.all(err <= 1e-3 * np.abs(g64) + 1e-4 * rms), int(np.argmax(err - 1e-3 * np.abs(g64)))
    assert abs(cs32 - cs64) <= 1e-3 * abs(cs64)


def _j_fp64(th, cs):
    c = C4
    s = CavitySolver(c["nx"], c["ny"], c["ra"], 0.71, cs, 0.9, 0.02, 42, precision="f64",
                     t_hot_profile=th, init_mode=L.CAV_INIT_ZERO, noise_amp=1e-4)
    s.step(c["ws"] - 1)
    s.nu_accumulate(True)
    s.step(c["n"] - c["ws"] + 1)
    hot, _, n = s.nu_accumulated()
    assert n == c["n"] - c["ws"] + 1
    return hot


def test_adjoint_c4_against_central_differences():
    """96x384, Ra=1e7, J = mean Nu_hot over steps 40 001-60 000, gradient
    w.r.t. the 384-value hot-wall profile (seeded +-0.01 around 0.5) and Cs;
    FP32 adjoint with checkpoints every 500 steps vs central FD (h = 1e-4) of
    FP64 forward runs."""
    c = C4
    th = profile(c["ny"])
    s = CavitySolver(c["nx"], c["ny"], c["ra"], 0.71, c["cs"], 0.9, 0.02, 42, precision="f32",
                     t_hot_profile=th, init_mode=L.CAV_INIT_ZERO, noise_amp=1e-4)
    J, gth, gcs, info = s.adjoint_nusselt(c["n"], c["ws"], c["ck"])
    ratio = (info["forward_ms"] + info["reverse_ms"]) / info["forward_ms"]
    print(f"C4 adjoint: J={J:.6f} dJ/dCs={gcs:.6e} forward {info['forward_ms']:.1f} ms "
          f"reverse {info['reverse_ms']:.1f} ms ratio {ratio:.2f}")
    h = 1e-4
    fd_cs = (_j_fp64(th, c["cs"] + h) - _j_fp64(th, c["cs"] - h)) / (2 * h)
    print(f"C4 dJ/dCs adjoint {gcs:.6e} FD {fd_cs:.6e}")
    assert abs(gcs - fd_cs) <= 1e-3 * abs(fd_cs)
    for iy in (1, 60, 191, 330, 382):
        tp, tm = th.copy(), th.copy()
        tp[iy] += h
        tm[iy] -= h
        fd = (_j_fp64(tp, c["cs"]) - _j_fp64(tm, c["cs"])) / (2 * h)
        print(f"C4 dJ/dtheta[{iy}] adjoint {gth[iy]:.6e} FD {fd:.6e}")
        assert abs(gth[iy] - fd) <= 1e-3 * abs(fd) + 1e-9
