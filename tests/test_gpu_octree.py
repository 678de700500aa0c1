"""The block-refined (octree) cavity on the GPU (cav_octree_*).

  * FP64 storage: every level's populations and moments bit-identical to the
    FP64 oracle (a restatement of src/octree/) after whole coarse steps, for
    2 and 3 levels, with and without the viscosity ramp and odd_exact;
  * the reference's own octree tests (src/octree/tests.rs) on the GPU path;
  * the interface couplings alone (coarse_to_fine / fine_to_coarse) against
    the moment identities of src/octree/tests.rs:136-320, restated on the
    cavity's block layout;
  * FP32 and FP32-arithmetic / binary16-storage against FP64, tolerances
    stated in each test.
"""
import numpy as np
import pytest

import oracle
from cfd_cavity_b200 import _lib as L
from cfd_cavity_b200.octree import OctreeSolver

pytestmark = pytest.mark.gpu

CX = np.array([0, 1, 0, 1, -1, -1, 0, -1, 1], dtype=float)
CY = np.array([0, 0, 1, 1, 1, 0, -1, -1, -1], dtype=float)
W = np.array([4 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 9, 1 / 9, 1 / 36, 1 / 36])
OPP = [0, 5, 6, 7, 8, 1, 2, 3, 4]


def n_levels(levels):
    return 3 if levels == 2 else 5


def assert_levels_equal(gpu, orc, levels):
    for lvl in range(n_levels(levels)):
        g = gpu.level(lvl, pops=True)
        o = orc.level(lvl, pops=True)
        assert (g["nx"], g["ny"]) == (o["nx"], o["ny"])
        for k in ("rho", "ux", "uy", "temp", "f", "g"):
            np.testing.assert_array_equal(g[k], o[k], err_msg=f"level {lvl} {k}")


@pytest.mark.parametrize("levels", [2, 3])
def test_fp64_bit_identical_to_oracle(levels):
    args = (32, 64, 4, 1.0e6, 0.71, 0.02, 42)
    gpu = OctreeSolver(*args, levels=levels, precision="f64")
    orc = oracle.OracleOctree(*args, levels=levels)
    assert_levels_equal(gpu, orc, levels)           # init_cavity
    gpu.step_cavity(1)
    orc.step_cavity(1)
    assert_levels_equal(gpu, orc, levels)
    gpu.step_cavity(40)                               # graph replays + single steps
    orc.step_cavity(40)
    assert_levels_equal(gpu, orc, levels)
    dg, do = gpu.diag(), orc.diag()
    for k in ("nu_hot", "nu_hot_link0", "nu_cold", "nu_hot_fine", "max_u"):
        assert dg[k] == do[k], k
    # mean rho: FP64 sums in another order (last-bit differences)
    for k in ("mass", "max_rho_dev", "max_rho_dev_ifaces"):
        assert abs(dg[k] - do[k]) <= 1e-14, k
    assert dg["finite"] == 1.0


@pytest.mark.parametrize("levels,odd_exact,nu_start_mult", [(3, True, 1.0), (3, False, 4.0), (2, True, 2.5)])
def test_fp64_bit_identical_variants(levels, odd_exact, nu_start_mult):
    args = (48, 96, 6, 1.0e7, 0.71, 0.03, 7)
    gpu = OctreeSolver(*args, odd_exact=odd_exact, levels=levels, nu_start_mult=nu_start_mult, precision="f64")
    orc = oracle.OracleOctree(*args, odd_exact=odd_exact, levels=levels, nu_start_mult=nu_start_mult)
    gpu.step_cavity(37)
    orc.step_cavity(37)
    assert_levels_equal(gpu, orc, levels)
    assert gpu.time_step == 37


def test_fp64_restart_bit_identical_to_oracle():
    """set_from_snapshot (src/octree/solver.rs:1080-1168): a Ra = 1e7 octree
    restarted from the fields of a Ra = 1e6 run of the same layout, then
    stepped; every level bit-identical to the oracle doing the same."""
    a_args = (32, 64, 4, 1.0e6, 0.71, 0.02, 42)
    b_args = (32, 64, 4, 1.0e7, 0.71, 0.02, 9)
    ga = OctreeSolver(*a_args, levels=3, precision="f64")
    oa = oracle.OracleOctree(*a_args, levels=3)
    ga.step_cavity(30)
    oa.step_cavity(30)
    gb = OctreeSolver(*b_args, levels=3, precision="f64")
    ob = oracle.OracleOctree(*b_args, levels=3)
    gb.step_cavity(5)
    ob.step_cavity(5)
    gb.restart_from(ga)
    ob.restart_from(oa)
    assert gb.time_step == 0
    assert_levels_equal(gb, ob, 3)
    gb.step_cavity(20)
    ob.step_cavity(20)
    assert_levels_equal(gb, ob, 3)


def test_reference_octree_kats_on_gpu():
    """src/octree/tests.rs:397-580 on the GPU path (FP64 and FP32)."""
    for prec in ("f64", "f32", "f32_f16"):
        sim = OctreeSolver(32, 64, 4, 1.0e6, 0.71, 0.02, 42, levels=2, precision=prec)
        d0 = sim.diag()
        assert abs(d0["nu_hot"] - 1.0) < 0.05 and abs(d0["nu_cold"] - 1.0) < 0.05
        for step in range(20):
            sim.step_cavity()
            d = sim.diag()
            if step < 10:
                assert abs(d["mass"] - 1.0) < 1e-6, (prec, step, d["mass"])
            assert d["max_rho_dev"] >= d["max_rho_dev_ifaces"]
            if step >= 5:
                assert d["max_rho_dev_ifaces"] < 1.0
        s3 = OctreeSolver(32, 64, 4, 1.0e6, 0.71, 0.02, 42, levels=3, precision=prec)
        i = s3.info()
        assert i["nx"][3] == 7 and i["nx"][4] == 7
        nu0 = i["nu"]
        tp2 = 0.5 + 3.0 * (4.0 * nu0)
        assert abs(i["tau_plus"][2] - tp2) < 1e-15
        assert abs(i["xi_even_sub"] - 0.5 * tp2 / i["tau_plus"][1]) < 1e-15
        for _ in range(10):
            s3.step_cavity()
            d = s3.diag()
            assert abs(d["mass"] - 1.0) < 1e-6
            assert d["max_rho_dev_ifaces"] < 1.0 and d["max_rho_dev"] >= d["max_rho_dev_ifaces"]
            assert s3.check_guards() == 0


def feq(rho, ux, uy):
    eu = CX[None, :] * ux[:, None] + CY[None, :] * uy[:, None]
    u2 = (ux * ux + uy * uy)[:, None]
    return W[None, :] * rho[:, None] * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * u2)


def bilinear(x, y, nx0, ny0):
    ix = int(min(max(np.floor(x), 0), nx0 - 2))
    iy = int(min(max(np.floor(y), 0), ny0 - 2))
    fx, fy = x - ix, y - iy
    return [(iy * nx0 + ix, (1 - fx) * (1 - fy)), (iy * nx0 + ix + 1, fx * (1 - fy)),
            ((iy + 1) * nx0 + ix, (1 - fx) * fy), ((iy + 1) * nx0 + ix + 1, fx * fy)]


def test_coarse_to_fine_conserves_moments():
    """src/octree/tests.rs:136-214 on the cavity blocks: every injected ghost
    carries the bilinear rho and T of the coarse grid to 1e-12 and the
    momentum rho u + xi_odd * (interpolated f^neq momentum)."""
    nx0, ny0, blw = 32, 64, 4
    sim = OctreeSolver(nx0, ny0, blw, 1.0e6, 0.71, 0.02, 42, levels=2, precision="f64")
    n = nx0 * ny0
    iy, ix = np.divmod(np.arange(n), nx0)
    uy = 0.01 * (ix - nx0 / 2) / (nx0 / 2)
    temp = 0.5 + 0.01 * (iy - ny0 / 2) / (ny0 / 2)
    rho = 1.0 + 1e-3 * np.sin(2 * np.pi * iy / ny0)
    f = feq(rho, np.zeros(n), uy) + 1e-4 * W[None, :] * CY[None, :]
    g = feq(temp, np.zeros(n), uy) + 1e-5 * W[None, :] * CX[None, :]
    rho_m, ux_m, uy_m, t_m = f.sum(1), (f * CX).sum(1) / f.sum(1), (f * CY).sum(1) / f.sum(1), g.sum(1)
    sim.set_level(0, rho_m, ux_m, uy_m, t_m, f, g)
    sim.couple(0)
    xi_odd = sim.info()["xi_odd"]
    fneq = f - feq(rho_m, ux_m, uy_m)
    for lvl, bx0 in ((1, 0), (2, nx0 - 1 - blw)):
        lv = sim.level(lvl, pops=True)
        nx1, ny1 = lv["nx"], lv["ny"]
        worst = 0.0
        for b in range(ny1):
            for a in range(nx1):
                if not (a == 0 or b == 0 or a == nx1 - 1 or b == ny1 - 1):
                    continue
                k = b * nx1 + a
                st = bilinear(bx0 - 0.5 + 0.5 * a, -0.5 + 0.5 * b, nx0, ny0)
                e_rho = sum(w * rho_m[kc] for kc, w in st)
                e_t = sum(w * t_m[kc] for kc, w in st)
                e_mx = sum(w * rho_m[kc] for kc, w in st) * sum(w * ux_m[kc] for kc, w in st) \
                    + xi_odd * sum(w * (fneq[kc] * CX).sum() for kc, w in st)
                e_my = sum(w * rho_m[kc] for kc, w in st) * sum(w * uy_m[kc] for kc, w in st) \
                    + xi_odd * sum(w * (fneq[kc] * CY).sum() for kc, w in st)
                fk, gk = lv["f"][k], lv["g"][k]
                worst = max(worst, abs(fk.sum() - e_rho), abs(gk.sum() - e_t),
                            abs((fk * CX).sum() - e_mx), abs((fk * CY).sum() - e_my))
                assert lv["rho"][k] == pytest.approx(fk.sum(), abs=1e-14)
        assert worst < 1e-12, worst


def test_fine_to_coarse_conserves_moments():
    """src/octree/tests.rs:216-320 on the cavity blocks: each coincident
    coarse node gets the 9-point weighted rho and T and the momentum
    rho u + (weighted f^neq momentum) / xi_odd, to 1e-12."""
    nx0, ny0, blw = 32, 64, 4
    sim = OctreeSolver(nx0, ny0, blw, 1.0e6, 0.71, 0.02, 42, levels=2, precision="f64")
    xi_odd = sim.info()["xi_odd"]
    for lvl, bx0 in ((1, 0), (2, nx0 - 1 - blw)):
        lv = sim.level(lvl)
        nx1, ny1 = lv["nx"], lv["ny"]
        n = nx1 * ny1
        b, a = np.divmod(np.arange(n), nx1)
        x = bx0 - 0.5 + 0.5 * a
        y = -0.5 + 0.5 * b
        uy = 0.02 * (x - nx0 / 2) / (nx0 / 2)
        temp = 0.5 + 0.01 * (y - ny0 / 2) / (ny0 / 2)
        rho = 1.0 + 1e-3 * np.sin(2 * np.pi * y / ny1)
        fneq0 = 2e-4 * W * CX * CY + 5e-4 * W * CX
        f = feq(rho, np.zeros(n), uy) + fneq0[None, :]
        g = feq(temp, np.zeros(n), uy) + (1e-5 * W * CY)[None, :]
        sim.set_level(lvl, rho, np.zeros(n), uy, temp, f, g)
    sim.couple(1)
    c = sim.level(0, pops=True)
    worst = 0.0
    checked = 0
    for lvl, bx0 in ((1, 0), (2, nx0 - 1 - blw)):
        lv = sim.level(lvl, pops=True)
        nx1 = lv["nx"]
        for cy in range(1, ny0 - 1):
            for cx in range(bx0, bx0 + blw):
                if cx == 0 or cx + 1 == nx0:
                    continue
                a, b = 2 * (cx - bx0) + 1, 2 * cy + 1
                ww = [0.25, 0.5, 0.25]
                e_rho = e_t = e_mx = e_my = fmx = fmy = 0.0
                for jb in range(3):
                    for ja in range(3):
                        kf = (b + jb - 1) * nx1 + (a + ja - 1)
                        w = ww[ja] * ww[jb]
                        r, u, v = lv["rho"][kf], lv["ux"][kf], lv["uy"][kf]
                        e_rho += w * r
                        e_t += w * lv["temp"][kf]
                        e_mx += w * r * u
                        e_my += w * r * v
                        fn = lv["f"][kf] - feq(np.array([r]), np.array([u]), np.array([v]))[0]
                        fmx += w * (fn * CX).sum()
                        fmy += w * (fn * CY).sum()
                kc = cy * nx0 + cx
                fk, gk = c["f"][kc], c["g"][kc]
                worst = max(worst, abs(fk.sum() - e_rho), abs(gk.sum() - e_t),
                            abs((fk * CX).sum() - (e_mx + fmx / xi_odd)),
                            abs((fk * CY).sum() - (e_my + fmy / xi_odd)))
                checked += 1
    assert checked == (blw - 1 + blw) * (ny0 - 2)
    assert worst < 1e-12, worst


@pytest.mark.parametrize("prec", ["f32", "f32_f16", "f32_f16g"])
@pytest.mark.parametrize("levels", [2, 3])
def test_fg_level_kernel_bit_identical(prec, levels):
    """The fine levels' step with a node's f and g halves on two threads
    (the default) and with one thread per node give the same state bit for
    bit: every level's populations and moments after 37 coarse steps (graph
    replays and single steps) across the viscosity ramp, with a switch of
    form half way (binary16 pairs rounded by one cvt.rs against each half
    rounded alone, the fixed-point g planes, FP32)."""
    args = (48, 96, 6, 1.0e7, 0.71, 0.03, 7)
    a = OctreeSolver(*args, levels=levels, precision=prec, nu_start_mult=2.5)
    b = OctreeSolver(*args, levels=levels, precision=prec, nu_start_mult=2.5)
    assert a.level_kernel() == L.CAV_OCT_LEVEL_FG
    b.set_level_kernel(L.CAV_OCT_LEVEL_NODE)
    assert b.level_kernel() == L.CAV_OCT_LEVEL_NODE
    a.step_cavity(20)
    b.step_cavity(20)
    b.set_level_kernel(L.CAV_OCT_LEVEL_FG)
    a.set_level_kernel(L.CAV_OCT_LEVEL_NODE)
    a.step_cavity(17)
    b.step_cavity(17)
    for lvl in range(n_levels(levels)):
        ga, gb = a.level(lvl, pops=True), b.level(lvl, pops=True)
        for k in ("rho", "ux", "uy", "temp", "f", "g"):
            np.testing.assert_array_equal(ga[k], gb[k], err_msg=f"level {lvl} {k}")
    assert a.diag() == b.diag()
    with pytest.raises(L.CavError) as e:
        a.set_level_kernel(5)
    assert e.value.code == L.CAV_ERR_ARG


@pytest.mark.parametrize("prec,tol_t,tol_nu", [("f32", 1e-4, 5e-4), ("f32_f16", 3e-3, 2e-3),
                                                ("f32_f16g", 5e-4, 1e-3)])
def test_reduced_precision_against_fp64(prec, tol_t, tol_nu):
    """64 x 256 base, bl_width 8, 3 levels, Ra = 1e7, 2000 coarse steps (the
    start-up plume is still growing, so rounding differences grow too):
    max |T - T_64| over every level <= tol_t (temperatures are O(0.5)) and
    |Nu - Nu_64| / Nu_64 <= tol_nu for the coarse and fine estimators.
    Measured on a B200: f32 2.8e-5 / 1.4e-4, f32_f16 6.8e-4 / 3.2e-4,
    f32_f16g 1.3e-4 / 1.3e-4."""
    args = (64, 256, 8, 1.0e7, 0.71, 0.02, 42)
    ref = OctreeSolver(*args, levels=3, precision="f64")
    red = OctreeSolver(*args, levels=3, precision=prec)
    ref.step_cavity(2000)
    red.step_cavity(2000)
    for lvl in range(5):
        a, b = ref.level(lvl), red.level(lvl)
        assert np.max(np.abs(a["temp"] - b["temp"])) <= tol_t, lvl
    dr, dd = ref.diag(), red.diag()
    for k in ("nu_hot", "nu_cold", "nu_hot_fine"):
        assert abs(dd[k] - dr[k]) <= tol_nu * abs(dr[k]), (k, dd[k], dr[k])
    assert abs(dd["mass"] - dr["mass"]) < 1e-5
    assert dd["finite"] == 1.0


def test_argument_checks():
    with pytest.raises(L.CavError) as e:
        OctreeSolver(32, 64, 1, 1e6, 0.71, 0.02, 42)
    assert e.value.code == L.CAV_ERR_ARG
    with pytest.raises(L.CavError):
        OctreeSolver(32, 64, 16, 1e6, 0.71, 0.02, 42)
    with pytest.raises(L.CavError):
        OctreeSolver(32, 64, 4, 1e6, 0.71, 0.02, 42, levels=4)
    s = OctreeSolver(32, 64, 4, 1e6, 0.71, 0.02, 42, levels=2)
    with pytest.raises(L.CavError):
        s.level(3)
    with pytest.raises(L.CavError):
        s.couple(2)
