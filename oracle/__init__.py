"""The oracle -- TEST INFRASTRUCTURE ONLY.

ctypes front end of the CPU FP64 restatement of the reference solver
(bbrangeo/cfd_cavity ``src/uniform/solver.rs``, ``post.rs``, ``rng.rs``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline use it, as the checker; the product library never does.

``OracleSolver`` mirrors the reference type ``uniform::solver::CavitySolver``
(``src/uniform/solver.rs:35-104``): same constructor arguments, ``step``,
``init_from_fields``, the ``pub(crate)`` phases the reference tests call
(``collide``, ``stream``, ``apply_bounce_back``,
``apply_thermal_boundary_conditions``, ``update_macroscopic``) and the
fields the reference callers read.  Parity status: see
``oracle/cavity_oracle.hpp``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcavity_oracle.so")
_lib = None

T_HOT = 0.5
T_COLD = -0.5
DELTA_T = 1.0
INIT_LINEAR = 0
INIT_ZERO = 1


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("ra", ctypes.c_double), ("pr", ctypes.c_double), ("cs", ctypes.c_double),
        ("pr_t", ctypes.c_double), ("utarget", ctypes.c_double),
        ("seed", ctypes.c_uint64), ("jobs", ctypes.c_int32),
        ("alpha_mult", ctypes.c_double), ("nu_start_mult", ctypes.c_double),
        ("has_nu_override", ctypes.c_int32), ("nu_override", ctypes.c_double),
        ("init_mode", ctypes.c_int32), ("noise_amp", ctypes.c_double),
        ("geq_order", ctypes.c_int32),
        ("t_hot_profile", ctypes.POINTER(ctypes.c_double)),
        ("t_cold", ctypes.c_double),
    ]


def build() -> str:
    """Compiles the oracle library with its Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, dp, i64 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.POINTER(ctypes.c_int32)]
        for name in ("orc_destroy", "orc_stream", "orc_bounce_back", "orc_thermal_bc",
                     "orc_macro", "orc_noslip"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = None
        L.orc_step.argtypes = [vp, i64]
        L.orc_collide.argtypes = [vp, i64]
        L.orc_set_time_step.argtypes = [vp, i64]
        L.orc_init_from_fields.argtypes = [vp, dp, dp, dp, dp]
        L.orc_get_fields.argtypes = [vp, dp, dp, dp, dp, dp, dp]
        L.orc_set_fields.argtypes = [vp, dp, dp, dp, dp, dp]
        L.orc_get_pops.argtypes = [vp, dp, dp]
        L.orc_set_pops.argtypes = [vp, dp, dp]
        L.orc_info.argtypes = [vp, dp]
        L.orc_diag.argtypes = [vp, dp]
        L.orc_feq.restype = ctypes.c_double
        L.orc_feq.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_geq.restype = ctypes.c_double
        L.orc_geq.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                              ctypes.c_int32]
        L.orc_weight.restype = ctypes.c_double
        L.orc_weight.argtypes = [ctypes.c_int32]
        L.orc_velocity.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_int32)]
        L.orc_nusselt.argtypes = [vp, dp, dp]
        L.orc_tl_nusselt.restype = ctypes.c_int
        L.orc_tl_nusselt.argtypes = [ctypes.POINTER(OrcParams), i64, i64, dp, ctypes.c_double, dp, dp]
        L.orc_avg_create.restype = vp
        L.orc_avg_create.argtypes = [i64]
        L.orc_avg_destroy.argtypes = [vp]
        L.orc_avg_accumulate.argtypes = [vp, vp]
        L.orc_avg_means.restype = i64
        L.orc_avg_means.argtypes = [vp, dp, dp, dp, dp, dp]
        L.orc_nusselt_from_mean.restype = ctypes.c_double
        L.orc_nusselt_from_mean.argtypes = [vp, dp, ctypes.c_int32]
        L.orc_set_dynamic_sgs.argtypes = [vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double]
        L.orc_compute_dynamic_sgs.argtypes = [vp]
        L.orc_dynamic_stats.argtypes = [vp, dp, dp, dp]
        L.orc_lilly_coefficient.restype = ctypes.c_double
        L.orc_lilly_coefficient.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_interpolate_field.argtypes = [dp, i64, i64, i64, i64, dp]
        L.orc_mixed_factor.restype = ctypes.c_double
        L.orc_mixed_factor.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        i32, d = ctypes.c_int32, ctypes.c_double
        L.orc_oct_create.restype = vp
        L.orc_oct_create.argtypes = [i32, i32, i32, d, d, d, ctypes.c_uint64, i32, i32, d, i32, d,
                                     ctypes.POINTER(i32)]
        L.orc_oct_destroy.argtypes = [vp]
        L.orc_oct_step.argtypes = [vp, i64]
        L.orc_oct_level_dims.restype = i32
        L.orc_oct_level_dims.argtypes = [vp, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]
        L.orc_oct_get_level.restype = i32
        L.orc_oct_get_level.argtypes = [vp, i32, dp, dp, dp, dp, dp, dp]
        L.orc_oct_info.argtypes = [vp, dp]
        L.orc_oct_diag.argtypes = [vp, dp]
        L.orc_oct_restart_level.restype = i32
        L.orc_oct_restart_level.argtypes = [vp, i32, dp, dp, dp, dp]
        L.orc_oct_set_time_step.argtypes = [vp, i64]
        L.orc_oct_set_dynamic_sgs.argtypes = [vp, i32, d, d, d]
        L.orc_oct_dynamic_stats.argtypes = [vp, dp]
        L.orc_oct_get_nut.restype = i32
        L.orc_oct_get_nut.argtypes = [vp, i32, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def lilly_coefficient(num, den):
    return lib().orc_lilly_coefficient(num, den)


def mixed_factor(a, b, alpha):
    return lib().orc_mixed_factor(a, b, alpha)


def interpolate_field(src, nx0, ny0, nx1, ny1):
    """interpolate_field (src/uniform/snapshot.rs:102-131)."""
    s = np.ascontiguousarray(src, dtype=np.float64).reshape(nx0 * ny0)
    d = np.empty(nx1 * ny1)
    lib().orc_interpolate_field(_dp(s), nx0, ny0, nx1, ny1, _dp(d))
    return d


def feq(i, rho, ux, uy):
    return lib().orc_feq(i, rho, ux, uy)


def geq(i, t, ux, uy, order=2):
    return lib().orc_geq(i, t, ux, uy, order)


def weights():
    return [lib().orc_weight(i) for i in range(9)]


def velocities():
    out = []
    for i in range(9):
        cx, cy = ctypes.c_int32(), ctypes.c_int32()
        lib().orc_velocity(i, ctypes.byref(cx), ctypes.byref(cy))
        out.append((cx.value, cy.value))
    return out


class OracleError(RuntimeError):
    pass


def tangent_nusselt(nx, ny, ra, pr, cs, pr_t, utarget, seed, n_steps, ws, dtheta=None, dcs=0.0,
                    *, jobs=1, nu_override=None, init_mode=INIT_LINEAR, noise_amp=1.0e-3,
                    geq_order=2, t_hot_profile=None, t_cold=T_COLD):
    """FP64 tangent-linear oracle: (J, dJ . v) with J the mean hot-wall Nusselt
    number over the states after s steps, s in [ws, n_steps], and
    v = (dtheta, dcs) a direction in (hot-wall theta profile, Cs)."""
    p = OrcParams()
    p.nx, p.ny, p.ra, p.pr, p.cs, p.pr_t, p.utarget = nx, ny, ra, pr, cs, pr_t, utarget
    p.seed, p.jobs, p.alpha_mult, p.nu_start_mult = seed, jobs, 1.0, 1.0
    p.has_nu_override = 0 if nu_override is None else 1
    p.nu_override = 0.0 if nu_override is None else nu_override
    p.init_mode, p.noise_amp, p.geq_order, p.t_cold = init_mode, noise_amp, geq_order, t_cold
    th = None
    if t_hot_profile is not None:
        th = np.ascontiguousarray(t_hot_profile, dtype=np.float64)
        p.t_hot_profile = _dp(th)
    dth = None if dtheta is None else np.ascontiguousarray(dtheta, dtype=np.float64)
    J, dJ = ctypes.c_double(), ctypes.c_double()
    rc = lib().orc_tl_nusselt(ctypes.byref(p), n_steps, ws, _dp(dth), dcs, ctypes.byref(J), ctypes.byref(dJ))
    if rc != 0:
        raise OracleError(f"orc_tl_nusselt failed with code {rc}")
    return J.value, dJ.value


class OracleSolver:
    """CPU FP64 restatement of ``CavitySolver`` (src/uniform/solver.rs:106-210).

    Positional arguments follow ``CavitySolver::new(nx, ny, ra, pr, cs, pr_t,
    utarget, seed, jobs, alpha_mult, nu_start_mult, nu_override)``; the
    keyword-only ones select the benchmark initial field and the unpinned
    ``geq`` form.
    """

    def __init__(self, nx, ny, ra, pr, cs, pr_t, utarget, seed, jobs=1, alpha_mult=1.0,
                 nu_start_mult=1.0, nu_override=None, *, init_mode=INIT_LINEAR,
                 noise_amp=1.0e-3, geq_order=2, t_hot_profile=None, t_cold=T_COLD):
        L = lib()
        p = OrcParams()
        p.nx, p.ny, p.ra, p.pr, p.cs, p.pr_t, p.utarget = nx, ny, ra, pr, cs, pr_t, utarget
        p.seed, p.jobs, p.alpha_mult, p.nu_start_mult = seed, jobs, alpha_mult, nu_start_mult
        p.has_nu_override = 0 if nu_override is None else 1
        p.nu_override = 0.0 if nu_override is None else nu_override
        p.init_mode, p.noise_amp, p.geq_order = init_mode, noise_amp, geq_order
        self._t_hot = None
        if t_hot_profile is not None:
            self._t_hot = np.ascontiguousarray(t_hot_profile, dtype=np.float64)
            assert self._t_hot.shape == (ny,)
            p.t_hot_profile = _dp(self._t_hot)
        p.t_cold = t_cold
        err = ctypes.c_int32(0)
        self._h = L.orc_create(ctypes.byref(p), ctypes.byref(err))
        if not self._h:
            raise OracleError(f"orc_create failed with code {err.value}")
        self._nx, self._ny = nx, ny

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    # -- API of CavitySolver -------------------------------------------------
    def nx(self):
        return self._nx

    def ny(self):
        return self._ny

    def idx(self, ix, iy):
        return iy * self._nx + ix

    def step(self, n: int = 1):
        lib().orc_step(self._h, n)

    def collide(self, step):
        lib().orc_collide(self._h, step)

    def stream(self):
        lib().orc_stream(self._h)

    def apply_bounce_back(self):
        lib().orc_bounce_back(self._h)

    def apply_thermal_boundary_conditions(self):
        lib().orc_thermal_bc(self._h)

    def update_macroscopic(self):
        lib().orc_macro(self._h)

    def enforce_wall_velocity(self):
        lib().orc_noslip(self._h)

    def init_from_fields(self, rho, ux, uy, t):
        n = self._nx * self._ny
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(n) for a in (rho, ux, uy, t)]
        lib().orc_init_from_fields(self._h, *[_dp(a) for a in arrs])

    def fields(self):
        n = self._nx * self._ny
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "temperature", "nu_t", "fy_node")}
        lib().orc_get_fields(self._h, *[_dp(out[k]) for k in
                                         ("rho", "ux", "uy", "temperature", "nu_t", "fy_node")])
        return out

    def set_fields(self, rho=None, ux=None, uy=None, temperature=None, fy_node=None):
        n = self._nx * self._ny
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(n)
                for a in (rho, ux, uy, temperature, fy_node)]
        lib().orc_set_fields(self._h, *[_dp(a) for a in arrs])

    def populations(self):
        n = self._nx * self._ny
        f = np.empty((n, 9))
        g = np.empty((n, 9))
        lib().orc_get_pops(self._h, _dp(f), _dp(g))
        return f, g

    def set_populations(self, f=None, g=None):
        n = self._nx * self._ny
        fa = None if f is None else np.ascontiguousarray(f, dtype=np.float64).reshape(n, 9)
        ga = None if g is None else np.ascontiguousarray(g, dtype=np.float64).reshape(n, 9)
        lib().orc_set_pops(self._h, _dp(fa), _dp(ga))

    def set_time_step(self, t):
        lib().orc_set_time_step(self._h, t)

    def info(self):
        out = np.empty(10)
        lib().orc_info(self._h, _dp(out))
        keys = ("nu", "alpha", "alpha_phys", "beta_eff", "lz", "lx", "tau", "tau_t",
                "time_step", "spin_up_steps")
        return dict(zip(keys, out.tolist()))

    def diag(self):
        out = np.empty(11)
        lib().orc_diag(self._h, _dp(out))
        keys = ("nusselt_hot", "nusselt_cold", "nusselt_hot_wall_link", "total_mass",
                "total_f_mass", "max_u", "max_uy", "nu_t_max", "finite", "y_plus_hot",
                "nusselt_volume")
        return dict(zip(keys, out.tolist()))

    # convenience accessors named like the reference's pub fields / fns
    @property
    def temperature(self):
        return self.fields()["temperature"]

    def total_mass(self):
        return self.diag()["total_mass"]

    def total_f_mass(self):
        return self.diag()["total_f_mass"]

    def nusselt(self):
        hot, cold = ctypes.c_double(), ctypes.c_double()
        lib().orc_nusselt(self._h, ctypes.byref(hot), ctypes.byref(cold))
        return hot.value, cold.value

    def nusselt_hot(self):
        return self.nusselt()[0]

    def nusselt_cold(self):
        return self.nusselt()[1]

    def set_dynamic_sgs(self, on, smag_alpha=0.5, nu_sm_min=-0.1, eta_test=2.0):
        """set_dynamic_sgs (src/uniform/solver.rs:215-220)."""
        lib().orc_set_dynamic_sgs(self._h, int(bool(on)), smag_alpha, nu_sm_min, eta_test)

    def compute_dynamic_sgs(self):
        lib().orc_compute_dynamic_sgs(self._h)

    def dynamic_stats(self):
        """(cs_dyn_mean, cs_dyn_max, kappa_dyn_mean, kappa_dyn_max, nu_t_pre, alpha_t_pre)."""
        n = self._nx * self._ny
        o, a, b = np.empty(4), np.empty(n), np.empty(n)
        a[:] = np.nan
        b[:] = np.nan
        lib().orc_dynamic_stats(self._h, _dp(o), _dp(a), _dp(b))
        return (*o.tolist(), a, b)

    def nusselt_from_mean(self, t_mean, hot=True):
        t = np.ascontiguousarray(t_mean, dtype=np.float64)
        return lib().orc_nusselt_from_mean(self._h, _dp(t), 1 if hot else 0)


class OracleAverager:
    """TimeAverager, src/uniform/post.rs:11-57."""

    def __init__(self, n):
        self._n = n
        self._a = lib().orc_avg_create(n)

    def __del__(self):
        a = getattr(self, "_a", None)
        if a:
            lib().orc_avg_destroy(a)
            self._a = None

    def accumulate(self, s: OracleSolver):
        lib().orc_avg_accumulate(self._a, s._h)

    def means(self):
        out = [np.empty(self._n) for _ in range(5)]
        cnt = lib().orc_avg_means(self._a, *[_dp(a) for a in out])
        return cnt, out


OCT_INFO_KEYS = ("nu", "alpha", "beta_eff_coarse", "tau_plus_l0", "tau_plus_l1", "tau_plus_l2",
                 "xi_even", "xi_odd", "xi_thermal", "xi_even_sub", "time_step", "n_coincident",
                 "n_ghosts")
OCT_DIAG_KEYS = ("nu_hot", "nu_hot_link0", "nu_cold", "nu_hot_fine", "max_u", "mass",
                 "max_rho_dev", "max_rho_dev_ifaces", "finite")
OCT_DYN_KEYS = ("cs_dyn_mean", "cs_dyn_max", "kappa_dyn_mean", "kappa_dyn_max", "nu_t_max",
                "xi_even", "xi_odd", "xi_th", "xi_b_hot_even", "xi_b_hot_odd", "xi_b_hot_th",
                "xi_b_cold_even", "xi_b_cold_odd", "xi_b_cold_th")


class OracleOctree:
    """CPU FP64 restatement of the block-refined ``octree::solver::CavitySolver``
    (src/octree/solver.rs:284-947): ``CavitySolver::new(nx0, ny0, bl_width,
    ra, pr, utarget, seed, jobs, odd_exact, levels, nu_start_mult,
    nu_override)`` and ``step_cavity``.  Levels: 0 coarse, 1/2 the hot/cold
    L1 blocks, 3/4 the hot/cold L2 strips (levels = 3)."""

    def __init__(self, nx0, ny0, bl_width, ra, pr, utarget, seed, jobs=1, odd_exact=False, levels=2,
                 nu_start_mult=1.0, nu_override=None):
        err = ctypes.c_int32(0)
        self._h = lib().orc_oct_create(nx0, ny0, bl_width, ra, pr, utarget, seed, int(odd_exact), levels,
                                       nu_start_mult, 0 if nu_override is None else 1,
                                       0.0 if nu_override is None else float(nu_override),
                                       ctypes.byref(err))
        if not self._h:
            raise OracleError(f"orc_oct_create failed with code {err.value}")
        self.levels = levels

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_oct_destroy(h)
            self._h = None

    def step_cavity(self, n: int = 1):
        lib().orc_oct_step(self._h, int(n))

    def level_dims(self, level):
        nx, ny = ctypes.c_int32(), ctypes.c_int32()
        if lib().orc_oct_level_dims(self._h, level, ctypes.byref(nx), ctypes.byref(ny)):
            raise OracleError(f"no level {level}")
        return nx.value, ny.value

    def level(self, level, pops=False):
        nx, ny = self.level_dims(level)
        n = nx * ny
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "temp")}
        f = np.empty((n, 9)) if pops else None
        g = np.empty((n, 9)) if pops else None
        lib().orc_oct_get_level(self._h, level, _dp(out["rho"]), _dp(out["ux"]), _dp(out["uy"]),
                                _dp(out["temp"]), _dp(f), _dp(g))
        if pops:
            out["f"], out["g"] = f, g
        out["nx"], out["ny"] = nx, ny
        return out

    def restart_from(self, other):
        """set_from_snapshot (src/octree/solver.rs:1080-1168) from another
        octree of the same layout, then time_step = 0."""
        for lvl in range(3 if self.levels == 2 else 5):
            d = other.level(lvl)
            lib().orc_oct_restart_level(self._h, lvl, _dp(d["rho"]), _dp(d["ux"]), _dp(d["uy"]),
                                        _dp(d["temp"]))
        lib().orc_oct_set_time_step(self._h, 0)

    def info(self):
        o = np.empty(len(OCT_INFO_KEYS))
        lib().orc_oct_info(self._h, _dp(o))
        return dict(zip(OCT_INFO_KEYS, o.tolist()))

    def diag(self):
        o = np.empty(len(OCT_DIAG_KEYS))
        lib().orc_oct_diag(self._h, _dp(o))
        return dict(zip(OCT_DIAG_KEYS, o.tolist()))

    def set_dynamic_sgs(self, on, smag_alpha=0.5, nu_sm_min=-0.1, eta_test=2.0):
        """set_dynamic_sgs (src/octree/solver.rs:476-481)."""
        lib().orc_oct_set_dynamic_sgs(self._h, int(bool(on)), float(smag_alpha), float(nu_sm_min),
                                      float(eta_test))

    def dynamic_stats(self):
        """cs_dyn_mean / _max, kappa_dyn_mean / _max (the L0 model of the last
        step), nu_t_max (all levels) and the current rescaling factors."""
        o = np.empty(len(OCT_DYN_KEYS))
        lib().orc_oct_dynamic_stats(self._h, _dp(o))
        return dict(zip(OCT_DYN_KEYS, o.tolist()))

    def nu_t(self, level):
        """(nu_t_pre, alpha_t_pre) of a level, as last computed."""
        nx, ny = self.level_dims(level)
        a, b = np.empty(nx * ny), np.empty(nx * ny)
        if lib().orc_oct_get_nut(self._h, level, _dp(a), _dp(b)):
            raise OracleError(f"no level {level}")
        return a, b
