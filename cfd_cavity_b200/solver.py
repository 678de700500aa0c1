"""Python mirror of the reference's ``uniform::solver::CavitySolver`` over the C ABI.

Same constructor arguments as ``CavitySolver::new``
(``src/uniform/solver.rs:108``), same methods (``step``,
``init_from_fields``, ``idx``, ``nx``, ``ny``, ``total_mass``,
``total_f_mass``) and the ``pub(crate)`` phases the reference tests call
(``collide``, ``stream``, ``apply_bounce_back``,
``apply_thermal_boundary_conditions``, ``update_macroscopic``,
``enforce_wall_velocity``; ``src/uniform/tests.rs:154-169``).  The fields the
reference's callers read directly (``lbm.rho``, ``lbm.temperature``,
``nu_t``, ``fy_node``, ``lbm.f`` ...) are properties that copy the device
state back.  All computation runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

T_HOT = 0.5
T_COLD = -0.5
DELTA_T = T_HOT - T_COLD


def _dp(a):
    return None if a is None else a.ctypes.data_as(L._dp)


class CavitySolver:
    """One cavity on one GPU (``CavitySolver``, src/uniform/solver.rs:35-104)."""

    def __init__(self, nx, ny, ra, pr, cs, pr_t, utarget, seed, jobs=1, alpha_mult=1.0,
                 nu_start_mult=1.0, nu_override=None, *, precision="f64",
                 init_mode=L.CAV_INIT_LINEAR, noise_amp=1.0e-3, geq_order=2,
                 t_hot_profile=None, t_cold=T_COLD, device=0):
        lib = L.load()
        p = L.CavParams()
        L.check(lib.cav_default_params(ctypes.byref(p)))
        p.nx, p.ny, p.ra, p.pr, p.cs, p.pr_t, p.utarget = nx, ny, ra, pr, cs, pr_t, utarget
        p.seed, p.jobs, p.alpha_mult, p.nu_start_mult = seed, jobs, alpha_mult, nu_start_mult
        p.has_nu_override = 0 if nu_override is None else 1
        p.nu_override = 0.0 if nu_override is None else float(nu_override)
        p.init_mode, p.noise_amp, p.geq_order = init_mode, noise_amp, geq_order
        self._t_hot = None
        if t_hot_profile is not None:
            self._t_hot = np.ascontiguousarray(t_hot_profile, dtype=np.float64)
            if self._t_hot.shape != (ny,):
                raise ValueError("t_hot_profile must have ny values")
            p.t_hot_profile = _dp(self._t_hot)
        p.t_cold = t_cold
        p.precision = L.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p.device = device
        h = ctypes.c_void_p()
        L.check(lib.cav_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self._nx, self._ny = nx, ny
        self.precision = precision

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            L.load().cav_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        L.check(rc, self._h)

    # -- CavitySolver methods --------------------------------------------------
    def nx(self):
        return self._nx

    def ny(self):
        return self._ny

    def idx(self, ix, iy):
        return iy * self._nx + ix

    def step(self, n: int = 1):
        """``n`` calls of ``CavitySolver::step`` (src/uniform/solver.rs:279-293)."""
        self._ck(L.load().cav_step(self._h, int(n)))

    def init_from_fields(self, rho, ux, uy, t):
        n = self._nx * self._ny
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(n) for a in (rho, ux, uy, t)]
        self._ck(L.load().cav_init_from_fields(self._h, *[_dp(a) for a in arrs]))

    def collide(self, step):
        self._ck(L.load().cav_debug_phase(self._h, L.CAV_PHASE_COLLIDE, int(step)))

    def stream(self):
        self._ck(L.load().cav_debug_phase(self._h, L.CAV_PHASE_STREAM, 0))

    def apply_bounce_back(self):
        self._ck(L.load().cav_debug_phase(self._h, L.CAV_PHASE_BOUNCE_BACK, 0))

    def apply_thermal_boundary_conditions(self):
        self._ck(L.load().cav_debug_phase(self._h, L.CAV_PHASE_THERMAL_BC, 0))

    def update_macroscopic(self):
        self._ck(L.load().cav_debug_phase(self._h, L.CAV_PHASE_MACRO, 0))

    def enforce_wall_velocity(self):
        self._ck(L.load().cav_debug_phase(self._h, L.CAV_PHASE_NOSLIP, 0))

    def set_time_step(self, t):
        self._ck(L.load().cav_set_time_step(self._h, int(t)))

    # -- state access ------------------------------------------------------------
    def fields(self):
        n = self._nx * self._ny
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "temperature", "nu_t", "fy_node")}
        self._ck(L.load().cav_get_fields(self._h, *[_dp(out[k]) for k in
                                                     ("rho", "ux", "uy", "temperature", "nu_t",
                                                      "fy_node")]))
        return out

    def set_fields(self, rho=None, ux=None, uy=None, temperature=None, fy_node=None):
        n = self._nx * self._ny
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(n)
                for a in (rho, ux, uy, temperature, fy_node)]
        self._ck(L.load().cav_set_fields(self._h, *[_dp(a) for a in arrs]))

    def populations(self):
        n = self._nx * self._ny
        f = np.empty((n, 9))
        g = np.empty((n, 9))
        self._ck(L.load().cav_get_populations(self._h, _dp(f), _dp(g)))
        return f, g

    def set_populations(self, f=None, g=None):
        n = self._nx * self._ny
        fa = None if f is None else np.ascontiguousarray(f, dtype=np.float64).reshape(n, 9)
        ga = None if g is None else np.ascontiguousarray(g, dtype=np.float64).reshape(n, 9)
        self._ck(L.load().cav_set_populations(self._h, _dp(fa), _dp(ga)))

    def info(self):
        i = L.CavInfo()
        self._ck(L.load().cav_get_info(self._h, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in L.CavInfo._fields_}

    def diag(self):
        d = L.CavDiag()
        self._ck(L.load().cav_diag(self._h, ctypes.byref(d)))
        return {k: getattr(d, k) for k, _ in L.CavDiag._fields_}

    def check_guards(self, max_u_abort=0.10):
        """Status of the driver's guards (src/main.rs:209-276), 0 when all pass."""
        return L.load().cav_check_guards(self._h, max_u_abort)

    def sync(self):
        self._ck(L.load().cav_sync(self._h))

    def stream_handle(self):
        s = ctypes.c_void_p()
        self._ck(L.load().cav_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def set_step_kernel(self, kernel):
        """Kernel of the fused step: 0 one node per thread, 1 two x-adjacent
        nodes per thread, 2 the same pairs with their f and g halves on two
        warps (16-bit formats: 2 is the default up to 70 000 nodes, 1
        above); same bits."""
        self._ck(L.load().cav_set_step_kernel(self._h, int(kernel)))

    def step_kernel(self):
        k = ctypes.c_int32()
        self._ck(L.load().cav_get_step_kernel(self._h, ctypes.byref(k)))
        return k.value

    def launch_count(self):
        n = ctypes.c_int64()
        self._ck(L.load().cav_launch_count(self._h, ctypes.byref(n)))
        return n.value

    # -- reference field names -----------------------------------------------------
    @property
    def temperature(self):
        return self.fields()["temperature"]

    @property
    def rho(self):
        return self.fields()["rho"]

    @property
    def ux(self):
        return self.fields()["ux"]

    @property
    def uy(self):
        return self.fields()["uy"]

    @property
    def nu_t(self):
        return self.fields()["nu_t"]

    @property
    def fy_node(self):
        return self.fields()["fy_node"]

    def __getattr__(self, name):
        if name in ("nu", "alpha", "alpha_phys", "beta_eff", "lz", "lx", "tau", "tau_t",
                    "time_step", "spin_up_steps"):
            return self.info()[name]
        raise AttributeError(name)

    def total_mass(self):
        """``total_mass`` (src/uniform/solver.rs:1012-1014), FP64 device reduction."""
        return self.diag()["total_mass"]

    def total_f_mass(self):
        """``total_f_mass`` (src/uniform/solver.rs:1018-1020)."""
        return self.diag()["total_f_mass"]

    # -- snapshots -----------------------------------------------------------------
    def write_snapshot(self, path):
        """The fields to a CAVSNAP1 file (snapshot::write_snapshot_atomic)."""
        self._ck(L.load().cav_snapshot_write(self._h, str(path).encode()))

    def restart_from_snapshot(self, path):
        """The driver's --restart: CAVSNAP1 file, bilinear regrid when the grid
        differs, equilibrium populations, time step 0 (on the device)."""
        self._ck(L.load().cav_restart_from_snapshot(self._h, str(path).encode()))

    # -- dynamic mixed-scale subgrid model ---------------------------------------
    def set_dynamic_sgs(self, dynamic_smag, smag_alpha=0.5, nu_sm_min=-0.1, eta_test=2.0):
        """``set_dynamic_sgs`` (src/uniform/solver.rs:215-220)."""
        self._ck(L.load().cav_set_dynamic_sgs(self._h, 1 if dynamic_smag else 0, smag_alpha, nu_sm_min,
                                              eta_test))

    def dynamic_stats(self):
        """cs_dyn_mean, cs_dyn_max, kappa_dyn_mean, kappa_dyn_max of the last step."""
        o = np.empty(4)
        self._ck(L.load().cav_dynamic_sgs_stats(self._h, _dp(o)))
        return dict(zip(("cs_dyn_mean", "cs_dyn_max", "kappa_dyn_mean", "kappa_dyn_max"), o.tolist()))

    # -- adjoint -----------------------------------------------------------------
    def adjoint_nusselt(self, n_steps, window_start, checkpoint_every=500):
        """Gradients of J = mean over s in [window_start, n_steps] of the hot-wall
        Nusselt number (post.rs:68-78) w.r.t. the hot-wall theta profile and
        Cs, by the discrete adjoint with checkpoint-and-recompute.  Starts from
        step 0 and leaves the solver at step n_steps.  Returns
        (J, dJ/dtheta_w [ny], dJ/dCs, info)."""
        spec = L.CavAdjointSpec(int(n_steps), int(window_start), int(checkpoint_every))
        res = L.CavAdjointResult()
        gth = np.empty(self._ny)
        self._ck(L.load().cav_adjoint_run(self._h, ctypes.byref(spec), _dp(gth), ctypes.byref(res)))
        info = {"forward_ms": res.forward_ms, "reverse_ms": res.reverse_ms,
                "checkpoints": res.checkpoints}
        return res.objective, gth, res.grad_cs, info

    # -- per-step Nusselt accumulation --------------------------------------------
    def nu_accumulate(self, enable=True):
        self._ck(L.load().cav_nu_accumulate(self._h, 1 if enable else 0))

    def nu_accumulated(self):
        hot, cold, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        self._ck(L.load().cav_nu_accumulated(self._h, ctypes.byref(hot), ctypes.byref(cold),
                                             ctypes.byref(n)))
        return hot.value, cold.value, n.value


class TimeAverager:
    """``TimeAverager`` (src/uniform/post.rs:11-57), accumulated on the device."""

    def __init__(self, solver: CavitySolver):
        self.s = solver
        self.s._ck(L.load().cav_reset_means(self.s._h))

    def accumulate(self, s: CavitySolver | None = None):
        s = s or self.s
        s._ck(L.load().cav_sample(s._h))

    def means(self):
        n = self.s._nx * self.s._ny
        out = [np.empty(n) for _ in range(5)]
        cnt = ctypes.c_int64()
        self.s._ck(L.load().cav_get_means(self.s._h, *[_dp(a) for a in out], ctypes.byref(cnt)))
        return cnt.value, out

    def nusselt_from_mean(self, hot=True):
        v = ctypes.c_double()
        self.s._ck(L.load().cav_nusselt_from_mean(self.s._h, 1 if hot else 0, ctypes.byref(v)))
        return v.value


def write_snapshot_fields(path, nx, ny, rho, ux, uy, t):
    """write_snapshot_atomic (src/uniform/snapshot.rs:13-61), host only."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(nx * ny) for a in (rho, ux, uy, t)]
    L.check(L.load().cav_snapshot_write_fields(str(path).encode(), nx, ny, *[_dp(a) for a in arrs]))


def read_snapshot_fields(path):
    """read_snapshot (src/uniform/snapshot.rs:64-97): (nx, ny, rho, ux, uy, t)."""
    nx, ny = ctypes.c_int64(), ctypes.c_int64()
    lib = L.load()
    L.check(lib.cav_snapshot_read_fields(str(path).encode(), ctypes.byref(nx), ctypes.byref(ny), None, None,
                                         None, None))
    n = nx.value * ny.value
    out = [np.empty(n) for _ in range(4)]
    L.check(lib.cav_snapshot_read_fields(str(path).encode(), ctypes.byref(nx), ctypes.byref(ny),
                                         *[_dp(a) for a in out]))
    return (nx.value, ny.value, *out)
