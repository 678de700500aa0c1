"""Python mirror of the reference's block-refined ``octree::solver::CavitySolver``
(``src/octree/solver.rs:284-1206``) over the ``cav_octree_*`` C ABI.

Same constructor arguments as ``CavitySolver::new(nx0, ny0, bl_width, ra,
pr, utarget, seed, jobs, odd_exact, levels, nu_start_mult, nu_override)``,
``step_cavity``, ``noise_stats``, ``max_u_all``, ``check_guards`` and the
Nusselt estimators of ``src/octree/cavity.rs:672-741``.  The level fields
the reference tests read (``sim.coarse.rho``, ``block.fine.temp`` ...) come
back through ``level()``.  All computation runs in the CUDA library.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

COARSE, HOT_L1, COLD_L1, HOT_L2, COLD_L2 = range(5)
OCT_DYN_KEYS = ("cs_dyn_mean", "cs_dyn_max", "kappa_dyn_mean", "kappa_dyn_max", "nu_t_max",
                "xi_even", "xi_odd", "xi_th", "xi_b_hot_even", "xi_b_hot_odd", "xi_b_hot_th",
                "xi_b_cold_even", "xi_b_cold_odd", "xi_b_cold_th")


def _dp(a):
    return None if a is None else a.ctypes.data_as(L._dp)


class OctreeSolver:
    def __init__(self, nx0, ny0, bl_width, ra, pr, utarget, seed, jobs=1, odd_exact=False, levels=2,
                 nu_start_mult=1.0, nu_override=None, *, precision="f64", device=0, cs=0.0,
                 pr_t=0.9):
        lib = L.load()
        p = L.CavOctreeParams()
        L.check_octree(lib.cav_octree_default_params(ctypes.byref(p)))
        p.nx0, p.ny0, p.bl_width = nx0, ny0, bl_width
        p.ra, p.pr, p.utarget, p.seed, p.jobs = ra, pr, utarget, seed, jobs
        p.odd_exact, p.levels, p.nu_start_mult = int(bool(odd_exact)), levels, nu_start_mult
        p.has_nu_override = 0 if nu_override is None else 1
        p.nu_override = 0.0 if nu_override is None else float(nu_override)
        p.precision = L.OCT_PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p.device = device
        p.cs, p.pr_t = cs, pr_t
        h = ctypes.c_void_p()
        L.check_octree(lib.cav_octree_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.precision = precision
        self.levels = levels
        self.nx0, self.ny0 = nx0, ny0

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            L.load().cav_octree_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        L.check_octree(rc, self._h)

    def step_cavity(self, n: int = 1):
        """``n`` calls of ``step_cavity`` (src/octree/solver.rs:647-947)."""
        self._ck(L.load().cav_octree_step(self._h, int(n)))

    def info(self):
        i = L.CavOctreeInfo()
        self._ck(L.load().cav_octree_get_info(self._h, ctypes.byref(i)))
        out = {}
        for k, _ in L.CavOctreeInfo._fields_:
            v = getattr(i, k)
            out[k] = list(v) if isinstance(v, ctypes.Array) else v
        return out

    def n_nodes_total(self):
        """``n_nodes_total`` (src/octree/solver.rs:475-486)."""
        return self.info()["n_nodes_total"]

    def level(self, lvl, pops=False):
        """Fields of level ``lvl`` (0 coarse, 1/2 hot/cold L1, 3/4 hot/cold L2)."""
        i = self.info()
        nx, ny = i["nx"][lvl], i["ny"][lvl]
        n = nx * ny
        out = {k: np.empty(n) for k in ("rho", "ux", "uy", "temp")}
        f = np.empty((n, 9)) if pops else None
        g = np.empty((n, 9)) if pops else None
        self._ck(L.load().cav_octree_get_level(self._h, lvl, _dp(out["rho"]), _dp(out["ux"]),
                                               _dp(out["uy"]), _dp(out["temp"]), _dp(f), _dp(g)))
        if pops:
            out["f"], out["g"] = f, g
        out["nx"], out["ny"] = nx, ny
        return out

    def set_level(self, lvl, rho=None, ux=None, uy=None, temp=None, f=None, g=None):
        def c(a, shape=None):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            return a
        arrs = [c(a) for a in (rho, ux, uy, temp, f, g)]
        self._ck(L.load().cav_octree_set_level(self._h, lvl, *[_dp(a) for a in arrs]))

    def set_time_step(self, t):
        self._ck(L.load().cav_octree_set_time_step(self._h, int(t)))

    def restart_from(self, other: "OctreeSolver"):
        """``set_from_snapshot`` (src/octree/solver.rs:1080-1168) from another
        solver with the same layout: every level restarts at the equilibrium
        of the other's fields, then the time step (and the ramps) restart at 0."""
        n = 3 if self.levels == 2 else 5
        if other.levels != self.levels or other.info()["nx"] != self.info()["nx"] \
                or other.info()["ny"] != self.info()["ny"]:
            raise ValueError("restart needs the same level layout")
        for lvl in range(n):
            d = other.level(lvl)
            self._ck(L.load().cav_octree_restart_level(self._h, lvl, _dp(d["rho"]), _dp(d["ux"]),
                                                       _dp(d["uy"]), _dp(d["temp"])))
        self.set_time_step(0)

    def write_snapshot(self, path, step=None):
        """``snapshot`` + ``write_snapshot_atomic`` (src/octree/snapshot.rs:147-165)."""
        st = self.time_step if step is None else step
        self._ck(L.load().cav_octree_snapshot_write(self._h, str(path).encode(), int(st)))

    def restart_from_snapshot(self, path):
        """``set_from_snapshot`` of an OCTSNAP1 file (same layout), time step 0."""
        self._ck(L.load().cav_octree_restart_from_snapshot(self._h, str(path).encode()))

    def couple(self, which):
        """One coupling: 0 coarse_to_fine L0->L1, 1 fine_to_coarse L1->L0,
        2 / 3 the same between L1 and L2 (src/octree/interface.rs:137-206)."""
        self._ck(L.load().cav_octree_couple(self._h, int(which)))

    def diag(self):
        d = L.CavOctreeDiag()
        self._ck(L.load().cav_octree_diag(self._h, ctypes.byref(d)))
        return {k: getattr(d, k) for k, _ in L.CavOctreeDiag._fields_}

    def noise_stats(self):
        """``noise_stats`` (src/octree/solver.rs:954-1003)."""
        d = self.diag()
        return {"max_rho_dev": d["max_rho_dev"], "max_rho_dev_ifaces": d["max_rho_dev_ifaces"],
                "masse": d["mass"]}

    def max_u_all(self):
        return self.diag()["max_u"]

    def nusselt_hot(self):
        return self.diag()["nu_hot"]

    def nusselt_cold(self):
        return self.diag()["nu_cold"]

    def nusselt_hot_link0(self):
        return self.diag()["nu_hot_link0"]

    def nusselt_hot_fine(self):
        return self.diag()["nu_hot_fine"]

    def check_guards(self, max_u_abort=0.10):
        """``check_guards`` (src/octree/solver.rs:1019-1038): 0 when all pass."""
        return L.load().cav_octree_check_guards(self._h, max_u_abort)

    def sync(self):
        self._ck(L.load().cav_octree_sync(self._h))

    def stream_handle(self):
        s = ctypes.c_void_p()
        self._ck(L.load().cav_octree_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def launch_count(self):
        n = ctypes.c_int64()
        self._ck(L.load().cav_octree_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def set_level_kernel(self, kind):
        """The fine levels' step kernel: ``CAV_OCT_LEVEL_NODE`` (one thread
        per node) or ``CAV_OCT_LEVEL_FG`` (a node's f and g halves on two
        threads, the default where it applies); same results bit for bit."""
        self._ck(L.load().cav_octree_set_level_kernel(self._h, int(kind)))

    def level_kernel(self):
        k = ctypes.c_int32()
        self._ck(L.load().cav_octree_get_level_kernel(self._h, ctypes.byref(k)))
        return k.value

    def set_dynamic_sgs(self, on, smag_alpha=0.5, nu_sm_min=-0.1, eta_test=2.0):
        """``set_dynamic_sgs`` (src/octree/solver.rs:476-481): the dynamic
        mixed-scale model on every level (src/octree/smag.rs)."""
        self._ck(L.load().cav_octree_set_dynamic_sgs(self._h, int(bool(on)), float(smag_alpha),
                                                     float(nu_sm_min), float(eta_test)))

    def dynamic_stats(self):
        """``cs_dyn_mean`` / ``cs_dyn_max`` / ``kappa_dyn_mean`` /
        ``kappa_dyn_max`` of the last L0 model, ``nu_t_max`` over every level,
        and the rescaling factors in use (xi A, xi B of each strip)."""
        o = np.empty(len(OCT_DYN_KEYS))
        self._ck(L.load().cav_octree_dynamic_stats(self._h, _dp(o)))
        return dict(zip(OCT_DYN_KEYS, o.tolist()))

    def nu_t(self, lvl):
        """(nu_t_pre, alpha_t_pre) of a level as last computed by the model."""
        i = self.info()
        n = i["nx"][lvl] * i["ny"][lvl]
        a, b = np.empty(n), np.empty(n)
        self._ck(L.load().cav_octree_get_nu_t(self._h, int(lvl), _dp(a), _dp(b)))
        return a, b

    @property
    def time_step(self):
        return self.info()["time_step"]
