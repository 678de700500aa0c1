"""Python mirror of the batch C ABI (``cav_batch_*``): many cavities advanced
in lockstep by one kernel launch per lattice step.

The reference runs one cavity per process (``src/main.rs:42-443``); a batch
is a set of ``CavitySolver::new`` objects stepped together.  Each cavity of a
batch evolves bit-identically to the same cavity created alone.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .solver import _dp

C3_SIZES = ((64, 256), (96, 384), (128, 512))


class Xorshift64Star:
    """xorshift64* (the reference's generator, src/uniform/rng.rs:5-31)."""

    def __init__(self, seed: int):
        self.s = (seed | 1) & 0xFFFFFFFFFFFFFFFF

    def next_u64(self) -> int:
        x = self.s
        x ^= x >> 12
        x ^= (x << 25) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 27
        self.s = x
        return (x * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF

    def next_f64(self) -> float:
        return (self.next_u64() >> 11) / float(1 << 53)


def sweep_configs(n=64, seed=2024, sizes=C3_SIZES, ra_range=(1e6, 1e8), cs_range=(0.08, 0.12)):
    """The batched sweep: per cavity Ra log-uniform in ra_range, a grid drawn
    uniformly from `sizes`, Cs uniform in cs_range, all from one seed; every
    cavity starts from theta = 0 + U(+-1e-4) noise with its own seed."""
    rng = Xorshift64Star(seed)
    lo, hi = np.log10(ra_range[0]), np.log10(ra_range[1])
    out = []
    for i in range(n):
        ra = 10.0 ** (lo + (hi - lo) * rng.next_f64())
        nx, ny = sizes[min(int(len(sizes) * rng.next_f64()), len(sizes) - 1)]
        cs = cs_range[0] + (cs_range[1] - cs_range[0]) * rng.next_f64()
        out.append(dict(nx=nx, ny=ny, ra=ra, cs=cs, seed=seed * 1000 + i))
    return out


def make_params(nx, ny, ra, cs=0.1, *, pr=0.71, pr_t=0.9, utarget=0.02, seed=42, precision="f16sr",
                init_mode=L.CAV_INIT_ZERO, noise_amp=1e-4, device=0, nu_override=None,
                alpha_mult=1.0, nu_start_mult=1.0, geq_order=2, t_cold=-0.5):
    p = L.CavParams()
    L.check(L.load().cav_default_params(ctypes.byref(p)))
    p.nx, p.ny, p.ra, p.pr, p.cs, p.pr_t, p.utarget, p.seed = nx, ny, ra, pr, cs, pr_t, utarget, seed
    p.alpha_mult, p.nu_start_mult = alpha_mult, nu_start_mult
    p.has_nu_override = 0 if nu_override is None else 1
    p.nu_override = 0.0 if nu_override is None else float(nu_override)
    p.init_mode, p.noise_amp, p.geq_order, p.t_cold = init_mode, noise_amp, geq_order, t_cold
    p.precision = L.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    p.device = device
    return p


class CavityBatch:
    """A batch of cavities (``cav_batch``)."""

    def __init__(self, configs, precision="f16sr", device=0, **common):
        ps = (L.CavParams * len(configs))()
        for i, c in enumerate(configs):
            kw = dict(common)
            kw.update({k: v for k, v in c.items() if k not in ("nx", "ny", "ra")})
            ps[i] = make_params(c["nx"], c["ny"], c["ra"], precision=precision, device=device, **kw)
        h = ctypes.c_void_p()
        L.check_batch(L.load().cav_batch_create(ps, len(configs), ctypes.byref(h)))
        self._b = h
        self.sizes = [(c["nx"], c["ny"]) for c in configs]

    def close(self):
        b = getattr(self, "_b", None)
        if b:
            L.load().cav_batch_destroy(b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        L.check_batch(rc, self._b)

    def __len__(self):
        return len(self.sizes)

    def step(self, n=1):
        self._ck(L.load().cav_batch_step(self._b, int(n)))

    def fields(self, i):
        nx, ny = self.sizes[i]
        out = {k: np.empty(nx * ny) for k in ("rho", "ux", "uy", "temperature", "nu_t", "fy_node")}
        self._ck(L.load().cav_batch_get_fields(self._b, i, *[_dp(out[k]) for k in
                                                            ("rho", "ux", "uy", "temperature", "nu_t",
                                                             "fy_node")]))
        return out

    def populations(self, i):
        nx, ny = self.sizes[i]
        f = np.empty((nx * ny, 9))
        g = np.empty((nx * ny, 9))
        self._ck(L.load().cav_batch_get_populations(self._b, i, _dp(f), _dp(g)))
        return f, g

    def diag(self, i):
        d = L.CavDiag()
        self._ck(L.load().cav_batch_diag(self._b, i, ctypes.byref(d)))
        return {k: getattr(d, k) for k, _ in L.CavDiag._fields_}

    def info(self):
        n, nodes, t = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        self._ck(L.load().cav_batch_info(self._b, ctypes.byref(n), ctypes.byref(nodes), ctypes.byref(t)))
        return {"n_cavities": n.value, "total_nodes": nodes.value, "time_step": t.value}

    @staticmethod
    def _used(t):
        """The kernel and the tuning fields it uses (cav_batch_tuning)."""
        k = t.kernel
        if k == 0:
            return {"kernel": 0, "rows_per_item": t.rows_per_item, "ctas_per_sm": t.ctas_per_sm}
        if k in (1, 2):
            return {"kernel": k, "ctas_per_sm": t.ctas_per_sm}
        if k == 6:
            return {"kernel": 6, "rows_per_item": t.rows_per_item, "ctas_per_sm": t.ctas_per_sm}
        return {"kernel": k, "rows_per_item": t.rows_per_item}

    def tuning(self):
        """The current kernel and the tuning fields it uses."""
        t = L.CavBatchTuning()
        self._ck(L.load().cav_batch_get_tuning(self._b, ctypes.byref(t)))
        return self._used(t)

    def set_tuning(self, rows_per_item, ctas_per_sm, kernel=3):
        """kernel 0: the persistent global-memory kernel (rows_per_item,
        ctas_per_sm); 1 / 2: the TMA tile kernel in tile shape 1 or 2
        (ctas_per_sm); 3: one CTA per 32-column x rows_per_item item, one
        node per thread (1, 2, 4 or 8 rows); 4: the same items, two rows per
        thread on packed FP32x2 arithmetic (2, 4 or 8 rows); 5: one CTA per
        64-column x rows_per_item item, two x-adjacent nodes per thread
        (16-bit formats; 1, 2, 4 or 8 rows); 6: the node-pair body on
        TMA-staged tiles of 64 columns x rows_per_item rows (4 or 8),
        ctas_per_sm persistent CTAs per SM (16-bit formats)."""
        t = L.CavBatchTuning(rows_per_item, ctas_per_sm, int(kernel))
        self._ck(L.load().cav_batch_set_tuning(self._b, ctypes.byref(t)))

    def autotune(self, trial_steps=64):
        """Times every candidate kernel / parameter set three times on a twin
        batch (median kept), applies the fastest; returns it as tuning()."""
        t = L.CavBatchTuning()
        self._ck(L.load().cav_batch_autotune(self._b, int(trial_steps), ctypes.byref(t)))
        return self._used(t)

    def debug_stall_copies(self, on):
        """Test of the tile kernel's bounded waits: arm the barriers but issue
        no copy (the next sync raises CAV_ERR_TIMEOUT)."""
        self._ck(L.load().cav_batch_debug_stall_copies(self._b, int(bool(on))))

    def sync(self):
        self._ck(L.load().cav_batch_sync(self._b))

    def stream_handle(self):
        s = ctypes.c_void_p()
        self._ck(L.load().cav_batch_get_stream(self._b, ctypes.byref(s)))
        return s.value or 0

    def launch_count(self):
        n = ctypes.c_int64()
        self._ck(L.load().cav_batch_launch_count(self._b, ctypes.byref(n)))
        return n.value
