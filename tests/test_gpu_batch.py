"""Batched cavities (cav_batch_*): one launch per step over many cavities of
uneven size and Ra.  Each cavity of a batch must evolve bit-identically to
the same cavity created alone (same kernel body, same per-step scalars, same
rounding stream), whatever the tile / grid tuning."""
import numpy as np
import pytest

from cfd_cavity_b200 import CavitySolver, CavityBatch, sweep_configs
from cfd_cavity_b200 import _lib as L

pytestmark = pytest.mark.gpu

MIXED = [
    dict(nx=64, ny=256, ra=1e6, cs=0.10, seed=1),
    dict(nx=96, ny=384, ra=3e7, cs=0.08, seed=2),
    dict(nx=37, ny=61, ra=2e5, cs=0.12, seed=3),
    dict(nx=128, ny=512, ra=1e8, cs=0.11, seed=4),
]


def single(c, precision):
    return CavitySolver(c["nx"], c["ny"], c["ra"], 0.71, c["cs"], 0.9, 0.02, c["seed"],
                        precision=precision, init_mode=L.CAV_INIT_ZERO, noise_amp=1e-4)


@pytest.mark.parametrize("precision,kernel", [("f64", 3), ("f32", 3), ("f32", 4), ("f16sr", 3), ("f16sr", 5),
                                              ("f16gsr", 5), ("bf16sr", 5), ("f16", 5), ("f16sr", 6), ("f16gsr", 6),
                                              ("bf16sr", 6), ("bf16", 6)])
def test_batch_is_bitwise_equal_to_single_cavities(precision, kernel):
    """Every cavity of the batch against the same cavity created alone (its
    default single-cavity kernel: node pairs for the 16-bit formats)."""
    b = CavityBatch(MIXED, precision=precision)
    b.set_tuning(4, 3, kernel=kernel)
    singles = [single(c, precision) for c in MIXED]
    for n in (1, 150, 137):  # spin-up steps (table rows), graph replays, remainders
        b.step(n)
        for s in singles:
            s.step(n)
    assert b.info()["time_step"] == 288
    for i, s in enumerate(singles):
        fb, fs = b.fields(i), s.fields()
        for k in fb:
            assert np.array_equal(fb[k], fs[k]), (i, k)
        pb, ps = b.populations(i), s.populations()
        assert np.array_equal(pb[0], ps[0]) and np.array_equal(pb[1], ps[1])


@pytest.mark.parametrize("precision", ["f64", "f32", "f16sr", "bf16", "f16gsr"])
def test_batch_tuning_does_not_change_results(precision):
    """Tile heights, grid sizes and the kernel (persistent or one CTA per item
    from global memory, TMA-staged shared-memory tiles, two nodes per thread
    on packed FP32x2 lanes) change no bit."""
    a = CavityBatch(MIXED, precision=precision)
    b = CavityBatch(MIXED, precision=precision)
    a.set_tuning(3, 2, kernel=0)
    b.set_tuning(32, 16, kernel=1)
    a.step(100)
    b.step(40)
    b.set_tuning(2, 7, kernel=3)
    b.step(20)
    b.set_tuning(5, 1, kernel=2)
    b.step(15)
    b.set_tuning(8, 1, kernel=4)
    b.step(5)
    b.set_tuning(1, 1, kernel=5)
    b.step(5)
    b.set_tuning(8, 1, kernel=5)
    b.step(5)
    b.set_tuning(8, 3, kernel=6)
    b.step(5)
    b.set_tuning(4, 2, kernel=6)
    b.step(5)
    for i in range(len(MIXED)):
        fa, fb = a.fields(i), b.fields(i)
        for k in fa:
            assert np.array_equal(fa[k], fb[k]), (i, k)
        pa, pb = a.populations(i), b.populations(i)
        assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1])


def test_autotune_picks_a_candidate_and_leaves_the_state_alone():
    b = CavityBatch(MIXED[:2], precision="f16sr")
    ref = CavityBatch(MIXED[:2], precision="f16sr")
    b.step(10)
    ref.step(10)
    t = b.autotune(trial_steps=16)
    assert t["kernel"] in (0, 1, 2, 3, 4, 5, 6)
    if t["kernel"] == 0:
        assert t["rows_per_item"] in (4, 8, 16) and t["ctas_per_sm"] in (4, 8, 16)
    elif t["kernel"] in (1, 2):
        assert set(t) == {"kernel", "ctas_per_sm"} and t["ctas_per_sm"] in (1, 2, 3, 4)
    elif t["kernel"] == 6:
        assert t["rows_per_item"] in (4, 8) and t["ctas_per_sm"] in (3, 4, 5)
    else:
        assert set(t) == {"kernel", "rows_per_item"} and t["rows_per_item"] in (1, 2, 4, 8)
    assert b.tuning() == t
    assert b.info()["time_step"] == 10
    b.step(70)
    ref.step(70)
    assert np.array_equal(b.fields(1)["temperature"], ref.fields(1)["temperature"])


def test_item_heights_outside_a_kernels_range_are_rejected():
    b = CavityBatch(MIXED[:2], precision="f16sr")
    for rows, kernel in ((3, 3), (16, 5), (1, 4), (2, 6)):
        with pytest.raises(L.CavError) as e:
            b.set_tuning(rows, 8, kernel=kernel)
        assert e.value.code == L.CAV_ERR_ARG


def test_sweep_batch_runs_and_conserves_mass():
    """The 64-cavity sweep (Ra log-uniform in [1e6, 1e8], three grids, Cs in
    [0.08, 0.12]) in 16-bit storage: finite, mass conserved, per-cavity
    diagnostics available."""
    cfg = sweep_configs(64)
    b = CavityBatch(cfg, precision="f16sr")
    assert b.info()["total_nodes"] == sum(c["nx"] * c["ny"] for c in cfg)
    m0 = [b.diag(i)["total_f_mass"] for i in (0, 31, 63)]
    b.step(600)
    for j, i in enumerate((0, 31, 63)):
        d = b.diag(i)
        assert d["finite"] == 1
        assert abs(d["total_f_mass"] - m0[j]) / m0[j] < 1e-4
        assert d["max_u"] < 0.1


def test_tile_kernel_bounded_wait_reports_timeout_and_device_stays_usable():
    """The tile kernel's mbarrier waits give up after about a second: with
    the copies withheld (nothing in flight), the step reports CAV_ERR_TIMEOUT
    at the next sync instead of hanging, and the batch (and the device) run
    normally afterwards."""
    import time

    b = CavityBatch(MIXED[:2], precision="f16sr")
    b.set_tuning(16, 2, kernel=1)
    b.step(3)
    b.sync()
    b.debug_stall_copies(True)
    t0 = time.perf_counter()
    b.step(1)
    with pytest.raises(L.CavError) as e:
        b.sync()
    assert e.value.code == L.CAV_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 30.0
    b.debug_stall_copies(False)
    b.step(5)
    b.sync()
    ref = CavityBatch(MIXED[:2], precision="f16sr")
    ref.step(20)
    assert np.all(np.isfinite(ref.fields(1)["temperature"]))
