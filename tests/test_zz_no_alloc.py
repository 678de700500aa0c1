"""cav_diag_noalloc: the diagnostics on caller-owned device memory, with no
allocation by the library.

It exists for callers that cannot let the library call cudaMalloc (their own
allocator already holds the device memory they may use, or their loop cannot
take the device-wide synchronisation cudaMalloc / cudaFree may cause).  The
test keeps a cavity state in device buffers it owns (allocated here with
torch, i.e. by the caller), calls the entry point through the C ABI twice in
a row, and checks each result against cav_diag on the same state, within the
1e-12 relative tolerance of the other diagnostics tests.  This file is
collected last on purpose; it passes alone in a fresh process (its first call
then does the one-time scratch set-up) and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from cfd_cavity_b200 import CavitySolver
from cfd_cavity_b200 import _lib as L

pytestmark = pytest.mark.gpu

KEYS = ["nusselt_hot", "nusselt_cold", "nusselt_hot_wall_link", "total_mass", "total_f_mass",
        "max_u", "max_uy", "nu_t_max", "y_plus_hot", "nusselt_volume"]
MAX_ROWS = 8192  # CAV_NOALLOC_MAX_ROWS in include/cavity.h


def _fn():
    lib = L.load()
    fn = lib.cav_diag_noalloc
    vp = ctypes.c_void_p
    fn.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                   ctypes.c_double, vp, vp]
    fn.restype = ctypes.c_int32
    return fn


def _device_state(s, torch):
    """Copies the solver's state into device buffers owned by the caller."""
    fl = s.fields()
    f, _ = s.populations()
    dev = {k: torch.from_numpy(fl[k]).cuda() for k in ("rho", "ux", "uy", "temperature", "nu_t")}
    dev["f"] = torch.from_numpy(np.ascontiguousarray(f)).cuda()
    return dev


def _call(fn, dev, s, out, torch, stream=None):
    info = s.info()
    st = stream if stream is not None else torch.cuda.current_stream()
    rc = fn(dev["rho"].data_ptr(), dev["ux"].data_ptr(), dev["uy"].data_ptr(),
            dev["temperature"].data_ptr(), dev["nu_t"].data_ptr(), dev["f"].data_ptr(),
            s.nx(), s.ny(), info["nu"], info["lz"], out.data_ptr(), st.cuda_stream)
    st.synchronize()
    return rc, out.cpu().numpy().copy()


def _check(vals, ref):
    for j, k in enumerate(KEYS):
        assert abs(vals[j] - ref[k]) <= 1e-12 * max(abs(ref[k]), 1e-30), (k, vals[j], ref[k])
    assert vals[10] == 1.0 and ref["finite"] == 1


def test_noalloc_diagnostics_match_cav_diag_on_two_calls():
    torch = pytest.importorskip("torch")
    fn = _fn()
    s = CavitySolver(64, 256, 1e6, 0.71, 0.1, 0.9, 0.02, 42, precision="f64",
                     init_mode=L.CAV_INIT_ZERO, noise_amp=1e-4)
    out = torch.full((11,), float("nan"), dtype=torch.float64, device="cuda")

    s.step(500)
    dev = _device_state(s, torch)
    rc, first = _call(fn, dev, s, out, torch)
    assert rc == L.CAV_OK
    _check(first, s.diag())

    # second call in a row, on a later state: nothing stale from the first
    s.step(300)
    dev = _device_state(s, torch)
    rc, second = _call(fn, dev, s, out, torch)
    assert rc == L.CAV_OK
    _check(second, s.diag())
    assert not np.array_equal(first[:10], second[:10])

    # and the same input twice gives the same bits (fixed-order reduction)
    rc, again = _call(fn, dev, s, out, torch)
    assert rc == L.CAV_OK
    assert np.array_equal(second, again)


def test_noalloc_rejects_more_rows_than_its_scratch():
    torch = pytest.importorskip("torch")
    fn = _fn()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    rc = fn(p, p, p, p, p, p, 4, MAX_ROWS + 1, 0.01, float(MAX_ROWS), p, None)
    assert rc == L.CAV_ERR_ARG
    rc = fn(p, p, p, p, p, p, 4, 3, 0.01, 2.0, p, None)
    assert rc == L.CAV_ERR_ARG


def test_noalloc_at_the_row_limit_on_a_side_stream():
    """ny equal to the scratch's row count (its last row in use), on a
    caller-created stream rather than the default one."""
    torch = pytest.importorskip("torch")
    fn = _fn()
    s = CavitySolver(4, MAX_ROWS, 1e6, 0.71, 0.1, 0.9, 0.02, 7, precision="f64")
    s.step(40)
    dev = _device_state(s, torch)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        out = torch.full((11,), float("nan"), dtype=torch.float64, device="cuda")
        rc, vals = _call(fn, dev, s, out, torch, stream=side)
    assert rc == L.CAV_OK
    _check(vals, s.diag())
