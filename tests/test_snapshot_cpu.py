"""Snapshot files (CAVSNAP1, src/uniform/snapshot.rs:10-131) through the
host-only entry points, and interpolate_field on the oracle: the reference's
snapshot tests (src/uniform/tests.rs:15-110), no GPU needed."""
import os
import struct

import numpy as np
import pytest

import oracle
from cfd_cavity_b200 import _lib as L
from cfd_cavity_b200.solver import read_snapshot_fields, write_snapshot_fields

T_HOT, T_COLD = 0.5, -0.5


def fields(nx, ny, a=1e-4, b=0.001, c=-0.002):
    n = nx * ny
    k = np.arange(n, dtype=np.float64)
    return 1.0 + a * k, b * k, c * k, 0.5 - k / n


def test_snapshot_atomic_write_roundtrips_and_leaves_no_temporary(tmp_path):
    """src/uniform/tests.rs:17-60."""
    nx, ny = 10, 14
    rho, ux, uy, t = fields(nx, ny)
    path = tmp_path / "snapshot.bin"
    write_snapshot_fields(path, nx, ny, rho, ux, uy, t)
    rnx, rny, rr, ru, rv, rt = read_snapshot_fields(path)
    assert (rnx, rny) == (nx, ny)
    for a, b in ((rr, rho), (ru, ux), (rv, uy), (rt, t)):
        np.testing.assert_array_equal(a, b)
    rho2 = np.full(nx * ny, 2.0)
    write_snapshot_fields(path, nx, ny, rho2, ux, uy, t)
    np.testing.assert_array_equal(read_snapshot_fields(path)[2], rho2)
    assert not [p for p in os.listdir(tmp_path) if p.endswith(".tmp")]


def test_snapshot_file_layout_is_the_reference_format(tmp_path):
    """CAVSNAP1 magic, nx, ny as u64 LE, then rho, ux, uy, T as LE f64
    (src/uniform/snapshot.rs:13-31): decoded here independently."""
    nx, ny = 12, 20
    rho, ux, uy, t = fields(nx, ny, 0.001, 0.01, -0.02)
    path = tmp_path / "s.bin"
    write_snapshot_fields(path, nx, ny, rho, ux, uy, t)
    raw = path.read_bytes()
    assert raw[:8] == b"CAVSNAP1"
    assert struct.unpack("<QQ", raw[8:24]) == (nx, ny)
    assert len(raw) == 24 + 4 * nx * ny * 8
    body = np.frombuffer(raw[24:], dtype="<f8").reshape(4, nx * ny)
    for a, b in zip(body, (rho, ux, uy, t)):
        np.testing.assert_array_equal(a, b)


def test_snapshot_read_errors(tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTASNAP" + bytes(40))
    with pytest.raises(L.CavError) as e:
        read_snapshot_fields(bad)
    assert e.value.code == L.CAV_ERR_IO
    nx, ny = 4, 5
    good = tmp_path / "good.bin"
    write_snapshot_fields(good, nx, ny, *fields(nx, ny))
    short = tmp_path / "short.bin"
    short.write_bytes(good.read_bytes()[:-8])
    with pytest.raises(L.CavError) as e:
        read_snapshot_fields(short)
    assert e.value.code == L.CAV_ERR_IO
    with pytest.raises(L.CavError):
        read_snapshot_fields(tmp_path / "missing.bin")


def test_interpolate_same_grid_identity():
    """src/uniform/tests.rs:89-94."""
    src = np.ones(5 * 9)
    np.testing.assert_array_equal(oracle.interpolate_field(src, 5, 9, 5, 9), src)


def test_interpolate_grid_change_linear_field_exact():
    """src/uniform/tests.rs:96-120: 8x32 -> 16x64 keeps a linear T exact."""
    nx0, ny0 = 8, 32
    xf = np.tile(np.arange(nx0) / (nx0 - 1), ny0)
    t0 = T_HOT + (T_COLD - T_HOT) * xf
    t1 = oracle.interpolate_field(t0, nx0, ny0, 16, 64).reshape(64, 16)
    exact = T_HOT + (T_COLD - T_HOT) * (np.arange(16) / 15.0)
    assert np.max(np.abs(t1 - exact[None, :])) < 1e-12
