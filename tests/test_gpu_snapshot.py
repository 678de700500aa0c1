"""Snapshots and the restart from them on the GPU path.

Uniform cavity (--restart, src/uniform/snapshot.rs + solver.rs:232-262): a
CAVSNAP1 file written from the device, read into a cavity of another size
(bilinear regrid on the device) and stepped, is bit-identical in FP64 to the
oracle doing interpolate_field + init_from_fields + the same steps.  Octree
(OCTSNAP1, src/octree/snapshot.rs and tests.rs:783-965): the round trip is
byte-identical, a restart equals the oracle's set_from_snapshot bit for bit,
and a layout mismatch is an error.
"""
import struct

import numpy as np
import pytest

import oracle
from cfd_cavity_b200 import CavitySolver
from cfd_cavity_b200 import _lib as L
from cfd_cavity_b200.octree import OctreeSolver
from cfd_cavity_b200.solver import read_snapshot_fields

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dst", [(64, 256), (96, 384)])
def test_uniform_restart_with_regrid_matches_oracle(tmp_path, dst):
    src = CavitySolver(64, 256, 1e7, 0.71, 0.1, 0.9, 0.02, 42, precision="f64")
    src.step(200)
    path = tmp_path / "snap.bin"
    src.write_snapshot(path)
    nx0, ny0, r, u, v, t = read_snapshot_fields(path)
    f = src.fields()
    for a, k in ((r, "rho"), (u, "ux"), (v, "uy"), (t, "temperature")):
        np.testing.assert_array_equal(a, f[k])
    nx1, ny1 = dst
    g = CavitySolver(nx1, ny1, 1e8, 0.71, 0.1, 0.9, 0.02, 7, precision="f64")
    g.restart_from_snapshot(path)
    assert g.info()["time_step"] == 0
    o = oracle.OracleSolver(nx1, ny1, 1e8, 0.71, 0.1, 0.9, 0.02, 7)
    fi = [oracle.interpolate_field(a, nx0, ny0, nx1, ny1) for a in (r, u, v, t)]
    o.init_from_fields(*fi)
    gf, of = g.fields(), o.fields()
    for k in ("rho", "ux", "uy", "temperature"):
        np.testing.assert_array_equal(gf[k], of[k])
    g.step(30)
    o.step(30)
    gf, of = g.fields(), o.fields()
    for k in ("rho", "ux", "uy", "temperature", "nu_t"):
        np.testing.assert_array_equal(gf[k], of[k])


def test_uniform_restart_16bit_storage(tmp_path):
    src = CavitySolver(64, 256, 1e7, 0.71, 0.1, 0.9, 0.02, 42, precision="f32")
    src.step(100)
    path = tmp_path / "s.bin"
    src.write_snapshot(path)
    g = CavitySolver(128, 512, 1e8, 0.71, 0.1, 0.9, 0.02, 7, precision="f16sr")
    g.restart_from_snapshot(path)
    g.step(50)
    assert g.diag()["finite"] == 1


def octree_pair(levels=3, seed=42, bl=4):
    args = (32, 64, bl, 1.0e6, 0.71, 0.02, seed)
    return OctreeSolver(*args, levels=levels, precision="f64"), oracle.OracleOctree(*args, levels=levels)


def test_octree_snapshot_roundtrip_and_restart(tmp_path):
    """src/octree/tests.rs:796-948."""
    g, o = octree_pair()
    g.step_cavity(5)
    o.step_cavity(5)
    p1 = tmp_path / "oct1.bin"
    g.write_snapshot(p1, step=5)
    raw = p1.read_bytes()
    assert raw[:8] == b"OCTSNAP1"
    version, levels, step, ng = struct.unpack("<IIQI", raw[8:28])
    assert (version, levels, step, ng) == (1, 3, 5, 5)
    dims = [struct.unpack("<QQ", raw[28 + 16 * i:44 + 16 * i]) for i in range(ng)]
    info = g.info()
    assert dims == [(info["nx"][i], info["ny"][i]) for i in range(5)]
    # restart another solver of the same layout; equals the oracle's set_from_snapshot
    g2, o2 = octree_pair(seed=9)
    g2.restart_from_snapshot(p1)
    o2.restart_from(o)
    assert g2.time_step == 0
    for lvl in range(5):
        a, b = g2.level(lvl, pops=True), o2.level(lvl, pops=True)
        for k in ("rho", "ux", "uy", "temp", "f", "g"):
            np.testing.assert_array_equal(a[k], b[k])
    # byte-identical round trip
    p2 = tmp_path / "oct2.bin"
    g2.write_snapshot(p2, step=5)
    assert p2.read_bytes() == raw
    g2.step_cavity(7)
    o2.step_cavity(7)
    for lvl in range(5):
        np.testing.assert_array_equal(g2.level(lvl)["temp"], o2.level(lvl)["temp"])


def test_octree_restart_layout_mismatch_is_error(tmp_path):
    """src/octree/tests.rs:950-965."""
    g, _ = octree_pair()
    g.step_cavity(2)
    p = tmp_path / "o.bin"
    g.write_snapshot(p)
    other, _ = octree_pair(bl=6)
    with pytest.raises(L.CavError) as e:
        other.restart_from_snapshot(p)
    assert e.value.code == L.CAV_ERR_ARG
    assert "layout" in str(e.value)
    two, _ = octree_pair(levels=2)
    with pytest.raises(L.CavError):
        two.restart_from_snapshot(p)
