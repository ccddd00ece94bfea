"""Checkpoint and restore on the GPU (ccs_checkpoint_save / ccs_checkpoint_load).

A run saved mid-impact -- full phase, a loose list, two monopoles -- and
restored into a fresh engine holds the same state bit for bit, and both then
take the same step: the pair sets are equal and the state agrees to the 1e-5
of its scale that float-atomic deposits leave.  The library's file parses
with the Python reader (its CRC is zlib's), a file written by the Python
writer loads, the field step's settings survive, and a save off a block
boundary or a corrupted file is refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scaled_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return 0.0 if s == 0 else float(np.abs(a - b).max() / s)


def same_state(x, y):
    return all(np.array_equal(x[k], y[k]) for k in ("pos", "vel", "aux", "q", "mat"))


def test_impact_checkpoint_continues(ccmod, tmp_path):
    from cosmic_collisions_b200 import checkpoint as ck, configs
    a, b = ccmod.NBody(0), ccmod.NBody(0)
    try:
        a.build(configs.small_impact_opt(16384))
        a.run_to(1.0)
        if a.sim.stepNo % 8:
            a.steps(8 - a.sim.stepNo % 8)
        a.sync()
        path = tmp_path / "run.ckpt"
        data = a.save(path)
        r = ck.read(path)                                   # the library's CRC is zlib's
        sa = a.read_state()
        assert np.array_equal(r["pos"], sa["pos"]) and np.array_equal(r["q"], sa["q"])
        assert r["ppCount"] == a.pp["count"] > 0
        b.load(data)
        assert bytes(b.sim) == bytes(a.sim)
        assert same_state(b.read_state(), sa)
        assert b.ref == a.ref and b.analyses == a.analyses and b.pp == a.pp
        assert bytes(b.report) == bytes(a.report)
        a.step(False, False)                                # a mesh step: grid, mesh, P3M, contacts
        b.step(False, False)
        x, y = a.read_state(), b.read_state()
        assert np.array_equal(x["aux"][:, 3], y["aux"][:, 3])
        for k in ("pos", "vel"):
            assert scaled_err(y[k][:, :3], x[k][:, :3]) < 1e-5, k
        assert scaled_err(y["aux"][:, :3], x["aux"][:, :3]) < 1e-5
        # off a block boundary: refused
        with pytest.raises(ccmod.CCSError, match="checkpoint"):
            a.save()
        bad = bytearray(data)
        bad[-5] ^= 0x40
        with pytest.raises(ccmod.CCSError, match="checksum"):
            b.load(bytes(bad))
    finally:
        a.close()
        b.close()


def test_python_written_checkpoint_loads_with_the_field_step(ccmod):
    from cosmic_collisions_b200 import checkpoint as ck, configs as cf
    sim, pos, vel, mat = cf.crater_patch(16384)
    q = np.zeros(len(pos), np.float32)
    data = ck.write(sim, pos, vel, np.zeros_like(pos), q, mat, field=(cf.CRATER_G, cf.MAT_FROZEN, 1.0, 1.0))
    a, b = ccmod.NBody(0), ccmod.NBody(0)
    try:
        a.load(data)
        u = a.uniforms()
        assert u.field == 1.0 and u.frozen == 0.0 and u.invM == 1.0
        assert np.array_equal(a.read_state()["pos"], pos)
        a.step(True, False)
        a.step(False, False)                                # stepNo 2: a field-step boundary
        b.load(a.save())
        a.step(False, False)
        b.step(False, False)
        x, y = a.read_state(), b.read_state()
        assert np.array_equal(x["aux"], y["aux"])          # the field, and the same pair counts
        for k in ("pos", "vel"):
            assert scaled_err(y[k][:, :3], x[k][:, :3]) < 1e-5, k
    finally:
        a.close()
        b.close()
