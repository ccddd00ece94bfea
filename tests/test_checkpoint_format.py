"""The checkpoint format on the CPU: the Python reader and writer against each other, corruption and
truncation refused, and the header laid out as include/ccstep.h declares it (compiled with gcc)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def sample(N=4096, field=True):
    from cosmic_collisions_b200 import checkpoint as ck, configs
    s, p, v, m = configs.crater_patch(N)
    rng = np.random.default_rng(5)
    aux = rng.normal(size=(N, 4)).astype(np.float32)
    q = rng.uniform(0, 1, N).astype(np.float32)
    data = ck.write(s, p, v, aux, q, m, pp_list=np.arange(0, N, 97), pp_loose=123, mesh_every=8,
                    field=(configs.CRATER_G, configs.MAT_FROZEN, 1.0, 1.0) if field else None,
                    mono_a=(1, 2, 3, 4), extra=b'{"x": 1}')
    return data, (s, p, v, aux, q, m)


def test_roundtrip():
    from cosmic_collisions_b200 import checkpoint as ck
    data, (s, p, v, aux, q, m) = sample()
    r = ck.read(data)
    assert bytes(r["sim"]) == bytes(s)
    for name, a in (("pos", p), ("vel", v), ("aux", aux), ("q", q), ("mat", m)):
        assert np.array_equal(r[name], a), name
    assert not r["home"].any()
    assert r["ppCount"] == len(r["pp_list"]) and r["ppLoose"] == 123 and r["flags"] == 2
    assert list(r["monoA"]) == [1, 2, 3, 4] and r["extra"] == b'{"x": 1}'
    assert r["field"][3] == 0.0 and r["field"][1] == pytest.approx(-0.0981)


def test_corruption_and_truncation_are_refused():
    from cosmic_collisions_b200 import checkpoint as ck
    data, _ = sample(field=False)
    bad = bytearray(data)
    bad[C.sizeof(ck.Header) + 1000] ^= 1
    with pytest.raises(ValueError, match="checksum"):
        ck.read(bytes(bad))
    with pytest.raises(ValueError, match="sizes"):
        ck.read(data[:-1])
    with pytest.raises(ValueError, match="version-1"):
        ck.read(b"XXXXXXXX" + data[8:])
    with pytest.raises(ValueError, match="shorter"):
        ck.read(data[:100])


def test_header_layout_matches_the_c_header(tmp_path):
    from cosmic_collisions_b200 import _lib as L, checkpoint as ck
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ccstep.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu\\n", sizeof(ccs_checkpoint_header), '
                   'offsetof(ccs_checkpoint_header, field), offsetof(ccs_checkpoint_header, checksum), '
                   'sizeof(ccs_sim)); return 0; }\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [C.sizeof(ck.Header), ck.Header.field.offset, ck.Header.checksum.offset, C.sizeof(L.Sim)]
