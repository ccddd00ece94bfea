"""The checkpoint format of ccs_checkpoint_save / ccs_checkpoint_load, read and written without a GPU.

A checkpoint holds a run's whole state at a step whose successor rebuilds
everything derived from it (the contact grid, the mesh, the pairwise pass), so
a restored run continues as the saved one would.  Layout (little-endian): the
144-byte header `ccs_checkpoint_header`; the run scalars (`ccs_sim`); pos4,
vel4, aux4 (float32 x 4 per particle), q, mat (float32), home4 (float32 x 4);
the loose list (int32 x ppCount); the caller's own bytes.  The checksum is the
CRC-32 of zlib (IEEE 802.3 polynomial) over everything after the header.  The
reference has no such format (its runTo replays a run from the build,
index.html:592-600); the snapshots the learned correction trains on and long
runs need one.
"""
import ctypes as C
import os
import zlib

import numpy as np

from . import _lib as L

MAGIC = b"CCSCKPT1"
VERSION = 1


class Header(C.Structure):
    _fields_ = [("magic", C.c_char * 8), ("version", C.c_uint32), ("headerBytes", C.c_uint32),
                ("simBytes", C.c_uint32), ("flags", C.c_uint32), ("N", C.c_int32), ("meshEvery", C.c_int32),
                ("ppCount", C.c_int32), ("ppLoose", C.c_int32), ("field", C.c_double * 6),
                ("monoA", C.c_float * 4), ("monoB", C.c_float * 4), ("extraBytes", C.c_uint64),
                ("payloadBytes", C.c_uint64), ("checksum", C.c_uint64)]


def _sizes(N, pp, extra):
    return [("sim", C.sizeof(L.Sim)), ("pos", 16 * N), ("vel", 16 * N), ("aux", 16 * N), ("q", 4 * N),
            ("mat", 4 * N), ("home", 16 * N), ("pp_list", 4 * pp), ("extra", extra)]


def read(data, verify=True):
    """Parse a checkpoint (bytes, or a path): a dict of the header's fields, `sim` (a ccs_sim struct), the
    state arrays, `pp_list` and `extra` (bytes).  Raises ValueError on a malformed or corrupted one."""
    if isinstance(data, (str, os.PathLike)):
        with open(data, "rb") as f:
            data = f.read()
    data = bytes(data)
    hb = C.sizeof(Header)
    if len(data) < hb:
        raise ValueError("checkpoint: shorter than its header")
    h = Header.from_buffer_copy(data[:hb])
    if h.magic != MAGIC or h.version != VERSION or h.headerBytes != hb or h.simBytes != C.sizeof(L.Sim):
        raise ValueError("checkpoint: not a version-1 checkpoint of this layout")
    sizes = _sizes(h.N, h.ppCount, h.extraBytes)
    if h.N <= 0 or h.ppCount < 0 or h.payloadBytes != sum(s for _, s in sizes) or len(data) < hb + h.payloadBytes:
        raise ValueError("checkpoint: sizes do not add up")
    payload = data[hb:hb + h.payloadBytes]
    if verify and zlib.crc32(payload) != h.checksum:
        raise ValueError("checkpoint: checksum mismatch")
    out = {f[0]: getattr(h, f[0]) for f in Header._fields_}
    out["field"] = list(h.field)
    out["monoA"] = np.array(h.monoA, np.float32)
    out["monoB"] = np.array(h.monoB, np.float32)
    at = 0
    for name, n in sizes:
        chunk = payload[at:at + n]
        at += n
        if name == "sim":
            out[name] = L.Sim.from_buffer_copy(chunk)
        elif name == "pp_list":
            out[name] = np.frombuffer(chunk, np.int32).copy()
        elif name == "extra":
            out[name] = chunk
        elif name in ("q", "mat"):
            out[name] = np.frombuffer(chunk, np.float32).copy()
        else:
            out[name] = np.frombuffer(chunk, np.float32).reshape(-1, 4).copy()
    return out


def write(sim, pos, vel, aux, q, mat, home=None, pp_list=(), pp_loose=0, mesh_every=8, field=None,
          mono_a=(0, 0, 0, 0), mono_b=(0, 0, 0, 0), extra=b""):
    """Make a checkpoint from host arrays (a state built or stepped elsewhere, e.g. by the oracle).
    field = (g[3], frozen, invM, cpIron) for the field step.  Returns bytes for ccs_checkpoint_load."""
    N = int(sim.N)
    pva = [np.ascontiguousarray(a, np.float32) for a in (pos, vel, aux)]
    qa, ma = np.ascontiguousarray(q, np.float32), np.ascontiguousarray(mat, np.float32)
    ho = np.zeros((N, 4), np.float32) if home is None else np.ascontiguousarray(home, np.float32)
    pl = np.ascontiguousarray(pp_list, np.int32)
    if any(a.shape != (N, 4) for a in pva + [ho]) or qa.shape != (N,) or ma.shape != (N,):
        raise ValueError("checkpoint: pos, vel, aux, home must be N x 4 and q, mat N")
    payload = b"".join([bytes(sim)] + [a.tobytes() for a in pva + [qa, ma, ho, pl]] + [bytes(extra)])
    h = Header()
    h.magic = MAGIC
    h.version, h.headerBytes, h.simBytes = VERSION, C.sizeof(Header), C.sizeof(L.Sim)
    h.flags = 2 if field is not None else 0
    h.N, h.meshEvery, h.ppCount, h.ppLoose = N, int(mesh_every), len(pl), int(pp_loose)
    g, frozen, inv_m, cp_iron = field if field is not None else ((0.0, 0.0, 0.0), -1.0, 1.0, 1.0)
    for k in range(3):
        h.field[k] = float(g[k])
    h.field[3], h.field[4], h.field[5] = float(frozen), float(inv_m), float(cp_iron)
    for k in range(4):
        h.monoA[k], h.monoB[k] = float(mono_a[k]), float(mono_b[k])
    h.extraBytes, h.payloadBytes = len(extra), len(payload)
    h.checksum = zlib.crc32(payload)
    return bytes(h) + payload
