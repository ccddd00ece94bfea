"""Writes tests/golden/oracle_golden.json: regression fixtures of the CPU oracle.

The reference ships no golden vectors and cannot run here (WebGL2 + JavaScript),
so these fixtures pin the oracle against itself: any change to the oracle's
restatement that moves a seed's random stream, the body builder, the pair
table, the seat table or one scheduled step shows up as a mismatch.  They are
NOT reference outputs.  Regenerate only after a deliberate oracle change:

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden():
    from oracle import oracle as O
    O.build()
    out = {"mulberry": {str(s): O.mulberry_seq(s, 8).tolist() for s in (1234567, 99, 777)},
           "maclaurin": {str(f): O.maclaurin(f) for f in (0.18, 0.2, 0.55)}}
    f, p = O.pair_table()
    out["pair_table"] = {"f": f.tolist(), "p": p.tolist()}
    sim, pos, vel, mat, home = O.build_run(O.make_opt(16384))
    out["build_16384"] = {"pos": sha(pos), "mat": sha(mat), "home": sha(home), "a": sim.a, "dt": sim.dt,
                          "n1": sim.n1, "n2": sim.n2, "t": sim.t, "k": sim.k, "c": sim.c}
    u = O.make_uni(sim)
    out["seats_16384"] = sha(O.slots(u, pos))
    e = O.Engine(sim, pos, vel, mat)
    e.step(True, False)
    out["step0_16384"] = {"pos": sha(e.buf("pos")), "vel": sha(e.buf("vel")), "aux": sha(e.buf("aux")),
                          "fineA": sha(e.buf("fineA")), "forceA": sha(e.buf("forceA"))}
    return out


if __name__ == "__main__":
    path = os.path.join(HERE, "oracle_golden.json")
    with open(path, "w") as fh:
        json.dump(golden(), fh, indent=1, sort_keys=True)
    print(path)
