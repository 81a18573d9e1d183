"""Generate the golden fixtures in this directory from the reference's own
CPU build (oracle/_ref, made by ``sh oracle/ref/build.sh``).

Each fixture holds the synthetic input state and the reference's output
arrays at a few points of the run, with one OpenMP thread (the reference's
Langevin noise stream depends on the thread count).  Run from the repo root:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refjob as rj  # noqa: E402
from spilady_b200.lattice import initial_state  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

ATOM_KEEP = ["rx", "ry", "rz", "px", "py", "pz", "fx", "fy", "fz", "sx", "sy",
             "sz", "Hx", "Hy", "Hz", "HLx", "HLy", "HLz", "rho", "pe", "ke",
             "me", "me0", "sum_Jij_sj"]

CASES = {
    # name: (mode, ncell, seed, tilt, steps per dump, number of dumps)
    "nve_6": ("nve", 6, 1, 0.05, 1, 3),
    "lang_6": ("lang", 6, 2, 0.3, 1, 3),
    "langte_6": ("langte", 6, 3, 0.35, 1, 3),
    "nve_16": ("nve", 16, 4, 0.05, 100, 1),
}


def make(name):
    mode, ncell, seed, tilt, every, ndump = CASES[name]
    params, r, p, s = initial_state(ncell, seed=seed, tilt=tilt)
    ops = [(rj.OP_DUMP, 0)]
    for _ in range(ndump):
        ops += [(rj.OP_CORE, every), (rj.OP_DUMP, 0)]
    dumps = rj.run(mode, params, r, p, s, ops=ops, threads=1)
    out = {"r0": r, "p0": p, "s0": s, "box": np.array(params["box"]),
           "step": params["step"], "mode": mode, "every": every,
           "ngroups": dumps[0].ngroups,
           "groups": np.concatenate([[len(g)] + list(g) for g in dumps[0].groups])}
    cols = [rj.ATOM_FIELDS.index(k) for k in ATOM_KEEP]
    out["atom_fields"] = np.array(ATOM_KEEP)
    out["atoms"] = np.stack([d.atoms[:, cols] for d in dumps])
    out["cells"] = np.stack([d.cells for d in dumps])
    out["cell_fields"] = np.array(rj.CELL_FIELDS)
    out["lists"] = np.stack([d.lists for d in dumps])
    out["cell_of"] = np.stack([d.a("cell").astype(np.int32) for d in dumps])
    if name == "nve_16":   # large case: keep only what the parity tests read
        keep = [ATOM_KEEP.index(k) for k in ("rx", "ry", "rz", "px", "py", "pz",
                                             "fx", "fy", "fz", "sx", "sy", "sz",
                                             "rho", "pe", "ke", "me", "me0")]
        out["atoms"] = out["atoms"][:, :, keep]
        out["atom_fields"] = out["atom_fields"][keep]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, mode, "atoms", r.shape[0], "groups", dumps[0].ngroups)


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        make(n)
