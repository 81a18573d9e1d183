"""Generate the golden fixtures in this directory from the reference's own
CPU build (oracle/_ref, made by ``sh oracle/ref/build.sh``).

Each fixture holds the synthetic input state and the reference's output
arrays at a few points of the run, with one OpenMP thread (the reference's
Langevin noise stream depends on the thread count).  Run from the repo root:

    python tests/golden/make_golden.py            # the trajectory fixtures
    python tests/golden/make_golden.py adjoint    # the reference's FD gradient
    python tests/golden/make_golden.py long       # the reference's long runs
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


def make_adjoint_fd(path=os.path.join(HERE, "adjoint_ref_fd.npz"), K=10, threads=16):
    """The reference's own gradient of L = sum |f|^2 + |Heff_H|^2 in the 36
    potential parameters, by FP64 central differences (h = 1e-6 of each, 1e-6
    for a zero one) of its CPU code: the "param" build reads the parameters
    from theta.in.  One configuration (bcc Fe 8^3 cells, positions +N(0, 0.05
    A), spin tilt 0.2 rad), and after K NVE steps of 1 fs.  Heff_H is the
    field check_temperature recomputes for every atom."""
    from concurrent.futures import ThreadPoolExecutor
    params, r, p, s = initial_state(8, seed=21, tilt=0.2, temperature=300.0, pos_sigma=0.05)
    theta = np.array(DEFAULT_THETA)
    h = np.where(theta != 0.0, 1e-6 * np.abs(theta), 1e-6)

    def loss(th, steps):
        ops = ([(rj.OP_CORE, steps)] if steps else []) + [(rj.OP_CHECK, steps - 1),
                                                          (rj.OP_DUMP, 0)]
        d = rj.run("param", params, r, p, s, ops=ops,
                   inputs={"theta.in": " ".join("%.17g" % x for x in th)})[-1]
        return float((d.vec("f") ** 2).sum() + (d.vec("H") ** 2).sum())

    jobs = []
    for steps in (0, K):
        for k in range(len(theta)):
            for sgn in (1.0, -1.0):
                t = theta.copy()
                t[k] += sgn * h[k]
                jobs.append((t, steps))
    with ThreadPoolExecutor(threads) as ex:
        vals = list(ex.map(lambda j: loss(*j), jobs))
    v = np.array(vals).reshape(2, len(theta), 2)
    fd = (v[:, :, 0] - v[:, :, 1]) / (2 * h)
    np.savez_compressed(path, theta=theta, h=h, K=K, dL_config=fd[0], dL_traj=fd[1],
                        L_config=loss(theta, 0), L_traj=loss(theta, K))
    print("adjoint_ref_fd", path)


def read_lines(text):
    return np.array([[float(x) for x in l.split()] for l in text.splitlines() if l.strip()])


def make_long_runs(path=os.path.join(HERE, "long_runs_ref.npz"), threads=16):
    """The reference's long runs, for the statistical checks: its print-out
    lines every step (check.cpp with interval_of_print_out 1).
      NVE: bcc Fe 16^3 cells (8,192 atoms), spins tilted 0.05 rad, 300 K
           momenta, dt 1 fs, 1,000 steps: the total energy per atom (pe + ke +
           me + me0), whose drift the engine's may not exceed;
      Langevin spin + lattice at 300 K: 10^3 cells (2,000 atoms), 3,000 steps:
           Tl, Ts_R, Ts_L and |<m>|, whose equilibrium averages the engine's
           must match within their error bars (the noise streams differ).
    OpenMP threads change only the rounding of NVE and the reference's own
    noise stream of the Langevin run."""
    never = [(rj.OP_CONFIG_INTERVAL, 10**9)]
    params, r, p, s = initial_state(16, seed=4, tilt=0.05, temperature=300.0)
    _, t = rj.run("nve", params, r, p, s, ops=never + [(rj.OP_STEP, 1000)], threads=threads,
                  files=True)
    enr = read_lines(t["enr-ref.dat"])
    e_nve = enr[:, 2] + enr[:, 3] + enr[:, 4] + enr[:, 5]
    params, r, p, s = initial_state(10, seed=7, tilt=0.05, temperature=300.0)
    _, t = rj.run("lang", params, r, p, s, ops=never + [(rj.OP_STEP, 3000)], threads=threads,
                  files=True)
    tmp = read_lines(t["tmp-ref.dat"])
    spn = read_lines(t["spn-ref.dat"])
    np.savez_compressed(path, nve_E=e_nve, nve_steps=1000,
                        lang_Tl=tmp[:, 2], lang_TsR=tmp[:, 3], lang_TsL=tmp[:, 4],
                        lang_m=spn[:, 9], lang_steps=3000)
    print("long_runs_ref", path)


# the potential's 36 constants in sld_adjoint_theta_default's order (DD05.cpp,
# JijFe.cpp): F a, b; f coefficients, knots; phi coefficients, knots; J A, rc;
# Landau A, B, C, D
DEFAULT_THETA = [
    4.100199340884814, 1.565647547483517,
    0.9332056681088162, -1.162558782567700, -0.3502026949249225, 0.4287820835430028,
    4.907925057809273, -5.307049068415304,
    3.0, 2.8666666666666666, 2.7333333333333333, 2.6, 2.4, 2.3,
    -0.1960674387419232, 0.3687525935422963, -1.505333614924853, 4.948907078156191,
    -4.894613262753399, 3.468897724782442, -1.792218099820337, 80.22069592246987,
    4.1, 3.8, 3.5, 3.2, 2.9, 2.6, 2.4, 2.3,
    0.870, 3.75,
    -0.744824, 0.345295, -0.00790205, 0.0,
]


if __name__ == "__main__":
    args = sys.argv[1:]
    if args == ["adjoint"]:
        make_adjoint_fd()
    elif args == ["long"]:
        make_long_runs()
    else:
        for n in (args or CASES):
            make(n)
