"""Test infrastructure: run the reference's own CPU build (oracle/_ref) on a
synthetic state and read back its per-atom / per-cell arrays.

The binaries are made by ``oracle/ref/build.sh`` from the reference sources;
the job/dump layout is documented in ``oracle/ref/harness.cpp``.  Only the
tests, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg use this.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

OP_DUMP, OP_LINKS, OP_RHO, OP_FORCE, OP_DS, OP_DP, OP_DR, OP_DTE, OP_TEMP, \
    OP_CORE, OP_CHECK_ENERGY, OP_STEP, OP_CONFIG_INTERVAL, OP_WRITE_CONFIG, \
    OP_CHECK, OP_QINIT, OP_QFILTER, OP_STATS = range(18)
# OP_SET + k sets an input variable of the baro / dtstep builds (harness.cpp)
OP_SET = 100
SET_VARS = {"pressure": 0, "baro_damping_time": 1, "stress_xx": 2, "stress_yx": 3,
            "stress_yy": 4, "stress_zx": 5, "stress_zy": 6, "stress_zz": 7,
            "interval_of_scale_pressure": 8, "interval_of_scale_stress": 9,
            "displace_limit": 10, "phi_limit": 11, "Msteps_quantum": 12,
            "Nfrequency_quantum": 13}


def set_ops(**values):
    """Ops that set the given input variables (names as in variables.in)."""
    return [(OP_SET + SET_VARS[k], float(v)) for k, v in values.items()]

ATOM_FIELDS = [
    "rx", "ry", "rz", "px", "py", "pz", "fx", "fy", "fz", "sx", "sy", "sz",
    "s0", "Hx", "Hy", "Hz", "HLx", "HLy", "HLz", "rho", "pe", "ke", "me",
    "me0", "vir", "st11", "st22", "st33", "st12", "st23", "st31",
    "sum_Jij_sj", "local_volume", "cell",
]
CELL_FIELDS = ["count", "Te", "Ee", "Tl", "Ts_R", "Ts_L", "Gel", "Ges"]


def binary(mode: str) -> str:
    return os.path.join(REF_DIR, f"spilady_ref_{mode}")


def available(mode: str = "nve") -> bool:
    return os.access(binary(mode), os.X_OK)


@dataclass
class Dump:
    natom: int
    ncells: int
    ngroups: int
    total_time: float
    wall: float
    atoms: np.ndarray          # (natom, len(ATOM_FIELDS))
    cells: np.ndarray          # (ncells, len(CELL_FIELDS))
    lists: np.ndarray          # concatenated cell member lists, head->tail
    groups: list = field(default_factory=list)  # list of int arrays (cells)

    def a(self, name):
        return self.atoms[:, ATOM_FIELDS.index(name)]

    def vec(self, prefix):
        names = {"r": ("rx", "ry", "rz"), "p": ("px", "py", "pz"),
                 "f": ("fx", "fy", "fz"), "s": ("sx", "sy", "sz"),
                 "H": ("Hx", "Hy", "Hz"), "HL": ("HLx", "HLy", "HLz")}[prefix]
        return np.stack([self.a(n) for n in names], axis=1)

    def c(self, name):
        return self.cells[:, CELL_FIELDS.index(name)]


def write_job(path, params, r, p, s, te=None, ops=(), threads=1):
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    n = r.shape[0]
    p = np.ascontiguousarray(p, dtype=np.float64).reshape(n, 3)
    s = np.ascontiguousarray(s, dtype=np.float64).reshape(n, 3)
    te = np.zeros(0) if te is None else np.ascontiguousarray(te, np.float64)
    box = list(params["box"])
    with open(path, "wb") as f:
        f.write(struct.pack("<5i", 0x534C4431, n, threads, te.size, len(ops)))
        f.write(struct.pack(
            "<17d", *box, params["step"], params["temperature"],
            params["atmass"], params["gamma_L_over_mass"],
            params["gamma_S_HL"], params["rcut_pot"], params["rcut_mag"],
            params["rcut_max"], params["min_length_link_cell"],
            params["kappa_e"], 0.0))
        f.write(struct.pack("<i", int(params["random_seed"])))
        f.write(r.tobytes())
        f.write(p.tobytes())
        f.write(s.tobytes())
        f.write(te.tobytes())
        for code, arg in ops:
            f.write(struct.pack("<id", code, float(arg)))


def read_dumps(path):
    data = open(path, "rb").read()
    off = 0
    out = []
    while off < len(data):
        tag, natom, ncells, ngroups = struct.unpack_from("<4i", data, off)
        off += 16
        assert tag == 0x44554D50, "bad dump tag"
        total_time, wall = struct.unpack_from("<2d", data, off)
        off += 16
        na = natom * len(ATOM_FIELDS)
        atoms = np.frombuffer(data, np.float64, na, off).reshape(natom, len(ATOM_FIELDS))
        off += 8 * na
        nc = ncells * len(CELL_FIELDS)
        cells = np.frombuffer(data, np.float64, nc, off).reshape(ncells, len(CELL_FIELDS))
        off += 8 * nc
        (nl,) = struct.unpack_from("<i", data, off)
        off += 4
        lists = np.frombuffer(data, np.int32, nl, off)
        off += 4 * nl
        (ng,) = struct.unpack_from("<i", data, off)
        off += 4
        g = np.frombuffer(data, np.int32, ng, off)
        off += 4 * ng
        groups, k = [], 0
        while k < ng:
            m = int(g[k])
            groups.append(np.array(g[k + 1:k + 1 + m]))
            k += 1 + m
        out.append(Dump(natom, ncells, ngroups, total_time, wall,
                        atoms.copy(), cells.copy(), lists.copy(), groups))
    return out


def run(mode, params, r, p, s, te=None, ops=(), threads=1, timeout=3600,
        files=False, inputs=None):
    """Run the reference harness in a scratch directory; return the dumps,
    and with ``files`` also a dict of the ``.dat`` files the reference wrote
    there (name -> text: its enr-/tmp-/.../con-/cel- output).  ``inputs``
    (name -> text) are written into the working directory first, e.g. the
    extfield.in / extforce.in files the extf build reads."""
    exe = binary(mode)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(f"{exe} missing: run sh oracle/ref/build.sh")
    with tempfile.TemporaryDirectory(prefix="sldref_") as tmp:
        job = os.path.join(tmp, "job.bin")
        out = os.path.join(tmp, "out.bin")
        write_job(job, params, r, p, s, te, ops, threads)
        for name, text in (inputs or {}).items():
            with open(os.path.join(tmp, name), "w") as fh:
                fh.write(text)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        res = subprocess.run([exe, job, out], cwd=tmp, env=env,
                             stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                             timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"reference harness failed ({res.returncode}):"
                               f" {res.stderr.decode()[-2000:]}")
        dumps = read_dumps(out)
        if not files:
            return dumps
        texts = {}
        for name in sorted(os.listdir(tmp)):
            if name.endswith(".dat") and name not in (inputs or {}):
                with open(os.path.join(tmp, name)) as fh:
                    texts[name] = fh.read()
        return dumps, texts
