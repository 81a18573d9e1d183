"""Test infrastructure: ctypes wrapper of the C restatement (the oracle).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
The library is built by ``make -C oracle`` into ``oracle/_build``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsld_oracle.so")

RNG_MWC, RNG_PHILOX = 0, 1


class Params(C.Structure):
    _fields_ = [
        ("box", C.c_double * 6), ("step", C.c_double),
        ("temperature", C.c_double), ("atmass", C.c_double),
        ("gamma_L_over_mass", C.c_double), ("gamma_S_HL", C.c_double),
        ("rcut_pot", C.c_double), ("rcut_mag", C.c_double),
        ("rcut_max", C.c_double), ("min_length_link_cell", C.c_double),
        ("kappa_e", C.c_double), ("random_seed", C.c_int),
        ("spinlang", C.c_int), ("lattlang", C.c_int), ("eltemp", C.c_int),
        ("localcolmot", C.c_int), ("renormalize", C.c_int), ("rng", C.c_int),
        ("te_mesh", C.c_int), ("te_nloop", C.c_int),
        ("interval_of_print_out", C.c_int),
        ("quantum", C.c_int), ("msteps_quantum", C.c_int), ("nfrequency_quantum", C.c_int),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(C.c_double)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(Params), C.c_int, P, P, P, P]
        L.orc_destroy.argtypes = [C.c_void_p]
        for name in ("orc_links", "orc_rho", "orc_force", "orc_temperature"):
            getattr(L, name).argtypes = [C.c_void_p]
        for name in ("orc_core_ds", "orc_core_dp", "orc_core_dr", "orc_core_dte"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_double]
        L.orc_run.argtypes = [C.c_void_p, C.c_int]
        L.orc_averages.argtypes = [C.c_void_p, P]
        L.orc_quantum_filter.argtypes = [C.c_void_p, P, C.c_int]
        for name in ("orc_natom", "orc_ncells", "orc_nte", "orc_ngroups"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = C.c_int
        L.orc_get.argtypes = [C.c_void_p, C.c_char_p, P]
        L.orc_get.restype = C.c_int
        L.orc_lists.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.orc_total_time.argtypes = [C.c_void_p]
        L.orc_total_time.restype = C.c_double
        L.orc_philox_normals.argtypes = [C.c_uint, C.c_uint, C.c_uint,
                                         C.c_ulonglong, P]
        L.orc_philox4x32.argtypes = [C.POINTER(C.c_uint)] * 3
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_params(params, *, spinlang=False, lattlang=False, eltemp=False,
                localcolmot=False, renormalize=False, rng=RNG_PHILOX,
                te_mesh=0, te_nloop=50, quantum=False, msteps_quantum=50,
                nfrequency_quantum=150):
    P = Params()
    P.box[:] = list(params["box"])
    for k in ("step", "temperature", "atmass", "gamma_L_over_mass",
              "gamma_S_HL", "rcut_pot", "rcut_mag", "rcut_max",
              "min_length_link_cell", "kappa_e"):
        setattr(P, k, float(params[k]))
    P.random_seed = int(params["random_seed"])
    P.spinlang, P.lattlang, P.eltemp = int(spinlang), int(lattlang), int(eltemp)
    P.localcolmot, P.renormalize = int(localcolmot), int(renormalize)
    P.rng, P.te_mesh, P.te_nloop = rng, te_mesh, te_nloop
    P.interval_of_print_out = 1
    P.quantum, P.msteps_quantum = int(quantum), int(msteps_quantum)
    P.nfrequency_quantum = int(nfrequency_quantum)
    return P


class System:
    """One oracle system; methods carry the reference's function names."""

    def __init__(self, params, r, p, s, te=None, **switches):
        self.L = lib()
        self.P = make_params(params, **switches)
        r = np.ascontiguousarray(r, np.float64)
        p = np.ascontiguousarray(p, np.float64)
        s = np.ascontiguousarray(s, np.float64)
        te_arr = None if te is None else np.ascontiguousarray(te, np.float64)
        h = self.L.orc_create(C.byref(self.P), r.shape[0], _dp(r), _dp(p),
                              _dp(s), None if te_arr is None else _dp(te_arr))
        if not h:
            raise ValueError("oracle rejected the input")
        self.h = C.c_void_p(h)
        self.natom = r.shape[0]

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def links(self): self.L.orc_links(self.h)
    def calculate_rho(self): self.L.orc_rho(self.h)
    def calculate_force_energy(self): self.L.orc_force(self.h)
    def calculate_temperature(self): self.L.orc_temperature(self.h)
    def core_ds(self, dt): self.L.orc_core_ds(self.h, dt)
    def core_dp(self, dt): self.L.orc_core_dp(self.h, dt)
    def core_dr(self, dt): self.L.orc_core_dr(self.h, dt)
    def core_dTe(self, dt): self.L.orc_core_dte(self.h, dt)
    def run(self, nsteps): self.L.orc_run(self.h, nsteps)

    @property
    def ncells(self): return self.L.orc_ncells(self.h)

    @property
    def nte(self): return self.L.orc_nte(self.h)

    @property
    def ngroups(self): return self.L.orc_ngroups(self.h)

    def get(self, name):
        per_te = name in ("Te", "Ee", "Tl", "Ts_R", "Ts_L", "Gel", "Ges", "count")
        width = {"r": 3, "p": 3, "f": 3, "s": 3, "H": 3, "HL": 3, "stress": 6}.get(name, 1)
        n = (self.nte if per_te else self.natom) * width
        out = np.empty(n, np.float64)
        got = self.L.orc_get(self.h, name.encode(), _dp(out))
        if got < 0:
            raise KeyError(name)
        return out.reshape(-1, width) if width > 1 else out

    def lists(self):
        out = np.empty(self.natom, np.int32)
        self.L.orc_lists(self.h, out.ctypes.data_as(C.POINTER(C.c_int)))
        return out

    def averages(self):
        out = np.empty(10, np.float64)
        self.L.orc_averages(self.h, _dp(out))
        return dict(zip(["pe", "ke", "me", "me0", "Ee", "Tl", "Te", "sx", "sy", "sz"], out))

    def quantum_filter(self):
        out = np.zeros(100000)
        n = self.L.orc_quantum_filter(self.h, _dp(out), len(out))
        return out[:n]


def philox4x32(ctr, key):
    c = (C.c_uint * 4)(*ctr)
    k = (C.c_uint * 2)(*key)
    o = (C.c_uint * 4)()
    lib().orc_philox4x32(c, k, o)
    return list(o)


def philox_normals(seed, replica, atom, epoch):
    out = np.empty(3, np.float64)
    lib().orc_philox_normals(seed, replica, atom, epoch, _dp(out))
    return out
