"""Python binding of the C ABI in include/sld.h.

``Engine`` mirrors the reference's step functions by name (links,
calculate_rho, calculate_force_energy, core_ds, core_dp, core_dr, core_dTe,
calculate_temperature, core) over one device context.  The CUDA library is
required: importing works without it, but creating an Engine fails loudly
when ``spilady_b200/_lib/libsld_b200.so`` is missing or no GPU is present.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsld_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "sld.h")

FP64, SPLIT, FP64_ANALYTIC = 0, 1, 2
# control.h's Hamiltonian switch
SLDHL, SLDH, MD, SDH, SDHL = 0, 1, 2, 3, 4
HAMILTONIANS = {"SLDHL": SLDHL, "SLDH": SLDH, "MD": MD, "SDH": SDH, "SDHL": SDHL}

ERRORS = {
    -1: "SLD_ERR_ARG", -2: "SLD_ERR_CUDA", -3: "SLD_ERR_GEOMETRY",
    -4: "SLD_ERR_CAPACITY", -5: "SLD_ERR_TABLE", -6: "SLD_ERR_NAN",
    -7: "SLD_ERR_IO", -8: "SLD_ERR_STATE", -9: "SLD_ERR_NOMEM",
    -10: "SLD_ERR_TIMEOUT",
}


class SldError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)}")


class Params(C.Structure):
    _fields_ = [
        ("box", C.c_double * 6), ("step", C.c_double),
        ("temperature", C.c_double), ("atmass", C.c_double),
        ("gamma_L_over_mass", C.c_double), ("gamma_S_HL", C.c_double),
        ("rcut_pot", C.c_double), ("rcut_mag", C.c_double),
        ("rcut_max", C.c_double), ("min_length_link_cell", C.c_double),
        ("kappa_e", C.c_double), ("random_seed", C.c_int),
        ("spinlang", C.c_int), ("lattlang", C.c_int), ("eltemp", C.c_int),
        ("localcolmot", C.c_int), ("renormalize_energy", C.c_int),
        ("te_mesh", C.c_int), ("te_nloop", C.c_int),
        ("interval_of_print_out", C.c_int), ("precision", C.c_int),
        ("device", C.c_int), ("replica", C.c_int),
        ("interval_of_config_out", C.c_int),
        ("pressure_control", C.c_int), ("stress_control", C.c_int),
        ("change_step", C.c_int), ("interval_of_scale_pressure", C.c_int),
        ("interval_of_scale_stress", C.c_int), ("pressure", C.c_double),
        ("stress", C.c_double * 6), ("baro_damping_time", C.c_double),
        ("displace_limit", C.c_double), ("phi_limit", C.c_double),
        ("quantum_noise", C.c_int), ("msteps_quantum", C.c_int),
        ("nfrequency_quantum", C.c_int),
        ("hamiltonian", C.c_int), ("gamma_S_H", C.c_double),
    ]


_lib = None


def lib():
    """Load the engine library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not built: run make -C spilady_b200/csrc")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.sld_params_default.argtypes = [C.POINTER(Params)]
        L.sld_read_variables.argtypes = [C.c_char_p, C.POINTER(Params)]
        L.sld_create.argtypes = [C.POINTER(vp), C.POINTER(Params), C.c_int, P, P, P, P]
        L.sld_create_from_config.argtypes = [C.POINTER(vp), C.POINTER(Params),
                                             C.c_char_p, C.c_char_p]
        L.sld_destroy.argtypes = [vp]
        L.sld_destroy.restype = None
        L.sld_set_state.argtypes = [vp, P, P, P]
        for n in ("sld_links", "sld_calculate_rho", "sld_calculate_force_energy",
                  "sld_calculate_temperature", "sld_sync"):
            getattr(L, n).argtypes = [vp]
        for n in ("sld_core_ds", "sld_core_dp", "sld_core_dr", "sld_core_dTe"):
            getattr(L, n).argtypes = [vp, C.c_double]
        L.sld_run.argtypes = [vp, C.c_int]
        L.sld_get.argtypes = [vp, C.c_char_p, P, C.c_long]
        L.sld_get.restype = C.c_long
        L.sld_get_cell_lists.argtypes = [vp, C.POINTER(C.c_int)]
        L.sld_averages.argtypes = [vp, P]
        L.sld_info.argtypes = [vp, C.POINTER(C.c_int)]
        L.sld_virial.argtypes = [vp, P]
        L.sld_total_time.argtypes = [vp, P]
        L.sld_last_run_ms.argtypes = [vp, P]
        L.sld_profile_step.argtypes = [vp, P]
        L.sld_step_kernel_count.argtypes = [vp, C.POINTER(C.c_int)]
        L.sld_batch_create.argtypes = [C.POINTER(vp), C.POINTER(vp), C.c_int]
        L.sld_batch_run.argtypes = [vp, C.c_int]
        L.sld_batch_last_run_ms.argtypes = [vp, P]
        L.sld_batch_destroy.argtypes = [vp]
        L.sld_batch_destroy.restype = None
        L.sld_check.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int]
        L.sld_scale.argtypes = [vp, C.c_int, P]
        L.sld_quantum_filter.argtypes = [vp, P, C.c_int]
        L.sld_autotune.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        for n in ("sld_set_external_field", "sld_set_external_force"):
            getattr(L, n).argtypes = [vp, P]
        for n in ("sld_read_external_field", "sld_read_external_force"):
            getattr(L, n).argtypes = [vp, C.c_char_p]
        L.sld_write_config.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int, C.c_int]
        L.sld_adjoint_theta_default.argtypes = [P]
        L.sld_adjoint_config.argtypes = [vp, P, P, P, P]
        L.sld_adjoint_trajectory.argtypes = [vp, P, C.c_int, C.c_int, P, P]
        L.sld_adjoint_jacobians.argtypes = [vp, P, P, P, P, P]
        L.sld_error_string.argtypes = [C.c_int]
        L.sld_error_string.restype = C.c_char_p
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(rc, where):
    if rc != 0:
        raise SldError(rc, where)


def make_params(params, *, spinlang=False, lattlang=False, eltemp=False,
                localcolmot=False, renormalize=False, te_mesh=0, te_nloop=50,
                precision=FP64, device=0, interval_of_print_out=1, replica=0,
                interval_of_config_out=1000, pressure_control=False,
                stress_control=False, change_step=False, hamiltonian=SLDHL,
                quantum_noise=False, msteps_quantum=50, nfrequency_quantum=150):
    """sld_params from a variables.in-style dict plus the control switches."""
    P = Params()
    lib().sld_params_default(C.byref(P))
    P.box[:] = list(params["box"])
    for k in ("step", "temperature", "atmass", "gamma_L_over_mass",
              "gamma_S_HL", "rcut_pot", "rcut_mag", "rcut_max",
              "min_length_link_cell", "kappa_e"):
        if k in params:
            setattr(P, k, float(params[k]))
    P.random_seed = int(params.get("random_seed", 1234))
    P.spinlang, P.lattlang, P.eltemp = int(spinlang), int(lattlang), int(eltemp)
    P.localcolmot, P.renormalize_energy = int(localcolmot), int(renormalize)
    P.te_mesh, P.te_nloop = int(te_mesh), int(te_nloop)
    P.precision, P.device = int(precision), int(device)
    P.interval_of_print_out = int(interval_of_print_out)
    P.replica = int(replica)
    P.interval_of_config_out = int(interval_of_config_out)
    P.pressure_control, P.stress_control = int(pressure_control), int(stress_control)
    P.change_step = int(change_step)
    P.hamiltonian = HAMILTONIANS[hamiltonian] if isinstance(hamiltonian, str) else int(hamiltonian)
    P.quantum_noise, P.msteps_quantum = int(quantum_noise), int(msteps_quantum)
    P.nfrequency_quantum = int(nfrequency_quantum)
    if "gamma_S_H" in params:
        P.gamma_S_H = float(params["gamma_S_H"])
    # barostat / time-step variables, variables.in names (read_variables.cpp:197-241)
    for k in ("pressure", "baro_damping_time", "displace_limit", "phi_limit"):
        if k in params:
            setattr(P, k, float(params[k]))
    for k in ("interval_of_scale_pressure", "interval_of_scale_stress"):
        if k in params:
            setattr(P, k, int(params[k]))
    for j, k in enumerate(("stress_xx", "stress_yx", "stress_yy", "stress_zx",
                           "stress_zy", "stress_zz")):
        if k in params:
            P.stress[j] = float(params[k])
    return P


VEC_FIELDS = {"r": 3, "p": 3, "f": 3, "s": 3, "H": 3, "HL": 3, "stress": 6}
CELL_FIELDS = ("Te", "Ee", "Tl", "Ts_R", "Ts_L", "Gel", "Ges", "count")


ADJ_NTHETA = 36


def adjoint_theta_default():
    """The potential's 36 parameters (DD05 embedding, density and pair
    terms, J(r), Landau), in sld_adjoint_*'s order."""
    th = np.zeros(ADJ_NTHETA)
    _check(lib().sld_adjoint_theta_default(_dp(th)), "adjoint_theta_default")
    return th


class Engine:
    """One spin-lattice system on one GPU."""

    def __init__(self, params, r, p, s, te=None, **switches):
        L = lib()
        self.L = L
        self.P = make_params(params, **switches)
        r = np.ascontiguousarray(r, np.float64).reshape(-1, 3)
        p = np.ascontiguousarray(p, np.float64).reshape(-1, 3)
        s = np.ascontiguousarray(s, np.float64).reshape(-1, 3)
        te_arr = None if te is None else np.ascontiguousarray(te, np.float64)
        h = C.c_void_p()
        _check(L.sld_create(C.byref(h), C.byref(self.P), r.shape[0], _dp(r),
                            _dp(p), _dp(s), None if te_arr is None else _dp(te_arr)),
               "sld_create")
        self._attach(h)

    def _attach(self, h):
        self.h = h
        info = (C.c_int * 6)()
        _check(self.L.sld_info(self.h, info), "sld_info")
        self.natom = info[0]
        self.ncells, self.ngroups, self.nte = info[1], info[2], info[3]

    @classmethod
    def from_config(cls, params, con_path, te_path=None, **switches):
        """A system read from a con- file (read_config.cpp format) and,
        optionally, a readTe file; box and natom come from the file."""
        self = cls.__new__(cls)
        self.L = lib()
        self.P = make_params(params, **switches)
        h = C.c_void_p()
        _check(self.L.sld_create_from_config(
            C.byref(h), C.byref(self.P), str(con_path).encode(),
            None if te_path is None else str(te_path).encode()), "sld_create_from_config")
        self._attach(h)
        return self

    def close(self):
        if getattr(self, "h", None):
            self.L.sld_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # the reference's step functions
    def links(self): _check(self.L.sld_links(self.h), "links")
    def calculate_rho(self): _check(self.L.sld_calculate_rho(self.h), "calculate_rho")
    def calculate_force_energy(self):
        _check(self.L.sld_calculate_force_energy(self.h), "calculate_force_energy")
    def calculate_temperature(self):
        _check(self.L.sld_calculate_temperature(self.h), "calculate_temperature")
    def core_ds(self, dt): _check(self.L.sld_core_ds(self.h, dt), "core_ds")
    def core_dp(self, dt): _check(self.L.sld_core_dp(self.h, dt), "core_dp")
    def core_dr(self, dt): _check(self.L.sld_core_dr(self.h, dt), "core_dr")
    def core_dTe(self, dt): _check(self.L.sld_core_dTe(self.h, dt), "core_dTe")

    def run(self, nsteps):
        _check(self.L.sld_run(self.h, int(nsteps)), "run")

    def core(self):
        self.run(1)

    def sync(self):
        _check(self.L.sld_sync(self.h), "sync")

    def set_state(self, r, p, s):
        r = np.ascontiguousarray(r, np.float64)
        p = np.ascontiguousarray(p, np.float64)
        s = np.ascontiguousarray(s, np.float64)
        _check(self.L.sld_set_state(self.h, _dp(r), _dp(p), _dp(s)), "set_state")

    def get(self, name, out=None):
        """A field in caller order; into ``out`` (a C-contiguous float64 array
        of the field's size, e.g. pinned host memory) when given."""
        width = VEC_FIELDS.get(name, 1)
        n = (self.nte if name in CELL_FIELDS else self.natom) * width
        if out is None:
            out = np.empty(n, np.float64)
        elif out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"] or out.size != n:
            raise ValueError(f"get({name}): out must be C-contiguous float64 of {n} values")
        got = self.L.sld_get(self.h, name.encode(), _dp(out), n)
        if got < 0:
            raise SldError(int(got), f"get({name})")
        return out.reshape(-1, width) if width > 1 else out

    def cell_lists(self):
        out = np.empty(self.natom, np.int32)
        _check(self.L.sld_get_cell_lists(self.h, out.ctypes.data_as(C.POINTER(C.c_int))),
               "cell_lists")
        return out

    def averages(self):
        out = np.empty(10, np.float64)
        _check(self.L.sld_averages(self.h, _dp(out)), "averages")
        return dict(zip(["pe", "ke", "me", "me0", "Ee", "Tl", "Te", "sx", "sy", "sz"], out))

    def virial(self):
        out = np.empty(1, np.float64)
        _check(self.L.sld_virial(self.h, _dp(out)), "virial")
        return float(out[0])

    def total_time(self):
        out = np.empty(1, np.float64)
        _check(self.L.sld_total_time(self.h, _dp(out)), "total_time")
        return float(out[0])

    PHASES = ("links", "core_dTe", "core_dp", "core_ds", "core_dr", "calculate_rho",
              "calculate_force_energy", "calculate_temperature", "check_energy", "bookkeeping")

    def profile_step(self):
        """One step run phase by phase; device ms per phase (CUDA events)."""
        out = np.zeros(10, np.float64)
        _check(self.L.sld_profile_step(self.h, _dp(out)), "profile_step")
        return dict(zip(self.PHASES, out))

    def step_kernel_count(self):
        n = C.c_int()
        _check(self.L.sld_step_kernel_count(self.h, C.byref(n)), "step_kernel_count")
        return n.value

    def check(self, out_dir, out_body, current_step):
        """check(current_step): append the enr-/tmp-/str-/prs-/spn- lines."""
        _check(self.L.sld_check(self.h, str(out_dir).encode(), out_body.encode(),
                                int(current_step)), "check")

    def write_config(self, out_dir, out_body, current_step, heff_as_reference=False):
        """write_config(current_step): con- (and cel-) files."""
        _check(self.L.sld_write_config(self.h, str(out_dir).encode(), out_body.encode(),
                                       int(current_step), 1 if heff_as_reference else 0),
               "write_config")

    def autotune(self, steps=3):
        """Choose the launch shapes by timing captured steps; the state is
        left unchanged.  Returns the chosen shapes."""
        out = (C.c_int * 8)()
        _check(self.L.sld_autotune(self.h, int(steps), out), "autotune")
        return dict(zip(("sweep_block", "pair_block", "force_block", "temp_block",
                         "dte_mode", "dte_threads", "sweep_cap"), list(out)))

    def quantum_filter(self):
        out = np.zeros(100000)
        n = self.L.sld_quantum_filter(self.h, _dp(out), len(out))
        if n < 0:
            raise SldError(int(n), "quantum_filter")
        return out[:n]

    def set_external_field(self, H):
        """Per-atom external field (natom x 3, eV), or None to remove."""
        a = None if H is None else np.ascontiguousarray(H, np.float64).reshape(-1, 3)
        _check(self.L.sld_set_external_field(self.h, None if a is None else _dp(a)),
               "set_external_field")

    def set_external_force(self, f):
        """Per-atom external force (natom x 3, eV/A), or None to remove."""
        a = None if f is None else np.ascontiguousarray(f, np.float64).reshape(-1, 3)
        _check(self.L.sld_set_external_force(self.h, None if a is None else _dp(a)),
               "set_external_force")

    def read_external_field(self, path):
        _check(self.L.sld_read_external_field(self.h, str(path).encode()), "read_external_field")

    def read_external_force(self, path):
        _check(self.L.sld_read_external_force(self.h, str(path).encode()), "read_external_force")

    def scale(self, current_step):
        """scale(current_step): barostats and adaptive time step; returns
        (displace_max, phi_max, new step)."""
        out = np.zeros(3, np.float64)
        _check(self.L.sld_scale(self.h, int(current_step), _dp(out)), "scale")
        return tuple(float(x) for x in out)

    def adjoint_config(self, theta):
        """(E, L, sum|f|^2, sum|H|^2), dE/dtheta, dL/dtheta at the current
        configuration."""
        th = np.ascontiguousarray(theta, np.float64)
        out, dE, dL = np.zeros(4), np.zeros(ADJ_NTHETA), np.zeros(ADJ_NTHETA)
        _check(self.L.sld_adjoint_config(self.h, _dp(th), _dp(out), _dp(dE), _dp(dL)),
               "adjoint_config")
        return out, dE, dL

    def adjoint_jacobians(self, theta):
        """Forces f, fields H (natom x 3) and their Jacobians in theta
        (natom x 3 x 36 each)."""
        th = np.ascontiguousarray(theta, np.float64)
        n = self.natom
        f, H = np.zeros((n, 3)), np.zeros((n, 3))
        dF, dH = np.zeros((n, 3, ADJ_NTHETA)), np.zeros((n, 3, ADJ_NTHETA))
        _check(self.L.sld_adjoint_jacobians(self.h, _dp(th), _dp(f), _dp(H), _dp(dF), _dp(dH)),
               "adjoint_jacobians")
        return f, H, dF, dH

    def adjoint_trajectory(self, theta, nsteps, checkpoint_every=20, grad=True):
        """Loss after nsteps NVE steps and (grad) its gradient in theta."""
        th = np.ascontiguousarray(theta, np.float64)
        Lv, dL = np.zeros(1), np.zeros(ADJ_NTHETA)
        _check(self.L.sld_adjoint_trajectory(self.h, _dp(th), int(nsteps), int(checkpoint_every),
                                             _dp(Lv), _dp(dL) if grad else None),
               "adjoint_trajectory")
        return (float(Lv[0]), dL) if grad else float(Lv[0])

    def last_run_ms(self):
        out = np.empty(1, np.float64)
        _check(self.L.sld_last_run_ms(self.h, _dp(out)), "last_run_ms")
        return float(out[0])


class Batch:
    """Several engines (independent replicas on one device) advanced
    together: each step is one CUDA graph holding every engine's step.  Each
    engine ends as if it had run alone; destroy the batch before its engines."""

    def __init__(self, engines):
        self.L = lib()
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e.h for e in self.engines])
        h = C.c_void_p()
        _check(self.L.sld_batch_create(C.byref(h), arr, len(self.engines)), "batch_create")
        self.h = h

    def run(self, nsteps):
        _check(self.L.sld_batch_run(self.h, int(nsteps)), "batch_run")

    def check(self, out_dir, out_body, current_step):
        """check(current_step): append the enr-/tmp-/str-/prs-/spn- lines."""
        _check(self.L.sld_check(self.h, str(out_dir).encode(), out_body.encode(),
                                int(current_step)), "check")

    def write_config(self, out_dir, out_body, current_step, heff_as_reference=False):
        """write_config(current_step): con- (and cel-) files."""
        _check(self.L.sld_write_config(self.h, str(out_dir).encode(), out_body.encode(),
                                       int(current_step), 1 if heff_as_reference else 0),
               "write_config")

    def autotune(self, steps=3):
        """Choose the launch shapes by timing captured steps; the state is
        left unchanged.  Returns the chosen shapes."""
        out = (C.c_int * 8)()
        _check(self.L.sld_autotune(self.h, int(steps), out), "autotune")
        return dict(zip(("sweep_block", "pair_block", "force_block", "temp_block",
                         "dte_mode", "dte_threads", "sweep_cap"), list(out)))

    def quantum_filter(self):
        out = np.zeros(100000)
        n = self.L.sld_quantum_filter(self.h, _dp(out), len(out))
        if n < 0:
            raise SldError(int(n), "quantum_filter")
        return out[:n]

    def set_external_field(self, H):
        """Per-atom external field (natom x 3, eV), or None to remove."""
        a = None if H is None else np.ascontiguousarray(H, np.float64).reshape(-1, 3)
        _check(self.L.sld_set_external_field(self.h, None if a is None else _dp(a)),
               "set_external_field")

    def set_external_force(self, f):
        """Per-atom external force (natom x 3, eV/A), or None to remove."""
        a = None if f is None else np.ascontiguousarray(f, np.float64).reshape(-1, 3)
        _check(self.L.sld_set_external_force(self.h, None if a is None else _dp(a)),
               "set_external_force")

    def read_external_field(self, path):
        _check(self.L.sld_read_external_field(self.h, str(path).encode()), "read_external_field")

    def read_external_force(self, path):
        _check(self.L.sld_read_external_force(self.h, str(path).encode()), "read_external_force")

    def scale(self, current_step):
        """scale(current_step): barostats and adaptive time step; returns
        (displace_max, phi_max, new step)."""
        out = np.zeros(3, np.float64)
        _check(self.L.sld_scale(self.h, int(current_step), _dp(out)), "scale")
        return tuple(float(x) for x in out)

    def adjoint_config(self, theta):
        """(E, L, sum|f|^2, sum|H|^2), dE/dtheta, dL/dtheta at the current
        configuration."""
        th = np.ascontiguousarray(theta, np.float64)
        out, dE, dL = np.zeros(4), np.zeros(ADJ_NTHETA), np.zeros(ADJ_NTHETA)
        _check(self.L.sld_adjoint_config(self.h, _dp(th), _dp(out), _dp(dE), _dp(dL)),
               "adjoint_config")
        return out, dE, dL

    def adjoint_jacobians(self, theta):
        """Forces f, fields H (natom x 3) and their Jacobians in theta
        (natom x 3 x 36 each)."""
        th = np.ascontiguousarray(theta, np.float64)
        n = self.natom
        f, H = np.zeros((n, 3)), np.zeros((n, 3))
        dF, dH = np.zeros((n, 3, ADJ_NTHETA)), np.zeros((n, 3, ADJ_NTHETA))
        _check(self.L.sld_adjoint_jacobians(self.h, _dp(th), _dp(f), _dp(H), _dp(dF), _dp(dH)),
               "adjoint_jacobians")
        return f, H, dF, dH

    def adjoint_trajectory(self, theta, nsteps, checkpoint_every=20, grad=True):
        """Loss after nsteps NVE steps and (grad) its gradient in theta."""
        th = np.ascontiguousarray(theta, np.float64)
        Lv, dL = np.zeros(1), np.zeros(ADJ_NTHETA)
        _check(self.L.sld_adjoint_trajectory(self.h, _dp(th), int(nsteps), int(checkpoint_every),
                                             _dp(Lv), _dp(dL) if grad else None),
               "adjoint_trajectory")
        return (float(Lv[0]), dL) if grad else float(Lv[0])

    def last_run_ms(self):
        out = np.empty(1, np.float64)
        _check(self.L.sld_batch_last_run_ms(self.h, _dp(out)), "batch_last_run_ms")
        return float(out[0])

    def close(self):
        if getattr(self, "h", None):
            self.L.sld_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def header_symbols(path=HEADER):
    """Entry points declared in include/sld.h."""
    import re
    text = open(path).read()
    return sorted(set(re.findall(r"\b(sld_[a-z_A-Z0-9]+)\s*\(", text)))
