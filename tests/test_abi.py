"""The C-ABI library loads on a CPU-only machine and exports every entry
point include/sld.h declares; host-side validation works without a GPU."""
import ctypes as C
import os

import numpy as np
import pytest

from spilady_b200 import engine


def test_library_exports_every_declared_symbol():
    L = engine.lib()
    syms = engine.header_symbols()
    assert "sld_create" in syms and "sld_run" in syms
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_params_default_are_reference_defaults():
    P = engine.Params()
    assert engine.lib().sld_params_default(C.byref(P)) == 0
    assert P.step == 1e-15 and P.temperature == 300.0 and P.atmass == 55.847
    assert P.gamma_L_over_mass == 6e11 and P.gamma_S_HL == 5.88e13
    assert P.rcut_pot == 4.1001 and P.rcut_mag == 3.7501 and P.min_length_link_cell == 4.11
    assert P.te_nloop == 50 and P.random_seed == 1234


def test_read_variables(tmp_path):
    f = tmp_path / "variables.in"
    f.write_text("out_body X\nstep 5e-16\ntemperature 450\ngamma_S_HL 1.5e13\n"
                 "unknown_key 7\nrcut_mag 3.5\nspinlang 1\neltemp 1\nte_mesh 16\n")
    P = engine.Params()
    L = engine.lib()
    L.sld_params_default(C.byref(P))
    assert L.sld_read_variables(str(f).encode(), C.byref(P)) == 0
    assert P.step == 5e-16 and P.temperature == 450 and P.gamma_S_HL == 1.5e13
    assert P.rcut_mag == 3.5 and P.spinlang == 1 and P.eltemp == 1 and P.te_mesh == 16
    assert L.sld_read_variables(str(tmp_path / "missing").encode(), C.byref(P)) == -7


def _create(params, r, p, s, **sw):
    L = engine.lib()
    P = engine.make_params(params, **sw)
    h = C.c_void_p()
    dp = lambda a: np.ascontiguousarray(a, np.float64).ctypes.data_as(C.POINTER(C.c_double))
    return L.sld_create(C.byref(h), C.byref(P), r.shape[0], dp(r), dp(p), dp(s), None)


def test_geometry_rejected_before_touching_the_device():
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(2, seed=1)        # 2 link cells per axis
    assert _create(params, r, p, s) == -3


def test_invalid_switch_combination_rejected():
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(5, seed=1)
    assert _create(params, r, p, s, eltemp=True) == -1        # eltemp needs both thermostats
    assert _create(params, r, p, s, localcolmot=True) == -1   # needs lattlang


def test_error_strings():
    L = engine.lib()
    for code in range(0, -10, -1):
        assert L.sld_error_string(code)


def test_error_strings_cover_every_code():
    L = engine.lib()
    L.sld_error_string.restype = C.c_char_p
    for code in range(0, -11, -1):
        msg = L.sld_error_string(code).decode()
        assert msg and msg != "unknown error", code
        if code < 0:
            assert code in engine.ERRORS, code


def test_read_variables_other_switches(tmp_path):
    # the keys of the switches that are compile-time in the reference
    # (control.h) and of the variables behind them (read_variables.cpp:197-250)
    f = tmp_path / "variables.in"
    f.write_text("hamiltonian SDHL\ngamma_S_H 0.02\nPRESSURE 1\nSTRESS 1\nchangestep 1\n"
                 "pressure 2.5\nstress_yx -0.5\nbaro_damping_time 3e-13\n"
                 "interval_of_scale_pressure 7\ndisplace_limit 0.02\nphi_limit 0.3\n"
                 "quantumnoise 1\nMsteps_quantum 20\nNfrequency_quantum 64\n"
                 "interval_of_config_out 25\n")
    P = engine.Params()
    L = engine.lib()
    L.sld_params_default(C.byref(P))
    assert P.interval_of_config_out == 1000 and P.msteps_quantum == 50
    assert P.nfrequency_quantum == 150 and P.baro_damping_time == 1e-13
    assert L.sld_read_variables(str(f).encode(), C.byref(P)) == 0
    assert P.hamiltonian == engine.SDHL and P.gamma_S_H == 0.02
    assert P.pressure_control == 1 and P.stress_control == 1 and P.change_step == 1
    assert P.pressure == 2.5 and P.stress[1] == -0.5 and P.baro_damping_time == 3e-13
    assert P.interval_of_scale_pressure == 7 and P.displace_limit == 0.02
    assert P.phi_limit == 0.3 and P.quantum_noise == 1 and P.msteps_quantum == 20
    assert P.nfrequency_quantum == 64 and P.interval_of_config_out == 25


def test_hamiltonian_switch_combinations_rejected():
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(5, seed=1)
    E = engine
    assert _create(params, r, p, s, hamiltonian=E.MD, spinlang=True) == -1     # no spins
    assert _create(params, r, p, s, hamiltonian=E.SDH, lattlang=True) == -1    # no lattice
    assert _create(params, r, p, s, hamiltonian=E.SDHL, pressure_control=True) == -1
    assert _create(params, r, p, s, hamiltonian=E.MD, lattlang=True, eltemp=True,
                   spinlang=False, quantum_noise=True, change_step=True) == -1
    assert _create(params, r, p, s, quantum_noise=True) == -1                  # needs lattlang
    assert _create(params, r, p, s, hamiltonian=7) == -1
