"""The other Hamiltonians of control.h (MD, SDH, SDHL, SLDH) against the
reference built with each: the main-loop body with its output calls, the
output files token by token and the final state array by array.

The Langevin cases run at zero temperature, where the noise amplitude is
zero: the runs are deterministic, and the damping parts of the thermostats
(the lattice friction, the Heisenberg scheme's damped precession, the
Heisenberg-Landau relaxation) are what they test.
"""
import os

import numpy as np
import pytest

from conftest import relerr
from oracle import refjob as rj
from spilady_b200.lattice import initial_state
from test_gpu_output import compare_text, read_all

pytestmark = pytest.mark.gpu

TOL_STATE = 1e-10
TOL_FILE = 1e-10

CASES = {
    # name: (reference build, hamiltonian, switches)
    "md": ("md", "MD", {}),
    "md_lang": ("md_lang", "MD", dict(lattlang=True)),
    "sdh": ("sdh", "SDH", {}),
    "sdh_lang": ("sdh_lang", "SDH", dict(spinlang=True)),
    "sdhl": ("sdhl", "SDHL", {}),
    "sdhl_lang": ("sdhl_lang", "SDHL", dict(spinlang=True)),
    "sldh": ("sldh", "SLDH", {}),
    "sldh_lang": ("sldh_lang", "SLDH", dict(spinlang=True, lattlang=True)),
    # with the electron temperature, renormalisation and zero friction (the
    # noise amplitude is zero; Te moves by diffusion and the renormalisation)
    "md_te": ("md_te", "MD", dict(lattlang=True, eltemp=True, renormalize=True)),
    "sdh_te": ("sdh_te", "SDH", dict(spinlang=True, eltemp=True, renormalize=True)),
    "sdhl_te": ("sdhl_te", "SDHL", dict(spinlang=True, eltemp=True, renormalize=True)),
    "sldh_te": ("sldh_te", "SLDH", dict(spinlang=True, lattlang=True, eltemp=True,
                                        localcolmot=True, renormalize=True)),
}

# what each Hamiltonian has (struct.h:44-118)
LATT = {"MD", "SLDH", "SLDHL"}
SPIN = {"SDH", "SDHL", "SLDH", "SLDHL"}
HL = {"SDHL", "SLDHL"}


def engine_mod():
    from spilady_b200 import engine
    return engine


@pytest.mark.parametrize("case", sorted(CASES))
def test_hamiltonian_matches_reference(case, tmp_path):
    build, ham, sw = CASES[case]
    if not rj.available(build):
        pytest.skip("reference build missing")
    params, r, p, s = initial_state(6, seed=31, tilt=0.35, temperature=300.0)
    te = None
    if case.endswith("_lang"):
        params = dict(params, temperature=0.0)
    if ham in ("SDH", "SLDH"):
        # the harness passes the spin damping in one slot: gamma_S_H here
        params = dict(params, gamma_S_H=8e-3, gamma_S_HL=8e-3)
    if case.endswith("_te"):
        params = dict(params, gamma_L_over_mass=0.0, gamma_S_HL=0.0, gamma_S_H=0.0)
    E = engine_mod()
    if case.endswith("_te"):
        probe = E.Engine(params, r, p, s, hamiltonian=ham, **sw)
        k = np.arange(probe.ncells)
        te = 300.0 + 40.0 * (k % 7) + 5.0 * (k % 3)
        probe.close()
    nsteps = 3
    dumps, ref = rj.run(build, params, r, p, s, te=te,
                        ops=[(rj.OP_STEP, nsteps), (rj.OP_DUMP, 0)], files=True)
    e = E.Engine(params, r, p, s, te=te, hamiltonian=ham, interval_of_config_out=1, **sw)
    d = tmp_path / "out"
    d.mkdir()
    if sw.get("renormalize"):
        # the harness's set-up prints the reference energy (check_energy(-1))
        d0 = tmp_path / "init"
        d0.mkdir()
        e.check(d0, "b200", -1)
        (d / "enr-b200.dat").write_text((d0 / "enr-b200.dat").read_text())
    for k in range(nsteps):
        e.run(1)
        e.check(d, "b200", k)
        e.write_config(d, "b200", k, heff_as_reference=True)
    ours = read_all(d)
    assert sorted(ours) == sorted(n.replace("-ref", "-b200") for n in ref)
    worst = {n: compare_text(ours[n], ref[n.replace("-b200", "-ref")], TOL_FILE, n)
             for n in sorted(ours)}
    D = dumps[0]
    names = ["r"]
    if ham in LATT:
        names += ["p", "f"]
    if ham in SPIN:
        names += ["s", "H"]
    if ham in HL:
        names += ["HL"]
    errs = {}
    for name in names:
        errs[name] = relerr(e.get(name), D.vec(name))
        assert errs[name] <= TOL_STATE, f"{case} {name}: {errs[name]:.2e}"
    scal = []
    if ham in LATT:
        scal += ["pe", "ke", "rho"]
    if ham in SPIN:
        scal += ["me", "me0"]
    for name in scal:
        errs[name] = relerr(e.get(name), D.a(name))
        assert errs[name] <= TOL_STATE, f"{case} {name}: {errs[name]:.2e}"
    if te is not None:
        errs["Te"] = relerr(e.get("Te"), D.c("Te"))
        assert errs["Te"] <= TOL_STATE, f"{case} Te: {errs['Te']:.2e}"
    print(case, " ".join(f"{k}:{v:.1e}" for k, v in errs.items()),
          "files", f"{max(worst.values()):.1e}")
