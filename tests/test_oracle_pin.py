"""The oracle (C restatement, oracle/sld_oracle.c) against the reference's
own CPU build: the committed golden fixtures (tests/golden, made by
tests/golden/make_golden.py from oracle/_ref) and, where the reference build
is present, a live run.  With the reference's random stream (MWC, one
thread) the restatement reproduces the reference bit for bit."""
import os
import sys

import numpy as np
import pytest

from conftest import load_golden, relerr
from oracle import orc, refjob
from oracle import refjob as rj
from spilady_b200.lattice import default_params, initial_state

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SWITCHES = {
    "nve": {},
    "lang": dict(spinlang=True, lattlang=True),
    "langte": dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True,
                   renormalize=True),
}

VEC = {"r": ["rx", "ry", "rz"], "p": ["px", "py", "pz"], "f": ["fx", "fy", "fz"],
       "s": ["sx", "sy", "sz"], "H": ["Hx", "Hy", "Hz"], "HL": ["HLx", "HLy", "HLz"]}
SCAL = {"rho": "rho", "pe": "pe", "ke": "ke", "me": "me", "me0": "me0",
        "sumJ": "sum_Jij_sj"}


def golden_field(g, k, name):
    fields = list(g["atom_fields"])
    if name in VEC:
        if not all(c in fields for c in VEC[name]):
            return None
        return np.stack([g["atoms"][k][:, fields.index(c)] for c in VEC[name]], 1)
    key = SCAL[name]
    if key not in fields:
        return None
    return g["atoms"][k][:, fields.index(key)]


def params_from(g):
    L = g["box"][0]
    p = default_params(1)
    p["box"] = tuple(g["box"])
    p["step"] = float(g["step"])
    return p


@pytest.mark.parametrize("name", ["nve_6", "lang_6", "langte_6", "nve_16"])
def test_oracle_matches_reference_fixture(name):
    g = load_golden(name)
    mode = str(g["mode"])
    sysm = orc.System(params_from(g), g["r0"], g["p0"], g["s0"], rng=orc.RNG_MWC,
                      **SWITCHES[mode])
    assert sysm.ngroups == int(g["ngroups"])
    every = int(g["every"])
    for k in range(g["atoms"].shape[0]):
        if k:
            sysm.run(every)
        for name_ in list(VEC) + list(SCAL):
            ref = golden_field(g, k, name_)
            if ref is None:
                continue
            got = sysm.get(name_)
            if name_ == "HL" and mode == "nve":
                continue
            assert np.array_equal(got, ref), f"{name} dump {k} field {name_}: {relerr(got, ref)}"
        assert np.array_equal(sysm.lists(), g["lists"][k])
        if mode == "langte":
            ci = list(g["cell_fields"])
            for c in ("Te", "Tl", "Ts_L", "Ts_R", "Gel", "Ges"):
                ref = g["cells"][k][:, ci.index(c)]
                got = sysm.get(c)
                assert np.array_equal(got, ref), f"{name} cell {c}"


def test_colour_groups_match_reference_fixture():
    g = load_golden("nve_16")
    grp = g["groups"]
    # 16^3 bcc -> 11^3 link cells -> 18 colour groups (the reference's printout)
    assert int(g["ngroups"]) == 18
    total, k, ng = 0, 0, 0
    while k < len(grp):
        m = int(grp[k]); total += m; k += 1 + m; ng += 1
    assert ng == 18 and total == 11 ** 3


@pytest.mark.skipif(not refjob.available("nve"), reason="reference build absent")
def test_oracle_matches_live_reference_subops():
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(5, seed=7, tilt=0.2)
    ops = [(refjob.OP_LINKS, 0), (refjob.OP_DP, 5e-16), (refjob.OP_DS, 5e-16),
           (refjob.OP_DR, 1e-15), (refjob.OP_RHO, 0), (refjob.OP_FORCE, 0),
           (refjob.OP_DUMP, 0)]
    d = refjob.run("nve", params, r, p, s, ops=ops)[0]
    o = orc.System(params, r, p, s, rng=orc.RNG_MWC)
    o.links(); o.core_dp(5e-16); o.core_ds(5e-16); o.core_dr(1e-15)
    o.calculate_rho(); o.calculate_force_energy()
    for n in ("r", "p", "s", "f"):
        assert np.array_equal(o.get(n), d.vec(n))
    assert np.array_equal(o.get("rho"), d.a("rho"))


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10
    assert orc.philox4x32([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert orc.philox4x32([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [
        0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert orc.philox4x32([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                          [0xA4093822, 0x299F31D0]) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_philox_normal_moments():
    x = np.array([orc.philox_normals(1234, 0, a, e) for a in range(2000) for e in range(5)])
    assert abs(x.mean()) < 0.03
    assert abs(x.var() - 1.0) < 0.05
    # independent components
    c = np.corrcoef(x.T)
    assert np.max(np.abs(c - np.eye(3))) < 0.05


def test_oracle_rejects_two_cell_box():
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(2, seed=1)
    with pytest.raises(ValueError):
        orc.System(params, r, p, s)


def test_quantum_filter_matches_the_references():
    # initial_quantum_noise's filter, as the reference built with quantumnoise
    # makes it, against the oracle's restatement: bit for bit
    from oracle import orc
    if not rj.available("quant"):
        pytest.skip("reference build missing")
    params, r, p, s = initial_state(6, seed=5)
    ops = rj.set_ops(Msteps_quantum=3, Nfrequency_quantum=12) + [(rj.OP_QINIT, 0),
                                                                 (rj.OP_QFILTER, 0)]
    _, t = rj.run("quant", params, r, p, s, ops=ops, files=True)
    ref = np.array([float(x) for x in t["qfilter.dat"].split()])
    o = orc.System(params, r, p, s, lattlang=True, quantum=True, msteps_quantum=3,
                   nfrequency_quantum=12)
    assert len(ref) == 24 and np.array_equal(o.quantum_filter(), ref)


def test_param_build_is_the_stock_build_at_the_default_constants():
    # the param build (the potential's constants from theta.in, for finite
    # differences of the reference's code) gives the stock build's forces
    # and fields at the default constants, bit for bit
    if not (rj.available("param") and rj.available("nve")):
        pytest.skip("reference build missing")
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import DEFAULT_THETA
    params, r, p, s = initial_state(6, seed=6, tilt=0.2, pos_sigma=0.05)
    ops = [(rj.OP_CORE, 2), (rj.OP_CHECK, 1), (rj.OP_DUMP, 0)]
    a = rj.run("param", params, r, p, s, ops=ops,
               inputs={"theta.in": " ".join("%.17g" % x for x in DEFAULT_THETA)})[0]
    b = rj.run("nve", params, r, p, s, ops=ops)[0]
    assert np.array_equal(a.atoms, b.atoms)


@pytest.mark.skipif(not refjob.available("langte"), reason="reference build absent")
def test_oracle_matches_live_reference_langte_20cubed():
    # 20^3 cells: 13^3 link cells in 18 colour groups (the colour count of the
    # 89^3 link cells of the 128^3 box); three spin-lattice-electron steps
    # with the reference's own noise stream (MWC, one thread): bit for bit
    params, r, p, s = initial_state(20, seed=21, tilt=0.35)
    d = refjob.run("langte", params, r, p, s, ops=[(refjob.OP_CORE, 3), (refjob.OP_DUMP, 0)])[0]
    o = orc.System(params, r, p, s, rng=orc.RNG_MWC, **SWITCHES["langte"])
    assert o.ngroups == d.ngroups == 18
    o.run(3)
    for n in ("r", "p", "s", "f", "H", "HL"):
        assert np.array_equal(o.get(n), d.vec(n)), n
    for n in ("rho", "pe", "me", "me0", "ke"):
        assert np.array_equal(o.get(n), d.a(SCAL[n])), n
    for c in ("Te", "Tl", "Ts_L", "Ts_R"):
        assert np.array_equal(o.get(c), d.c(c)), c
    assert np.array_equal(o.lists(), d.lists)
