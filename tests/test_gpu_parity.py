"""GPU parity: the CUDA engine (through the C ABI) against the oracle.

FP64 form tolerances (norm-wise relative, max|a-b| / max|b|):
  - one sub-operation or one step:             1e-11
  - a few Langevin / Te steps (Philox noise):  1e-10
  - 100 NVE steps against the reference fixture: 1e-8 (chaotic growth of
    last-bit differences from transcendental functions and FMA)
Integer data (cell lists, colour groups) must match exactly.
"""
import numpy as np
import pytest

from conftest import load_golden, relerr
from oracle import orc
from spilady_b200.lattice import initial_state, default_params

pytestmark = pytest.mark.gpu

TOL1 = 1e-11


def engine_mod():
    from spilady_b200 import engine
    return engine


def pair(ncell, seed, tilt=0.05, temperature=300.0, te=None, pos_sigma=0.0, **sw):
    params, r, p, s = initial_state(ncell, seed=seed, tilt=tilt,
                                    temperature=temperature, pos_sigma=pos_sigma)
    o = orc.System(params, r, p, s, te=te, rng=orc.RNG_PHILOX, **sw)
    e = engine_mod().Engine(params, r, p, s, te=te, **sw)
    return params, o, e


def compare(o, e, names, tol, where=""):
    for n in names:
        a, b = e.get(n), o.get(n)
        err = relerr(a, b)
        assert err <= tol, f"{where} {n}: rel err {err:.3e} > {tol:.0e}"


ATOM = ["r", "p", "f", "s", "rho", "pe", "me", "me0", "ke"]


def test_initial_rho_force_energy():
    params, o, e = pair(6, seed=1)
    compare(o, e, ATOM + ["stress"], TOL1, "init")
    assert np.array_equal(e.cell_lists(), o.lists())
    assert e.ngroups == o.ngroups and e.ncells == o.ncells
    # the per-atom virial is split differently; the total is the reference's
    assert abs(e.virial() - o.get("vir").sum()) <= 1e-11 * abs(o.get("vir")).sum()


def test_subops_nve_sequence():
    params, o, e = pair(6, seed=2, tilt=0.3)
    dt = params["step"]
    seq = [("links", ()), ("core_dp", (dt / 2,)), ("core_ds", (dt / 2,)),
           ("core_dr", (dt,)), ("calculate_rho", ()), ("core_ds", (dt / 2,)),
           ("calculate_force_energy", ()), ("core_dp", (dt / 2,))]
    for name, args in seq:
        getattr(o, name)(*args)
        getattr(e, name)(*args)
        compare(o, e, ATOM + ["H"], TOL1, name)


def test_nve_steps_match_oracle_and_graph_replay():
    params, o, e = pair(8, seed=3, tilt=0.2)
    for k in range(3):
        o.run(1)
        e.run(1)
        compare(o, e, ATOM + ["H"], 1e-10, f"step {k}")
    assert np.array_equal(e.cell_lists(), o.lists())


def test_links_order_with_many_movers():
    # hot lattice and a small cell edge: many atoms change cell every step
    params, o, e = pair(6, seed=4, temperature=3000.0, tilt=0.2)
    for k in range(6):
        o.run(1)
        e.run(1)
        assert np.array_equal(e.cell_lists(), o.lists()), f"step {k}"
        assert np.array_equal(e.get("cell").astype(int), o.get("cell").astype(int))


def test_langevin_spin_lattice_matches_oracle():
    params, o, e = pair(6, seed=5, tilt=0.3, spinlang=True, lattlang=True)
    for k in range(3):
        o.run(1)
        e.run(1)
        compare(o, e, ATOM + ["H", "HL", "sumJ"], 1e-10, f"lang step {k}")


def test_langevin_subops_draw_the_same_noise():
    params, o, e = pair(6, seed=6, tilt=0.3, spinlang=True, lattlang=True,
                        localcolmot=True)
    dt = params["step"]
    for name, args in [("core_dp", (dt / 2,)), ("core_ds", (dt / 2,)),
                       ("core_dp", (dt / 2,)), ("core_ds", (dt / 2,))]:
        getattr(o, name)(*args)
        getattr(e, name)(*args)
        compare(o, e, ["p", "s", "ke"], TOL1, name)


def test_electron_temperature_link_cells():
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True, renormalize=True)
    params, o, e = pair(6, seed=7, tilt=0.35, **sw)
    compare(o, e, ["Te", "Tl", "Ts_L", "Ts_R", "Gel", "Ges"], TOL1, "init")
    for k in range(3):
        o.run(1)
        e.run(1)
        compare(o, e, ATOM + ["Te", "Tl", "Ts_L", "Ges", "Gel"], 1e-10, f"te step {k}")


def test_electron_temperature_mesh():
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True, renormalize=True,
              te_mesh=4)
    params0 = default_params(8)
    from spilady_b200.lattice import hot_spot_te
    te = hot_spot_te(4, params0["box"][0], peak=1500.0, background=300.0, sigma=6.0)
    params, o, e = pair(8, seed=8, tilt=0.35, te=te, **sw)
    compare(o, e, ["Te", "Tl", "Ts_L", "Gel", "Ges", "count"], TOL1, "mesh init")
    for k in range(2):
        o.run(1)
        e.run(1)
        compare(o, e, ATOM + ["Te", "Tl", "Ts_L"], 1e-10, f"mesh step {k}")


def test_core_dte_alone():
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True)
    params, o, e = pair(6, seed=9, tilt=0.35, **sw)
    o.core_dTe(5e-16)
    e.core_dTe(5e-16)
    compare(o, e, ["Te", "Ee"], TOL1, "core_dTe")


def test_nve_100_steps_against_reference_fixture():
    g = load_golden("nve_16")
    p = default_params(16)
    e = engine_mod().Engine(p, g["r0"], g["p0"], g["s0"])
    fields = list(g["atom_fields"])
    col = lambda k, n: g["atoms"][k][:, fields.index(n)]
    assert e.ngroups == int(g["ngroups"])
    e.run(int(g["every"]))
    for name, cols in [("s", ("sx", "sy", "sz")), ("r", ("rx", "ry", "rz")),
                       ("p", ("px", "py", "pz")), ("f", ("fx", "fy", "fz"))]:
        ref = np.stack([col(1, c) for c in cols], 1)
        err = relerr(e.get(name), ref)
        assert err <= 1e-8, f"{name}: {err:.3e}"
    assert np.array_equal(e.cell_lists(), g["lists"][1])


def test_deterministic_replay():
    params, r, p, s = initial_state(6, seed=10, tilt=0.3)
    E = engine_mod().Engine
    a = E(params, r, p, s, spinlang=True, lattlang=True)
    b = E(params, r, p, s, spinlang=True, lattlang=True)
    a.run(3)
    b.run(3)
    for n in ("r", "p", "s"):
        assert np.array_equal(a.get(n), b.get(n))


def test_averages_and_time():
    params, o, e = pair(6, seed=11, tilt=0.2)
    o.run(2)
    e.run(2)
    ao, ae = o.averages(), e.averages()
    for k in ("pe", "ke", "me", "me0", "Tl", "sx", "sy", "sz"):
        assert abs(ae[k] - ao[k]) <= 1e-10 * max(abs(ao[k]), 1e-30), k
    assert abs(e.total_time() - 2 * params["step"]) < 1e-30
    e.sync()


# ---------------------------------------------------------------- split form
# The split form evaluates the DD05 / exchange forms in FP32 with the
# reference's seven-point derivatives (the exact derivative plus the stencil
# term of a knot within 3 r/1000) and F(rho), F'(rho) from the reference's
# tables: the functions of the reference's tables.  It is held to 1e-5
# against the oracle and against the FP64 form (the reference's arithmetic
# on the GPU).  FP64_ANALYTIC, the functional forms with their exact
# derivatives (the adjoint's model), differs from the tables by the tables'
# seven-point derivatives near the knots: bcc Fe's second shell (2.8665 A)
# sits on the density knot at 2.8667 A.
SPLIT_TOL = 1e-5      # split form vs the oracle / the FP64 form
TABLE_TOL = 1e-4      # exact-derivative analytic forms vs the reference's tables


def _three(ncell, seed, **sw):
    eng = engine_mod()
    params, r, p, s = initial_state(ncell, seed=seed, tilt=0.3, pos_sigma=0.05)
    return (params, eng.Engine(params, r, p, s, **sw),
            eng.Engine(params, r, p, s, precision=eng.FP64_ANALYTIC, **sw),
            eng.Engine(params, r, p, s, precision=eng.SPLIT, **sw))


def test_split_form_forces_and_fields_against_fp64():
    params, tab, an, sp = _three(8, 12, spinlang=True, lattlang=True)
    assert relerr(sp.get("rho"), tab.get("rho")) <= 1e-6
    for n in ("f", "pe", "me", "me0", "stress"):
        err = relerr(sp.get(n), tab.get(n))
        assert err <= SPLIT_TOL, f"split {n}: {err:.3e}"
        err = relerr(an.get(n), tab.get(n))
        assert err <= TABLE_TOL, f"analytic vs tables {n}: {err:.3e}"
    dt = params["step"]
    for e in (tab, an, sp):
        e.core_ds(dt / 2)
    for n in ("H", "s"):
        err = relerr(sp.get(n), tab.get(n))
        assert err <= SPLIT_TOL, f"split {n}: {err:.3e}"


@pytest.mark.parametrize("ncell", [8, 20])
def test_split_form_one_step_against_fp64_and_oracle(ncell):
    # one Langevin step (Philox noise, the same draws in all four): the split
    # form against the oracle at 1e-5, the FP64 forms against it at 1e-10.
    # 20^3 cells have 13^3 link cells in 18 colour groups (the colour count of
    # the 89^3 link cells of the 128^3 box)
    sw = dict(spinlang=True, lattlang=True, localcolmot=True)
    params, tab, an, sp = _three(ncell, 13, **sw)
    params_, r, p, s = initial_state(ncell, seed=13, tilt=0.3, pos_sigma=0.05)
    o = orc.System(params_, r, p, s, rng=orc.RNG_PHILOX, **sw)
    assert sp.ngroups == o.ngroups
    for n in ("f", "rho", "pe", "me"):
        err = relerr(sp.get(n), o.get(n))
        assert err <= SPLIT_TOL, f"start state: split vs oracle {n}: {err:.3e}"
    o.run(1)
    for e in (tab, an, sp):
        e.run(1)
    for n in ("r", "p", "s", "f", "H", "rho", "pe", "me"):
        err = relerr(tab.get(n), o.get(n))
        assert err <= 1e-10, f"FP64 form vs oracle {n}: {err:.3e}"
        err = relerr(an.get(n), o.get(n))
        assert err <= TABLE_TOL, f"analytic FP64 form vs oracle {n}: {err:.3e}"
        err = relerr(sp.get(n), tab.get(n))
        assert err <= SPLIT_TOL, f"split vs FP64 form {n}: {err:.3e}"
        err = relerr(sp.get(n), o.get(n))
        assert err <= SPLIT_TOL, f"split vs oracle {n}: {err:.3e}"


def test_split_form_electron_mesh_runs_and_tracks_fp64():
    eng = engine_mod()
    from spilady_b200.lattice import hot_spot_te
    params, r, p, s = initial_state(8, seed=14, tilt=0.35)
    te = hot_spot_te(4, params["box"][0], peak=1500.0, sigma=6.0)
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True, renormalize=True,
              te_mesh=4)
    a = eng.Engine(params, r, p, s, te=te, precision=eng.FP64, **sw)
    b = eng.Engine(params, r, p, s, te=te, precision=eng.SPLIT, **sw)
    a.run(3)
    b.run(3)
    b.sync()
    for n in ("s", "p", "Te"):
        err = relerr(b.get(n), a.get(n))
        assert err <= SPLIT_TOL, f"{n}: {err:.3e}"


# ------------------------------------------------------ sweep schedules
def _run_with_sweep_mode(mode, monkeypatch, precision):
    monkeypatch.setenv("SLD_SWEEP_MODE", str(mode))
    eng = engine_mod()
    params, r, p, s = initial_state(8, seed=15, tilt=0.3, temperature=600.0)
    e = eng.Engine(params, r, p, s, spinlang=True, lattlang=True, localcolmot=True,
                   precision=precision)
    e.run(3)
    e.core_ds(params["step"] / 2)
    e.sync()
    out = {n: e.get(n) for n in ("s", "H", "HL", "sumJ", "p", "r")}
    e.close()
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_sweep_schedules_give_identical_bits(monkeypatch, precision):
    # one launch per colour group with the pipelined walk (2) and the
    # data-flow schedule of the same walk (3) visit the cells in orders the
    # reference's dependencies cannot tell apart: bit for bit the same.  The
    # plain walk (1) is separate code: the same bits in the split form, whose
    # sums are rounded step by step; in FP64 the compiler may fuse a
    # different product of a two-product sum in its integrator (last bit).
    ref = _run_with_sweep_mode(3, monkeypatch, precision)
    got = _run_with_sweep_mode(2, monkeypatch, precision)
    for n, a in ref.items():
        assert np.array_equal(got[n], a), f"mode 2 {n}"

    got = _run_with_sweep_mode(1, monkeypatch, precision)
    for n, a in ref.items():
        if precision == 1:
            assert np.array_equal(got[n], a), f"mode 1 {n}"
        else:
            assert relerr(got[n], a) <= 1e-14, f"mode 1 {n}: {relerr(got[n], a):.2e}"


# ------------------------------------------------------ core_dTe kernels
@pytest.mark.parametrize("mode", [3, 2, 1, 0])
@pytest.mark.parametrize("precision", [0, 2])
def test_core_dte_kernels_and_forms(monkeypatch, mode, precision):
    # hub by levels (3) and by colour phases (2), cluster (1) and one-CTA (0)
    # kernels, with the reference's
    # heat-capacity expressions (FP64 form) and with the fitted ones (the
    # split form's, here in its FP64 twin): one core_dTe and one full step
    monkeypatch.setenv("SLD_DTE_MODE", str(mode))
    from spilady_b200.lattice import hot_spot_te
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True, renormalize=True,
              te_mesh=4)
    params, r, p, s = initial_state(8, seed=16, tilt=0.35)
    te = hot_spot_te(4, params["box"][0], peak=3000.0, background=300.0, sigma=6.0)
    o = orc.System(params, r, p, s, te=te, rng=orc.RNG_PHILOX, **sw)
    e = engine_mod().Engine(params, r, p, s, te=te, precision=precision, **sw)
    o.core_dTe(5e-16)
    e.core_dTe(5e-16)
    compare(o, e, ["Te", "Ee"], TOL1, f"core_dTe mode {mode}")
    if precision == 0:
        o.run(1)
        e.run(1)
        compare(o, e, ATOM + ["Te", "Tl"], 1e-10, f"step, dTe mode {mode}")


@pytest.mark.parametrize("cells", [10, 8])
@pytest.mark.parametrize("precision", [0, 2])
def test_core_dte_levels_give_the_phase_bits(monkeypatch, cells, precision):
    # the hub's sweep by levels against the same hub by colour phases: every
    # update reads the values of the sequential sweep, so the bits agree.  Te
    # on the link cells (6^3 at 10^3 unit cells: 8 colours, 7 levels; 5^3 at
    # 8^3: 20 colours, irregular levels and double tasks inside the sweep),
    # whose lattice and spin temperatures are fixed-order sums (a Te mesh
    # sums them with atomics, whose order is not fixed)
    from spilady_b200.lattice import hot_spot_te
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True, renormalize=True)
    params, r, p, s = initial_state(cells, seed=16, tilt=0.35)
    mesh = {10: 6, 8: 5}[cells]
    te = hot_spot_te(mesh, params["box"][0], peak=3000.0, background=300.0, sigma=6.0)
    out = {}
    for mode in (2, 3):
        monkeypatch.setenv("SLD_DTE_MODE", str(mode))
        e = engine_mod().Engine(params, r, p, s, te=te, precision=precision, **sw)
        assert e.ncells == mesh ** 3
        e.core_dTe(5e-16)
        out[mode] = {n: e.get(n) for n in ("Te", "Ee")}
        e.close()
    for n in ("Te", "Ee"):
        assert np.array_equal(out[2][n], out[3][n]), n


@pytest.mark.parametrize("precision", [0, 1])
def test_atoms_wrapped_by_the_drift_keep_their_pairs(precision):
    # Atoms that the drift carries across the box's high faces are wrapped to
    # the low side (periodic_CPU.cpp:31-50) but stay linked in their old cell
    # until the next links; the reference still finds their pairs (find_image
    # on every pair).  The lattice is shifted so that the sites of highest x,
    # y and z sit 0.002 A below the faces, and those atoms move outwards.
    eng = engine_mod()
    params, r, p, s = initial_state(6, seed=17, tilt=0.3, temperature=300.0, pos_sigma=0.05)
    L = params["box"][0]
    r = r + (L - 0.002 - r.max(axis=0))
    sigma = p.std()
    for ax in range(3):
        sel = r[:, ax] > L - 0.003
        assert sel.any()
        p[sel, ax] = 20.0 * sigma   # about 0.04 A per step
    p -= p.mean(axis=0)
    o = orc.System(params, r, p, s, rng=orc.RNG_PHILOX)
    e = eng.Engine(params, r, p, s, precision=precision)
    tol = 1e-10 if precision == 0 else SPLIT_TOL
    for k in range(2):
        o.run(1)
        e.run(1)
        e.sync()
        if k == 0:
            # some atoms were wrapped by the first drift
            assert np.any(e.get("r") < 0.1)
        for n in ("r", "p", "s", "f", "rho", "pe", "me"):
            err = relerr(e.get(n), o.get(n))
            assert err <= tol, f"step {k} {n}: {err:.3e}"
