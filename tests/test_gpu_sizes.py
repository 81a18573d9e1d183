"""GPU parity at the larger sizes: the engine (through the C ABI) against the
oracle on the colourings and cell grids of the benchmark-sized boxes.

- 20^3 cells (16,000 atoms): 13^3 link cells in 18 colour groups, the colour
  count of the 89^3 link cells of the 128^3 box; three spin-lattice-electron
  steps (Te on the link cells, Philox noise drawn the same in both);
- 64^3 cells (524,288 atoms): 44^3 link cells in 8 colour groups; one NVE
  step;
- 128^3 cells (4,194,304 atoms): the benchmark's start state (Te on a 16^3
  mesh with its hot spot), rho, forces, per-atom energies and the cell
  temperatures against the oracle's calculate_rho / calculate_force_energy /
  calculate_temperature.

Tolerances (max|a-b| / max|b|): FP64 form 1e-11 for the start state, 1e-10
after steps; split form 1e-5.
"""
import numpy as np
import pytest

from conftest import relerr
from oracle import orc
from spilady_b200.lattice import hot_spot_te, initial_state

pytestmark = pytest.mark.gpu

SPLIT_TOL = 1e-5
ATOM = ["r", "p", "f", "s", "H", "rho", "pe", "me", "me0", "ke"]


def engine_mod():
    from spilady_b200 import engine
    return engine


def _compare(e, o, names, tol, where):
    for n in names:
        err = relerr(e.get(n), o.get(n))
        assert err <= tol, f"{where} {n}: rel err {err:.3e} > {tol:.0e}"


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_langte_20cubed_three_steps(precision):
    # a thermal start state (positions displaced by 0.05 A, about the
    # vibration amplitude of bcc Fe at 300 K).  On a perfect lattice the net
    # forces nearly vanish by symmetry: the split form's FP32 pair terms, each
    # rounded to about 1e-7 of its ~1 eV/A, then come to 1e-5 of the small net
    # force, and the FP64 form's electron temperature, relaxed towards cell
    # temperatures of almost motionless atoms, carries the transcendental
    # functions' last-bit differences to 1e-9
    E = engine_mod()
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True, renormalize=True)
    params, r, p, s = initial_state(20, seed=21, tilt=0.35, temperature=300.0, pos_sigma=0.05)
    prec = E.FP64 if precision == "fp64" else E.SPLIT
    tol = 1e-10 if precision == "fp64" else SPLIT_TOL
    e = E.Engine(params, r, p, s, precision=prec, **sw)
    o = orc.System(params, r, p, s, rng=orc.RNG_PHILOX, **sw)
    assert e.ncells == 13 ** 3 and e.ngroups == o.ngroups == 18
    for k in range(3):
        o.run(1)
        e.run(1)
        e.sync()
        errs = {n: relerr(e.get(n), o.get(n)) for n in ATOM + ["Te", "Ee", "Tl", "Ts_L", "Ts_R"]}
        print(f"{precision} step {k}: " + " ".join(f"{n} {v:.1e}" for n, v in errs.items()))
        _compare(e, o, ATOM + ["Te", "Ee", "Tl", "Ts_L", "Ts_R"], tol, f"{precision} step {k}")
    assert np.array_equal(e.cell_lists(), o.lists())
    e.close()


def test_nve_64cubed_one_step():
    E = engine_mod()
    params, r, p, s = initial_state(64, seed=22, tilt=0.05, temperature=300.0)
    e = E.Engine(params, r, p, s)
    o = orc.System(params, r, p, s, rng=orc.RNG_PHILOX)
    assert e.ncells == 44 ** 3 and e.ngroups == o.ngroups == 8
    _compare(e, o, ["f", "rho", "pe", "me"], 1e-11, "start")
    o.run(1)
    e.run(1)
    e.sync()
    _compare(e, o, ATOM, 1e-10, "step")
    assert np.array_equal(e.cell_lists(), o.lists())
    e.close()


def _bench_start_state():
    # the benchmark's 4.19M-atom start state (bench.py workload())
    params, r, p, s = initial_state(128, seed=2026, tilt=0.35, temperature=300.0)
    params["step"] = 0.5e-15
    te = hot_spot_te(16, params["box"][0], peak=3000.0, background=300.0, sigma=20.0)
    sw = dict(spinlang=True, lattlang=True, eltemp=True, localcolmot=True, renormalize=True,
              te_mesh=16)
    return params, r, p, s, te, sw


def test_bench_start_state_128cubed():
    E = engine_mod()
    params, r, p, s, te, sw = _bench_start_state()
    o = orc.System(params, r, p, s, te=te, rng=orc.RNG_PHILOX, **sw)
    assert o.ncells == 89 ** 3
    ref = {n: o.get(n) for n in ("f", "rho", "pe", "me", "me0", "Tl", "Ts_L", "Ts_R")}
    ngroups = o.ngroups
    del o
    for prec, tol in ((E.FP64, 1e-11), (E.SPLIT, SPLIT_TOL)):
        e = E.Engine(params, r, p, s, te=te, precision=prec, **sw)
        assert e.ngroups == ngroups
        for n, b in ref.items():
            # cell temperatures on a Te mesh are sums with atomics (order not
            # fixed): rounding-level differences in both forms
            t = max(tol, 1e-10) if n in ("Tl", "Ts_L", "Ts_R") else tol
            err = relerr(e.get(n), b)
            assert err <= t, f"precision {prec} {n}: rel err {err:.3e} > {t:.0e}"
        e.close()
