"""Long runs against the reference's own (tests/golden/long_runs_ref.npz,
made by ``tests/golden/make_golden.py long`` from the reference's CPU build):

- NVE energy drift: 1,000 steps of 1 fs, bcc Fe 16^3 cells; the largest
  departure of the total energy per atom from its start may not exceed the
  reference's by more than a factor stated below;
- Langevin equilibrium: 3,000 steps at 300 K, 10^3 cells; the noise streams
  differ, so the averages of Tl, Ts_R, Ts_L and |<m>| over steps 1,000-3,000
  are compared within error bars, estimated from eight engine replicas with
  independent noise.

Both runs print through sld_check, the same lines the reference prints.
"""
import numpy as np
import pytest

from conftest import load_golden
from spilady_b200.lattice import initial_state

pytestmark = pytest.mark.gpu


def engine_mod():
    from spilady_b200 import engine
    return engine


def lines(path):
    return np.array([[float(x) for x in l.split()] for l in open(path) if l.strip()])


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_nve_energy_drift_no_worse_than_reference(precision, tmp_path):
    E = engine_mod()
    g = load_golden("long_runs_ref")
    ref = g["nve_E"]
    params, r, p, s = initial_state(16, seed=4, tilt=0.05, temperature=300.0)
    prec = E.FP64 if precision == "fp64" else E.SPLIT
    e = E.Engine(params, r, p, s, precision=prec)
    for k in range(int(g["nve_steps"])):
        e.run(1)
        e.check(tmp_path, "b200", k)
    enr = lines(tmp_path / "enr-b200.dat")
    ours = enr[:, 2] + enr[:, 3] + enr[:, 4] + enr[:, 5]
    d_ref = np.max(np.abs(ref - ref[0]))
    d_ours = np.max(np.abs(ours - ours[0]))
    print(f"{precision}: max |E - E0| per atom {d_ours:.2e} eV, reference {d_ref:.2e} eV")
    # the FP64 form is the reference's arithmetic; the split form's FP32
    # forces add their own rounding to the energy's fluctuation
    limit = 1.5 if precision == "fp64" else 2.0
    assert d_ours <= limit * d_ref


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_langevin_equilibrium_matches_reference(precision, tmp_path):
    # the split form too: FP32 pair terms and fields, FP32 Box-Muller normals
    E = engine_mod()
    g = load_golden("long_runs_ref")
    n = int(g["lang_steps"])
    params, r, p, s = initial_state(10, seed=7, tilt=0.05, temperature=300.0)
    reps = 8
    prec = E.FP64 if precision == "fp64" else E.SPLIT
    engines = [E.Engine(params, r, p, s, spinlang=True, lattlang=True, replica=k, precision=prec)
               for k in range(reps)]
    batch = E.Batch(engines)
    for k in range(n):
        batch.run(1)
        for q, e in enumerate(engines):
            e.check(tmp_path, f"r{q}", k)
    batch.close()
    window = slice(1000, n)
    cols = {"Tl": ("tmp", 2, "lang_Tl"), "Ts_R": ("tmp", 3, "lang_TsR"),
            "Ts_L": ("tmp", 4, "lang_TsL"), "|m|": ("spn", 9, "lang_m")}
    for name, (f, c, key) in cols.items():
        ours = np.array([lines(tmp_path / f"{f}-r{q}.dat")[window, c].mean() for q in range(reps)])
        theirs = g[key][window].mean()
        spread = ours.std(ddof=1)
        # one reference realisation against the mean of eight: the standard
        # deviation of their difference is spread * sqrt(1 + 1/8)
        z = abs(theirs - ours.mean()) / (spread * np.sqrt(1.0 + 1.0 / reps))
        print(f"{precision} {name}: engine {ours.mean():.3f} +- {spread:.3f}, reference "
              f"{theirs:.3f}, z {z:.2f}")
        assert z <= 4.0, f"{name}: {z:.2f} standard deviations apart"
