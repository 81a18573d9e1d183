"""The quantum thermostat (control.h's quantumnoise): its filter against the
reference's own (initial_quantum_noise, read from the reference built with
quantumnoise) and against the oracle; the dynamics against the oracle with
the same counter-based normals, number for number."""
import numpy as np
import pytest

from conftest import relerr
from oracle import orc
from oracle import refjob as rj
from spilady_b200.lattice import initial_state

pytestmark = pytest.mark.gpu

Q = dict(quantum_noise=True, msteps_quantum=2, nfrequency_quantum=8)


def test_quantum_filter_is_the_references():
    from spilady_b200 import engine
    params, r, p, s = initial_state(6, seed=51)
    e = engine.Engine(params, r, p, s, lattlang=True, **Q)
    h = e.quantum_filter()
    o = orc.System(params, r, p, s, lattlang=True, quantum=True, msteps_quantum=2,
                   nfrequency_quantum=8)
    assert np.array_equal(h, o.quantum_filter())
    if rj.available("quant"):
        ops = rj.set_ops(Msteps_quantum=2, Nfrequency_quantum=8) + [(rj.OP_QINIT, 0),
                                                                    (rj.OP_QFILTER, 0)]
        _, t = rj.run("quant", params, r, p, s, ops=ops, files=True)
        ref = np.array([float(x) for x in t["qfilter.dat"].split()])
        assert np.array_equal(h, ref)


@pytest.mark.parametrize("sw", [dict(lattlang=True), dict(lattlang=True, spinlang=True,
                                                           localcolmot=True)],
                         ids=["lattice", "spin-lattice-localcolmot"])
def test_quantum_dynamics_match_oracle(sw):
    from spilady_b200 import engine
    params, r, p, s = initial_state(6, seed=52, tilt=0.3)
    e = engine.Engine(params, r, p, s, **sw, **Q)
    o = orc.System(params, r, p, s, rng=orc.RNG_PHILOX, quantum=True, msteps_quantum=2,
                   nfrequency_quantum=8, **sw)
    for k in range(6):     # the noise changes every other kick: three updates
        e.run(1)
        o.run(1)
        for name in ("r", "p", "s"):
            err = relerr(e.get(name), o.get(name))
            assert err <= 1e-10, f"step {k} {name}: {err:.2e}"
