"""Batched replicas (sld_batch_*): systems of different sizes, temperatures
and noise streams advanced together end exactly as each would alone."""
import numpy as np
import pytest

from spilady_b200.lattice import initial_state

pytestmark = pytest.mark.gpu

SW = dict(spinlang=True, lattlang=True, localcolmot=True)


def _replicas(precision):
    from spilady_b200 import engine
    out = []
    for k, (edge, temp) in enumerate([(6, 150.0), (7, 600.0), (8, 1100.0)]):
        params, r, p, s = initial_state(edge, seed=30 + k, tilt=0.2, temperature=temp)
        params["temperature"] = temp
        out.append(engine.Engine(params, r, p, s, precision=precision, replica=k + 1, **SW))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_each_replica_alone(precision):
    from spilady_b200 import engine
    alone = _replicas(precision)
    for e in alone:
        e.run(5)
    batched = _replicas(precision)
    b = engine.Batch(batched)
    b.run(2)
    batched[1].run(1)          # a replica stepped on its own between batch runs
    b.run(2)
    batched[0].run(1)
    batched[2].run(1)          # every replica has now taken 5 steps
    b.close()
    for k, (a, e) in enumerate(zip(alone, batched)):
        for n in ("r", "p", "s", "f"):
            assert np.array_equal(a.get(n), e.get(n)), f"replica {k} {n}"


def test_replicas_draw_different_noise():
    from spilady_b200 import engine
    params, r, p, s = initial_state(6, seed=40, tilt=0.2)
    a = engine.Engine(params, r, p, s, replica=1, **SW)
    b = engine.Engine(params, r, p, s, replica=2, **SW)
    a.run(1)
    b.run(1)
    assert not np.array_equal(a.get("p"), b.get("p"))


def test_autotune_keeps_the_state_and_the_results():
    # launch shapes change no arithmetic (a thread per cell or atom whatever
    # the block), so the tuned context steps on with the same bits
    from spilady_b200 import engine
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(8, seed=61, tilt=0.2)
    a = engine.Engine(params, r, p, s, spinlang=True, lattlang=True, precision=engine.SPLIT)
    b = engine.Engine(params, r, p, s, spinlang=True, lattlang=True, precision=engine.SPLIT)
    a.run(2)
    b.run(2)
    shapes = a.autotune(steps=2)
    assert shapes["sweep_block"] in (0, 64, 96, 128)
    for n in ("r", "p", "s"):
        assert np.array_equal(a.get(n), b.get(n)), n
    a.run(3)
    b.run(3)
    for n in ("r", "p", "s", "f"):
        assert np.array_equal(a.get(n), b.get(n)), n
