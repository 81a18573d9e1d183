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


def test_capped_sweep_grid_gives_the_same_bits(monkeypatch):
    # a cap on the sweep's CTAs per SM makes each thread walk several cells
    # of its colour group; the cells of a group are independent, so the
    # result is the same bit for bit.  96^3 unit cells: 66^3 link cells,
    # colour groups of 35,937 cells, more than one CTA per SM's threads
    from spilady_b200 import engine
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(96, seed=62, tilt=0.2)
    out = {}
    for cap in ("0", "1"):
        monkeypatch.setenv("SLD_SWEEP_CAP", cap)
        e = engine.Engine(params, r, p, s, spinlang=True, lattlang=True, precision=engine.SPLIT)
        assert e.ngroups == 8
        e.run(2)
        out[cap] = {n: e.get(n) for n in ("s", "H", "p")}
        e.close()
    for n in ("s", "H", "p"):
        assert np.array_equal(out["0"][n], out["1"][n]), n


def test_capped_side_branch_grids_give_the_same_bits(monkeypatch):
    # caps on the CTAs per SM of the sweeps, the pair pass and the EAM force
    # pass (each thread then takes several cells or atoms) change no
    # arithmetic: the step ends with the same bits
    from spilady_b200 import engine
    from spilady_b200.lattice import initial_state
    params, r, p, s = initial_state(48, seed=63, tilt=0.2)
    out = {}
    for caps in (("0", "0", "0"), ("2", "1", "1")):
        for name, v in zip(("SLD_SWEEP_CAP", "SLD_PAIR_CAP", "SLD_FORCE_CAP"), caps):
            monkeypatch.setenv(name, v)
        e = engine.Engine(params, r, p, s, spinlang=True, lattlang=True, precision=engine.SPLIT)
        e.run(2)
        out[caps] = {n: e.get(n) for n in ("s", "p", "r", "f", "rho")}
        e.close()
    a, b = out.values()
    for n in a:
        assert np.array_equal(a[n], b[n]), n
