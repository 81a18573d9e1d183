"""Failure reporting on the GPU: inputs that break the kernels' assumptions
end in an error code from the host, quickly, and never fault or trap."""
import numpy as np
import pytest

from spilady_b200.lattice import initial_state

pytestmark = pytest.mark.gpu


@pytest.mark.timeout(300)
def test_overfull_link_cell_reports_capacity():
    # every atom of a 6^3 box piled into one link cell: links flags the cell
    # (more than SLD_MAX_CELL_ATOMS), every per-cell walk stops at that bound,
    # and create returns SLD_ERR_CAPACITY instead of walking 432 atoms per
    # thread (or, at millions of atoms, sorting them in one thread)
    from spilady_b200 import engine
    params, r, p, s = initial_state(6, seed=1)
    rng = np.random.default_rng(3)
    r = rng.uniform(0.2, 1.2, size=r.shape)
    with pytest.raises(engine.SldError) as err:
        engine.Engine(params, r, p, s)
    assert err.value.code == -4



@pytest.mark.timeout(300)
def test_sweep_schedule_wait_runs_out_and_reports(monkeypatch):
    # The data-flow schedule of the spin sweeps (SLD_SWEEP_MODE=3) waits on
    # its neighbours' flags with a bounded number of polls.  Here every wait
    # asks for a tag that no warp writes (SLD_FLOW_STALL) with a small bound
    # (SLD_FLOW_POLLS): the kernel gives up, every warp leaves, and the host
    # reads SLD_ERR_TIMEOUT instead of the GPU hanging.  A fresh context then
    # steps as the oracle does.
    from oracle import orc
    from spilady_b200 import engine
    from conftest import relerr
    sw = dict(spinlang=True, lattlang=True)
    params, r, p, s = initial_state(6, seed=31, tilt=0.3)
    monkeypatch.setenv("SLD_SWEEP_MODE", "3")
    monkeypatch.setenv("SLD_FLOW_POLLS", "4096")
    monkeypatch.setenv("SLD_FLOW_STALL", "7")
    e = engine.Engine(params, r, p, s, **sw)
    with pytest.raises(engine.SldError) as err:
        e.run(1)
        e.sync()
    assert err.value.code == -10
    e.close()
    monkeypatch.delenv("SLD_FLOW_STALL")
    monkeypatch.delenv("SLD_FLOW_POLLS")
    e = engine.Engine(params, r, p, s, **sw)
    o = orc.System(params, r, p, s, rng=orc.RNG_PHILOX, **sw)
    e.run(2)
    o.run(2)
    e.sync()
    for n in ("r", "p", "s", "f"):
        assert relerr(e.get(n), o.get(n)) <= 1e-10, n
    e.close()


def test_entry_points_keep_the_callers_device():
    # every entry point makes its context's device current and gives the
    # caller's back: the context lives on the last device, the caller keeps
    # device 0 current throughout (with one GPU both are device 0)
    import torch
    from spilady_b200 import engine
    from conftest import relerr
    dev = torch.cuda.device_count() - 1
    params, r, p, s = initial_state(6, seed=32, tilt=0.3)
    torch.cuda.set_device(0)
    a = engine.Engine(params, r, p, s, device=dev, spinlang=True, lattlang=True)
    assert torch.cuda.current_device() == 0
    H = np.tile([0.0, 0.0, 0.01], (a.natom, 1))
    a.set_external_field(H)
    a.run(2)
    a.sync()
    assert torch.cuda.current_device() == 0
    b = engine.Engine(params, r, p, s, device=0, spinlang=True, lattlang=True)
    b.set_external_field(H)
    b.run(2)
    for n in ("r", "s"):
        assert relerr(a.get(n), b.get(n)) <= 1e-13, n
    assert torch.cuda.current_device() == 0
    a.close()
    b.close()
