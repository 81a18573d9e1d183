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

