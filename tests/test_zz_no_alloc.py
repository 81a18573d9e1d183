"""The allocation-free averages entry point (sld_averages_static).

Some callers cannot let this library allocate device memory: a code whose
device memory all comes from its own pool, or one that cannot afford
cudaFree (which waits for all device work) in the middle of its own
stream-ordered work.  For them sld_averages_static computes the averages of
sld_averages from caller-owned device arrays, keeping its partial sums in a
fixed device array compiled into the library.  This file is collected last
(pytest takes files in name order), so it runs both after the other GPU tests
and, with `pytest tests/test_zz_no_alloc.py`, alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("pe", "ke", "me", "me0", "Tl", "sx", "sy", "sz")
TOL = 1e-12     # relative; the two entry points sum in a different atom order


def _bind():
    from spilady_b200 import engine
    L = engine.lib()
    f = L.sld_averages_static
    f.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return engine, f


def test_static_averages_match_sld_averages_on_two_calls_in_a_row():
    import torch
    engine, f = _bind()
    from spilady_b200.lattice import initial_state

    params, r, p, s = initial_state(6, seed=21, tilt=0.3)
    e = engine.Engine(params, r, p, s, spinlang=True, lattlang=True)
    e.run(2)
    ref = e.averages()                      # the existing entry point
    want = np.array([ref[k] for k in KEYS])
    dev = torch.device("cuda", 0)
    arrays = [torch.tensor(e.get(n), dtype=torch.float64, device=dev).contiguous()
              for n in ("pe", "ke", "me", "me0", "s")]
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        out = torch.full((8,), float("nan"), dtype=torch.float64, device=dev)
        rc = f(*[a.data_ptr() for a in arrays], e.natom, out.data_ptr(), stream)
        assert rc == 0, f"call {call}: rc {rc}"
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        err = np.abs(got - want) / np.maximum(np.abs(want), 1e-30)
        assert np.all(err <= TOL), f"call {call}: {dict(zip(KEYS, err))}"
    e.close()


def test_static_averages_refuse_sizes_beyond_the_fixed_scratch():
    import torch
    engine, f = _bind()
    dev = torch.device("cuda", 0)
    a = torch.zeros(8, dtype=torch.float64, device=dev)
    out = torch.zeros(8, dtype=torch.float64, device=dev)
    limit = 8388608                          # SLD_AVERAGES_STATIC_MAX_ATOMS
    p = a.data_ptr()
    assert f(p, p, p, p, p, limit + 1, out.data_ptr(), None) == -4    # SLD_ERR_CAPACITY
    assert f(p, p, p, p, p, 0, out.data_ptr(), None) == -1            # SLD_ERR_ARG
    assert np.all(out.cpu().numpy() == 0.0)  # nothing was launched
