"""External field and force (control.h's extfield, extforce) against the
reference built with both, reading the same extfield.in / extforce.in files:
the main-loop body with its output calls, the files token by token and the
final state array by array."""
import numpy as np
import pytest

from conftest import relerr
from oracle import refjob as rj
from spilady_b200.lattice import initial_state
from test_gpu_output import compare_text, read_all

pytestmark = pytest.mark.gpu


def per_atom_file(v):
    lines = [str(len(v))] + [f"{i} {x:.17g} {y:.17g} {z:.17g}" for i, (x, y, z) in enumerate(v)]
    return "\n".join(lines) + "\n"


def test_external_field_and_force_match_reference(tmp_path):
    if not rj.available("extf"):
        pytest.skip("reference build missing")
    from spilady_b200 import engine
    params, r, p, s = initial_state(6, seed=41, tilt=0.3, temperature=300.0)
    rng = np.random.default_rng(41)
    H_tesla = rng.normal(0.0, 20.0, size=r.shape)        # a strong, uneven field
    f_ext = rng.normal(0.0, 0.05, size=r.shape)          # eV/A
    inputs = {"extfield.in": per_atom_file(H_tesla), "extforce.in": per_atom_file(f_ext)}
    for name, text in inputs.items():
        (tmp_path / name).write_text(text)
    nsteps = 3
    dumps, ref = rj.run("extf", params, r, p, s, ops=[(rj.OP_STEP, nsteps), (rj.OP_DUMP, 0)],
                        files=True, inputs=inputs)
    e = engine.Engine(params, r, p, s, interval_of_config_out=1)
    e.read_external_field(tmp_path / "extfield.in")
    e.read_external_force(tmp_path / "extforce.in")
    d = tmp_path / "out"
    d.mkdir()
    for k in range(nsteps):
        e.run(1)
        e.check(d, "b200", k)
        e.write_config(d, "b200", k, heff_as_reference=True)
    ours = read_all(d)
    assert sorted(ours) == sorted(n.replace("-ref", "-b200") for n in ref)
    worst = max(compare_text(ours[n], ref[n.replace("-b200", "-ref")], 1e-10, n) for n in ours)
    D = dumps[0]
    errs = {n: relerr(e.get(n), D.vec(n)) for n in ("r", "p", "f", "s", "H", "HL")}
    errs.update({n: relerr(e.get(n), D.a(n)) for n in ("pe", "me", "me0")})
    print("extf", " ".join(f"{k}:{v:.1e}" for k, v in errs.items()), f"files {worst:.1e}")
    for n, v in errs.items():
        assert v <= 1e-10, f"{n}: {v:.2e}"
    # removing both gives back the plain step
    e.set_external_field(None)
    e.set_external_force(None)
    plain = engine.Engine(params, r, p, s)
    e2 = engine.Engine(params, r, p, s)
    e2.set_external_field(np.zeros(r.shape))
    e2.set_external_force(np.zeros(r.shape))
    e2.set_external_field(None)
    e2.set_external_force(None)
    e2.run(2)
    plain.run(2)
    for n in ("r", "p", "s"):
        assert np.array_equal(e2.get(n), plain.get(n)), n
