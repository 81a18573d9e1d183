"""The drop-in on the reference's own driver: SPILADY's unmodified main loop
(spilady.cpp:43-62, calling core.cpp:31-76 and check.cpp:31-47) linked with
oracle/ref/core_B200.cpp, which backs the step functions with the engine's C
ABI (include/sld.h), against the same main loop on the reference's own CPU
step functions.  Both read the same variables.in and configuration file
(read_variables.cpp, read_config.cpp), run three NVE steps and write their
enr-/tmp-/str-/prs-/spn- files and final configuration with the reference's
own output code; the files agree to 1e-10 relative, column by column.

The binaries come from oracle/ref/build.sh (modes main_nve and b200_nve).
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import orc, refjob
from spilady_b200.lattice import initial_state

pytestmark = pytest.mark.gpu

NSTEPS = 3


def write_inputs(d, params, o, r, p, s):
    """variables.in and the configuration file, with the start state's
    forces, densities and energies (the reference's own arithmetic, from the
    oracle), as read_config expects them (read_config.cpp:39-116)."""
    n = r.shape[0]
    f, rho, ke, pe = o.get("f"), o.get("rho"), o.get("ke"), o.get("pe")
    H, HL, me, me0, st = o.get("H"), o.get("HL"), o.get("me"), o.get("me0"), o.get("stress")
    box = params["box"]
    lv = box[0] * box[2] * box[5] / n
    g = lambda x: "%.17g" % x
    with open(os.path.join(d, "con-start.in"), "w") as fh:
        fh.write(f"{n} 0 SLDHL\n{g(box[0])} {g(box[1])} {g(box[2])}\n"
                 f"{g(box[3])} {g(box[4])} {g(box[5])}\n")
        for i in range(n):
            s0 = float(np.sqrt(np.sum(s[i] ** 2)))
            cols = ([*r[i], *p[i], *f[i], *st[i], rho[i], ke[i], pe[i], *s[i], s0, *H[i], *HL[i],
                     me[i], me0[i], lv])
            fh.write(f"{i} Fe " + " ".join(g(x) for x in cols) + "\n")
    keys = {"out_body": "dropin", "no_of_production_steps": NSTEPS, "step": params["step"],
            "interval_of_print_out": 1, "interval_of_config_out": 100000,
            "interval_of_vsim": 100000, "in_config": "con-start.in",
            "temperature": params["temperature"], "atmass": params["atmass"],
            "random_seed": params["random_seed"], "rcut_pot": params["rcut_pot"],
            "rcut_mag": params["rcut_mag"], "rcut_max": params["rcut_max"],
            "min_length_link_cell": params["min_length_link_cell"], "OMP_threads": 1}
    with open(os.path.join(d, "variables.in"), "w") as fh:
        for k, v in keys.items():
            fh.write(f"{k} {v}\n")


def run_main(binary, d):
    res = subprocess.run([binary], cwd=d, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]


def columns(path):
    return np.array([[float(x) for x in line.split()] for line in open(path) if line.strip()])


@pytest.mark.skipif(not (refjob.available("main_nve") and refjob.available("b200_nve")),
                    reason="reference builds missing (sh oracle/ref/build.sh)")
def test_reference_main_loop_on_the_engine(tmp_path):
    params, r, p, s = initial_state(6, seed=41, tilt=0.3, temperature=300.0, pos_sigma=0.05)
    o = orc.System(params, r, p, s, rng=orc.RNG_MWC)
    stock, b200 = tmp_path / "stock", tmp_path / "b200"
    for d in (stock, b200):
        d.mkdir()
        write_inputs(str(d), params, o, r, p, s)
    run_main(refjob.binary("main_nve"), str(stock))
    run_main(refjob.binary("b200_nve"), str(b200))
    for kind in ("enr", "tmp", "str", "prs", "spn"):
        a = columns(stock / f"{kind}-dropin.dat")
        b = columns(b200 / f"{kind}-dropin.dat")
        # the start's line (step -1, written before the loop) and one per step
        assert a.shape == b.shape and a.shape[0] == NSTEPS + 1, kind
        scale = np.maximum(np.abs(a), 1e-300)
        err = np.max(np.abs(b - a) / np.maximum(scale, np.max(np.abs(a), axis=0) * 1e-6))
        assert err <= 1e-10, f"{kind}: {err:.3e}"
    ends = sorted(x.name for x in stock.iterdir() if x.name.startswith("con-dropin"))
    assert ends, "no configuration written"
    for name in ends:
        a = np.loadtxt(stock / name, skiprows=3, usecols=range(2, 8))
        b = np.loadtxt(b200 / name, skiprows=3, usecols=range(2, 8))
        err = np.max(np.abs(b - a)) / np.max(np.abs(a))
        assert err <= 1e-10, f"{name}: {err:.3e}"
