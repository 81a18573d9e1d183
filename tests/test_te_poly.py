"""The fitted heat-capacity functions of the split form (te_poly.h, made by
spilady_b200/csrc/gen_te_poly.py) against the model they replace
(heatcapacity_CPU.cpp:33-57) evaluated in 40-digit arithmetic."""
import os
import re

import mpmath as mp
import numpy as np

HDR = os.path.join(os.path.dirname(__file__), "..", "spilady_b200", "csrc", "te_poly.h")


def _polys():
    text = open(HDR).read()
    out = {}
    for name in ("te_poly_logcosh", "te_poly_inv_logcosh", "te_poly_coth"):
        body = text[text.index(f"double {name}(double t)"):]
        body = body[:body.index("return p;")]
        coef = [float(x) for x in re.findall(r"([-+0-9.e]+)\)?;", body)]
        mid = float(re.search(rf"#define {name}_MID ([-+0-9.e]+)", text).group(1))
        inv = float(re.search(rf"#define {name}_INV_HALF ([-+0-9.e]+)", text).group(1))
        out[name] = (coef, mid, inv)   # coef[0] is the leading coefficient
    out["u_max"] = float(re.search(r"#define TE_U_MAX ([-+0-9.e]+)", text).group(1))
    return out


def _horner64(coef, t):
    p = np.float64(coef[0])
    for c in coef[1:]:
        p = p * t + c
    return p


def test_fitted_forms_are_within_two_ulp():
    mp.mp.dps = 40
    P = _polys()
    rng = np.random.default_rng(5)
    u = np.concatenate([rng.uniform(0.0, P["u_max"], 300), [1e-6, 0.06, 0.6, P["u_max"]]])
    worst = {}
    for ui in u:
        v = ui * ui
        c, mid, inv = P["te_poly_logcosh"]
        y = v * _horner64(c, (v - mid) * inv)
        ref = mp.log(mp.cosh(mp.mpf(ui)))
        worst["logcosh"] = max(worst.get("logcosh", 0), abs(float((y - ref) / ref)))
        yr = float(ref)
        c, mid, inv = P["te_poly_inv_logcosh"]
        uu = np.sqrt(yr * _horner64(c, (yr - mid) * inv))
        worst["inverse"] = max(worst.get("inverse", 0), abs(uu - ui) / ui)
        c, mid, inv = P["te_poly_coth"]
        co = 1.0 / ui + ui * _horner64(c, (v - mid) * inv)
        ref = mp.coth(mp.mpf(ui))
        worst["coth"] = max(worst.get("coth", 0), abs(float((co - ref) / ref)))
    # float64 Horner without fused multiply-adds, the square root and the
    # input rounding: a few ulp
    assert worst["logcosh"] < 6e-16, worst
    assert worst["coth"] < 6e-16, worst
    assert worst["inverse"] < 1e-15, worst
