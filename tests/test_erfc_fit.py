"""The erfc approximation of the pair kernel (blade_b200/csrc/erfc_fit.h, an
own fit of Hastings' form erfc(x) = exp(-x^2) P6(1/(1 + p x)); no reference
coefficients): the polynomial evaluated in FP32 with the kernel's even/odd
FMA order against FP64 erfc over the whole range the path uses, x = beta r in
[0, beta rCut] for beta rCut up to 6."""
import os
import re

import numpy as np
from scipy.special import erfcx

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "blade_b200", "csrc", "erfc_fit.h")
MAX_REL = 1.0e-6   # FP32 evaluation of erfc(x) exp(x^2)


def _coefficients():
    text = open(HEADER).read()
    v = {m.group(1): np.float32(float(m.group(2))) for m in re.finditer(r"kErfc(\w+) = ([-0-9.e+]+)f", text)}
    return v["P"], [v[f"C{k}"] for k in range(7)]


def _fma(a, b, c):
    """FP32 fused multiply-add (the product is exact in FP64)."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def test_erfcx_polynomial_in_fp32():
    p, c = _coefficients()
    x = np.linspace(0.0, 6.0, 200001).astype(np.float32)
    t = (np.float32(1) / _fma(np.full_like(x, p), x, np.ones_like(x))).astype(np.float32)
    t2 = (t * t).astype(np.float32)
    f = lambda v: np.full_like(t, v)
    pe = _fma(f(c[6]), t2, f(c[4]))
    pe = _fma(pe, t2, f(c[2]))
    pe = _fma(pe, t2, f(c[0]))
    po = _fma(f(c[5]), t2, f(c[3]))
    po = _fma(po, t2, f(c[1]))
    val = _fma(po, t, pe)
    rel = np.abs(val.astype(np.float64) / erfcx(x.astype(np.float64)) - 1)
    assert rel.max() <= MAX_REL, rel.max()
