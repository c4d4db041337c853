"""The backprojector's polynomial asin (asin_half in csrc/backproject_quad.cu) against the FP64
arcsin on its domain |x| <= 0.5.

The coefficients are read from the kernel source, and the evaluation repeats the kernel's
float32 operations: round-to-nearest products and fused multiply-adds (emulated in FP64 and
rounded once, which is exact for float32 operands).  Bar: within 1 ulp everywhere on the
domain."""
import re
from pathlib import Path

import numpy as np

SRC = Path(__file__).resolve().parent.parent / "listctrecons_b200" / "csrc" / "backproject_quad.cu"


def _coefficients():
    src = SRC.read_text()
    body = src[src.index("float asin_half(float x)"):]
    body = body[: body.index("}")]
    lits = [float(v) for v in re.findall(r"(\d+\.\d+)f", body)]
    assert len(lits) == 5, lits
    # fmaf(fmaf(fmaf(fmaf(c4, t, c3), t, c2), t, c1), t, c0): literals appear as c4, c3, c2, c1, c0
    return [np.float32(v) for v in lits]


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def test_asin_half_within_one_ulp():
    c4, c3, c2, c1, c0 = _coefficients()
    x = np.linspace(-0.5, 0.5, 400001, dtype=np.float32)
    t = (x * x).astype(np.float32)
    p = np.full_like(t, c4)
    for c in (c3, c2, c1, c0):
        p = _fma32(p, t, np.full_like(t, c))
    got = _fma32((x * t).astype(np.float32), p, x)
    ref = np.arcsin(x.astype(np.float64))
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    err = np.abs(got.astype(np.float64) - ref) / ulp
    assert err.max() <= 1.0, err.max()
    assert np.all(np.sign(got) == np.sign(x))
