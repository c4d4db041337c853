"""CPU checks of the learned-correction oracle (oracle/cnn_oracle.c): the forward pass against an
independent numpy restatement, the backward pass against central finite differences of the
loss (pure FP64 mode), and the bfloat16 rounding used at the GPU's storage points."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as orc  # noqa: E402


def _init_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    out = []
    for cin, cout in zip(orc.CNN_CIN, orc.CNN_COUT):
        std = scale * np.sqrt(2.0 / (9 * cin))
        out.append(rng.normal(0.0, std, size=cout * cin * 9))
        out.append(rng.normal(0.0, 0.05, size=cout))
    p = np.concatenate(out)
    assert p.size == orc.cnn_param_count()
    return p


def _np_forward(params, in5, k_in, bf16):
    """Independent restatement: zero-padded 3x3 cross-correlation, ReLU between layers."""
    def q(a):
        if not bf16:
            return a
        f = a.astype(np.float32).view(np.uint32).astype(np.uint64)
        f = (f + 0x7FFF + ((f >> 16) & 1)) & 0xFFFF0000
        return f.astype(np.uint32).view(np.float32).astype(np.float64)

    B, _, H, W = in5.shape
    a = q((np.float32(k_in) * in5.astype(np.float32)).astype(np.float64))  # [B][5][H][W]
    off = 0
    for l, (cin, cout) in enumerate(zip(orc.CNN_CIN, orc.CNN_COUT)):
        w = q(params[off: off + cout * cin * 9]).reshape(cout, cin, 3, 3)
        b = params[off + cout * cin * 9: off + cout * cin * 9 + cout]
        off += cout * cin * 9 + cout
        ap = np.pad(a, ((0, 0), (0, 0), (1, 1), (1, 1)))
        z = np.zeros((B, cout, H, W))
        for ky in range(3):
            for kx in range(3):
                z += np.einsum("oi,bihw->bohw", w[:, :, ky, kx], ap[:, :, ky: ky + H, kx: kx + W])
        z += b[None, :, None, None]
        a = q(np.maximum(z, 0.0)) if l < 7 else z
    return a[:, 0]


@pytest.mark.parametrize("bf16", [False, True])
def test_forward_matches_numpy(bf16):
    rng = np.random.default_rng(3)
    p = _init_params(1)
    x = rng.normal(0.5, 0.3, size=(2, 5, 9, 11)).astype(np.float32)
    r = orc.cnn_forward(p, x, k_in=1.7, bf16=bf16)
    ref = _np_forward(p, x, 1.7, bf16)
    tol = 1e-12 if not bf16 else 1e-6  # bf16: rounding ties may differ by the summation order
    assert np.max(np.abs(r - ref)) <= tol * max(1.0, np.max(np.abs(ref))), np.max(np.abs(r - ref))


def test_backward_finite_differences():
    rng = np.random.default_rng(5)
    p = _init_params(2)
    x = rng.normal(0.5, 0.3, size=(1, 5, 6, 7)).astype(np.float32)
    t = rng.normal(0.5, 0.3, size=(1, 6, 7)).astype(np.float32)
    k_in, s = 1.3, 0.9
    loss, g = orc.cnn_loss_grad(p, x, t, k_in, s, bf16=False)
    assert loss > 0
    # a sample of weights and biases in every layer
    idx, off = [], 0
    for cin, cout in zip(orc.CNN_CIN, orc.CNN_COUT):
        nw = cout * cin * 9
        idx += list(rng.choice(np.arange(off, off + nw), size=6, replace=False))
        idx += list(rng.choice(np.arange(off + nw, off + nw + cout), size=min(2, cout), replace=False))
        off += nw + cout
    fd, an = [], []
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = orc.cnn_loss_grad(pp, x, t, k_in, s, bf16=False)
        lm, _ = orc.cnn_loss_grad(pm, x, t, k_in, s, bf16=False)
        fd.append((lp - lm) / (2 * h))
        an.append(g[i])
    fd, an = np.array(fd), np.array(an)
    err = np.linalg.norm(fd - an) / np.linalg.norm(an)
    assert err < 1e-5, (err, fd, an)


def test_bf16_gradient_close_to_fp64():
    """The bf16 storage points perturb the gradient only at the bf16 level."""
    rng = np.random.default_rng(7)
    p = _init_params(3)
    x = rng.normal(0.5, 0.3, size=(1, 5, 8, 8)).astype(np.float32)
    t = rng.normal(0.5, 0.3, size=(1, 8, 8)).astype(np.float32)
    _, g64 = orc.cnn_loss_grad(p, x, t, 1.0, 1.0, bf16=False)
    _, g16 = orc.cnn_loss_grad(p, x, t, 1.0, 1.0, bf16=True)
    err = np.linalg.norm(g16 - g64) / np.linalg.norm(g64)
    assert 0 < err < 5e-2, err
