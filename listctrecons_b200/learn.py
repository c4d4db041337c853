"""Learned 2.5D residual correction after backprojection (no reference counterpart).

Host side of the lct_cnn_* C ABI, training-pair generation on the GPU, training and evaluation.

Pairs: a seeded random-ellipsoid phantom (scan.Phantom.random) -> analytic helical fan-beam
line integrals with Poisson noise (lct_sim_project) -> FDK through lct_recon (the product path)
-> FDK volume; the target is the phantom voxelised on the FDK voxel grid (lct_voxelise; voxel
(ix, iy, k) of block b centred at ((ix - wx) dx, (iy - wy) dy, block_start_b + k dz dir)).

Plain FDK is the starting point: `plain = calib * fdk`, with `calib` the least-squares scale of the
training volumes onto their phantoms (the reference's FDK normalisation is about twice the
parallel-beam value).  The network sees in_scale * plain (in_scale = 1 / mu_water), predicts a
residual r, and the corrected volume is plain + r / in_scale wherever |r / in_scale| <= bound
(the acceptance gate), else plain.  Errors against the phantom are reported for both.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .recon import BLOCK_SLICES, Plan, Reconstruction
from .scan import MU_WATER, Phantom, ScanGeometry, simulate_gpu

N_PARAMS = 57249
CIN = (5, 32, 32, 32, 32, 32, 32, 32)
COUT = (32, 32, 32, 32, 32, 32, 32, 1)
# 1/mm: largest accepted |corrected - plain|.  On the learned configuration plain FDK is off by
# several mu_water where photons starve (40 overlapping ellipsoids, I0 = 1e5) and at pitch 1.5;
# a 2 mu_water gate rejects about 15% of the voxels and keeps little of the correction, 10 mu_water
# about 1% (the benchmark reports the sweep).
DEFAULT_BOUND = 10.0 * MU_WATER


def _torch():
    import torch

    return torch


def _stream():
    return _torch().cuda.current_stream().cuda_stream


def layer_slices():
    """(weight slice, bias slice, weight shape) of every layer in the flat parameter vector."""
    out, off = [], 0
    for cin, cout in zip(CIN, COUT):
        nw = cout * cin * 9
        out.append((slice(off, off + nw), slice(off + nw, off + nw + cout), (cout, cin, 3, 3)))
        off += nw + cout
    return out


class CNN:
    """lct_cnn: weights (FP32 master + Adam state) and a workspace for max_slices slices of
    ny x nx.  train=False keeps two activation buffers (inference only)."""

    def __init__(self, max_slices: int, ny: int, nx: int, train: bool = True, seed: int = 0):
        self._lib = capi.load()
        h = C.c_void_p()
        capi.check(self._lib.lct_cnn_create(max_slices, ny, nx, capi.CNN_TRAIN if train else 0,
                                            int(seed), C.byref(h)), "lct_cnn_create")
        self._h = h
        self.max_slices, self.ny, self.nx, self.train = max_slices, ny, nx, train

    # parameters --------------------------------------------------------------------------
    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, dtype=np.float32)
        capi.check(self._lib.lct_cnn_get_params(self._h, p.ctypes.data, 0), "lct_cnn_get_params")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters, got {p.size}")
        capi.check(self._lib.lct_cnn_set_params(self._h, p.ctypes.data, 0), "lct_cnn_set_params")

    def grads(self) -> np.ndarray:
        g = np.zeros(N_PARAMS, dtype=np.float32)
        capi.check(self._lib.lct_cnn_get_grads(self._h, g.ctypes.data, 0), "lct_cnn_get_grads")
        return g

    def set_scales(self, calib: float, in_scale: float) -> None:
        capi.check(self._lib.lct_cnn_set_scales(self._h, float(calib), float(in_scale)),
                   "lct_cnn_set_scales")

    def scales(self) -> tuple[float, float]:
        c, s = C.c_float(), C.c_float()
        capi.check(self._lib.lct_cnn_get_scales(self._h, C.byref(c), C.byref(s)))
        return c.value, s.value

    def copy_from(self, other: "CNN") -> None:
        self.set_params(other.params())
        self.set_scales(*other.scales())

    # training ----------------------------------------------------------------------------
    def forward(self, in5, resid=None):
        torch = _torch()
        n = in5.shape[0]
        if resid is None:
            resid = torch.empty((n, self.ny, self.nx), dtype=torch.float32, device=in5.device)
        capi.check(self._lib.lct_cnn_forward(self._h, in5.data_ptr(), n, resid.data_ptr(),
                                             _stream()), "lct_cnn_forward")
        return resid

    def backward(self, in5, target) -> None:
        capi.check(self._lib.lct_cnn_backward(self._h, in5.data_ptr(), target.data_ptr(),
                                              in5.shape[0], _stream()), "lct_cnn_backward")

    def adam_step(self, lr: float, beta1=0.9, beta2=0.999, eps=1e-8) -> None:
        capi.check(self._lib.lct_cnn_adam_step(self._h, lr, beta1, beta2, eps, _stream()),
                   "lct_cnn_adam_step")

    def train_step(self, in5, target, lr: float) -> None:
        capi.check(self._lib.lct_cnn_train_step(self._h, in5.data_ptr(), target.data_ptr(),
                                                in5.shape[0], lr, _stream()), "lct_cnn_train_step")

    def last_loss(self) -> float:
        v = C.c_double()
        capi.check(self._lib.lct_cnn_last_loss(self._h, C.byref(v)), "lct_cnn_last_loss")
        return v.value

    # inference ---------------------------------------------------------------------------
    def infer_volume(self, vol, bound: float = DEFAULT_BOUND, out=None, count: bool = True):
        """Corrected volume (phantom units) of a device FDK volume [nz][ny][nx]; returns
        (out, rejected voxel count or None)."""
        torch = _torch()
        if out is None:
            out = torch.empty_like(vol)
        n = C.c_int64()
        capi.check(self._lib.lct_cnn_infer_volume(self._h, vol.data_ptr(), out.data_ptr(),
                                                  vol.shape[0], float(bound),
                                                  C.byref(n) if count else None, _stream()),
                   "lct_cnn_infer_volume")
        return out, (n.value if count else None)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.lct_cnn_destroy(h)
            self._h = None


def voxelise_gpu(phantom: Phantom, nx, ny, nz, x0, y0, z0, dx, dy, dz, ss=4, out=None):
    """lct_voxelise into a CUDA tensor [nz][ny][nx]."""
    torch = _torch()
    ell = torch.as_tensor(np.ascontiguousarray(phantom.records), dtype=torch.float64, device="cuda")
    if out is None:
        out = torch.empty((nz, ny, nx), dtype=torch.float32, device="cuda")
    capi.check(capi.load().lct_voxelise(ell.data_ptr(), len(phantom.records), nx, ny, nz, x0, y0,
                                        z0, dx, dy, dz, ss, out.data_ptr(), _stream()),
               "lct_voxelise")
    return out


# ------------------------------------------------------------------------------------------
# training pairs
# ------------------------------------------------------------------------------------------
@dataclass
class PairSpec:
    geo: ScanGeometry          # readings and max_blocks already set
    n_ellipsoids: int = 40
    i0: float = 1e5
    semi: tuple = (5.0, 80.0)
    density: tuple = (0.0, 2.0)
    ss: int = 4                # voxelisation sub-samples per axis


# recon options of the training pairs and of the learned configuration: the mixed-precision path
# (tensor-core BF16x6 Toeplitz filter, FP64-geometry exact interpolation), Ram-Lak taps
def mixed_opts() -> dict:
    return dict(filter_mode=capi.FILTER_BF16X6, interp=capi.INTERP_EXACT,
                filter_kind=capi.FILTER_RAMLAK)


def pair_spec(ns=736, nt=64, ds=0.6, npt=1152, pitch=1.5, nx=256, dx=1.0, dz=1.0, nz=64,
              n_ellipsoids=40, i0=1e5) -> PairSpec:
    """A training geometry: scan length = the planner minimum for nz slices (nz / 32 blocks).
    The defaults are the 736 x 64 @ 0.6 mm, pitch 1.5, 256 x 256 x 64 @ 1 mm configuration."""
    geo = ScanGeometry(ns=ns, nt=nt, ds=ds, dt=ds, npt=npt, pitch=pitch, nx=nx, ny=nx, dx=dx,
                       dz=dz).with_blocks(nz // BLOCK_SLICES)
    return PairSpec(geo=geo, n_ellipsoids=n_ellipsoids, i0=i0)


class PairGenerator:
    """Seeded (FDK volume, voxelised phantom) pairs of one geometry, all on the GPU."""

    def __init__(self, spec: PairSpec, **recon_opts):
        torch = _torch()
        self.spec = spec
        self.plan = Plan(spec.geo)
        self.rec = Reconstruction(self.plan, **recon_opts)
        info = self.plan.info
        self.nb = info.n_blocks_run
        self.ig = info.ig
        self.blocks = self.plan.blocks[info.first_block: info.first_block + self.nb]
        zs = [b.block_start for b in self.blocks] + [b.block_end for b in self.blocks]
        self.z_lo, self.z_hi = min(zs), max(zs)
        self.fov = 0.5 * min(spec.geo.nx * spec.geo.dx, spec.geo.ny * spec.geo.dx)
        self.shape = self.rec.image_shape
        self.fan = torch.empty((self.rec.fan_count, spec.geo.nt, spec.geo.ns), dtype=torch.float32,
                               device="cuda")

    def phantom(self, seed: int) -> Phantom:
        s = self.spec
        return Phantom.random(s.n_ellipsoids, seed=seed, fov_radius=self.fov, z_lo=self.z_lo,
                              z_hi=self.z_hi, semi=s.semi, density=s.density)

    def target(self, ph: Phantom, out=None):
        torch = _torch()
        ig = self.ig
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device="cuda")
        for i, b in enumerate(self.blocks):
            zdir = 1.0 if b.block_end >= b.block_start else -1.0
            voxelise_gpu(ph, ig.nx, ig.ny, BLOCK_SLICES, -ig.wx * ig.dx, -ig.wy * ig.dy,
                         b.block_start, ig.dx, ig.dy, zdir * ig.dz, ss=self.spec.ss,
                         out=out[i * BLOCK_SLICES:(i + 1) * BLOCK_SLICES])
        return out

    def pair(self, seed: int):
        ph = self.phantom(seed)
        f0 = self.rec.fan_first
        simulate_gpu(self.spec.geo, ph, i0=self.spec.i0, seed=seed, v0=f0,
                     v1=f0 + self.rec.fan_count, out=self.fan)
        fdk = self.rec.run(self.fan, fan_view0=f0)
        return fdk, self.target(ph)


def stack5(vol, z):
    """[len(z)][5][ny][nx]: slices z-2..z+2 of vol (edge slices replicated)."""
    torch = _torch()
    z = torch.as_tensor(z, device=vol.device).long()
    idx = (z[:, None] + torch.arange(-2, 3, device=vol.device)[None, :]).clamp_(0, vol.shape[0] - 1)
    return vol[idx]


def fit_calibration(pairs) -> float:
    """Least-squares scale of FDK volumes onto their phantoms."""
    num = sum(float((f.double() * t.double()).sum()) for f, t in pairs)
    den = sum(float((f.double() * f.double()).sum()) for f, _ in pairs)
    return num / den


def sample_batch(pairs, n: int, rng: np.random.Generator):
    """n random (5-slice input, target slice) examples from the pair pool."""
    torch = _torch()
    ins, tgts = [], []
    which = rng.integers(0, len(pairs), size=n)
    for p in np.unique(which):
        fdk, tgt = pairs[p]
        z = rng.integers(0, fdk.shape[0], size=int((which == p).sum()))
        ins.append(stack5(fdk, z))
        tgts.append(tgt[torch.as_tensor(z, device=tgt.device).long()])
    return torch.cat(ins).contiguous(), torch.cat(tgts).contiguous()


def train(cnn: CNN, pairs, steps: int, batch: int, lr: float = 1e-3, seed: int = 0,
          lr_final: float | None = None, log_every: int = 0, log=print) -> list[float]:
    """Adam on random slices of the pair pool; cosine decay from lr to lr_final."""
    rng = np.random.default_rng(seed)
    losses = []
    lr_final = lr * 0.05 if lr_final is None else lr_final
    for it in range(steps):
        x, t = sample_batch(pairs, batch, rng)
        a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * it / max(steps - 1, 1)))
        cnn.train_step(x, t, float(a))
        if log_every and (it % log_every == 0 or it == steps - 1):
            losses.append(cnn.last_loss())
            log(f"step {it:5d}  lr {a:.2e}  loss {losses[-1]:.4e}")
    return losses


def errors(vol, target) -> dict:
    d = (vol.double() - target.double())
    return {"rmse": float(d.pow(2).mean().sqrt()),
            "rel_l2": float(d.norm() / target.double().norm())}


def plain_error_percentiles(pairs, calib: float, qs=(50.0, 90.0, 99.0, 99.9)) -> dict:
    """Percentiles of plain FDK's per-voxel error |calib * fdk - phantom|, in units of mu_water,
    over every voxel of the first 64 pairs."""
    torch = _torch()
    err = torch.cat([((f.double() * calib - t.double()).abs() / MU_WATER).flatten().float()
                     for f, t in pairs[:64]])
    # a seeded subsample keeps torch.quantile within its input-size limit
    if err.numel() > 8_000_000:
        g = torch.Generator(device=err.device).manual_seed(0)
        err = err[torch.randint(0, err.numel(), (8_000_000,), device=err.device, generator=g)]
    qv = torch.quantile(err, torch.tensor([q / 100.0 for q in qs], device=err.device))
    return {f"p{q:g}": float(v) for q, v in zip(qs, qv)}


def evaluate(cnn: CNN, pairs, bound: float = DEFAULT_BOUND) -> dict:
    """Error against the phantom of plain (calibrated) FDK and of the corrected volume."""
    calib, _ = cnn.scales()
    plain_se = corr_se = ref_sq = 0.0
    rejected = voxels = 0
    for fdk, tgt in pairs:
        out, rej = cnn.infer_volume(fdk, bound)
        t = tgt.double()
        plain_se += float((fdk.double() * calib - t).pow(2).sum())
        corr_se += float((out.double() - t).pow(2).sum())
        ref_sq += float(t.pow(2).sum())
        rejected += rej
        voxels += fdk.numel()
    return {"plain_rmse": (plain_se / voxels) ** 0.5, "corrected_rmse": (corr_se / voxels) ** 0.5,
            "plain_rel_l2": (plain_se / ref_sq) ** 0.5, "corrected_rel_l2": (corr_se / ref_sq) ** 0.5,
            "rejected_fraction": rejected / voxels, "bound": bound, "calib": calib,
            "volumes": len(pairs)}


# ------------------------------------------------------------------------------------------
# weights files and the training command
# ------------------------------------------------------------------------------------------
def save_weights(path, cnn: CNN, meta: dict, bound: float | None = None) -> None:
    import json
    from pathlib import Path

    calib, in_scale = cnn.scales()
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    extra = {} if bound is None else {"bound": np.float32(bound)}
    np.savez(path, params=cnn.params(), calib=np.float32(calib), in_scale=np.float32(in_scale),
             meta=np.array(json.dumps(meta)), **extra)


def load_weights(path) -> dict:
    """params, calib, in_scale, meta and the acceptance-gate bound stored with the network
    (1/mm; DEFAULT_BOUND for files that carry none)."""
    import json

    with np.load(path) as z:
        return {"params": z["params"].astype(np.float32), "calib": float(z["calib"]),
                "in_scale": float(z["in_scale"]), "meta": json.loads(str(z["meta"])),
                "bound": float(z["bound"]) if "bound" in z.files else DEFAULT_BOUND}


def cnn_from_weights(path, max_slices: int, ny: int, nx: int, train: bool = False) -> CNN:
    w = load_weights(path)
    c = CNN(max_slices, ny, nx, train=train)
    c.set_params(w["params"])
    c.set_scales(w["calib"], w["in_scale"])
    return c


def _train_main(argv=None) -> int:
    """python -m listctrecons_b200.learn train --out FILE [...]: seeded training pairs of the
    736 x 64 @ 0.6 mm, pitch 1.5, 256 x 256 x 64 @ 1 mm configuration (40 ellipsoids), Adam on
    the GPU, evaluation on held-out seeds; writes the weights and a JSON summary."""
    import argparse
    import json
    import time

    torch = _torch()
    ap = argparse.ArgumentParser(prog="python -m listctrecons_b200.learn train")
    ap.add_argument("--out", required=True)
    ap.add_argument("--pairs", type=int, default=256)
    ap.add_argument("--test-pairs", type=int, default=8)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--i0", type=float, default=1e5,
                    help="photons per ray: 1e5 starves where 40 overlapping ellipsoids stack up "
                         "(counts clamp at 1); 1e12 never clamps, so plain FDK's error is its "
                         "cone-beam / helical artefacts and blur")
    ap.add_argument("--gate-percentile", type=float, default=99.0,
                    help="acceptance-gate bound stored with the network: this percentile of "
                         "plain FDK's per-voxel error on the training pairs")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    spec = pair_spec(i0=a.i0)
    gen = PairGenerator(spec, **mixed_opts())
    t0 = time.perf_counter()
    pairs = [tuple(x.clone() for x in gen.pair(100000 * (a.seed + 1) + i)) for i in range(a.pairs)]
    test = [tuple(x.clone() for x in gen.pair(900000 + 1000 * a.seed + i))
            for i in range(a.test_pairs)]
    torch.cuda.synchronize()
    t_pairs = time.perf_counter() - t0
    _, H, W = gen.shape
    cnn = CNN(a.batch, H, W, train=True, seed=a.seed)
    cnn.set_scales(fit_calibration(pairs), 1.0 / MU_WATER)
    t0 = time.perf_counter()
    train(cnn, pairs, steps=a.steps, batch=a.batch, lr=a.lr, seed=a.seed, log_every=500)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    inf = CNN(32, H, W, train=False)
    inf.copy_from(cnn)
    calib = cnn.scales()[0]
    pct = plain_error_percentiles(pairs, calib, qs=(50.0, 90.0, a.gate_percentile, 99.9))
    bound = pct[f"p{a.gate_percentile:g}"] * MU_WATER
    meta = {
        "geometry": f"736x64@0.6mm, 1152 views/rot, pitch 1.5, 256x256x64@1mm, 40 ellipsoids, "
                    f"I0={a.i0:g}",
        "i0": a.i0,
        "plain_error_percentiles_mu_water": pct,
        "bound_per_mm": bound,
        "bound_rule": f"p{a.gate_percentile:g} of plain FDK's per-voxel error on the training "
                      "pairs: the correction may move a voxel as far as plain FDK's own errors "
                      "reach, no further",
        "recon": "scan mode, Ram-Lak, BF16x6 tensor-core filter, exact interpolation",
        "train_pairs": a.pairs, "train_seeds": f"{100000 * (a.seed + 1)}+i",
        "test_pairs": a.test_pairs, "test_seeds": f"{900000 + 1000 * a.seed}+i",
        "steps": a.steps, "batch_slices": a.batch, "lr": a.lr, "seed": a.seed,
        "pair_generation_s": t_pairs, "training_s": t_train,
        "eval_gated": evaluate(inf, test, bound=bound),
        "eval_ungated": evaluate(inf, test, bound=1e30),
    }
    save_weights(a.out, cnn, meta, bound=bound)
    print(json.dumps(meta), flush=True)
    return 0


def _infer_main(argv=None) -> int:
    """python -m listctrecons_b200.learn infer [...]: times lct_cnn_infer_volume on a seeded
    random device volume (CUDA events around each pass after one warm-up pass)."""
    import argparse
    import json

    torch = _torch()
    ap = argparse.ArgumentParser(prog="python -m listctrecons_b200.learn infer")
    ap.add_argument("--weights", default=None, help="weights file (default: He-init)")
    ap.add_argument("--nz", type=int, default=16)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--max-slices", type=int, default=16)
    ap.add_argument("--repeat", type=int, default=4)
    ap.add_argument("--bound", type=float, default=DEFAULT_BOUND / MU_WATER, help="x mu_water")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    g = torch.Generator(device="cuda").manual_seed(1)
    vol = torch.rand((a.nz, a.ny, a.nx), device="cuda", generator=g)
    out = torch.empty_like(vol)
    if a.weights:
        cnn = cnn_from_weights(a.weights, a.max_slices, a.ny, a.nx)
    else:
        cnn = CNN(a.max_slices, a.ny, a.nx, train=False)
        cnn.set_scales(0.5, 1.0 / MU_WATER)
    cnn.infer_volume(vol, a.bound * MU_WATER, out=out, count=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for _ in range(a.repeat):
        e0.record()
        cnn.infer_volume(vol, a.bound * MU_WATER, out=out, count=False)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    n = vol.numel()
    best = min(ms)
    print(json.dumps({"volume": [a.nz, a.ny, a.nx], "ms": best, "ms_all": ms,
                      "tflops": n * 114048 / best / 1e9}), flush=True)
    return 0


if __name__ == "__main__":
    import sys

    if len(sys.argv) > 1 and sys.argv[1] == "train":
        sys.exit(_train_main(sys.argv[2:]))
    if len(sys.argv) > 1 and sys.argv[1] == "infer":
        sys.exit(_infer_main(sys.argv[2:]))
    print("usage: python -m listctrecons_b200.learn train --out FILE [--pairs N] [--steps N]\n"
          "       python -m listctrecons_b200.learn infer [--nz N --ny N --nx N] [--weights F]")
    sys.exit(2)
