"""Learned warm start for the LBFGS minimiser.

A small convolutional network (``magnumaf.ConvNet``, trained with the library's
own CUDA kernels) maps an initial magnetisation and the material/field
parameters to a proposal for the relaxed state; LBFGS then finishes from the
proposal.  Plain LBFGS from the user's initial state stays both the fallback
(a proposal with non-finite values or a higher energy than the initial state
is discarded) and the arbiter: the minimiser's own stopping criteria decide when
a state is relaxed, and the final energy and residual torque max|m x H|/Ms are
reported for both starts.

Workload (thin film, 2 nm cells, one layer): exchange A, interface DMI D
(axis z), uniaxial anisotropy Ku (axis z), Zeeman field Bz along z, each drawn
uniformly per sample from PARAM_RANGES; the initial state is a smooth random
field (a few low Fourier modes).  Training pairs come from the GPU LBFGS run
from those initial states.

    python -m magnumaf.warmstart --n-train 512 --n-test 32 --mesh 64 64 --out result.json

The default network has 8 layers of width 16 with dilations 1, 2, 4, 8, 16, 32,
2, 1 (a receptive field of 133 cells, the whole 64 x 64 sample).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time
from typing import Dict, List

import numpy as np

import magnumaf as M

PARAM_RANGES = {
    "Ms": (5.0e5, 1.2e6),   # A/m
    "A": (1.0e-11, 2.0e-11),  # J/m
    "D": (1.0e-3, 4.0e-3),  # J/m^2
    "Ku": (5.0e5, 1.2e6),   # J/m^3
    "Bz": (0.0, 0.2),       # T
}
# the warm-start configuration of the benchmarks (128 x 128 cells of 2 nm): every
# parameter uniform per sample in these ranges, the initial state random on the
# unit sphere cell by cell
PARAM_RANGES_128 = {
    "Ms": (4.0e5, 1.2e6),
    "A": (0.5e-11, 2.0e-11),
    "D": (0.0, 4.0e-3),
    "Ku": (0.0, 1.2e6),
    "Bz": (-0.2, 0.2),
}
SCALE = {"Ms": 1e6, "A": 1e-11, "D": 1e-3, "Ku": 1e6, "Bz": 0.1}
KEYS = ["Ms", "A", "D", "Ku", "Bz"]
CIN = 3 + len(KEYS)
DX = 2e-9


def sample_params(rng, ranges=None) -> Dict[str, float]:
    ranges = ranges or PARAM_RANGES
    return {k: float(rng.uniform(*ranges[k])) for k in KEYS}


def random_sphere_m(rng, nx: int, ny: int) -> np.ndarray:
    """(nx, ny, 1, 3) unit vectors drawn uniformly on the sphere, cell by cell."""
    m = rng.normal(size=(nx, ny, 1, 3))
    return m / np.linalg.norm(m, axis=3, keepdims=True)


def smooth_random_m(rng, nx: int, ny: int, kmax: int = 4) -> np.ndarray:
    """(nx, ny, 1, 3) unit vectors from a sum of random low-order Fourier modes."""
    x = np.arange(nx)[:, None] / nx
    y = np.arange(ny)[None, :] / ny
    m = np.zeros((nx, ny, 3))
    for c in range(3):
        f = np.zeros((nx, ny))
        for kx in range(kmax + 1):
            for ky in range(kmax + 1):
                a, ph = rng.normal() / (1 + kx + ky), rng.uniform(0, 2 * math.pi)
                f += a * np.cos(2 * math.pi * (kx * x + ky * y) + ph)
        m[..., c] = f
    m /= np.linalg.norm(m, axis=2, keepdims=True)
    return m[:, :, None, :]


def terms_for(p: Dict[str, float]) -> list:
    return [M.ExchangeField(p["A"]), M.DmiField(p["D"]), M.UniaxialAnisotropyField(p["Ku"]),
            M.ExternalField.uniform(0.0, 0.0, p["Bz"] / M.Constants.mu0)]


def to_chw(m: np.ndarray) -> np.ndarray:
    """(nx, ny, 1, 3) -> [3][ny][nx]"""
    return np.ascontiguousarray(np.transpose(m[:, :, 0, :], (2, 1, 0)))


def from_chw(y: np.ndarray) -> np.ndarray:
    """[3][ny][nx] -> (nx, ny, 1, 3)"""
    return np.ascontiguousarray(np.transpose(y, (2, 1, 0))[:, :, None, :])


def features(m: np.ndarray, p: Dict[str, float]) -> np.ndarray:
    """[CIN][ny][nx] float32: m, then one constant map per scaled parameter."""
    mc = to_chw(m)
    maps = [np.full(mc.shape[1:], p[k] / SCALE[k]) for k in KEYS]
    return np.concatenate([mc, np.stack(maps)]).astype(np.float32)


def propose(net, m0: np.ndarray, p: Dict[str, float]) -> np.ndarray:
    """The network's proposal for the relaxed state of (m0, p), (nx, ny, 1, 3)."""
    import torch

    nx, ny = m0.shape[0], m0.shape[1]
    x = torch.from_numpy(features(m0, p)[None]).cuda()
    if isinstance(net, M.ConvNet):
        y = torch.empty((1, 3, ny, nx), dtype=torch.float32, device="cuda")
        net.forward(x.data_ptr(), 1, ny, nx, y.data_ptr())
        return from_chw(y[0].double().cpu().numpy())
    y = net.forward(x.data_ptr(), 1, ny, nx)  # U-net: [ny nx][3], pixel-major
    return np.ascontiguousarray(np.transpose(y.double().cpu().numpy().reshape(ny, nx, 3), (1, 0, 2))[:, :, None, :])


def relax(m0: np.ndarray, p: Dict[str, float], cnn=None, tol: float = 1e-6, maxiter: int = 1000):
    """LBFGS relaxation from m0, or from the network's proposal when cnn (a
    ConvNet or a UNet) is given.  Returns (m, info): info has E, iterations,
    fevals, torque = max|m x H|/Ms, seconds (network included), used_proposal."""
    import torch

    nx, ny = m0.shape[0], m0.shape[1]
    mesh = M.Mesh(nx, ny, 1, DX, DX, DX)
    terms = terms_for(p)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    start = m0
    used = False
    if cnn is not None:
        prop = propose(cnn, m0, p)
        if np.all(np.isfinite(prop)):
            s0 = M.State(mesh, p["Ms"], m0)
            s1 = M.State(mesh, p["Ms"], prop)
            e0 = sum(t.Energy_in_J(s0) for t in terms)
            e1 = sum(t.Energy_in_J(s1) for t in terms)
            if e1 <= e0:
                start, used = prop, True
    state = M.State(mesh, p["Ms"], start)
    mini = M.LBFGS_Minimizer(terms, tol=tol, maxiter=maxiter)
    E = mini.minimize(state)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    st = mini.stats()
    return np.asarray(state.m), {"E": E, "iterations": st["iterations"], "fevals": st["fevals"],
                                 "torque": st["grad_max"] / p["Ms"], "seconds": dt, "used_proposal": used}


def generate(n: int, nx: int, ny: int, seed: int, tol: float = 1e-6, maxiter: int = 1000, ranges=None,
             sphere: bool = False, workers: int = 1):
    """n samples (x [CIN][ny][nx], target [3][ny][nx], params, m0, info) relaxed by the GPU LBFGS.
    ranges: the parameter ranges (PARAM_RANGES by default); sphere: initial states
    random on the unit sphere cell by cell instead of smooth random fields."""
    rng = np.random.default_rng(seed)
    draws = []
    for _ in range(n):
        p = sample_params(rng, ranges)
        m0 = random_sphere_m(rng, nx, ny) if sphere else smooth_random_m(rng, nx, ny)
        draws.append((p, m0))
    # independent relaxations on their own states and streams, several at a time
    # (the seconds they report then include the others' GPU time)
    import concurrent.futures as cf

    with cf.ThreadPoolExecutor(max_workers=max(1, workers)) as ex:
        res = list(ex.map(lambda d: relax(d[1], d[0], None, tol, maxiter), draws))
    return [(features(m0, p), to_chw(m).astype(np.float32), p, m0, info) for (p, m0), (m, info) in zip(draws, res)]


def train(cnn, samples, steps: int, batch: int, lr: float, seed: int = 0) -> List[float]:
    """Adam on random minibatches; the dataset stays on the device.  Returns the losses.
    A UNet takes its targets pixel-major ([B H W][3])."""
    import torch

    X = torch.from_numpy(np.stack([s[0] for s in samples])).cuda()
    tg = np.stack([s[1] for s in samples])
    if not isinstance(cnn, M.ConvNet):
        tg = np.ascontiguousarray(np.transpose(tg, (0, 2, 3, 1)))
    T = torch.from_numpy(tg).cuda()
    n, _, H, W = X.shape
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    for k in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g).cuda()
        xb = X.index_select(0, idx).contiguous()
        tb = T.index_select(0, idx).contiguous()
        lr_k = lr * 0.5 * (1 + math.cos(math.pi * k / steps))
        losses.append(cnn.train_step(xb.data_ptr(), tb.data_ptr(), batch, H, W, lr_k))
    return losses


def evaluate(cnn: M.ConvNet, tests, tol: float = 1e-6, maxiter: int = 1000, plain_runs=None) -> dict:
    """Plain and warm-started LBFGS on each test sample; plain_runs (the info
    dicts of earlier plain relaxations of the same samples) skips the plain runs."""
    rows = []
    for i, (x, t, p, m0, _) in enumerate(tests):
        plain = plain_runs[i] if plain_runs is not None else relax(m0, p, None, tol, maxiter)[1]
        _, warm = relax(m0, p, cnn, tol, maxiter)
        rows.append((plain, warm))
    tp = sum(r[0]["seconds"] for r in rows)
    tw = sum(r[1]["seconds"] for r in rows)
    dE = [abs(r[1]["E"] - r[0]["E"]) / abs(r[0]["E"]) for r in rows]
    return {
        "samples": len(rows),
        "plain_seconds": tp, "warm_seconds": tw, "speedup": tp / tw,
        "plain_iterations": float(np.mean([r[0]["iterations"] for r in rows])),
        "warm_iterations": float(np.mean([r[1]["iterations"] for r in rows])),
        "proposals_used": int(sum(r[1]["used_proposal"] for r in rows)),
        "rel_energy_diff_median": float(np.median(dE)), "rel_energy_diff_max": float(np.max(dE)),
        "equal_energy_1e-6": float(np.mean([d <= 1e-6 for d in dE])),
        "warm_iterations_equal_energy": float(np.mean([r[1]["iterations"] for r, d in zip(rows, dE) if d <= 1e-6]
                                                      or [float("nan")])),
        "plain_iterations_equal_energy": float(np.mean([r[0]["iterations"] for r, d in zip(rows, dE) if d <= 1e-6]
                                                       or [float("nan")])),
        "torque_plain_max": float(max(r[0]["torque"] for r in rows)),
        "torque_warm_max": float(max(r[1]["torque"] for r in rows)),
    }


PRETRAINED_128 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_unet_128.npz")


def pretrained_unet():
    """The U-net trained by ``python -m magnumaf.warmstart --net unet --config128 --mesh 128 128
    --n-train 1200 --n-test 48 --steps 4000 --batch 16 --lr 2e-3 --maxiter 2000 --workers 6``
    (1200 GPU-LBFGS relaxations of 128 x 128 films, the configuration's parameter ranges,
    sphere-random initial states, seed 0)."""
    from .unet import UNet

    net = UNet(CIN, seed=0)
    net.set_params(np.load(PRETRAINED_128)["params"])
    return net


def gain(net, n: int, nx: int, ny: int, seed: int, tol: float = 1e-6, maxiter: int = 2000) -> dict:
    """Plain against warm-started LBFGS on n fresh samples of the 128 x 128
    configuration (seed not used in training), relaxed one at a time."""
    tests = generate(n, nx, ny, seed, tol=tol, maxiter=maxiter, ranges=PARAM_RANGES_128, sphere=True)
    res = evaluate(net, tests, tol=tol, maxiter=maxiter, plain_runs=[t[4] for t in tests])
    res["seed"] = seed
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-train", type=int, default=512)
    ap.add_argument("--n-test", type=int, default=32)
    ap.add_argument("--mesh", type=int, nargs=2, default=[64, 64])
    ap.add_argument("--net", choices=["convnet", "unet"], default="convnet")
    ap.add_argument("--config128", action="store_true",
                    help="the 128x128 configuration's parameter ranges and sphere-random initial states")
    ap.add_argument("--maxiter", type=int, default=1000)
    ap.add_argument("--workers", type=int, default=1, help="concurrent relaxations while generating training data")
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--width", type=int, default=16)
    ap.add_argument("--depth", type=int, default=8)
    # receptive field 1 + 2*(1+2+4+8+16+32+2+1) = 133 cells: the whole 64x64 sample
    ap.add_argument("--dilation", default="1,2,4,8,16,32,2,1",
                    help="comma-separated dilation per layer ('' for none)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--gain", type=int, default=0, metavar="N",
                    help="only evaluate the pretrained 128 x 128 U-net on N held-out samples (seed --gain-seed)")
    ap.add_argument("--gain-seed", type=int, default=50_000)
    a = ap.parse_args()
    if a.gain:
        res = gain(pretrained_unet(), a.gain, 128, 128, seed=a.gain_seed)
        print(json.dumps(res), flush=True)
        if a.out:
            with open(a.out, "w") as f:
                f.write(json.dumps(res) + "\n")
        return
    t0 = time.perf_counter()
    ranges = PARAM_RANGES_128 if a.config128 else None
    train_set = generate(a.n_train, a.mesh[0], a.mesh[1], a.seed, maxiter=a.maxiter, ranges=ranges,
                         sphere=a.config128, workers=a.workers)
    # held-out samples relaxed one at a time: their seconds are the plain method's wall time
    test_set = generate(a.n_test, a.mesh[0], a.mesh[1], a.seed + 10_000, maxiter=a.maxiter, ranges=ranges,
                        sphere=a.config128)
    t1 = time.perf_counter()
    if a.net == "unet":
        from .unet import UNet

        cnn = UNet(CIN, seed=a.seed)
        arch = {"net": "unet", "widths": list(cnn.widths), "layers": len(cnn.layers)}
    else:
        dil = [int(v) for v in a.dilation.split(",")] if a.dilation else None
        cnn = M.ConvNet(CIN, a.width, a.depth, seed=a.seed, dilation=dil)
        arch = {"net": "convnet", "width": a.width, "depth": a.depth, "dilation": cnn.dilation}
    losses = train(cnn, train_set, a.steps, a.batch, a.lr, a.seed)
    t2 = time.perf_counter()
    res = evaluate(cnn, test_set, maxiter=a.maxiter, plain_runs=[s[4] for s in test_set])
    res.update({"mesh": a.mesh, "n_train": a.n_train, "train_steps": a.steps, "batch": a.batch,
                "params": cnn.n_params, "config128": a.config128,
                "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-20:])),
                "generate_seconds": t1 - t0, "train_seconds": t2 - t1, **arch})
    line = json.dumps(res)
    print(line, flush=True)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")
        np.save(a.out + ".params.npy", cnn.get_params())


if __name__ == "__main__":
    main()
