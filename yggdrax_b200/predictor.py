"""Learned row-capacity predictor for the one-pass traversal.

A small MLP (12 -> 64 -> 64 -> 2, ReLU, fp32) maps per-node features of the
tree geometry to log2(1 + far row length) and log2(1 + near row length).
The traversal's ``"learned"`` mode sizes its rows from these predictions and
walks once instead of count-then-fill; rows that outgrow their prediction
are completed from a log, so the lists stay exact.  Features, inference,
training (forward / backward / Adam) and the capacity kernel are
hand-written CUDA (``csrc/predictor.cu``); this module drives them.

The package ships trained parameters (``predictor_weights.npz``: ``params``
plus the calibrated ``slack_far`` / ``slack_near`` / ``add``).  They were
produced by :func:`main` from plain-path traversals of uniform cubes,
Plummer spheres and Plummer-clump mixtures (seeds 100-299) and calibrated on
seeds 300-319.
"""

from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .dtypes import INDEX_BITS

N_INPUTS = 12
N_HIDDEN = 64
N_PARAMS = N_INPUTS * N_HIDDEN + N_HIDDEN + N_HIDDEN * N_HIDDEN + N_HIDDEN + N_HIDDEN * 2 + 2
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "predictor_weights.npz")
MAC_CODES = {"bh": 0, "dehnen": 1, "engblom": 2}

_DEFAULT: dict = {}


class Calibration(dict):
    """``slack_far`` / ``slack_near`` (log2 head-room added to the
    prediction) and ``add`` (entries added to every capacity)."""


def load_weights(path: str = WEIGHTS_PATH):
    """(params float32 [N_PARAMS], Calibration) from an ``.npz`` file."""
    z = np.load(path)
    params = np.asarray(z["params"], dtype=np.float32)
    if params.shape != (N_PARAMS,):
        raise ValueError(f"predictor weights have shape {params.shape}, expected ({N_PARAMS},)")
    cal = Calibration(slack_far=float(z["slack_far"]), slack_near=float(z["slack_near"]),
                      add=int(z["add"]))
    return params, cal


def save_weights(path: str, params, cal: dict, **extra) -> None:
    np.savez(path, params=np.asarray(params, dtype=np.float32),
             slack_far=np.float32(cal["slack_far"]), slack_near=np.float32(cal["slack_near"]),
             add=np.int32(cal["add"]), **extra)


def set_predictor(params, calibration: Optional[dict] = None) -> None:
    """Use these parameters (flat float32, N_PARAMS) and calibration for the
    learned traversal mode on every device (``None`` restores the shipped
    weights)."""
    _DEFAULT.clear()
    if params is None:
        _OVERRIDE.clear()
        return
    p = np.asarray(params.detach().cpu() if isinstance(params, torch.Tensor) else params,
                   dtype=np.float32).ravel()
    if p.shape != (N_PARAMS,):
        raise ValueError(f"predictor parameters have shape {p.shape}, expected ({N_PARAMS},)")
    cal = Calibration(slack_far=0.0, slack_near=0.0, add=8)
    cal.update(calibration or {})
    _OVERRIDE["params"], _OVERRIDE["cal"] = p, cal


_OVERRIDE: dict = {}


def default_predictor(dev):
    """The parameters in use on ``dev`` (cached) and their calibration."""
    key = str(dev)
    if _OVERRIDE and key not in _DEFAULT:
        _DEFAULT[key] = (torch.from_numpy(_OVERRIDE["params"]).to(dev), _OVERRIDE["cal"])
    if key not in _DEFAULT:
        if not os.path.exists(WEIGHTS_PATH):
            raise RuntimeError(f"no trained predictor weights at {WEIGHTS_PATH}; run "
                               "`python -m yggdrax_b200.predictor` on a GPU to train them")
        params, cal = load_weights()
        _DEFAULT[key] = (torch.from_numpy(params).to(dev), cal)
    return _DEFAULT[key]


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases, in the flat layout of the kernels."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((N_INPUTS, N_HIDDEN), (N_HIDDEN, N_HIDDEN), (N_HIDDEN, 2)):
        bound = math.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-bound, bound, (fan_in, fan_out)).astype(np.float32).ravel())
        parts.append(np.zeros(fan_out, np.float32))
    return np.concatenate(parts)


def node_features(topology, geometry, theta: float, mac_type: str) -> torch.Tensor:
    """(total, N_INPUTS) float32 features of every node (on the device)."""
    from .interactions import _root_of
    from .tree import _dev_of

    lib = L.lib()
    d = _dev_of(topology)
    total = int(topology.parent.shape[0])
    ni = int(topology.left_child.shape[0])
    dev = topology.parent.device
    root = _root_of(topology, d)
    X = torch.empty((total, N_INPUTS), dtype=torch.float32, device=dev)
    L.check(lib.ygx_node_features(
        L.ptr(geometry.center.contiguous().float()), L.ptr(geometry.radius.contiguous().float()),
        L.ptr(geometry.max_extent.contiguous().float()), L.ptr(d.level32), L.ptr(d.parent32),
        total, ni, L.ptr(topology.node_ranges.contiguous()), INDEX_BITS, root, float(theta),
        MAC_CODES[mac_type], L.ptr(X), L.stream_handle(dev)), "ygx_node_features")
    return X




def forward(params: torch.Tensor, X: torch.Tensor) -> torch.Tensor:
    """(n, 2) predictions of log2(1 + far length), log2(1 + near length)."""
    lib = L.lib()
    out = torch.empty((X.shape[0], 2), dtype=torch.float32, device=X.device)
    L.check(lib.ygx_mlp_forward(L.ptr(params), L.ptr(X.contiguous()), int(X.shape[0]),
                                L.ptr(out), L.stream_handle(X.device)), "ygx_mlp_forward")
    return out


def gradients(params: torch.Tensor, X: torch.Tensor, Y: torch.Tensor, mask: torch.Tensor):
    """Masked-MSE loss and its gradient w.r.t. the flat parameters."""
    lib = L.lib()
    dev = X.device
    B = int(X.shape[0])
    ws = L.workspace(lib.ygx_mlp_workspace_size(B), dev)
    grads = torch.empty(N_PARAMS, dtype=torch.float32, device=dev)
    loss = torch.empty(1, dtype=torch.float32, device=dev)
    L.check(lib.ygx_mlp_gradients(L.ptr(params), L.ptr(X.contiguous()), L.ptr(Y.contiguous()),
                                  L.ptr(mask.contiguous()), B, L.ptr(grads), L.ptr(loss),
                                  L.ptr(ws), ws.numel(), L.stream_handle(dev)),
            "ygx_mlp_gradients")
    return float(loss.item()), grads


def targets_of(topology, walk_far_counts, walk_near_counts, leafpos32):
    """Targets (log2(1 + length)) and mask for every node: far for all nodes,
    near for leaves."""
    total = int(topology.parent.shape[0])
    ni = int(topology.left_child.shape[0])
    dev = topology.parent.device
    Y = torch.zeros((total, 2), dtype=torch.float32, device=dev)
    M = torch.zeros((total, 2), dtype=torch.float32, device=dev)
    Y[:, 0] = torch.log2(1.0 + walk_far_counts.to(torch.float32))
    M[:, 0] = 1.0
    leaves = torch.arange(ni, total, device=dev)
    Y[ni:, 1] = torch.log2(1.0 + walk_near_counts.to(torch.float32)[leafpos32[leaves].long()])
    M[ni:, 1] = 1.0
    return Y, M


def train(X: torch.Tensor, Y: torch.Tensor, mask: torch.Tensor, *, steps: int = 6000,
          batch: int = 32768, lr: float = 2e-3, lr_end: float = 5e-5, seed: int = 0,
          params: Optional[np.ndarray] = None, log_every: int = 0) -> torch.Tensor:
    """Adam on random minibatches (cosine learning-rate decay); all device work
    in the library's training kernels."""
    lib = L.lib()
    dev = X.device
    n = int(X.shape[0])
    p = torch.from_numpy(init_params(seed) if params is None else params).to(dev)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    B = min(batch, n)
    ws = L.workspace(lib.ygx_mlp_workspace_size(B), dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    st = L.stream_handle(dev)
    for step in range(1, steps + 1):
        idx = torch.randint(0, n, (B,), device=dev, generator=gen)
        xb, yb, mb = X[idx].contiguous(), Y[idx].contiguous(), mask[idx].contiguous()
        cur = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * (step - 1) / steps))
        L.check(lib.ygx_mlp_train_step(L.ptr(p), L.ptr(m), L.ptr(v), step, float(cur),
                                       L.ptr(xb), L.ptr(yb), L.ptr(mb), B, L.ptr(loss),
                                       L.ptr(ws), ws.numel(), st), "ygx_mlp_train_step")
        if log_every and step % log_every == 0:
            print(f"step {step} loss {float(loss.item()):.4f} lr {cur:.2e}", flush=True)
    return p


def calibrate(pred: torch.Tensor, Y: torch.Tensor, mask: torch.Tensor, *,
              quantile: float = 0.95, add: int = 8) -> Calibration:
    """Per-output log2 slack such that `quantile` of the rows fit."""
    out = {}
    for j, name in enumerate(("slack_far", "slack_near")):
        sel = mask[:, j] > 0
        r = (Y[sel, j] - pred[sel, j]).float()
        out[name] = float(torch.quantile(r[:: max(1, r.numel() // 2_000_000)], quantile).item())
    return Calibration(add=add, **out)


def _dataset(seed: int):
    """One training configuration: a distribution of the C1-C3 kinds at a
    scaled-down size, a leaf size and a MAC."""
    from . import inputs

    rng = np.random.default_rng(seed)
    kind = ("uniform", "plummer", "clumps")[seed % 3]
    n = int(np.exp(rng.uniform(np.log(32768), np.log(4194304))))
    if kind == "uniform":
        pos, mass = inputs.uniform_cube(n, seed)
    elif kind == "plummer":
        pos, mass = inputs.plummer(n, seed)
    else:
        pos, mass = inputs.plummer_clumps(n, seed, clumps=int(rng.integers(4, 65)))
    leaf = int(rng.choice([16, 32]))
    mac, theta = [("dehnen", 0.6), ("dehnen", 0.5), ("bh", 0.5), ("dehnen", 0.7)][
        int(rng.integers(0, 4))]
    return pos, mass, leaf, mac, theta


def training_samples(seed: int, dev, max_nodes: int = 65536):
    """Features and exact row-length targets of one plain-path traversal."""
    import yggdrax_b200 as yb
    from .interactions import _leaf_ordering

    pos, mass, leaf, mac, theta = _dataset(seed)
    P = torch.from_numpy(pos).to(dev)
    M = torch.from_numpy(mass).to(dev)
    tree, ps = yb.build_tree(P, M, leaf_size=leaf, return_reordered=True)[:2]
    geom = yb.compute_tree_geometry(tree, ps)
    inter, nbrs = yb.build_interactions_and_neighbors(tree, geom, theta=theta, mac_type=mac)
    topo = tree.topology if hasattr(tree, "topology") else tree
    total = int(topo.parent.shape[0])
    ni = int(topo.left_child.shape[0])
    _, leafpos32, _, _ = _leaf_ordering(topo, total, ni, dev)
    X = node_features(topo, geom, theta, mac)
    Y, Mk = targets_of(topo, inter.counts, nbrs.counts, leafpos32)
    if total > max_nodes:  # a random subset keeps large systems from dominating
        g = torch.Generator(device=dev)
        g.manual_seed(seed)
        keep = torch.randperm(total, device=dev, generator=g)[:max_nodes]
        X, Y, Mk = X[keep], Y[keep], Mk[keep]
    return X, Y, Mk


def main(argv=None) -> int:
    """Train on seeds 100-299, calibrate on 300-319, write the weights file."""
    import argparse

    import yggdrax_b200 as yb

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=WEIGHTS_PATH)
    ap.add_argument("--train-seeds", default="100:300")
    ap.add_argument("--cal-seeds", default="300:320")
    ap.add_argument("--steps", type=int, default=10000)
    args = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    yb.set_reference_limits(False)
    yb.set_dense_neighbor_budget(1 << 28)

    def collect(spec):
        a, b = (int(x) for x in spec.split(":"))
        xs, ys, ms = [], [], []
        for s in range(a, b):
            X, Y, Mk = training_samples(s, dev)
            xs.append(X), ys.append(Y), ms.append(Mk)
        return torch.cat(xs), torch.cat(ys), torch.cat(ms)

    X, Y, Mk = collect(args.train_seeds)
    print(f"training samples: {X.shape[0]}", flush=True)
    p = train(X, Y, Mk, steps=args.steps, log_every=500)
    Xc, Yc, Mc = collect(args.cal_seeds)
    cal = calibrate(forward(p, Xc), Yc, Mc)
    loss_cal, _ = gradients(p, Xc, Yc, Mc)
    print(f"calibration: {dict(cal)}, held-out loss {loss_cal:.4f}", flush=True)
    save_weights(args.out, p.cpu().numpy(), cal, train_samples=np.int64(X.shape[0]),
                 heldout_loss=np.float32(loss_cal))
    print("wrote", args.out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
