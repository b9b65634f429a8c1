"""Row-nnz predictor for the learned sparse product.

A 5 -> 64 -> 64 -> 1 MLP (ReLU, FP32) predicts log2(1 + output nnz) of each
C-tile row from five features of the row (log2 of the A-row nnz over all
stages, of the row's intermediate products and of its longest referenced B
row, and the tile's row/column coordinates).  Training data are the exact
per-row counts of the symbolic phase; training and inference run in the
library's own CUDA kernels (bclx_mlp_train / bclx_mlp_predict).  The learned
product (bclx_spgemm_learned_run) uses the predictions to cut heavy rows into
accumulator-sized items without a symbolic pass; rows it mispredicts are
redone by the exact two-phase path, so results never change.
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, List, Optional, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import call

IN = 5


def num_params() -> int:
    return int(_lib.load().bclx_mlp_num_params())


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases, in the kernels' layout; the output bias
    starts at 8 (log2 counts of a few hundred)."""
    rng = np.random.default_rng(seed)
    W1 = rng.standard_normal((5, 64)) * np.sqrt(2 / 5)
    W2 = rng.standard_normal((64, 64)) * np.sqrt(2 / 64)
    w3 = rng.standard_normal(64) * np.sqrt(1 / 64)
    p = np.concatenate([W1.ravel(), np.zeros(64), W2.ravel(), np.zeros(64), w3, [8.0]]).astype(np.float32)
    assert p.size == num_params()
    return p


class RowNnzPredictor:
    """Parameters live on the device; fit() and predict() run the CUDA kernels."""

    def __init__(self, params: Optional[np.ndarray] = None, seed: int = 0, device: Optional[int] = None):
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        dev = torch.cuda.current_device() if device is None else device
        self.params = torch.from_numpy(p.copy()).to(torch.device("cuda", dev))
        self.device = dev

    def _ctx(self):
        from .containers import context
        return context(self.device).use_current_stream()

    def fit(self, X: torch.Tensor, y: torch.Tensor, steps: int = 400, lr: float = 3e-3) -> np.ndarray:
        """Full-batch Adam; returns the loss before each step."""
        X = X.contiguous().float()
        y = y.contiguous().float()
        losses = np.zeros(steps, dtype=np.float32)
        call("bclx_mlp_train", self._ctx(), ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(y.data_ptr()),
             X.shape[0], ctypes.c_void_p(self.params.data_ptr()), steps, ctypes.c_float(lr),
             losses.ctypes.data_as(ctypes.c_void_p))
        return losses

    def predict(self, X: torch.Tensor) -> torch.Tensor:
        X = X.contiguous().float()
        out = torch.empty(X.shape[0], dtype=torch.float32, device=X.device)
        call("bclx_mlp_predict", self._ctx(), ctypes.c_void_p(X.data_ptr()), X.shape[0],
             ctypes.c_void_p(self.params.data_ptr()), ctypes.c_void_p(out.data_ptr()))
        return out

    def gradient(self, X: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
        g = torch.empty(num_params() + 1, dtype=torch.float32, device=X.device)
        call("bclx_mlp_gradient", self._ctx(), ctypes.c_void_p(X.contiguous().data_ptr()),
             ctypes.c_void_p(y.contiguous().data_ptr()), X.shape[0], ctypes.c_void_p(self.params.data_ptr()),
             ctypes.c_void_p(g.data_ptr()))
        return g

    def save(self, path: str) -> None:
        np.save(path, self.params.cpu().numpy())

    @classmethod
    def load(cls, path: str, device: Optional[int] = None) -> "RowNnzPredictor":
        return cls(np.load(path), device=device)


def row_samples(a, b) -> Tuple[torch.Tensor, torch.Tensor]:
    """Features and exact targets log2(1 + nnz) of every row of C = A*B that
    has products (the symbolic phase supplies the counts)."""
    from .containers import _out_grid, context, spgemm_symbolic
    plan, out, trp, toff, nnz = spgemm_symbolic(a, b)
    nri = a.gm * b.gn * a.tm
    X = torch.empty((nri, IN), dtype=torch.float32, device="cuda")
    ub = torch.empty(nri, dtype=torch.int32, device="cuda")
    cnt = torch.empty(nri, dtype=torch.int32, device="cuda")
    h = context(a.device).use_current_stream()
    ag, bg = a.spgrid(), b.spgrid()
    call("bclx_spgemm_row_features", h, ctypes.byref(ag), ctypes.byref(bg), ctypes.byref(out),
         ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(ub.data_ptr()))
    call("bclx_spgemm_plan_row_counts", plan.h, ctypes.c_void_p(cnt.data_ptr()))
    plan.close()
    keep = ub > 0
    return X[keep], torch.log2(1.0 + cnt[keep].float())


def training_set(scales: Iterable[int] = (14, 15, 16, 17, 18), n_rmat: int = 32,
                 stencil_grids: Iterable[int] = (32, 48, 64), tile_grids=(4, 8, 16), seed: int = 1000,
                 max_rows: int = 4_000_000):
    """Rows of C = A*A for n_rmat seeded R-MAT matrices spread over `scales`
    and 27-point stencils on g^3 grids, each on one of `tile_grids` tile grids
    (tiles at most 16384 wide)."""
    from . import gen
    from .containers import BlockCustom, SPMatrix
    scales = list(scales)
    Xs, ys = [], []
    for i in range(n_rmat):
        s = scales[i % len(scales)]
        a = gen.rmat(s, seed=seed + i)
        G = max(tile_grids[i % len(tile_grids)], -(-a.m // 16384))
        t = -(-a.m // G)
        A = SPMatrix.from_csr(a, BlockCustom((t, t)))
        X, y = row_samples(A, A)
        Xs.append(X)
        ys.append(y)
    for k, gsz in enumerate(stencil_grids):
        a = gen.stencil27(gsz)
        G = max(tile_grids[k % len(tile_grids)], -(-a.m // 16384))
        t = -(-a.m // G)
        A = SPMatrix.from_csr(a, BlockCustom((t, t)))
        X, y = row_samples(A, A)
        Xs.append(X)
        ys.append(y)
    X = torch.cat(Xs)
    y = torch.cat(ys)
    if X.shape[0] > max_rows:
        g = torch.Generator(device="cpu").manual_seed(seed)
        idx = torch.randperm(X.shape[0], generator=g)[:max_rows].to(X.device)
        X, y = X[idx], y[idx]
    return X, y


PACKAGED_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "row_nnz_mlp.npy")


def default_model_path() -> str:
    """The trained weights shipped with the package, else the local cache."""
    if os.path.exists(PACKAGED_MODEL):
        return PACKAGED_MODEL
    from .gen import cache_dir
    return os.path.join(cache_dir(), "row_nnz_mlp.npy")


def get_default(train_if_missing: bool = True, **kw) -> RowNnzPredictor:
    """The cached trained predictor, training it first if there is none."""
    path = default_model_path()
    if os.path.exists(path):
        return RowNnzPredictor.load(path)
    if not train_if_missing:
        raise FileNotFoundError(path)
    X, y = training_set(**kw)
    m = RowNnzPredictor(seed=0)
    m.fit(X, y, steps=600, lr=3e-3)
    m.save(path)
    return m


def _main():
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="train the row-nnz predictor on the GPU")
    ap.add_argument("--out", default=None)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--lr", type=float, default=3e-3)
    args = ap.parse_args()
    t0 = time.time()
    X, y = training_set()
    t1 = time.time()
    m = RowNnzPredictor(seed=0)
    losses = m.fit(X, y, steps=args.steps, lr=args.lr)
    torch.cuda.synchronize()
    t2 = time.time()
    pred = m.predict(X)
    err = (torch.exp2(pred) - torch.exp2(y)).abs() / torch.exp2(y)
    out = args.out or default_model_path()
    m.save(out)
    print(json.dumps({"samples": int(X.shape[0]), "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                      "median_rel_err_count": float(err.median()), "p90_rel_err_count": float(err.quantile(0.9)),
                      "data_s": t1 - t0, "train_s": t2 - t1, "out": out}))


if __name__ == "__main__":
    _main()
