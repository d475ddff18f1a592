"""Learned scheduler: the cost model that orders deep-level work.

The device miner splits the deep levels into root units (one position of a
top-level class).  With ``scheduler="learned"`` the miners start root units in
order of a predicted subtree cost instead of the plain order (more later class
members first).  The predictor is a one-hidden-layer FP32 MLP; its forward,
backward and Adam kernels live in ``libcupami_b200.so`` and run on the GPU.
The order never changes which itemsets are found or their supports.

Training data are traces the exact miner emits itself: mining with
``collect_trace`` records, for every root unit, its features and
``log1p(intersections in its subtree)``.  ``python -m cupami_b200.costmodel``
regenerates the shipped model from synthetic training databases (seeds that
the benchmark workloads do not use).
"""

from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

import numpy as np

from . import _native

MODEL_PATH = Path(__file__).resolve().parent / "models" / "costmodel.json"


def sizes():
    nf, npar = ctypes.c_uint32(), ctypes.c_uint32()
    _native.library().cpm_costmodel_params(ctypes.byref(nf), ctypes.byref(npar))
    return nf.value, npar.value


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a if shape is None else a.reshape(shape)


def train(X, y, epochs=600, lr=3e-3, seed=0, ctx=None):
    """Fit the MLP on the GPU; returns (params, loss per epoch)."""
    ctx = ctx or _native.context(0)
    nf, npar = sizes()
    X = _f32(X, (-1, nf))
    y = _f32(y)
    params = np.zeros(npar, dtype=np.float32)
    hist = np.zeros(epochs, dtype=np.float32)
    with ctx.lock:
        ctx.check(_native.library().cpm_costmodel_train(ctx.handle, X.ctypes.data, y.ctypes.data, y.size, epochs,
                                                        ctypes.c_float(lr), seed, params.ctypes.data,
                                                        hist.ctypes.data))
    return params, hist


def predict(params, X, ctx=None):
    """Predicted log1p(subtree intersections) per row of X."""
    ctx = ctx or _native.context(0)
    nf, _ = sizes()
    X = _f32(X, (-1, nf))
    params = _f32(params)
    y = np.zeros(X.shape[0], dtype=np.float32)
    with ctx.lock:
        ctx.check(_native.library().cpm_costmodel_predict(ctx.handle, params.ctypes.data, X.ctypes.data,
                                                          X.shape[0], y.ctypes.data))
    return y


def gradient(params, X, y, ctx=None):
    """(gradient of the standardised half-MSE per parameter, loss) from the device kernels."""
    ctx = ctx or _native.context(0)
    nf, npar = sizes()
    X = _f32(X, (-1, nf))
    y = _f32(y)
    params = _f32(params)
    g = np.zeros(npar, dtype=np.float32)
    loss = ctypes.c_float()
    with ctx.lock:
        ctx.check(_native.library().cpm_costmodel_gradient(ctx.handle, params.ctypes.data, X.ctypes.data,
                                                           y.ctypes.data, y.size, g.ctypes.data,
                                                           ctypes.byref(loss)))
    return g, loss.value


def save(params, path=MODEL_PATH, meta=None):
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps({"params": [float(v) for v in np.asarray(params, dtype=np.float32)],
                                "meta": meta or {}}, indent=0))


def load(path=MODEL_PATH):
    d = json.loads(Path(path).read_text())
    return np.asarray(d["params"], dtype=np.float32)


def use(params, ctx=None):
    """Make ``params`` the model of the context's learned scheduler (None unloads)."""
    ctx = ctx or _native.context(0)
    p = None if params is None else _f32(params)
    ctx.check(_native.library().cpm_costmodel_set(ctx.handle, None if p is None else p.ctypes.data))
    ctx.model_loaded = p is not None


def ensure_default(ctx):
    """Load the shipped model into ``ctx`` once (no model file: plain order)."""
    if getattr(ctx, "model_loaded", False):
        return True
    if not MODEL_PATH.exists():
        return False
    use(load(), ctx)
    return True


def trace(csr, minSup):
    """(features, log1p(subtree intersections)) of every root unit of one database."""
    db = _native.Database.from_ids(_native.context(0), csr.offsets, csr.items)
    opts = _native.Opts()
    _native.library().cpm_default_opts(ctypes.byref(opts))
    opts.collect_trace = 1
    n = int(np.count_nonzero(np.diff(csr.offsets.astype(np.int64)) > 0))
    from .frequentPattern.cuApriori import cuApriori

    res = db.mine(cuApriori._getSupportCount(minSup, n), _native.CPM_ECLAT, opts)
    db.close()
    nf, _ = sizes()
    return res.trace if res.trace is not None else (np.zeros((0, nf), np.float32), np.zeros(0, np.float32))


def training_databases():
    """Synthetic training databases of the dense and batched families.

    Seeds 1000+ are not used by any benchmark workload."""
    from . import datasets

    out = []
    for k in range(6):
        out.append((datasets.dense_bernoulli(n=16384 * (1 + k % 2), n_items=96 + 8 * k, seed=1000 + k), 0.6))
    for k, csr in enumerate(datasets.batched_zipf(n_db=48, seed=1100, limit=48)):
        out.append((csr, 0.01))
    for k in range(3):
        out.append((datasets.planted_zipf(n=40000, n_items=600, seed=1200 + k), 0.005))
    return out


def main(argv):
    out = Path(argv[1]) if len(argv) > 1 else MODEL_PATH
    xs, ys = [], []
    for csr, ms in training_databases():
        X, y = trace(csr, ms)
        xs.append(X)
        ys.append(y)
    X = np.concatenate(xs)
    y = np.concatenate(ys)
    params, hist = train(X, y, epochs=800, lr=3e-3, seed=7)
    pred = predict(params, X)
    rank = np.corrcoef(np.argsort(np.argsort(pred)), np.argsort(np.argsort(y)))[0, 1]
    meta = {"samples": int(y.size), "final_loss": float(hist[-1]), "first_loss": float(hist[0]),
            "train_spearman": float(rank), "epochs": 800, "lr": 3e-3, "seed": 7}
    save(params, out, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main(sys.argv)
