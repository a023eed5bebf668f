"""Learned insertion proposal: training data, the network's trainer and its parameters.

The network (csrc/mlp.cu) maps a voxel's 4x4x4 local density of solvent
first sites to a logit; the engine turns the logits of all voxels into the
proposal q_v = eps / V + (1 - eps) softmax(s)_v and weights every insertion
by p/q (csrc/proposal.cu).  Training data come from plain uniform insertion:
the features of each insertion's voxel and a label that marks insertions
whose total solute-solvent energy lies below a quantile of the uniform
energies, i.e. where the solute fits.  Uniform insertion stays the yardstick:
the importance weights make the learned run estimate the uniform-insertion
distributions.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from .engine import ErmodError

NIN, NH = 64, 128


def layout():
    """Offsets of W1, b1, W2, b2, W3, b3, w4, b4 in the parameter vector."""
    o = {}
    n = 0
    for name, size in (("W1", NH * NIN), ("b1", NH), ("W2", NH * NH), ("b2", NH), ("W3", NH * NH), ("b3", NH),
                       ("w4", NH), ("b4", 1)):
        o[name] = (n, size)
        n += size
    o["n"] = n
    return o


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weight matrices, zero biases (FP32)."""
    rng = np.random.default_rng(seed)
    L = layout()
    p = np.zeros(L["n"], dtype=np.float32)
    for name, fan_in in (("W1", NIN), ("W2", NH), ("W3", NH), ("w4", NH)):
        off, size = L[name]
        p[off:off + size] = rng.normal(0.0, np.sqrt(2.0 / fan_in), size)
    return p


def labels_from_energies(etot: np.ndarray, quantile: float = 0.1, threshold: float | None = None):
    """1 for insertions with total energy below `threshold` (default: the `quantile` of `etot`)."""
    thr = float(np.quantile(etot, quantile)) if threshold is None else threshold
    return (etot < thr).astype(np.float32), thr


class Trainer:
    """The device trainer (ermod_mlp_*): Adam on FP32 master weights, BF16 weights in every pass."""

    def __init__(self, params: np.ndarray, max_batch: int = 4096, device: int = 0):
        self.lib = A.load_library()
        p = np.ascontiguousarray(params, dtype=np.float32)
        self.h = C.c_void_p()
        rc = self.lib.ermod_mlp_create(C.byref(self.h), device, max_batch, A.ptr(p, C.c_float))
        if rc != 0:
            raise ErmodError(rc, "mlp_create")
        self.max_batch = max_batch
        self.n = int(self.lib.ermod_mlp_nparams())

    def close(self):
        if getattr(self, "h", None):
            self.lib.ermod_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def forward(self, x: np.ndarray) -> np.ndarray:
        """Logits of any number of samples, in batches of at most max_batch."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros(len(x), dtype=np.float32)
        for i in range(0, len(x), self.max_batch):
            xb = np.ascontiguousarray(x[i:i + self.max_batch])
            ob = np.zeros(len(xb), dtype=np.float32)
            rc = self.lib.ermod_mlp_forward(self.h, A.ptr(xb, C.c_float), len(xb), A.ptr(ob, C.c_float))
            if rc != 0:
                raise ErmodError(rc, "mlp_forward")
            out[i:i + len(xb)] = ob
        return out

    def activations(self, n: int) -> np.ndarray:
        """The hidden activations [3][n][128] of the last forward or gradient pass (n samples)."""
        a = np.zeros((3, n, 128), dtype=np.float32)
        rc = self.lib.ermod_mlp_activations(self.h, n, A.ptr(a, C.c_float))
        if rc != 0:
            raise ErmodError(rc, "mlp_activations")
        return a

    def gradients(self, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(self.n, dtype=np.float32)
        loss = C.c_double()
        rc = self.lib.ermod_mlp_gradients(self.h, A.ptr(x, C.c_float), A.ptr(y, C.c_float), len(x),
                                          A.ptr(g, C.c_float), C.byref(loss))
        if rc != 0:
            raise ErmodError(rc, "mlp_gradients")
        return g, loss.value

    def step(self, x: np.ndarray, y: np.ndarray, lr: float) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = C.c_double()
        rc = self.lib.ermod_mlp_train_step(self.h, A.ptr(x, C.c_float), A.ptr(y, C.c_float), len(x), lr,
                                           C.byref(loss))
        if rc != 0:
            raise ErmodError(rc, "mlp_train_step")
        return loss.value

    def params(self) -> np.ndarray:
        p = np.zeros(self.n, dtype=np.float32)
        rc = self.lib.ermod_mlp_get_params(self.h, A.ptr(p, C.c_float))
        if rc != 0:
            raise ErmodError(rc, "mlp_get_params")
        return p

    def fit(self, x: np.ndarray, y: np.ndarray, epochs: int = 3, batch: int = 2048, lr: float = 1e-3,
            seed: int = 0) -> list[float]:
        """Mini-batch Adam over shuffled data; returns the mean loss of each epoch."""
        rng = np.random.default_rng(seed)
        batch = min(batch, self.max_batch)
        hist = []
        for _ in range(epochs):
            order = rng.permutation(len(x))
            losses = []
            for i in range(0, len(order) - batch + 1, batch):
                idx = order[i:i + batch]
                losses.append(self.step(x[idx], y[idx], lr))
            hist.append(float(np.mean(losses)) if losses else float("nan"))
        return hist


def collect_uniform_samples(engine, frames, stnum0: int = 1):
    """Run uniform-insertion frames [(sitepos, cell)] on `engine` (proposal grid configured) and return
    the per-insertion features, total energies and voxels of all of them."""
    fs, es, vs = [], [], []
    for i, (pos, cell) in enumerate(frames):
        engine.engconst(stnum0 + i, pos, cell)
        f, e, v = engine.insertion_samples()
        fs.append(f)
        es.append(e)
        vs.append(v)
    return np.concatenate(fs), np.concatenate(es), np.concatenate(vs)
