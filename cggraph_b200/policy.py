"""The learned per-iteration scheduler: trace collection, GPU training,
loading.

The network (24 features -> 64 -> 64 -> 14 log-cost predictions, FP32) lives
in the engine; this module drives its C entry points (cgb_policy_*):

* ``collect(graph, alg, root)`` -- counterfactual samples of one run: at each
  BFS level the three variants (binned push, chunked push, bottom-up pull),
  at the first SSSP bucket boundary the rest of the run under each of the
  seven delta multipliers (x 1/4 .. x 16),
  at each large SSSP near round the four round variants (sparse frontier
  binned or chunked, dense frontier, pull), timed from the same snapshot;
* ``train(X, T, M)`` -- masked-MSE training on the GPU by the engine's own
  forward / backward / Adam kernels;
* ``load(params)`` -- makes a network the policy of CGB_SCHED_LEARNED runs;
  ``load_default()`` loads the weights shipped with the package
  (``policy_weights.npy``, made by ``python -m cggraph_b200.train_policy``).
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

from . import _lib as L
from ._lib import check

NF, NO, NP = L.POLICY_FEATURES, L.POLICY_OUTPUTS, L.POLICY_PARAMS
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "policy_weights.npy")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def collect(graph, algorithm: int, root: int, options=None, max_samples: int = 8192):
    X = np.zeros((max_samples, NF), np.float32)
    T = np.zeros((max_samples, NO), np.float32)
    M = np.zeros((max_samples, NO), np.uint8)
    n = ctypes.c_uint32()
    check(L.lib().cgb_policy_collect(graph.handle, int(algorithm), int(root),
                                     ctypes.byref(options) if options else None, X.ctypes.data, T.ctypes.data,
                                     M.ctypes.data, max_samples, ctypes.byref(n)))
    k = n.value
    return X[:k].copy(), T[:k].copy(), M[:k].copy()


def train(X, T, M, epochs: int = 300, batch: int = 256, lr: float = 3e-3, seed: int = 0,
          init: Optional[np.ndarray] = None) -> Tuple[np.ndarray, float]:
    X, T = _f32(X), _f32(T)
    M = np.ascontiguousarray(M, dtype=np.uint8)
    out = np.zeros(NP, np.float32)
    loss = ctypes.c_float()
    init = _f32(init) if init is not None else None
    check(L.lib().cgb_policy_train(X.ctypes.data, T.ctypes.data, M.ctypes.data, len(X), epochs, batch, lr, seed,
                                   init.ctypes.data if init is not None else None, out.ctypes.data,
                                   ctypes.byref(loss)))
    return out, float(loss.value)


def forward(params, X) -> np.ndarray:
    params, X = _f32(params), _f32(X)
    Y = np.zeros((len(X), NO), np.float32)
    check(L.lib().cgb_policy_forward(params.ctypes.data, X.ctypes.data, len(X), Y.ctypes.data))
    return Y


def loss_grad(params, X, T, M):
    params, X, T = _f32(params), _f32(X), _f32(T)
    M = np.ascontiguousarray(M, dtype=np.uint8)
    loss = ctypes.c_float()
    grad = np.zeros(NP, np.float32)
    check(L.lib().cgb_policy_loss_grad(params.ctypes.data, X.ctypes.data, T.ctypes.data, M.ctypes.data, len(X),
                                       ctypes.byref(loss), grad.ctypes.data))
    return float(loss.value), grad


def load(params: Optional[np.ndarray]) -> None:
    """Make `params` the policy of the current device (None: heuristic only)."""
    if params is None:
        check(L.lib().cgb_policy_load(None))
        return
    p = _f32(params)
    assert p.size == NP
    check(L.lib().cgb_policy_load(p.ctypes.data))


def load_default() -> bool:
    if not os.path.exists(DEFAULT_WEIGHTS):
        return False
    load(np.load(DEFAULT_WEIGHTS))
    return True


# output heads (include/cgb200.h)
BFS_LEVEL = [0, 1, 9]            # binned push, pull, chunked push
SSSP_DELTA = list(range(2, 9))   # x 1/4 .. x 16
SSSP_ROUND = [10, 11, 12, 13]    # sparse binned, sparse chunked, dense, pull


def decisions(params, X) -> dict:
    """What the policy would choose for each sample, before the confidence
    margin: BFS level variant (0 push, 1 pull, 2 chunked push), SSSP delta
    index (0..6: x 1/4 .. x 16), SSSP round variant (0..3)."""
    Y = forward(params, X)
    return {"bfs_level": np.argmin(Y[:, BFS_LEVEL], axis=1), "delta": np.argmin(Y[:, SSSP_DELTA], axis=1),
            "round": np.argmin(Y[:, SSSP_ROUND], axis=1)}
