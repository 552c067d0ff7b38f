"""Repair-vs-recompute selection on the GPU.

The reference chooses, per update batch, between ``IncrementalBFS.apply``
(repair) and ``graph.apply`` + ``recompute`` (full) in its benchmark harnesses
(benchmarks/publication_policy_bfs.cpp:46-335) with a hand-tuned heuristic.

* ``MLPSelector`` trains the 16-64-64-2 network with the library's own
  kernels (vx_selector_train) on standardised log times and predicts both arms;
* ``Heuristic`` is the reference's adaptive selector, restated in the library
  (vx_heuristic_*), used as fallback and baseline.

The features of a batch come from ``vx_bfs_stage`` + ``vx_bfs_staged_features``;
the chosen arm runs with ``vx_bfs_run_repair`` or ``vx_bfs_run_full``.  The
regret study that trains and scores the network lives beside the benchmarks
(``workloads/selector_study.py``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import capi

N_FEATURES = 16
N_PARAMS = 5378

_f32p = C.POINTER(C.c_float)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)


def _lib():
    lib = capi()
    sig = {
        "vx_bfs_stage": (C.c_int, [C.c_void_p, _u32p, _u32p, _u8p, C.c_size_t]),
        "vx_bfs_staged_features": (C.c_int, [C.c_void_p, C.c_float, _f32p]),
        "vx_bfs_run_repair": (C.c_int, [C.c_void_p]),
        "vx_bfs_run_full": (C.c_int, [C.c_void_p]),
        "vx_selector_create": (C.c_int, [C.c_uint64, C.POINTER(C.c_void_p)]),
        "vx_selector_destroy": (C.c_int, [C.c_void_p]),
        "vx_selector_train": (C.c_int, [C.c_void_p, _f32p, _f32p, C.c_size_t, C.c_uint32, C.c_uint32, C.c_float,
                                        C.c_uint32, _f32p]),
        "vx_selector_gradients": (C.c_int, [C.c_void_p, _f32p, _f32p, C.c_size_t, _f32p, _f32p]),
        "vx_selector_predict": (C.c_int, [C.c_void_p, _f32p, C.c_size_t, _f32p]),
        "vx_selector_set_params": (C.c_int, [C.c_void_p, _f32p]),
        "vx_selector_get_params": (C.c_int, [C.c_void_p, _f32p]),
        "vx_heuristic_create": (C.c_int, [C.c_size_t, C.c_double, C.c_double, C.POINTER(C.c_void_p)]),
        "vx_heuristic_destroy": (C.c_int, [C.c_void_p]),
        "vx_heuristic_decide": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_int)]),
        "vx_heuristic_observe": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        from . import last_error

        raise RuntimeError(f"vx_b200 error {rc}: {last_error()}")


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class MLPSelector:
    """The 16-64-64-2 network on the GPU (vx_selector_*)."""

    def __init__(self, seed: int = 1):
        self.lib = _lib()
        self.h = C.c_void_p()
        _check(self.lib.vx_selector_create(seed, C.byref(self.h)))
        self.mu = np.zeros(2)
        self.sd = np.ones(2)
        self.margin = 0.0  # log-ratio margin full must win by (fit calibrates it)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.vx_selector_destroy(self.h)
            self.h = None

    @property
    def params(self) -> np.ndarray:
        out = np.empty(N_PARAMS, np.float32)
        _check(self.lib.vx_selector_get_params(self.h, out.ctypes.data_as(_f32p)))
        return out

    @params.setter
    def params(self, p) -> None:
        p = _f32(p)
        assert p.size == N_PARAMS
        _check(self.lib.vx_selector_set_params(self.h, p.ctypes.data_as(_f32p)))

    def gradients(self, X, Y):
        X, Y = _f32(X), _f32(Y)
        g = np.empty(N_PARAMS, np.float32)
        loss = C.c_float()
        _check(self.lib.vx_selector_gradients(self.h, X.ctypes.data_as(_f32p), Y.ctypes.data_as(_f32p), len(X),
                                              g.ctypes.data_as(_f32p), C.byref(loss)))
        return g, loss.value

    def targets(self, t_repair, t_full) -> np.ndarray:
        """Network targets: the mean log time of the two arms and the log
        ratio full/repair, each standardised with the training set's moments
        (fit sets them).  The second output carries the decision, so it gets a
        unit-variance target of its own."""
        lr, lf = np.log(t_repair), np.log(t_full)
        raw = np.stack([(lr + lf) / 2, lf - lr], axis=1)
        return _f32((raw - self.mu) / self.sd)

    def fit(self, X, t_repair, t_full, epochs: int = 300, batch: int = 32, lr: float = 3e-3, seed: int = 7,
            calib=None) -> float:
        """Trains on (features, both arms' times in us) with the library's Adam
        kernel, then calibrates the decision margin on calib = (X, t_repair,
        t_full), batches the network was not fitted on (default: the training
        batches themselves)."""
        lr_, lf_ = np.log(t_repair), np.log(t_full)
        raw = np.stack([(lr_ + lf_) / 2, lf_ - lr_], axis=1)
        self.mu = raw.mean(0)
        self.sd = raw.std(0) + 1e-6
        Y = self.targets(t_repair, t_full)
        X = _f32(X)
        loss = C.c_float()
        _check(self.lib.vx_selector_train(self.h, X.ctypes.data_as(_f32p), Y.ctypes.data_as(_f32p), len(X), epochs,
                                          batch, lr, seed, C.byref(loss)))
        self.margin = self.calibrate_margin(*(calib if calib is not None else (X, t_repair, t_full)))
        return loss.value

    # candidate margins of the predicted log ratio log(t_full / t_repair)
    MARGINS = (0.0, 0.02, 0.05, 0.1, 0.2, 0.4, 0.8, np.inf)

    def calibrate_margin(self, X, t_repair, t_full) -> float:
        """The margin by which the predicted full time must undercut the
        predicted repair time before full is chosen, picked on the given
        batches: the candidate with the smallest mean regret there (an
        infinite margin is always repair; ties go to the larger margin, the
        cheaper mistake).  Prediction errors otherwise send batches to the
        full arm whose rare wins do not pay for its losses."""
        Y = self.predict_log(X)
        d = Y[:, 1] - Y[:, 0]
        oracle = np.minimum(t_repair, t_full)
        best, best_r = 0.0, np.inf
        for m in self.MARGINS:
            full = np.isfinite(d) & (d <= -m)
            r = float(np.mean(np.maximum(0.0, (np.where(full, t_full, t_repair) - oracle) / oracle)))
            if r <= best_r:
                best, best_r = m, r
        return best

    def predict_raw(self, X) -> np.ndarray:
        """The network's two outputs for each row of X (standardised units)."""
        X = _f32(X).reshape(-1, N_FEATURES)
        Y = np.empty((len(X), 2), np.float32)
        if len(X):
            _check(self.lib.vx_selector_predict(self.h, X.ctypes.data_as(_f32p), len(X), Y.ctypes.data_as(_f32p)))
        return Y

    def predict_log(self, X) -> np.ndarray:
        """Predicted natural-log execution times (us) of (repair, full)."""
        Y = self.predict_raw(X).astype(np.float64) * self.sd + self.mu
        return np.stack([Y[:, 0] - Y[:, 1] / 2, Y[:, 0] + Y[:, 1] / 2], axis=1)

    def choose_full(self, X):
        """(choose_full, ok): full where its predicted log time undercuts
        repair's by the calibrated margin (with margin 0, full wins ties); ok
        is False where a prediction is not finite, and the caller then falls
        back to the heuristic."""
        Y = self.predict_log(X)
        ok = np.all(np.isfinite(Y), axis=1)
        return np.where(ok, Y[:, 1] - Y[:, 0] <= -self.margin, False), ok


class Heuristic:
    """The reference's adaptive selector (publication_policy_bfs.cpp:163-235)."""

    def __init__(self, vertices: int, initial_reachable_fraction: float, initial_full_us: float):
        self.lib = _lib()
        self.h = C.c_void_p()
        _check(self.lib.vx_heuristic_create(vertices, initial_reachable_fraction, initial_full_us, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.vx_heuristic_destroy(self.h)
            self.h = None

    def decide(self, update_fraction: float, shallow_fraction: float) -> bool:
        out = C.c_int()
        _check(self.lib.vx_heuristic_decide(self.h, update_fraction, shallow_fraction, C.byref(out)))
        return bool(out.value)

    def observe(self, full: bool, execution_us: float, affected_fraction: float) -> None:
        _check(self.lib.vx_heuristic_observe(self.h, int(full), execution_us, affected_fraction))
