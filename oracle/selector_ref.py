"""Oracle (test infrastructure only): fp64 restatements for the selector.

* ``forward`` / ``loss_and_grad``: the 16-64-64-2 ReLU network and its
  mean-squared-error gradient in float64, with the parameter layout of the
  library (W1[64x16], b1, W2[64x64], b2, W3[2x64], b3; row-major, out x in).
  The gradient of the library's kernel is checked against it.
* ``AdaptivePolicy``: an independent Python restatement of the reference's
  adaptive selector, benchmarks/publication_policy_bfs.cpp:79-94 (state),
  :163-235 (decision) and :285-320 (EMA updates), constants from
  benchmarks/adaptive_policy_bfs.cpp:21-31.  The library's C++ restatement
  (vx_heuristic_*) is checked against it decision by decision.

Only tests import this module; nothing in the product path does.
"""
from __future__ import annotations

import math

import numpy as np

IN, H, OUT = 16, 64, 2
O_W1 = 0
O_B1 = O_W1 + H * IN
O_W2 = O_B1 + H
O_B2 = O_W2 + H * H
O_W3 = O_B2 + H
O_B3 = O_W3 + OUT * H
N_PARAMS = O_B3 + OUT


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    assert P.size == N_PARAMS
    W1 = P[O_W1:O_B1].reshape(H, IN)
    b1 = P[O_B1:O_W2]
    W2 = P[O_W2:O_B2].reshape(H, H)
    b2 = P[O_B2:O_W3]
    W3 = P[O_W3:O_B3].reshape(OUT, H)
    b3 = P[O_B3:]
    return W1, b1, W2, b2, W3, b3


def forward(P, X):
    W1, b1, W2, b2, W3, b3 = unpack(P)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3.T + b3


def loss_and_grad(P, X, Y):
    """loss = mean over samples and outputs of (y - target)^2."""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ W3.T + b3
    d = y - Y
    loss = float(np.mean(d * d))
    dy = 2.0 * d / d.size
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    d2 = (dy @ W3) * (z2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (z1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


class AdaptivePolicy:
    """publication_policy_bfs.cpp 'adaptive' policy state machine."""

    PREFLIGHT_FULL_UPDATE = 0.05
    VERY_SPARSE_REACH = 0.02
    SPARSE_REACH = 0.20
    SPARSE_REACH_FULL_UPDATE = 0.0025
    LEARNED_FULL_MARGIN = 1.25
    FRESH_AGE = 4
    EMA_ALPHA = 0.25

    def __init__(self, vertices, initial_reachable_fraction, initial_full_us):
        self.initial_reachable_fraction = initial_reachable_fraction
        self.previous_affected_fraction = 0.0
        self.ema_incremental_us = 0.0
        self.ema_full_us = initial_full_us
        self.last_incremental_update_fraction = 0.0
        self.ema_incremental_rel_error = 0.0
        self.ema_full_rel_error = 0.0
        self.have_incremental_error = False
        self.have_full_error = False
        self.have_incremental = False
        self.have_full = True
        self.incremental_age = self.FRESH_AGE + 1
        self.full_age = 0
        self.large_scale = vertices >= 200000
        self.first_batch = True
        self.pred_inc = 0.0
        self.pred_full = 0.0
        self.update_fraction = 0.0

    def decide(self, update_fraction, shallow_fraction):
        self.update_fraction = update_fraction
        clamp = lambda x, lo, hi: min(hi, max(lo, x))
        if self.large_scale:
            scale = (math.sqrt((update_fraction + 1e-12) / (self.last_incremental_update_fraction + 1e-12))
                     if self.have_incremental else 1.0)
            scale = clamp(scale, 0.5, 2.5)
            pi = (self.ema_incremental_us * scale * (1.0 + 3.0 * self.previous_affected_fraction)
                  if self.have_incremental else 0.0)
            pf = self.ema_full_us
            iu = clamp(self.ema_incremental_rel_error, 0.05, 0.35) if self.have_incremental_error else 0.35
            fu = clamp(self.ema_full_rel_error, 0.05, 0.35) if self.have_full_error else 0.20
            self.pred_inc, self.pred_full = pi, pf
            if update_fraction >= self.PREFLIGHT_FULL_UPDATE:
                return True
            if self.first_batch and shallow_fraction > 0.0:
                return True
            if not self.have_incremental:
                return False
            return pi * (1.0 - iu) > pf * (1.0 + fu)
        pi = self.ema_incremental_us * (1.0 + 2.0 * self.previous_affected_fraction) if self.have_incremental else 0.0
        pf = self.ema_full_us if self.have_full else 0.0
        self.pred_inc, self.pred_full = pi, pf
        fresh = (self.have_incremental and self.have_full and self.incremental_age <= self.FRESH_AGE
                 and self.full_age <= self.FRESH_AGE)
        if update_fraction >= self.PREFLIGHT_FULL_UPDATE:
            return True
        if self.initial_reachable_fraction <= self.VERY_SPARSE_REACH:
            return True
        if self.initial_reachable_fraction < self.SPARSE_REACH and update_fraction >= self.SPARSE_REACH_FULL_UPDATE:
            return True
        return fresh and pi > pf * self.LEARNED_FULL_MARGIN

    def observe(self, observed_full, execution_us, affected_fraction):
        a = self.EMA_ALPHA
        self.incremental_age += 1
        self.full_age += 1
        if self.large_scale and self.pred_inc > 0.0 and self.pred_full > 0.0:
            if observed_full:
                rel = abs(execution_us - self.pred_full) / max(1.0, self.pred_full)
                self.ema_full_rel_error = (1 - a) * self.ema_full_rel_error + a * rel if self.have_full_error else rel
                self.have_full_error = True
            else:
                rel = abs(execution_us - self.pred_inc) / max(1.0, self.pred_inc)
                self.ema_incremental_rel_error = ((1 - a) * self.ema_incremental_rel_error + a * rel
                                                  if self.have_incremental_error else rel)
                self.have_incremental_error = True
        if observed_full:
            self.ema_full_us = (1 - a) * self.ema_full_us + a * execution_us if self.have_full else execution_us
            self.have_full = True
            self.full_age = 0
            self.previous_affected_fraction = 0.0
        else:
            self.ema_incremental_us = ((1 - a) * self.ema_incremental_us + a * execution_us
                                       if self.have_incremental else execution_us)
            self.have_incremental = True
            self.incremental_age = 0
            self.last_incremental_update_fraction = self.update_fraction
            self.previous_affected_fraction = affected_fraction
        self.first_batch = False
