"""CPU: the selector's host logic.

* the library's restatement of the reference's adaptive heuristic
  (vx_heuristic_*) against the oracle's independent Python restatement, on
  random decision/observation sequences in both of its modes;
* the fp64 oracle gradient against central finite differences, so the GPU
  gradient check below it rests on a verified reference;
* the first-batch shallow-deletion feature on a hand-checked example.
"""
import numpy as np
import pytest

from oracle import selector_ref as ref
from velographx_b200 import selector as sel
from workloads import selector_study as study


@pytest.mark.parametrize("vertices,reach", [(1000, 0.9), (1000, 0.1), (1000, 0.01), (1 << 20, 0.7)])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_heuristic_matches_oracle_restatement(vertices, reach, seed):
    rng = np.random.default_rng(seed)
    full0 = float(rng.uniform(50, 5000))
    h = sel.Heuristic(vertices, reach, full0)
    o = ref.AdaptivePolicy(vertices, reach, full0)
    decisions = 0
    for i in range(400):
        # update fractions spanning the preflight and sparse-reach thresholds
        uf = float(10 ** rng.uniform(-6, -0.8))
        shallow = float(rng.random() < 0.3) * float(rng.random()) if i == 0 else 0.0
        a = h.decide(uf, shallow)
        b = o.decide(uf, shallow)
        assert a == b, (i, uf)
        decisions += a
        t = float(rng.lognormal(np.log(full0 if a else full0 / 4), 0.8))
        aff = 0.0 if a else float(rng.uniform(0, 0.3))
        h.observe(a, t, aff)
        o.observe(a, t, aff)
    assert 0 <= decisions <= 400


def test_heuristic_mixes_arms_in_both_modes():
    for vertices in (1000, 1 << 20):
        h = sel.Heuristic(vertices, 0.9, 100.0)
        picks = []
        for i in range(60):
            full = h.decide(1e-4, 0.0)
            picks.append(full)
            # repair costs grow until full becomes the cheaper arm
            h.observe(full, 100.0 if full else 100.0 * (1 + i), 0.01)
        assert any(picks) and not all(picks)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    P = rng.normal(0, 0.3, ref.N_PARAMS)
    X = rng.normal(0, 1, (9, ref.IN))
    Y = rng.normal(0, 1, (9, ref.OUT))
    loss, g = ref.loss_and_grad(P, X, Y)
    assert g.shape == (ref.N_PARAMS,)
    idx = rng.choice(ref.N_PARAMS, 200, replace=False)
    idx = np.concatenate([idx, np.arange(ref.O_B3, ref.N_PARAMS), [ref.O_B1, ref.O_W3]])
    eps = 1e-6
    for p in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[p] += eps
        Pm[p] -= eps
        fd = (ref.loss_and_grad(Pp, X, Y)[0] - ref.loss_and_grad(Pm, X, Y)[0]) / (2 * eps)
        assert abs(fd - g[p]) <= 1e-6 + 1e-5 * abs(fd), p
    assert np.isclose(loss, np.mean((ref.forward(P, X) - Y) ** 2))


def test_shallow_parent_deletion_fraction_example():
    U = 0xFFFFFFFF
    dist = np.array([0, 1, 2, 3, 4, U, 1], np.uint32)
    src = np.array([0, 2, 3, 4, 1, 5, 0, 6], np.uint32)
    dst = np.array([1, 1, 4, 3, 6, 4, 6, 0], np.uint32)
    add = np.array([0, 0, 0, 0, 0, 0, 1, 0], np.uint8)
    # 0-1 tree arc (d=1); 2-1 reversed tree arc at depth 2; 3-4 at depth 4 (too deep);
    # 4-3 reversed at depth 4; 1-6 not a tree arc; 5 unreachable; 0-6 an insertion;
    # 6-0 reversed tree arc at depth 1
    assert study.shallow_parent_deletion_fraction(src, dst, add, dist) == pytest.approx(3 / 8)
