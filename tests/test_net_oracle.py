"""The candidate network's CPU oracle (no GPU): its analytic gradients agree with central finite
differences of its own loss, so the oracle the GPU training kernels are checked against is itself
pinned; and the parameter count matches the library's."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import candidate_net_oracle as cno  # noqa: E402


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    crops = rng.integers(0, 256, (n, 2, 24, 24)).astype(np.uint8)
    part = rng.integers(-1, 4, n)
    i4 = rng.integers(-1, 9, (n, 16))
    mv = rng.normal(0, 1.5, (n, 2))
    mvv = rng.integers(0, 2, n)
    part[0], i4[0, 0], mvv[0] = 2, 5, 1
    return crops, part, i4, mv, mvv


def test_parameter_count_matches_the_library():
    from ragdoll_b200.engine import lib
    assert lib().rg_net_param_count() == cno.N_PARAMS == 19599


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    flat = rng.normal(0, 0.15, cno.N_PARAMS)
    crops, part, i4, mv, mvv = _batch(2, 2)
    loss, grads, _ = cno.forward_backward(flat, crops, part, i4, mv, mvv, 0.5)
    assert np.isfinite(loss)
    idx = np.concatenate([rng.choice(np.arange(0, 608), 6), rng.choice(np.arange(608, 9856), 6),
                          rng.choice(np.arange(9856, 19104), 6), np.arange(19104, 19599, 37)])
    eps = 1e-6
    for i in idx:
        a, b = flat.copy(), flat.copy()
        a[i] += eps
        b[i] -= eps
        num = (cno.forward_backward(a, crops, part, i4, mv, mvv, 0.5)[0] -
               cno.forward_backward(b, crops, part, i4, mv, mvv, 0.5)[0]) / (2 * eps)
        assert abs(num - grads[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, grads[i])
