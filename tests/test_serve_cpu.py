"""CPU: the served loop's host-side pieces: request-set generation and argument checks that fail
before any device work."""
import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
from gpu_betweennesscentrality_b200 import capi
from gpu_betweennesscentrality_b200.serve import log_uniform_sizes, request_sets
from util import grid_lines


def test_log_uniform_sizes_cover_the_range():
    rng = np.random.default_rng(0)
    s = log_uniform_sizes(rng, 20000, 1, 8192)
    assert s.min() == 1 and s.max() <= 8192 and s.max() > 4000
    # log-uniform: about half of the sizes below the geometric midpoint
    assert 0.45 < np.mean(s < np.sqrt(8192)) < 0.55


def test_request_sets_are_seeded_and_repeat_free():
    a = request_sets(1000, 10, 1, 5000, seed=4)
    b = request_sets(1000, 10, 1, 5000, seed=4)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    for x in a:
        assert 1 <= x.shape[0] <= 1000 and np.unique(x).shape[0] == x.shape[0] and x.max() < 1000


def test_serve_and_autotune_need_a_device_index():
    n, u, v, w = grid_lines(200, seed=1)
    g = Q.Graph()
    g.ReadLines(n, u, v, w)
    idx = g.build_index(upload=False)
    with pytest.raises(Q.QbcError) as e:
        idx.serve()
    assert e.value.code == capi.QBC_EINVAL
    with pytest.raises(Q.QbcError):
        idx.autotune(np.arange(10))
    with pytest.raises(Q.QbcError):
        idx.set_tuning(queue_depth=5)
    idx.set_tuning(queue_depth=256)
    assert idx.get_tuning()["queue_depth"] == 256
