"""Shared helpers of the tests (graph generation, known-answer graphs)."""
import os

import numpy as np

from gpu_betweennesscentrality_b200 import synth

# BC agreement: FP64 sums in a different order than the reference's atomics
BC_RTOL = 1e-9


def lines_of(edges, n):
    """Undirected (a, b, w) 0-based edges -> both-direction 1-based arc lines."""
    e = np.asarray(edges, np.int64).reshape(-1, 3)
    u = np.empty(2 * e.shape[0], np.int32)
    v = np.empty_like(u)
    w = np.empty_like(u)
    u[0::2], v[0::2], w[0::2] = e[:, 0] + 1, e[:, 1] + 1, e[:, 2]
    u[1::2], v[1::2], w[1::2] = e[:, 1] + 1, e[:, 0] + 1, e[:, 2]
    return n, u, v, w


def grid_lines(n_target, seed=1, shortcut_frac=0.0):
    g = synth.grid_graph(n_target, seed=seed, shortcut_frac=shortcut_frac)
    u, v, w = g.arcs()
    return g.n, u, v, w


KNOWN = {
    # name: (n, edges, expected BC or None)
    "path3": (3, [(0, 1, 1), (1, 2, 1)], [0.0, 1.0, 0.0]),
    "star5": (6, [(0, i, 2) for i in range(1, 6)], [10.0, 0, 0, 0, 0, 0]),
    "cycle4": (4, [(0, 1, 1), (1, 2, 1), (2, 3, 1), (3, 0, 1)], [0.5, 0.5, 0.5, 0.5]),
    "diamond": (4, [(0, 1, 1), (0, 2, 1), (1, 3, 1), (2, 3, 1)], [0.5, 0.5, 0.5, 0.5]),
    "single": (1, [], [0.0]),
    "pair": (2, [(0, 1, 7)], [0.0, 0.0]),
    "grid3x3": (9, [(r * 3 + c, r * 3 + c + 1, 1) for r in range(3) for c in range(2)] +
                [(r * 3 + c, (r + 1) * 3 + c, 1) for r in range(2) for c in range(3)], None),
    "path40": (40, [(i, i + 1, 1 + (i % 3)) for i in range(39)], [float(i * (39 - i)) for i in range(40)]),
}


def unit_grid_lines(r=24, c=24):
    """Unit-weight r x c grid: the shortest-path counts from a corner are binomial coefficients, so
    at 24 x 24 they exceed 2^32 and the 32-bit count arithmetic wraps (C(46,23) = 8.2e12)."""
    edges = [(i * c + j, i * c + j + 1, 1) for i in range(r) for j in range(c - 1)]
    edges += [(i * c + j, (i + 1) * c + j, 1) for i in range(r - 1) for j in range(c)]
    return lines_of(edges, r * c)
