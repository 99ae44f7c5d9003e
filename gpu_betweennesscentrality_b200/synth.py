"""Seeded synthetic road-like graphs, order files and query batches.

The reference ships one real road graph (data/roadData/LosAngeles.txt) and no generator.  The
workloads here are perturbed 2-D grids in the reference's text formats:

* graph file (README.md:18, src/Graph.cpp:11-36): ``n m`` then ``m`` lines ``u v w``, 1-based,
  one directed arc per line; every undirected edge is written in both directions;
* order file (src/buildIndex.cpp:13-20): ``n`` then ``n`` lines ``id order``, 0-based ids;
* query batch (RQ.cu:595-601): ``q`` then ``q`` 1-based ids.

Grid recipe: R = floor(sqrt(n)), C = ceil(n / R) vertices on a jittered lattice (spacing 100,
jitter +-30).  A random spanning tree (minimum spanning tree under i.i.d. uniform keys) keeps the
graph connected; ``delete_frac`` of all lattice edges is then removed from the non-tree edges
(0.27 reproduces ~2.8k edges at 2k vertices and ~72k at 50k).  Weight = round(euclid * U[0.8,1.2])
clipped to 1..1000.  Shortcuts: ``shortcut_frac * n`` distinct non-adjacent random pairs with
weights U{500..5000}.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np


@dataclasses.dataclass
class EdgeList:
    """Undirected simple graph, 0-based endpoints, one row per edge."""

    n: int
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray

    @property
    def m_undirected(self) -> int:
        return int(self.u.shape[0])

    def arcs(self):
        """Both directions interleaved (u->v then v->u), 1-based, as the graph file lists them."""
        a = np.empty(2 * self.m_undirected, dtype=np.int32)
        b = np.empty_like(a)
        ww = np.empty_like(a)
        a[0::2], b[0::2] = self.u + 1, self.v + 1
        a[1::2], b[1::2] = self.v + 1, self.u + 1
        ww[0::2] = ww[1::2] = self.w
        return a, b, ww


def grid_graph(n_target: int, seed: int = 1, delete_frac: float = 0.27, shortcut_frac: float = 0.0,
               spacing: float = 100.0, jitter: float = 30.0) -> EdgeList:
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import minimum_spanning_tree

    rng = np.random.default_rng(seed)
    R = max(1, int(np.floor(np.sqrt(n_target))))
    C = int(np.ceil(n_target / R))
    N = R * C
    ids = np.arange(N)
    xs = (ids % C) * spacing + rng.uniform(-jitter, jitter, N)
    ys = (ids // C) * spacing + rng.uniform(-jitter, jitter, N)
    grid = ids.reshape(R, C)
    eh = np.stack([grid[:, :-1].ravel(), grid[:, 1:].ravel()], 1)
    ev = np.stack([grid[:-1, :].ravel(), grid[1:, :].ravel()], 1)
    E = np.concatenate([eh, ev]).astype(np.int64)
    keys = rng.uniform(1.0, 2.0, E.shape[0])
    mst = minimum_spanning_tree(coo_matrix((keys, (E[:, 0], E[:, 1])), shape=(N, N)).tocsr()).tocoo()
    tree = set(zip(np.minimum(mst.row, mst.col).tolist(), np.maximum(mst.row, mst.col).tolist()))
    is_tree = np.fromiter(((int(a), int(b)) in tree for a, b in E), dtype=bool, count=E.shape[0])
    non_tree = np.flatnonzero(~is_tree)
    n_del = min(int(round(delete_frac * E.shape[0])), non_tree.shape[0])
    drop = rng.choice(non_tree, size=n_del, replace=False) if n_del else np.empty(0, np.int64)
    keep = np.ones(E.shape[0], dtype=bool)
    keep[drop] = False
    E = E[keep]
    d = np.hypot(xs[E[:, 0]] - xs[E[:, 1]], ys[E[:, 0]] - ys[E[:, 1]])
    w = np.clip(np.rint(d * rng.uniform(0.8, 1.2, E.shape[0])), 1, 1000).astype(np.int32)
    u, v = E[:, 0].astype(np.int32), E[:, 1].astype(np.int32)
    n_sc = int(round(shortcut_frac * N))
    if n_sc:
        present = set(zip(np.minimum(u, v).tolist(), np.maximum(u, v).tolist()))
        su, sv = [], []
        while len(su) < n_sc:
            a, b = rng.integers(0, N, size=2)
            a, b = int(min(a, b)), int(max(a, b))
            if a == b or (a, b) in present:
                continue
            present.add((a, b))
            su.append(a)
            sv.append(b)
        sw = rng.integers(500, 5001, size=n_sc).astype(np.int32)
        u = np.concatenate([u, np.asarray(su, np.int32)])
        v = np.concatenate([v, np.asarray(sv, np.int32)])
        w = np.concatenate([w, sw])
    return EdgeList(N, u, v, w)


def query_set(n: int, q: int, seed: int = 2) -> np.ndarray:
    """q distinct 0-based vertex ids drawn uniformly."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(q, n), replace=False)).astype(np.int32)


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count))).astype(np.int64).clip(lo, hi)


def write_graph(path: str, g: EdgeList) -> None:
    a, b, w = g.arcs()
    with open(path, "w") as f:
        f.write(f"{g.n} {a.shape[0]}\n")
        np.savetxt(f, np.stack([a, b, w], 1), fmt="%d")


def read_graph_lines(path: str):
    """Raw lines of a graph file: (n, u1, v1, w) as int32 arrays, 1-based, unmodified."""
    with open(path) as f:
        n, m = map(int, f.readline().split())
        data = np.loadtxt(f, dtype=np.int64, max_rows=m, ndmin=2)
    if data.shape[0] != m:
        raise ValueError(f"{path}: expected {m} arc lines, found {data.shape[0]}")
    return n, data[:, 0].astype(np.int32), data[:, 1].astype(np.int32), data[:, 2].astype(np.int32)


def write_order(path: str, node_order: np.ndarray) -> None:
    """node_order[vid] = contraction rank (0 first), 0-based ids."""
    n = node_order.shape[0]
    with open(path, "w") as f:
        f.write(f"{n}\n")
        np.savetxt(f, np.stack([np.arange(n), node_order], 1), fmt="%d")


def write_query(path: str, ids0: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write(f"{ids0.shape[0]}\n")
        np.savetxt(f, ids0.reshape(-1, 1) + 1, fmt="%d")


def cached_graph(cache_dir: str, n_target: int, seed: int = 1, shortcut_frac: float = 0.0,
                 delete_frac: float = 0.27) -> str:
    """Write (once) and return the path of a generated graph file."""
    os.makedirs(cache_dir, exist_ok=True)
    tag = f"grid_{n_target}_s{seed}_d{int(delete_frac * 1000)}_sc{int(shortcut_frac * 1000)}.txt"
    path = os.path.join(cache_dir, tag)
    if not os.path.exists(path):
        tmp = path + f".tmp{os.getpid()}"
        write_graph(tmp, grid_graph(n_target, seed=seed, delete_frac=delete_frac, shortcut_frac=shortcut_frac))
        os.replace(tmp, path)
    return path
