"""Writes the committed golden inputs: a seeded 2,024-vertex perturbed grid (the 2k config), its
min-degree order file (0-based, the order-file format of src/buildIndex.cpp:13-20) and a 10-vertex
query batch (RQ.cu:595-601 format).

    python tests/golden/make_inputs.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from gpu_betweennesscentrality_b200 import synth  # noqa: E402


def main():
    g = synth.grid_graph(2000, seed=1)
    synth.write_graph(os.path.join(HERE, "g2k.txt"), g)
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
    import pyoracle

    n, u, v, w = synth.read_graph_lines(os.path.join(HERE, "g2k.txt"))
    tc = pyoracle.TreeCount(n, u, v, w)  # TreeDecomp::Reduce min-degree order
    order = np.empty(n, np.int32)
    order[tc.del_order - 1] = np.arange(n)
    synth.write_order(os.path.join(HERE, "g2k.order"), order)
    synth.write_query(os.path.join(HERE, "g2k.query"), synth.query_set(n, 10, seed=2))


if __name__ == "__main__":
    main()
