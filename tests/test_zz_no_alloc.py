"""GPU: the allocation-free single-source entry point (qbc_bc_source_static).

It serves callers that cannot allocate device memory when they need BC (a process whose memory
manager already holds the GPU's memory, or a latency-bound loop that must not call cudaMalloc /
cudaFree).  Its scratch is a static device array inside the library, so its output must match the
allocating entry point's (qbc_bc_sources) within the suite's BC tolerance, including on repeated
calls that reuse the array.  This file is collected last on purpose.
"""
import ctypes as C
import os

import numpy as np
import pytest

import gpu_betweennesscentrality_b200 as Q
from conftest import GOLDEN, rel_err
from gpu_betweennesscentrality_b200 import capi, synth
from util import BC_RTOL, lines_of

pytestmark = pytest.mark.gpu


def _static_call(idx, source, d_bc_ptr):
    capi.check(capi.lib().qbc_bc_source_static(idx.h, int(source), C.c_void_p(d_bc_ptr), None))


def test_static_entry_matches_allocating_entry_two_calls():
    import torch

    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    idx = g.build_index()
    d_bc = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    s1, s2 = 5, 1234
    _static_call(idx, s1, d_bc.data_ptr())
    torch.cuda.synchronize()
    first = d_bc.cpu().numpy().copy()
    assert rel_err(first, idx.bc_sources(np.array([s1], np.int32))) <= BC_RTOL
    _static_call(idx, s2, d_bc.data_ptr())  # second call reuses the static scratch, accumulates
    torch.cuda.synchronize()
    both = d_bc.cpu().numpy()
    assert rel_err(both, idx.bc_sources(np.array([s1, s2], np.int32))) <= BC_RTOL
    assert np.any(both != first)


def test_static_entry_h2h_index():
    import torch

    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    idx = g.build_index(Q.QBC_INDEX_H2H, Q.read_order(os.path.join(GOLDEN, "g2k.order"), n))
    d_bc = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    for s in (0, 999):
        _static_call(idx, s, d_bc.data_ptr())
    torch.cuda.synchronize()
    assert rel_err(d_bc.cpu().numpy(), idx.bc_sources(np.array([0, 999], np.int32))) <= BC_RTOL


def test_static_entry_allocates_no_device_memory():
    """after a first call (which looks up the array's address), further calls leave the device's
    free memory and the index's own device bytes unchanged"""
    import torch

    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    idx = g.build_index()
    d_bc = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    _static_call(idx, 0, d_bc.data_ptr())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    bytes0 = int(idx.info()[5])
    for s in range(1, 40):
        _static_call(idx, s, d_bc.data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0 and int(idx.info()[5]) == bytes0
    assert rel_err(d_bc.cpu().numpy(), idx.bc_sources(np.arange(40, dtype=np.int32))) <= BC_RTOL


def test_static_entry_csr_index():
    """the label-free index runs the shortest-path sweep in the static array"""
    import torch

    n, u, v, w = synth.read_graph_lines(os.path.join(GOLDEN, "g2k.txt"))
    g = Q.Graph(device=0)
    g.ReadLines(n, u, v, w)
    idx = g.build_index(Q.QBC_INDEX_CSR)
    d_bc = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    for s in (3, 1500):
        _static_call(idx, s, d_bc.data_ptr())
    torch.cuda.synchronize()
    assert rel_err(d_bc.cpu().numpy(), idx.bc_sources(np.array([3, 1500], np.int32))) <= BC_RTOL


def test_static_entry_rejects_trees_taller_than_its_label_kernel():
    """a 6,000-vertex path has a tree of ~6,000 levels: refused with QBC_EINVAL by the static entry
    point on a label index, served by the batched path and by the static entry point on a CSR index"""
    import torch

    n = 6000
    nn, u, v, w = lines_of([(i, i + 1, 1 + i % 3) for i in range(n - 1)], n)
    g = Q.Graph(device=0)
    g.ReadLines(nn, u, v, w)
    idx = g.build_index()
    assert int(idx.info()[3]) > 5200
    d_bc = torch.zeros(n, dtype=torch.float64, device="cuda:0")
    with pytest.raises(Q.QbcError) as e:
        _static_call(idx, 0, d_bc.data_ptr())
    assert e.value.code == capi.QBC_EINVAL and "tree height" in str(e.value)
    csr = g.build_index(Q.QBC_INDEX_CSR)
    _static_call(csr, 0, d_bc.data_ptr())
    torch.cuda.synchronize()
    assert rel_err(d_bc.cpu().numpy(), csr.bc_sources(np.array([0], np.int32))) <= BC_RTOL


def test_static_entry_rejects_graphs_above_the_limit():
    n = 131073  # one more than QBC_STATIC_MAX_VERTICES: a star stays tiny to index
    nn, u, v, w = lines_of([(0, i, 1) for i in range(1, n)], n)
    g = Q.Graph(device=0)
    g.ReadLines(nn, u, v, w)
    idx = g.build_index(upload=False)
    with pytest.raises(Q.QbcError) as e:
        capi.check(capi.lib().qbc_bc_source_static(idx.h, 0, C.c_void_p(16), None))
    assert e.value.code == capi.QBC_EINVAL and "131072" in str(e.value)
