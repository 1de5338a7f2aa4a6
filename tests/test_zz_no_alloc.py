"""felog_build_alias_noalloc: alias tables for callers that cannot allocate.

Some callers cannot call cudaMalloc (their device memory belongs to their own
allocator, or they must not grow their footprint once running).  This entry
point builds the same tables as felog_build_alias from buffers the caller
already owns, using a fixed device array for its worklists.  The test calls it
through the C ABI twice in a row (the second call reuses the array the first
one left behind) and compares both results with felog_build_alias on the same
graph.  The tables are deterministic, so the comparison is exact.  The device
buffers of the test itself come from torch: the test plays the caller, and the
entry point allocates nothing, which the test checks by reading the device's
free memory around the second call.
"""
import ctypes

import numpy as np
import pytest

import felog_b200 as fb

pytestmark = pytest.mark.gpu


def _graph():
    g = fb.synth_graph(seed=2, v_target=2048, e_target=8192, abcd=(0.6, 0.15, 0.15, 0.1), lognormal=True)
    return g["edges"], g["v_num"]


def test_noalloc_alias_matches_allocating_entry_point_twice():
    import torch

    edges, V = _graph()
    f = fb.Felog(v_num=V)
    f.load_graph(edges, V)
    f.build_alias()
    prob_ref, alias_ref = f.alias()
    row_ptr, _, weight = f.csr()
    M = len(weight)
    assert M <= 1 << 22
    dev = torch.device("cuda:0")
    d_row = torch.from_numpy(row_ptr.astype(np.int64)).to(dev)
    d_w = torch.from_numpy(weight.astype(np.float32)).to(dev)
    for call in range(2):
        d_prob = torch.full((M,), -1.0, dtype=torch.float32, device=dev)
        d_alias = torch.full((M,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        fb.build_alias_noalloc(d_row.data_ptr(), d_w.data_ptr(), V, M, d_prob.data_ptr(), d_alias.data_ptr())
        torch.cuda.synchronize()
        if call == 1:
            # the first call may map the fixed array; the second one changes nothing
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        np.testing.assert_array_equal(d_prob.cpu().numpy(), prob_ref, err_msg=f"call {call}")
        np.testing.assert_array_equal(d_alias.cpu().numpy().view(np.uint32), alias_ref, err_msg=f"call {call}")
    f.close()


def test_noalloc_alias_rejects_oversized_graphs_and_bad_weights():
    import torch

    L = fb.gpu_lib()
    big = (1 << 22) + 1
    st = L.felog_build_alias_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), 10, big, ctypes.c_void_p(16),
                                     ctypes.c_void_p(16), None)
    assert st == 1  # FELOG_INVALID_ARG, before any device access
    dev = torch.device("cuda:0")
    row = torch.tensor([0, 2, 3], dtype=torch.int64, device=dev)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float32, device=dev)
    prob = torch.zeros(3, dtype=torch.float32, device=dev)
    alias = torch.zeros(3, dtype=torch.int32, device=dev)
    with pytest.raises(fb.FelogError) as ei:
        fb.build_alias_noalloc(row.data_ptr(), w.data_ptr(), 2, 3, prob.data_ptr(), alias.data_ptr())
    assert ei.value.status == 1
    # the error word is cleared by the next call
    w[1] = 2.0
    fb.build_alias_noalloc(row.data_ptr(), w.data_ptr(), 2, 3, prob.data_ptr(), alias.data_ptr())


def test_noalloc_alias_rejects_inconsistent_row_ptr():
    import torch

    dev = torch.device("cuda:0")
    # vertex 1's range ends past e_num (5 > 4), vertex 2's range runs backwards;
    # every buffer is large enough for the offsets, so the test itself never
    # writes out of bounds
    row = torch.tensor([0, 2, 5, 3], dtype=torch.int64, device=dev)
    w = torch.ones(8, dtype=torch.float32, device=dev)
    prob = torch.zeros(8, dtype=torch.float32, device=dev)
    alias = torch.zeros(8, dtype=torch.int32, device=dev)
    with pytest.raises(fb.FelogError) as ei:
        fb.build_alias_noalloc(row.data_ptr(), w.data_ptr(), 3, 4, prob.data_ptr(), alias.data_ptr())
    assert ei.value.status == 1
    L = fb.gpu_lib()
    assert L.felog_build_alias_noalloc(row.data_ptr(), w.data_ptr(), 0, 4, prob.data_ptr(), alias.data_ptr(),
                                       None) == 1  # edges without vertices
    # a consistent CSR over the same buffers succeeds afterwards
    row2 = torch.tensor([0, 2, 3, 4], dtype=torch.int64, device=dev)
    fb.build_alias_noalloc(row2.data_ptr(), w.data_ptr(), 3, 4, prob.data_ptr(), alias.data_ptr())
    torch.cuda.synchronize()
    assert torch.all(prob[:4] == 1.0)
