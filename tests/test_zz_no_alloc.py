"""pmc_coag_gpu_bin_sort_noalloc against the context's sort.

The no-alloc entry point serves callers that cannot allocate device memory
while they call us (a host model whose device memory is all pre-assigned by
its own allocator).  It must give the same
bins and per-cell counts as pmc_coag_gpu_sort, which allocates its scratch,
and keep doing so on consecutive calls that reuse its static scratch array.
This file is collected last so a failure here does not hide other results."""
import ctypes

import numpy as np
import pytest

import partmc_b200 as pm
from partmc_b200 import _lib, aero_dist

pytestmark = pytest.mark.gpu


def sequential_vtot(vol):
    # the library sums species volumes in species order; numpy's sum may not
    v = vol[:, 0].copy()
    for s in range(1, vol.shape[1]):
        v = v + vol[:, s]
    return v


def context_sort(pop):
    st = pm.AeroState(pop.aero_data, pop.awa)
    st.add_particles(pop.vol, pop.group)
    edges, counts, bins = st.sort()
    return edges, counts, bins


def noalloc_sort(pop, edges):
    import torch
    n = pop.n_part
    n_bin = len(edges) - 1
    n_class = pop.awa.n_class
    vt = torch.from_numpy(sequential_vtot(pop.vol)).cuda()
    cls = torch.ones(n, dtype=torch.int32, device="cuda")
    b = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    cnt = torch.full((n_bin * n_class,), -7, dtype=torch.int32, device="cuda")
    start = torch.full((n_bin * n_class + 1,), -7, dtype=torch.int32, device="cuda")
    lst = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = _lib.lib().pmc_coag_gpu_bin_sort_noalloc(
        n, ctypes.c_void_p(vt.data_ptr()), ctypes.c_void_p(cls.data_ptr()), n_bin, n_class,
        float(edges[0]), float(edges[-1]), ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(cnt.data_ptr()),
        ctypes.c_void_p(start.data_ptr()), ctypes.c_void_p(lst.data_ptr()),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.STATUS_NAMES.get(rc, rc)
    torch.cuda.synchronize()
    return b.cpu().numpy(), cnt.cpu().numpy(), start.cpu().numpy(), lst.cpu().numpy()


def test_noalloc_sort_matches_context_sort_twice(gpu_lib):
    pops = [aero_dist.brown_20spec(30000, seed=31), aero_dist.brown_bimodal(50000, seed=32)]
    for call, pop in enumerate(pops + pops[:1]):  # consecutive calls, scratch reused
        edges, counts, bins = context_sort(pop)
        b, cnt, start, lst = noalloc_sort(pop, edges)
        n_bin = len(edges) - 1
        assert np.array_equal(b, bins), call
        assert np.array_equal(cnt.reshape(1, n_bin).T, counts), call
        assert start[0] == 0 and np.array_equal(np.diff(start), cnt)
        # list: every particle once, grouped by bin, increasing inside a bin
        assert np.array_equal(np.sort(lst), np.arange(pop.n_part))
        for k in range(n_bin):
            seg = lst[start[k]:start[k + 1]]
            assert (b[seg] == k + 1).all() and (np.diff(seg) > 0).all()


def test_noalloc_rejects_sizes_over_its_limit(gpu_lib):
    L = _lib.lib()
    null = ctypes.c_void_p(0)
    rc = L.pmc_coag_gpu_bin_sort_noalloc((1 << 21) + 1, null, null, 40, 1, 1e-9, 1e-5, null, null, null, null,
                                         null)
    assert rc == 1 or rc == 3  # arguments are checked before sizes
    import torch
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = ctypes.c_void_p(d.data_ptr())
    rc = L.pmc_coag_gpu_bin_sort_noalloc((1 << 21) + 1, p, p, 40, 1, 1e-9, 1e-5, p, p, p, p, null)
    assert rc == 3  # PMC_ERR_CAPACITY
    rc = L.pmc_coag_gpu_bin_sort_noalloc(10, p, p, 300, 4, 1e-9, 1e-5, p, p, p, p, null)
    assert rc == 3
