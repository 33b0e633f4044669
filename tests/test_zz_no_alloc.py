"""pmc_coag_gpu_bin_sort_noalloc against the context's sort.

The no-alloc entry point serves callers that cannot allocate device memory
while they call us (a host model whose device memory is all pre-assigned by
its own allocator).  It must give the same bins and per-cell counts as
pmc_coag_gpu_sort, which allocates its scratch, and keep doing so on
consecutive calls that reuse its static scratch array: with one and with
three weight classes, and on a grid that leaves particles below and above
it (those get bin 0 or n_bin + 1 and stay out of the lists).
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


def context_sort(pop, cls=None, awa=None):
    st = pm.AeroState(pop.aero_data, pop.awa if awa is None else awa)
    st.add_particles(pop.vol, pop.group if cls is None else 1, weight_class=cls)
    edges, counts, bins = st.sort()
    return edges, counts, bins


def noalloc_sort(pop, edges, cls=None, n_class=1):
    import torch
    n = pop.n_part
    n_bin = len(edges) - 1
    vt = torch.from_numpy(sequential_vtot(pop.vol)).cuda()
    if cls is None:
        cls = np.ones(n, dtype=np.int32)
    cls = torch.from_numpy(np.ascontiguousarray(cls, dtype=np.int32)).cuda()
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


def check_list(b, cls, cnt, start, lst, n_bin, n_class):
    """list_dev holds start[n_bin*n_class] entries: every on-grid particle
    once, grouped by cell (bin fastest), increasing inside a cell."""
    n_cells = n_bin * n_class
    assert start[0] == 0 and np.array_equal(np.diff(start), cnt)
    on = (b >= 1) & (b <= n_bin)
    assert start[n_cells] == on.sum()
    assert np.array_equal(np.sort(lst[:start[n_cells]]), np.flatnonzero(on))
    for c in range(n_cells):
        seg = lst[start[c]:start[c + 1]]
        assert (b[seg] - 1 + n_bin * (cls[seg] - 1) == c).all() and (np.diff(seg) > 0).all()


def test_noalloc_sort_three_classes_matches_context_sort(gpu_lib):
    """The cell key bin + n_bin * (class - 1) with three weight classes,
    particles spread over the classes at random."""
    pop = aero_dist.brown_bimodal(40000, seed=33)
    cls = np.random.default_rng(5).integers(1, 4, pop.n_part).astype(np.int32)
    awa = pm.AeroWeightArray.flat(n_class=3)
    for call in range(2):  # two calls in a row on the shared scratch
        edges, counts, bins = context_sort(pop, cls, awa)
        n_bin = len(edges) - 1
        b, cnt, start, lst = noalloc_sort(pop, edges, cls, 3)
        assert np.array_equal(b, bins), call
        assert np.array_equal(cnt.reshape(3, n_bin).T, counts), call
        check_list(b, cls, cnt, start, lst, n_bin, 3)


def test_noalloc_sort_particles_off_the_grid(gpu_lib):
    """A grid narrower than the population: particles below it get bin 0,
    above it n_bin + 1, and neither is counted or listed.  The expected bins
    come from the oracle's bin_grid_find restatement."""
    from oracle import oracle as O
    pop = aero_dist.brown_bimodal(30000, seed=34)
    cls = np.random.default_rng(6).integers(1, 3, pop.n_part).astype(np.int32)
    r = np.array([O.vol2rad(v) for v in sequential_vtot(pop.vol)])
    lo, hi = np.quantile(r, [0.1, 0.9])
    n_bin = 25
    want = np.array([O.bin_find(n_bin, lo, hi, x) for x in r], dtype=np.int32)
    want = np.clip(want, 0, n_bin + 1)
    assert (want == 0).sum() > 1000 and (want == n_bin + 1).sum() > 1000
    for call in range(2):
        b, cnt, start, lst = noalloc_sort(pop, np.geomspace(lo, hi, n_bin + 1), cls, 2)
        assert np.array_equal(b, want), call
        on = (want >= 1) & (want <= n_bin)
        key = want[on] - 1 + n_bin * (cls[on] - 1)
        assert np.array_equal(cnt, np.bincount(key, minlength=2 * n_bin)), call
        check_list(b, cls, cnt, start, lst, n_bin, 2)


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
