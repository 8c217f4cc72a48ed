"""The allocation-free entry point, checked against mce_count.

mce_count_oriented_noalloc serves callers that cannot allocate device
memory (a process whose GPU memory another allocator owns, or a loop that
cannot afford cudaMalloc's device synchronisation).  It searches an oriented
graph the caller already holds in device memory, using a fixed array inside
the library as scratch.  This file is collected last so that a failure here
cannot stop the other tests from running first.
"""
import ctypes as C

import numpy as np
import pytest

import mce_b200 as mce

pytestmark = pytest.mark.gpu


def oriented_on_device(g):
    """The graph's oriented CSR and its roots as torch tensors on cuda:0."""
    import torch
    with mce.Graph.from_host(g) as dg:
        ref = dg.count()
        split, cs = dg.split_csr()
    dplus = g.row_ptr[1:g.n + 1] - split
    roots = np.nonzero(dplus > 0)[0].astype(np.int32)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
           for k, v in dict(rp=g.row_ptr[:g.n + 1].astype(np.int32), split=split, cs=cs,
                            roots=roots).items()}
    return ref, dev


def call(dev, hist, n_roots=None):
    import torch
    k = len(dev["roots"]) if n_roots is None else n_roots
    return mce._lib.mce_count_oriented_noalloc(
        C.c_void_p(dev["rp"].data_ptr()), C.c_void_p(dev["split"].data_ptr()),
        C.c_void_p(dev["cs"].data_ptr()), len(dev["split"]), C.c_void_p(dev["roots"].data_ptr()),
        k, C.c_void_p(hist.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_matches_mce_count_twice():
    import torch
    # ER(10000, 0.002) + 20 planted cliques: every root has <= 32 later and
    # <= 1024 earlier neighbours, so the whole graph fits the entry point
    g = mce.gen_er(10000, 0.002, 1, 20, 6, 12)
    ref, dev = oriented_on_device(g)
    hist = torch.zeros(mce.HIST_MAX, dtype=torch.int64, device="cuda")
    for _ in range(2):  # the second call reuses the scratch the first one left
        assert call(dev, hist) == mce.OK
        h = hist.cpu().numpy().astype(np.uint64)
        assert np.array_equal(h, ref.hist)  # bit-exact, like every count test
        assert int(h.sum()) == ref.total


def test_noalloc_rejects_roots_beyond_its_limit():
    import torch
    from graphs import complete
    ref, dev = oriented_on_device(complete(40))  # root 0 has 39 later neighbours
    hist = torch.zeros(mce.HIST_MAX, dtype=torch.int64, device="cuda")
    assert call(dev, hist) == mce.ELIMIT
    assert int(hist.sum().item()) == 0


@pytest.mark.parametrize("bad", ["n", "-1"])
def test_noalloc_rejects_root_ids_outside_the_graph(bad):
    import torch
    g = mce.gen_er(2000, 0.004, 3, 4, 5, 8)
    ref, dev = oriented_on_device(g)
    roots = dev["roots"].clone()
    roots[len(roots) // 2] = g.n if bad == "n" else -1
    hist = torch.full((mce.HIST_MAX,), 7, dtype=torch.int64, device="cuda")
    assert call(dict(dev, roots=roots), hist) == mce.EINVAL
    # caught before the search: the histogram is left as it was
    assert bool((hist == 7).all().item())
    # the scratch stays usable: a good call right after gives the full answer
    assert call(dev, hist) == mce.OK
    assert np.array_equal(hist.cpu().numpy().astype(np.uint64), ref.hist)
