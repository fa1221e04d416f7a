"""The allocation-free single-n entry point against the regular one.

gb_check_single_batch_noalloc exists for callers that cannot allocate
device memory (stream capture, foreign memory pools, real-time loops); it
keeps its counters and candidate-prime table in a fixed file-scope device
array instead.  This file is collected last so that a failure here leaves
every other test already run; it also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(gbmod):
    L = gbmod.load()
    f = L.gb_check_single_batch_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_uint64, ctypes.c_void_p]
    return f


def _run_noalloc(gbmod, ns, p_limit=0):
    import torch
    f = _noalloc(gbmod)
    n_dev = torch.from_numpy(ns.view(np.int64)).cuda()
    p_dev = torch.full_like(n_dev, -1)
    q_dev = torch.full_like(n_dev, -1)
    s = torch.cuda.current_stream()
    st = f(n_dev.data_ptr(), len(ns), p_dev.data_ptr(), q_dev.data_ptr(), p_limit, s.cuda_stream)
    assert st == 0, st
    s.synchronize()
    return (p_dev.cpu().numpy().view(np.uint64), q_dev.cpu().numpy().view(np.uint64))


def test_noalloc_matches_regular_entry_point_twice(ctx, gbmod):
    limit = 65521  # the allocation-free table's reach (GB_NOALLOC_P_LIMIT)
    rng = np.random.default_rng(11)
    first = (rng.integers(2, 2**63, size=5000, dtype=np.uint64) * 2).astype(np.uint64)
    second = np.concatenate([np.array([4, 6, 8, 2**64 - 2, 10**18, 10**12], dtype=np.uint64),
                             (rng.integers(2, 2**40, size=3000, dtype=np.uint64) * 2)]).astype(np.uint64)
    for ns in (first, second):  # two calls in a row share the fixed scratch
        p, q = _run_noalloc(gbmod, ns)
        p_ref, q_ref, _ = ctx.check_single(ns, p_limit=limit)
        np.testing.assert_array_equal(p, p_ref)
        np.testing.assert_array_equal(q, q_ref)
        assert (p > 0).all()


def test_noalloc_rejects_bound_beyond_its_table(gbmod):
    import torch
    f = _noalloc(gbmod)
    n = torch.tensor([100], dtype=torch.int64, device="cuda")
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = f(n.data_ptr(), 1, out.data_ptr(), out.data_ptr(), 65522, torch.cuda.current_stream().cuda_stream)
    assert st == gbmod.GB_EINVAL
