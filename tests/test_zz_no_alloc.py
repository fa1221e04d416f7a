"""The allocation-free single-n entry point against the regular one and the oracle.

gb_check_single_batch_noalloc exists for callers that cannot allocate
device memory (stream capture, foreign memory pools, real-time loops); it
keeps its counters and candidate-prime table in a fixed file-scope device
array instead.  This file is collected last so that a failure here leaves
every other test already run; it also passes when run alone.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


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


@pytest.mark.parametrize("p_limit", [0, 97, 1000])
def test_noalloc_matches_the_oracle(gbmod, oracle, p_limit):
    """Against the CPU oracle directly (not only another CUDA path): small
    n below 2^21 (q may be a prime below the filter's trial divisors), n
    near 2^64, and bounds low enough that some n find no p (p = q = 0)."""
    rng = np.random.default_rng(23 + p_limit)
    ns = np.concatenate([
        np.arange(4, 4000, 2, dtype=np.uint64),
        (rng.integers(2, 1 << 20, size=2000, dtype=np.uint64) * 2),
        np.array([(1 << 21) - 2, 1 << 21, 2**64 - 2, 2**63, 2**32 + 2], dtype=np.uint64),
        (rng.integers(2, 2**63, size=4000, dtype=np.uint64) * 2),
    ]).astype(np.uint64)
    want = oracle.single_minp(ns, p_limit=p_limit or 65521)
    for _ in range(2):  # a second call over the same scratch
        p, q = _run_noalloc(gbmod, ns, p_limit)
        bad = np.nonzero(p != want)[0]
        assert bad.size == 0, (ns[bad[:8]], p[bad[:8]], want[bad[:8]])
        np.testing.assert_array_equal(q, np.where(want > 0, ns - want, 0))
    if p_limit:
        assert (want == 0).any()


# A child process that calls the entry point from the primary context, from a
# second context created on the same device, and from the primary context
# again: the fixed array exists once per context, so each context must get
# its own table (a table cached per device would leave the second context's
# array all zero and every p = 0).  Buffers come from the driver API, so the
# child needs neither torch nor a gb context.
_CHILD = r"""
import ctypes as C, sys
import numpy as np
sys.path.insert(0, sys.argv[1] + "/tests")
import oracle_lib
cu = C.CDLL("libcuda.so.1")
def ok(r, what):
    if r != 0:
        raise SystemExit(f"{what} failed: {r}")
gb = C.CDLL(sys.argv[1] + "/goldbach-gpu_b200/libgoldbach_b200.so")
f = gb.gb_check_single_batch_noalloc
f.restype = C.c_int
f.argtypes = [C.c_uint64, C.c_size_t, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p]
ok(cu.cuInit(0), "cuInit")
dev = C.c_int()
ok(cu.cuDeviceGet(C.byref(dev), 0), "cuDeviceGet")
rng = np.random.default_rng(5)
ns = (rng.integers(2, 2**63, size=4096, dtype=np.uint64) * 2).astype(np.uint64)
want = oracle_lib.Oracle().single_minp(ns, p_limit=65521)

def buffers():
    b = [C.c_uint64() for _ in range(3)]
    for x in b:
        ok(cu.cuMemAlloc_v2(C.byref(x), C.c_size_t(ns.nbytes)), "cuMemAlloc")
    ok(cu.cuMemcpyHtoD_v2(b[0], C.c_void_p(ns.ctypes.data), C.c_size_t(ns.nbytes)), "HtoD")
    return b

def check(b, label):
    st = f(b[0].value, len(ns), b[1].value, b[2].value, 0, None)
    if st != 0:
        raise SystemExit(f"{label}: status {st}")
    ok(cu.cuCtxSynchronize(), "sync")
    p = np.zeros_like(ns)
    ok(cu.cuMemcpyDtoH_v2(C.c_void_p(p.ctypes.data), b[1], C.c_size_t(ns.nbytes)), "DtoH")
    if not np.array_equal(p, want):
        raise SystemExit(f"{label}: {int((p != want).sum())} of {len(ns)} differ from the oracle")

prim = C.c_void_p()
ok(cu.cuDevicePrimaryCtxRetain(C.byref(prim), dev), "retain")
ok(cu.cuCtxSetCurrent(prim), "set current")
bp = buffers()
check(bp, "primary context")
ctx2 = C.c_void_p()
ok(cu.cuCtxCreate_v2(C.byref(ctx2), 0, dev), "cuCtxCreate")  # now current
b2 = buffers()
check(b2, "second context, first call")
check(b2, "second context, second call")
for x in b2:
    ok(cu.cuMemFree_v2(x), "free")
ok(cu.cuCtxDestroy_v2(ctx2), "cuCtxDestroy")
ok(cu.cuCtxSetCurrent(prim), "set current")
check(bp, "primary context again")
print("contexts ok")
"""


def test_noalloc_builds_its_table_in_every_context():
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "contexts ok" in r.stdout, (r.stdout[-2000:], r.stderr[-2000:])


def test_noalloc_rejects_bound_beyond_its_table(gbmod):
    import torch
    f = _noalloc(gbmod)
    n = torch.tensor([100], dtype=torch.int64, device="cuda")
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = f(n.data_ptr(), 1, out.data_ptr(), out.data_ptr(), 65522, torch.cuda.current_stream().cuda_stream)
    assert st == gbmod.GB_EINVAL
