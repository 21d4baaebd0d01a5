"""btk_direct_sum_noalloc: the direct sum with static device scratch.

Collected last (file name) so that it also runs after every other GPU test
has used the device. Every case goes through the C ABI and compares against
btk_direct_sum (which allocates its scratch per call) bit for bit, on two
calls in a row with different source sets (the second smaller, so stale
scratch beyond its count is present and must not be read). The allocation
check reads the high-water mark of the device's default memory pool, the
pool the library's own stream-ordered allocations draw from: it rises under
btk_direct_sum and must stay at zero under the no-alloc entry point.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_SOURCES = 1 << 18


def _problem(rng, dim, nt, ns):
    t = tuple(rng.random(nt) for _ in range(dim))
    s = tuple(rng.random(ns) for _ in range(dim))
    q = rng.standard_normal(ns)
    return t, s, q


def _run(lib, fn, dim, kind, eps, t, s, q):
    import torch
    from barytreek_b200 import _lib, treecode
    dev = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in t]
    src = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in s]
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    nc = treecode.ncomp(dim, kind)
    out = torch.full((nc, len(t[0])), float("nan"), dtype=torch.float64, device="cuda")
    z_t = _lib.ptr(dev[2]) if dim == 3 else None
    z_s = _lib.ptr(src[2]) if dim == 3 else None
    _lib.check(getattr(lib, fn)(dim, kind, eps, len(t[0]), _lib.ptr(dev[0]), _lib.ptr(dev[1]), z_t, len(s[0]),
                                _lib.ptr(src[0]), _lib.ptr(src[1]), z_s, _lib.ptr(qd), _lib.ptr(out), None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("dim,kind", [(2, 0), (2, 2), (3, 0), (3, 1), (3, 2)])
def test_two_calls_in_a_row_match_direct_sum(dim, kind, lib):
    rng = np.random.default_rng(100 + 10 * dim + kind)
    first = _problem(rng, dim, 700, 5000)
    second = _problem(rng, dim, 500, 3001)
    for t, s, q in (first, second):
        a = _run(lib, "btk_direct_sum_noalloc", dim, kind, 1e-4, t, s, q)
        b = _run(lib, "btk_direct_sum", dim, kind, 1e-4, t, s, q)
        assert np.isfinite(a).all()
        assert np.array_equal(a, b)


def test_limit_and_empty_sources(lib):
    import torch
    from barytreek_b200 import _lib
    rng = np.random.default_rng(7)
    t, s, q = _problem(rng, 3, 64, MAX_SOURCES)
    a = _run(lib, "btk_direct_sum_noalloc", 3, 2, 1e-4, t, s, q)
    b = _run(lib, "btk_direct_sum", 3, 2, 1e-4, t, s, q)
    assert np.array_equal(a, b)
    x = torch.zeros(MAX_SOURCES + 1, dtype=torch.float64, device="cuda")
    p = _lib.ptr(x)
    # no sources (valid pointers, count 0): every output is zero
    out = torch.full((4, 64), float("nan"), dtype=torch.float64, device="cuda")
    _lib.check(lib.btk_direct_sum_noalloc(3, 2, 1e-4, 64, p, p, p, 0, p, p, p, p, _lib.ptr(out), None))
    torch.cuda.synchronize()
    assert not out.cpu().numpy().any()
    st = lib.btk_direct_sum_noalloc(3, 0, 0.0, 1, p, p, p, MAX_SOURCES + 1, p, p, p, p, p, None)
    assert st == 1  # BTK_ERR_INVALID_ARGUMENT
    assert b"static scratch" in lib.btk_last_error()


def _pool_high_water(reset):
    import torch
    from cuda.bindings import driver, runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    attr = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
    if reset:
        # the high-water mark restarts at the pool's current use (memory that
        # earlier work still holds, such as the drop-in entry points' cached
        # state), which this returns
        (err,) = rt.cudaMemPoolSetAttribute(pool, attr, driver.cuuint64_t(0))
        assert err == rt.cudaError_t.cudaSuccess
        err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
        assert err == rt.cudaError_t.cudaSuccess
        return int(v)
    err, v = rt.cudaMemPoolGetAttribute(pool, attr)
    assert err == rt.cudaError_t.cudaSuccess
    return int(v)


def test_no_device_allocation(lib):
    rng = np.random.default_rng(11)
    t, s, q = _problem(rng, 3, 256, 20000)
    _run(lib, "btk_direct_sum_noalloc", 3, 2, 1e-4, t, s, q)  # first call on the device: setup
    base = _pool_high_water(reset=True)
    _run(lib, "btk_direct_sum", 3, 2, 1e-4, t, s, q)
    assert _pool_high_water(reset=False) > base  # the check sees the allocating entry point
    base = _pool_high_water(reset=True)
    for _ in range(2):
        _run(lib, "btk_direct_sum_noalloc", 3, 2, 1e-4, t, s, q)
    assert _pool_high_water(reset=False) == base
