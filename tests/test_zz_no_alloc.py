"""mog_direct_sum_noalloc (fixed scratch, no device allocation) against
mog_direct_sum (stream-ordered allocation), both called through the C ABI.

Collected last on purpose: it must give the same answers in a process
where the other tests have already run as in a fresh one."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

PAIRS = 1 << 19   # scratch capacity in (target, chunk) pairs


def _lib():
    from mog_solver_b200 import _lib

    return _lib, _lib.lib()


def _sets(nt, ns, seed, world=100.0):
    rng = np.random.default_rng(seed)
    t = np.zeros((nt, 4), np.float32)
    t[:, :3] = rng.uniform(0, world, (nt, 3))
    s = np.zeros((ns, 4), np.float32)
    s[:, :3] = rng.uniform(0, world, (ns, 3))
    s[:, 3] = rng.uniform(0.5, 1.5, ns) / ns
    return torch.from_numpy(t).cuda(), torch.from_numpy(s).cuda()


def _call(fn, T, S, world, g_eff, soft):
    out = torch.full((T.shape[0], 3), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = fn(T.data_ptr(), T.shape[0], S.data_ptr(), S.shape[0], world, g_eff, soft, out.data_ptr(),
            ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


@pytest.mark.parametrize("nt,ns", [(1000, 5000), (16384, 300000), (3, 1)])
def test_noalloc_matches_allocating_entry_twice_in_a_row(nt, ns):
    L, lib = _lib()
    world, g_eff = 100.0, 0.0123
    # two calls in a row with different inputs: the second must not see
    # anything the first left in the scratch
    for seed, soft in ((nt, 0.0), (nt + 7, 1.5)):
        T, S = _sets(nt, ns, seed, world)
        rc_a, ref = _call(lib.mog_direct_sum, T, S, world, g_eff, soft)
        rc_b, got = _call(lib.mog_direct_sum_noalloc, T, S, world, g_eff, soft)
        assert rc_a == L.MOG_OK and rc_b == L.MOG_OK, L.lib().mog_last_error()
        assert np.isfinite(got).all()
        # same chunking and summation order: bit for bit
        assert np.array_equal(got, ref)


def test_noalloc_leaves_device_memory_unchanged():
    """The point of the entry point: after the first call on a device (which
    loads its kernels), further calls take no device memory at all."""
    L, lib = _lib()
    T, S = _sets(4096, 100000, 3)
    out = torch.empty((T.shape[0], 3), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def call():
        rc = lib.mog_direct_sum_noalloc(T.data_ptr(), T.shape[0], S.data_ptr(), S.shape[0], 100.0,
                                        1.0, 0.0, out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == L.MOG_OK, lib.mog_last_error()

    call()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_noalloc_rejects_requests_beyond_the_scratch():
    L, lib = _lib()
    ns = 300000                       # 32 source chunks
    T, S = _sets(PAIRS // 32 + 1, ns, 11)
    rc, out = _call(lib.mog_direct_sum_noalloc, T, S, 100.0, 1.0, 0.0)
    assert rc == L.MOG_ERR_ARG
    assert b"scratch" in lib.mog_last_error()
    assert np.isnan(out).all()        # nothing was launched
    # the largest request that fits still runs
    T2 = T[: PAIRS // 32].contiguous()
    rc2, _ = _call(lib.mog_direct_sum_noalloc, T2, S, 100.0, 1.0, 0.0)
    assert rc2 == L.MOG_OK
