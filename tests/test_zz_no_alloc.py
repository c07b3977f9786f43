"""GPU test of the allocation-free in-place forward NTT.

ckks_ntt_forward_inplace_static serves callers that cannot let the library
allocate device memory (their device memory is reserved up front by their own
arena or a serving framework, or their deployment forbids device allocation
after start-up): it stages the transform's intermediate in a fixed 16 MiB
device array compiled into the library. Its output must equal the regular
entry point's word for word (exact integer arithmetic: tolerance zero), on
consecutive calls that reuse the shared array, and oversized batches must be
rejected. The default memory pool's high-water mark (where the library's
stream-ordered workspaces come from) must not move across a call, while the
regular in-place entry point does move it. This file is collected last and
also passes on its own.
"""
import ctypes

import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def _reference_forward(ctx, x):
    import torch
    d = cb.as_u64_tensor(x)
    out = torch.empty_like(d)
    rc = cb.lib().ckks_ntt_forward(ctx.handle, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                   x.shape[0], 0, x.shape[1], None)
    cb.check(rc)
    torch.cuda.synchronize()
    return cb.to_numpy_u64(out)


def _static_forward(ctx, x, limb_begin=0):
    import torch
    d = cb.as_u64_tensor(x)
    rc = cb.lib().ckks_ntt_forward_inplace_static(ctx.handle, ctypes.c_void_p(d.data_ptr()), x.shape[0],
                                                  limb_begin, x.shape[1], None)
    cb.check(rc)
    torch.cuda.synchronize()
    return cb.to_numpy_u64(d)


class _Pool:
    """The current device's default memory pool through the driver API
    (cuDeviceGetDefaultMemPool / cuMemPoolGet/SetAttribute, attribute 8 =
    CU_MEMPOOL_ATTR_USED_MEM_HIGH, attribute 7 = USED_MEM_CURRENT)."""

    def __init__(self):
        import torch
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def reset_high(self):
        zero = ctypes.c_uint64(0)
        assert self.cu.cuMemPoolSetAttribute(self.pool, 8, ctypes.byref(zero)) == 0

    def high(self):
        v = ctypes.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, 8, ctypes.byref(v)) == 0
        return v.value


def test_static_scratch_ntt_allocates_nothing(cuda):
    import torch
    import ckks_b200.params as params
    n = 1 << 14
    q = params.primes_below_bits(50, n, 4)
    ctx = cb.Context(14, q)
    rng = np.random.default_rng(5)
    x = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(3)])
    d = cb.as_u64_tensor(x)
    pool = _Pool()
    torch.cuda.synchronize()
    pool.reset_high()
    base = pool.high()
    cb.check(cb.lib().ckks_ntt_forward_inplace_static(ctx.handle, ctypes.c_void_p(d.data_ptr()), 3, 0, 4, None))
    torch.cuda.synchronize()
    assert pool.high() == base, "the static entry point drew on the device memory pool"
    # the regular in-place transform stages through a pool workspace: the probe sees it
    cb.check(cb.lib().ckks_ntt_forward(ctx.handle, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                       3, 0, 4, None))
    torch.cuda.synchronize()
    assert pool.high() > base


def test_static_scratch_limb_subrange_and_full_capacity(cuda):
    import ckks_b200.params as params
    n = 1 << 16
    q = params.primes_below_bits(50, n, 6)
    ctx = cb.Context(16, q)
    rng = np.random.default_rng(9)
    # limbs 2..4 of the basis (limb_begin > 0)
    sub = q[2:5]
    x = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in sub]) for _ in range(2)])
    import torch
    d = cb.as_u64_tensor(x)
    ref = torch.empty_like(d)
    cb.check(cb.lib().ckks_ntt_forward(ctx.handle, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                       2, 2, 3, None))
    assert np.array_equal(_static_forward(ctx, x, limb_begin=2), cb.to_numpy_u64(ref))
    # exactly the capacity: 8 polys x 4 limbs x 2^16 = 2^21 words
    y = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q[:4]]) for _ in range(8)])
    assert np.array_equal(_static_forward(ctx, y), _reference_forward(ctx, y))


def test_static_scratch_ntt_matches_regular_entry_point(cuda):
    import ckks_b200.params as params
    for log_n, limbs, polys in [(12, 3, 5), (16, 4, 2)]:
        n = 1 << log_n
        q = params.primes_below_bits(50, n, limbs)
        ctx = cb.Context(log_n, q)
        rng = np.random.default_rng(log_n)
        for call in range(2):  # two calls in a row share the static array
            x = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q]) for _ in range(polys)])
            assert np.array_equal(_static_forward(ctx, x), _reference_forward(ctx, x)), (log_n, call)


def test_static_scratch_rejects_oversized_batches(cuda):
    import ckks_b200.params as params
    n = 1 << 16
    q = params.primes_below_bits(50, n, 4)
    ctx = cb.Context(16, q)
    import torch
    d = torch.zeros((9, 4, n), dtype=torch.int64, device="cuda")  # 9 * 4 * 2^16 > 2^21 words
    rc = cb.lib().ckks_ntt_forward_inplace_static(ctx.handle, ctypes.c_void_p(d.data_ptr()), 9, 0, 4, None)
    assert rc == -1
    assert b"exceeds the fixed scratch" in cb.lib().ckks_last_error_string()
