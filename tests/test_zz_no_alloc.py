"""GPU test of the allocation-free in-place forward NTT.

ckks_ntt_forward_inplace_static serves callers that cannot let the library
allocate device memory (their device memory is reserved up front by their own
arena or a serving framework, or their deployment forbids device allocation
after start-up): it stages the transform's intermediate in a fixed 16 MiB
device array compiled into the library. Its output must equal the regular
entry point's word for word (exact integer arithmetic: tolerance zero), on
consecutive calls that reuse the shared array, and oversized batches must be
rejected. This file is collected last and also passes on its own.
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
