"""GPU parity of the FP64 CKKS encode/decode (ckks/embedding.rs:57-349,
application_support/ckks.rs:39-130) with the oracle's restatement of the
reference's operation order: encoded residues equal word for word and decoded
doubles equal bit for bit (tolerance zero), including values beyond 2^63
after scaling and uniformly random residues (large CRT values)."""
import numpy as np
import pytest

import ckks_b200 as cb

pytestmark = pytest.mark.gpu


def host(t):
    return cb.to_numpy_u64(t)


@pytest.mark.parametrize("log_n,limbs,scale_log", [(10, 3, 40), (12, 3, 50), (16, 4, 50), (11, 5, 90)])
def test_encode_bit_exact(oracle, cuda, log_n, limbs, scale_log):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(50, n, limbs)]
    ctx = cb.Context(log_n, q)
    rng = np.random.default_rng(log_n)
    msgs = rng.uniform(-1, 1, (3, n // 2)) + 1j * rng.uniform(-1, 1, (3, n // 2))
    scale = 2.0 ** scale_log
    got = host(cb.encode(ctx, msgs, limbs, scale))
    for i in range(3):
        assert np.array_equal(got[i], oracle.encode(msgs[i], q, scale)), i
    # a lower level (Q prefix)
    got2 = host(cb.encode(ctx, msgs[:1], 2, scale))
    assert np.array_equal(got2[0], oracle.encode(msgs[0], q[:2], scale))


@pytest.mark.parametrize("log_n,limbs", [(10, 3), (13, 6), (16, 24)])
def test_decode_bit_exact(oracle, cuda, log_n, limbs):
    n = 1 << log_n
    q = [int(x) for x in oracle.primes_below_bits(50, n, limbs)]
    ctx = cb.Context(log_n, q)
    rng = np.random.default_rng(100 + log_n)
    scale = 2.0 ** 40
    # uniformly random residues: centred CRT values up to Q/2 (at most 16 limbs,
    # so that Q/2 / scale stays inside the double range)
    qr = q[:min(limbs, 16)]
    polys = np.stack([np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in qr]) for _ in range(2)])
    got = cb.decode(ctx, cb.as_u64_tensor(polys), scale).cpu().numpy()
    for i in range(2):
        want = oracle.decode(qr, polys[i], scale)
        assert np.all(np.isfinite(want))
        assert np.array_equal(got[i].view(np.float64), want.view(np.float64)), i
    # an encoded message decodes bit-exactly too, and close to the message
    msg = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    pt = cb.encode(ctx, msg[None], limbs, scale)
    dec = cb.decode(ctx, pt, scale).cpu().numpy()[0]
    assert np.array_equal(dec.view(np.float64), oracle.decode(q, host(pt)[0], scale).view(np.float64))
    assert np.max(np.abs(dec - msg)) < 2.0 ** -30


def test_embed_errors(oracle, cuda):
    n = 1 << 10
    q = [int(x) for x in oracle.primes_below_bits(50, n, 2)]
    ctx = cb.Context(10, q)
    import torch
    s = torch.zeros((1, n // 2), dtype=torch.complex128, device="cuda")
    with pytest.raises(cb.CkksError):
        cb.encode(ctx, s, 3, 2.0 ** 40)  # more limbs than the context has
    with pytest.raises(cb.CkksError):
        cb.encode(ctx, s, 2, -1.0)
