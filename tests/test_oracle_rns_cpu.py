"""CPU checks of the oracle's ordinary RNS key switch without auxiliary limbs
(rns_galois_key.rs:439-469, rns_key_switch.rs:2438-2524 and 1842-1905): a
rotation with the block Galois key decrypts to the rotated slots, and
relinearizing a tensor with the block relinearization key decrypts to the
slot-wise product (decoded relative error below 1e-3, inside the reference's
1e-2 bound of tests/r30_9a_13_hybrid_65536.rs).

Without auxiliary limbs the switch adds sum_i d_i e_i with block digits d_i
below Q_i, about Q_i sigma sqrt(N) in size, so the scale must sit well above
it: 30-bit limbs here, scales 2^60 (singleton blocks) and 2^90 (two-limb
blocks) for rotations, 2^55 per factor for products."""
import numpy as np
import pytest


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def setup(oracle):
    n = 1 << 10
    q = [int(x) for x in oracle.primes_below_bits(30, n, 4)]
    rng = np.random.default_rng(3)
    s = rng.integers(-1, 2, n).astype(np.int8)
    return n, q, s, rng


@pytest.mark.parametrize("blocks", [[1, 1, 1, 1], [2, 2], [1, 1, 2]])
def test_rns_rotation_decrypts_to_rotated_slots(oracle, setup, blocks):
    n, q, s, rng = setup
    scale = 2.0 ** (60 if max(blocks) == 1 else 90)
    slots = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ct = oracle.encrypt(q, s, oracle.encode(slots, q, scale), seed=11)
    for steps in (1, 5):
        k = int(oracle.L.oracle_rotation_exponent_left(n, steps))
        key = oracle.rns_key(q, blocks, s, k, seed=21 + steps)
        out = oracle.rns_rotate(q, blocks, key, k, ct)
        dec = oracle.decode(q, oracle.decrypt(q, s, out), scale)
        assert rel_l2(dec, np.roll(slots, -steps)) < 1e-3


@pytest.mark.parametrize("blocks", [[1, 1, 1, 1], [2, 2]])
def test_rns_relinearization_decrypts_to_product(oracle, setup, blocks):
    n, q, s, rng = setup
    scale = 2.0 ** 55
    x = rng.uniform(-1, 1, n // 2) + 0j
    y = rng.uniform(-1, 1, n // 2) + 0j
    cx = oracle.encrypt(q, s, oracle.encode(x, q, scale), seed=31)
    cy = oracle.encrypt(q, s, oracle.encode(y, q, scale), seed=32)
    quad = oracle.tensor(q, cx, cy)
    key = oracle.rns_relin_key(q, blocks, s, seed=41)
    out = oracle.rns_relinearize(q, blocks, quad, key)
    dec = oracle.decode(q, oracle.decrypt(q, s, out), scale * scale)
    assert rel_l2(dec, x * y) < 1e-3
