"""The arithmetic of the tensor-core Park Mod-PP-MM (csrc/park.cu), restated
on the CPU and checked against the oracle's Reference backend
(ccmm/park.rs:1405-1620).

The device kernel sums, per output, P_j = sum_(k,i) a_i[k] w_ij[k] of unsigned
8-bit products in 32 bits and returns sum_j 2^(8j) P_j mod q, where a_i are the
bytes of lhs mod q and w_ij the bytes of 2^(8i) (rhs mod q) mod q. These tests
pin that identity, the inner-sum length per launch (every P_j below 2^31 in
the worst case, one block more would not be) and the tile widths, with the
same constants the kernel uses.
"""
import numpy as np
import pytest


def nbytes(q):
    return ((q - 1).bit_length() + 7) // 8


def cols_per_tile(nb):  # nb * ct <= 256, a multiple of 16
    c = (256 // nb) // 8 * 8
    return c - 8 if (c * nb) % 16 else c


def blocks_per_launch(nb):  # 32-deep inner blocks per launch
    return (0x7FFFFFFF // (65025 * nb)) // 32


def byte_planes(x, nb):
    return [((x >> np.uint64(8 * i)) & np.uint64(255)).astype(np.int64) for i in range(nb)]


def park_tc_restated(lhs, rhs, q):
    nb = nbytes(q)
    a = lhs % np.uint64(q)
    b = rhs % np.uint64(q)
    a_planes = byte_planes(a, nb)
    # weights W_i = 2^(8i) b mod q, exact in Python integers
    w = [b]
    for _ in range(1, nb):
        w.append(np.array([[(int(v) << 8) % q for v in row] for row in w[-1]], dtype=np.uint64))
    w_planes = [byte_planes(wi, nb) for wi in w]  # w_planes[i][j]
    inner = lhs.shape[1]
    chunk = 32 * blocks_per_launch(nb)
    out = np.zeros((lhs.shape[0], rhs.shape[1]), dtype=object)
    for k0 in range(0, inner, chunk):
        k1 = min(inner, k0 + chunk)
        part = np.zeros_like(out)
        for j in range(nb):
            P = sum(a_planes[i][:, k0:k1] @ w_planes[i][j][k0:k1, :] for i in range(nb))
            assert P.max(initial=0) < 2**31
            part = part + (P.astype(object) << (8 * j))
        out = (out + part % q) % q
    return out.astype(np.uint64)


@pytest.mark.parametrize("q", [2, 17, 257, 65537, 2**31 - 1, 0x7ffff6001, 2**47 - 115, 0xfffffffffffc001,
                               2**64 - 59, 2**64 - 1])
def test_restated_tensor_core_identity_matches_oracle(oracle, q):
    rng = np.random.default_rng(q % 1000)
    lhs = rng.integers(0, 2**64, (9, 37), dtype=np.uint64)  # entries at and above q
    rhs = rng.integers(0, 2**64, (37, 11), dtype=np.uint64)
    assert np.array_equal(park_tc_restated(lhs, rhs, q), oracle.park_mod_pp_mm(lhs, rhs, q))


def test_chunked_inner_sum_matches_oracle(oracle):
    q = 251  # one byte: 33,024 terms per launch
    rng = np.random.default_rng(3)
    lhs = rng.integers(0, q, (2, 33100), dtype=np.uint64)
    rhs = rng.integers(0, q, (33100, 3), dtype=np.uint64)
    assert np.array_equal(park_tc_restated(lhs, rhs, q), oracle.park_mod_pp_mm(lhs, rhs, q))


@pytest.mark.parametrize("nb", range(1, 9))
def test_launch_length_and_tile_width(nb):
    terms = 32 * blocks_per_launch(nb)
    # worst case: every product 255 x 255 over nb byte planes of every inner index
    assert nb * terms * 255 * 255 < 2**31
    assert nb * (terms + 32) * 255 * 255 >= 2**31
    ct = cols_per_tile(nb)
    assert ct % 8 == 0 and (nb * ct) % 16 == 0 and nb * ct <= 256
    assert nb * (ct + 8) > 256 or (nb * (ct + 8)) % 16  # the widest such tile
