"""CPU tests: the oracle pinned to the reference's own constants and Python
oracles (tests/golden/golden.json, made by tests/golden/make_golden.py), to
exact big-integer definitions, and the product's host-side parameter search.
No GPU needed."""
import json
import os

import numpy as np
import pytest

import ckks_b200 as cb
import ckks_b200.params as params

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def test_prime_search_matches_reference_generator(oracle):
    # security/p6a/generate_candidates.py:53-73 (the reference's own search)
    for key, want in GOLDEN["primes"].items():
        bits, n, count = map(int, key.split("_"))
        assert [int(x) for x in oracle.primes_below_bits(bits, n, count)] == want, key
        assert params.primes_below_bits(bits, n, count) == want, key


def test_prime_pool_of_parameters_rs(oracle):
    # ckks/parameters.rs:345-362: every pooled modulus is an NTT-friendly prime for N=2^15
    for q in GOLDEN["pool_32768"]:
        assert oracle.L.oracle_is_prime(q) == 1 and (q - 1) % (2 * 32768) == 0
        assert params.is_prime(q)
    # the 50-bit search at N=2^15 visits those primes in descending order
    found = GOLDEN["primes"]["50_32768_14"]
    assert all(found[i] > found[i + 1] for i in range(len(found) - 1))
    assert found[0] == GOLDEN["pool_32768"][0]


def test_psi_constants(oracle):
    # ring/ntt_parameter_sets.rs:7-10, smallest-generator rule of ring/ntt_params.rs:16-50
    for case in GOLDEN["psi"]:
        assert oracle.root(case["q"], case["n"]) == case["psi"]
        if case["q"] < (1 << 62):
            assert params.negacyclic_root(case["q"], case["n"]) == case["psi"]
    # roots of the reference's prime search (same smallest-generator rule): the 60-bit
    # prime of the N=2^12 chain and the first 50-bit prime for N=2^16
    assert oracle.root(0xfffffffffffc001, 4096) == 431606828070683274
    assert oracle.root(0x3ffffffd20001, 65536) == 1077102403560341
    assert params.negacyclic_root(0x3ffffffd20001, 65536) == 1077102403560341


@pytest.mark.parametrize("q,n", [(97, 8), (12289, 16), (12289, 256), (40961, 512), (0x3ffffffd20001, 64)])
def test_ntt_matches_definition(oracle, q, n):
    # radix-2 prepared NTT vs the O(N^2) definition (ring/ntt_params.rs:87-141)
    rng = np.random.default_rng(q + n)
    a = rng.integers(0, q, n, dtype=np.uint64)
    A = oracle.ntt_forward([q], a.reshape(1, n))[0]
    assert np.array_equal(A, oracle.ntt_forward_reference(q, a))
    psi = oracle.root(q, n)
    for k in (0, 1, n - 1):
        assert int(A[k]) == sum(int(a[j]) * pow(psi, (2 * k + 1) * j, q) for j in range(n)) % q
    assert np.array_equal(oracle.ntt_inverse([q], A.reshape(1, n))[0], a)


def test_shoup_and_barrett_edges(oracle):
    # ring/modulus.rs:331-456: Shoup and Barrett vs u128 % on edge operands
    for q in [268_238_849, 68_712_923_137, 0x3ffffffd20001, 0xfffffffffffc001]:
        vals = [0, 1, 2, q // 2, q - 2, q - 1]
        for a in vals:
            wq = oracle.L.oracle_shoup_quotient(a, q)
            for b in vals:
                assert oracle.L.oracle_shoup_mul(b, a, wq, q) == (a * b) % q
                assert oracle.L.oracle_barrett_mul(a, b, q) == (a * b) % q


def centred(x, m):
    x %= m
    return x - m if x > m // 2 else x


def test_crt_decompose_moddown_rescale_vs_bigint(oracle):
    rng = np.random.default_rng(3)
    n = 64
    q = [int(x) for x in oracle.primes_below_bits(50, 1024, 4)]
    p = [int(x) for x in oracle.primes_below_bits(60, 1024, 2)]
    Q = int(np.prod([1] + q, dtype=object))
    P = p[0] * p[1]
    x = np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q])
    vals = oracle.crt(q, x)
    assert all(v < Q and all(v % m == int(x[i][c]) for i, m in enumerate(q)) for c, v in enumerate(vals))
    for base_log in (8, 20, 32):
        d = oracle.bounded_decompose(q, x, base_log)
        B = 1 << base_log
        assert d.shape[0] == -(-(Q.bit_length() + 1) // base_log)
        for c in range(n):
            v, ds = centred(vals[c], Q), []
            for _ in range(d.shape[0]):
                r = v % B
                dig = r - B if r >= B // 2 else r
                ds.append(dig)
                v = (v - dig) // B
            assert v == 0 and ds == [int(t) for t in d[:, c]]
    # ModDown (auxiliary_modulus.rs:48-81 reference: round(centred(x)/P) mod Q)
    y = np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q + p])
    md = oracle.mod_down(q, p, y)
    full = oracle.crt(q + p, y)
    for c in range(n):
        xc = centred(full[c], Q * P)
        rounded = (abs(xc) + P // 2) // P * (1 if xc >= 0 else -1)
        assert [int(md[i][c]) for i in range(len(q))] == [rounded % m for m in q]
    # rescale (rns_rescale.rs:107-167) == round(centred / q_L) on the remaining basis
    rs = oracle.rescale(q, x)
    for c in range(n):
        xc = centred(vals[c], Q)
        ql = q[-1]
        r = (abs(xc) + ql // 2) // ql * (1 if xc >= 0 else -1)
        assert [int(rs[i][c]) for i in range(3)] == [r % m for m in q[:3]]


def test_rescale_matches_grafting_spec_oracle(oracle):
    # tools/grafting_spec_oracle.py ckks_rescale on the toy chain 12289, 40961, 65537
    g = GOLDEN["rescale"]
    q = g["moduli"]
    x = np.array([[v % m for v in g["values"]] for m in q], np.uint64)
    out = oracle.rescale(q, x)
    got = oracle.crt(q[:2], out)
    assert got == g["rescaled"]


def test_embedding_matches_reference_oracle(oracle):
    # ckks/embedding.rs FFT form vs tools/ckks_embedding_oracle.py O(N^2) form
    for case in GOLDEN["embedding"]:
        slots = np.array([complex(a, b) for a, b in case["slots"]])
        co = oracle.slots_to_coefficients(slots)
        assert np.max(np.abs(co - np.array(case["coefficients"]))) < 1e-12
        back = oracle.coefficients_to_slots(np.array(case["coefficients"]))
        want = np.array([complex(a, b) for a, b in case["slots_back"]])
        assert np.max(np.abs(back - want)) < 1e-12


def test_hoisted_digits_equal_redecomposition(oracle):
    # grafting/bounded_gadget.rs:446-500
    rng = np.random.default_rng(5)
    n = 256
    q = [int(x) for x in oracle.primes_below_bits(40, n, 3)]
    x = np.stack([rng.integers(0, m, n, dtype=np.uint64) for m in q])
    for base_log in (4, 16):
        d = oracle.bounded_decompose(q, x, base_log)
        for k in (3, 5, 2 * n - 1):
            assert np.array_equal(oracle.bounded_automorphism_hoisted(d, base_log, k),
                                  oracle.bounded_decompose(q, oracle.automorphism_coef(q, x, k), base_log))


def test_rotation_decodes_to_rotated_slots(oracle):
    # decoded error of a hybrid-QP rotation (tests/r30_9a_13_hybrid_65536.rs:256-262 bound 0.01)
    rng = np.random.default_rng(9)
    n = 256
    q = [int(x) for x in oracle.primes_below_bits(50, n, 3)]
    p = [int(x) for x in oracle.primes_below_bits(60, n, 1)]
    s = rng.integers(-1, 2, n).astype(np.int8)
    slots = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ct = oracle.encrypt(q, s, oracle.encode(slots, q, 2.0 ** 40), seed=3)
    k = int(oracle.L.oracle_rotation_exponent_left(n, 3))
    key = oracle.hybrid_key(q, p, s, k, 20, seed=4)
    out = oracle.hybrid_rotate(q, p, key, k, 20, ct)
    dec = oracle.decode(q, oracle.decrypt(q, s, out), 2.0 ** 40)
    assert np.linalg.norm(dec - np.roll(slots, -3)) / np.linalg.norm(slots) < 1e-6


def test_multiply_chain_decodes(oracle):
    # HMult -> bounded relinearize (base 2^20) -> rescale -> rotate by 1 on the
    # N=2^12 chain q = 60 + 40 + 40 bits, P = 60 bits (ckks/rns_multiply.rs:262-300)
    q = [0xfffffffffffc001, 0xfffffdc001, 0xfffffc6001]
    p = [0xffffffffffe8001]
    n = 4096
    assert all(params.is_prime(m) and (m - 1) % (2 * n) == 0 for m in q + p)
    rng = np.random.default_rng(12)
    s = rng.integers(-1, 2, n).astype(np.int8)
    scale = 2.0 ** 40
    a = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    b = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    cx = oracle.encrypt(q, s, oracle.encode(a, q, scale), seed=1)
    cy = oracle.encrypt(q, s, oracle.encode(b, q, scale), seed=2)
    rel = oracle.relinearize(q, oracle.tensor(q, cx, cy), oracle.relin_key(q, s, 20, seed=3), 20)
    resc = oracle.rescale(q, rel.reshape(2, 3, n))
    k = int(oracle.L.oracle_rotation_exponent_left(n, 1))
    rot = oracle.hybrid_rotate(q[:2], p, oracle.hybrid_key(q[:2], p, s, k, 20, seed=4), k, 20, resc)
    dec = oracle.decode(q[:2], oracle.decrypt(q[:2], s, rot), scale * scale / q[-1])
    err = np.linalg.norm(dec - np.roll(a * b, -1)) / np.linalg.norm(a * b)
    assert err < 1e-4, err
