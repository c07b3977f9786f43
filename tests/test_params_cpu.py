"""The named parameter sets reproduce the reference's prime chains (host-side
search through the library's C ABI; no GPU call): C1's [60, 40, 40] + P60 at
N=2^12, the 24 x 50-bit + 3 x 60-bit chain at N=2^16 and the 14 x 50-bit +
2 x 60-bit chain at N=2^15 (ckks/parameters.rs:345-362 for the last)."""
import ckks_b200.params as params


def test_multiply_chain():
    q, p = params.config("multiply").moduli()
    assert q == [0xfffffffffffc001, 0xfffffdc001, 0xfffffc6001]
    assert p == [0xffffffffffe8001]


def test_rotation_and_ccmm_chains():
    q, p = params.config("rotation").moduli()
    assert len(q) == 24 and q[0] == 0x3ffffffd20001 and q[-1] == 0x3fffffc3c0001
    assert p == [0xffffffffffc0001, 0xfffffffff840001, 0xfffffffff6a0001]
    assert params.config("fft2").moduli() == (q, p)
    qc, pc = params.config("ccmm").moduli()
    assert len(qc) == 14 and qc[0] == 0x3ffffffdf0001 and qc[-1] == 0x3fffffea60001
    assert pc == [0xffffffffffc0001, 0xfffffffff840001]
    for m in q + p + qc + pc:
        assert params.is_prime(m)
    assert params.negacyclic_root(q[0], 1 << 16) == 1077102403560341


def test_ntt_chain_extends_rotation_pool():
    q, p = params.config("ntt").moduli()
    assert len(q) == 32 and not p
    assert q[:24] == params.config("rotation").moduli()[0]
