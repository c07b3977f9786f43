"""Regenerates the golden fixtures of tests/test_oracle_golden.py.

Runs only where the reference checkout is present (its Python oracles are
imported from there); the GPU box and the tests read the committed JSON.

Usage: python tests/golden/make_golden.py <reference checkout>
(or set CCMM_REFERENCE to the checkout's root).
Sources:
  security/p6a/generate_candidates.py  -- the reference's prime search
  tools/ckks_embedding_oracle.py       -- O(N^2) canonical embedding
  tools/grafting_spec_oracle.py        -- centred rescale semantics
  src/ring/ntt_parameter_sets.rs        -- psi constants (read as text)
  src/ckks/parameters.rs                -- prime pools (read as text)
"""
import importlib.util
import json
import os
import random
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CCMM_REFERENCE")
HERE = os.path.dirname(os.path.abspath(__file__))
if not REF or not os.path.isdir(REF):
    sys.exit("usage: make_golden.py <reference checkout>  (or CCMM_REFERENCE=<checkout>)")


def load(path, name):
    spec = importlib.util.spec_from_file_location(name, os.path.join(REF, path))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    gen = load("security/p6a/generate_candidates.py", "ref_generate_candidates")
    emb = load("tools/ckks_embedding_oracle.py", "ref_embedding_oracle")
    spec = load("tools/grafting_spec_oracle.py", "ref_grafting_spec_oracle")
    out = {}
    out["primes"] = {
        "%d_%d_%d" % (b, n, c): gen.primes_below_bits(b, n, c)
        for (b, n, c) in [(50, 65536, 32), (60, 65536, 3), (50, 32768, 14), (60, 32768, 2), (60, 4096, 2),
                          (40, 4096, 2), (55, 65536, 4)]
    }
    src = open(os.path.join(REF, "src/ring/ntt_parameter_sets.rs")).read()
    consts = dict(re.findall(r"pub const (NTT(?:32|64)_(?:MODULUS|PSI)): u\d+ = ([0-9_]+);", src))
    out["psi"] = [
        {"q": int(consts["NTT32_MODULUS"].replace("_", "")), "n": 4096, "psi": int(consts["NTT32_PSI"].replace("_", ""))},
        {"q": int(consts["NTT64_MODULUS"].replace("_", "")), "n": 4096, "psi": int(consts["NTT64_PSI"].replace("_", ""))},
    ]
    par = open(os.path.join(REF, "src/ckks/parameters.rs")).read()
    block = par[par.index("const RESEARCH_32768_DEPTH_MODULUS_POOL"):]
    block = block[:block.index("];")]
    out["pool_32768"] = [int(x, 16) for x in re.findall(r"0x([0-9a-f]+)", block)]
    emb_cases = []
    for degree in (8, 16, 32):
        rng = random.Random(1000 + degree)
        slots = [complex(rng.uniform(-1, 1), rng.uniform(-1, 1)) for _ in range(degree // 2)]
        coeffs = emb.slots_to_coefficients(slots)
        back = emb.coefficients_to_slots(coeffs)
        emb_cases.append({"degree": degree, "slots": [[z.real, z.imag] for z in slots], "coefficients": coeffs,
                          "slots_back": [[z.real, z.imag] for z in back]})
    out["embedding"] = emb_cases
    q0, q1, q2 = 12_289, 40_961, 65_537
    Q0, Q1 = q0 * q1 * q2, q0 * q1
    vals = [0, 1, q2 // 2, q2 // 2 + 1, q2 - 1, Q0 - 1] + [random.Random(7).randrange(Q0) for _ in range(8)]
    out["rescale"] = {"moduli": [q0, q1, q2], "values": vals,
                      "rescaled": [spec.ckks_rescale(v, Q0, q2, Q1) for v in vals]}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
