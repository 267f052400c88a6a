"""Extract the reference's golden vectors (hard-coded Montgomery limbs) into
tests/golden/reference_vectors.json.

The reference pins its GPU pairing code with limbs copied from runs of its
Rust oracle (ic_bls12_381 0.10.1) and pasted into standalone CUDA test mains.
This script reads those files as text, by file and line range, and stores the
64-bit little-endian Montgomery limbs (R = 2^384) as hex strings.  It is run
once in a container that has the reference checked out; the JSON it writes is
the committed fixture, so nothing at test time needs the reference.

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT (the reference's checkout)")
REF = sys.argv[1]
HEX_C = re.compile(r"0x([0-9a-fA-F]+)(?:ULL|ull)?")


def lines(path, lo, hi):
    with open(os.path.join(REF, path)) as f:
        all_lines = f.read().split("\n")
    return "\n".join(all_lines[lo - 1:hi])


def c_hex(path, lo, hi, strip_comments=True):
    """All 0x... literals in lines lo..hi (1-based, inclusive)."""
    text = lines(path, lo, hi)
    if strip_comments:
        text = re.sub(r"//[^\n]*", "", text)
    return ["%016x" % int(h, 16) for h in HEX_C.findall(text)]


def bracket_hex(path, line_no):
    """Comma-separated bare hex words inside [...] on one line."""
    text = lines(path, line_no, line_no)
    inner = text[text.index("[") + 1:text.index("]")]
    return ["%016x" % int(w.strip(), 16) for w in inner.split(",")]


def main():
    out = {"source": "Menese-Protocol/ICP-GPU test sources (limbs: u64 LE, Montgomery R=2^384)"}

    out["g2_gen_coeffs"] = {"cite": "cuda/g2_coeffs.h:4-549",
                            "limbs": c_hex("cuda/g2_coeffs.h", 4, 549)}
    out["pk42_coeffs"] = {"cite": "cuda/pk42_coeffs.h:2-411",
                          "limbs": c_hex("cuda/pk42_coeffs.h", 2, 411)}
    assert len(out["g2_gen_coeffs"]["limbs"]) == 2448
    assert len(out["pk42_coeffs"]["limbs"]) == 2448

    out["g1_generator"] = {"cite": "cuda/test_full_pairing.cu:402-407",
                           "limbs": c_hex("cuda/test_full_pairing.cu", 402, 407)}
    # Known bad: y.c0 (lines 297-299) is not the generator's; the point is off
    # the curve.  The generator is pinned instead by the full G2_COEFFS table.
    out["g2_generator_known_bad"] = {"cite": "cuda/test_miller_v2.cu:291-302",
                                     "limbs": c_hex("cuda/test_miller_v2.cu", 291, 302),
                                     "order": "x.c0, x.c1, y.c0, y.c1",
                                     "note": "y.c0 is wrong in the reference source; not on the curve"}
    out["sig_294_g1"] = {"cite": "cuda/test_bls_verify.cu:115-120",
                         "limbs": c_hex("cuda/test_bls_verify.cu", 115, 120)}
    out["neg_hm_7_g1"] = {"cite": "cuda/test_bls_verify.cu:124-129",
                          "limbs": c_hex("cuda/test_bls_verify.cu", 124, 129)}
    out["ml_2pair_c000"] = {"cite": "cuda/test_bls_verify.cu:147",
                            "what": "multi_miller_loop[(294*G1, G2), (-7*G1, 42*G2)] c0.c0.c0",
                            "limbs": bracket_hex("cuda/test_bls_verify.cu", 147)}
    out["ml_g1_g2"] = {"cite": "cuda/test_final_exp.cu:288-300",
                       "what": "miller_loop(G1, G2), all 12 Fp in tower order",
                       "limbs": c_hex("cuda/test_final_exp.cu", 289, 300)}
    out["pairing_g1_g2"] = {"cite": "lib/test_cyc_sq.cu:141-153",
                            "what": "final_exponentiation(miller_loop(G1, G2))",
                            "limbs": c_hex("lib/test_cyc_sq.cu", 142, 153)}
    out["cycsq_pairing_c000"] = {"cite": "lib/test_cyc_sq.cu:175-176",
                                 "what": "cyclotomic_square(e(G1,G2)).c0.c0.c0",
                                 "limbs": c_hex("lib/test_cyc_sq.cu", 175, 176)}
    out["frob6_c1"] = {"cite": "gpu-crypto/cuda/field_sppark.cuh:117",
                       "what": "Fp6 Frobenius coefficient for c1 (Fp2 = (0, this))",
                       "limbs": c_hex("gpu-crypto/cuda/field_sppark.cuh", 117, 117)}
    out["frob6_c2"] = {"cite": "gpu-crypto/cuda/field_sppark.cuh:119",
                       "what": "Fp6 Frobenius coefficient for c2 (Fp2 = (this, 0))",
                       "limbs": c_hex("gpu-crypto/cuda/field_sppark.cuh", 119, 119)}
    out["frob12"] = {"cite": "gpu-crypto/cuda/field_sppark.cuh:162-163",
                     "what": "Fp12 Frobenius coefficient (c0 limbs then c1 limbs)",
                     "limbs": c_hex("gpu-crypto/cuda/field_sppark.cuh", 162, 163)}
    out["mont_one"] = {"cite": "gpu-crypto/cuda/api.cu:85-86",
                       "limbs": c_hex("gpu-crypto/cuda/api.cu", 85, 86)}
    out["mont_6"] = {"cite": "lib/test_sppark_fp.cu:72-73",
                     "limbs": c_hex("lib/test_sppark_fp.cu", 72, 73)}
    out["mont_minus7_limb0"] = {"cite": "lib/test_sppark_fp2.cu:67",
                                "limbs": c_hex("lib/test_sppark_fp2.cu", 67, 67)}
    out["mont_22_limb0"] = {"cite": "lib/test_sppark_fp2.cu:69",
                            "limbs": c_hex("lib/test_sppark_fp2.cu", 69, 69)}

    sizes = {"g1_generator": 12, "g2_generator_known_bad": 24, "sig_294_g1": 12, "neg_hm_7_g1": 12,
             "ml_2pair_c000": 6, "ml_g1_g2": 72, "pairing_g1_g2": 72, "cycsq_pairing_c000": 6,
             "frob6_c1": 6, "frob6_c2": 6, "frob12": 12, "mont_one": 6, "mont_6": 6,
             "mont_minus7_limb0": 1, "mont_22_limb0": 1}
    for k, n in sizes.items():
        assert len(out[k]["limbs"]) == n, (k, len(out[k]["limbs"]))

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main()
