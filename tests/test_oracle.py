"""CPU tests: the oracle against the reference's golden vectors, the C++ oracle
against the Python one, and the decoding rules.  No GPU needed."""
import random

import numpy as np
import pytest

import bls_ref as B
import cpu as C
import workload_py as W


def _fp12(golden, key):
    return B.f12_from_mont_limbs([int(x) for x in golden[key]])


# ---------------------------------------------------------------- Python oracle pins

def test_small_montgomery_constants(golden):
    assert B.mont_limbs(1) == list(golden["mont_one"])
    assert B.mont_limbs(6) == list(golden["mont_6"])
    assert B.mont_limbs(-7)[0] == golden["mont_minus7_limb0"][0]
    assert B.mont_limbs(22)[0] == golden["mont_22_limb0"][0]


def test_frobenius_constants(golden):
    assert B.FROB6_C1 == (0, B.from_mont_limbs(golden["frob6_c1"]))
    assert B.FROB6_C2 == (B.from_mont_limbs(golden["frob6_c2"]), 0)
    f = golden["frob12"]
    assert B.FROB12_C1 == (B.from_mont_limbs(f[:6]), B.from_mont_limbs(f[6:]))


def test_generators(golden):
    assert B.g1_from_mont_u64(golden["g1_generator"]) == B.G1_GEN
    assert B.g1_on_curve(B.G1_GEN) and B.g2_on_curve(B.G2_GEN)
    # the reference's hard-coded G2 generator has a wrong y.c0: off the curve
    bad = golden["g2_generator_known_bad"]
    q = ((B.from_mont_limbs(bad[0:6]), B.from_mont_limbs(bad[6:12])),
         (B.from_mont_limbs(bad[12:18]), B.from_mont_limbs(bad[18:24])))
    assert q[0] == B.G2_GEN[0] and not B.g2_on_curve(q)


def test_line_tables(golden):
    assert B.coeffs_to_limbs(B.g2_prepare(B.G2_GEN)) == list(golden["g2_gen_coeffs"])
    assert B.coeffs_to_limbs(B.g2_prepare(B.g2_mul(B.G2_GEN, 42))) == list(golden["pk42_coeffs"])


def test_miller_and_pairing(golden):
    co = B.coeffs_from_limbs(golden["g2_gen_coeffs"])
    ml = B.multi_miller_loop([(B.G1_GEN, co, False)])
    assert B.f12_mont_limbs(ml) == list(golden["ml_g1_g2"])
    gt = B.final_exponentiation(ml)
    assert B.f12_mont_limbs(gt) == list(golden["pairing_g1_g2"])
    cs = B.f12_cyclotomic_square(gt)
    assert B.f12_mont_limbs(cs)[:6] == list(golden["cycsq_pairing_c000"])
    # on the cyclotomic subgroup the Granger-Scott square is the square
    assert cs == B.f12_mul(gt, gt)


def test_verify_kat(golden):
    """sk = 42, H(m) = 7 G1, sig = 294 G1 (gpu-crypto/src/lib.rs:198-221) and the
    G1-generator forgery (lib.rs:224-242)."""
    sig = B.g1_from_mont_u64(golden["sig_294_g1"])
    nhm = B.g1_from_mont_u64(golden["neg_hm_7_g1"])
    assert sig == B.g1_mul(B.G1_GEN, 294) and nhm == B.g1_neg(B.g1_mul(B.G1_GEN, 7))
    co = B.coeffs_from_limbs(golden["g2_gen_coeffs"])
    pk = B.coeffs_from_limbs(golden["pk42_coeffs"])
    ok, ml, gt = B.verify(sig, nhm, co, pk)
    assert ok and B.f12_mont_limbs(ml)[:6] == list(golden["ml_2pair_c000"])
    assert B.f12_is_one(gt)
    assert not B.verify(B.G1_GEN, nhm, co, pk)[0]


def test_identity_pairs_are_skipped(golden):
    co = B.coeffs_from_limbs(golden["g2_gen_coeffs"])
    pk = B.coeffs_from_limbs(golden["pk42_coeffs"])
    # sig = identity, -H = identity: both pairs skipped, Miller value 1
    ok, ml, gt = B.verify(None, None, co, pk)
    assert ok and ml == B.F12_ONE
    # sig = identity only: e(-H, pk) != 1 for a real H
    assert not B.verify(None, B.g1_neg(B.G1_GEN), co, pk)[0]


# ---------------------------------------------------------------- C++ oracle pins

def test_cpp_line_tables(golden):
    q = np.array(W.g2_affine_u64(B.G2_GEN), dtype=np.uint64)
    assert (C.g2_prepare(q) == golden["g2_gen_coeffs"]).all()
    q42 = np.array(W.g2_affine_u64(B.g2_mul(B.G2_GEN, 42)), dtype=np.uint64)
    assert (C.g2_prepare(q42) == golden["pk42_coeffs"]).all()


def test_cpp_final_exp_and_cycsq(golden):
    assert (C.final_exp(golden["ml_g1_g2"]) == golden["pairing_g1_g2"]).all()
    assert (C.cyclotomic_square(golden["pairing_g1_g2"])[:6] == golden["cycsq_pairing_c000"]).all()


def test_cpp_verify_kat(golden):
    sig = golden["sig_294_g1"][None]
    nhm = golden["neg_hm_7_g1"][None]
    res, ml, gt = C.verify_batch(sig, nhm, golden["g2_gen_coeffs"], golden["pk42_coeffs"][None], want_values=True)
    assert res[0] == 1
    assert (ml[0, :6] == golden["ml_2pair_c000"]).all()
    assert C.verify_batch(golden["g1_generator"][None], nhm, golden["g2_gen_coeffs"], golden["pk42_coeffs"][None])[0] == 0
    # identity -H(m) (x = 0, y = R): the pair drops out, leaving e(G1, G2)
    ident = np.array([0] * 6 + B.mont_limbs(1), dtype=np.uint64)[None]
    res, ml, gt = C.verify_batch(golden["g1_generator"][None], ident, golden["g2_gen_coeffs"],
                                 golden["pk42_coeffs"][None], want_values=True)
    assert (ml[0] == golden["ml_g1_g2"]).all() and (gt[0] == golden["pairing_g1_g2"]).all()


def test_cpp_matches_python_random_batch():
    wl = W.plain_config(n=8, seed=7)
    g2 = np.array(B.coeffs_to_limbs(B.g2_prepare(B.G2_GEN)), dtype=np.uint64)
    res, ml, gt = C.verify_batch(wl["sigs"], wl["nhms"], g2, wl["pk_tabs"], want_values=True, nthreads=4)
    assert (res == wl["expect"]).all()
    co = B.coeffs_from_limbs([int(x) for x in g2])
    for i in (0, 7):
        ok, mlp, gtp = B.verify(B.g1_from_mont_u64(wl["sigs"][i]), B.g1_from_mont_u64(wl["nhms"][i]), co,
                                B.coeffs_from_limbs([int(x) for x in wl["pk_tabs"][i]]))
        assert ok == bool(res[i])
        assert B.f12_mont_limbs(mlp) == list(ml[i]) and B.f12_mont_limbs(gtp) == list(gt[i])


def test_cpp_garbage_points_match_python():
    """Points off the curve still define a Miller value and a final exponentiation
    (through the same formulas); both oracles must agree on them too."""
    rng = random.Random(3)
    g2 = np.array(B.coeffs_to_limbs(B.g2_prepare(B.G2_GEN)), dtype=np.uint64)
    s = [rng.randrange(1, B.P), rng.randrange(1, B.P)]
    h = [rng.randrange(1, B.P), rng.randrange(1, B.P)]
    sig = np.array(B.mont_limbs(s[0]) + B.mont_limbs(s[1]), dtype=np.uint64)[None]
    nhm = np.array(B.mont_limbs(h[0]) + B.mont_limbs(h[1]), dtype=np.uint64)[None]
    res, ml, gt = C.verify_batch(sig, nhm, g2, g2[None], want_values=True)
    co = B.coeffs_from_limbs([int(x) for x in g2])
    ok, mlp, gtp = B.verify((s[0], s[1]), (h[0], h[1]), co, co)
    assert B.f12_mont_limbs(mlp) == list(ml[0]) and B.f12_mont_limbs(gtp) == list(gt[0])


# ---------------------------------------------------------------- decoding

def test_decompress_valid_and_identity():
    rng = random.Random(11)
    pts = [B.g1_mul(B.G1_GEN, rng.randrange(1, B.R_ORDER)) for _ in range(12)] + [None, B.G1_GEN]
    comp = b"".join(B.g1_compress(p) for p in pts)
    for p, c in zip(pts, [comp[48 * i:48 * i + 48] for i in range(len(pts))]):
        assert B.g1_decompress(c) == (B.ST_OK, p)
    st, xy = C.g1_decompress(np.frombuffer(comp, dtype=np.uint8))
    assert (st == 0).all()
    for i, p in enumerate(pts):
        assert list(xy[i]) == B.g1_to_mont_u64(p)


def test_decompress_invalid_reasons():
    rng = W.SplitMix64(99)
    cases = W.invalid_encodings(rng, B.g1_mul(B.G1_GEN, 5))
    for b, want in cases:
        assert B.g1_decompress(b)[0] == want
    st, _ = C.g1_decompress(np.frombuffer(b"".join(b for b, _ in cases), dtype=np.uint8))
    assert list(st) == [w for _, w in cases]


def test_compressed_verify_statuses():
    wl = W.plain_config(n=4, seed=5)
    g2 = np.array(B.coeffs_to_limbs(B.g2_prepare(B.G2_GEN)), dtype=np.uint64)
    comp = [B.g1_compress(p) for p in wl["sig_points"]]
    bad = W.invalid_encodings(W.SplitMix64(1), wl["sig_points"][0])
    comp[1] = bad[0][0]
    comp[2] = bad[-1][0]
    res = C.verify_compressed_batch(np.frombuffer(b"".join(comp), dtype=np.uint8), wl["nhms"], g2, wl["pk_tabs"])
    assert list(res) == [1, -B.ST_BAD_FLAGS, -B.ST_NOT_IN_SUBGROUP, wl["expect"][3]]


# ---------------------------------------------------------------- hash to G1

def test_expand_message_xmd_shape_and_determinism():
    a = B.expand_message_xmd(b"abc", W.DST, 128)
    assert len(a) == 128 and a == B.expand_message_xmd(b"abc", W.DST, 128)
    assert a != B.expand_message_xmd(b"abd", W.DST, 128)
    assert B.expand_message_xmd(b"abc", W.DST, 32) != a[:32]


def test_sswu_curve_z_and_map():
    """E' is isogenous to E (its points have orders dividing #E(Fp) = h r), Z
    is the RFC's search result, and the map lands on E' with sgn0(y) = sgn0(u)"""
    assert B.N_G1_CURVE == 0x396c8c005555e1568c00aaab0000aaab * B.R_ORDER
    x = 5
    while not B.fp_is_square(B._g_iso(x)):
        x += 1
    assert B._iso_mul((x, B.fp_sqrt(B._g_iso(x))), B.N_G1_CURVE) is None
    assert B.SSWU_Z == 11
    for u in (0, 1, 2, 12345, B.P - 1):
        x, y = B.map_to_curve_sswu(u)
        assert (y * y - B._g_iso(x)) % B.P == 0 and (y & 1) == (u & 1)


def test_isogeny_lands_on_e_and_adds():
    pts = [B.map_to_curve_sswu(u) for u in (3, 77, 2**300 + 5)]
    imgs = [B.iso_map(q) for q in pts]
    assert all(q is not None and B.g1_on_curve(q) for q in imgs)
    assert B.iso_map(B._iso_add(pts[0], pts[1])) == B.g1_add(imgs[0], imgs[1])
    assert B.iso_map(B._iso_mul(pts[2], 11)) == B.g1_mul(imgs[2], 11)
    assert B.iso_map(B._ISO_KERNEL[0]) is None          # the kernel maps to the identity


def test_hash_to_g1_in_subgroup():
    for m in (b"", b"abc", bytes(range(32))):
        h = B.hash_to_g1(m, W.DST)
        assert B.g1_on_curve(h) and B.g1_in_subgroup(h)
    assert B.hash_to_g1(b"abc", W.DST) != B.hash_to_g1(b"abd", W.DST)


# ---------------------------------------------------------------- workload generator vs oracle

def test_generator_sha256_and_xmd():
    import hashlib
    import workload as WL
    L = WL.wl()
    for m in (b"", b"abc", bytes(range(200))):
        o = np.zeros(32, np.uint8)
        a = np.frombuffer(m, np.uint8) if m else np.zeros(1, np.uint8)
        L.wl_sha256(a.ctypes.data, len(m), o.ctypes.data)
        assert bytes(o) == hashlib.sha256(m).digest()
    o = np.zeros(128, np.uint8)
    m = np.frombuffer(b"abc", np.uint8)
    d = np.frombuffer(W.DST, np.uint8)
    L.wl_expand_message_xmd(m.ctypes.data, 3, d.ctypes.data, len(W.DST), o.ctypes.data, 128)
    assert bytes(o) == B.expand_message_xmd(b"abc", W.DST, 128)


def test_generator_hash_sign_keys_match_oracle():
    import workload as WL
    msgs = [bytes([i]) * 32 for i in range(4)]
    h = WL.hash_to_g1(msgs)
    for i, m in enumerate(msgs):
        assert list(h[i]) == B.g1_to_mont_u64(B.hash_to_g1(m, W.DST))
    k = [5, 2**200 + 17]
    sc = np.array([WL.scalar_limbs(x) for x in k], dtype=np.uint64)
    s = WL.g1_mul(h[:2], sc)
    for i in range(2):
        assert list(s[i]) == B.g1_to_mont_u64(B.g1_mul(B.hash_to_g1(msgs[i], W.DST), k[i]))
    pk = WL.g2_mul_gen(sc)
    for i in range(2):
        q = B.g2_mul(B.G2_GEN, k[i])
        assert list(pk[i]) == W.g2_affine_u64(q)
        assert bytes(WL.g2_compress(pk[i:i + 1])[0]) == B.g2_compress(q)
        assert B.g2_decompress(B.g2_compress(q)) == (B.ST_OK, q)
        assert list(WL.g2_prepare(pk[i:i + 1])[0]) == B.coeffs_to_limbs(B.g2_prepare(q))
    comp = WL.g1_compress(s)
    for i in range(2):
        assert bytes(comp[i]) == B.g1_compress(B.g1_from_mont_u64(s[i]))


def test_generator_configs_verify_as_expected():
    import workload as WL
    g2 = np.array(B.coeffs_to_limbs(B.g2_prepare(B.G2_GEN)), dtype=np.uint64)
    c = WL.config_keyset(256, 40, seed=2)
    r = C.verify_batch(c["sigs"], c["nhms"], g2, c["pk_tables"], pk_index=c["pk_index"], nthreads=8)
    assert (r == c["expect"]).all() and (r == 0).sum() == 32
    cc = WL.config_compressed(512, 40, seed=3, invalid_frac=0.05)
    r = C.verify_compressed_batch(cc["sigs_compressed"].reshape(-1), cc["nhms"], g2, cc["pk_tables"],
                                  pk_index=cc["pk_index"], nthreads=8)
    assert (r == cc["expect"]).all()
    assert set(np.unique(r[r < 0])) == {-1, -2, -3, -4}
