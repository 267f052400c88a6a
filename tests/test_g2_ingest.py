"""On-device public-key ingest: 96-byte compressed G2 keys decoded, validated,
prepared and normalised on the GPU (bls_g2_decompress_status,
bls_pk_register_compressed).  The reference's callers do this on the CPU per
item (G2Affine::from_compressed + G2Prepared::from,
ic-integration/patches/ic-gpu-consensus.patch:458-461); the tables are pinned
by the reference's cuda/g2_coeffs.h and cuda/pk42_coeffs.h, the decode statuses
by the oracle's from_compressed rules."""
import os
import re

import numpy as np
import pytest

import bls_ref as B
import bls_gpu as G
import cpu as C
import workload_py as W

HERE = os.path.dirname(os.path.abspath(__file__))
G2_CUH = os.path.join(HERE, "..", "icp-gpu_b200", "csrc", "g2.cuh")
G1_CUH = os.path.join(HERE, "..", "icp-gpu_b200", "csrc", "g1.cuh")


# ------------------------------------------------------------------ CPU side

def _u64_array(text, name):
    return sum(w << (64 * i) for i, w in enumerate(_u64_words(text, name)))


def test_device_constants():
    """The exponents of the device's square roots: (p + 1) / 4 in the Fp
    square root, which the G2 decoder's Fp2 square root calls, and (p - 3) / 4
    in the Fp2 square root itself; 379 bits each."""
    text = open(G1_CUH).read()
    body = text[text.index("fp_sqrt_candidate(const fp& a)"):]
    e = _u64_array(body, "e")
    assert e == (B.P + 1) // 4 and e.bit_length() == 379
    assert "fp_pow_ool(a, e, 379)" in body
    g2 = open(G2_CUH).read()
    assert "fp_sqrt_candidate(" in g2
    e2 = _u64_array(g2[g2.index("static __device__ __noinline__ fp2 fp2_sqrt"):], "e")
    assert e2 == (B.P - 3) // 4 and e2.bit_length() == 379 and "fp_pow_ool(d, e, 379)" in g2


def _psi_constants():
    text = open(G2_CUH).read()
    cx1, cy0, cy1 = (B.from_mont_limbs(_u64_words(text, n)) for n in ("cx1", "cy0", "cy1"))
    return (0, cx1), (cy0, cy1)


def _u64_words(text, name):
    m = re.search(r"const uint64_t %s\[\d\] = \{([^}]*)\}" % name, text)
    return [int(w, 16) for w in re.findall(r"0x([0-9a-f]+)ULL", m.group(1))]


X_BLS = -0xd201000000010000


def psi_test(pt):
    """The device's subgroup test restated: psi(P) == [x] P."""
    cx, cy = _psi_constants()
    psi = (B.f2_mul(B.f2_conj(pt[0]), cx), B.f2_mul(B.f2_conj(pt[1]), cy))
    m = B.g2_mul(pt, -X_BLS)
    return m is not None and (m[0], B.f2_neg(m[1])) == psi


def test_psi_constants_and_subgroup_test():
    cx, cy = _psi_constants()
    xi = (1, 1)
    assert cx == B.f2_inv(B.f2_pow(xi, (B.P - 1) // 3))
    assert cy == B.f2_inv(B.f2_pow(xi, (B.P - 1) // 2))
    text = open(G2_CUH).read()
    assert "0xd201000000010000ULL" in text and "i = 62" in text
    # agrees with [r] P == O on subgroup points and on twist points outside G2
    for k in (1, 42, 0x1234567):
        assert psi_test(B.g2_mul(B.G2_GEN, k))
    rng = W.SplitMix64(31)
    for _ in range(6):
        x, y2 = W.g2_random_x(rng, True)
        pt = (x, B.f2_sqrt(y2))
        assert psi_test(pt) == B.g2_in_subgroup(pt) == False   # noqa: E712
    # a point of G2 plus a small-order-free cofactor component stays outside
    x, y2 = W.g2_random_x(rng, True)
    q = B.g2_add(B.G2_GEN, (x, B.f2_sqrt(y2)))
    assert not psi_test(q) and not B.g2_in_subgroup(q)


def sqrt_norm(a):
    """The device's Fp2 square root (the norm method of csrc/g2.cuh), restated
    on integers: (root, ok, branch).  For a1 = 0: sqrt(a0) or u sqrt(-a0); else
    g = sqrt(a0^2 + a1^2), d = (a0 + g) / 2, t = d^((p-3)/4), and x = (d t,
    a1 t / 2) when d t^2 = 1 (d a square), else (a1 t / 2, -d t)."""
    P = B.P
    half = lambda v: v * pow(2, P - 2, P) % P
    a0, a1 = a
    if a1 == 0:
        t = pow(a0, (P + 1) // 4, P)
        if t * t % P == a0:
            x, branch = (t, 0), "fp-square"
        else:
            x, branch = (0, pow(-a0 % P, (P + 1) // 4, P)), "fp-non-square"
    else:
        n = (a0 * a0 + a1 * a1) % P
        g = pow(n, (P + 1) // 4, P)
        if g * g % P != n:
            return (0, 0), False, "norm-non-square"
        d = half(a0 + g)
        t = pow(d, (P - 3) // 4, P)
        dt, h = d * t % P, half(a1 * t % P)
        if dt * t % P == 1:
            x, branch = (dt, h), "d-square"
        else:
            x, branch = (h, -dt % P), "d-non-square"
    return x, B.f2_sqr(x) == a, branch


def test_sqrt_norm_method_restatement():
    """Every branch of the device's Fp2 square root, on squares and
    non-squares: the root squares back exactly when the input is a square."""
    rng = W.SplitMix64(2024)
    cases = [(0, 0), (B.P - 1, 0), (B.P - 4, 0), (5, 0), (0, 1), (4, 4)]
    for _ in range(40):
        cases.append((rng.scalar() % B.P, rng.scalar() % B.P))
    for _ in range(20):
        t = (rng.scalar() % B.P, rng.scalar() % B.P)
        cases.append(B.f2_sqr(t))                           # squares for sure
        cases.append((rng.scalar() % B.P, 0))                # Fp elements: always squares in Fp2
    seen = set()
    for a in cases:
        x, ok, branch = sqrt_norm(a)
        seen.add(branch)
        assert ok == B.f2_is_square(a), a
        if ok:
            assert B.f2_sqr(x) == a
    assert seen == {"fp-square", "fp-non-square", "norm-non-square", "d-square", "d-non-square"}, seen


def test_oracle_g2_round_trip_and_rejects():
    for k in (1, 42, 7 * 294):
        q = B.g2_mul(B.G2_GEN, k)
        for pt in (q, (q[0], B.f2_neg(q[1]))):
            st, back = B.g2_decompress(B.g2_compress(pt))
            assert st == B.ST_OK and back == pt
    assert B.g2_decompress(bytes([0xC0]) + bytes(95)) == (B.ST_OK, None)
    rng = W.SplitMix64(7)
    for enc, want in W.invalid_g2_encodings(rng, B.G2_GEN):
        assert B.g2_decompress(enc)[0] == want


def test_workload_g2_encoding_matches_oracle():
    rng = W.SplitMix64(11)
    sks = np.array([W.WL.scalar_limbs(rng.scalar()) for _ in range(4)], dtype=np.uint64)
    q = W.WL.g2_mul_gen(sks)
    enc = W.WL.g2_compress(q)
    for i in range(4):
        st, pt = B.g2_decompress(bytes(enc[i]))
        assert st == B.ST_OK
        assert np.array(W.g2_affine_u64(pt), dtype=np.uint64).tolist() == q[i].tolist()


# ------------------------------------------------------------------ GPU side

@pytest.fixture(scope="module")
def keys():
    rng = W.SplitMix64(99)
    sks = np.array([W.WL.scalar_limbs(rng.scalar()) for _ in range(24)], dtype=np.uint64)
    q = W.WL.g2_mul_gen(sks)
    return {"q": q, "enc": W.WL.g2_compress(q), "tables": W.WL.g2_prepare(q)}


@pytest.fixture(scope="module", params=[6, 1], ids=["fp2lanes6", "thread"])
def ctx(request):
    G.init()
    with G.Context(lanes=request.param, max_pks=256) as c:
        yield c


def _neg_y(q):
    out = q.copy()
    for k in (12, 18):
        y = B.from_mont_limbs(q[k:k + 6])
        out[k:k + 6] = B.mont_limbs((-y) % B.P)
    return out


@pytest.mark.gpu
def test_g2_decompress_valid(ctx, keys):
    enc = keys["enc"].copy()
    flipped = enc.copy()
    flipped[:, 0] ^= 0x20                                    # the other root: -Q
    st, q = ctx.g2_decompress(np.concatenate([enc, flipped]).tobytes())
    n = enc.shape[0]
    assert (st == 0).all()
    assert (q[:n] == keys["q"]).all()
    assert (q[n:] == np.stack([_neg_y(r) for r in keys["q"]])).all()


@pytest.mark.gpu
def test_g2_decompress_rejects(ctx):
    rng = W.SplitMix64(5)
    cases = W.invalid_g2_encodings(rng, B.G2_GEN)
    cases.append((bytes([0xC0]) + bytes(95), B.ST_OK))        # identity
    st, q = ctx.g2_decompress(b"".join(c[0] for c in cases))
    assert st.tolist() == [c[1] for c in cases]
    assert st.tolist() == [B.g2_decompress(c[0])[0] for c in cases]
    assert (q == 0).all()


@pytest.mark.gpu
def test_register_compressed_tables_pinned(ctx, golden, keys):
    gen = B.g2_compress(B.G2_GEN)
    pk42 = B.g2_compress(B.g2_mul(B.G2_GEN, 42))
    ids, st = ctx.register_pk_compressed(gen + pk42 + keys["enc"].tobytes())
    assert (st == 0).all()
    assert list(ids) == list(range(ids[0], ids[0] + len(ids)))
    assert (ctx.pk_table(ids[0]) == golden["g2_gen_coeffs"]).all()
    assert (ctx.pk_table(ids[1]) == golden["pk42_coeffs"]).all()
    for i in range(keys["enc"].shape[0]):
        assert (ctx.pk_table(ids[2 + i]) == keys["tables"][i]).all()


@pytest.mark.gpu
def test_register_compressed_all_or_nothing(ctx, keys):
    first, _ = ctx.register_pk_compressed(keys["enc"][:1].tobytes())
    bad = bytearray(keys["enc"][1].tobytes())
    bad[0] &= 0x7F
    batch = keys["enc"][:1].tobytes() + bytes(bad) + keys["enc"][2:3].tobytes()
    with pytest.raises(G.GpuError) as e:
        ctx.register_pk_compressed(batch)
    assert e.value.status.tolist() == [0, B.ST_BAD_FLAGS, 0]
    nxt, _ = ctx.register_pk_compressed(keys["enc"][2:3].tobytes())
    assert nxt[0] == first[0] + 1                             # the failed call registered nothing
    assert (ctx.pk_table(int(nxt[0])) == keys["tables"][2]).all()


@pytest.mark.gpu
def test_verify_through_compressed_keys(ctx, golden):
    wl = W.plain_config(n=64, seed=3)
    enc = W.WL.g2_compress(wl["pk_affine"])
    ids, _ = ctx.register_pk_compressed(enc.tobytes())
    res, ml, gt = ctx.verify(wl["sigs"], wl["nhms"], ids, want_values=True)
    assert (res == wl["expect"]).all()
    want, wml, wgt = C.verify_batch(wl["sigs"], wl["nhms"], golden["g2_gen_coeffs"], wl["pk_tabs"],
                                    want_values=True, nthreads=4)
    assert (res == want).all() and (ml == wml).all() and (gt == wgt).all()


@pytest.mark.gpu
def test_identity_key(ctx, golden):
    ids, st = ctx.register_pk_compressed(bytes([0xC0]) + bytes(95))
    assert st.tolist() == [0]
    ident = np.array([0] * 6 + B.mont_limbs(1), dtype=np.uint64)
    sigs = np.stack([ident, golden["g1_generator"], golden["sig_294_g1"]])
    nhms = np.stack([golden["neg_hm_7_g1"]] * 3)
    res, ml, gt = ctx.verify(sigs, nhms, [int(ids[0])] * 3, want_values=True)
    want, wml, wgt = C.verify_batch(sigs, nhms, golden["g2_gen_coeffs"], golden["g2_gen_coeffs"][None],
                                    pk_index=np.zeros(3, dtype=np.int32), pk_inf=np.ones(1, dtype=np.uint8),
                                    want_values=True)
    assert res.tolist() == want.tolist() == [1, 0, 0]
    assert (ml == wml).all() and (gt == wgt).all()


@pytest.mark.gpu
def test_register_affine_batch_tables_pinned(ctx, golden, keys):
    """n affine keys in one call (one launch of the table kernel and one of the
    normalisation): the same tables as the reference's golden ones and the
    workload's, consecutive ids, and the same verify results as keys
    registered one at a time."""
    (x0, x1), (y0, y1) = B.g2_mul(B.G2_GEN, 42)
    q42 = np.array(B.mont_limbs(x0) + B.mont_limbs(x1) + B.mont_limbs(y0) + B.mont_limbs(y1), dtype=np.uint64)
    qs = np.concatenate([q42[None], keys["q"]])
    ids = ctx.register_pk_affine_batch(qs)
    assert list(ids) == list(range(ids[0], ids[0] + len(ids)))
    assert (ctx.pk_table(int(ids[0])) == golden["pk42_coeffs"]).all()
    for i in range(keys["q"].shape[0]):
        assert (ctx.pk_table(int(ids[1 + i])) == keys["tables"][i]).all()
    wl = W.plain_config(n=64, seed=4)
    batch_ids = ctx.register_pk_affine_batch(wl["pk_affine"])
    single_ids = np.array([ctx.register_pk_affine(q) for q in wl["pk_affine"]], dtype=np.int32)
    a = ctx.verify(wl["sigs"], wl["nhms"], batch_ids)
    b = ctx.verify(wl["sigs"], wl["nhms"], single_ids)
    assert (a == wl["expect"]).all() and (b == a).all()
    assert ctx.register_pk_affine_batch(np.zeros((0, 24), dtype=np.uint64)).size == 0
