"""Random-linear-combination batch verification (bls_verify_batch_rlc): the
combined check e(sum r_i sig_i, G2) * prod_k e(sum_{pk_i = k} r_i (-H(m_i)), pk_k)
== 1 with per-item fallback.  Results must equal bls_verify_batch's item for
item; the aggregated points are checked bit for bit against the oracle's
group arithmetic, and the combination rule itself against the oracle's
pairing on the CPU."""
import numpy as np
import pytest

import bls_ref as B
import bls_gpu as G
import workload_py as W


ITEM_FIELDS = ("sigs", "nhms", "pk_index", "expect")


def _valid_subset(wl):
    keep = np.nonzero(wl["expect"] == 1)[0]
    return {k: (wl[k][keep] if k in ITEM_FIELDS else wl[k]) for k in wl}


# the device uses r = a + lambda b for a 64-bit scalar b:a, lambda = -x^2 mod r
# (the eigenvalue of phi(x, y) = (beta x, y) on G1)
LAMBDA = (-(0xd201000000010000 ** 2)) % B.R_ORDER


def effective(k):
    k = int(k)
    return ((k & 0xffffffff) + LAMBDA * (k >> 32)) % B.R_ORDER


def _oracle_aggregate(sigs, nhms, keys_of_items, r):
    s, t = None, {}
    for i in range(len(r)):
        s = B.g1_add(s, B.g1_mul(B.g1_from_mont_u64(sigs[i].tolist()), r[i]))
        k = int(keys_of_items[i])
        t[k] = B.g1_add(t.get(k), B.g1_mul(B.g1_from_mont_u64(nhms[i].tolist()), r[i]))
    return s, t


def test_lambda_is_a_cube_root_of_unity():
    assert (LAMBDA * LAMBDA + LAMBDA + 1) % B.R_ORDER == 0
    g = B.g1_mul(B.G1_GEN, 5)
    assert effective(3 | (7 << 32)) == (3 + 7 * LAMBDA) % B.R_ORDER
    assert B.g1_mul(g, effective(1 << 32)) == B.g1_mul(g, LAMBDA)


# ------------------------------------------------------------------ CPU side

def test_combination_rule_on_the_oracle(golden):
    """The combined pairing product is one for a valid batch and not for a batch
    with one bad item (three items, two keys, oracle pairing)."""
    wl = W.WL.config_keyset(8, 2, seed=9)
    g2c = B.coeffs_from_limbs(golden["g2_gen_coeffs"].tolist())
    pkc = [B.coeffs_from_limbs(t.tolist()) for t in wl["pk_tables"]]
    idx = [i for i in range(8) if wl["expect"][i] == 1][:3]
    r = [0x9e3779b97f4a7c15, 0x1234567890abcdef, 0xfedcba9876543211]

    def combined(sig_override=None):
        sigs = wl["sigs"][idx].copy()
        if sig_override is not None:
            sigs[0] = sig_override
        s, t = _oracle_aggregate(sigs, wl["nhms"][idx], wl["pk_index"][idx], r)
        pairs = [(s, g2c, s is None)] + [(t[k], pkc[k], t[k] is None) for k in sorted(t)]
        pairs = [(p if p is not None else (0, 0), c, skip) for p, c, skip in pairs]
        return B.f12_is_one(B.final_exponentiation(B.multi_miller_loop(pairs)))

    assert combined()
    assert not combined(golden["g1_generator"])


# ------------------------------------------------------------------ GPU side

@pytest.fixture(scope="module", params=[6, 1], ids=["fp2lanes6", "thread"])
def ctx(request):
    G.init()
    with G.Context(lanes=request.param) as c:
        yield c


@pytest.fixture(scope="module")
def keyset():
    return W.WL.config_keyset(512, 40, seed=31)


def _ids(ctx, wl):
    ids = np.array([ctx.register_pk_affine(q) for q in wl["pk_affine"]], dtype=np.int32)
    return ids[wl["pk_index"]]


@pytest.mark.gpu
def test_valid_batch_combined(ctx, keyset):
    wl = _valid_subset(keyset)
    ids = _ids(ctx, wl)
    res, comb = ctx.verify_rlc(wl["sigs"], wl["nhms"], ids)
    assert comb == 1 and (res == 1).all()
    assert (res == ctx.verify(wl["sigs"], wl["nhms"], ids)).all()


@pytest.mark.gpu
def test_aggregates_bit_exact(ctx, keyset):
    wl = _valid_subset(keyset)
    n = 48
    sigs, nhms, ids = wl["sigs"][:n], wl["nhms"][:n], _ids(ctx, wl)[:n]
    rng = W.SplitMix64(4)
    r = np.array([rng.next() | 1 for _ in range(n)], dtype=np.uint64)
    res, comb, agg = ctx.verify_rlc(sigs, nhms, ids, scalars=r, want_agg=True)
    assert comb == 1
    s, t = _oracle_aggregate(sigs, nhms, ids, [effective(k) for k in r])
    assert agg[0].tolist() == B.g1_to_mont_u64(s)
    for j, k in enumerate(sorted(set(ids.tolist()))):
        assert agg[1 + j].tolist() == B.g1_to_mont_u64(t[k])


@pytest.mark.gpu
def test_corrupted_batch_falls_back(ctx, keyset):
    ids = _ids(ctx, keyset)
    res, comb = ctx.verify_rlc(keyset["sigs"], keyset["nhms"], ids)
    assert comb == 0
    assert (res == keyset["expect"]).all()
    assert (res == ctx.verify(keyset["sigs"], keyset["nhms"], ids)).all()


@pytest.mark.gpu
def test_compressed_with_bad_encodings(ctx, keyset):
    wl = _valid_subset(keyset)
    ids = _ids(ctx, wl)
    enc = W.WL.g1_compress(wl["sigs"]).copy()
    rng = W.SplitMix64(12)
    bad = W.invalid_encodings(rng, B.G1_GEN)
    for j, (b, _) in enumerate(bad):
        enc[5 + 7 * j] = np.frombuffer(b, dtype=np.uint8)
    res, comb = ctx.verify_rlc(enc.tobytes(), wl["nhms"], ids, compressed=True)
    want = ctx.verify(enc.tobytes(), wl["nhms"], ids, compressed=True)
    assert comb == 1
    assert (res == want).all()
    assert [int(res[5 + 7 * j]) for j in range(len(bad))] == [-st for _, st in bad]


@pytest.mark.gpu
def test_point_outside_g1_forces_item_path(ctx, keyset):
    wl = _valid_subset(keyset)
    ids = _ids(ctx, wl)
    sigs = wl["sigs"].copy()
    pt = W.random_curve_point_not_in_g1(W.SplitMix64(3))
    sigs[10] = np.array(B.g1_to_mont_u64(pt), dtype=np.uint64)      # on the curve, not in G1
    sigs[11, 0] ^= np.uint64(1)                                      # off the curve
    res, comb = ctx.verify_rlc(sigs, wl["nhms"], ids)
    assert comb == 0
    assert (res == ctx.verify(sigs, wl["nhms"], ids)).all()


@pytest.mark.gpu
def test_identity_points_and_keys(ctx, golden, keyset):
    wl = _valid_subset(keyset)
    ids = list(_ids(ctx, wl)[:16])
    ident_pk, _ = ctx.register_pk_compressed(bytes([0xC0]) + bytes(95))
    ident = np.array([0] * 6 + B.mont_limbs(1), dtype=np.uint64)
    sigs = np.concatenate([wl["sigs"][:16], ident[None], ident[None]])
    nhms = np.concatenate([wl["nhms"][:16], golden["neg_hm_7_g1"][None], ident[None]])
    ids = np.array(ids + [int(ident_pk[0]), ids[0]], dtype=np.int32)
    res, comb = ctx.verify_rlc(sigs, nhms, ids)
    assert comb == 1 and (res == 1).all()
    assert (res == ctx.verify(sigs, nhms, ids)).all()


@pytest.mark.gpu
def test_many_keys(ctx):
    wl = _valid_subset(W.WL.config_plain(300, seed=8))
    ids = _ids(ctx, wl)
    assert len(set(ids.tolist())) > 256
    res, comb = ctx.verify_rlc(wl["sigs"], wl["nhms"], ids)
    assert comb == 1 and (res == 1).all()


@pytest.mark.gpu
def test_zero_scalar_rejected(ctx, keyset):
    ids = _ids(ctx, keyset)[:4]
    with pytest.raises(G.GpuError):
        ctx.verify_rlc(keyset["sigs"][:4], keyset["nhms"][:4], ids, scalars=[1, 2, 0, 3])
