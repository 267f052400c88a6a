"""GPU parity: the CUDA path through the C ABI against the oracle, bit for bit
(accept bits, decode statuses, Miller-loop and Gt values, line tables)."""
import numpy as np
import pytest

import bls_ref as B
import bls_gpu as G
import cpu as C
import workload_py as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(6, 384), (6, 64), (8, 0), (4, 0), (1, 0)],
                ids=["fp2lanes6-wide", "fp2lanes6-five", "lanes8", "lanes4", "thread"])
def ctx(request):
    G.init()
    lanes, tpb = request.param
    with G.Context(lanes=lanes, threads_per_block=tpb) as c:
        yield c


@pytest.fixture(scope="module")
def plain64():
    return W.plain_config(n=64, seed=1)


def test_golden_kat_reference_abi(golden):
    sig = golden["sig_294_g1"][None]
    nhm = golden["neg_hm_7_g1"][None]
    assert G.batch_bls_verify(sig, nhm, golden["g2_gen_coeffs"], golden["pk42_coeffs"][None]) == [True]
    assert G.batch_bls_verify(golden["g1_generator"][None], nhm, golden["g2_gen_coeffs"],
                              golden["pk42_coeffs"][None]) == [False]


def test_golden_values_extended_api(ctx, golden):
    pk = ctx.register_pk_coeffs(golden["pk42_coeffs"])
    g = ctx.register_pk_coeffs(golden["g2_gen_coeffs"])
    ident = np.array([0] * 6 + B.mont_limbs(1), dtype=np.uint64)
    sigs = np.stack([golden["sig_294_g1"], golden["g1_generator"]])
    nhms = np.stack([golden["neg_hm_7_g1"], ident])
    res, ml, gt = ctx.verify(sigs, nhms, [pk, g], want_values=True)
    assert list(res) == [1, 0]
    assert (ml[0, :6] == golden["ml_2pair_c000"]).all()
    # item 1: e(G1, G2) alone (identity pair skipped): full 72-limb pins
    assert (ml[1] == golden["ml_g1_g2"]).all()
    assert (gt[1] == golden["pairing_g1_g2"]).all()


def test_generator_table_on_device(ctx, golden):
    assert (ctx.pk_table(-1) == golden["g2_gen_coeffs"]).all()


def test_pk_register_affine_matches_oracle(ctx, golden, plain64):
    q42 = np.array(W.g2_affine_u64(B.g2_mul(B.G2_GEN, 42)), dtype=np.uint64)
    assert (ctx.pk_table(ctx.register_pk_affine(q42)) == golden["pk42_coeffs"]).all()
    for i in (0, 5):
        pid = ctx.register_pk_affine(plain64["pk_affine"][i])
        assert (ctx.pk_table(pid) == plain64["pk_tabs"][i]).all()


def test_plain_config_reference_abi(golden, plain64):
    wl = plain64
    got = G.batch_bls_verify(wl["sigs"], wl["nhms"], golden["g2_gen_coeffs"], wl["pk_tabs"])
    assert [int(x) for x in got] == list(wl["expect"])
    want = C.verify_batch(wl["sigs"], wl["nhms"], golden["g2_gen_coeffs"], wl["pk_tabs"], nthreads=4)
    assert (np.array(got, dtype=np.int32) == want).all()


def test_plain_config_values(ctx, golden, plain64):
    wl = plain64
    ids = [ctx.register_pk_coeffs(t) for t in wl["pk_tabs"]]
    res, ml, gt = ctx.verify(wl["sigs"], wl["nhms"], ids, want_values=True)
    want, wml, wgt = C.verify_batch(wl["sigs"], wl["nhms"], golden["g2_gen_coeffs"], wl["pk_tabs"],
                                    want_values=True, nthreads=4)
    assert (res == want).all() and (res == wl["expect"]).all()
    assert (ml == wml).all()
    assert (gt == wgt).all()


def test_garbage_points_bit_exact(ctx, golden):
    """Off-curve inputs through the raw layout: same Miller and Gt values as the oracle."""
    rng = np.random.default_rng(4)
    vals = [int(rng.integers(1, 2**63)) * 7919 % B.P for _ in range(16)]
    sigs = np.array([B.mont_limbs(vals[2 * i]) + B.mont_limbs(vals[2 * i + 1]) for i in range(4)], dtype=np.uint64)
    nhms = np.array([B.mont_limbs(vals[8 + 2 * i]) + B.mont_limbs(vals[9 + 2 * i]) for i in range(4)], dtype=np.uint64)
    pk = ctx.register_pk_coeffs(golden["pk42_coeffs"])
    res, ml, gt = ctx.verify(sigs, nhms, [pk] * 4, want_values=True)
    want, wml, wgt = C.verify_batch(sigs, nhms, golden["g2_gen_coeffs"], golden["pk42_coeffs"][None],
                                    pk_index=np.zeros(4, np.int32), want_values=True)
    assert (res == want).all() and (ml == wml).all() and (gt == wgt).all()


def test_identity_inputs(ctx, golden):
    ident = np.array([0] * 6 + B.mont_limbs(1), dtype=np.uint64)
    zero = np.zeros(12, dtype=np.uint64)
    pk = ctx.register_pk_coeffs(golden["pk42_coeffs"])
    pk_inf = ctx.register_pk_coeffs(golden["pk42_coeffs"], is_identity=True)
    sigs = np.stack([ident, zero, golden["sig_294_g1"], ident])
    nhms = np.stack([ident, zero, golden["neg_hm_7_g1"], golden["neg_hm_7_g1"]])
    ids = [pk, pk, pk_inf, pk_inf]
    res, ml, gt = ctx.verify(sigs, nhms, ids, want_values=True)
    # both pairs skipped -> 1; sig only with pk identity -> e(294 G1, G2) != 1
    assert list(res) == [1, 1, 0, 1]
    one = np.array(B.f12_mont_limbs(B.F12_ONE), dtype=np.uint64)
    assert (gt[0] == one).all() and (ml[0] == one).all()


def test_compressed_path_statuses(ctx, golden, plain64):
    wl = plain64
    n = 24
    comp = [B.g1_compress(p) for p in wl["sig_points"][:n]]
    expect = list(wl["expect"][:n])
    bad = W.invalid_encodings(W.SplitMix64(3), wl["sig_points"][0])
    for k, (b, st) in enumerate(bad):
        comp[2 + 3 * k] = b
        expect[2 + 3 * k] = -st
    ids = [ctx.register_pk_coeffs(t) for t in wl["pk_tabs"][:n]]
    res = ctx.verify(b"".join(comp), wl["nhms"][:n], ids, compressed=True)
    assert list(res) == expect
    want = C.verify_compressed_batch(np.frombuffer(b"".join(comp), dtype=np.uint8), wl["nhms"][:n],
                                     golden["g2_gen_coeffs"], wl["pk_tabs"][:n])
    assert (res == want).all()


def test_decompress_abi_and_statuses(ctx, plain64):
    pts = plain64["sig_points"][:16]
    comp = b"".join(B.g1_compress(p) for p in pts)
    out = G.g1_decompress_batch(comp)
    assert all(list(out[i]) == B.g1_to_mont_u64(p) for i, p in enumerate(pts))
    bad = W.invalid_encodings(W.SplitMix64(8), pts[0])
    blob = comp + b"".join(b for b, _ in bad) + B.g1_compress(None)
    st, xy = ctx.g1_decompress(blob)
    want_st, want_xy = C.g1_decompress(np.frombuffer(blob, dtype=np.uint8))
    assert (st == want_st).all() and (xy == want_xy).all()
    assert list(st[16:]) == [s for _, s in bad] + [0]
    # the reference ABI refuses batches holding an invalid point or the identity
    with pytest.raises(G.GpuError):
        G.g1_decompress_batch(comp + bad[0][0])
    with pytest.raises(G.GpuError):
        G.g1_decompress_batch(B.g1_compress(None))


def test_empty_and_single(ctx, golden):
    assert G.batch_bls_verify(np.zeros((0, 12)), np.zeros((0, 12)), golden["g2_gen_coeffs"], np.zeros((0, 2448))) == []
    pk = ctx.register_pk_coeffs(golden["pk42_coeffs"])
    assert list(ctx.verify(golden["sig_294_g1"][None], golden["neg_hm_7_g1"][None], [pk])) == [1]
    with pytest.raises(G.GpuError):
        ctx.verify(golden["sig_294_g1"][None], golden["neg_hm_7_g1"][None], [10**6])


def test_imad_chain_ceiling_is_plausible():
    """The measured carry-chain ceiling lies between 1 T and the nominal peak
    (SMs x 64 IMAD per clock x 2.1 GHz)."""
    import torch
    with G.Context() as c:
        rate = c.imad_chain_rate()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert 1e12 < rate < sms * 64 * 2.1e9


def test_limb_layout_rates_are_plausible():
    """The autotuner's limb-layout points: each layout's product rate is
    positive and below what the nominal IMAD peak allows for its multiply
    count (216, 225 and 196 multiplies per product), and the 32-bit
    carry-chain layout the verify kernels use is the fastest of the three."""
    import torch
    with G.Context() as c:
        rates = c.limb_layout_rates()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert len(rates) == 3
    for r, muls in zip(rates, (216, 225, 196)):
        assert 1e9 < r < sms * 64 * 2.1e9 / muls
    assert rates[0] == max(rates)
