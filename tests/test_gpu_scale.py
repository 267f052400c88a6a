"""Batches far larger than one wave of the verify kernel (888 resident blocks of
five verifications on a B200), with ragged sizes: every result against the
workload's known answer, and the same items verified in one call and in
uneven chunks give the same results.  And concurrent callers: the reference
ABI and one shared context called from several host threads at once (the
reference's library is not thread-safe; this one's entry points are)."""
import threading

import numpy as np
import pytest

import bls_gpu as G
import cpu as C
import workload_py as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    G.init()
    with G.Context(lanes=6) as c:
        yield c


@pytest.fixture(scope="module")
def big():
    return W.WL.config_keyset(40003, 40, seed=41)


def _ids(ctx, wl):
    ids = np.array([ctx.register_pk_affine(q) for q in wl["pk_affine"]], dtype=np.int32)
    return ids[wl["pk_index"]]


def test_multi_wave_batch_is_exact(ctx, big):
    ids = _ids(ctx, big)
    res = ctx.verify(big["sigs"], big["nhms"], ids)
    assert (res == big["expect"]).all()
    assert (big["expect"] == 0).sum() > 4000          # 1 in 8 corrupted, both kinds


def test_chunked_equals_one_call(ctx, big):
    ids = _ids(ctx, big)
    whole = ctx.verify(big["sigs"], big["nhms"], ids)
    cuts = [0, 1, 6, 4099, 17000, 33333, len(ids)]
    parts = [ctx.verify(big["sigs"][a:b], big["nhms"][a:b], ids[a:b]) for a, b in zip(cuts, cuts[1:])]
    assert (np.concatenate(parts) == whole).all()


def test_compressed_multi_wave_with_invalid(ctx):
    wl = W.WL.config_compressed(n=20011, nkeys=40, seed=43)
    ids = _ids(ctx, wl)
    res = ctx.verify(wl["sigs_compressed"], wl["nhms"], ids, compressed=True)
    assert (res == wl["expect"]).all()
    assert (wl["expect"] < 0).sum() == round(0.02 * 20011)


def _run_threads(fn, n):
    errors = []

    def body(k):
        try:
            fn(k)
        except Exception as e:          # noqa: BLE001 - reported below
            errors.append(repr(e))
    th = [threading.Thread(target=body, args=(k,)) for k in range(n)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors


def test_reference_abi_concurrent_callers(golden):
    wls = [W.plain_config(n=24 + 7 * k, seed=60 + k) for k in range(4)]

    def call(k):
        wl = wls[k]
        for _ in range(3):
            got = G.batch_bls_verify(wl["sigs"], wl["nhms"], golden["g2_gen_coeffs"], wl["pk_tabs"])
            assert [int(x) for x in got] == list(wl["expect"])
    _run_threads(call, 4)


def test_shared_context_concurrent_callers(ctx, big):
    ids = _ids(ctx, big)
    cuts = [0, 5000, 9001, 16384, 20000]

    def call(k):
        a, b = cuts[k], cuts[k + 1]
        for _ in range(2):
            r = ctx.verify(big["sigs"][a:b], big["nhms"][a:b], ids[a:b])
            assert (r == big["expect"][a:b]).all()
    _run_threads(call, 4)


def test_reference_abi_repeated_tables(golden, big):
    """4,096 items over 40 keys through the reference's entry point: one table
    per item, repeated; the library copies the distinct ones with an index."""
    n = 4096
    tabs = np.ascontiguousarray(big["pk_tables"][big["pk_index"][:n]])
    got = G.batch_bls_verify(big["sigs"][:n], big["nhms"][:n], golden["g2_gen_coeffs"], tabs)
    assert [int(x) for x in got] == list(big["expect"][:n])


def test_reference_abi_fingerprint_twins(golden, big):
    """Tables equal to a key's table except in the last word share its
    fingerprint but must not share its id: every result equals the oracle's on
    the same per-item tables."""
    n = 600
    tabs = np.ascontiguousarray(big["pk_tables"][big["pk_index"][:n]])
    twins = np.arange(3, n, 7)
    tabs[twins, -1] ^= np.uint64(1)
    got = np.array(G.batch_bls_verify(big["sigs"][:n], big["nhms"][:n], golden["g2_gen_coeffs"], tabs),
                   dtype=np.int32)
    want = C.verify_batch(big["sigs"][:n], big["nhms"][:n], golden["g2_gen_coeffs"], tabs, nthreads=8)
    assert (got == want).all()
    untouched = np.setdiff1d(np.arange(n), twins)
    assert (got[untouched] == big["expect"][untouched]).all()


def test_reference_abi_repeat_call_uses_cached_tables(golden, big):
    """The same tables again (found by exact content among the tables seen
    before, so nothing but the index crosses), then a batch mixing cached and
    new tables: the same results as the first call and the oracle."""
    n = 3000
    tabs = np.ascontiguousarray(big["pk_tables"][big["pk_index"][:n]])
    for _ in range(2):
        got = G.batch_bls_verify(big["sigs"][:n], big["nhms"][:n], golden["g2_gen_coeffs"], tabs)
        assert [int(x) for x in got] == list(big["expect"][:n])
    mixed = tabs.copy()
    mixed[::5, 100] ^= np.uint64(1 << 7)     # some tables the library has not seen
    got = np.array(G.batch_bls_verify(big["sigs"][:n], big["nhms"][:n], golden["g2_gen_coeffs"], mixed),
                   dtype=np.int32)
    want = C.verify_batch(big["sigs"][:n], big["nhms"][:n], golden["g2_gen_coeffs"], mixed, nthreads=8)
    assert (got == want).all()


def test_reference_abi_other_generator_table(golden, big):
    """A caller's generator table that is not the context's own: the tables
    cross as they are and the results equal the oracle's with that table."""
    n = 400
    tabs = np.ascontiguousarray(big["pk_tables"][big["pk_index"][:n]])
    g2 = golden["pk42_coeffs"]
    got = np.array(G.batch_bls_verify(big["sigs"][:n], big["nhms"][:n], g2, tabs), dtype=np.int32)
    want = C.verify_batch(big["sigs"][:n], big["nhms"][:n], g2, tabs, nthreads=8)
    assert (got == want).all()
