"""Pairing-value parity at the workloads' own sizes.

The reference pins its verifier by the Miller-loop and pairing values of
whole verifications (cuda/test_bls_verify.cu:147-172, cuda/test_final_exp.cu:
288-325), not only by accept bits.  A wrong Gt whose "is one" bit happens to
agree would pass an accept-bit test, and what changes between a small batch and
a large one is exactly the kernel's scheduling (waves, claims from the work
counter, graph replay).  So here every item of each large batch is compared
with the oracle (oracle/cpu_verifier.cpp on all host threads) on all 72 limbs
of its Miller value and its Gt value, as well as its accept bit:

  * the 4,096-item keyset workload over 40 resident keys (the bench's headline
    batch, same seed);
  * a 40,003-item keyset batch, many waves of the kernel;
  * an 8,192-item slice of the 65,536-item compressed workload (2% invalid
    encodings: values of the valid items, decode statuses of the others);
  * the batching workload (256 requests, sizes log-uniform in [1, 2048], 1-40
    keys each, 76,123 items) through bls_verify_requests in both modes, at
    accept-bit level against the oracle (that entry point returns no values).
"""
import os

import numpy as np
import pytest

import bls_gpu as G
import cpu as C
import workload as WL

pytestmark = pytest.mark.gpu

NT = max(1, os.cpu_count() or 1)
# R mod p, the Montgomery form of 1 (6 x u64 little-endian)
ONE_MONT = np.array([0x760900000002FFFD, 0xEBF4000BC40C0002, 0x5F48985753C758BA,
                     0x77CE585370525745, 0x5C071A97A256EC6D, 0x15F65EC3FA80E493], dtype=np.uint64)


@pytest.fixture(scope="module", params=[384, 64], ids=["wide", "five"])
def ctx(request):
    G.init()
    with G.Context(lanes=6, threads_per_block=request.param) as c:
        yield c


@pytest.fixture(scope="module")
def keyset4096():
    return WL.config_keyset(4096, 40, seed=2)


@pytest.fixture(scope="module")
def keyset40003():
    return WL.config_keyset(40003, 40, seed=41)


@pytest.fixture(scope="module")
def compressed65536():
    return WL.config_compressed(65536, 40, seed=3)


@pytest.fixture(scope="module")
def requests256():
    return WL.config_requests(256, 2048, 40, seed=4)


def _register(ctx, wl):
    return ctx.register_pk_affine_batch(wl["pk_affine"])


@pytest.fixture(scope="module")
def g2_table(ctx):
    return ctx.pk_table(-1)


def _check_values(ctx, g2_table, wl, ids):
    res, ml, gt = ctx.verify(wl["sigs"], wl["nhms"], ids[wl["pk_index"]], want_values=True)
    wres, wml, wgt = C.verify_batch(wl["sigs"], wl["nhms"], g2_table, wl["pk_tables"], pk_index=wl["pk_index"],
                                    nthreads=NT, want_values=True)
    assert (res == wl["expect"]).all()
    assert (res == wres).all()
    bad_ml = np.nonzero((ml != wml).any(axis=1))[0]
    bad_gt = np.nonzero((gt != wgt).any(axis=1))[0]
    assert bad_ml.size == 0, ("Miller values differ", bad_ml[:10])
    assert bad_gt.size == 0, ("Gt values differ", bad_gt[:10])
    # the accept bit is exactly "Gt is one": R mod p in c0.c0.c0, zeros elsewhere
    one = np.zeros(72, dtype=np.uint64)
    one[:6] = ONE_MONT
    assert ((gt == one).all(axis=1) == (res == 1)).all()


def test_keyset_4096_values_exact(ctx, g2_table, keyset4096):
    _check_values(ctx, g2_table, keyset4096, _register(ctx, keyset4096))


def test_keyset_multi_wave_values_exact(ctx, g2_table, keyset40003):
    _check_values(ctx, g2_table, keyset40003, _register(ctx, keyset40003))


def test_compressed_slice_values_exact(ctx, g2_table, compressed65536):
    full = compressed65536
    n = 8192
    comp = np.ascontiguousarray(full["sigs_compressed"][:n])
    nhms = full["nhms"][:n]
    pk_index = full["pk_index"][:n]
    expect = full["expect"][:n]
    assert (expect < 0).sum() >= 100                  # the slice carries every kind of invalid encoding
    ids = _register(ctx, full)
    res, ml, gt = ctx.verify(comp.reshape(-1), nhms, ids[pk_index], compressed=True, want_values=True)
    assert (res == expect).all()
    st, xy = C.g1_decompress(comp.reshape(-1), nthreads=NT)
    assert (res[st != 0] == -st[st != 0]).all()
    ok = np.nonzero(st == 0)[0]
    wres, wml, wgt = C.verify_batch(xy[ok], nhms[ok], g2_table, full["pk_tables"], pk_index=pk_index[ok],
                                    nthreads=NT, want_values=True)
    assert (res[ok] == wres).all()
    assert (ml[ok] == wml).all()
    assert (gt[ok] == wgt).all()


@pytest.mark.parametrize("mode", [G.MODE_PLAIN, G.MODE_PERSISTENT])
def test_batching_workload_full_size(ctx, g2_table, mode, requests256):
    wl = requests256
    assert len(wl["offsets"]) == 257 and len(wl["expect"]) > 60000
    ids = _register(ctx, wl)
    off = wl["offsets"]
    reqs = [(wl["sigs"][a:b], wl["nhms"][a:b], ids[wl["pk_index"][a:b]]) for a, b in zip(off[:-1], off[1:])]
    got = np.concatenate(ctx.verify_requests(reqs, mode=mode))
    assert (got == wl["expect"]).all()
    want = C.verify_batch(wl["sigs"], wl["nhms"], g2_table, wl["pk_tables"], pk_index=wl["pk_index"], nthreads=NT)
    assert (got == want).all()
    if mode == G.MODE_PERSISTENT:                     # graph replay of the same shapes
        again = np.concatenate(ctx.verify_requests(reqs, mode=mode))
        assert (again == got).all()
