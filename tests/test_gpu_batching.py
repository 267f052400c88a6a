"""GPU tests of batched execution: many uneven requests in one persistent,
graph-replayed launch give the same results as one launch per request and as
the expected accept bits; the autotuner's pick stays bit-exact."""
import numpy as np
import pytest

import bls_gpu as G
import workload as WL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wl():
    return WL.config_requests(nreq=24, max_size=96, nkeys=40, seed=4)


def _requests(ctx, wl):
    ids = np.array([ctx.register_pk_affine(q) for q in wl["pk_affine"]], dtype=np.int32)
    off = wl["offsets"]
    reqs = []
    for r in range(len(off) - 1):
        a, b = off[r], off[r + 1]
        reqs.append((wl["sigs"][a:b], wl["nhms"][a:b], ids[wl["pk_index"][a:b]]))
    return reqs


@pytest.mark.parametrize("lanes", [6, 8, 4])
def test_persistent_equals_plain_and_expected(wl, lanes):
    with G.Context(lanes=lanes) as ctx:
        reqs = _requests(ctx, wl)
        plain = ctx.verify_requests(reqs, mode=G.MODE_PLAIN)
        pers = ctx.verify_requests(reqs, mode=G.MODE_PERSISTENT)
        again = ctx.verify_requests(reqs, mode=G.MODE_PERSISTENT)   # graph replay
        want = np.split(wl["expect"], wl["offsets"][1:-1])
        for p, q, r, w in zip(plain, pers, again, want):
            assert (p == w).all() and (q == w).all() and (r == w).all()
        # a different shape re-captures
        fewer = ctx.verify_requests(reqs[:5], mode=G.MODE_PERSISTENT)
        for q, w in zip(fewer, want[:5]):
            assert (q == w).all()


def test_persistent_compressed_with_invalid(wl):
    cc = WL.config_compressed(300, 40, seed=9, invalid_frac=0.05)
    with G.Context() as ctx:
        ids = np.array([ctx.register_pk_affine(q) for q in cc["pk_affine"]], dtype=np.int32)
        cuts = [0, 7, 60, 61, 200, 300]
        reqs = [(cc["sigs_compressed"][a:b], cc["nhms"][a:b], ids[cc["pk_index"][a:b]]) for a, b in zip(cuts, cuts[1:])]
        out = ctx.verify_requests(reqs, compressed=True, mode=G.MODE_PERSISTENT)
        assert (np.concatenate(out) == cc["expect"]).all()


def test_autotune_pick_is_exact(wl):
    import torch
    with G.Context() as ctx:
        ids = np.array([ctx.register_pk_affine(q) for q in wl["pk_affine"]], dtype=np.int32)
        n = len(wl["expect"])
        d_sigs = torch.from_numpy(wl["sigs"].view(np.int64)).cuda()
        d_nhms = torch.from_numpy(wl["nhms"].view(np.int64)).cuda()
        d_ids = torch.from_numpy(ids[wl["pk_index"]]).cuda()
        pts = ctx.autotune(n, d_sigs.data_ptr(), d_nhms.data_ptr(), d_ids.data_ptr(), repeats=2)
        assert len(pts) >= 4 and all(p[3] > 0 for p in pts)
        assert {p[1] for p in pts if p[0] == 6} == {64, 384}          # both block shapes swept
        res = ctx.verify(wl["sigs"], wl["nhms"], ids[wl["pk_index"]])
        assert (res == wl["expect"]).all()


def test_request_argument_errors(wl):
    with G.Context() as ctx:
        reqs = _requests(ctx, wl)[:2]
        bad = [(reqs[0][0], reqs[0][1], np.full(len(reqs[0][2]), 999, dtype=np.int32))]
        with pytest.raises(G.GpuError):
            ctx.verify_requests(bad)
        assert ctx.verify_requests([]) == []
