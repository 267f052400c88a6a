"""bls_verify_compressed_noalloc: the verify entry point for callers that
cannot allocate device memory while they verify (a host process that owns all
device memory through its own allocator, or a path that cannot take
cudaMalloc's device-wide synchronisation).

It works only on the caller's device buffers plus a fixed scratch array inside
the library.  Here it must give exactly what the existing entry point
(bls_verify_batch with compressed signatures) gives, for every lane width it
accepts, on two calls in a row that share that scratch; it must report a key
index outside the caller's tables as -BLS_ST_BAD_KEY_INDEX without reading a
table for it, honour identity-key flags, and refuse a batch larger than the
scratch holds.  This file is collected last so that a run stopping at the first
failure has already run every other test; it also passes alone in a fresh
process."""
import numpy as np
import pytest

import bls_gpu as G
import workload as WL

ST_BAD_KEY_INDEX = 5


def test_rejects_batches_beyond_the_scratch_capacity():
    # returns before touching the GPU, so it runs anywhere
    rc = G.verify_compressed_noalloc(1, 1, 1, 1, None, 1, 1, 1, G.NOALLOC_MAX_ITEMS + 1, 6, None)
    assert rc == G.BLS_ERR_INVALID


def test_rejects_bad_arguments_before_launching():
    # no tables, a NULL key index array, an unsupported lane width: all refused on the host
    assert G.verify_compressed_noalloc(1, 1, 1, 1, None, 0, 1, 1, 4, 6, None) == G.BLS_ERR_INVALID
    assert G.verify_compressed_noalloc(1, 1, 1, 1, None, 3, None, 1, 4, 6, None) == G.BLS_ERR_INVALID
    assert G.verify_compressed_noalloc(1, 1, 1, 1, None, 3, 1, 1, 4, 3, None) == G.BLS_ERR_INVALID
    assert G.verify_compressed_noalloc(1, 1, 1, 1, None, 3, 1, 1, 0, 6, None) == G.BLS_OK


def _batches():
    b1 = WL.config_compressed(700, 40, seed=21, invalid_frac=0.05)
    b2 = WL.config_compressed(300, 40, seed=22, invalid_frac=0.1)
    # batch 2 adds a 41st table flagged as the identity key (a copy of table 0)
    # and a few key indices outside [0, 41)
    b2["pk_tables"] = np.concatenate([b2["pk_tables"], b2["pk_tables"][:1]])
    b2["identity"] = np.zeros(41, dtype=np.uint8)
    b2["identity"][40] = 1
    idx = b2["pk_index"].astype(np.int32).copy()
    idx[[3, 50, 51, 120]] = 40
    bad = np.array([7, 8, 99, 200, 299])
    idx[bad] = [41, -1, 1000, -7, 41]
    b2["pk_index"] = idx
    b2["bad_index"] = bad
    return [b1, b2]


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [6, 8, 4, 2])
def test_noalloc_matches_existing_entry_point_twice(lanes):
    import torch

    G.init()
    batches = _batches()
    with G.Context() as ctx:
        g2 = ctx.pk_table(-1)
        wants = []
        for cc in batches:
            ident = cc.get("identity", np.zeros(len(cc["pk_tables"]), dtype=np.uint8))
            ids = np.array([ctx.register_pk_coeffs(t, is_identity=bool(f)) for t, f in zip(cc["pk_tables"], ident)],
                           dtype=np.int32)
            safe = np.clip(cc["pk_index"], 0, len(ids) - 1)
            want = ctx.verify(cc["sigs_compressed"].reshape(-1), cc["nhms"], ids[safe], compressed=True)
            if "bad_index" in cc:
                b = cc["bad_index"]
                want[b] = np.where(want[b] >= 0, -ST_BAD_KEY_INDEX, want[b])
            wants.append(want)
    assert (wants[0] == batches[0]["expect"]).all()
    stream = torch.cuda.current_stream()
    d_g2 = torch.from_numpy(g2.view(np.int64)).cuda()
    for cc, want in zip(batches, wants):
        n = len(want)
        d_sigs = torch.from_numpy(np.ascontiguousarray(cc["sigs_compressed"].reshape(-1))).cuda()
        d_nhms = torch.from_numpy(cc["nhms"].view(np.int64)).cuda()
        d_tabs = torch.from_numpy(np.ascontiguousarray(cc["pk_tables"]).view(np.int64)).cuda()
        d_idx = torch.from_numpy(cc["pk_index"].astype(np.int32)).cuda()
        d_ident = torch.from_numpy(cc["identity"]).cuda() if "identity" in cc else None
        d_res = torch.full((n,), -99, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = G.verify_compressed_noalloc(d_sigs.data_ptr(), d_nhms.data_ptr(), d_g2.data_ptr(), d_tabs.data_ptr(),
                                         d_ident.data_ptr() if d_ident is not None else None,
                                         len(cc["pk_tables"]), d_idx.data_ptr(), d_res.data_ptr(), n, lanes,
                                         stream.cuda_stream)
        assert rc == G.BLS_OK, G.last_error()
        torch.cuda.synchronize()
        got = d_res.cpu().numpy()
        assert (got == want).all(), np.nonzero(got != want)
    # the identity-key items and the bad indices really were exercised
    assert (wants[1][batches[1]["bad_index"]] < 0).all()
    assert (wants[1][[3, 50, 51, 120]] != 1).all()
