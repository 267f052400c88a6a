"""bls_verify_compressed_noalloc: the verify entry point for callers that
cannot allocate device memory while they verify (inside a stream capture,
under a host process that owns all device memory through its own allocator,
or on a path that cannot take cudaMalloc's device-wide synchronisation).

It works only on the caller's device buffers plus a fixed scratch array inside
the library.  Here it must give exactly what the existing entry point
(bls_verify_batch with compressed signatures) gives, on two calls in a row that
share that scratch, and it must refuse a batch larger than the scratch holds.
This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import numpy as np
import pytest

import bls_gpu as G
import workload as WL


def test_rejects_batches_beyond_the_scratch_capacity():
    # returns before touching the GPU, so it runs anywhere
    rc = G.verify_compressed_noalloc(1, 1, 1, 1, 1, 1, G.NOALLOC_MAX_ITEMS + 1, 8, None)
    assert rc == G.BLS_ERR_INVALID


@pytest.mark.gpu
def test_noalloc_matches_existing_entry_point_twice():
    import torch

    G.init()
    batches = [WL.config_compressed(700, 40, seed=21, invalid_frac=0.05),
               WL.config_compressed(300, 40, seed=22, invalid_frac=0.1)]
    with G.Context() as ctx:
        g2 = ctx.pk_table(-1)
        wants = []
        for cc in batches:
            ids = np.array([ctx.register_pk_coeffs(t) for t in cc["pk_tables"]], dtype=np.int32)
            wants.append(ctx.verify(cc["sigs_compressed"].reshape(-1), cc["nhms"], ids[cc["pk_index"]],
                                    compressed=True))
    stream = torch.cuda.current_stream()
    d_g2 = torch.from_numpy(g2.view(np.int64)).cuda()
    for cc, want in zip(batches, wants):
        assert (want == cc["expect"]).all()
        n = len(want)
        d_sigs = torch.from_numpy(np.ascontiguousarray(cc["sigs_compressed"].reshape(-1))).cuda()
        d_nhms = torch.from_numpy(cc["nhms"].view(np.int64)).cuda()
        d_tabs = torch.from_numpy(np.ascontiguousarray(cc["pk_tables"]).view(np.int64)).cuda()
        d_idx = torch.from_numpy(cc["pk_index"].astype(np.int32)).cuda()
        d_res = torch.full((n,), -99, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        rc = G.verify_compressed_noalloc(d_sigs.data_ptr(), d_nhms.data_ptr(), d_g2.data_ptr(), d_tabs.data_ptr(),
                                         d_idx.data_ptr(), d_res.data_ptr(), n, 8, stream.cuda_stream)
        assert rc == G.BLS_OK, G.last_error()
        torch.cuda.synchronize()
        got = d_res.cpu().numpy()
        assert (got == want).all()
