"""Key ids that name no registered table, given where the host cannot check
them: device-resident batches (bls_verify_batch_device) and the autotuner's
device sample.  Every verify kernel reads the key's line table by its id, so
each one checks the id against the context's table count first: an item with
an id outside [0, keys) reads no table and gets -BLS_ST_BAD_KEY_INDEX, a
compressed signature that failed to decode keeps its own decode status, and
every other item's result is unchanged.  Bad ids are negative, equal to the
table count, and the largest int32."""
import numpy as np
import pytest

import bls_gpu as G
import workload as WL

pytestmark = pytest.mark.gpu

BAD_KEY_INDEX = 5


@pytest.fixture(scope="module")
def wl():
    return WL.config_compressed(256, 8, seed=11, invalid_frac=0.05)


def _bad_ids(ids, nkeys):
    ids = ids.copy()
    bad = np.zeros(len(ids), dtype=bool)
    for k, v in ((3, -1), (17, nkeys), (40, 2**31 - 1), (41, nkeys + 5), (200, -(2**31))):
        ids[k] = v
        bad[k] = True
    return ids, bad


def _device_verify(ctx, sigs, nhms, ids, compressed):
    import torch
    dev = torch.device("cuda", 0)
    d_s = torch.from_numpy(np.ascontiguousarray(sigs).reshape(-1).view(np.uint8)).to(dev)
    d_h = torch.from_numpy(np.ascontiguousarray(nhms).view(np.int64)).to(dev)
    d_i = torch.from_numpy(np.ascontiguousarray(ids, dtype=np.int32)).to(dev)
    d_r = torch.zeros(len(ids), dtype=torch.int32, device=dev)
    ctx.verify_device(len(ids), d_s.data_ptr(), d_h.data_ptr(), d_i.data_ptr(), d_r.data_ptr(),
                      compressed=compressed)
    ctx.sync()
    return d_r.cpu().numpy()


@pytest.mark.parametrize("lanes,tpb", [(6, 384), (6, 64), (8, 0), (4, 0), (1, 0)])
@pytest.mark.parametrize("compressed", [False, True])
def test_device_batch_with_unknown_key_ids(wl, lanes, tpb, compressed):
    with G.Context(lanes=lanes, threads_per_block=tpb) as ctx:
        reg = np.asarray(ctx.register_pk_affine_batch(wl["pk_affine"]), dtype=np.int32)
        good_ids = reg[wl["pk_index"]]
        ids, bad = _bad_ids(good_ids, len(reg))
        expect = wl["expect"]
        if compressed:
            sigs, nhms, sel = wl["sigs_compressed"], wl["nhms"], np.arange(len(expect))
        else:
            sel = np.nonzero(expect >= 0)[0]      # affine inputs: the decodable items only
            sigs, nhms = wl["sigs"][sel], wl["nhms"][sel]
        # a bad id gives -5 unless the signature already failed to decode
        want = np.where(bad & (expect >= 0), -BAD_KEY_INDEX, expect)[sel]
        got = _device_verify(ctx, sigs, nhms, ids[sel], compressed)
        assert (got == want).all(), np.nonzero(got != want)
        assert (want == -BAD_KEY_INDEX).sum() >= 3
        # the same context then verifies the batch with its real ids exactly
        again = _device_verify(ctx, sigs, nhms, good_ids[sel], compressed)
        assert (again == expect[sel]).all()
