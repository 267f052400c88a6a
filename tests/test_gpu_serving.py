"""GPU tests of the serving loop (bls_server_*): requests submitted from
several threads while others are on the device are batched together, and each
request's results are identical to verifying it alone and to the expected
accept bits (exact integer results: the tolerance is zero)."""
import threading

import numpy as np
import pytest

import bls_gpu as G
import workload as WL

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool():
    return WL.config_pool(n=1024, nkeys=40, seed=5)


def _ids(ctx, pool):
    return np.array([ctx.register_pk_affine(q) for q in pool["pk_affine"]], dtype=np.int32)


def _requests(pool, nreq, max_size, seed):
    rng = np.random.default_rng(seed)
    n = len(pool["expect"])
    out = []
    for _ in range(nreq):
        s = int(min(max_size, max(1, np.exp(rng.uniform() * np.log(max_size + 1)))))
        idx = (int(rng.integers(n)) + np.arange(s)) % n
        out.append(idx)
    return out


def test_mix_equals_alone_and_expected(pool):
    with G.Context() as ctx:
        ids = _ids(ctx, pool)
        pk_ids = ids[pool["pk_index"]]
        reqs = _requests(pool, 60, 200, seed=1)
        alone = [ctx.verify(pool["sigs"][ix], pool["nhms"][ix], pk_ids[ix]) for ix in reqs]
        with G.Server(ctx, slots=3, max_batch_items=512) as srv:
            tickets = [None] * len(reqs)

            def submit(k0):
                for k in range(k0, len(reqs), 3):
                    ix = reqs[k]
                    tickets[k] = srv.submit(pool["sigs"][ix], pool["nhms"][ix], pk_ids[ix])

            th = [threading.Thread(target=submit, args=(k,)) for k in range(3)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            for k, (ticket, t_sub, res) in enumerate(tickets):
                t_done = srv.wait(ticket, timeout_ms=60000)
                assert t_done >= t_sub
                assert (res == alone[k]).all()
                assert (res == pool["expect"][reqs[k]]).all()
            st = srv.stats()
        assert st["items"] == sum(len(ix) for ix in reqs)
        # requests arriving together were batched: fewer launches than requests
        assert 1 <= st["launches"] < len(reqs)
        assert st["max_batch"] <= 512


def test_compressed_stream_with_invalid():
    cc = WL.config_compressed(256, 40, seed=9, invalid_frac=0.05)
    with G.Context() as ctx:
        ids = np.array([ctx.register_pk_affine(q) for q in cc["pk_affine"]], dtype=np.int32)
        pk_ids = ids[cc["pk_index"]]
        cuts = [0, 1, 40, 41, 130, 256]
        with G.Server(ctx, compressed=True, slots=2, max_batch_items=128) as srv:
            tk = []
            for a, b in zip(cuts, cuts[1:]):
                tk.append((a, b, srv.submit(cc["sigs_compressed"][a:b], cc["nhms"][a:b], pk_ids[a:b])))
            for a, b, (ticket, _, res) in tk:
                srv.wait(ticket, timeout_ms=60000)
                assert (res == cc["expect"][a:b]).all()


def test_admission_and_argument_errors(pool):
    with G.Context() as ctx:
        ids = _ids(ctx, pool)
        # a budget too small for one slot is refused
        with pytest.raises(G.GpuError):
            G.Server(ctx, max_batch_items=4096, mem_cap_bytes=1 << 16)
        with G.Server(ctx, slots=8, max_batch_items=64, mem_cap_bytes=64 * 400 * 2 + 1024) as srv:
            bad = np.full(3, 999, dtype=np.int32)
            with pytest.raises(G.GpuError):
                srv.submit(pool["sigs"][:3], pool["nhms"][:3], bad)
            with pytest.raises(G.GpuError):   # larger than a slot
                n = 65
                srv.submit(pool["sigs"][:n], pool["nhms"][:n], ids[pool["pk_index"][:n]])
            t, _, res = srv.submit(pool["sigs"][:5], pool["nhms"][:5], ids[pool["pk_index"][:5]])
            srv.wait(t, timeout_ms=60000)
            assert (res == pool["expect"][:5]).all()
            with pytest.raises(G.GpuError):   # unknown ticket: times out
                srv.wait(t + 1000, timeout_ms=10)


def _submit_all(srv, pool, pk_ids, reqs, threads=3):
    tickets = [None] * len(reqs)

    def submit(k0):
        for k in range(k0, len(reqs), threads):
            ix = reqs[k]
            tickets[k] = srv.submit(pool["sigs"][ix], pool["nhms"][ix], pk_ids[ix])

    th = [threading.Thread(target=submit, args=(k,)) for k in range(threads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return tickets


@pytest.mark.parametrize("shape", [384, 64], ids=["wide", "five"])
def test_ring_mode_equals_alone(pool, shape):
    """Ring mode: one persistent kernel takes items as they are published; every
    request's results equal verifying it alone, for sizes from 1 upwards and a
    ring smaller than the stream (admission waits for ring space), with both
    block shapes of the kernel."""
    with G.Context(threads_per_block=shape) as ctx:
        ids = _ids(ctx, pool)
        pk_ids = ids[pool["pk_index"]]
        reqs = _requests(pool, 80, 300, seed=3) + [np.array([7]), np.array([8, 9])]
        alone = [ctx.verify(pool["sigs"][ix], pool["nhms"][ix], pk_ids[ix]) for ix in reqs]
        with G.Server(ctx, max_batch_items=512, mode=G.SERVE_RING, ring_items=1000) as srv:
            tickets = _submit_all(srv, pool, pk_ids, reqs)
            for k, (ticket, t_sub, res) in enumerate(tickets):
                t_done = srv.wait(ticket, timeout_ms=60000)
                assert t_done >= t_sub
                assert (res == alone[k]).all()
                assert (res == pool["expect"][reqs[k]]).all()
            st = srv.stats()
        assert st["items"] == sum(len(ix) for ix in reqs)
        assert st["launches"] >= 1


@pytest.mark.parametrize("shape", [384, 64], ids=["wide", "five"])
def test_ring_mode_idle_relaunch(pool, shape):
    """The ring kernel leaves after 20 ms without work; a later request relaunches it."""
    import time
    with G.Context(threads_per_block=shape) as ctx:
        ids = _ids(ctx, pool)
        pk_ids = ids[pool["pk_index"]]
        with G.Server(ctx, max_batch_items=64, mode=G.SERVE_RING) as srv:
            for a in (0, 30, 60):
                t, _, res = srv.submit(pool["sigs"][a:a + 17], pool["nhms"][a:a + 17], pk_ids[a:a + 17])
                srv.wait(t, timeout_ms=60000)
                assert (res == pool["expect"][a:a + 17]).all()
                time.sleep(0.1)
            st = srv.stats()
        assert st["launches"] == 3


@pytest.mark.parametrize("shape", [384, 64], ids=["wide", "five"])
def test_ring_mode_compressed_with_invalid(shape):
    """Ring mode with 48-byte signatures (the certifier's shares): the
    dispatcher decodes each published range on the device before the kernel
    can claim it.  Requests submitted from several threads, with invalid
    encodings of every kind among them, give exactly the results of verifying
    each request alone and the workload's known answers."""
    cc = WL.config_compressed(600, 40, seed=19, invalid_frac=0.05)
    with G.Context(threads_per_block=shape) as ctx:
        ids = ctx.register_pk_affine_batch(cc["pk_affine"])
        pk_ids = ids[cc["pk_index"]]
        comp = cc["sigs_compressed"]
        rng = np.random.default_rng(7)
        cuts = np.unique(np.concatenate([[0, 1, 2, 600], rng.integers(3, 600, 40)]))
        reqs = [np.arange(a, b) for a, b in zip(cuts[:-1], cuts[1:])]
        alone = [ctx.verify(comp[ix].reshape(-1), cc["nhms"][ix], pk_ids[ix], compressed=True) for ix in reqs]
        with G.Server(ctx, compressed=True, max_batch_items=256, mode=G.SERVE_RING, ring_items=400) as srv:
            tickets = [None] * len(reqs)

            def submit(k0):
                for k in range(k0, len(reqs), 3):
                    ix = reqs[k]
                    tickets[k] = srv.submit(comp[ix], cc["nhms"][ix], pk_ids[ix])

            th = [threading.Thread(target=submit, args=(k,)) for k in range(3)]
            for t in th:
                t.start()
            for t in th:
                t.join()
            for k, (ticket, _, res) in enumerate(tickets):
                srv.wait(ticket, timeout_ms=60000)
                assert (res == alone[k]).all()
                assert (res == cc["expect"][reqs[k]]).all()
    assert (cc["expect"] < 0).sum() == 30
