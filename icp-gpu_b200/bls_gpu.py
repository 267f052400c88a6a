"""Python host binding of libbls_gpu.so (ctypes over the C ABI in include/bls_gpu.h).

It mirrors the reference's Rust FFI crate (gpu-crypto/src/lib.rs,
ic-integration/gpu_crypto/lib.rs): `init`, `batch_bls_verify`, `bls_verify`,
`g1_decompress_batch`, with the same argument meaning and error behaviour
(an error return from the library raises `GpuError`, the Rust crate's `Err`).
`Context` wraps the extended API: device-resident public-key tables,
compressed signatures with per-item decode status, and Miller / Gt values.

There is no CPU path here.  If the shared library is missing or cannot load,
every call raises; nothing falls back to a CPU implementation.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbls_gpu.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "bls_gpu.h")

G2_COEFF_U64S = 68 * 36     # 2448, gpu-crypto/src/lib.rs:29
G1_U64S = 12                # gpu-crypto/src/lib.rs:30

BLS_OK = 0
BLS_ERR_NODEV = -1
BLS_ERR_INVALID = -2
BLS_ERR_CUDA = -3
BLS_ERR_NOMEM = -4
BLS_ERR_TIMEOUT = -5
BLS_ERR_FULL = -6

BLS_ACCEPT = 1
BLS_REJECT = 0
ST_OK, ST_BAD_FLAGS, ST_X_NOT_CANONICAL, ST_NOT_ON_CURVE, ST_NOT_IN_SUBGROUP = 0, 1, 2, 3, 4
SIG_AFFINE, SIG_COMPRESSED = 0, 1


class GpuError(RuntimeError):
    def __init__(self, msg, status=None):
        super().__init__(msg)
        self.status = status   # per-item decode status of a failed registration


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_batch", ctypes.c_int), ("max_pks", ctypes.c_int),
                ("mem_cap_bytes", ctypes.c_size_t), ("threads_per_block", ctypes.c_int),
                ("blocks_per_sm", ctypes.c_int), ("lanes_per_pairing", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("sigs", ctypes.c_void_p), ("neg_hms", ctypes.c_void_p),
                ("pk_ids", ctypes.c_void_p), ("results", ctypes.c_void_p)]


class TunePoint(ctypes.Structure):
    _fields_ = [("lanes_per_pairing", ctypes.c_int), ("threads_per_block", ctypes.c_int),
                ("blocks_per_sm", ctypes.c_int), ("ms", ctypes.c_float)]


MODE_PLAIN, MODE_PERSISTENT = 0, 1


class ServerConfig(ctypes.Structure):
    _fields_ = [("sig_format", ctypes.c_int), ("slots", ctypes.c_int), ("max_batch_items", ctypes.c_int),
                ("mem_cap_bytes", ctypes.c_size_t), ("mode", ctypes.c_int), ("ring_items", ctypes.c_int),
                ("ring_blocks_per_sm", ctypes.c_int), ("ring_blocks", ctypes.c_int)]


SERVE_SLOTS = 0
SERVE_RING = 1


class Batch(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("sig_format", ctypes.c_int), ("sigs", ctypes.c_void_p),
                ("neg_hms", ctypes.c_void_p), ("pk_ids", ctypes.c_void_p),
                ("miller_out", ctypes.c_void_p), ("gt_out", ctypes.c_void_p)]


_lib = None


def lib():
    """Load libbls_gpu.so (raises if it is absent: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GpuError("libbls_gpu.so not built (run `make -C icp-gpu_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        P, I = ctypes.c_void_p, ctypes.c_int
        L.gpu_crypto_init.restype = I
        L.gpu_batch_bls_verify.argtypes = [P, P, P, P, P, I]
        L.gpu_batch_sha256.argtypes = [P, P, I, I]
        L.gpu_g1_decompress_batch.argtypes = [P, P, I]
        L.gpu_g1_decompress.argtypes = [P, P]
        L.gpu_msm_g1.argtypes = [P, P, ctypes.c_size_t, P]
        L.gpu_jacobian_to_affine.argtypes = [P, P]
        L.bls_ref_cache_stats.argtypes = [P, P, P]
        L.bls_config_default.argtypes = [ctypes.POINTER(Config), I]
        L.bls_config_default.restype = None
        L.bls_ctx_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(P)]
        L.bls_ctx_destroy.argtypes = [P]
        L.bls_ctx_destroy.restype = None
        L.bls_last_error.restype = ctypes.c_char_p
        L.bls_pk_register_coeffs.argtypes = [P, P, I, ctypes.POINTER(ctypes.c_int32)]
        L.bls_pk_register_affine.argtypes = [P, P, ctypes.POINTER(ctypes.c_int32)]
        L.bls_pk_register_compressed.argtypes = [P, P, I, P, P]
        L.bls_pk_register_affine_batch.argtypes = [P, P, I, P]
        L.bls_g2_decompress_status.argtypes = [P, P, I, P, P]
        L.bls_pk_table.argtypes = [P, ctypes.c_int32, P]
        L.bls_verify_batch.argtypes = [P, ctypes.POINTER(Batch), P]
        L.bls_verify_batch_device.argtypes = [P, ctypes.POINTER(Batch), P]
        L.bls_ctx_sync.argtypes = [P]
        L.bls_ctx_stream.argtypes = [P]
        L.bls_ctx_stream.restype = P
        L.bls_g1_decompress_status.argtypes = [P, P, I, P, P]
        L.bls_neg_hash_to_g1.argtypes = [P, P, P, I, P, I, P]
        L.bls_imad_chain_rate.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
        L.bls_imad_pipe_rates.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.bls_limb_layout_rates.argtypes = [P, ctypes.POINTER(ctypes.c_double), I]
        L.bls_verify_batch_rlc.argtypes = [P, ctypes.POINTER(Batch), P, P, ctypes.POINTER(I), P]
        L.bls_verify_messages.argtypes = [P, I, P, P, P, P, I, P, I, P]
        L.bls_verify_requests.argtypes = [P, ctypes.POINTER(Request), I, I, I]
        L.bls_verify_compressed_noalloc.argtypes = [P, P, P, P, P, I, P, P, I, I, P]
        L.bls_server_create.argtypes = [P, ctypes.POINTER(ServerConfig), ctypes.POINTER(P)]
        L.bls_server_destroy.argtypes = [P]
        L.bls_server_destroy.restype = None
        L.bls_server_submit.argtypes = [P, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.c_int64)]
        L.bls_server_wait.argtypes = [P, ctypes.c_uint64, I, ctypes.POINTER(ctypes.c_int64)]
        L.bls_server_stats.argtypes = [P] + [ctypes.POINTER(ctypes.c_uint64)] * 3
        L.bls_autotune.argtypes = [P, ctypes.POINTER(Batch), I, ctypes.POINTER(TunePoint), I, ctypes.POINTER(I)]
        _lib = L
    return _lib


def pack_messages(msgs):
    """Messages back to back (uint8) and their n + 1 byte offsets (uint32)."""
    off = np.zeros(len(msgs) + 1, dtype=np.uint32)
    off[1:] = np.cumsum([len(m) for m in msgs], dtype=np.uint64).astype(np.uint32)
    buf = np.frombuffer(b"".join(bytes(m) for m in msgs) or b"\0", dtype=np.uint8).copy()
    return buf, off


def last_error():
    return lib().bls_last_error().decode()


def _u64(a, shape_last=None):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    if shape_last is not None:
        a = a.reshape(-1, shape_last)
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data


# ----------------------------------------------------------------------------
# the reference crate's API (gpu-crypto/src/lib.rs)
# ----------------------------------------------------------------------------

def init():
    """gpu-crypto/src/lib.rs:36-39: Ok when a CUDA device is present."""
    if lib().gpu_crypto_init() != 0:
        raise GpuError("No CUDA GPU found")


def batch_bls_verify(sigs, neg_hm_points, g2_prepared, pk_prepared):
    """gpu-crypto/src/lib.rs:82-125.  sigs, neg_hm_points: (M, 12) u64 affine
    Montgomery; g2_prepared: (2448,) u64; pk_prepared: (M, 2448) u64.
    Returns a list of M bools; raises GpuError when the kernel call fails."""
    sigs = _u64(sigs, G1_U64S)
    nhms = _u64(neg_hm_points, G1_U64S)
    g2 = _u64(g2_prepared).reshape(-1)
    pk = _u64(pk_prepared, G2_COEFF_U64S)
    m = sigs.shape[0]
    assert nhms.shape[0] == m and pk.shape[0] == m and g2.size == G2_COEFF_U64S
    if m == 0:
        return []
    res = np.zeros(m, dtype=np.int32)
    ret = lib().gpu_batch_bls_verify(_ptr(sigs), _ptr(nhms), _ptr(g2), _ptr(pk), _ptr(res), m)
    if ret != 0:
        raise GpuError("GPU kernel failed: " + last_error())
    return (res == 1).tolist()


def ref_cache_stats():
    """The reference entry point's table cache: (resident tables, capacity,
    times it was emptied to make room)."""
    res, cap, fl = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_uint64(0)
    if lib().bls_ref_cache_stats(ctypes.byref(res), ctypes.byref(cap), ctypes.byref(fl)) != 0:
        raise GpuError("bls_ref_cache_stats failed: " + last_error())
    return res.value, cap.value, fl.value


def bls_verify(sig, neg_hm, g2_prepared, pk_prepared):
    """gpu-crypto/src/lib.rs:129-148 without its CPU fallback: raises instead."""
    return batch_bls_verify(_u64(sig, 12), _u64(neg_hm, 12), g2_prepared, _u64(pk_prepared, G2_COEFF_U64S))[0]


def g1_decompress_batch(compressed_points):
    """ic-integration/gpu_crypto/lib.rs:189-223: bytes of n x 48 -> (n, 12) u64."""
    b = bytes(compressed_points)
    if len(b) % 48 != 0:
        raise GpuError("Input must be multiple of 48 bytes")
    n = len(b) // 48
    if n == 0:
        return np.zeros((0, 12), dtype=np.uint64)
    src = np.frombuffer(b, dtype=np.uint8)
    out = np.zeros((n, 12), dtype=np.uint64)
    if lib().gpu_g1_decompress_batch(_ptr(src), _ptr(out), n) != 0:
        raise GpuError("GPU decompression failed: " + last_error())
    return out


# ----------------------------------------------------------------------------
# extended API
# ----------------------------------------------------------------------------

NOALLOC_MAX_ITEMS = 8192


def verify_compressed_noalloc(sigs48_ptr, nhms_ptr, g2_ptr, pk_tables_ptr, pk_identity_ptr, n_tables, pk_index_ptr,
                              results_ptr, n, lanes=6, stream=None):
    """Enqueue a verify of n compressed signatures on `stream` using only
    caller-owned device buffers (raw device pointers; pk_identity_ptr may be
    None); the library allocates nothing.  Returns the library status code
    (0 = enqueued)."""
    return lib().bls_verify_compressed_noalloc(sigs48_ptr, nhms_ptr, g2_ptr, pk_tables_ptr, pk_identity_ptr,
                                               n_tables, pk_index_ptr, results_ptr, n, lanes, stream)


class Context:
    """A device context: stream, buffers and resident public-key tables."""

    def __init__(self, device=0, max_batch=0, max_pks=0, mem_cap_bytes=0, lanes=0, blocks_per_sm=0,
                 threads_per_block=0):
        L = lib()
        cfg = Config()
        L.bls_config_default(ctypes.byref(cfg), device)
        if max_batch:
            cfg.max_batch = max_batch
        if max_pks:
            cfg.max_pks = max_pks
        cfg.mem_cap_bytes = mem_cap_bytes
        cfg.lanes_per_pairing = lanes
        cfg.blocks_per_sm = blocks_per_sm
        cfg.threads_per_block = threads_per_block
        h = ctypes.c_void_p()
        rc = L.bls_ctx_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != BLS_OK:
            raise GpuError("bls_ctx_create failed (%d): %s" % (rc, last_error()))
        self.h = h
        self.lib = L

    def close(self):
        if self.h:
            self.lib.bls_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != BLS_OK:
            raise GpuError("%s failed (%d): %s" % (what, rc, last_error()))

    def register_pk_coeffs(self, coeffs, is_identity=False):
        c = _u64(coeffs).reshape(-1)
        assert c.size == G2_COEFF_U64S
        pid = ctypes.c_int32()
        self._check(self.lib.bls_pk_register_coeffs(self.h, _ptr(c), int(is_identity), ctypes.byref(pid)),
                    "bls_pk_register_coeffs")
        return pid.value

    def register_pk_affine(self, q24):
        q = _u64(q24).reshape(-1)
        assert q.size == 24
        pid = ctypes.c_int32()
        self._check(self.lib.bls_pk_register_affine(self.h, _ptr(q), ctypes.byref(pid)), "bls_pk_register_affine")
        return pid.value

    def register_pk_affine_batch(self, q24s):
        """Register n affine keys ((n, 24) u64) in one call; returns their ids."""
        q = _u64(q24s).reshape(-1, 24)
        ids = np.full(q.shape[0], -1, dtype=np.int32)
        self._check(self.lib.bls_pk_register_affine_batch(self.h, _ptr(q), q.shape[0], _ptr(ids)),
                    "bls_pk_register_affine_batch")
        return ids

    def register_pk_compressed(self, pks96):
        """Decode, validate and prepare n 96-byte keys on the GPU.  Returns
        (ids, status); raises GpuError (registering none) when a key fails."""
        src = np.ascontiguousarray(np.frombuffer(bytes(pks96), dtype=np.uint8))
        assert src.size % 96 == 0
        n = src.size // 96
        ids = np.full(n, -1, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rc = self.lib.bls_pk_register_compressed(self.h, _ptr(src), n, _ptr(ids), _ptr(st))
        if rc != BLS_OK:
            raise GpuError("bls_pk_register_compressed failed (%d): %s" % (rc, last_error()), status=st)
        return ids, st

    def g2_decompress(self, compressed):
        """(status (n,) int32, q (n, 24) u64: x.c0, x.c1, y.c0, y.c1 Montgomery)."""
        src = np.ascontiguousarray(np.frombuffer(bytes(compressed), dtype=np.uint8))
        assert src.size % 96 == 0
        n = src.size // 96
        q = np.zeros((n, 24), dtype=np.uint64)
        st = np.zeros(n, dtype=np.int32)
        self._check(self.lib.bls_g2_decompress_status(self.h, _ptr(src), n, _ptr(q), _ptr(st)),
                    "bls_g2_decompress_status")
        return st, q

    def pk_table(self, pk_id):
        out = np.zeros(G2_COEFF_U64S, dtype=np.uint64)
        self._check(self.lib.bls_pk_table(self.h, pk_id, _ptr(out)), "bls_pk_table")
        return out

    def verify(self, sigs, neg_hms, pk_ids, compressed=False, want_values=False):
        """results (n,) int32: 1 accept, 0 reject, -status for a decode failure;
        with want_values also the Miller-loop and Gt values, (n, 72) u64 each."""
        nhms = _u64(neg_hms, 12)
        n = nhms.shape[0]
        if compressed:
            s = np.ascontiguousarray(np.frombuffer(bytes(sigs), dtype=np.uint8) if not isinstance(sigs, np.ndarray)
                                     else sigs, dtype=np.uint8).reshape(-1)
            assert s.size == 48 * n
        else:
            s = _u64(sigs, 12)
            assert s.shape[0] == n
        ids = np.ascontiguousarray(pk_ids, dtype=np.int32).reshape(-1)
        assert ids.size == n
        res = np.zeros(n, dtype=np.int32)
        ml = np.zeros((n, 72), dtype=np.uint64) if want_values else None
        gt = np.zeros((n, 72), dtype=np.uint64) if want_values else None
        b = Batch(n, SIG_COMPRESSED if compressed else SIG_AFFINE, _ptr(s), _ptr(nhms), _ptr(ids), _ptr(ml), _ptr(gt))
        self._check(self.lib.bls_verify_batch(self.h, ctypes.byref(b), _ptr(res)), "bls_verify_batch")
        return (res, ml, gt) if want_values else res

    def verify_rlc(self, sigs, neg_hms, pk_ids, compressed=False, scalars=None, want_agg=False):
        """Random-linear-combination batch verification: (results, combined[, agg])."""
        nhms = _u64(neg_hms, 12)
        n = nhms.shape[0]
        if compressed:
            s = np.ascontiguousarray(np.frombuffer(bytes(sigs), dtype=np.uint8) if not isinstance(sigs, np.ndarray)
                                     else sigs, dtype=np.uint8).reshape(-1)
            assert s.size == 48 * n
        else:
            s = _u64(sigs, 12)
            assert s.shape[0] == n
        ids = np.ascontiguousarray(pk_ids, dtype=np.int32).reshape(-1)
        assert ids.size == n
        r = None if scalars is None else np.ascontiguousarray(scalars, dtype=np.uint64).reshape(-1)
        res = np.zeros(n, dtype=np.int32)
        comb = ctypes.c_int(0)
        agg = np.zeros((1 + len(set(ids.tolist())), 12), dtype=np.uint64) if want_agg else None
        b = Batch(n, SIG_COMPRESSED if compressed else SIG_AFFINE, _ptr(s), _ptr(nhms), _ptr(ids), None, None)
        self._check(self.lib.bls_verify_batch_rlc(self.h, ctypes.byref(b), _ptr(r), _ptr(res), ctypes.byref(comb),
                                                  _ptr(agg)), "bls_verify_batch_rlc")
        return (res, comb.value, agg) if want_agg else (res, comb.value)

    def verify_device(self, n, sigs_ptr, nhms_ptr, ids_ptr, res_ptr, compressed=False, ml_ptr=None, gt_ptr=None):
        """Enqueue a verify on device-resident arrays (raw device pointers)."""
        b = Batch(n, SIG_COMPRESSED if compressed else SIG_AFFINE, sigs_ptr, nhms_ptr, ids_ptr, ml_ptr, gt_ptr)
        self._check(self.lib.bls_verify_batch_device(self.h, ctypes.byref(b), res_ptr), "bls_verify_batch_device")

    def sync(self):
        self._check(self.lib.bls_ctx_sync(self.h), "bls_ctx_sync")

    def stream(self):
        return self.lib.bls_ctx_stream(self.h)

    def neg_hash_to_g1(self, msgs, dst):
        """-H(m) for each message (RFC 9380 hash_to_curve, SSWU suite) on the GPU: (n, 12) u64."""
        buf, off = pack_messages(msgs)
        d = np.frombuffer(bytes(dst), dtype=np.uint8).copy()
        out = np.zeros((len(msgs), 12), dtype=np.uint64)
        self._check(self.lib.bls_neg_hash_to_g1(self.h, _ptr(buf), _ptr(off), len(msgs), _ptr(d) if d.size else None,
                                                d.size, _ptr(out)), "bls_neg_hash_to_g1")
        return out

    def verify_messages(self, sigs, msgs, pk_ids, dst, compressed=False):
        """results (n,) int32 as verify(), with -H(m_i) computed on the GPU from the message bytes."""
        n = len(msgs)
        if compressed:
            s = np.ascontiguousarray(np.frombuffer(bytes(sigs), dtype=np.uint8) if not isinstance(sigs, np.ndarray)
                                     else sigs, dtype=np.uint8).reshape(-1)
            assert s.size == 48 * n
        else:
            s = _u64(sigs, 12)
            assert s.shape[0] == n
        buf, off = pack_messages(msgs)
        d = np.frombuffer(bytes(dst), dtype=np.uint8).copy()
        ids = np.ascontiguousarray(pk_ids, dtype=np.int32).reshape(-1)
        assert ids.size == n
        res = np.zeros(n, dtype=np.int32)
        self._check(self.lib.bls_verify_messages(self.h, SIG_COMPRESSED if compressed else SIG_AFFINE, _ptr(s),
                                                 _ptr(buf), _ptr(off), _ptr(ids), n, _ptr(d) if d.size else None,
                                                 d.size, _ptr(res)), "bls_verify_messages")
        return res

    def imad_chain_rate(self):
        """IMAD-pipe instructions/s of the carry-chain product loop (bls_imad_chain_rate)."""
        v = ctypes.c_double(0.0)
        self._check(self.lib.bls_imad_chain_rate(self.h, ctypes.byref(v)), "bls_imad_chain_rate")
        return v.value

    def imad_pipe_rates(self):
        """(mul.lo, mul.hi) thread instructions per second on the whole device (bls_imad_pipe_rates)."""
        lo, hi = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._check(self.lib.bls_imad_pipe_rates(self.h, ctypes.byref(lo), ctypes.byref(hi)), "bls_imad_pipe_rates")
        return lo.value, hi.value

    def limb_layout_rates(self):
        """Products/s of the three limb layouts in the verify kernel's setting
        (bls_limb_layout_rates): [12 x 32-bit Karatsuba carry chains,
        15 x 26-bit signed wide columns, 14 x 28-bit wide columns]."""
        v = (ctypes.c_double * 3)()
        self._check(self.lib.bls_limb_layout_rates(self.h, v, 3), "bls_limb_layout_rates")
        return list(v)

    def g1_decompress(self, compressed):
        src = np.ascontiguousarray(np.frombuffer(bytes(compressed), dtype=np.uint8))
        n = src.size // 48
        xy = np.zeros((n, 12), dtype=np.uint64)
        st = np.zeros(n, dtype=np.int32)
        self._check(self.lib.bls_g1_decompress_status(self.h, _ptr(src), n, _ptr(xy), _ptr(st)),
                    "bls_g1_decompress_status")
        return st, xy

    def verify_requests(self, requests, compressed=False, mode=MODE_PERSISTENT):
        """requests: list of (sigs, neg_hms, pk_ids); returns a list of int32
        result arrays.  MODE_PLAIN launches once per request; MODE_PERSISTENT
        runs all of them in one graph-replayed persistent launch."""
        keep, reqs, outs = [], [], []
        for sigs, nhms, ids in requests:
            nhms = _u64(nhms, 12)
            n = nhms.shape[0]
            s = (np.ascontiguousarray(sigs, dtype=np.uint8).reshape(-1) if compressed else _u64(sigs, 12))
            ids = np.ascontiguousarray(ids, dtype=np.int32).reshape(-1)
            res = np.zeros(n, dtype=np.int32)
            keep += [s, nhms, ids]
            outs.append(res)
            reqs.append(Request(n, _ptr(s), _ptr(nhms), _ptr(ids), _ptr(res)))
        arr = (Request * max(1, len(reqs)))(*reqs)
        self._check(self.lib.bls_verify_requests(self.h, arr, len(reqs), SIG_COMPRESSED if compressed else SIG_AFFINE,
                                                 mode), "bls_verify_requests")
        return outs

    def autotune(self, n, sigs_ptr, nhms_ptr, ids_ptr, compressed=False, repeats=3):
        """Time every kernel configuration on a device-resident sample and keep
        the fastest; returns [(lanes, threads_per_block, blocks_per_sm, ms), ...]."""
        b = Batch(n, SIG_COMPRESSED if compressed else SIG_AFFINE, sigs_ptr, nhms_ptr, ids_ptr, None, None)
        pts = (TunePoint * 32)()
        npts = ctypes.c_int()
        self._check(self.lib.bls_autotune(self.h, ctypes.byref(b), repeats, pts, 32, ctypes.byref(npts)),
                    "bls_autotune")
        return [(pts[i].lanes_per_pairing, pts[i].threads_per_block, pts[i].blocks_per_sm, pts[i].ms)
                for i in range(npts.value)]


class Server:
    """Continuous-batching verify server on a Context (bls_server_*)."""

    def __init__(self, ctx, compressed=False, slots=0, max_batch_items=0, mem_cap_bytes=0, mode=SERVE_SLOTS,
                 ring_items=0, ring_blocks_per_sm=0, ring_blocks=0):
        cfg = ServerConfig(SIG_COMPRESSED if compressed else SIG_AFFINE, slots, max_batch_items, mem_cap_bytes, mode,
                           ring_items, ring_blocks_per_sm, ring_blocks)
        h = ctypes.c_void_p()
        rc = ctx.lib.bls_server_create(ctx.h, ctypes.byref(cfg), ctypes.byref(h))
        if rc != BLS_OK:
            raise GpuError("bls_server_create failed (%d)" % rc)
        self.h, self.lib, self.compressed = h, ctx.lib, compressed
        self._keep = {}

    def submit(self, sigs, nhms, ids):
        """Queue a request; returns (ticket, submit_ns, results array filled on completion)."""
        nhms = _u64(nhms, 12)
        n = nhms.shape[0]
        s = np.ascontiguousarray(sigs, dtype=np.uint8).reshape(-1) if self.compressed else _u64(sigs, 12)
        ids = np.ascontiguousarray(ids, dtype=np.int32).reshape(-1)
        res = np.zeros(n, dtype=np.int32)
        req = Request(n, _ptr(s), _ptr(nhms), _ptr(ids), _ptr(res))
        t = ctypes.c_uint64()
        ns = ctypes.c_int64()
        rc = self.lib.bls_server_submit(self.h, ctypes.byref(req), ctypes.byref(t), ctypes.byref(ns))
        if rc != BLS_OK:
            raise GpuError("bls_server_submit failed (%d)" % rc)
        self._keep[t.value] = res
        return t.value, ns.value, res

    def wait(self, ticket, timeout_ms=-1):
        """Block until the ticket completes; returns its completion time (ns)."""
        ns = ctypes.c_int64()
        rc = self.lib.bls_server_wait(self.h, ticket, timeout_ms, ctypes.byref(ns))
        if rc != BLS_OK:
            raise GpuError("bls_server_wait failed (%d)" % rc)
        self._keep.pop(ticket, None)
        return ns.value

    def stats(self):
        v = [ctypes.c_uint64() for _ in range(3)]
        self.lib.bls_server_stats(self.h, *[ctypes.byref(x) for x in v])
        return {"launches": v[0].value, "items": v[1].value, "max_batch": v[2].value}

    def close(self):
        if self.h:
            self.lib.bls_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
