"""Seeded synthetic verify workloads (the five bench configurations).

The reference benchmarks one repeated test vector (cuda/bench_bls_verify.cu:
122-247); these workloads instead draw fresh keys, messages and signatures
from a seed, with known expected results, standing in for the IC replica's
traffic.  Keys, hashes, signatures, encodings and line tables come from
libbls_workload.so (C++, host CPU): the caller's side of the verify path.

Definitions (one SplitMix64 stream per config seed):
  scalar   4 draws -> 255-bit little-endian integer, rejected unless in [1, r)
  message  4 draws -> 32 bytes (little-endian words)
  H(m)     RFC 9380 hash_to_curve to G1, suite BLS12381G1_XMD:SHA-256_SSWU_RO_
           (ic_bls12_381's): SHA-256 expander, DST below, simplified SWU map
           on the 11-isogenous curve, isogeny to E
  sig      sk * H(m);  the verifier receives -H(m') for the message it checks
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
DST = b"BLS_BENCH_G1_XMD:SHA-256_SSWU_RO_"
R_ORDER = 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001
P_MOD = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
M64 = (1 << 64) - 1

# decode statuses (include/bls_gpu.h)
ST_BAD_FLAGS, ST_X_NOT_CANONICAL, ST_NOT_ON_CURVE, ST_NOT_IN_SUBGROUP = 1, 2, 3, 4

_wl = None


def wl():
    global _wl
    if _wl is None:
        path = os.path.join(_HERE, "libbls_workload.so")
        if not os.path.exists(path):
            raise RuntimeError("libbls_workload.so not built (run `make -C icp-gpu_b200`)")
        L = ctypes.CDLL(path)
        P, I = ctypes.c_void_p, ctypes.c_int
        L.wl_num_threads.restype = I
        L.wl_sha256.argtypes = [P, ctypes.c_size_t, P]
        L.wl_expand_message_xmd.argtypes = [P, ctypes.c_size_t, P, ctypes.c_size_t, P, ctypes.c_size_t]
        L.wl_hash_to_g1.argtypes = [P, I, I, P, I, P, I]
        L.wl_g1_mul.argtypes = [P, P, I, P, I]
        L.wl_g1_neg.argtypes = [P, I, P]
        L.wl_g2_mul_gen.argtypes = [P, I, P, I]
        L.wl_g2_prepare.argtypes = [P, I, P, I]
        L.wl_g1_compress.argtypes = [P, I, P]
        L.wl_g2_compress.argtypes = [P, I, P]
        L.wl_special_points.argtypes = [ctypes.c_uint64, I, I, P]
        _wl = L
    return _wl


def _p(a):
    return a.ctypes.data


def nthreads():
    return max(1, wl().wl_num_threads())


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & M64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def scalar(self):
        while True:
            v = 0
            for i in range(4):
                v |= self.next() << (64 * i)
            v &= (1 << 255) - 1
            if 0 < v < R_ORDER:
                return v

    def msg(self):
        return b"".join(self.next().to_bytes(8, "little") for _ in range(4))

    def below(self, n):
        return self.next() % n

    def uniform(self):
        return (self.next() >> 11) / float(1 << 53)


def scalar_limbs(k):
    return [(k >> (64 * i)) & M64 for i in range(4)]


# ---------------------------------------------------------------- primitives

def hash_to_g1(msgs, msg_len=32):
    msgs = np.ascontiguousarray(np.frombuffer(b"".join(msgs), dtype=np.uint8))
    n = msgs.size // msg_len
    out = np.zeros((n, 12), dtype=np.uint64)
    dst = np.frombuffer(DST, dtype=np.uint8)
    wl().wl_hash_to_g1(_p(msgs), msg_len, n, _p(dst), len(DST), _p(out), nthreads())
    return out


def g1_mul(points, scalars):
    points = np.ascontiguousarray(points, dtype=np.uint64)
    sc = np.ascontiguousarray(scalars, dtype=np.uint64)
    out = np.zeros_like(points)
    wl().wl_g1_mul(_p(points), _p(sc), points.shape[0], _p(out), nthreads())
    return out


def g1_neg(points):
    points = np.ascontiguousarray(points, dtype=np.uint64)
    out = np.zeros_like(points)
    wl().wl_g1_neg(_p(points), points.shape[0], _p(out))
    return out


def g1_compress(points):
    points = np.ascontiguousarray(points, dtype=np.uint64)
    out = np.zeros((points.shape[0], 48), dtype=np.uint8)
    wl().wl_g1_compress(_p(points), points.shape[0], _p(out))
    return out


def g2_mul_gen(scalars):
    sc = np.ascontiguousarray(scalars, dtype=np.uint64)
    out = np.zeros((sc.shape[0], 24), dtype=np.uint64)
    wl().wl_g2_mul_gen(_p(sc), sc.shape[0], _p(out), nthreads())
    return out


def g2_compress(q):
    q = np.ascontiguousarray(q, dtype=np.uint64)
    out = np.zeros((q.shape[0], 96), dtype=np.uint8)
    wl().wl_g2_compress(_p(q), q.shape[0], _p(out))
    return out


def g2_prepare(q):
    q = np.ascontiguousarray(q, dtype=np.uint64)
    out = np.zeros((q.shape[0], 2448), dtype=np.uint64)
    wl().wl_g2_prepare(_p(q), q.shape[0], _p(out), nthreads())
    return out


def special_points(seed, n, mode):
    out = np.zeros((n, 48), dtype=np.uint8)
    wl().wl_special_points(seed & M64, n, mode, _p(out))
    return out


# ---------------------------------------------------------------- configs

def _keys(rng, nkeys, with_tables=True):
    sks = [rng.scalar() for _ in range(nkeys)]
    sk_limbs = np.array([scalar_limbs(k) for k in sks], dtype=np.uint64)
    pk_aff = g2_mul_gen(sk_limbs)
    keys = {"sk": sk_limbs, "pk_affine": pk_aff, "pk_compressed": g2_compress(pk_aff)}
    if with_tables:
        keys["pk_tables"] = g2_prepare(pk_aff)
    return keys


def _items(rng, keys, key_of_item, corrupt):
    """Sign one fresh message per item with key_of_item[i]; corrupt[i] in
    {0: none, 1: message flip, 2: wrong key}.  Returns sigs, -H(m'), the pk
    index each item is verified against, and the expected accept bit."""
    n = len(key_of_item)
    nkeys = keys["sk"].shape[0]
    msgs, checked, pk_index, expect = [], [], np.array(key_of_item, dtype=np.int32), np.ones(n, dtype=np.int32)
    for i in range(n):
        m = rng.msg()
        msgs.append(m)
        if corrupt[i] == 1:
            b = bytearray(m)
            b[rng.below(32)] ^= 1 << rng.below(8)
            checked.append(bytes(b))
            expect[i] = 0
        else:
            checked.append(m)
            if corrupt[i] == 2 and nkeys > 1:
                pk_index[i] = (key_of_item[i] + 1 + rng.below(nkeys - 1)) % nkeys
                expect[i] = 0
    h_signed = hash_to_g1(msgs)
    sigs = g1_mul(h_signed, keys["sk"][np.array(key_of_item, dtype=np.int64)])
    flip = np.array([corrupt[i] == 1 for i in range(n)])
    h_checked = h_signed.copy()
    if flip.any():
        h_checked[flip] = hash_to_g1([checked[i] for i in range(n) if flip[i]])
    return {"sigs": sigs, "nhms": g1_neg(h_checked), "pk_index": pk_index, "expect": expect, "msgs": checked}


def config_plain(n=64, seed=1):
    """Plain workload: n keys, one signature each, every 8th message bit-flipped."""
    rng = SplitMix64(seed)
    keys = _keys(rng, n)
    corrupt = [1 if i % 8 == 7 else 0 for i in range(n)]
    it = _items(rng, keys, list(range(n)), corrupt)
    return {**keys, **it, "name": "plain-%d" % n}


def _split_corruption(n):
    # 1 in 8 corrupted, alternating message flip and wrong key
    return [0 if i % 8 != 7 else (1 if (i // 8) % 2 == 0 else 2) for i in range(n)]


def config_keyset(n=4096, nkeys=40, seed=2):
    """Key-set workload: n verifications over nkeys resident keys (key i % nkeys)."""
    rng = SplitMix64(seed)
    keys = _keys(rng, nkeys)
    it = _items(rng, keys, [i % nkeys for i in range(n)], _split_corruption(n))
    return {**keys, **it, "name": "keyset-%d-%d" % (n, nkeys)}


def config_compressed(n=65536, nkeys=40, seed=3, invalid_frac=0.02):
    """Compressed workload: n compressed signatures; invalid_frac of them are invalid
    encodings, the reason per index known: bad flags (three kinds), x >= p, x
    off the curve, a curve point outside the subgroup."""
    rng = SplitMix64(seed)
    keys = _keys(rng, nkeys)
    it = _items(rng, keys, [i % nkeys for i in range(n)], _split_corruption(n))
    comp = g1_compress(it["sigs"])
    n_bad = int(round(invalid_frac * n))
    bad_pos = []
    seen = set()
    while len(bad_pos) < n_bad:
        p = rng.below(n)
        if p not in seen:
            seen.add(p)
            bad_pos.append(p)
    kinds = 6
    per_kind = [bad_pos[k::kinds] for k in range(kinds)]
    expect = it["expect"].copy()
    # 0: compression bit clear
    for p in per_kind[0]:
        comp[p, 0] &= 0x7F
        expect[p] = -ST_BAD_FLAGS
    # 1: infinity flag with a non-zero payload
    for p in per_kind[1]:
        comp[p, 0] |= 0xC0
        expect[p] = -ST_BAD_FLAGS
    # 2: infinity with the sort flag, zero payload
    for p in per_kind[2]:
        comp[p] = 0
        comp[p, 0] = 0xE0
        expect[p] = -ST_BAD_FLAGS
    # 3: x >= p (p plus a small offset, flags valid)
    for p in per_kind[3]:
        x = P_MOD + rng.below(1 << 32)
        b = bytearray(x.to_bytes(48, "big"))
        b[0] |= 0x80
        comp[p] = np.frombuffer(bytes(b), dtype=np.uint8)
        expect[p] = -ST_X_NOT_CANONICAL
    # 4: x^3 + 4 not a square
    nr = special_points(rng.next(), len(per_kind[4]), 0)
    for j, p in enumerate(per_kind[4]):
        comp[p] = nr[j]
        expect[p] = -ST_NOT_ON_CURVE
    # 5: on the curve, outside the subgroup
    ns = special_points(rng.next(), len(per_kind[5]), 1)
    for j, p in enumerate(per_kind[5]):
        comp[p] = ns[j]
        expect[p] = -ST_NOT_IN_SUBGROUP
    return {**keys, **it, "sigs_compressed": comp, "expect": expect, "invalid_positions": np.array(bad_pos),
            "name": "compressed-%d" % n}


def loguniform_sizes(rng, count, hi):
    """floor(exp(U * ln(hi + 1))) clipped to [1, hi]: log-uniform on [1, hi]."""
    out = []
    for _ in range(count):
        out.append(min(hi, max(1, int(math.exp(rng.uniform() * math.log(hi + 1))))))
    return out


def config_requests(nreq=256, max_size=2048, nkeys=40, seed=4):
    """Batching workload: nreq requests of log-uniform size in [1, max_size], each over
    1..nkeys keys drawn from the pool.  Items are concatenated; offsets[r] is
    the first item of request r."""
    rng = SplitMix64(seed)
    keys = _keys(rng, nkeys)
    sizes = loguniform_sizes(rng, nreq, max_size)
    key_of_item = []
    for s in sizes:
        k = 1 + rng.below(nkeys)
        start = rng.below(nkeys)
        ks = [(start + j) % nkeys for j in range(k)]
        key_of_item.extend(ks[j % k] for j in range(s))
    n = len(key_of_item)
    it = _items(rng, keys, key_of_item, _split_corruption(n))
    offsets = np.zeros(nreq + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    return {**keys, **it, "offsets": offsets, "sizes": np.array(sizes), "name": "requests-%d" % nreq}


def config_pool(n=8192, nkeys=40, seed=5):
    """Item pool the serving stream draws its requests from."""
    rng = SplitMix64(seed)
    keys = _keys(rng, nkeys)
    it = _items(rng, keys, [i % nkeys for i in range(n)], _split_corruption(n))
    return {**keys, **it, "name": "pool-%d" % n}


def poisson_stream(duration_s, rate_per_s, max_size=512, pool_size=8192, seed=6):
    """Arrival times (Poisson, rate per second), sizes log-uniform in
    [1, max_size], and for each request the pool indices of its items."""
    rng = SplitMix64(seed)
    t, arrivals, sizes, starts = 0.0, [], [], []
    while True:
        t += -math.log(1.0 - rng.uniform()) / rate_per_s
        if t >= duration_s:
            break
        arrivals.append(t)
        s = loguniform_sizes(rng, 1, max_size)[0]
        sizes.append(s)
        starts.append(rng.below(pool_size))
    return np.array(arrivals), np.array(sizes, dtype=np.int64), np.array(starts, dtype=np.int64)
