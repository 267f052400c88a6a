"""ctypes binding of the C++ CPU oracle (oracle/cpu_verifier.cpp).

TEST INFRASTRUCTURE ONLY: the checker and the timed CPU baseline.  Nothing in
the GPU library imports this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle_cpu.so")
        if not os.path.exists(path):
            raise RuntimeError("CPU oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.oc_verify_batch.argtypes = [P, P, P, P, P, P, ctypes.c_int, P, P, P, ctypes.c_int]
        L.oc_verify_compressed_batch.argtypes = [P, P, P, P, P, P, ctypes.c_int, P, ctypes.c_int]
        L.oc_g1_decompress.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int]
        L.oc_g2_prepare.argtypes = [P, P]
        L.oc_final_exp.argtypes = [P, P]
        L.oc_cyclotomic_square.argtypes = [P, P]
        L.oc_fp_mul.argtypes = [P, P, P]
        L.oc_num_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data


def num_threads():
    return lib().oc_num_threads()


def verify_batch(sigs, nhms, g2c, pkc, pk_index=None, pk_inf=None, nthreads=1, want_values=False):
    """sigs/nhms: (n,12) u64; g2c: (2448,) u64; pkc: (k,2448) u64.
    Returns results (n,) int32 [, ml (n,72), gt (n,72)]."""
    sigs = np.ascontiguousarray(sigs, dtype=np.uint64)
    nhms = np.ascontiguousarray(nhms, dtype=np.uint64)
    g2c = np.ascontiguousarray(g2c, dtype=np.uint64)
    pkc = np.ascontiguousarray(pkc, dtype=np.uint64)
    n = sigs.shape[0]
    if pk_index is not None:
        pk_index = np.ascontiguousarray(pk_index, dtype=np.int32)
    if pk_inf is not None:
        pk_inf = np.ascontiguousarray(pk_inf, dtype=np.uint8)
    res = np.zeros(n, dtype=np.int32)
    ml = np.zeros((n, 72), dtype=np.uint64) if want_values else None
    gt = np.zeros((n, 72), dtype=np.uint64) if want_values else None
    rc = lib().oc_verify_batch(_p(sigs), _p(nhms), _p(g2c), _p(pkc), _p(pk_index), _p(pk_inf), n,
                               _p(res), _p(ml), _p(gt), nthreads)
    assert rc == 0
    return (res, ml, gt) if want_values else res


def verify_compressed_batch(sigs48, nhms, g2c, pkc, pk_index=None, pk_inf=None, nthreads=1):
    sigs48 = np.ascontiguousarray(sigs48, dtype=np.uint8)
    nhms = np.ascontiguousarray(nhms, dtype=np.uint64)
    g2c = np.ascontiguousarray(g2c, dtype=np.uint64)
    pkc = np.ascontiguousarray(pkc, dtype=np.uint64)
    n = nhms.shape[0]
    if pk_index is not None:
        pk_index = np.ascontiguousarray(pk_index, dtype=np.int32)
    if pk_inf is not None:
        pk_inf = np.ascontiguousarray(pk_inf, dtype=np.uint8)
    res = np.zeros(n, dtype=np.int32)
    rc = lib().oc_verify_compressed_batch(_p(sigs48), _p(nhms), _p(g2c), _p(pkc), _p(pk_index),
                                          _p(pk_inf), n, _p(res), nthreads)
    assert rc == 0
    return res


def g1_decompress(sigs48, nthreads=1):
    sigs48 = np.ascontiguousarray(sigs48, dtype=np.uint8)
    n = sigs48.size // 48
    out = np.zeros((n, 12), dtype=np.uint64)
    st = np.zeros(n, dtype=np.int32)
    assert lib().oc_g1_decompress(_p(sigs48), n, _p(out), _p(st), nthreads) == 0
    return st, out


def g2_prepare(q24):
    q24 = np.ascontiguousarray(q24, dtype=np.uint64)
    out = np.zeros(2448, dtype=np.uint64)
    assert lib().oc_g2_prepare(_p(q24), _p(out)) == 0
    return out


def final_exp(ml72):
    ml72 = np.ascontiguousarray(ml72, dtype=np.uint64)
    out = np.zeros(72, dtype=np.uint64)
    lib().oc_final_exp(_p(ml72), _p(out))
    return out


def cyclotomic_square(f72):
    f72 = np.ascontiguousarray(f72, dtype=np.uint64)
    out = np.zeros(72, dtype=np.uint64)
    lib().oc_cyclotomic_square(_p(f72), _p(out))
    return out
