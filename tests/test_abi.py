"""CPU tests of the C ABI boundary: the library loads, exports every symbol the
header declares, validates arguments without touching a GPU, and reports a
missing device the way the reference does."""
import ctypes
import os
import re

import numpy as np
import pytest

import bls_gpu as G


def _declared_functions():
    with open(G.HEADER_PATH) as f:
        text = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*\b([a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while")))


def test_header_declares_reference_symbols():
    names = _declared_functions()
    for ref in ("gpu_crypto_init", "gpu_batch_bls_verify", "gpu_batch_sha256", "gpu_g1_decompress_batch",
                "gpu_g1_decompress", "gpu_msm_g1", "gpu_jacobian_to_affine"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(G.LIB_PATH)
    missing = [n for n in _declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_dlopen_symbol_check_of_ic_crate():
    """ic-integration/gpu_crypto/lib.rs:103-107 rejects the library unless all
    three symbols resolve."""
    L = ctypes.CDLL(G.LIB_PATH, mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for n in ("gpu_msm_g1", "gpu_jacobian_to_affine", "gpu_g1_decompress_batch"):
        assert getattr(L, n) is not None


def test_argument_validation_needs_no_gpu():
    L = G.lib()
    z = np.zeros(2448, dtype=np.uint64)
    r = np.zeros(1, dtype=np.int32)
    p = z.ctypes.data
    # M == 0: nothing to do (lib.rs:92 never calls with 0, the C side tolerates it)
    assert L.gpu_batch_bls_verify(p, p, p, p, r.ctypes.data, 0) == 0
    assert L.gpu_batch_bls_verify(p, p, p, p, r.ctypes.data, -1) == -1
    assert L.gpu_batch_bls_verify(None, p, p, p, r.ctypes.data, 1) == -1
    assert L.gpu_g1_decompress_batch(p, p, 0) == -1
    assert L.gpu_g1_decompress_batch(None, p, 3) == -1
    # out-of-scope entry points are -1 stubs (callers keep their CPU path)
    assert L.gpu_batch_sha256(p, p, 1, 64) == -1
    assert L.gpu_msm_g1(p, p, 1, p) == -1
    assert L.gpu_jacobian_to_affine(p, p) == -1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_behaviour():
    L = G.lib()
    assert L.gpu_crypto_init() == -1
    with pytest.raises(G.GpuError):
        G.init()
    with pytest.raises(G.GpuError):
        G.Context()
    z = np.zeros(2448, dtype=np.uint64)
    r = np.zeros(1, dtype=np.int32)
    assert L.gpu_batch_bls_verify(z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data, r.ctypes.data, 1) == -1
    assert G.last_error() != ""
    with pytest.raises(G.GpuError):
        G.ref_cache_stats()


def test_reference_cache_capacity_is_checked_before_any_device_work():
    """A capacity outside 1 .. 65536 is refused when the reference entry
    point's context is first created, before any device call (a fresh process,
    since that context lives for the life of the process)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import bls_gpu as G\n"
            "assert G.lib().bls_ref_cache_stats(None, None, None) == -1\n"
            "assert 'BLS_REF_TABLE_CACHE' in G.last_error(), G.last_error()\n")
    env = dict(os.environ, BLS_REF_TABLE_CACHE="0", PYTHONPATH=os.path.join(root, "icp-gpu_b200"))
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]


def test_python_binding_shapes_without_gpu():
    assert G.batch_bls_verify(np.zeros((0, 12)), np.zeros((0, 12)), np.zeros(2448), np.zeros((0, 2448))) == []
    with pytest.raises(G.GpuError):
        G.g1_decompress_batch(b"\x00" * 47)
