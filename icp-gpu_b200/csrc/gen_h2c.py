"""Constants of the device hash-to-G1 (h2c.cuh), derived here rather than typed in.

  SHA-256 (FIPS 180-4 section 4.2.2 / 5.3.3): K[t] = first 32 bits of the
    fractional part of the cube root of the t-th prime; H0 the same for the
    square roots of the first eight primes.
  Shallue-van de Woestijne map for y^2 = x^3 + 4 (RFC 9380 section 6.6.1): Z
    from the search of appendix H.1, then c1 = g(Z), c2 = -Z / 2,
    c3 = sqrt(-g(Z) (3 Z^2)) with sgn0(c3) = 0, c4 = -4 g(Z) / (3 Z^2).
  Field conversion of 64-byte strings (RFC 9380 section 5.2, L = 64): a
    value hi 2^256 + lo becomes Montgomery form as mont_mul(lo, R^2) +
    mont_mul(hi, 2^256 R^2).
  Cofactor clearing of G1 (RFC 9380 section 8.8.1): h_eff = 1 - x.

Writes h2c.inc next to this file (run `python gen_h2c.py`).
"""
import os
from math import isqrt

P = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
R = 1 << 384
X_BLS = -0xd201000000010000
B = 4


def primes(n):
    out, c = [], 2
    while len(out) < n:
        if all(c % q for q in out):
            out.append(c)
        c += 1
    return out


def icbrt(n):
    lo, hi = 0, 1 << (n.bit_length() // 3 + 2)
    while lo < hi:
        m = (lo + hi + 1) // 2
        if m ** 3 <= n:
            lo = m
        else:
            hi = m - 1
    return lo


SHA256_K = [icbrt(q << 96) & 0xffffffff for q in primes(64)]
SHA256_H0 = [isqrt(q << 64) & 0xffffffff for q in primes(8)]


def is_square(a):
    return a % P == 0 or pow(a, (P - 1) // 2, P) == 1


def sqrt(a):
    r = pow(a, (P + 1) // 4, P)
    assert r * r % P == a % P
    return r


def inv(a):
    return pow(a, P - 2, P)


def g(x):
    return (x * x * x + B) % P


def find_z_svdw():
    """RFC 9380 appendix H.1 with A = 0, B = 4."""
    ctr = 1
    while True:
        for z in (ctr % P, (-ctr) % P):
            gz = g(z)
            if gz == 0:
                continue
            h = (-(3 * z * z) * inv(4 * gz % P)) % P
            if h == 0 or not is_square(h):
                continue
            if is_square(gz) or is_square(g((-z) * inv(2) % P)):
                return z
        ctr += 1


SVDW_Z = find_z_svdw()
SVDW_C1 = g(SVDW_Z)
SVDW_C2 = (-SVDW_Z) * inv(2) % P
_c3 = sqrt((-SVDW_C1 * (3 * SVDW_Z * SVDW_Z)) % P)
SVDW_C3 = _c3 if _c3 % 2 == 0 else (-_c3) % P
SVDW_C4 = (-4 * SVDW_C1) * inv(3 * SVDW_Z * SVDW_Z % P) % P
H_EFF = 1 - X_BLS
K256 = (1 << 256) * R * R % P       # raw operand: mont_mul(hi, K256) = hi 2^256 R


def limbs64(v):
    return [(v >> (64 * i)) & (2 ** 64 - 1) for i in range(6)]


def mont(v):
    return limbs64(v * R % P)


def emit():
    L = ["// Generated by gen_h2c.py: constants of the device hash-to-G1.", "#pragma once", "#include <cstdint>",
         "namespace bls {", "namespace h2c {"]

    def arr(name, vals, fmt, ty):
        L.append("__device__ __constant__ %s %s[%d] = {%s};" % (ty, name, len(vals), ", ".join(fmt % v for v in vals)))

    arr("kSha256K", SHA256_K, "0x%08xu", "uint32_t")
    arr("kSha256H0", SHA256_H0, "0x%08xu", "uint32_t")
    for name, v in (("kZ", SVDW_Z), ("kC1", SVDW_C1), ("kC2", SVDW_C2), ("kC3", SVDW_C3), ("kC4", SVDW_C4)):
        arr(name, mont(v), "0x%016xull", "uint64_t")
    arr("kK256", limbs64(K256), "0x%016xull", "uint64_t")
    arr("kPMinus2", limbs64(P - 2), "0x%016xull", "uint64_t")
    L.append("constexpr uint64_t kHEff = 0x%016xull;  // 1 - x" % H_EFF)
    L.append("}  // namespace h2c")
    L.append("}  // namespace bls")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "h2c.inc")
    with open(out, "w") as f:
        f.write("\n".join(L) + "\n")


if __name__ == "__main__":
    emit()
