"""Constants of the hash to G1 (h2c.cuh on the device, the workload generator
on the host), derived here rather than typed in.

  SHA-256 (FIPS 180-4 section 4.2.2 / 5.3.3): K[t] = first 32 bits of the
    fractional part of the cube root of the t-th prime; H0 the same for the
    square roots of the first eight primes.
  Simplified SWU map for BLS12-381 G1 (RFC 9380 sections 6.6.2, 6.6.3 and
    8.8.1, the suite BLS12381G1_XMD:SHA-256_SSWU_RO_ that ic_bls12_381's
    hash_to_curve implements): the map runs on E': y^2 = x^3 + A' x + B',
    which is 11-isogenous to E: y^2 = x^3 + 4, and an 11-isogeny carries its
    points to E.
    * A' and B' are the suite's published coefficients.  They are accepted
      only because random points of E' are killed by #E(Fp) = h r (curves
      isogenous over Fp have the same order), which a mistyped digit would
      not survive (check_isogenous_curve).
    * Z is the result of the RFC's search (appendix H.2, find_z_sswu).
    * The isogeny E' -> E is derived, not typed: its kernel polynomial D is
      the product of the five rational roots of the 11-division polynomial of
      E'; Velu's formulas in Kohel's form give the codomain y^2 = x^3 + b''
      and the map x -> N(x) / D(x)^2, y -> y (N' D - 2 N D') / D^3; the
      isomorphism (x, y) -> (u^2 x, u^3 y) onto y^2 = x^3 + 4 is fixed among
      its six choices by two published coefficients of the suite's map, the
      constant terms of its x and y numerators (k_(1,0) and k_(3,0) of the
      RFC's appendix E.2), each of which the derived map must reproduce in
      full (derive_isogeny).
  Field conversion of 64-byte strings (RFC 9380 section 5.2, L = 64): a
    value hi 2^256 + lo becomes Montgomery form as mont_mul(lo, R^2) +
    mont_mul(hi, 2^256 R^2).
  Cofactor clearing of G1 (RFC 9380 section 8.8.1): h_eff = 1 - x.

Writes h2c.inc next to this file (run `python gen_h2c.py`).  The header's
arrays are `__device__ __constant__` unless the includer defines
BLS_H2C_CONST (the host workload generator defines it as `static const`).
"""
import os
import random
from math import isqrt

P = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
R = 1 << 384
X_BLS = -0xd201000000010000
B = 4
N_E = P + 1 - (X_BLS + 1)          # #E(Fp): the trace of Frobenius of a BLS12 curve is x + 1


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


# ------------------------------------------------------------------ E' and Z
ISO_A = 0x144698a3b8e9433d693a02c96d4982b0ea985383ee66a8d8e8981aefd881ac98936f8da0e0f97f5cf428082d584c1d
ISO_B = 0x12e2908d11688030018b12e8753eee3b2016c1f0f24f4070a0b9c14fcef35ef55a23215a316ceaa5d1cc48e98e172be0
# constant terms of the suite's x and y numerators (RFC 9380 appendix E.2)
K_X0 = 0x11a05f2b1e833340b809101dd99815856b303e88a2d7005ff2627b56cdb4e2c85610c2d5f2e62d6eaeac1662734649b7
K_Y0 = 0x90d97c81ba24ee0259d1f094980dcfa11ad138e48a869522b52af6c956543d3cd0c7aee9b3ba3c2be9845719707bb33


def g_iso(x):
    return (x * x * x + ISO_A * x + ISO_B) % P


def ec_add(p1, p2, a):
    """affine addition on y^2 = x^3 + a x + b (None is the identity)"""
    if p1 is None:
        return p2
    if p2 is None:
        return p1
    (x1, y1), (x2, y2) = p1, p2
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        lam = (3 * x1 * x1 + a) * inv(2 * y1) % P
    else:
        lam = (y2 - y1) * inv((x2 - x1) % P) % P
    x3 = (lam * lam - x1 - x2) % P
    return (x3, (lam * (x1 - x3) - y1) % P)


def ec_mul(pt, k, a):
    acc = None
    while k:
        if k & 1:
            acc = ec_add(acc, pt, a)
        pt = ec_add(pt, pt, a)
        k >>= 1
    return acc


def check_isogenous_curve(trials=3):
    """#E'(Fp) = #E(Fp): random points of E' have order dividing N_E."""
    rng = random.Random(2024)
    for _ in range(trials):
        while True:
            x = rng.randrange(P)
            if is_square(g_iso(x)):
                break
        assert ec_mul((x, sqrt(g_iso(x))), N_E, ISO_A) is None, "E' is not isogenous to E"


def find_z_sswu():
    """RFC 9380 appendix H.2: Z non-square, Z != -1, g(x) - Z irreducible
    (a cubic without roots in Fp), g(B / (Z A)) square; smallest |Z| first,
    positive before negative."""
    ctr = 1
    while True:
        for z in (ctr % P, (-ctr) % P):
            if is_square(z) or z == P - 1:
                continue
            gz = [(ISO_B - z) % P, ISO_A, 0, 1]
            xpz = poly_powmod([0, 1], P, gz)
            if len(poly_gcd(gz, poly_sub(xpz, [0, 1]))) > 1:
                continue
            if not is_square(g_iso(ISO_B * inv(z * ISO_A % P) % P)):
                continue
            return z
        ctr += 1


# ------------------------------------------------------------------ polynomials over Fp (index = degree)
def _trim(a):
    while a and a[-1] % P == 0:
        a.pop()
    return a


def poly_add(a, b):
    n = max(len(a), len(b))
    return _trim([((a[i] if i < len(a) else 0) + (b[i] if i < len(b) else 0)) % P for i in range(n)])


def poly_sub(a, b):
    n = max(len(a), len(b))
    return _trim([((a[i] if i < len(a) else 0) - (b[i] if i < len(b) else 0)) % P for i in range(n)])


def poly_mul(a, b):
    if not a or not b:
        return []
    r = [0] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        if x:
            for j, y in enumerate(b):
                r[i + j] += x * y
    return _trim([v % P for v in r])


def poly_scale(a, c):
    return _trim([x * c % P for x in a])


def poly_divmod(a, b):
    a = a[:]
    q = [0] * max(1, len(a) - len(b) + 1)
    lead = inv(b[-1])
    while len(a) >= len(b) and a:
        c = a[-1] * lead % P
        d = len(a) - len(b)
        q[d] = c
        for i, y in enumerate(b):
            a[i + d] = (a[i + d] - c * y) % P
        _trim(a)
    return _trim(q), a


def poly_gcd(a, b):
    while b:
        a, b = b, poly_divmod(a, b)[1]
    return poly_scale(a, inv(a[-1])) if a else a


def poly_powmod(a, e, m):
    r, a = [1], poly_divmod(a, m)[1]
    while e:
        if e & 1:
            r = poly_divmod(poly_mul(r, a), m)[1]
        a = poly_divmod(poly_mul(a, a), m)[1]
        e >>= 1
    return r


def poly_deriv(a):
    return _trim([i * a[i] % P for i in range(1, len(a))])


def poly_eval(a, x):
    r = 0
    for c in reversed(a):
        r = (r * x + c) % P
    return r


def division_poly_11(a, b):
    """psi_11 of y^2 = x^3 + a x + b (a polynomial in x; even-index psi_n are
    y g_n with g_n in Fp[x], and y^2 = f(x))."""
    f = [b, a, 0, 1]
    f2 = poly_mul(f, f)
    psi1 = [1]
    psi3 = _trim([(-a * a) % P, 12 * b % P, 6 * a % P, 0, 3])
    g2 = [2]
    g4 = poly_scale(_trim([(-8 * b * b - a ** 3) % P, (-4 * a * b) % P, (-5 * a * a) % P, 20 * b % P,
                           5 * a % P, 0, 1]), 4)
    cube = lambda v: poly_mul(v, poly_mul(v, v))  # noqa: E731
    psi5 = poly_sub(poly_mul(f2, poly_mul(g4, cube(g2))), cube(psi3))                # psi4 psi2^3 - psi1 psi3^3
    g6 = poly_scale(poly_mul(poly_sub(poly_mul(psi5, poly_mul(g2, g2)), poly_mul(psi1, poly_mul(g4, g4))), psi3),
                    inv(2))                                                          # (psi5 psi2^2 - psi1 psi4^2) psi3 / 2y
    psi7 = poly_sub(poly_mul(psi5, cube(psi3)), poly_mul(f2, poly_mul(g2, cube(g4))))  # psi5 psi3^3 - psi2 psi4^3
    return poly_sub(poly_mul(psi7, cube(psi5)), poly_mul(f2, poly_mul(g4, cube(g6))))  # psi7 psi5^3 - psi4 psi6^3


def _cube_root(a):
    """a cube root of a in Fp (p - 1 = 3^2 s): a^(1/3) up to the 3-Sylow part,
    then a search over that subgroup's nine elements"""
    s = P - 1
    while s % 3 == 0:
        s //= 3
    z = 2
    while pow(z, (P - 1) // 3, P) == 1:
        z += 1
    c = pow(z, s, P)                     # generates the 3-Sylow subgroup
    r = pow(a, pow(3, -1, s), P)        # r^3 = a times an element of the 3-Sylow subgroup
    err = pow(r, 3, P) * inv(a) % P
    target, c3, cj = inv(err), pow(c, 3, P), 1
    for j in range(9):
        if cj == target:
            return r * pow(c, j, P) % P
        cj = cj * c3 % P
    raise AssertionError("no cube root")


def derive_isogeny():
    """(x_num, x_den, y_num, y_den) of the 11-isogeny E' -> E, coefficient
    lists (index = degree); x_den (degree 10) and y_den (degree 15) monic."""
    psi = division_poly_11(ISO_A, ISO_B)
    assert len(psi) - 1 == 60
    psi = poly_scale(psi, inv(psi[-1]))
    xp = poly_powmod([0, 1], P, psi)
    D = poly_gcd(psi, poly_sub(xp, [0, 1]))          # the rational roots of psi_11
    assert len(D) - 1 == 5, "the kernel polynomial has five rational roots"
    d, a, b = 5, ISO_A, ISO_B
    s1, s2, s3 = (-D[4]) % P, D[3] % P, (-D[2]) % P
    v = (6 * (s1 * s1 - 2 * s2) + 2 * d * a) % P
    w = (10 * (s1 ** 3 - 3 * s1 * s2 + 3 * s3) + 6 * a * s1 + 4 * b * d) % P
    a2, b2 = (a - 5 * v) % P, (b - 7 * w) % P      # codomain y^2 = x^3 + a2 x + b2
    assert a2 == 0, "the codomain has j = 0"
    f = [b, a, 0, 1]
    Dp, Dpp = poly_deriv(D), poly_deriv(poly_deriv(D))
    # Kohel: X = (2d + 1) x - 2 s1 - 2 (3 x^2 + a) D'/D + 4 f (D'^2 - D D'') / D^2
    N = poly_add(poly_mul(poly_sub([0, 2 * d + 1], [2 * s1 % P]), poly_mul(D, D)),
                 poly_sub(poly_scale(poly_mul(f, poly_sub(poly_mul(Dp, Dp), poly_mul(D, Dpp))), 4),
                          poly_scale(poly_mul([a, 0, 3], poly_mul(Dp, D)), 2)))
    Y = poly_sub(poly_mul(poly_deriv(N), D), poly_scale(poly_mul(N, Dp), 2))
    # (x, y) -> (u^2 x, u^3 y) onto y^2 = x^3 + 4: u^6 = 4 / b2
    t = 4 * inv(b2) % P
    u2_0 = _cube_root(t)
    z = 2
    while pow(z, (P - 1) // 3, P) == 1:
        z += 1
    zeta = pow(z, (P - 1) // 3, P)        # a primitive cube root of unity
    u2 = [c for c in (u2_0, u2_0 * zeta % P, u2_0 * zeta * zeta % P) if N[0] * c % P == K_X0]
    u3 = [c for c in (sqrt(t), (-sqrt(t)) % P) if Y[0] * c % P == K_Y0]
    assert len(u2) == 1 and len(u3) == 1, "the published coefficients pin one isomorphism"
    assert pow(u2[0], 3, P) == t and u3[0] * u3[0] % P == t
    x_num, y_num = poly_scale(N, u2[0]), poly_scale(Y, u3[0])
    x_den, y_den = poly_mul(D, D), poly_mul(poly_mul(D, D), D)
    assert (len(x_num), len(x_den), len(y_num), len(y_den)) == (12, 11, 16, 16)
    return x_num, x_den, y_num, y_den


check_isogenous_curve()
SSWU_Z = find_z_sswu()
SSWU_C1 = (-ISO_B) * inv(ISO_A) % P                 # -B' / A'
SSWU_C2 = ISO_B * inv(SSWU_Z * ISO_A % P) % P       # B' / (Z A'), x1 when tv1 = 0
SQRT_RATIO_E = (P - 3) // 4                          # sqrt_ratio for p = 3 mod 4 (RFC 9380 F.2.1.2): c1
SQRT_MINUS_Z = sqrt((-SSWU_Z) % P)                   # and c2 = sqrt(-Z) (any root: sgn0 fixes y)
ISO_X_NUM, ISO_X_DEN, ISO_Y_NUM, ISO_Y_DEN = derive_isogeny()
H_EFF = 1 - X_BLS
K256 = (1 << 256) * R * R % P       # raw operand: mont_mul(hi, K256) = hi 2^256 R


def iso_map(x, y):
    """E' -> E (affine; None for the identity)"""
    xd, yd = poly_eval(ISO_X_DEN, x), poly_eval(ISO_Y_DEN, x)
    if xd == 0 or yd == 0:
        return None
    return (poly_eval(ISO_X_NUM, x) * inv(xd) % P, y * poly_eval(ISO_Y_NUM, x) * inv(yd) % P)


def limbs64(v):
    return [(v >> (64 * i)) & (2 ** 64 - 1) for i in range(6)]


def mont(v):
    return limbs64(v * R % P)


def emit():
    L = ["// Generated by gen_h2c.py: constants of the hash to G1.", "#pragma once", "#include <cstdint>",
         "#ifndef BLS_H2C_CONST", "#define BLS_H2C_CONST __device__ __constant__", "#endif",
         "namespace bls {", "namespace h2c {"]

    def arr(name, vals, fmt, ty):
        L.append("BLS_H2C_CONST %s %s[%d] = {%s};" % (ty, name, len(vals), ", ".join(fmt % v for v in vals)))

    def fparr(name, coeffs):
        arr(name, [w for c in coeffs for w in mont(c)], "0x%016xull", "uint64_t")

    arr("kSha256K", SHA256_K, "0x%08xu", "uint32_t")
    arr("kSha256H0", SHA256_H0, "0x%08xu", "uint32_t")
    L.append("// E': y^2 = x^3 + A' x + B', the SSWU map's Z, -B'/A' and B'/(Z A') (Montgomery)")
    for name, v in (("kIsoA", ISO_A), ("kIsoB", ISO_B), ("kZ", SSWU_Z), ("kSswuC1", SSWU_C1), ("kSswuC2", SSWU_C2),
                    ("kSqrtMinusZ", SQRT_MINUS_Z)):
        fparr(name, [v])
    arr("kSqrtRatioE", limbs64(SQRT_RATIO_E), "0x%016xull", "uint64_t")
    L.append("constexpr int kSqrtRatioBits = %d;  // (p - 3) / 4" % SQRT_RATIO_E.bit_length())
    L.append("// the 11-isogeny E' -> E: coefficients by degree; the denominators are monic")
    L.append("// (leading 1 not stored): x = x_num / x_den, y = y' y_num / y_den")
    fparr("kIsoXNum", ISO_X_NUM)
    fparr("kIsoXDen", ISO_X_DEN[:-1])
    fparr("kIsoYNum", ISO_Y_NUM)
    fparr("kIsoYDen", ISO_Y_DEN[:-1])
    arr("kK256", limbs64(K256), "0x%016xull", "uint64_t")
    arr("kR3", [(R ** 3 % P >> (32 * i)) & 0xffffffff for i in range(12)], "0x%08xu", "uint32_t")
    L.append("constexpr uint64_t kHEff = 0x%016xull;  // 1 - x" % H_EFF)
    L.append("constexpr int kIsoXNumLen = %d, kIsoXDenLen = %d, kIsoYNumLen = %d, kIsoYDenLen = %d;"
             % (len(ISO_X_NUM), len(ISO_X_DEN) - 1, len(ISO_Y_NUM), len(ISO_Y_DEN) - 1))
    L.append("}  // namespace h2c")
    L.append("}  // namespace bls")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "h2c.inc")
    with open(out, "w") as f:
        f.write("\n".join(L) + "\n")


if __name__ == "__main__":
    emit()
