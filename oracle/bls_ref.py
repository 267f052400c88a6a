"""BLS12-381 verify path, restated in pure Python big integers.

TEST INFRASTRUCTURE ONLY.  This module is the checker: tests, the smoke run
and the CPU-baseline leg of the bench may call it; the GPU library never does.

It restates the reference's CPU-verifier semantics (ic_bls12_381 0.10.1, as
mirrored by the reference's GPU code) for small cases:

  * the tower Fp2 = Fp[u]/(u^2+1), Fp6 = Fp2[v]/(v^3-(1+u)), Fp12 = Fp6[w]/(w^2-v)
    (gpu-crypto/cuda/field_sppark.cuh:52-197);
  * the two-pair Miller loop over precomputed line coefficients
    (gpu-crypto/cuda/api.cu:22-52);
  * the final exponentiation chain (gpu-crypto/cuda/api.cu:54-78), including the
    Granger-Scott cyclotomic squaring formula (field_sppark.cuh:174-197), which
    is applied exactly where the reference applies it;
  * the identity test of the verify (gpu-crypto/cuda/api.cu:80-91);
  * G2 line-coefficient precomputation, Algorithms 26/27 of eprint 2010/354 as
    restated at cuda/test_miller_v2.cu:148-229 (ic_bls12_381 G2Prepared layout:
    68 coefficients of (Fp2, Fp2, Fp2));
  * G1/G2 point decompression with the ZCash flag rules and the checks that
    ic_bls12_381's from_compressed performs (the reference's GPU decoder,
    cuda/decompress.cu:140-188, performs none of them);
  * hash-to-G1 following RFC 9380's hash_to_curve construction
    (expand_message_xmd with SHA-256, hash_to_field, map_to_curve, clear_cofactor)
    for the suite BLS12381G1_XMD:SHA-256_SSWU_RO_ that ic_bls12_381 implements:
    the simplified SWU map of section 6.6.2 on the 11-isogenous curve E' and
    the 11-isogeny to E, evaluated pointwise by Velu's formulas.

Field elements are canonical Python ints in [0, p).  Montgomery limbs (R = 2^384,
6 x u64 little-endian) are produced only at the boundary (`mont_limbs`).
"""
import hashlib

P = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
R_ORDER = 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001
MONT_R = 1 << 384
MONT_RINV = pow(MONT_R, -1, P)
BLS_X = 0xd201000000010000          # |x|; the curve parameter x is negative
BLS_X_IS_NEG = True
H_EFF_G1 = 0xd201000000010001       # 1 - x, the G1 cofactor-clearing scalar (RFC 9380 8.8.1)
B_G1 = 4

# ----------------------------------------------------------------------------
# Montgomery boundary
# ----------------------------------------------------------------------------

def mont_limbs(a):
    """Canonical a -> 6 u64 limbs of a*R mod p, little-endian."""
    m = (a % P) * MONT_R % P
    return [(m >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(6)]


def from_mont_limbs(limbs):
    m = 0
    for i, w in enumerate(limbs):
        m |= int(w) << (64 * i)
    return m * MONT_RINV % P


def raw_limbs_int(limbs):
    m = 0
    for i, w in enumerate(limbs):
        m |= int(w) << (64 * i)
    return m


# ----------------------------------------------------------------------------
# Fp
# ----------------------------------------------------------------------------

def fp_inv(a):
    """Fermat inversion a^(p-2); maps 0 to 0 (field_sppark.cuh:40-50)."""
    return pow(a, P - 2, P)


def fp_sqrt(a):
    """a^((p+1)/4) (p = 3 mod 4); caller checks the square (cuda/decompress.cu:16-40)."""
    return pow(a, (P + 1) // 4, P)


def fp_is_square(a):
    return a == 0 or pow(a, (P - 1) // 2, P) == 1


def fp_lex_largest(a):
    """ic_bls12_381 Fp::lexicographically_largest: a > (p-1)/2."""
    return a > (P - 1) // 2


# ----------------------------------------------------------------------------
# Fp2 = Fp[u]/(u^2 + 1)         (field_sppark.cuh:52-83)
# ----------------------------------------------------------------------------
F2_ZERO = (0, 0)
F2_ONE = (1, 0)


def f2_add(a, b):
    return ((a[0] + b[0]) % P, (a[1] + b[1]) % P)


def f2_sub(a, b):
    return ((a[0] - b[0]) % P, (a[1] - b[1]) % P)


def f2_neg(a):
    return ((-a[0]) % P, (-a[1]) % P)


def f2_conj(a):
    return (a[0], (-a[1]) % P)


def f2_mul_nr(a):
    """times the non-residue xi = 1 + u."""
    return ((a[0] - a[1]) % P, (a[0] + a[1]) % P)


def f2_mul(a, b):
    t0 = a[0] * b[0]
    t1 = a[1] * b[1]
    return ((t0 - t1) % P, ((a[0] + a[1]) * (b[0] + b[1]) - t0 - t1) % P)


def f2_sqr(a):
    return ((a[0] + a[1]) * (a[0] - a[1]) % P, 2 * a[0] * a[1] % P)


def f2_mul_fp(a, s):
    return (a[0] * s % P, a[1] * s % P)


def f2_inv(a):
    n = (a[0] * a[0] + a[1] * a[1]) % P
    i = fp_inv(n)
    return (a[0] * i % P, (-a[1] * i) % P)


def f2_is_zero(a):
    return a[0] == 0 and a[1] == 0


def f2_pow(a, e):
    r = F2_ONE
    base = a
    while e:
        if e & 1:
            r = f2_mul(r, base)
        base = f2_sqr(base)
        e >>= 1
    return r


def f2_is_square(a):
    """a is a square in Fp2 iff its norm is a square in Fp."""
    return fp_is_square((a[0] * a[0] + a[1] * a[1]) % P)


def f2_sqrt(a):
    """Some square root of a square a in Fp2 (p = 3 mod 4), or None."""
    if f2_is_zero(a):
        return F2_ZERO
    # complex method: a = a0 + a1 u, |a| = sqrt(a0^2 + a1^2)
    n = (a[0] * a[0] + a[1] * a[1]) % P
    if not fp_is_square(n):
        return None
    alpha = fp_sqrt(n)
    for s in (alpha, (-alpha) % P):
        d = (a[0] + s) * fp_inv(2) % P
        if fp_is_square(d):
            x0 = fp_sqrt(d)
            if x0 == 0:
                continue
            x1 = a[1] * fp_inv(2 * x0 % P) % P
            cand = (x0, x1)
            if f2_sqr(cand) == (a[0] % P, a[1] % P):
                return cand
    if a[1] == 0:   # a in Fp and a non-square there: sqrt = sqrt(-a0) * u
        t = (-a[0]) % P
        if fp_is_square(t):
            cand = (0, fp_sqrt(t))
            if f2_sqr(cand) == a:
                return cand
    return None


def f2_lex_largest(a):
    """ic_bls12_381 Fp2::lexicographically_largest."""
    return fp_lex_largest(a[1]) or (a[1] == 0 and fp_lex_largest(a[0]))


# ----------------------------------------------------------------------------
# Fp6 = Fp2[v]/(v^3 - xi)       (field_sppark.cuh:85-134)
# ----------------------------------------------------------------------------
F6_ZERO = (F2_ZERO, F2_ZERO, F2_ZERO)
F6_ONE = (F2_ONE, F2_ZERO, F2_ZERO)


def f6_add(a, b):
    return (f2_add(a[0], b[0]), f2_add(a[1], b[1]), f2_add(a[2], b[2]))


def f6_sub(a, b):
    return (f2_sub(a[0], b[0]), f2_sub(a[1], b[1]), f2_sub(a[2], b[2]))


def f6_neg(a):
    return (f2_neg(a[0]), f2_neg(a[1]), f2_neg(a[2]))


def f6_mul_by_v(a):
    return (f2_mul_nr(a[2]), a[0], a[1])


def f6_mul(a, b):
    aa = f2_mul(a[0], b[0])
    bb = f2_mul(a[1], b[1])
    cc = f2_mul(a[2], b[2])
    c0 = f2_add(aa, f2_mul_nr(f2_sub(f2_sub(f2_mul(f2_add(a[1], a[2]), f2_add(b[1], b[2])), bb), cc)))
    c1 = f2_add(f2_sub(f2_sub(f2_mul(f2_add(a[0], a[1]), f2_add(b[0], b[1])), aa), bb), f2_mul_nr(cc))
    c2 = f2_add(f2_sub(f2_sub(f2_mul(f2_add(a[0], a[2]), f2_add(b[0], b[2])), aa), cc), bb)
    return (c0, c1, c2)


def f6_inv(f):
    """field_sppark.cuh:104-111 (norm to Fp2, then Fp2 inversion)."""
    c0s, c1s, c2s = f2_sqr(f[0]), f2_sqr(f[1]), f2_sqr(f[2])
    c01, c02, c12 = f2_mul(f[0], f[1]), f2_mul(f[0], f[2]), f2_mul(f[1], f[2])
    t0 = f2_sub(c0s, f2_mul_nr(c12))
    t1 = f2_sub(f2_mul_nr(c2s), c01)
    t2 = f2_sub(c1s, c02)
    sc = f2_add(f2_mul(f[0], t0), f2_mul_nr(f2_add(f2_mul(f[2], t1), f2_mul(f[1], t2))))
    si = f2_inv(sc)
    return (f2_mul(t0, si), f2_mul(t1, si), f2_mul(t2, si))


# Frobenius coefficients, derived (and pinned against field_sppark.cuh:113-166)
XI = (1, 1)
FROB6_C1 = f2_pow(XI, (P - 1) // 3)          # multiplies c1 after conjugation
FROB6_C2 = f2_pow(XI, 2 * (P - 1) // 3)      # multiplies c2 after conjugation
FROB12_C1 = f2_pow(XI, (P - 1) // 6)         # multiplies every Fp2 of c1


def f6_frob(f):
    return (f2_conj(f[0]), f2_mul(f2_conj(f[1]), FROB6_C1), f2_mul(f2_conj(f[2]), FROB6_C2))


def f6_mul_by_01(s, c0, c1):
    """Sparse product s * (c0 + c1 v) (field_sppark.cuh:126-131)."""
    aa = f2_mul(s[0], c0)
    bb = f2_mul(s[1], c1)
    t1 = f2_add(f2_mul_nr(f2_mul(s[2], c1)), aa)
    t2 = f2_sub(f2_sub(f2_mul(f2_add(c0, c1), f2_add(s[0], s[1])), aa), bb)
    t3 = f2_add(f2_mul(s[2], c0), bb)
    return (t1, t2, t3)


def f6_mul_by_1(s, c1):
    """Sparse product s * (c1 v) (field_sppark.cuh:132-134)."""
    return (f2_mul_nr(f2_mul(s[2], c1)), f2_mul(s[0], c1), f2_mul(s[1], c1))


# ----------------------------------------------------------------------------
# Fp12 = Fp6[w]/(w^2 - v)       (field_sppark.cuh:136-197)
# ----------------------------------------------------------------------------
F12_ONE = (F6_ONE, F6_ZERO)


def f12_mul(a, b):
    aa = f6_mul(a[0], b[0])
    bb = f6_mul(a[1], b[1])
    return (f6_add(aa, f6_mul_by_v(bb)),
            f6_sub(f6_sub(f6_mul(f6_add(a[0], a[1]), f6_add(b[0], b[1])), aa), bb))


def f12_sqr(a):
    ab = f6_mul(a[0], a[1])
    s1 = f6_add(a[0], a[1])
    s2 = f6_add(a[0], f6_mul_by_v(a[1]))
    return (f6_sub(f6_sub(f6_mul(s2, s1), ab), f6_mul_by_v(ab)), f6_add(ab, ab))


def f12_conj(a):
    return (a[0], f6_neg(a[1]))


def f12_inv(f):
    t = f6_sub(f6_mul(f[0], f[0]), f6_mul_by_v(f6_mul(f[1], f[1])))
    ti = f6_inv(t)
    return (f6_mul(f[0], ti), f6_neg(f6_mul(f[1], ti)))


def f12_frob(f):
    c0 = f6_frob(f[0])
    c1 = f6_frob(f[1])
    return (c0, (f2_mul(c1[0], FROB12_C1), f2_mul(c1[1], FROB12_C1), f2_mul(c1[2], FROB12_C1)))


def f12_mul_by_014(f, c0, c1, c4):
    """f * (c0 + c1 v + c4 v w) (field_sppark.cuh:168-172)."""
    aa = f6_mul_by_01(f[0], c0, c1)
    bb = f6_mul_by_1(f[1], c4)
    o = f2_add(c1, c4)
    c1n = f6_sub(f6_sub(f6_mul_by_01(f6_add(f[1], f[0]), c0, o), aa), bb)
    c0n = f6_add(f6_mul_by_v(bb), aa)
    return (c0n, c1n)


def _fp4_square(a, b):
    t0 = f2_sqr(a)
    t1 = f2_sqr(b)
    out0 = f2_add(f2_mul_nr(t1), t0)
    out1 = f2_sub(f2_sub(f2_sqr(f2_add(a, b)), t0), t1)
    return out0, out1


def f12_cyclotomic_square(f):
    """Granger-Scott squaring (field_sppark.cuh:174-197).  Equals f^2 only on
    the cyclotomic subgroup; the formula itself is what must match."""
    z0, z4, z3 = f[0]
    z2, z1, z5 = f[1]
    A0, A1 = _fp4_square(z0, z1)
    z0 = f2_sub(A0, z0)
    z0 = f2_add(f2_add(z0, z0), A0)
    z1 = f2_add(A1, z1)
    z1 = f2_add(f2_add(z1, z1), A1)
    B0, B1 = _fp4_square(z2, z3)
    C0, C1 = _fp4_square(z4, z5)
    z4 = f2_sub(B0, z4)
    z4 = f2_add(f2_add(z4, z4), B0)
    z5 = f2_add(B1, z5)
    z5 = f2_add(f2_add(z5, z5), B1)
    nr_c1 = f2_mul_nr(C1)
    z2 = f2_add(nr_c1, z2)
    z2 = f2_add(f2_add(z2, z2), nr_c1)
    z3 = f2_sub(C0, z3)
    z3 = f2_add(f2_add(z3, z3), C0)
    return ((z0, z4, z3), (z2, z1, z5))


def f12_flat(f):
    """Fp12 -> 12 canonical Fp in the reference's memory order
    (c0.c0.c0, c0.c0.c1, c0.c1.c0, ..., c1.c2.c1)."""
    out = []
    for f6 in f:
        for f2 in f6:
            out.extend(f2)
    return out


def f12_from_flat(v):
    v = [x % P for x in v]
    f2s = [(v[2 * i], v[2 * i + 1]) for i in range(6)]
    return ((f2s[0], f2s[1], f2s[2]), (f2s[3], f2s[4], f2s[5]))


def f12_mont_limbs(f):
    out = []
    for x in f12_flat(f):
        out.extend(mont_limbs(x))
    return out


def f12_from_mont_limbs(limbs):
    return f12_from_flat([from_mont_limbs(limbs[6 * i:6 * i + 6]) for i in range(12)])


# ----------------------------------------------------------------------------
# Miller loop over precomputed lines (gpu-crypto/cuda/api.cu:22-52)
# ----------------------------------------------------------------------------

def _loop_bits():
    """Bits of |x| >> 1 from the MSB, skipping up to and including the first 1."""
    bits = []
    found = False
    for b in range(63, -1, -1):
        bit = ((BLS_X >> 1) >> b) & 1 == 1
        if not found:
            found = bit
            continue
        bits.append(bit)
    return bits


LOOP_BITS = _loop_bits()        # 62 entries; 5 set
N_COEFFS = 68


def _ell(f, coeff, px, py):
    c0, c1, c2 = coeff
    return f12_mul_by_014(f, c2, f2_mul_fp(c1, px), f2_mul_fp(c0, py))


def multi_miller_loop(pairs):
    """pairs: list of (P, coeffs, skip).  P = (x, y) canonical affine G1,
    coeffs = 68 x (c0, c1, c2) Fp2 triples; skip=True drops the pair (the
    ic_bls12_381 rule for an identity P or Q).  Returns the conjugated f."""
    f = F12_ONE
    ci = 0
    for bit in LOOP_BITS:
        for (pt, co, skip) in pairs:
            if not skip:
                f = _ell(f, co[ci], pt[0], pt[1])
        ci += 1
        if bit:
            for (pt, co, skip) in pairs:
                if not skip:
                    f = _ell(f, co[ci], pt[0], pt[1])
            ci += 1
        f = f12_sqr(f)
    for (pt, co, skip) in pairs:
        if not skip:
            f = _ell(f, co[ci], pt[0], pt[1])
    assert ci + 1 == N_COEFFS
    return f12_conj(f)


# ----------------------------------------------------------------------------
# Final exponentiation (gpu-crypto/cuda/api.cu:54-78)
# ----------------------------------------------------------------------------

def cyc_exp(f):
    """f^x for x = -|x|: square-and-multiply over |x| with the Granger-Scott
    square, then conjugate (api.cu:54-63)."""
    t = F12_ONE
    found = False
    for i in range(63, -1, -1):
        if found:
            t = f12_cyclotomic_square(t)
        bit = (BLS_X >> i) & 1 == 1
        if not found:
            found = bit
            if not bit:
                continue
        if bit:
            t = f12_mul(t, f)
    return f12_conj(t)


def final_exponentiation(fi):
    f = fi
    t0 = f12_conj(f)
    t1 = f12_inv(f)
    t2 = f12_mul(t0, t1)
    t1 = t2
    t2 = f12_mul(f12_frob(f12_frob(t2)), t1)
    f = t2
    t1 = f12_conj(f12_cyclotomic_square(t2))
    t3 = cyc_exp(t2)
    t4 = f12_mul(t1, t3)
    t1 = cyc_exp(t4)
    t4 = f12_conj(t4)
    f = f12_mul(f, t4)
    t4 = f12_cyclotomic_square(t3)
    t0 = cyc_exp(t1)
    t3 = f12_mul(t3, t0)
    t3 = f12_frob(f12_frob(t3))
    f = f12_mul(f, t3)
    t4 = f12_mul(t4, cyc_exp(t0))
    f = f12_mul(f, cyc_exp(t4))
    t4 = f12_mul(t4, f12_conj(t2))
    t2 = f12_mul(t2, t1)
    t2 = f12_frob(f12_frob(f12_frob(t2)))
    f = f12_mul(f, t2)
    t4 = f12_frob(t4)
    f = f12_mul(f, t4)
    return f


def f12_is_one(f):
    return f == F12_ONE


# ----------------------------------------------------------------------------
# Curve groups (affine canonical coordinates, None = identity)
# ----------------------------------------------------------------------------
G1_GEN = (
    0x17f1d3a73197d7942695638c4fa9ac0fc3688c4f9774b905a14e3a3f171bac586c55e83ff97a1aeffb3af00adb22c6bb,
    0x08b3f481e3aaa0f1a09e30ed741d8ae4fcf5e095d5d00af600db18cb2c04b3edd03cc744a2888ae40caa232946c5e7e1,
)
G2_GEN = (
    (0x024aa2b2f08f0a91260805272dc51051c6e47ad4fa403b02b4510b647ae3d1770bac0326a805bbefd48056c8c121bdb8,
     0x13e02b6052719f607dacd3a088274f65596bd0d09920b61ab5da61bbdc7f5049334cf11213945d57e5ac7d055d042b7e),
    (0x0ce5d527727d6e118cc9cdc6da2e351aadfd9baa8cbdd3a76d429a695160d12c923ac9cc3baca289e193548608b82801,
     0x0606c4a02ea734cc32acd2b02bc28b99cb3e287e85a763af267492ab572e99ab3f370d275cec1da1aaa9075ff05f79be),
)
B_G2 = (4, 4)   # 4(1 + u)


def g1_on_curve(pt):
    if pt is None:
        return True
    x, y = pt
    return (y * y - x * x * x - B_G1) % P == 0


def g1_add(a, b):
    if a is None:
        return b
    if b is None:
        return a
    x1, y1 = a
    x2, y2 = b
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        lam = 3 * x1 * x1 * fp_inv(2 * y1 % P) % P
    else:
        lam = (y2 - y1) * fp_inv((x2 - x1) % P) % P
    x3 = (lam * lam - x1 - x2) % P
    return (x3, (lam * (x1 - x3) - y1) % P)


def g1_neg(a):
    return None if a is None else (a[0], (-a[1]) % P)


def g1_mul(a, k):
    r = None
    q = a
    while k:
        if k & 1:
            r = g1_add(r, q)
        q = g1_add(q, q)
        k >>= 1
    return r


def g1_in_subgroup(pt):
    return g1_mul(pt, R_ORDER) is None


def g2_on_curve(pt):
    if pt is None:
        return True
    x, y = pt
    return f2_sub(f2_sqr(y), f2_add(f2_mul(f2_sqr(x), x), B_G2)) == F2_ZERO


def g2_add(a, b):
    if a is None:
        return b
    if b is None:
        return a
    x1, y1 = a
    x2, y2 = b
    if x1 == x2:
        if f2_add(y1, y2) == F2_ZERO:
            return None
        lam = f2_mul(f2_mul_fp(f2_sqr(x1), 3), f2_inv(f2_add(y1, y1)))
    else:
        lam = f2_mul(f2_sub(y2, y1), f2_inv(f2_sub(x2, x1)))
    x3 = f2_sub(f2_sub(f2_sqr(lam), x1), x2)
    return (x3, f2_sub(f2_mul(lam, f2_sub(x1, x3)), y1))


def g2_mul(a, k):
    r = None
    q = a
    while k:
        if k & 1:
            r = g2_add(r, q)
        q = g2_add(q, q)
        k >>= 1
    return r


def g2_in_subgroup(pt):
    return g2_mul(pt, R_ORDER) is None


# ----------------------------------------------------------------------------
# G2 line coefficients (G2Prepared), cuda/test_miller_v2.cu:148-229
# (Algorithms 26 and 27 of eprint 2010/354, homogeneous projective X, Y, Z)
# ----------------------------------------------------------------------------

def _doubling_step(r):
    X, Y, Z = r
    tmp0 = f2_sqr(X)
    tmp1 = f2_sqr(Y)
    tmp2 = f2_sqr(tmp1)
    tmp3 = f2_sub(f2_sqr(f2_add(tmp1, X)), f2_add(tmp0, tmp2))
    tmp3 = f2_add(tmp3, tmp3)
    tmp4 = f2_add(f2_add(tmp0, tmp0), tmp0)
    tmp6 = f2_add(X, tmp4)
    tmp5 = f2_sqr(tmp4)
    zsq = f2_sqr(Z)
    X = f2_sub(f2_sub(tmp5, tmp3), tmp3)
    Z = f2_sub(f2_sqr(f2_add(Z, Y)), f2_add(tmp1, zsq))
    Y = f2_mul(f2_sub(tmp3, X), tmp4)
    tmp2 = f2_add(tmp2, tmp2)
    tmp2 = f2_add(tmp2, tmp2)
    tmp2 = f2_add(tmp2, tmp2)
    Y = f2_sub(Y, tmp2)
    tmp3 = f2_mul(tmp4, zsq)
    tmp3 = f2_add(tmp3, tmp3)
    tmp3 = f2_neg(tmp3)
    tmp6 = f2_sub(f2_sqr(tmp6), f2_add(tmp0, tmp5))
    tmp1 = f2_add(tmp1, tmp1)
    tmp1 = f2_add(tmp1, tmp1)
    tmp6 = f2_sub(tmp6, tmp1)
    tmp0 = f2_mul(Z, zsq)
    tmp0 = f2_add(tmp0, tmp0)
    return (X, Y, Z), (tmp0, tmp3, tmp6)


def _addition_step(r, q):
    X, Y, Z = r
    qx, qy = q
    zsq = f2_sqr(Z)
    ysq = f2_sqr(qy)
    t0 = f2_mul(zsq, qx)
    t1 = f2_mul(f2_sub(f2_sqr(f2_add(qy, Z)), f2_add(ysq, zsq)), zsq)
    t2 = f2_sub(t0, X)
    t3 = f2_sqr(t2)
    t4 = f2_add(t3, t3)
    t4 = f2_add(t4, t4)
    t5 = f2_mul(t4, t2)
    t6 = f2_sub(f2_sub(t1, Y), Y)
    t9 = f2_mul(t6, qx)
    t7 = f2_mul(t4, X)
    Xn = f2_sub(f2_sub(f2_sub(f2_sqr(t6), t5), t7), t7)
    Zn = f2_sub(f2_sqr(f2_add(Z, t2)), f2_add(zsq, t3))
    t10 = f2_add(qy, Zn)
    t8 = f2_mul(f2_sub(t7, Xn), t6)
    t0b = f2_mul(Y, t5)
    t0b = f2_add(t0b, t0b)
    Yn = f2_sub(t8, t0b)
    t10 = f2_sub(f2_sqr(t10), ysq)
    ztsq = f2_sqr(Zn)
    t10 = f2_sub(t10, ztsq)
    t9 = f2_sub(f2_add(t9, t9), t10)
    t10o = f2_add(Zn, Zn)
    t6 = f2_neg(t6)
    t1o = f2_add(t6, t6)
    return (Xn, Yn, Zn), (t10o, t1o, t9)


def g2_prepare(q):
    """68 line coefficients (c0, c1, c2) for affine canonical Q (not identity)."""
    r = (q[0], q[1], F2_ONE)
    coeffs = []
    for bit in LOOP_BITS:
        r, c = _doubling_step(r)
        coeffs.append(c)
        if bit:
            r, c = _addition_step(r, q)
            coeffs.append(c)
    r, c = _doubling_step(r)
    coeffs.append(c)
    assert len(coeffs) == N_COEFFS
    return coeffs


def coeffs_to_limbs(coeffs):
    out = []
    for (c0, c1, c2) in coeffs:
        for f2 in (c0, c1, c2):
            out.extend(mont_limbs(f2[0]))
            out.extend(mont_limbs(f2[1]))
    return out


def coeffs_from_limbs(limbs):
    assert len(limbs) == N_COEFFS * 36
    co = []
    for i in range(N_COEFFS):
        b = 36 * i
        f = [from_mont_limbs(limbs[b + 6 * k:b + 6 * k + 6]) for k in range(6)]
        co.append(((f[0], f[1]), (f[2], f[3]), (f[4], f[5])))
    return co


# ----------------------------------------------------------------------------
# Verify (gpu-crypto/cuda/api.cu:80-91 / ic_bls12_381 multi_miller_loop)
# ----------------------------------------------------------------------------

def verify(sig, neg_hm, g2_coeffs, pk_coeffs, pk_is_identity=False):
    """e(sig, G2) * e(-H(m), pk) == 1.  sig / neg_hm: affine canonical, or None
    for the identity (its pair is skipped).  Returns (ok, miller, gt)."""
    dummy = (0, 0)
    pairs = [(sig if sig is not None else dummy, g2_coeffs, sig is None),
             (neg_hm if neg_hm is not None else dummy, pk_coeffs, neg_hm is None or pk_is_identity)]
    ml = multi_miller_loop(pairs)
    gt = final_exponentiation(ml)
    return f12_is_one(gt), ml, gt


# ----------------------------------------------------------------------------
# Serialization (ZCash BLS12-381 format, as ic_bls12_381 reads it)
# ----------------------------------------------------------------------------
# Per-item decode status codes shared with the GPU library.
ST_OK = 0
ST_BAD_FLAGS = 1
ST_X_NOT_CANONICAL = 2
ST_NOT_ON_CURVE = 3
ST_NOT_IN_SUBGROUP = 4


def g1_compress(pt):
    if pt is None:
        b = bytearray(48)
        b[0] = 0xC0
        return bytes(b)
    x, y = pt
    b = bytearray(x.to_bytes(48, "big"))
    b[0] |= 0x80
    if fp_lex_largest(y):
        b[0] |= 0x20
    return bytes(b)


def g1_decompress(b, check_subgroup=True):
    """Returns (status, point) where point is None for the identity."""
    assert len(b) == 48
    comp = (b[0] >> 7) & 1
    inf = (b[0] >> 6) & 1
    sort = (b[0] >> 5) & 1
    xb = bytearray(b)
    xb[0] &= 0x1F
    x = int.from_bytes(xb, "big")
    if not comp:
        return ST_BAD_FLAGS, None
    if inf:
        if sort or x != 0:
            return ST_BAD_FLAGS, None
        return ST_OK, None
    if x >= P:
        return ST_X_NOT_CANONICAL, None
    y2 = (x * x * x + B_G1) % P
    y = fp_sqrt(y2)
    if y * y % P != y2:
        return ST_NOT_ON_CURVE, None
    if fp_lex_largest(y) != bool(sort):
        y = (-y) % P
    pt = (x, y)
    if check_subgroup and not g1_in_subgroup(pt):
        return ST_NOT_IN_SUBGROUP, None
    return ST_OK, pt


def g2_compress(pt):
    if pt is None:
        b = bytearray(96)
        b[0] = 0xC0
        return bytes(b)
    x, y = pt
    b = bytearray(x[1].to_bytes(48, "big") + x[0].to_bytes(48, "big"))
    b[0] |= 0x80
    if f2_lex_largest(y):
        b[0] |= 0x20
    return bytes(b)


def g2_decompress(b, check_subgroup=True):
    assert len(b) == 96
    comp = (b[0] >> 7) & 1
    inf = (b[0] >> 6) & 1
    sort = (b[0] >> 5) & 1
    xb = bytearray(b)
    xb[0] &= 0x1F
    x1 = int.from_bytes(xb[:48], "big")
    x0 = int.from_bytes(xb[48:], "big")
    if not comp:
        return ST_BAD_FLAGS, None
    if inf:
        if sort or x0 != 0 or x1 != 0:
            return ST_BAD_FLAGS, None
        return ST_OK, None
    if x0 >= P or x1 >= P:
        return ST_X_NOT_CANONICAL, None
    x = (x0, x1)
    y2 = f2_add(f2_mul(f2_sqr(x), x), B_G2)
    y = f2_sqrt(y2)
    if y is None:
        return ST_NOT_ON_CURVE, None
    if f2_lex_largest(y) != bool(sort):
        y = f2_neg(y)
    pt = (x, y)
    if check_subgroup and not g2_in_subgroup(pt):
        return ST_NOT_IN_SUBGROUP, None
    return ST_OK, pt


def g1_to_mont_u64(pt):
    """ABI layout of an affine G1 point: x[6], y[6] Montgomery u64 limbs."""
    if pt is None:
        return [0] * 6 + mont_limbs(1)   # ic_bls12_381 identity: x = 0, y = 1
    return mont_limbs(pt[0]) + mont_limbs(pt[1])


def g1_from_mont_u64(limbs):
    return (from_mont_limbs(limbs[:6]), from_mont_limbs(limbs[6:12]))


# ----------------------------------------------------------------------------
# Hash to G1: RFC 9380 hash_to_curve, suite BLS12381G1_XMD:SHA-256_SSWU_RO_
# ----------------------------------------------------------------------------

def expand_message_xmd(msg, dst, len_in_bytes):
    """RFC 9380 section 5.3.1 with H = SHA-256 (b = 32, s = 64 bytes)."""
    b_in, s_in = 32, 64
    ell = (len_in_bytes + b_in - 1) // b_in
    assert ell <= 255 and len_in_bytes <= 65535 and len(dst) <= 255
    dst_prime = dst + bytes([len(dst)])
    msg_prime = bytes(s_in) + msg + len_in_bytes.to_bytes(2, "big") + b"\x00" + dst_prime
    b0 = hashlib.sha256(msg_prime).digest()
    bi = hashlib.sha256(b0 + b"\x01" + dst_prime).digest()
    out = bi
    for i in range(2, ell + 1):
        bi = hashlib.sha256(bytes(x ^ y for x, y in zip(b0, bi)) + bytes([i]) + dst_prime).digest()
        out += bi
    return out[:len_in_bytes]


def hash_to_field_fp(msg, dst, count=2):
    """RFC 9380 section 5.2 for Fp (m = 1, L = 64)."""
    L = 64
    ub = expand_message_xmd(msg, dst, count * L)
    return [int.from_bytes(ub[L * i:L * (i + 1)], "big") % P for i in range(count)]


def _sgn0(x):
    return x & 1


# E': y^2 = x^3 + A' x + B', 11-isogenous to E (RFC 9380 section 8.8.1).  The
# published coefficients are accepted because points of E' have orders that
# divide #E(Fp) (tests/test_oracle.py checks it).
SSWU_A = 0x144698a3b8e9433d693a02c96d4982b0ea985383ee66a8d8e8981aefd881ac98936f8da0e0f97f5cf428082d584c1d
SSWU_B = 0x12e2908d11688030018b12e8753eee3b2016c1f0f24f4070a0b9c14fcef35ef55a23215a316ceaa5d1cc48e98e172be0
# constant terms of the x and y numerators of the suite's isogeny map (RFC 9380
# appendix E.2): they fix which of the six isomorphisms onto y^2 = x^3 + 4
# the map uses
ISO_X_NUM0 = 0x11a05f2b1e833340b809101dd99815856b303e88a2d7005ff2627b56cdb4e2c85610c2d5f2e62d6eaeac1662734649b7
ISO_Y_NUM0 = 0x90d97c81ba24ee0259d1f094980dcfa11ad138e48a869522b52af6c956543d3cd0c7aee9b3ba3c2be9845719707bb33
N_G1_CURVE = P + BLS_X                   # #E(Fp) = p + 1 - t, trace t = x + 1 = 1 - |x|


def _g_iso(x):
    return (x * x * x + SSWU_A * x + SSWU_B) % P


def _iso_add(a, b):
    """affine addition on E' (None is the identity)"""
    if a is None:
        return b
    if b is None:
        return a
    (x1, y1), (x2, y2) = a, b
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        lam = (3 * x1 * x1 + SSWU_A) * fp_inv(2 * y1 % P) % P
    else:
        lam = (y2 - y1) * fp_inv((x2 - x1) % P) % P
    x3 = (lam * lam - x1 - x2) % P
    return (x3, (lam * (x1 - x3) - y1) % P)


def _iso_mul(a, k):
    r = None
    while k:
        if k & 1:
            r = _iso_add(r, a)
        a = _iso_add(a, a)
        k >>= 1
    return r


def _ptrim(a):
    while a and a[-1] % P == 0:
        a = a[:-1]
    return a


def _pmul(a, b):
    r = [0] * (len(a) + len(b) - 1) if a and b else []
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            r[i + j] = (r[i + j] + x * y) % P
    return _ptrim(r)


def _prem(a, b):
    """a mod b (coefficient lists, index = degree; b nonzero)"""
    a, inv_lead = list(a), fp_inv(b[-1])
    while len(a) >= len(b):
        c, d = a[-1] * inv_lead % P, len(a) - len(b)
        for i, y in enumerate(b):
            a[d + i] = (a[d + i] - c * y) % P
        a = _ptrim(a)
    return a


def _cubic_has_root(c0, c1):
    """x^3 + c1 x + c0 has a root in Fp iff gcd(x^p - x, it) is not 1"""
    cubic, xp, base, e = [c0 % P, c1 % P, 0, 1], [1], [0, 1], P
    while e:
        if e & 1:
            xp = _prem(_pmul(xp, base), cubic)
        base = _prem(_pmul(base, base), cubic)
        e >>= 1
    a, b = cubic, _ptrim([(xp[i] if i < len(xp) else 0) - (1 if i == 1 else 0) for i in range(3)])
    b = [v % P for v in b]
    while b:
        a, b = b, _prem(a, b)
    return len(a) > 1


def _find_z_sswu():
    """RFC 9380 appendix H.2: Z non-square, Z != -1, g(x) - Z irreducible,
    g(B / (Z A)) square; smallest |Z| first, positive before negative."""
    ctr = 1
    while True:
        for z in (ctr % P, (-ctr) % P):
            if fp_is_square(z) or z == P - 1:
                continue
            if _cubic_has_root((SSWU_B - z) % P, SSWU_A):
                continue
            if not fp_is_square(_g_iso(SSWU_B * fp_inv(z * SSWU_A % P) % P)):
                continue
            return z
        ctr += 1


SSWU_Z = _find_z_sswu()


def map_to_curve_sswu(u):
    """RFC 9380 section 6.6.2 (the map's definition, steps 1-10) to E'."""
    tv1 = (SSWU_Z * SSWU_Z * pow(u, 4, P) + SSWU_Z * u * u) % P
    tv1 = fp_inv(tv1) if tv1 else 0
    if tv1 == 0:
        x1 = SSWU_B * fp_inv(SSWU_Z * SSWU_A % P) % P
    else:
        x1 = (-SSWU_B) * fp_inv(SSWU_A) % P * (1 + tv1) % P
    gx1 = _g_iso(x1)
    x2 = SSWU_Z * u * u % P * x1 % P
    if fp_is_square(gx1):
        x, y = x1, fp_sqrt(gx1)
    else:
        x, y = x2, fp_sqrt(_g_iso(x2))
    if _sgn0(u) != _sgn0(y):
        y = (-y) % P
    return (x, y)


def _iso_kernel():
    """the five points of a rational subgroup of order 11 of E', one of each
    pair +-Q: (N / 11) times points of E' until the result is not O"""
    x = 1
    while True:
        x += 1
        if not fp_is_square(_g_iso(x)):
            continue
        q = _iso_mul((x, fp_sqrt(_g_iso(x))), N_G1_CURVE // 11)
        if q is not None:
            assert _iso_mul(q, 11) is None
            out, acc = [], q
            for _ in range(5):
                out.append(acc)
                acc = _iso_add(acc, q)
            return out


_ISO_KERNEL = _iso_kernel()


def _velu(x):
    """Velu's isogeny with the kernel above at abscissa x: (X(x), X'(x)), the
    image being (X, y X'); None at a kernel abscissa"""
    X, dX = x, 1
    for xq, yq in _ISO_KERNEL:
        h = (x - xq) % P
        if h == 0:
            return None
        v = (6 * xq * xq + 2 * SSWU_A) % P
        w = 4 * yq * yq % P
        hi = fp_inv(h)
        X = (X + v * hi + w * hi * hi) % P
        dX = (dX - v * hi * hi - 2 * w * hi * hi % P * hi) % P
    return X, dX


def _iso_normalisation():
    """(u^2, u^3) of the isomorphism onto y^2 = x^3 + 4, fixed by the suite's
    two published coefficients: x_num(0) = u^2 X(0) D(0)^2 and
    y_num(0) = u^3 X'(0) D(0)^3, D the kernel polynomial"""
    d0 = 1
    for xq, _ in _ISO_KERNEL:
        d0 = d0 * (-xq) % P
    X0, dX0 = _velu(0)
    u2 = ISO_X_NUM0 * fp_inv(X0 * d0 * d0 % P) % P
    u3 = ISO_Y_NUM0 * fp_inv(dX0 * pow(d0, 3, P) % P) % P
    assert pow(u2, 3, P) == u3 * u3 % P, "the two coefficients give one isomorphism"
    return u2, u3


ISO_U2, ISO_U3 = _iso_normalisation()


def iso_map(pt):
    """E' -> E (affine; None for the identity)"""
    if pt is None:
        return None
    x, y = pt
    v = _velu(x)
    if v is None:
        return None
    return (ISO_U2 * v[0] % P, ISO_U3 * y % P * v[1] % P)


def hash_to_g1(msg, dst):
    u0, u1 = hash_to_field_fp(msg, dst, 2)
    q = g1_add(iso_map(map_to_curve_sswu(u0)), iso_map(map_to_curve_sswu(u1)))
    return g1_mul(q, H_EFF_G1)
