"""Seeded BLS inputs built with the Python oracle, for small test cases.

The generation rules match the workload generator the bench uses (SplitMix64
stream, scalars by rejection in [1, r), 32-byte messages, RFC 9380 hash with the
bench domain string, 1-in-8 corruptions), so small cases here and the bench's
inputs come from one definition.
"""
import numpy as np

import bls_ref as B

DST = b"BLS_BENCH_G1_XMD:SHA-256_SVDW_RO_"
M64 = (1 << 64) - 1


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
            if 0 < v < B.R_ORDER:
                return v

    def msg(self):
        return b"".join(self.next().to_bytes(8, "little") for _ in range(4))

    def below(self, n):
        return self.next() % n


def g2_affine_u64(q):
    return B.mont_limbs(q[0][0]) + B.mont_limbs(q[0][1]) + B.mont_limbs(q[1][0]) + B.mont_limbs(q[1][1])


def plain_config(n=64, seed=1, corrupt_every=8):
    """n independent keys, one message each; item i with i % corrupt_every ==
    corrupt_every - 1 gets a one-bit message flip (expected reject)."""
    rng = SplitMix64(seed)
    sigs, nhms, pk_tabs, pk_aff, expect, sig_pts = [], [], [], [], [], []
    for i in range(n):
        sk = rng.scalar()
        msg = rng.msg()
        pk = B.g2_mul(B.G2_GEN, sk)
        h = B.hash_to_g1(msg, DST)
        sig = B.g1_mul(h, sk)
        ok = True
        if corrupt_every and i % corrupt_every == corrupt_every - 1:
            m2 = bytearray(msg)
            m2[rng.below(32)] ^= 1 << rng.below(8)
            h = B.hash_to_g1(bytes(m2), DST)
            ok = False
        sigs.append(B.g1_to_mont_u64(sig))
        sig_pts.append(sig)
        nhms.append(B.g1_to_mont_u64(B.g1_neg(h)))
        pk_tabs.append(B.coeffs_to_limbs(B.g2_prepare(pk)))
        pk_aff.append(g2_affine_u64(pk))
        expect.append(1 if ok else 0)
    return {
        "sigs": np.array(sigs, dtype=np.uint64), "nhms": np.array(nhms, dtype=np.uint64),
        "pk_tabs": np.array(pk_tabs, dtype=np.uint64), "pk_affine": np.array(pk_aff, dtype=np.uint64),
        "expect": np.array(expect, dtype=np.int32), "sig_points": sig_pts,
    }


def random_curve_point_not_in_g1(rng):
    """A point on y^2 = x^3 + 4 outside the order-r subgroup."""
    while True:
        x = rng.scalar() % B.P
        y2 = (x ** 3 + 4) % B.P
        if B.fp_is_square(y2):
            pt = (x, B.fp_sqrt(y2))
            if not B.g1_in_subgroup(pt):
                return pt


def x_not_on_curve(rng):
    while True:
        x = rng.scalar() % B.P
        if not B.fp_is_square((x ** 3 + 4) % B.P):
            return x


def invalid_encodings(rng, valid_point):
    """(bytes, expected status) for each invalid-encoding class."""
    out = []
    good = bytearray(B.g1_compress(valid_point))
    b = bytearray(good); b[0] &= 0x7F
    out.append((bytes(b), B.ST_BAD_FLAGS))                        # compression bit clear
    b = bytearray(48); b[0] = 0xC0; b[47] = 1
    out.append((bytes(b), B.ST_BAD_FLAGS))                        # infinity with payload
    b = bytearray(48); b[0] = 0xE0
    out.append((bytes(b), B.ST_BAD_FLAGS))                        # infinity with sort bit
    b = bytearray(B.P.to_bytes(48, "big")); b[0] |= 0x80
    out.append((bytes(b), B.ST_X_NOT_CANONICAL))                  # x = p
    b = bytearray(((1 << 381) - 1).to_bytes(48, "big")); b[0] |= 0x80
    out.append((bytes(b), B.ST_X_NOT_CANONICAL))                  # x = 2^381 - 1
    x = x_not_on_curve(rng)
    b = bytearray(x.to_bytes(48, "big")); b[0] |= 0x80
    out.append((bytes(b), B.ST_NOT_ON_CURVE))
    pt = random_curve_point_not_in_g1(rng)
    out.append((B.g1_compress(pt), B.ST_NOT_IN_SUBGROUP))
    return out
