"""Small test inputs: the bench's workload generator (icp-gpu_b200/workload.py)
plus invalid encodings built with the Python oracle."""
import numpy as np

import bls_ref as B

import workload as WL

DST = WL.DST
SplitMix64 = WL.SplitMix64


def g2_affine_u64(q):
    return B.mont_limbs(q[0][0]) + B.mont_limbs(q[0][1]) + B.mont_limbs(q[1][0]) + B.mont_limbs(q[1][1])


def plain_config(n=64, seed=1):
    """The plain workload from the workload generator, plus the signatures as oracle
    points (for encoding tests)."""
    c = WL.config_plain(n, seed)
    return {
        "sigs": c["sigs"], "nhms": c["nhms"], "pk_tabs": c["pk_tables"], "pk_affine": c["pk_affine"],
        "expect": c["expect"], "sig_points": [B.g1_from_mont_u64(s) for s in c["sigs"]], "msgs": c["msgs"],
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


def g2_random_x(rng, square):
    """x in Fp2 with x^3 + 4(1 + u) a square (square=True) or not."""
    while True:
        x = (rng.scalar() % B.P, rng.scalar() % B.P)
        y2 = B.f2_add(B.f2_mul(B.f2_sqr(x), x), B.B_G2)
        if B.f2_is_square(y2) == square:
            return x, y2


def g2_encode_x(x, flags):
    b = bytearray(x[1].to_bytes(48, "big") + x[0].to_bytes(48, "big"))
    b[0] |= flags
    return bytes(b)


def invalid_g2_encodings(rng, valid_point):
    """(bytes, expected status) for each invalid class of 96-byte G2 encodings."""
    out = []
    good = bytearray(B.g2_compress(valid_point))
    b = bytearray(good); b[0] &= 0x7F
    out.append((bytes(b), B.ST_BAD_FLAGS))                        # compression bit clear
    for pos in (95, 47, 1):                                       # infinity with payload in x.c0 / x.c1
        b = bytearray(96); b[0] = 0xC0; b[pos] = 1
        out.append((bytes(b), B.ST_BAD_FLAGS))
    b = bytearray(96); b[0] = 0xE0
    out.append((bytes(b), B.ST_BAD_FLAGS))                        # infinity with sort bit
    out.append((g2_encode_x((B.P, 0), 0x80), B.ST_X_NOT_CANONICAL))          # x.c0 = p
    out.append((g2_encode_x((0, B.P), 0x80), B.ST_X_NOT_CANONICAL))          # x.c1 = p
    out.append((g2_encode_x((1, (1 << 381) - 1), 0xA0), B.ST_X_NOT_CANONICAL))
    out.append((g2_encode_x(((1 << 381) - 1, 5), 0x80), B.ST_X_NOT_CANONICAL))
    x, _ = g2_random_x(rng, False)
    out.append((g2_encode_x(x, 0x80), B.ST_NOT_ON_CURVE))
    out.append((g2_encode_x(x, 0xA0), B.ST_NOT_ON_CURVE))
    x, y2 = g2_random_x(rng, True)                                # on the twist, outside G2
    out.append((g2_encode_x(x, 0x80), B.ST_NOT_IN_SUBGROUP))
    out.append((g2_encode_x(x, 0xA0), B.ST_NOT_IN_SUBGROUP))
    return out
