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
        "expect": c["expect"], "sig_points": [B.g1_from_mont_u64(s) for s in c["sigs"]],
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
