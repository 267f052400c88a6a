"""CPU tests of the generated tower programs (icp-gpu_b200/csrc/gen_programs.py):
each program, run in the bit-exact emulator on redundant inputs (any
representative below 8p), gives the oracle's value; the whole verify driven
through the programs reproduces the reference's golden Miller and Gt values."""
import random

import numpy as np
import pytest

import bls_ref as B
import gen_programs as G
import vm_emulator as E

LANES = [8, 4]


def rand_rep(rng, x):
    """a random representative of x below 8p, in Montgomery form"""
    m = x * G.R % G.P
    return m + G.P * rng.randrange(0, 7)


def rand_f12(rng):
    return [rng.randrange(G.P) for _ in range(12)]


def to_f12(vals):
    return B.f12_from_flat(vals)


@pytest.mark.parametrize("lanes", LANES)
def test_programs_against_oracle(lanes):
    rng = random.Random(lanes)
    m = E.Machine(lanes)
    for _ in range(3):
        a, b = rand_f12(rng), rand_f12(rng)
        m.set_group(3, [rand_rep(rng, v) for v in a])
        m.set_group(4, [rand_rep(rng, v) for v in b])
        checks = [
            ("MUL", (5, 3, 4), B.f12_mul(to_f12(a), to_f12(b))),
            ("FROB", (5, 3), B.f12_frob(to_f12(a))),
            ("CONJ", (5, 3), B.f12_conj(to_f12(a))),
            ("COPY", (5, 3), to_f12(a)),
            ("INV", (5, 3), B.f12_inv(to_f12(a))),
        ]
        for name, args, want in checks:
            m.call(name, *args)
            got = [v * B.MONT_RINV % B.P for v in m.group(5)]
            assert got == B.f12_flat(want), name
        for name, fn in (("SQR", B.f12_sqr), ("CYCSQR", B.f12_cyclotomic_square)):
            m.set_group(6, [rand_rep(rng, v) for v in a])
            m.call(name, 6)
            got = [v * B.MONT_RINV % B.P for v in m.group(6)]
            assert got == B.f12_flat(fn(to_f12(a))), name


@pytest.mark.parametrize("lanes", LANES)
def test_line2_against_oracle(lanes):
    rng = random.Random(17)
    m = E.Machine(lanes)
    f = rand_f12(rng)
    co = [[(rng.randrange(B.P), rng.randrange(B.P)) for _ in range(3)] for _ in range(2)]
    pts = [(rng.randrange(B.P), rng.randrange(B.P)) for _ in range(2)]
    m.set_group(0, [rand_rep(rng, v) for v in f])
    C = m.grp(1)
    for pair in range(2):
        for k in range(3):
            m.slots[C + 8 * pair + 2 * k] = rand_rep(rng, co[pair][k][0])
            m.slots[C + 8 * pair + 2 * k + 1] = rand_rep(rng, co[pair][k][1])
        m.slots[C + 8 * pair + 6] = rand_rep(rng, pts[pair][0])
        m.slots[C + 8 * pair + 7] = rand_rep(rng, pts[pair][1])
    m.call("LINE2", 0)
    want = to_f12(f)
    for pair in range(2):
        want = B._ell(want, tuple(co[pair]), pts[pair][0], pts[pair][1])
    assert [v * B.MONT_RINV % B.P for v in m.group(0)] == B.f12_flat(want)


@pytest.mark.parametrize("lanes", [8])
def test_full_verify_through_programs(lanes, golden):
    sig = B.g1_from_mont_u64(golden["sig_294_g1"])
    nhm = B.g1_from_mont_u64(golden["neg_hm_7_g1"])
    ml, gt = E.verify(lanes, sig, nhm, golden["g2_gen_coeffs"], golden["pk42_coeffs"])
    assert B.f12_mont_limbs(B.f12_from_flat(ml))[:6] == list(golden["ml_2pair_c000"])
    assert B.f12_from_flat(gt) == B.F12_ONE
    # e(G1, G2) alone: the second pair skipped
    ml, gt = E.verify(lanes, B.G1_GEN, None, golden["g2_gen_coeffs"], golden["pk42_coeffs"], skip2=True)
    assert B.f12_mont_limbs(B.f12_from_flat(ml)) == list(golden["ml_g1_g2"])
    assert B.f12_mont_limbs(B.f12_from_flat(gt)) == list(golden["pairing_g1_g2"])


def test_generated_header_is_current():
    """programs.inc matches what the generator produces now."""
    import os
    import tempfile
    path = os.path.join(os.path.dirname(G.__file__), "programs.inc")
    with tempfile.NamedTemporaryFile("r", suffix=".inc", delete=False) as tf:
        G.emit(G.LANE_OPTIONS, tf.name)
        fresh = open(tf.name).read()
    os.unlink(tf.name)
    assert open(path).read() == fresh
