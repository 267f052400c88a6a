"""CPU tests of the Fp2-lane tower programs (icp-gpu_b200/csrc/gen_fp2ops.py):
each program, run in the bit-exact emulator on redundant inputs (random
representatives below the slot bound 2^381 + p), gives the oracle's value; the
whole verify driven through the programs reproduces the reference's golden
Miller-loop and pairing values; the emitted tables are current."""
import os
import random
import tempfile

import pytest

import bls_ref as B
import fp2_emulator as E
import gen_fp2ops as G


def rep(rng, x):
    """a random representative of x (normal form) below the slot bound, Montgomery"""
    m = x * G.R % G.P
    while True:
        v = m + G.P * rng.randrange(0, 3)
        if v < G.SLOT_BOUND:
            return v


def rand_f12(rng):
    return [rng.randrange(G.P) for _ in range(12)]


def set_f12(m, g, flat, rng):
    m.set_group(g, [(rep(rng, flat[2 * i]), rep(rng, flat[2 * i + 1])) for i in range(6)])


def got(m, g):
    return [v * B.MONT_RINV % B.P for v in m.group_flat(g)]


def test_programs_against_oracle():
    rng = random.Random(5)
    m = E.Machine()
    for _ in range(3):
        a, b = rand_f12(rng), rand_f12(rng)
        fa, fb = B.f12_from_flat(a), B.f12_from_flat(b)
        checks = [
            ("MUL", (5, 3, 4), B.f12_mul(fa, fb)),
            ("SQR", (5, 3), B.f12_sqr(fa)),
            ("CYCSQR", (5, 3), B.f12_cyclotomic_square(fa)),
            ("FROB", (5, 3), B.f12_frob(fa)),
            ("CONJ", (5, 3), B.f12_conj(fa)),
            ("COPY", (5, 3), fa),
        ]
        for name, args, want in checks:
            set_f12(m, 3, a, rng)
            set_f12(m, 4, b, rng)
            m.call(name, *args)
            assert got(m, 5) == B.f12_flat(want), name
        # in place, as the driver calls them
        for name, fn in (("SQR", B.f12_sqr), ("CYCSQR", B.f12_cyclotomic_square), ("CONJ", B.f12_conj)):
            set_f12(m, 6, a, rng)
            m.call(name, 6, 6)
            assert got(m, 6) == B.f12_flat(fn(fa)), name + " in place"
        set_f12(m, 0, a, rng)
        m.inv(2, 0)
        assert got(m, 2) == B.f12_flat(B.f12_inv(fa)), "INV"


def test_lines_against_oracle():
    rng = random.Random(17)
    m = E.Machine()
    f = rand_f12(rng)
    co = [[(rng.randrange(B.P), rng.randrange(B.P)) for _ in range(3)] for _ in range(2)]
    pts = [(rng.randrange(B.P), rng.randrange(B.P)) for _ in range(2)]
    set_f12(m, 0, f, rng)
    C = m.region + E.C_OFF
    for pair in range(2):
        for k in range(3):
            m.slots[C + 6 * pair + k] = (rep(rng, co[pair][k][0]), rep(rng, co[pair][k][1]))
        m.slots[C + 6 * pair + G.C_PT] = (rep(rng, pts[pair][0]), rep(rng, pts[pair][1]))
    m.call("LSCALE", 0)
    m.call("LINE1", 0, 0)
    m.call("LINE2", 0, 0)
    want = B.f12_from_flat(f)
    for pair in range(2):
        want = B._ell(want, tuple(co[pair]), pts[pair][0], pts[pair][1])
    assert got(m, 0) == B.f12_flat(want)


def test_inverse_of_zero_is_zero():
    m = E.Machine()
    m.set_group(0, [(0, 0)] * 6)
    m.inv(2, 0)
    assert got(m, 2) == [0] * 12


@pytest.mark.parametrize("normalised", [False, True], ids=["raw-lines", "normalised-lines"])
def test_full_verify_through_programs(golden, normalised):
    sig = B.g1_from_mont_u64(golden["sig_294_g1"])
    nhm = B.g1_from_mont_u64(golden["neg_hm_7_g1"])
    ml, gt = E.verify(sig, nhm, golden["g2_gen_coeffs"], golden["pk42_coeffs"], normalised=normalised)
    assert B.f12_mont_limbs(B.f12_from_flat(ml))[:6] == list(golden["ml_2pair_c000"])
    assert B.f12_from_flat(gt) == B.F12_ONE
    # e(G1, G2) alone: the second pair skipped
    ml, gt = E.verify(B.G1_GEN, None, golden["g2_gen_coeffs"], golden["pk42_coeffs"], skip2=True,
                      normalised=normalised)
    assert B.f12_mont_limbs(B.f12_from_flat(ml)) == list(golden["ml_g1_g2"])
    assert B.f12_mont_limbs(B.f12_from_flat(gt)) == list(golden["pairing_g1_g2"])


def test_constant_slots_match_oracle():
    """the generator's Frobenius constants are the oracle's (conjugated)"""
    ks = G.k_slot_values()
    assert ks[0] == (0, 0) and ks[1] == (E.mont(1), 0)
    assert ks[2:7] == E.frob_constants()


def test_static_bounds_hold():
    """every output's worst-case accumulator fits the device's limits"""
    for name, outs, _ in G.build():
        for o in outs:
            if o is None or o.mode not in (G.M_SIMPLE, G.M_FULL):
                continue
            assert o.bias_re < 256 and o.bias_im < 256, name


def test_generated_header_is_current():
    path = os.path.join(os.path.dirname(G.__file__), "fp2ops.inc")
    with tempfile.NamedTemporaryFile("r", suffix=".inc", delete=False) as tf:
        G.emit(tf.name)
        fresh = open(tf.name).read()
    os.unlink(tf.name)
    assert open(path).read() == fresh


def test_bench_counts_match_the_sequence():
    """The own-work figures bench.py reports are the generated sequence's."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    progs = {i: fn() for i, (name, fn, _) in enumerate(G.PROGRAMS)}
    prods = redcs = 0
    for code, d, a, b, ci in G.driver_sequence(True):
        if code & G.COND_ML or code >= len(G.PROGRAMS):
            continue
        for o in progs[code]:
            if o is None:
                continue
            prods += G.half_products(o, 0) + G.half_products(o, 1)
            redcs += 2 if o.mode in (G.M_SIMPLE, G.M_FULL) else 0
    assert (prods, redcs) == (bench.OWN_PRODUCTS_PER_VERIFY, bench.OWN_REDC_PER_VERIFY)
