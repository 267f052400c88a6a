"""Python re-statement of the Fp2-lane verify kernel's driver (verify_fp2.cu)
over the generated descriptor tables (gen_fp2ops.py), bit-exact with the
device arithmetic: the same accumulators, biases, reductions and slot plan.
Test infrastructure: lets the CPU suite check the tables, the bounds and the
group plan of the final exponentiation against the oracle without a GPU."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "icp-gpu_b200", "csrc"))
import gen_fp2ops as G  # noqa: E402

import bls_ref as B  # noqa: E402

X_ABS = G.X_ABS


K_SLOTS = 8
GROUPS = 7
T_GROUP = G.T_GROUP  # inversion temporaries start at group 3 (13 slots)
C_OFF = 6 * GROUPS   # C area after the groups


def mont(x):
    return x * G.R % G.P


def f2m(a):
    return (mont(a[0]), mont(a[1]))


def frob_constants():
    """conj(g) for g in k1, k2, k12, k1 k12, k2 k12 (Montgomery Fp2)."""
    k1, k2, k12 = B.FROB6_C1, B.FROB6_C2, B.FROB12_C1
    gs = [k1, k2, k12, B.f2_mul(k1, k12), B.f2_mul(k2, k12)]
    return [f2m(B.f2_conj(g)) for g in gs]


class Machine:
    def __init__(self):
        self.e = G.Emulator(G.build())
        self.slots = {}
        ks = G.k_slot_values()
        for i, v in enumerate(ks):
            self.slots[i] = v
        self.region = K_SLOTS
        for s in range(self.region, self.region + C_OFF + 12):
            self.slots[s] = (0, 0)

    def grp(self, g):
        return self.region + 6 * g

    def call(self, name, d, a=0, b=0):
        bases = [self.grp(d), self.grp(a), self.grp(b), self.region + C_OFF, 0, self.grp(T_GROUP)]
        self.e.run(name, self.slots, bases)

    def inv(self, d, a):
        for k in range(1, 8):
            self.call("INV%d" % k, d, a)
        self.call("INV8", d, a)

    def set_group(self, g, f2s):
        for i, v in enumerate(f2s):
            self.slots[self.grp(g) + i] = v

    def group_flat(self, g):
        out = []
        for i in range(6):
            re, im = self.slots[self.grp(g) + i]
            out += [re % G.P, im % G.P]
        return out


def table_f2(tab, ci, k):
    w = [int(x) for x in tab[36 * ci + 12 * k: 36 * ci + 12 * k + 12]]
    return (sum(x << (64 * i) for i, x in enumerate(w[:6])), sum(x << (64 * i) for i, x in enumerate(w[6:])))


def normalise_table(tab):
    """(coefficient rows (c0 / c2, c1 / c2, 1) in Montgomery form, Miller
    correction factor): the line table divided row by row by its c2, and
    prod_i c2_i^(2^(squarings after line i)), both as Montgomery Fp2."""
    def dec(v):
        return (v[0] * B.MONT_RINV % B.P, v[1] * B.MONT_RINV % B.P)

    rows, corr = [], B.F2_ONE if hasattr(B, "F2_ONE") else (1, 0)
    ci = 0

    def line():
        nonlocal ci, corr
        c0, c1, c2 = (dec(table_f2(tab, ci, k)) for k in range(3))
        inv = B.f2_inv(c2)
        rows.append((f2m(B.f2_mul(c0, inv)), f2m(B.f2_mul(c1, inv)), (mont(1), 0)))
        corr = B.f2_mul(corr, c2)
        ci += 1

    for b in range(61, -1, -1):
        line()
        if ((X_ABS >> 1) >> b) & 1:
            line()
        corr = B.f2_mul(corr, corr)
    line()
    return rows, f2m(corr)


def verify(sig, nhm, g2_limbs, pk_limbs, skip1=False, skip2=False, normalised=False):
    """sig / nhm: canonical affine points; tables: 2448 u64.  Returns
    (miller, gt) as canonical flat Fp lists (normal form).  `normalised` runs
    the normalised-line sequence and multiplies the Miller value back by the
    two correction factors, as the kernel does for registered keys."""
    m = Machine()
    C = m.region + C_OFF
    one = mont(1)
    pts = [(0, 0) if skip1 else sig, (0, 0) if skip2 else nhm]
    for pair in range(2):
        m.slots[C + 6 * pair + G.C_PT] = (mont(pts[pair][0]), mont(pts[pair][1]))
    m.set_group(0, [(one, 0)] + [(0, 0)] * 5)
    norm = [normalise_table(g2_limbs), normalise_table(pk_limbs)] if normalised else None

    def load(ci):
        for pair, (tab, skip) in enumerate(((g2_limbs, skip1), (pk_limbs, skip2))):
            for k in range(3):
                if skip:
                    v = (one, 0) if k == 2 else (0, 0)
                elif normalised:
                    v = norm[pair][0][ci][k]
                else:
                    v = table_f2(tab, ci, k)
                m.slots[C + 6 * pair + k] = v

    names = [name for name, _, _ in G.PROGRAMS]
    ml = None
    for code, d, a, b, ci in G.driver_sequence(normalised):
        code &= ~G.COND_ML          # the Miller value is always wanted here
        if code == G.OP_LOAD_LINES:
            load(ci)
        elif code == G.OP_LOAD_CORR:
            for pair, skip in enumerate((skip1, skip2)):
                m.slots[C + 6 * pair + G.C_C2] = (one, 0) if skip else norm[pair][1]
        elif code == G.OP_MILLER_DONE:
            ml = [v * B.MONT_RINV % B.P for v in m.group_flat(d)]
        else:
            m.call(names[code], d, a, b)
    gt = [v * B.MONT_RINV % B.P for v in m.group_flat(G.gt_group(normalised))]
    return ml, gt
