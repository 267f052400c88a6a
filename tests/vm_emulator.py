"""Python re-statement of the lane-parallel kernel's driver (verify_vm.cu) over
the generated program tables, bit-exact with the device arithmetic.  Test
infrastructure: lets the CPU suite check the tables and the group plan of the
final exponentiation against the oracle without a GPU."""
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "icp-gpu_b200", "csrc"))
import gen_programs as G  # noqa: E402

import bls_ref as B  # noqa: E402

X_ABS = 0xD201000000010000
K_SLOTS = 8
GROUPS = 8


class Machine:
    def __init__(self, lanes):
        self.progs = {p.name: p for p in G.build_all(lanes)}
        self.ntemp = max(p.ntemp for p in self.progs.values())
        self.slots = {}
        one = G.R % G.P
        k = [0, one, 0, B.mont_limbs(0)[0] * 0 + self._m(B.FROB6_C1[1]), self._m(B.FROB6_C2[0]), 0,
             self._m(B.FROB12_C1[0]), self._m(B.FROB12_C1[1])]
        for i, v in enumerate(k):
            self.slots[i] = v
        self.region = K_SLOTS
        self.temp = self.region + 12 * GROUPS
        for s in range(self.region, self.temp + 96):
            self.slots[s] = 0

    @staticmethod
    def _m(x):
        return x * G.R % G.P

    def grp(self, g):
        return self.region + 12 * g

    def call(self, name, d, a=0, b=0):
        bases = [self.grp(d), self.grp(a), self.grp(b), self.grp(1), 0, self.temp, self.temp + 32, self.temp + 64]
        G.run_program(self.progs[name], self.slots, bases)

    def set_group(self, g, vals):
        for i, v in enumerate(vals):
            self.slots[self.grp(g) + i] = v

    def group(self, g):
        return [self.slots[self.grp(g) + i] % G.P for i in range(12)]


def cyc_exp(m, dst, x, spare):
    m.call("COPY", dst, x)
    cur, oth = dst, spare
    for i in range(62, -1, -1):
        m.call("CYCSQR", cur)
        if (X_ABS >> i) & 1:
            m.call("MUL", oth, cur, x)
            cur, oth = oth, cur
    m.call("CONJ", dst, cur)


def final_exp(m):
    c = m.call
    c("CONJ", 1, 0); c("INV", 2, 0); c("MUL", 3, 1, 2); c("FROB", 0, 3); c("FROB", 1, 0); c("MUL", 2, 1, 3)
    c("COPY", 0, 2); c("CYCSQR", 0); c("CONJ", 0, 0)
    cyc_exp(m, 1, 2, 3)
    c("MUL", 3, 0, 1)
    cyc_exp(m, 0, 3, 4)
    c("CONJ", 3, 3); c("MUL", 4, 2, 3); c("COPY", 3, 1); c("CYCSQR", 3)
    cyc_exp(m, 5, 0, 6)
    c("MUL", 6, 1, 5); c("FROB", 1, 6); c("FROB", 6, 1); c("MUL", 1, 4, 6)
    cyc_exp(m, 4, 5, 6)
    c("MUL", 5, 3, 4)
    cyc_exp(m, 3, 5, 4)
    c("MUL", 4, 1, 3); c("CONJ", 1, 2); c("MUL", 3, 5, 1); c("MUL", 1, 2, 0)
    c("FROB", 0, 1); c("FROB", 2, 0); c("FROB", 0, 2); c("MUL", 1, 4, 0); c("FROB", 2, 3); c("MUL", 0, 1, 2)


def verify(lanes, sig, nhm, g2_limbs, pk_limbs, skip1=False, skip2=False):
    """sig / nhm: canonical affine points; tables: 2448 u64.  Returns
    (miller, gt) as canonical flat Fp lists."""
    m = Machine(lanes)
    C = m.grp(1)
    one = G.R % G.P
    pts = [(0, 0) if skip1 else sig, (0, 0) if skip2 else nhm]
    for pair in range(2):
        m.slots[C + 8 * pair + 6] = pts[pair][0] * G.R % G.P
        m.slots[C + 8 * pair + 7] = pts[pair][1] * G.R % G.P
    m.set_group(0, [one] + [0] * 11)

    def load(ci):
        for pair, (tab, skip) in enumerate(((g2_limbs, skip1), (pk_limbs, skip2))):
            for k in range(6):
                if skip:
                    v = one if k == 4 else 0
                else:
                    w = tab[36 * ci + 6 * k: 36 * ci + 6 * k + 6]
                    v = sum(int(x) << (64 * i) for i, x in enumerate(w))
                m.slots[C + 8 * pair + k] = v

    ci = 0
    for b in range(61, -1, -1):
        load(ci); ci += 1
        m.call("LINE2", 0)
        if ((X_ABS >> 1) >> b) & 1:
            load(ci); ci += 1
            m.call("LINE2", 0)
        m.call("SQR", 0)
    load(ci)
    m.call("LINE2", 0)
    m.call("CONJ", 0, 0)
    ml = [v * B.MONT_RINV % B.P for v in m.group(0)]
    final_exp(m)
    gt = [v * B.MONT_RINV % B.P for v in m.group(0)]
    return ml, gt
