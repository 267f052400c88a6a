"""Tower-program generator for the lane-parallel verify kernel.

Each tower operation of the verify path (line evaluation, Fp12 squaring and
multiplication, cyclotomic squaring, Frobenius, inversion) is written here
once over symbolic Fp values, following the reference's formulas
(gpu-crypto/cuda/field_sppark.cuh:52-197, gpu-crypto/cuda/api.cu:22-78).  The
generator turns each into a straight-line program of Fp-level operations

  MUL  dst = REDC(A * B)       A, B: one slot, or a signed sum of slots
  LIN  dst = reduce(sum of signed slots)
  INV  dst = src^(p-2)         (one lane; Fermat, as field_sppark.cuh:40-50)

scheduled into rounds of at most T operations of one kind, so the T lanes that
own a pairing each take one operation per round without divergence.  Values
live in per-pairing shared-memory slots (one Fp, 48 bytes).  A slot reference
is base(3 bits) << 5 | offset(5 bits); the bases are supplied per call.  No
operation of a round writes a slot that an operation of the same round reads.

Arithmetic (the device kernel implements exactly this; `run_program` emulates
it bit for bit):
  * every slot holds an integer v with 0 <= v < 8p, congruent to the value;
  * MUL is a Montgomery product without the final subtraction: for a, b < 8p
    the result (a*b + M*p) / 2^384 is below 7.5p;
  * a signed sum starts from (number of negative units) * 8p, adds or
    subtracts each unit in a 13-word accumulator, then subtracts
    QP[acc >> 381] = floor(h * 2^381 / p) * p, leaving a value below 2.3p.
    At most 19 units per sum keep acc below 2^388 (h < 128).
Values are brought to canonical form (< p) only where they leave the kernel.

Outputs:
  programs.inc    C tables (written by `python gen_programs.py`)
  run_program()   a bit-exact Python emulator of the tables, used by the tests.
"""
import os
import sys

P = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
R = 1 << 384
PINV = pow(-P, -1, R)          # -p^-1 mod R
BOUND = 8 * P
QP = [(h << 381) // P * P for h in range(128)]

# slot bases
B_D, B_A, B_B, B_C, B_K, B_T0, B_T1, B_T2 = range(8)
K_ZERO, K_ONE = 0, 1           # constant slots (block-shared)
TEMP_SLOTS = 96                # T0, T1, T2
MAX_MUL_TERMS = 4              # units per MUL operand
MAX_LIN_TERMS = 8              # units per LIN
MAX_UNITS = 19

KIND_MUL, KIND_LIN, KIND_INV = 0, 1, 2


def ref(base, off):
    assert 0 <= off < 32
    return (base << 5) | off


ZERO_REF = ref(B_K, K_ZERO)


# --------------------------------------------------------------------------
# symbolic values
# --------------------------------------------------------------------------
class Lin:
    """A linear combination {atom: integer coefficient}."""
    __slots__ = ("t",)

    def __init__(self, t=None):
        self.t = {k: v for k, v in (t or {}).items() if v != 0}

    def __add__(self, o):
        r = dict(self.t)
        for k, v in o.t.items():
            r[k] = r.get(k, 0) + v
        return Lin(r)

    def __sub__(self, o):
        r = dict(self.t)
        for k, v in o.t.items():
            r[k] = r.get(k, 0) - v
        return Lin(r)

    def __neg__(self):
        return Lin({k: -v for k, v in self.t.items()})

    def scale(self, c):
        return Lin({k: c * v for k, v in self.t.items()})

    def units(self):
        return sum(abs(v) for v in self.t.values())

    def key(self):
        return tuple(sorted(self.t.items()))


class Node:
    __slots__ = ("id", "kind", "a", "b", "out_ref", "deps", "atom", "prio")

    def __init__(self, nid, kind, a, b):
        self.id, self.kind, self.a, self.b = nid, kind, a, b
        self.out_ref = None
        self.deps = set()
        self.atom = None
        self.prio = 0.0


class Builder:
    def __init__(self, name):
        self.name = name
        self.atoms = {}          # atom -> ("in", ref) | ("node", Node)
        self.nodes = []
        self.memo = {}
        self.outputs = []
        self._n = 0
        self._in = {}

    def _atom(self, desc):
        a = self._n
        self._n += 1
        self.atoms[a] = desc
        return a

    def inp(self, base, off):
        r = ref(base, off)
        if r not in self._in:
            self._in[r] = self._atom(("in", r))
        return Lin({self._in[r]: 1})

    def zero(self):
        return self.inp(B_K, K_ZERO)

    def _node(self, kind, a, b=None):
        n = Node(len(self.nodes), kind, a, b)
        n.atom = self._atom(("node", n))
        self.nodes.append(n)
        return n

    def lin(self, x):
        """Materialise x as one slot (memoised), splitting beyond MAX_LIN_TERMS."""
        if x.units() == 0:
            return self.zero()
        if len(x.t) == 1 and list(x.t.values())[0] == 1:
            return x
        k = x.key()
        if k in self.memo:
            return Lin({self.memo[k]: 1})
        y = self._fold(x, MAX_LIN_TERMS)
        n = self._node(KIND_LIN, y)
        self.memo[k] = n.atom
        return Lin({n.atom: 1})

    def _fold(self, x, limit):
        items = []
        for a, c in sorted(x.t.items()):
            items.extend([(a, 1 if c > 0 else -1)] * abs(c))
        while len(items) > limit:
            head, items = items[:limit], items[limit:]
            d = {}
            for a, s in head:
                d[a] = d.get(a, 0) + s
            n = self._node(KIND_LIN, Lin(d))
            items = [(n.atom, 1)] + items
        d = {}
        for a, s in items:
            d[a] = d.get(a, 0) + s
        return Lin(d)

    def _operand(self, x):
        """(Lin usable as a MUL operand, sign): single units are made positive
        and the sign moved to the product."""
        if x.units() == 0:
            return self.zero(), 1
        if len(x.t) == 1:
            (a, c), = x.t.items()
            if c == -1:
                return Lin({a: 1}), -1
            if c == 1:
                return x, 1
        if x.units() > MAX_MUL_TERMS:
            return self.lin(x), 1
        return x, 1

    def mul(self, a, b):
        a, sa = self._operand(a)
        b, sb = self._operand(b)
        n = self._node(KIND_MUL, a, b)
        return Lin({n.atom: sa * sb})

    def inv(self, a):
        a = self.lin(a)
        n = self._node(KIND_INV, a)
        return Lin({n.atom: 1})

    def out(self, base, off, x):
        self.outputs.append((ref(base, off), x))


# --------------------------------------------------------------------------
# tower formulas (field_sppark.cuh:52-197).  `m2` / `m6` materialise
# intermediate tower values so large sums are shared, not re-expanded.
# --------------------------------------------------------------------------
class Tower:
    def __init__(self, b, mat_fp2=True):
        self.b = b
        self.mat_fp2 = mat_fp2

    def m2(self, x):
        return (self.b.lin(x[0]), self.b.lin(x[1]))

    def f2_add(self, x, y): return (x[0] + y[0], x[1] + y[1])
    def f2_sub(self, x, y): return (x[0] - y[0], x[1] - y[1])
    def f2_neg(self, x): return (-x[0], -x[1])
    def f2_conj(self, x): return (x[0], -x[1])
    def f2_nr(self, x): return (x[0] - x[1], x[0] + x[1])
    def f2_dbl(self, x): return (x[0].scale(2), x[1].scale(2))

    def f2_mul(self, x, y):
        t0 = self.b.mul(x[0], y[0])
        t1 = self.b.mul(x[1], y[1])
        t2 = self.b.mul(x[0] + x[1], y[0] + y[1])
        r = (t0 - t1, t2 - t0 - t1)
        return self.m2(r) if self.mat_fp2 else r

    def f2_sqr(self, x):
        t = self.b.mul(x[0], x[1])
        s = self.b.mul(x[0] + x[1], x[0] - x[1])
        return (s, t.scale(2))

    def f2_mul_fp(self, x, s):
        return (self.b.mul(x[0], s), self.b.mul(x[1], s))

    def f6_add(self, x, y): return tuple(self.f2_add(a, b) for a, b in zip(x, y))
    def f6_sub(self, x, y): return tuple(self.f2_sub(a, b) for a, b in zip(x, y))
    def f6_neg(self, x): return tuple(self.f2_neg(a) for a in x)
    def f6_v(self, x): return (self.f2_nr(x[2]), x[0], x[1])
    def m6(self, x): return tuple(self.m2(a) for a in x)

    def f6_mul(self, a, b):
        aa = self.f2_mul(a[0], b[0])
        bb = self.f2_mul(a[1], b[1])
        cc = self.f2_mul(a[2], b[2])
        x = self.f2_mul(self.f2_add(a[1], a[2]), self.f2_add(b[1], b[2]))
        y = self.f2_mul(self.f2_add(a[0], a[1]), self.f2_add(b[0], b[1]))
        z = self.f2_mul(self.f2_add(a[0], a[2]), self.f2_add(b[0], b[2]))
        c0 = self.f2_add(aa, self.f2_nr(self.f2_sub(self.f2_sub(x, bb), cc)))
        c1 = self.f2_add(self.f2_sub(self.f2_sub(y, aa), bb), self.f2_nr(cc))
        c2 = self.f2_add(self.f2_sub(self.f2_sub(z, aa), cc), bb)
        return (c0, c1, c2)

    def f6_mul_by_01(self, s, c0, c1):
        aa = self.f2_mul(s[0], c0)
        bb = self.f2_mul(s[1], c1)
        t1 = self.f2_add(self.f2_nr(self.f2_mul(s[2], c1)), aa)
        t2 = self.f2_sub(self.f2_sub(self.f2_mul(self.f2_add(c0, c1), self.f2_add(s[0], s[1])), aa), bb)
        t3 = self.f2_add(self.f2_mul(s[2], c0), bb)
        return (t1, t2, t3)

    def f6_mul_by_1(self, s, c1):
        return (self.f2_nr(self.f2_mul(s[2], c1)), self.f2_mul(s[0], c1), self.f2_mul(s[1], c1))

    def f12_mul(self, a, b):
        sa = self.m6(self.f6_add(a[0], a[1]))
        sb = self.m6(self.f6_add(b[0], b[1]))
        aa = self.m6(self.f6_mul(a[0], b[0]))
        bb = self.m6(self.f6_mul(a[1], b[1]))
        s = self.f6_mul(sa, sb)
        return (self.f6_add(aa, self.f6_v(bb)), self.f6_sub(self.f6_sub(s, aa), bb))

    def f12_sqr(self, a):
        ab = self.m6(self.f6_mul(a[0], a[1]))
        x = self.m6(self.f6_add(a[0], self.f6_v(a[1])))
        y = self.m6(self.f6_add(a[0], a[1]))
        s = self.f6_mul(x, y)
        return (self.f6_sub(self.f6_sub(s, ab), self.f6_v(ab)), self.f6_add(ab, ab))

    def f12_mul_by_014(self, f, c0, c1, c4):
        aa = self.m6(self.f6_mul_by_01(f[0], c0, c1))
        bb = self.m6(self.f6_mul_by_1(f[1], c4))
        s = self.m6(self.f6_add(f[1], f[0]))
        o = self.m2(self.f2_add(c1, c4))
        t = self.f6_mul_by_01(s, c0, o)
        return (self.f6_add(self.f6_v(bb), aa), self.f6_sub(self.f6_sub(t, aa), bb))

    def fp4_square(self, a, b):
        t0 = self.m2(self.f2_sqr(a))
        t1 = self.m2(self.f2_sqr(b))
        o0 = self.f2_add(self.f2_nr(t1), t0)
        o1 = self.f2_sub(self.f2_sub(self.f2_sqr(self.f2_add(a, b)), t0), t1)
        return self.m2(o0), self.m2(o1)

    def f12_cyc_sqr(self, f):
        z0, z4, z3 = f[0]
        z2, z1, z5 = f[1]
        A0, A1 = self.fp4_square(z0, z1)
        B0, B1 = self.fp4_square(z2, z3)
        C0, C1 = self.fp4_square(z4, z5)
        z0 = self.f2_add(self.f2_dbl(self.f2_sub(A0, z0)), A0)
        z1 = self.f2_add(self.f2_dbl(self.f2_add(A1, z1)), A1)
        z4 = self.f2_add(self.f2_dbl(self.f2_sub(B0, z4)), B0)
        z5 = self.f2_add(self.f2_dbl(self.f2_add(B1, z5)), B1)
        nc1 = self.f2_nr(C1)
        z2 = self.f2_add(self.f2_dbl(self.f2_add(nc1, z2)), nc1)
        z3 = self.f2_add(self.f2_dbl(self.f2_sub(C0, z3)), C0)
        return ((z0, z4, z3), (z2, z1, z5))

    def f12_frob(self, f, k):
        k1, k2, k12 = k

        def f6_frob(x):
            return (self.f2_conj(x[0]), self.f2_mul(self.f2_conj(x[1]), k1), self.f2_mul(self.f2_conj(x[2]), k2))
        c0 = f6_frob(f[0])
        c1 = f6_frob(f[1])
        return (c0, tuple(self.f2_mul(x, k12) for x in c1))

    def f2_inv(self, a):
        n = self.b.mul(a[0], a[0]) + self.b.mul(a[1], a[1])
        i = self.b.inv(n)
        return (self.b.mul(a[0], i), -self.b.mul(a[1], i))

    def f6_inv(self, f):
        c0s, c1s, c2s = self.f2_sqr(f[0]), self.f2_sqr(f[1]), self.f2_sqr(f[2])
        c01, c02, c12 = self.f2_mul(f[0], f[1]), self.f2_mul(f[0], f[2]), self.f2_mul(f[1], f[2])
        t0 = self.m2(self.f2_sub(c0s, self.f2_nr(c12)))
        t1 = self.m2(self.f2_sub(self.f2_nr(c2s), c01))
        t2 = self.m2(self.f2_sub(c1s, c02))
        sc = self.f2_add(self.f2_mul(f[0], t0), self.f2_nr(self.f2_add(self.f2_mul(f[2], t1), self.f2_mul(f[1], t2))))
        si = self.f2_inv(self.m2(sc))
        return (self.f2_mul(t0, si), self.f2_mul(t1, si), self.f2_mul(t2, si))

    def f12_inv(self, f):
        t = self.m6(self.f6_sub(self.f6_mul(f[0], f[0]), self.f6_v(self.f6_mul(f[1], f[1]))))
        ti = self.m6(self.f6_inv(t))
        return (self.f6_mul(f[0], ti), self.f6_neg(self.f6_mul(f[1], ti)))


def unflat(v):
    f2 = [(v[2 * i], v[2 * i + 1]) for i in range(6)]
    return ((f2[0], f2[1], f2[2]), (f2[3], f2[4], f2[5]))


def flat(f):
    return [x for f6 in f for f2 in f6 for x in f2]


def f12_in(b, base):
    return unflat([b.inp(base, i) for i in range(12)])


# --------------------------------------------------------------------------
# programs.  D: Fp12 written; A / B: Fp12 inputs; C: auxiliary inputs.
# LINE2's C: pair 1 coefficient (c0, c1, c2) at C[0..5], point at C[6..7];
# pair 2 at C[8..13], C[14..15].  FROB's constants k1, k2, k12 at K[2..7].
# --------------------------------------------------------------------------
K_FROB = 2


def prog_line2(b, tw):
    f = f12_in(b, B_D)
    for pair in range(2):
        o = 8 * pair
        c0 = (b.inp(B_C, o + 0), b.inp(B_C, o + 1))
        c1 = (b.inp(B_C, o + 2), b.inp(B_C, o + 3))
        c2 = (b.inp(B_C, o + 4), b.inp(B_C, o + 5))
        px, py = b.inp(B_C, o + 6), b.inp(B_C, o + 7)
        f = tw.f12_mul_by_014(f, c2, tw.f2_mul_fp(c1, px), tw.f2_mul_fp(c0, py))
        if pair == 0:
            f = tuple(tw.m6(x) for x in f)
    for i, x in enumerate(flat(f)):
        b.out(B_D, i, x)


def prog_sqr(b, tw):
    for i, x in enumerate(flat(tw.f12_sqr(f12_in(b, B_D)))):
        b.out(B_D, i, x)


def prog_cycsqr(b, tw):
    for i, x in enumerate(flat(tw.f12_cyc_sqr(f12_in(b, B_D)))):
        b.out(B_D, i, x)


def prog_mul(b, tw):
    for i, x in enumerate(flat(tw.f12_mul(f12_in(b, B_A), f12_in(b, B_B)))):
        b.out(B_D, i, x)


def prog_frob(b, tw):
    k = [(b.inp(B_K, K_FROB + 2 * j), b.inp(B_K, K_FROB + 2 * j + 1)) for j in range(3)]
    for i, x in enumerate(flat(tw.f12_frob(f12_in(b, B_A), k))):
        b.out(B_D, i, x)


def prog_conj(b, tw):
    f = f12_in(b, B_A)
    for i, x in enumerate(flat((f[0], tuple((-a[0], -a[1]) for a in f[1])))):
        b.out(B_D, i, x)


def prog_copy(b, tw):
    for i in range(12):
        b.out(B_D, i, b.inp(B_A, i))


def prog_inv(b, tw):
    for i, x in enumerate(flat(tw.f12_inv(f12_in(b, B_A)))):
        b.out(B_D, i, x)


PROGRAMS = [
    ("LINE2", prog_line2, "D *= line(pair 1) * line(pair 2), coefficients and points in C (api.cu:37-38)"),
    ("SQR", prog_sqr, "D = D^2 (field_sppark.cuh:148-151)"),
    ("CYCSQR", prog_cycsqr, "D = cyclotomic square of D (field_sppark.cuh:174-197)"),
    ("MUL", prog_mul, "D = A * B (field_sppark.cuh:142-146)"),
    ("FROB", prog_frob, "D = Frobenius(A) (field_sppark.cuh:159-166)"),
    ("CONJ", prog_conj, "D = conjugate(A)"),
    ("COPY", prog_copy, "D = A"),
    ("INV", prog_inv, "D = A^-1 (field_sppark.cuh:153-157, 104-111, 79-83)"),
]


# --------------------------------------------------------------------------
# scheduling and slot allocation
# --------------------------------------------------------------------------
class Program:
    def __init__(self, name, rounds, ntemp):
        self.name, self.rounds, self.ntemp = name, rounds, ntemp
        self.nmul = sum(len(r[1]) for r in rounds if r[0] == KIND_MUL)
        self.nlin = sum(len(r[1]) for r in rounds if r[0] == KIND_LIN)


def _terms(x, atom_ref):
    t = []
    for a, c in sorted(x.t.items(), key=lambda kv: (-kv[1], kv[0])):
        t.extend([(atom_ref(a), 1 if c > 0 else -1)] * abs(c))
    return t


def compile_program(name, fn, lanes, mat_fp2=True):
    b = Builder(name)
    tw = Tower(b, mat_fp2=mat_fp2)
    fn(b, tw)
    for r, x in b.outputs:
        # a MUL result with +1 is written straight to its output slot, else a LIN
        if len(x.t) == 1:
            (a, c), = x.t.items()
            d = b.atoms[a]
            if c == 1 and d[0] == "node" and d[1].out_ref is None and d[1].kind == KIND_MUL:
                d[1].out_ref = r
                continue
        y = b._fold(x, MAX_LIN_TERMS) if x.units() else b.zero()
        n = b._node(KIND_LIN, y)
        n.out_ref = r
    nodes = b.nodes
    for n in nodes:
        for x in (n.a, n.b):
            if x is not None:
                assert x.units() <= MAX_UNITS
                for a in x.t:
                    d = b.atoms[a]
                    if d[0] == "node":
                        n.deps.add(d[1].id)
    users = {n.id: [] for n in nodes}
    for n in nodes:
        for d in n.deps:
            users[d].append(n.id)

    def cost(n):
        if n.kind == KIND_MUL:
            return 1.0 + 0.04 * (n.a.units() + n.b.units())
        if n.kind == KIND_LIN:
            return 0.05 + 0.04 * n.a.units()
        return 60.0
    for n in sorted(nodes, key=lambda n: -n.id):
        n.prio = cost(n) + max([nodes[u].prio for u in users[n.id]], default=0.0)

    done = {}
    remaining = set(n.id for n in nodes)
    rounds = []
    while remaining:
        r = len(rounds)
        ready = [nodes[i] for i in remaining if all(d in done and done[d] < r for d in nodes[i].deps)]
        ready.sort(key=lambda n: (-n.prio, n.id))
        head = ready[0]
        if head.kind == KIND_INV:
            pick = [head]
        elif head.kind == KIND_MUL:
            pick = [n for n in ready if n.kind == KIND_MUL][:lanes]
        else:
            lim = head.a.units()
            cand = [n for n in ready if n.kind == KIND_LIN]
            pick = [n for n in cand if n.a.units() <= lim][:lanes]
            if len(pick) < lanes:
                extra = [n for n in cand if n not in pick and n.a.units() <= lim + 2]
                pick += extra[:lanes - len(pick)]
        for n in pick:
            done[n.id] = r
            remaining.discard(n.id)
        rounds.append((head.kind, [n.id for n in pick]))

    last_use = {n.id: -1 for n in nodes}
    in_last = {}
    for n in nodes:
        for x in (n.a, n.b):
            if x is None:
                continue
            for a in x.t:
                d = b.atoms[a]
                if d[0] == "node":
                    last_use[d[1].id] = max(last_use[d[1].id], done[n.id])
                else:
                    in_last[d[1]] = max(in_last.get(d[1], -1), done[n.id])

    slot_of = {}
    free_at = {}
    copies = []
    for ri, (kind, ids) in enumerate(rounds):
        for i in ids:
            n = nodes[i]
            if n.out_ref is not None and in_last.get(n.out_ref, -1) < ri:
                slot_of[i] = n.out_ref
                continue
            if n.out_ref is not None:
                copies.append((n.out_ref, i))
            for s in range(TEMP_SLOTS):
                if free_at.get(s, 0) <= ri:
                    break
            else:
                raise RuntimeError("%s: out of temporary slots" % name)
            slot_of[i] = ref(B_T0 + s // 32, s % 32)
            lu = 10 ** 9 if n.out_ref is not None else last_use[i]
            free_at[s] = (lu + 1) if lu >= 0 else ri + 1

    def atom_ref(a):
        d = b.atoms[a]
        return d[1] if d[0] == "in" else slot_of[d[1].id]

    out_rounds = []
    for kind, ids in rounds:
        recs = []
        for i in ids:
            n = nodes[i]
            recs.append((slot_of[i], _terms(n.a, atom_ref), _terms(n.b, atom_ref) if n.b is not None else None))
        out_rounds.append((kind, recs))
    for k in range(0, len(copies), lanes):
        out_rounds.append((KIND_LIN, [(o, [(slot_of[i], 1)], None) for o, i in copies[k:k + lanes]]))
    ntemp = 0
    for s in slot_of.values():
        if (s >> 5) >= B_T0:
            ntemp = max(ntemp, ((s >> 5) - B_T0) * 32 + (s & 31) + 1)
    _check(name, out_rounds)
    return Program(name, out_rounds, ntemp)


def _check(name, rounds):
    for ri, (kind, recs) in enumerate(rounds):
        reads = set(r for _, a, bb in recs for r, _ in a + (bb or []))
        dsts = [d for d, _, _ in recs]
        assert not (set(dsts) & reads), "%s round %d writes a slot it reads" % (name, ri)
        assert len(dsts) == len(set(dsts))
        for _, a, bb in recs:
            if kind == KIND_MUL:
                for ops in (a, bb):
                    assert len(ops) <= MAX_MUL_TERMS
                    if len(ops) == 1:
                        assert ops[0][1] == 1, "%s: single-unit MUL operand must be positive" % name
            elif kind == KIND_INV:
                assert len(a) == 1 and a[0][1] == 1


# --------------------------------------------------------------------------
# bit-exact emulator of the device arithmetic
# --------------------------------------------------------------------------
def redc(a, b):
    assert 0 <= a < BOUND and 0 <= b < BOUND
    t = a * b
    m = (t * PINV) % R
    r = (t + m * P) >> 384
    assert r < BOUND
    return r


def signed_sum(terms, val):
    neg = sum(1 for _, s in terms if s < 0)
    acc = neg * BOUND
    for r, s in terms:
        acc += s * val(r)
    assert 0 <= acc < (1 << 388)
    acc -= QP[acc >> 381]
    assert 0 <= acc < BOUND
    return acc


def fp_inv_exact(x):
    """Fermat x^(p-2), right-to-left square-and-multiply over 381 exponent
    bits with the same REDC, on the representative."""
    r = R % P
    base = x
    e = P - 2
    for i in range(381):
        if (e >> i) & 1:
            r = redc(r, base)
        base = redc(base, base)
    return r


def run_program(prog, slots, bases):
    """slots: dict absolute slot -> integer representative (Montgomery form)."""
    def val(r):
        v = slots[bases[r >> 5] + (r & 31)]
        assert 0 <= v < BOUND
        return v

    for kind, recs in prog.rounds:
        out = []
        for dst, a, bb in recs:
            if kind == KIND_MUL:
                x = val(a[0][0]) if len(a) == 1 else signed_sum(a, val)
                y = val(bb[0][0]) if len(bb) == 1 else signed_sum(bb, val)
                out.append((dst, redc(x, y)))
            elif kind == KIND_LIN:
                out.append((dst, signed_sum(a, val)))
            else:
                out.append((dst, fp_inv_exact(val(a[0][0]))))
        for dst, v in out:
            slots[bases[dst >> 5] + (dst & 31)] = v


# --------------------------------------------------------------------------
# C emission
# --------------------------------------------------------------------------
def build_all(lanes):
    return [compile_program(n, fn, lanes) for n, fn, _ in PROGRAMS]


def emit(lane_options, path):
    L = ["// Generated by gen_programs.py (tower programs of the lane-parallel verify",
         "// kernel); do not edit, run `python gen_programs.py`.",
         "#pragma once", "#include <cstdint>", "", "namespace bls {", "namespace prog {", ""]
    for i, (n, _, doc) in enumerate(PROGRAMS):
        L.append("constexpr int P_%s = %d;  // %s" % (n, i, doc))
    L += ["constexpr int kNumPrograms = %d;" % len(PROGRAMS),
          "constexpr int kTempSlots = %d;" % TEMP_SLOTS,
          "constexpr int kKFrob = %d;" % K_FROB, ""]
    L.append("// QP[h] = floor(h * 2^381 / p) * p, 13 x 32-bit words padded to 16")
    L.append("__device__ const uint32_t kQP[128][16] = {")
    for q in QP:
        L.append("    {" + ", ".join("0x%08xu" % ((q >> (32 * i)) & 0xffffffff) for i in range(16)) + "},")
    L.append("};")
    L.append("")
    for lanes in lane_options:
        progs = build_all(lanes)
        rounds, ops, tab = [], [], []
        for p in progs:
            first = len(rounds)
            for kind, recs in p.rounds:
                na = max(len(a) for _, a, _ in recs)
                nb = max((len(bb) for _, _, bb in recs if bb), default=0)
                rounds.append((kind, len(ops), len(recs), na, nb))
                for dst, a, bb in recs:
                    bb = bb or []
                    ta = a + [(ZERO_REF, 1)] * (na - len(a))
                    tb = bb + [(ZERO_REF, 1)] * (nb - len(bb))
                    terms = ta + tb
                    assert len(terms) <= 8
                    sgn = sum(1 << k for k, (_, s) in enumerate(terms) if s < 0)
                    refs = [r for r, _ in terms] + [ZERO_REF] * (8 - len(terms))
                    ops.append((dst, sgn, refs))
            tab.append((first, len(rounds) - first, p.ntemp, p.nmul, p.nlin))
        L.append("// ---- %d lane(s) per pairing ----" % lanes)
        L.append("__device__ const uint32_t kProgT%d[%d][3] = {  // first round, rounds, temporaries" % (lanes, len(tab)))
        for (n, _, _), (f, c, tmp, nm, nl) in zip(PROGRAMS, tab):
            L.append("    {%du, %du, %du},  // %s: %d MUL, %d LIN" % (f, c, tmp, n, nm, nl))
        L.append("};")
        L.append("// round: kind | nops << 8 | na << 16 | nb << 24 ; first op")
        L.append("__device__ const uint32_t kRoundT%d[%d][2] = {" % (lanes, len(rounds)))
        for kind, fo, no, na, nb in rounds:
            L.append("    {0x%08xu, %du}," % (kind | (no << 8) | (na << 16) | (nb << 24), fo))
        L.append("};")
        L.append("// op: dst | sign bits << 8 ; slot refs 0-3 ; slot refs 4-7")
        L.append("__device__ const uint32_t kOpT%d[%d][3] = {" % (lanes, len(ops)))
        for dst, sgn, refs in ops:
            w1 = refs[0] | refs[1] << 8 | refs[2] << 16 | refs[3] << 24
            w2 = refs[4] | refs[5] << 8 | refs[6] << 16 | refs[7] << 24
            L.append("    {0x%04xu, 0x%08xu, 0x%08xu}," % (dst | (sgn << 8), w1, w2))
        L.append("};")
        L.append("constexpr int kMaxTempT%d = %d;" % (lanes, max(p.ntemp for p in progs)))
        L.append("")
    L += ["}  // namespace prog", "}  // namespace bls"]
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def summary(lanes):
    out = []
    for p in build_all(lanes):
        mr = [r for r in p.rounds if r[0] == KIND_MUL]
        lr = [r for r in p.rounds if r[0] == KIND_LIN]
        lin_units = sum(max(len(a) for _, a, _ in recs) for _, recs in lr)
        out.append("%-7s T=%d: %3d MUL / %3d rounds (%3.0f%% busy), %3d LIN / %3d rounds (%3d padded units), %2d temps"
                   % (p.name, lanes, p.nmul, len(mr), 100.0 * p.nmul / max(1, len(mr) * lanes), p.nlin, len(lr),
                      lin_units, p.ntemp))
    return out


LANE_OPTIONS = [1, 2, 4, 8]

if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    if "--summary" in sys.argv:
        for t in LANE_OPTIONS:
            print("\n".join(summary(t)))
    else:
        emit(LANE_OPTIONS, os.path.join(here, "programs.inc"))
