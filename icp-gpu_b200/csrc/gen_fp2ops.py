"""Generator of the Fp2-lane tower programs of the verify kernel (verify_fp2.cu).

Execution model.  Twelve threads own one pairing, in two halves (two warps
of a block); the thread pair (k, half 0) and (k, half 1) produces the k-th Fp2
coefficient (tower order c0.c0, c0.c1, c0.c2, c1.c0, c1.c1, c1.c2) of each
Fp12 result.  The products of an output are split between the two halves;
each half sums its share into both accumulators, the halves exchange one
accumulator through shared memory, and half 0 reduces the real part, half 1
the imaginary part.  Every coefficient of every tower operation on the verify path
(gpu-crypto/cuda/field_sppark.cuh:52-197, gpu-crypto/cuda/api.cu:22-78) is
written as one *output*:

    out = post( REDC(ACC_re), REDC(ACC_im) )
    ACC = bias + sum over terms of  alpha_j * U_j * V_j   (exact, 832-bit)

so a lane multiplies all the Fp2 products that feed its coefficient into two
double-width accumulators and performs one Montgomery reduction per Fp
(lazy reduction, Aranha et al., "Faster explicit formulas for computing
pairings over ordinary curves", EUROCRYPT 2011).  Karatsuba inside each Fp2
product; no intermediate result is rounded to Fp.

Term kinds (X, Y are Fp2 slots, x0/x1 their components):
  KARA   X*Y          U = (x0, x1, x0+x1)  V = (y0, y1, y0+y1)
  SQR    X^2          U = (x0+x1, 2 x0)    V = (x0-x1+3p, x1)
  FPMUL  X*y (y in Fp) U = (x0, x1)        V = (y, y)
  NORM   x0^2+x1^2    U = (x0, x1)         V = (x0, x1)
A KARA term times xi = 1 + u takes xi X = (x0 - x1 + 3p, x0 + x1) as its X; a
doubled KARA term takes 2 Y as its Y.  The per-product accumulator
coefficients (alpha for ACC_re, beta for ACC_im) are then all in {-1, 0, 1},
fixed by the kind and `xi`, and negated for a negative term.  Additive
multiples of p (the 3p above, the biases) leave every value unchanged mod p.

Post-processing of an output:
  SIMPLE  out = QP(r)                               r = REDC result
  FULL    out = QP(c_re * QP(r_re) + sum c_j z_j + bias)  (and im with c_im)
  LIN     out = QP(sum c_j z_j + bias)               (no product)
  INVFP   out = (x0^-1 in Montgomery form, 0)        (one lane)
QP(v) = v - QP[v >> 381], QP[h] = floor(h * 2^381 / p) * p: a value below
2^388 becomes one below 2^381 + p < 2.3p; every slot holds such a value.

Outputs:
  fp2ops.inc   descriptor tables (run `python gen_fp2ops.py`)
  Emulator     bit-exact Python model of the device arithmetic, used by the
               tests to check every program against the oracle on the CPU.
"""
import os
import sys

P = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
R = 1 << 384
NPRIME = (-pow(P, -1, 1 << 32)) % (1 << 32)
QP = [(h << 381) // P * P for h in range(128)]
SLOT_BOUND = (1 << 381) + P          # every slot value is below this
ACC_LIMIT = 1 << 771                 # accumulators stay below (REDC output < 2^388)
POST_LIMIT = 1 << 388                # QP input limit
K3P = 3 * P

# ---------------------------------------------------------------- refs
# A ref names one Fp2 slot: base (3 bits) << 4 | index (4 bits).
B_D, B_A, B_B, B_C, B_K, B_T = range(6)
BASE_NAMES = "DABCKT"


def ref(base, idx):
    assert 0 <= idx < 16
    return (base << 4) | idx


# block-shared constant slots (Fp2)
K_ZERO, K_ONE = 0, 1
K_FROB = 2     # 2..6: conj(k1), conj(k2), conj(k12), conj(k1 k12), conj(k2 k12)

# C area of a pairing: pair j (0, 1) at 6 j: coefficient c0, c1, c2, point (x, y), l2, l3
C_C0, C_C1, C_C2, C_PT, C_L2, C_L3 = range(6)

# ---------------------------------------------------------------- kinds
KARA, SQR, FPMUL, NORM, ONE = range(5)
# (alpha, beta) per product, plain and times xi
COEF = {
    (KARA, 0): ((1, -1, 0), (-1, -1, 1)),
    (KARA, 1): ((1, -1, 0), (-1, -1, 1)),     # xi applied to X
    (SQR, 0): ((1, 0), (0, 1)),                # second product is (2 x0) x1
    (SQR, 1): ((1, -1), (1, 1)),
    (FPMUL, 0): ((1, 0), (0, 1)),
    (FPMUL, 1): ((1, -1), (1, 1)),
    (NORM, 0): ((1, 1), (0, 0)),
}
NPROD = {KARA: 3, SQR: 2, FPMUL: 2, NORM: 2, ONE: 1}
M_SIMPLE, M_FULL, M_LIN, M_INVFP = range(4)


class Term:
    __slots__ = ("kind", "x", "y", "xi", "sign", "dbl", "yim")

    def __init__(self, kind, x, y=None, xi=0, sign=1, dbl=0, yim=0):
        self.kind, self.x, self.y, self.xi, self.sign, self.dbl, self.yim = kind, x, y, xi, sign, dbl, yim
        if kind in (SQR, NORM, ONE):
            self.y = x
        assert not (kind == NORM and xi)
        assert not (dbl and kind != KARA)

    def coefs(self):
        if self.kind == ONE:
            return [self.sign], [self.sign]
        a, b = COEF[(self.kind, self.xi)]
        return [self.sign * v for v in a], [self.sign * v for v in b]

    def operands(self, X, Y):
        """(U, V) integer pairs for the products, from component values.  A ONE
        term is X itself, placed in the high half of the accumulators (X R)."""
        x0, x1 = X
        if self.kind == ONE:
            return [(x0, x1)]
        if self.kind == KARA:
            if self.xi:
                x0, x1 = x0 - x1 + K3P, x0 + x1
            y0, y1 = Y
            if self.dbl:
                y0, y1 = 2 * y0, 2 * y1
            return [(x0, y0), (x1, y1), (x0 + x1, y0 + y1)]
        if self.kind == SQR:
            return [(x0 + x1, x0 - x1 + K3P), (2 * x0, x1)]
        if self.kind == FPMUL:
            y = Y[1] if self.yim else Y[0]
            return [(x0, y), (x1, y)]
        return [(x0, x0), (x1, x1)]


class Out:
    def __init__(self, dst, mode=M_SIMPLE, terms=(), lins=(), c_re=1, c_im=1):
        self.dst, self.mode, self.terms, self.lins = dst, mode, list(terms), list(lins)
        self.c_re, self.c_im = c_re, c_im
        if mode == M_SIMPLE and (lins or c_re != 1 or c_im != 1):
            self.mode = M_FULL
        self.bias_re = self.bias_im = self.bias_lin_re = self.bias_lin_im = 0


# ---------------------------------------------------------------- static bounds
def _operand_bounds(t):
    """exclusive upper bounds of (U, V) per product"""
    B = SLOT_BOUND
    if t.kind == KARA:
        bx0, bx1 = (B + K3P, 2 * B) if t.xi else (B, B)
        by = 2 * B if t.dbl else B
        return [(bx0, by), (bx1, by), (bx0 + bx1, 2 * by)]
    if t.kind == SQR:
        return [(2 * B, B + K3P), (2 * B, B)]
    if t.kind == ONE:
        return [(B, B)]
    return [(B, B), (B, B)]


def _prod_bounds(t):
    if t.kind == ONE:
        return [SLOT_BOUND * R]
    out = []
    for bu, bv in _operand_bounds(t):
        assert bu <= R and bv <= R, "operand bound"
        out.append(bu * bv)
    return out


def finish(o):
    """Fix the biases of an output from worst-case bounds and check limits."""
    if o.mode in (M_SIMPLE, M_FULL):
        pos = [0, 0]
        neg = [0, 0]
        for t in o.terms:
            al, be = t.coefs()
            for k, pb in enumerate(_prod_bounds(t)):
                for c, co in enumerate((al[k], be[k])):
                    if co > 0:
                        pos[c] += co * pb
                    else:
                        neg[c] += -co * pb
        o.bias_re = -(-neg[0] // (P * R))
        o.bias_im = -(-neg[1] // (P * R))
        for c, bk in enumerate((o.bias_re, o.bias_im)):
            assert bk < 256
            top = bk * P * R + pos[c]
            assert top < ACC_LIMIT, "accumulator bound"
            assert top // R + P < POST_LIMIT
    if o.mode in (M_FULL, M_LIN):
        for c, cc in enumerate((o.c_re, o.c_im)):
            negs = poss = 0
            if o.mode == M_FULL:      # c scales the REDC result, lins enter as they are
                negs, poss = (-cc if cc < 0 else 0) * SLOT_BOUND, (cc if cc > 0 else 0) * SLOT_BOUND
                mult = 1
            else:                     # c scales every lin term
                mult = cc
            for co, _ in o.lins:
                e = co * mult
                if e < 0:
                    negs += -e * SLOT_BOUND
                else:
                    poss += e * SLOT_BOUND
            bk = -(-negs // P)
            assert bk < 256
            if c == 0:
                o.bias_lin_re = bk
            else:
                o.bias_lin_im = bk
            assert bk * P + poss < POST_LIMIT
    return o


# ---------------------------------------------------------------- halves
def split_halves(o):
    """Assign the products of an output's terms to the two halves, balancing
    their counts: whole terms first (largest first, to the lighter half), then
    single products move from the heavier half while that narrows the gap.
    Returns two lists of (term index, product mask)."""
    load = [0, 0]
    masks = [dict(), dict()]
    for ti in sorted(range(len(o.terms)), key=lambda i: (-NPROD[o.terms[i].kind], i)):
        n = NPROD[o.terms[ti].kind]
        h = 0 if load[0] <= load[1] else 1
        masks[h][ti] = (1 << n) - 1
        load[h] += n
    while abs(load[0] - load[1]) >= 2:
        big = 0 if load[0] > load[1] else 1
        ti = max(masks[big])
        m = masks[big][ti]
        bit = m.bit_length() - 1
        masks[big][ti] = m & ~(1 << bit)
        if not masks[big][ti]:
            del masks[big][ti]
        masks[1 - big][ti] = masks[1 - big].get(ti, 0) | (1 << bit)
        load[big] -= 1
        load[1 - big] += 1
    halves = [sorted(masks[h].items()) for h in range(2)]
    # every product exactly once
    for ti, t in enumerate(o.terms):
        m0 = dict(halves[0]).get(ti, 0)
        m1 = dict(halves[1]).get(ti, 0)
        assert m0 & m1 == 0 and (m0 | m1) == (1 << NPROD[t.kind]) - 1
    return halves


def half_products(o, h):
    return sum(bin(m).count("1") for _, m in split_halves(o)[h]) if o.mode in (M_SIMPLE, M_FULL) else 0


# ---------------------------------------------------------------- tower helpers
# tower position t (0..5: c0.c0, c0.c1, c0.c2, c1.c0, c1.c1, c1.c2) <-> power of w
W_OF_T = [0, 2, 4, 1, 3, 5]
T_OF_W = [W_OF_T.index(k) for k in range(6)]


def prog_mul():
    """D = A * B (field_sppark.cuh:142-146): w-basis schoolbook, lazily."""
    outs = []
    for t in range(6):
        k = W_OF_T[t]
        terms = []
        for i in range(6):
            j = (k - i) % 6
            terms.append(Term(KARA, ref(B_A, T_OF_W[i]), ref(B_B, T_OF_W[j]), xi=int(i + j >= 6)))
        outs.append(finish(Out(ref(B_D, t), terms=terms)))
    return outs


def prog_sqr():
    """D = A^2 (field_sppark.cuh:148-151)."""
    outs = []
    for t in range(6):
        k = W_OF_T[t]
        terms = []
        for i in range(6):
            j = (k - i) % 6
            if i > j:
                continue
            xi = int(i + j >= 6)
            if i == j:
                terms.append(Term(SQR, ref(B_A, T_OF_W[i]), xi=xi))
            else:
                terms.append(Term(KARA, ref(B_A, T_OF_W[i]), ref(B_A, T_OF_W[j]), xi=xi, dbl=1))
        outs.append(finish(Out(ref(B_D, t), terms=terms)))
    return outs


def prog_line(pair):
    """D = A * (l0 + l2 w^2 + l3 w^3), the sparse line product of
    fp12_mul_by_014 (field_sppark.cuh:126-140) with l0 = c2, l2 = c1 * P.x,
    l3 = c0 * P.y (api.cu:37-38)."""
    o = 6 * pair
    lref = {0: ref(B_C, o + C_C2), 2: ref(B_C, o + C_L2), 3: ref(B_C, o + C_L3)}
    outs = []
    for t in range(6):
        k = W_OF_T[t]
        terms = []
        for j, lr in sorted(lref.items()):
            i = (k - j) % 6
            terms.append(Term(KARA, ref(B_A, T_OF_W[i]), lr, xi=int(k - j < 0)))
        outs.append(finish(Out(ref(B_D, t), terms=terms)))
    return outs


def prog_line_norm(pair):
    """D = A * (1 + l2 w^2 + l3 w^3): the line of prog_line divided by its c2
    (tables normalised once per key; the Miller value differs from the
    reference's by an Fp2 factor that the final exponentiation removes and
    that SCALE1 / SCALE2 multiply back when the Miller value is wanted)."""
    o = 6 * pair
    lref = {2: ref(B_C, o + C_L2), 3: ref(B_C, o + C_L3)}
    outs = []
    for t in range(6):
        k = W_OF_T[t]
        terms = [Term(ONE, ref(B_A, t))]
        for j, lr in sorted(lref.items()):
            i = (k - j) % 6
            terms.append(Term(KARA, ref(B_A, T_OF_W[i]), lr, xi=int(k - j < 0)))
        outs.append(finish(Out(ref(B_D, t), terms=terms)))
    return outs


def prog_scale(pair):
    """D = A * s, s the Fp2 in the C area's c2 slot of `pair` (a key's Miller
    correction factor)"""
    s_ref = ref(B_C, 6 * pair + C_C2)
    return [finish(Out(ref(B_D, t), terms=[Term(KARA, ref(B_A, t), s_ref)])) for t in range(6)]


def prog_lscale():
    """l2 = c1 * P.x, l3 = c0 * P.y for both pairs (api.cu:37-38)."""
    outs = []
    for pair in range(2):
        o = 6 * pair
        outs.append(finish(Out(ref(B_C, o + C_L2), terms=[Term(FPMUL, ref(B_C, o + C_C1), ref(B_C, o + C_PT))])))
        outs.append(finish(Out(ref(B_C, o + C_L3),
                               terms=[Term(FPMUL, ref(B_C, o + C_C0), ref(B_C, o + C_PT), yim=1)])))
    return outs + [None, None]


def prog_cycsqr():
    """D = Granger-Scott cyclotomic square of A (field_sppark.cuh:174-197)."""
    z = {0: 0, 4: 1, 3: 2, 2: 3, 1: 4, 5: 5}   # z_i -> tower position
    zr = {i: ref(B_A, t) for i, t in z.items()}
    outs = [None] * 6

    def sqr_out(i, a, b):     # z_i' = 3 (xi b^2 + a^2) - 2 z_i
        return finish(Out(ref(B_D, z[i]), terms=[Term(SQR, zr[b], xi=1), Term(SQR, zr[a])],
                          lins=[(-2, zr[i])], c_re=3, c_im=3))

    def mul_out(i, a, b, xi):  # z_i' = 6 xi^e a b + 2 z_i
        return finish(Out(ref(B_D, z[i]), terms=[Term(KARA, zr[a], zr[b], xi=xi)],
                          lins=[(2, zr[i])], c_re=6, c_im=6))
    outs[z[0]] = sqr_out(0, 0, 1)
    outs[z[1]] = mul_out(1, 0, 1, 0)
    outs[z[4]] = sqr_out(4, 2, 3)
    outs[z[5]] = mul_out(5, 2, 3, 0)
    outs[z[2]] = mul_out(2, 4, 5, 1)
    outs[z[3]] = sqr_out(3, 4, 5)
    return outs


def prog_frob():
    """D = Frobenius(A) (field_sppark.cuh:159-166): each coefficient is
    conj(a_t) * g_t = conj(a_t * conj(g_t)), g in {1, k1, k2, k12, k1 k12, k2 k12}."""
    gk = [None, K_FROB + 0, K_FROB + 1, K_FROB + 2, K_FROB + 3, K_FROB + 4]
    outs = []
    for t in range(6):
        if gk[t] is None:
            outs.append(finish(Out(ref(B_D, t), mode=M_LIN, lins=[(1, ref(B_A, t))], c_re=1, c_im=-1)))
        else:
            outs.append(finish(Out(ref(B_D, t), terms=[Term(KARA, ref(B_A, t), ref(B_K, gk[t]))], c_re=1, c_im=-1)))
    return outs


def prog_conj():
    """D = conjugate(A) = c0 - c1 w."""
    return [finish(Out(ref(B_D, t), mode=M_LIN, lins=[(1 if t < 3 else -1, ref(B_A, t))])) for t in range(6)]


def prog_copy():
    return [finish(Out(ref(B_D, t), mode=M_LIN, lins=[(1, ref(B_A, t))])) for t in range(6)]


# Fp12 inverse (field_sppark.cuh:153-157 -> 104-111 -> 79-83 -> 40-50), in steps.
# Temporaries (base T): 0-2 t = c0^2 - v c1^2, 3-5 (A, B, C), 6 F, 7 n, 8 n^-1,
# 9 F^-1, 10-12 t^-1.
def prog_inv1():
    a = [ref(B_A, t) for t in range(3)]
    b = [ref(B_A, 3 + t) for t in range(3)]
    T = lambda *args, **kw: Term(*args, **kw)
    o0 = Out(ref(B_T, 0), terms=[T(SQR, a[0]), T(KARA, a[1], a[2], xi=1, dbl=1), T(SQR, b[1], xi=1, sign=-1),
                                 T(KARA, b[0], b[2], xi=1, dbl=1, sign=-1)])
    o1 = Out(ref(B_T, 1), terms=[T(KARA, a[0], a[1], dbl=1), T(SQR, a[2], xi=1), T(SQR, b[0], sign=-1),
                                 T(KARA, b[1], b[2], xi=1, dbl=1, sign=-1)])
    o2 = Out(ref(B_T, 2), terms=[T(SQR, a[1]), T(KARA, a[0], a[2], dbl=1), T(KARA, b[0], b[1], dbl=1, sign=-1),
                                 T(SQR, b[2], xi=1, sign=-1)])
    return [finish(o0), finish(o1), finish(o2), None, None, None]


def prog_inv2():
    t = [ref(B_T, i) for i in range(3)]
    oA = Out(ref(B_T, 3), terms=[Term(SQR, t[0]), Term(KARA, t[1], t[2], xi=1, sign=-1)])
    oB = Out(ref(B_T, 4), terms=[Term(SQR, t[2], xi=1), Term(KARA, t[0], t[1], sign=-1)])
    oC = Out(ref(B_T, 5), terms=[Term(SQR, t[1]), Term(KARA, t[0], t[2], sign=-1)])
    return [finish(oA), finish(oB), finish(oC), None, None, None]


def prog_inv3():
    t = [ref(B_T, i) for i in range(3)]
    A, B, C = ref(B_T, 3), ref(B_T, 4), ref(B_T, 5)
    oF = Out(ref(B_T, 6), terms=[Term(KARA, t[0], A), Term(KARA, t[2], B, xi=1), Term(KARA, t[1], C, xi=1)])
    return [finish(oF), None, None, None, None, None]


def prog_inv4():
    return [finish(Out(ref(B_T, 7), terms=[Term(NORM, ref(B_T, 6))])), None, None, None, None, None]


def prog_inv5():
    o = Out(ref(B_T, 8), mode=M_INVFP, lins=[(1, ref(B_T, 7))])
    return [o, None, None, None, None, None]


def prog_inv6():
    o = Out(ref(B_T, 9), terms=[Term(FPMUL, ref(B_T, 6), ref(B_T, 8))], c_re=1, c_im=-1)
    return [finish(o), None, None, None, None, None]


def prog_inv7():
    return [finish(Out(ref(B_T, 10 + i), terms=[Term(KARA, ref(B_T, 3 + i), ref(B_T, 9))])) for i in range(3)] + \
        [None, None, None]


def prog_inv8():
    ti = [ref(B_T, 10 + i) for i in range(3)]
    outs = []
    for half in range(2):
        x = [ref(B_A, 3 * half + i) for i in range(3)]
        s = 1 if half == 0 else -1
        # Fp6 product (x0 + x1 v + x2 v^2)(t0 + t1 v + t2 v^2), v^3 = xi
        outs.append(finish(Out(ref(B_D, 3 * half + 0), terms=[Term(KARA, x[0], ti[0], sign=s),
                                                            Term(KARA, x[1], ti[2], xi=1, sign=s),
                                                            Term(KARA, x[2], ti[1], xi=1, sign=s)])))
        outs.append(finish(Out(ref(B_D, 3 * half + 1), terms=[Term(KARA, x[0], ti[1], sign=s),
                                                            Term(KARA, x[1], ti[0], sign=s),
                                                            Term(KARA, x[2], ti[2], xi=1, sign=s)])))
        outs.append(finish(Out(ref(B_D, 3 * half + 2), terms=[Term(KARA, x[0], ti[2], sign=s),
                                                            Term(KARA, x[1], ti[1], sign=s),
                                                            Term(KARA, x[2], ti[0], sign=s)])))
    return outs


PROGRAMS = [
    ("LSCALE", prog_lscale, "C: l2 = c1 * P.x, l3 = c0 * P.y for both pairs (api.cu:37-38)"),
    ("LINE1", lambda: prog_line(0), "D = A * line of pair 1 (field_sppark.cuh:126-140)"),
    ("LINE2", lambda: prog_line(1), "D = A * line of pair 2"),
    ("SQR", prog_sqr, "D = A^2 (field_sppark.cuh:148-151)"),
    ("CYCSQR", prog_cycsqr, "D = cyclotomic square of A (field_sppark.cuh:174-197)"),
    ("MUL", prog_mul, "D = A * B (field_sppark.cuh:142-146)"),
    ("FROB", prog_frob, "D = Frobenius(A) (field_sppark.cuh:159-166)"),
    ("CONJ", prog_conj, "D = conjugate(A)"),
    ("COPY", prog_copy, "D = A"),
    ("INV1", prog_inv1, "T0-2 = c0^2 - v c1^2 (field_sppark.cuh:153-157)"),
    ("INV2", prog_inv2, "T3-5 = Fp6 inverse cofactors (field_sppark.cuh:104-111)"),
    ("INV3", prog_inv3, "T6 = Fp6 norm to Fp2"),
    ("INV4", prog_inv4, "T7 = Fp2 norm to Fp (field_sppark.cuh:79-83)"),
    ("INV5", prog_inv5, "T8 = T7^-1 in Fp"),
    ("INV6", prog_inv6, "T9 = T6^-1"),
    ("INV7", prog_inv7, "T10-12 = Fp6 inverse"),
    ("INV8", prog_inv8, "D = A^-1"),
    ("LINE1N", lambda: prog_line_norm(0), "D = A * normalised line of pair 1"),
    ("LINE2N", lambda: prog_line_norm(1), "D = A * normalised line of pair 2"),
    ("SCALE1", lambda: prog_scale(0), "D = A * (Miller correction of pair 1)"),
    ("SCALE2", lambda: prog_scale(1), "D = A * (Miller correction of pair 2)"),
]


# ---------------------------------------------------------------- driver sequence
# The verify kernel runs one op sequence per verification (api.cu:30-52 Miller
# loop, api.cu:54-78 final exponentiation).  An op is a program on Fp12 groups
# (D, A, B), LOAD_LINES(ci) (both pairs' coefficient ci into the C area) or
# MILLER_DONE (the Miller value is complete in group 0).
X_ABS = 0xd201000000010000
OP_LOAD_CORR, OP_MILLER_DONE, OP_LOAD_LINES = 29, 30, 31
COND_ML = 1 << 21     # op runs only when the Miller value is wanted
NO_WAR = 1 << 22      # the op's program writes no slot it reads (set by encode_op)
T_GROUP = 3       # the inverse's temporaries start at group 3's slot 0
PHYS_GROUPS = 7   # Fp12 groups of the item area: one more than the final exponentiation's live values


def logical_sequence(normalised=False):
    """The op sequence of one verification over six logical Fp12 groups;
    `normalised`: the line tables are divided by their c2 (LINE1N / LINE2N)."""
    pid = {name: i for i, (name, _, _) in enumerate(PROGRAMS)}
    seq = []
    l1, l2 = ("LINE1N", "LINE2N") if normalised else ("LINE1", "LINE2")

    def prog(name, d, a=0, b=0):
        seq.append((pid[name], d, a, b, 0))

    def lines(ci):
        seq.append((OP_LOAD_LINES, 0, 0, 0, ci))
        prog("LSCALE", 0)
        prog(l1, 0, 0)
        prog(l2, 0, 0)

    ci = 0
    for bit in range(61, -1, -1):
        lines(ci)
        ci += 1
        if ((X_ABS >> 1) >> bit) & 1:
            lines(ci)
            ci += 1
        prog("SQR", 0, 0)
    lines(ci)
    prog("CONJ", 0, 0)
    if normalised:
        # Miller value = f * (generator's correction) * (key's correction), into group 1
        seq.append((OP_LOAD_CORR | COND_ML, 0, 0, 0, 0))
        seq.append((pid["SCALE1"] | COND_ML, 1, 0, 0, 0))
        seq.append((pid["SCALE2"] | COND_ML, 1, 1, 0, 0))
        seq.append((OP_MILLER_DONE, 1, 0, 0, 0))
    else:
        seq.append((OP_MILLER_DONE, 0, 0, 0, 0))

    def inv(d, a):
        for k in range(1, 9):
            prog("INV%d" % k, d, a)

    def cyc_exp(dst, x):
        # t = x (the leading bit), then square-and-multiply; the first square
        # reads x and writes dst, the rest run in place (programs may overwrite
        # their inputs)
        for i in range(62, -1, -1):
            prog("CYCSQR", dst, dst if i < 62 else x)
            if (X_ABS >> i) & 1:
                prog("MUL", dst, dst, x)
        prog("CONJ", dst, dst)

    # final exponentiation of group 0 into group 0: the reference's chain,
    # api.cu:65-78, over six groups
    prog("CONJ", 1, 0); inv(2, 0); prog("MUL", 3, 1, 2); prog("FROB", 0, 3); prog("FROB", 1, 0)
    prog("MUL", 2, 1, 3); prog("CYCSQR", 0, 2); prog("CONJ", 0, 0)
    cyc_exp(1, 2)
    prog("MUL", 3, 0, 1)
    cyc_exp(0, 3)
    prog("CONJ", 3, 3); prog("MUL", 4, 2, 3); prog("CYCSQR", 3, 1)
    cyc_exp(5, 0)
    prog("MUL", 1, 1, 5); prog("FROB", 1, 1); prog("FROB", 1, 1); prog("MUL", 1, 4, 1)
    cyc_exp(4, 5)
    prog("MUL", 5, 3, 4)
    cyc_exp(3, 5)
    prog("MUL", 4, 1, 3); prog("CONJ", 1, 2); prog("MUL", 3, 5, 1); prog("MUL", 1, 2, 0)
    prog("FROB", 0, 1); prog("FROB", 2, 0); prog("FROB", 0, 2); prog("MUL", 1, 4, 0); prog("FROB", 2, 3)
    prog("MUL", 0, 1, 2)
    return seq


def driver_sequence(normalised=False):
    """The op sequence of one verification as the kernels run it: the groups
    placed by place_groups; Gt ends in group gt_group(normalised)."""
    return place_groups(logical_sequence(normalised))[0]


def gt_group(normalised=False):
    """the physical group that holds Gt after driver_sequence(normalised)"""
    return place_groups(logical_sequence(normalised))[1]


def program_io(code):
    """(bases read, bases written) of program `code`"""
    reads, writes = set(), set()
    for o in PROGRAMS[code][1]():
        if o is None:
            continue
        writes.add(o.dst >> 4)
        reads.update(r >> 4 for t in o.terms for r in (t.x, t.y) if r is not None)
        reads.update(r >> 4 for _, r in o.lins)
    return reads, writes


def live_after(seq):
    """per op, the logical groups a later op still reads (the final value,
    group 0, counts as read at the end; ops that run only when the Miller
    value is wanted read but never end a value's life)"""
    n_prog = len(PROGRAMS)
    out = [None] * len(seq)
    cur = {0}
    for i in range(len(seq) - 1, -1, -1):
        code, d, a, b, _ = seq[i]
        c = code & ~COND_ML
        out[i] = set(cur)
        if c == OP_MILLER_DONE:
            cur.add(d)
            continue
        if c >= n_prog:
            continue
        rb, wb = program_io(c)
        if B_D in wb and not code & COND_ML:
            cur.discard(d)
        if B_A in rb:
            cur.add(a)
        if B_B in rb:
            cur.add(b)
    return out


def place_groups(seq):
    """Put the sequence's Fp12 values (logical groups 0..5) into PHYS_GROUPS
    physical groups so that as few programs as possible write a group they
    read: a result that would overwrite one of its operands (f = f^2,
    f = f * x) goes to a group whose value no later op reads, when there is
    one, and the value moves there.  Such a program writes only slots that
    none of its outputs reads, which lets the kernel store each output as
    soon as it is reduced (no block barrier between the reads and the
    stores; the op's NO_WAR flag).  Parts of the final exponentiation hold
    six live values, so with seven groups there is always one: every
    program of both sequences is out of place, which the 32-item kernel
    relies on (emit refuses a sequence where one is not).  Returns the placed
    sequence and the physical group of the final value (Gt)."""
    n_prog = len(PROGRAMS)
    live = live_after(seq)
    m = {0: 0}                             # logical group -> physical group (f = 1 starts in group 0)
    out = []
    for i, (code, d, a, b, ci) in enumerate(seq):
        c = code & ~COND_ML
        if c < n_prog:
            rb, wb = program_io(c)
            pa = m[a] if B_A in rb else 0
            pb = m[b] if B_B in rb else 0
            if B_D in wb:
                srcs = ({pa} if B_A in rb else set()) | ({pb} if B_B in rb else set())
                busy = {m[x] for x in live[i] if x != d and x in m} | srcs
                if d not in m or m[d] in busy:
                    free = [g for g in range(PHYS_GROUPS) if g not in busy]
                    m[d] = free[0] if free else m[d]
            out.append((code, m[d] if B_D in wb else 0, pa, pb, ci))
        elif c == OP_MILLER_DONE:
            out.append((code, m[d], a, b, ci))
        else:
            out.append((code, d, a, b, ci))
    return out, m[0]


def op_slots(op):
    """(slots read, slots written) of a program op, as (space, index) pairs:
    space 'g' is the item's group area (6 slots per group), 'c' the C area,
    'k' the constant slots"""
    code, d, a, b, ci = op
    code &= ~COND_ML
    base = {B_D: ("g", 6 * d), B_A: ("g", 6 * a), B_B: ("g", 6 * b), B_C: ("c", 0), B_K: ("k", 0),
            B_T: ("g", 6 * T_GROUP)}
    rd, wr = set(), set()
    for o in PROGRAMS[code][1]():
        if o is None:
            continue
        sp, off = base[o.dst >> 4]
        wr.add((sp, off + (o.dst & 15)))
        for r in [r for t in o.terms for r in (t.x, t.y) if r is not None] + [r for _, r in o.lins]:
            sp, off = base[r >> 4]
            rd.add((sp, off + (r & 15)))
    return rd, wr


def no_war(op):
    """the op writes no slot that any of its outputs reads"""
    code = op[0] & ~COND_ML
    if code >= len(PROGRAMS):
        return False
    rd, wr = op_slots(op)
    return not (rd & wr)


def t_slots_used():
    """Temporary slots (base T) any program reads or writes."""
    hi = -1
    for name, fn, _ in PROGRAMS:
        for o in fn():
            if o is None:
                continue
            refs = [o.dst] + [r for t in o.terms for r in (t.x, t.y) if r is not None] + \
                   [l[1] for l in o.lins]
            hi = max([hi] + [r & 15 for r in refs if isinstance(r, int) and (r >> 4) == B_T])
    return hi + 1


def groups_used(seqs):
    """Groups of six Fp2 slots the op sequences need per verification."""
    n_prog = len(PROGRAMS)
    t_slots = t_slots_used()
    hi = 0
    for seq in seqs:
        for code, d, a, b, _ in seq:
            code &= ~COND_ML
            if code < n_prog:
                hi = max(hi, d, a, b)
                if PROGRAMS[code][0].startswith("INV"):
                    hi = max(hi, T_GROUP + (t_slots - 1) // 6)
            elif code == OP_MILLER_DONE:
                hi = max(hi, d)
    return hi + 1


def encode_op(op):
    code, d, a, b, ci = op
    cond = code & COND_ML
    code &= ~COND_ML
    assert code < 32 and d < 8 and a < 8 and b < 8 and ci < 128
    return code | (d << 5) | (a << 8) | (b << 11) | (ci << 14) | cond | (NO_WAR if no_war(op) else 0)


def build():
    progs = []
    for name, fn, doc in PROGRAMS:
        outs = fn()
        assert len(outs) == 6
        progs.append((name, outs, doc))
    return progs


# ---------------------------------------------------------------- emulator
def redc(acc):
    assert 0 <= acc < ACC_LIMIT
    m = (-acc * pow(P, -1, R)) % R
    r = (acc + m * P) >> 384
    assert (acc + m * P) % R == 0
    return r


def qp(v):
    assert 0 <= v < POST_LIMIT, hex(v)
    r = v - QP[v >> 381]
    assert 0 <= r < SLOT_BOUND
    return r


def fp_inv_mont(x):
    """(x R^-1)^-1 R mod p, canonical; 0 for 0."""
    x %= P
    if x == 0:
        return 0
    return pow(x, -1, P) * R * R % P


class Emulator:
    """Slots: dict (absolute slot id) -> (re, im) integers.  `bases` maps the
    base codes to absolute slot ids of index 0."""

    def __init__(self, progs):
        self.progs = {name: outs for name, outs, _ in progs}

    @staticmethod
    def _acc(o, slots, bases):
        """both halves' partial accumulators (half 0 holds the bias), summed
        the way the device exchanges them"""
        parts = []
        for h, half in enumerate(split_halves(o)):
            acc = [o.bias_re * P * R, o.bias_im * P * R] if h == 0 else [0, 0]
            for ti, mask in half:
                t = o.terms[ti]
                X = slots[bases[t.x >> 4] + (t.x & 15)]
                Y = slots[bases[t.y >> 4] + (t.y & 15)] if t.y is not None else None
                al, be = t.coefs()
                if t.kind == ONE:
                    if mask & 1:
                        acc[0] += al[0] * X[0] * R
                        acc[1] += be[0] * X[1] * R
                    continue
                for k, (u, v) in enumerate(t.operands(X, Y)):
                    if not (mask >> k) & 1:
                        continue
                    assert 0 <= u < R and 0 <= v < R
                    pr = u * v
                    acc[0] += al[k] * pr
                    acc[1] += be[k] * pr
            parts.append(acc)
        return [parts[0][0] + parts[1][0], parts[0][1] + parts[1][1]]

    def run(self, name, slots, bases):
        outs = self.progs[name]
        res = []
        for o in outs:
            if o is None:
                continue
            if o.mode == M_INVFP:
                z = slots[bases[o.lins[0][1] >> 4] + (o.lins[0][1] & 15)]
                v = (fp_inv_mont(z[0]), 0)
            elif o.mode == M_LIN:
                v = []
                for c, cc in enumerate((o.c_re, o.c_im)):
                    s = (o.bias_lin_re, o.bias_lin_im)[c] * P
                    for co, r in o.lins:
                        s += cc * co * slots[bases[r >> 4] + (r & 15)][c]
                    v.append(qp(s))
                v = tuple(v)
            else:
                acc = self._acc(o, slots, bases)
                r = [redc(a) for a in acc]
                if o.mode == M_SIMPLE:
                    v = (qp(r[0]), qp(r[1]))
                else:
                    v = []
                    for c, cc in enumerate((o.c_re, o.c_im)):
                        s = (o.bias_lin_re, o.bias_lin_im)[c] * P + cc * qp(r[c])
                        for co, rr in o.lins:
                            s += co * slots[bases[rr >> 4] + (rr & 15)][c]
                        v.append(qp(s))
                    v = tuple(v)
            res.append((bases[o.dst >> 4] + (o.dst & 15), v))
        for d, v in res:      # every lane computes before any writes
            slots[d] = v


# ---------------------------------------------------------------- constants
def _f2_mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def _f2_pow(a, e):
    r = (1, 0)
    while e:
        if e & 1:
            r = _f2_mul(r, a)
        a = _f2_mul(a, a)
        e >>= 1
    return r


def frobenius_gammas():
    """g1 = xi^((p-1)/3), g2 = xi^(2(p-1)/3), g12 = xi^((p-1)/6) (normal form):
    the Frobenius constants of field_sppark.cuh:113-123 and 159-166."""
    xi = (1, 1)
    return _f2_pow(xi, (P - 1) // 3), _f2_pow(xi, 2 * (P - 1) // 3), _f2_pow(xi, (P - 1) // 6)


def k_slot_values():
    """Block-shared constant slots (Montgomery Fp2): 0, 1, then conj(g) for
    g in k1, k2, k12, k1 k12, k2 k12, then 0."""
    k1, k2, k12 = frobenius_gammas()
    gs = [k1, k2, k12, _f2_mul(k1, k12), _f2_mul(k2, k12)]
    mont = lambda v: v * R % P
    out = [(0, 0), (mont(1), 0)] + [(mont(g[0]), mont(-g[1] % P)) for g in gs] + [(0, 0)]
    return out


def _limbs32(v, n=12):
    return ["0x%08xu" % ((v >> (32 * i)) & 0xffffffff) for i in range(n)]


# ---------------------------------------------------------------- C emission
def encode_term(t, mask):
    w = t.kind | (t.xi << 3) | ((1 if t.sign < 0 else 0) << 4) | (t.dbl << 5) | (t.yim << 6)
    w |= t.x << 8
    w |= (t.y if t.y is not None else 0) << 16
    w |= mask << 24
    return w


def encode_out(o, h):
    """The descriptor of half h of an output.
       header: mode | nterms << 2 | nlin << 6 | dst << 8 | (c_re & 15) << 16 | (c_im & 15) << 20
       biases: re | im << 8 | lin_re << 16 | lin_im << 24 (accumulator biases in half 0 only);
       then terms (with the half's product mask in bits 24-26), then lins (coef & 15 | ref << 8)."""
    half = split_halves(o)[h] if o.mode in (M_SIMPLE, M_FULL) else []
    nt, nl = len(half), len(o.lins)
    assert nt < 16 and nl < 4
    hdr = o.mode | (nt << 2) | (nl << 6) | (o.dst << 8) | ((o.c_re & 15) << 16) | ((o.c_im & 15) << 20)
    bre, bim = (o.bias_re, o.bias_im) if h == 0 else (0, 0)
    bias = bre | (bim << 8) | (o.bias_lin_re << 16) | (o.bias_lin_im << 24)
    words = [hdr, bias] + [encode_term(o.terms[ti], m) for ti, m in half] + \
        [(co & 15) | (r << 8) for co, r in o.lins]
    return words


def emit(path):
    progs = build()
    L = ["// Generated by gen_fp2ops.py (Fp2-lane tower programs of the verify",
         "// kernel); do not edit, run `python gen_fp2ops.py`.",
         "#pragma once", "#include <cstdint>", "", "namespace bls {", "namespace f2 {", ""]
    for i, (n, _, doc) in enumerate(progs):
        L.append("constexpr int P_%s = %d;  // %s" % (n, i, doc))
    L.append("constexpr int kNumPrograms = %d;" % len(progs))
    L.append("constexpr uint32_t kModeSimple = %d, kModeFull = %d, kModeLin = %d, kModeInvFp = %d;"
             % (M_SIMPLE, M_FULL, M_LIN, M_INVFP))
    L.append("constexpr uint32_t kKara = %d, kSqr = %d, kFpMul = %d, kNorm = %d, kOne = %d;"
             % (KARA, SQR, FPMUL, NORM, ONE))
    L += ["constexpr int kKFrob = %d;" % K_FROB, ""]
    words, index = [], []
    for n, outs, _ in progs:
        row = []
        for h in range(2):
            for o in outs:
                if o is None:
                    row.append(0xffff)
                else:
                    row.append(len(words))
                    words.extend(encode_out(o, h))
            row += [0xffff, 0xffff]
        index.append(row)
    L.append("// per program, half (8 entries each) and lane: first word of the output")
    L.append("// descriptor (0xffff: none)")
    L.append("__device__ __constant__ uint16_t kOutIndex[%d][16] = {" % len(progs))
    for (n, _, _), row in zip(progs, index):
        L.append("    {%s},  // %s" % (", ".join("%d" % v for v in row), n))
    L.append("};")
    L.append("__device__ __constant__ uint32_t kDesc[%d] = {" % len(words))
    for i in range(0, len(words), 6):
        L.append("    " + ", ".join("0x%08xu" % w for w in words[i:i + 6]) + ",")
    L.append("};")
    L.append("// accumulator coefficients per (kind, xi): alpha0..2, beta0..2, 4 bits each, in {-1, 0, 1}")
    L.append("__device__ __constant__ uint32_t kCoef[10] = {")
    row = []
    for kind in range(5):
        for xi in range(2):
            al, be = COEF.get((kind, xi), ((0, 0, 0), (0, 0, 0)))
            al, be = list(al) + [0] * (3 - len(al)), list(be) + [0] * (3 - len(be))
            w = 0
            for k, v in enumerate(al + be):
                w |= (v & 15) << (4 * k)
            row.append("0x%08xu" % w)
    L.append("    " + ", ".join(row) + ",")
    L.append("};")
    L.append("// block-shared constant slots (Montgomery Fp2, re then im): 0, 1, conj of the")
    L.append("// Frobenius constants k1, k2, k12, k1 k12, k2 k12, 0")
    ks = k_slot_values()
    L.append("__device__ __constant__ uint32_t kKSlots[%d][24] = {" % len(ks))
    for re, im in ks:
        L.append("    {" + ", ".join(_limbs32(re) + _limbs32(im)) + "},")
    L.append("};")
    L.append("constexpr int kKSlotCount = %d;" % len(ks))
    L.append("// R^3 mod p: u * R^3 * R^-1 = u R^2 turns a plain inverse into Montgomery form")
    L.append("__device__ __constant__ uint32_t kR3[12] = {" + ", ".join(_limbs32(R * R * R % P)) + "};")
    L.append("// 3p, the offset of SQR's x0 - x1 + 3p")
    L.append("__device__ __constant__ uint32_t k3P[12] = {" + ", ".join(_limbs32(K3P)) + "};")
    L.append("// the verify op sequences (raw and normalised line tables): code | D << 5 | A << 8 | B << 11 |")
    L.append("// ci << 14; code < kNumPrograms is a program, kOpLoadLines loads line coefficient ci,")
    L.append("// kOpMillerDone marks the Miller value")
    L.append("// kOpLoadCorr loads the Miller correction factors; ops with kCondMl run only when the Miller")
    L.append("// value is wanted; kOpMillerDone emits group D")
    L.append("constexpr uint32_t kOpLoadCorr = %d, kOpMillerDone = %d, kOpLoadLines = %d, kCondMl = 0x%xu;"
             % (OP_LOAD_CORR, OP_MILLER_DONE, OP_LOAD_LINES, COND_ML))
    L.append("// kNoWar: the program writes no slot that any of its outputs reads, so its stores need")
    L.append("// no block barrier after the reads")
    L.append("constexpr uint32_t kNoWar = 0x%xu;" % NO_WAR)
    L.append("constexpr int kTGroup = %d;" % T_GROUP)
    max_bias = max(b for name, fn, _ in PROGRAMS for o in fn() if o is not None
                   for b in (o.bias_re, o.bias_im, o.bias_lin_re, o.bias_lin_im))
    L.append("// largest bias multiple k of any output (the kernel keeps k p for k = 0 .. kMaxBias)")
    L.append("constexpr int kMaxBias = %d;" % max_bias)
    seqs = [driver_sequence(False), driver_sequence(True)]
    for seq in seqs:   # verify_w.cu stores a program's outputs without a barrier after its reads
        assert all(no_war(op) for op in seq if (op[0] & ~COND_ML) < len(PROGRAMS))
    L.append("// Fp12 groups the sequences touch (operands, results, the inverse's temporaries)")
    L.append("constexpr int kGroupsUsed = %d;" % groups_used(seqs))
    L.append("// the group that holds Gt at the end of each sequence (raw, normalised)")
    L.append("__device__ __constant__ uint32_t kGtGroup[2] = {%d, %d};" % (gt_group(False), gt_group(True)))
    n = max(len(q) for q in seqs)
    L.append("constexpr int kSeqLenRaw = %d, kSeqLenNorm = %d;" % (len(seqs[0]), len(seqs[1])))
    L.append("__device__ __constant__ uint32_t kSeq[2][%d] = {" % n)
    for seq in seqs:
        words = [encode_op(op) for op in seq] + [0] * (n - len(seq))
        L.append("  {")
        for i in range(0, len(words), 8):
            L.append("    " + ", ".join("0x%05xu" % w for w in words[i:i + 8]) + ",")
        L.append("  },")
    L.append("};")
    L.append("// QP[h] = floor(h * 2^381 / p) * p, 13 words padded to 16")
    L.append("__device__ const uint32_t kQP2[128][16] = {")
    for q in QP:
        L.append("    {" + ", ".join("0x%08xu" % ((q >> (32 * i)) & 0xffffffff) for i in range(16)) + "},")
    L.append("};")
    L += ["", "}  // namespace f2", "}  // namespace bls"]
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def summary():
    out = []
    for n, outs, _ in build():
        per = []
        for o in outs:
            if o is None:
                per.append((0, 0))
            else:
                per.append((half_products(o, 0), half_products(o, 1)))
        mx = max(max(a, b) for a, b in per)
        tot = sum(a + b for a, b in per)
        redcs = sum(2 for o in outs if o is not None and o.mode in (M_SIMPLE, M_FULL))
        out.append("%-7s products per thread (half 0, half 1) %s  (max %2d, total %3d), REDC %2d"
                   % (n, per, mx, tot, redcs))
    return out


if __name__ == "__main__":
    if "--summary" in sys.argv:
        print("\n".join(summary()))
    else:
        emit(os.path.join(os.path.dirname(os.path.abspath(__file__)), "fp2ops.inc"))
