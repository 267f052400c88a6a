// BLS12-381 verify path restated in C++ on 6 x 64-bit limbs.
//
// TEST INFRASTRUCTURE ONLY: this is the checker and the timed CPU baseline.
// Tests, the smoke run and the bench's CPU leg load it; the GPU library never
// links or calls it.
//
// It follows the reference's verifier operation by operation:
//   tower arithmetic       gpu-crypto/cuda/field_sppark.cuh:40-197
//   Miller loop            gpu-crypto/cuda/api.cu:22-52
//   final exponentiation   gpu-crypto/cuda/api.cu:54-78
//   identity compare       gpu-crypto/cuda/api.cu:80-91
//   G2 line coefficients   cuda/test_miller_v2.cu:148-229 (eprint 2010/354 Alg. 26/27)
//   G1 decompression       cuda/decompress.cu:107-187 for the value path, plus the
//                          checks ic_bls12_381's G1Affine::from_compressed makes
//                          (flags, x < p, square, subgroup).
// Montgomery form with R = 2^384; every stored value is canonical (< p), so
// limbs compare bit for bit with ic_bls12_381's in-memory representation.
// The identity rule of ic_bls12_381's multi_miller_loop (a pair with an
// identity point contributes nothing) is applied to G1 inputs whose limbs are
// x = 0 and y in {0, R mod p}; no point of the curve has x = 0.
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>
#include <atomic>

typedef unsigned __int128 u128;

namespace oc {

static const uint64_t PM[6] = {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                               0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
static const uint64_t INV = 0x89f3fffcfffcfffdULL;  // -p^-1 mod 2^64
static const uint64_t ONE[6] = {0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL,
                                0x77ce585370525745ULL, 0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL};
static const uint64_t RR[6] = {0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL,
                               0x67eb88a9939d83c0ULL, 0x9a793e85b519952dULL, 0x11988fe592cae3aaULL};
static const uint64_t BLS_X = 0xd201000000010000ULL;

struct Fp { uint64_t l[6]; };

static inline bool geq_p(const uint64_t* a) {
    for (int i = 5; i >= 0; --i) {
        if (a[i] > PM[i]) return true;
        if (a[i] < PM[i]) return false;
    }
    return true;
}
static inline void sub_p(uint64_t* a) {
    uint64_t br = 0;
    for (int i = 0; i < 6; ++i) {
        u128 d = (u128)a[i] - PM[i] - br;
        a[i] = (uint64_t)d;
        br = (uint64_t)(d >> 64) & 1;
    }
}
static inline Fp fzero() { Fp r; memset(r.l, 0, 48); return r; }
static inline Fp fone() { Fp r; memcpy(r.l, ONE, 48); return r; }
static inline bool fis_zero(const Fp& a) {
    uint64_t o = 0;
    for (int i = 0; i < 6; ++i) o |= a.l[i];
    return o == 0;
}
static inline bool feq(const Fp& a, const Fp& b) { return memcmp(a.l, b.l, 48) == 0; }

static inline Fp fadd(const Fp& a, const Fp& b) {
    Fp r; uint64_t c = 0;
    for (int i = 0; i < 6; ++i) {
        u128 s = (u128)a.l[i] + b.l[i] + c;
        r.l[i] = (uint64_t)s; c = (uint64_t)(s >> 64);
    }
    if (c || geq_p(r.l)) sub_p(r.l);
    return r;
}
static inline Fp fsub(const Fp& a, const Fp& b) {
    Fp r; uint64_t br = 0;
    for (int i = 0; i < 6; ++i) {
        u128 d = (u128)a.l[i] - b.l[i] - br;
        r.l[i] = (uint64_t)d; br = (uint64_t)(d >> 64) & 1;
    }
    if (br) {
        uint64_t c = 0;
        for (int i = 0; i < 6; ++i) {
            u128 s = (u128)r.l[i] + PM[i] + c;
            r.l[i] = (uint64_t)s; c = (uint64_t)(s >> 64);
        }
    }
    return r;
}
static inline Fp fneg(const Fp& a) { return fsub(fzero(), a); }

// Montgomery product (CIOS, Koc-Acar-Kaliski 1996), result canonical.
static inline Fp fmul(const Fp& a, const Fp& b) {
    uint64_t t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 6; ++i) {
        uint64_t c = 0;
        for (int j = 0; j < 6; ++j) {
            u128 s = (u128)a.l[j] * b.l[i] + t[j] + c;
            t[j] = (uint64_t)s; c = (uint64_t)(s >> 64);
        }
        u128 s = (u128)t[6] + c; t[6] = (uint64_t)s; t[7] = (uint64_t)(s >> 64);
        uint64_t m = t[0] * INV;
        s = (u128)m * PM[0] + t[0]; c = (uint64_t)(s >> 64);
        for (int j = 1; j < 6; ++j) {
            s = (u128)m * PM[j] + t[j] + c;
            t[j - 1] = (uint64_t)s; c = (uint64_t)(s >> 64);
        }
        s = (u128)t[6] + c; t[5] = (uint64_t)s;
        t[6] = t[7] + (uint64_t)(s >> 64);
    }
    Fp r; memcpy(r.l, t, 48);
    if (t[6] || geq_p(r.l)) sub_p(r.l);
    return r;
}
static inline Fp fsqr(const Fp& a) { return fmul(a, a); }

static Fp fpow(const Fp& a, const uint64_t* e, int nlimbs) {
    Fp r = fone(), base = a;
    for (int w = 0; w < nlimbs; ++w)
        for (int b = 0; b < 64; ++b) {
            if ((e[w] >> b) & 1) r = fmul(r, base);
            base = fsqr(base);
        }
    return r;
}
// a^(p-2): Fermat inversion, 0 -> 0 (field_sppark.cuh:40-50)
static Fp finv(const Fp& a) {
    static const uint64_t E[6] = {0xb9feffffffffaaa9ULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                                  0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
    return fpow(a, E, 6);
}
// a^((p+1)/4) (cuda/decompress.cu:16-40)
static Fp fsqrt_cand(const Fp& a) {
    static const uint64_t E[6] = {0xee7fbfffffffeaabULL, 0x07aaffffac54ffffULL, 0xd9cc34a83dac3d89ULL,
                                  0xd91dd2e13ce144afULL, 0x92c6e9ed90d2eb35ULL, 0x0680447a8e5ff9a6ULL};
    return fpow(a, E, 6);
}
static Fp from_raw(const uint64_t* v) { Fp a; memcpy(a.l, v, 48); return a; }
static Fp to_mont(const uint64_t* v) { Fp rr; memcpy(rr.l, RR, 48); return fmul(from_raw(v), rr); }
static void from_mont(const Fp& a, uint64_t* out) {
    Fp one_raw = fzero(); one_raw.l[0] = 1;
    Fp r = fmul(a, one_raw);
    memcpy(out, r.l, 48);
}
// a > (p-1)/2 on the canonical integer
static bool lex_largest(const Fp& a) {
    static const uint64_t HALF[6] = {0xdcff7fffffffd555ULL, 0x0f55ffff58a9ffffULL, 0xb39869507b587b12ULL,
                                     0xb23ba5c279c2895fULL, 0x258dd3db21a5d66bULL, 0x0d0088f51cbff34dULL};
    uint64_t v[6]; from_mont(a, v);
    for (int i = 5; i >= 0; --i) {
        if (v[i] > HALF[i]) return true;
        if (v[i] < HALF[i]) return false;
    }
    return false;
}

// ---------------- Fp2 ----------------
struct Fp2 { Fp c0, c1; };
static inline Fp2 f2zero() { return {fzero(), fzero()}; }
static inline Fp2 f2one() { return {fone(), fzero()}; }
static inline Fp2 f2add(const Fp2& a, const Fp2& b) { return {fadd(a.c0, b.c0), fadd(a.c1, b.c1)}; }
static inline Fp2 f2sub(const Fp2& a, const Fp2& b) { return {fsub(a.c0, b.c0), fsub(a.c1, b.c1)}; }
static inline Fp2 f2neg(const Fp2& a) { return {fneg(a.c0), fneg(a.c1)}; }
static inline Fp2 f2conj(const Fp2& a) { return {a.c0, fneg(a.c1)}; }
static inline Fp2 f2mul_nr(const Fp2& a) { return {fsub(a.c0, a.c1), fadd(a.c0, a.c1)}; }
static inline Fp2 f2mul_fp(const Fp2& a, const Fp& s) { return {fmul(a.c0, s), fmul(a.c1, s)}; }
static inline Fp2 f2mul(const Fp2& a, const Fp2& b) {
    Fp t0 = fmul(a.c0, b.c0), t1 = fmul(a.c1, b.c1);
    return {fsub(t0, t1), fsub(fsub(fmul(fadd(a.c0, a.c1), fadd(b.c0, b.c1)), t0), t1)};
}
static inline Fp2 f2sqr(const Fp2& a) {
    Fp t = fmul(a.c0, a.c1);
    return {fmul(fadd(a.c0, a.c1), fsub(a.c0, a.c1)), fadd(t, t)};
}
static Fp2 f2inv(const Fp2& a) {
    Fp n = fadd(fsqr(a.c0), fsqr(a.c1));
    Fp i = finv(n);
    return {fmul(a.c0, i), fneg(fmul(a.c1, i))};
}
static inline bool f2is_zero(const Fp2& a) { return fis_zero(a.c0) && fis_zero(a.c1); }

// ---------------- Fp6 ----------------
struct Fp6 { Fp2 c0, c1, c2; };
static inline Fp6 f6zero() { return {f2zero(), f2zero(), f2zero()}; }
static inline Fp6 f6one() { return {f2one(), f2zero(), f2zero()}; }
static inline Fp6 f6add(const Fp6& a, const Fp6& b) { return {f2add(a.c0, b.c0), f2add(a.c1, b.c1), f2add(a.c2, b.c2)}; }
static inline Fp6 f6sub(const Fp6& a, const Fp6& b) { return {f2sub(a.c0, b.c0), f2sub(a.c1, b.c1), f2sub(a.c2, b.c2)}; }
static inline Fp6 f6neg(const Fp6& a) { return {f2neg(a.c0), f2neg(a.c1), f2neg(a.c2)}; }
static inline Fp6 f6mul_by_v(const Fp6& a) { return {f2mul_nr(a.c2), a.c0, a.c1}; }
static Fp6 f6mul(const Fp6& a, const Fp6& b) {
    Fp2 aa = f2mul(a.c0, b.c0), bb = f2mul(a.c1, b.c1), cc = f2mul(a.c2, b.c2);
    return {f2add(aa, f2mul_nr(f2sub(f2sub(f2mul(f2add(a.c1, a.c2), f2add(b.c1, b.c2)), bb), cc))),
            f2add(f2sub(f2sub(f2mul(f2add(a.c0, a.c1), f2add(b.c0, b.c1)), aa), bb), f2mul_nr(cc)),
            f2add(f2sub(f2sub(f2mul(f2add(a.c0, a.c2), f2add(b.c0, b.c2)), aa), cc), bb)};
}
static Fp6 f6inv(const Fp6& f) {
    Fp2 c0s = f2sqr(f.c0), c1s = f2sqr(f.c1), c2s = f2sqr(f.c2);
    Fp2 c01 = f2mul(f.c0, f.c1), c02 = f2mul(f.c0, f.c2), c12 = f2mul(f.c1, f.c2);
    Fp2 t0 = f2sub(c0s, f2mul_nr(c12)), t1 = f2sub(f2mul_nr(c2s), c01), t2 = f2sub(c1s, c02);
    Fp2 sc = f2add(f2mul(f.c0, t0), f2mul_nr(f2add(f2mul(f.c2, t1), f2mul(f.c1, t2))));
    Fp2 si = f2inv(sc);
    return {f2mul(t0, si), f2mul(t1, si), f2mul(t2, si)};
}
static const uint64_t FROB6_C1[6] = {0xcd03c9e48671f071ULL, 0x5dab22461fcda5d2ULL, 0x587042afd3851b95ULL,
                                     0x8eb60ebe01bacb9eULL, 0x03f97d6e83d050d2ULL, 0x18f0206554638741ULL};
static const uint64_t FROB6_C2[6] = {0x890dc9e4867545c3ULL, 0x2af322533285a5d5ULL, 0x50880866309b7e2cULL,
                                     0xa20d1b8c7e881024ULL, 0x14e4f04fe2db9068ULL, 0x14e56d3f1564853aULL};
static const uint64_t FROB12_C0[6] = {0x07089552b319d465ULL, 0xc6695f92b50a8313ULL, 0x97e83cccd117228fULL,
                                      0xa35baecab2dc29eeULL, 0x1ce393ea5daace4dULL, 0x08f2220fb0fb66ebULL};
static const uint64_t FROB12_C1[6] = {0xb2f66aad4ce5d646ULL, 0x5842a06bfc497cecULL, 0xcf4895d42599d394ULL,
                                      0xc11b9cba40a8e8d0ULL, 0x2e3813cbe5a0de89ULL, 0x110eefda88847fafULL};
static Fp6 f6frob(const Fp6& f) {
    Fp2 k1 = {fzero(), from_raw(FROB6_C1)};
    Fp2 k2 = {from_raw(FROB6_C2), fzero()};
    return {f2conj(f.c0), f2mul(f2conj(f.c1), k1), f2mul(f2conj(f.c2), k2)};
}
static Fp6 f6mul_by_01(const Fp6& s, const Fp2& c0, const Fp2& c1) {
    Fp2 aa = f2mul(s.c0, c0), bb = f2mul(s.c1, c1);
    return {f2add(f2mul_nr(f2mul(s.c2, c1)), aa),
            f2sub(f2sub(f2mul(f2add(c0, c1), f2add(s.c0, s.c1)), aa), bb),
            f2add(f2mul(s.c2, c0), bb)};
}
static Fp6 f6mul_by_1(const Fp6& s, const Fp2& c1) {
    return {f2mul_nr(f2mul(s.c2, c1)), f2mul(s.c0, c1), f2mul(s.c1, c1)};
}

// ---------------- Fp12 ----------------
struct Fp12 { Fp6 c0, c1; };
static inline Fp12 f12one() { return {f6one(), f6zero()}; }
static inline Fp12 f12conj(const Fp12& a) { return {a.c0, f6neg(a.c1)}; }
static Fp12 f12mul(const Fp12& a, const Fp12& b) {
    Fp6 aa = f6mul(a.c0, b.c0), bb = f6mul(a.c1, b.c1);
    return {f6add(aa, f6mul_by_v(bb)), f6sub(f6sub(f6mul(f6add(a.c0, a.c1), f6add(b.c0, b.c1)), aa), bb)};
}
static Fp12 f12sqr(const Fp12& a) {
    Fp6 ab = f6mul(a.c0, a.c1), s1 = f6add(a.c0, a.c1), s2 = f6add(a.c0, f6mul_by_v(a.c1));
    return {f6sub(f6sub(f6mul(s2, s1), ab), f6mul_by_v(ab)), f6add(ab, ab)};
}
static Fp12 f12inv(const Fp12& f) {
    Fp6 t = f6sub(f6mul(f.c0, f.c0), f6mul_by_v(f6mul(f.c1, f.c1)));
    Fp6 ti = f6inv(t);
    return {f6mul(f.c0, ti), f6neg(f6mul(f.c1, ti))};
}
static Fp12 f12frob(const Fp12& f) {
    Fp6 c0 = f6frob(f.c0), c1 = f6frob(f.c1);
    Fp2 co = {from_raw(FROB12_C0), from_raw(FROB12_C1)};
    return {c0, {f2mul(c1.c0, co), f2mul(c1.c1, co), f2mul(c1.c2, co)}};
}
static Fp12 f12mul_by_014(const Fp12& f, const Fp2& c0, const Fp2& c1, const Fp2& c4) {
    Fp6 aa = f6mul_by_01(f.c0, c0, c1), bb = f6mul_by_1(f.c1, c4);
    return {f6add(f6mul_by_v(bb), aa), f6sub(f6sub(f6mul_by_01(f6add(f.c1, f.c0), c0, f2add(c1, c4)), aa), bb)};
}
static void fp4_square(const Fp2& a, const Fp2& b, Fp2& o0, Fp2& o1) {
    Fp2 t0 = f2sqr(a), t1 = f2sqr(b);
    o0 = f2add(f2mul_nr(t1), t0);
    o1 = f2sub(f2sub(f2sqr(f2add(a, b)), t0), t1);
}
static Fp12 f12cyc_sqr(const Fp12& f) {
    Fp2 z0 = f.c0.c0, z4 = f.c0.c1, z3 = f.c0.c2, z2 = f.c1.c0, z1 = f.c1.c1, z5 = f.c1.c2;
    Fp2 A0, A1; fp4_square(z0, z1, A0, A1);
    z0 = f2sub(A0, z0); z0 = f2add(f2add(z0, z0), A0);
    z1 = f2add(A1, z1); z1 = f2add(f2add(z1, z1), A1);
    Fp2 B0, B1; fp4_square(z2, z3, B0, B1);
    Fp2 C0, C1; fp4_square(z4, z5, C0, C1);
    z4 = f2sub(B0, z4); z4 = f2add(f2add(z4, z4), B0);
    z5 = f2add(B1, z5); z5 = f2add(f2add(z5, z5), B1);
    Fp2 nr = f2mul_nr(C1);
    z2 = f2add(nr, z2); z2 = f2add(f2add(z2, z2), nr);
    z3 = f2sub(C0, z3); z3 = f2add(f2add(z3, z3), C0);
    return {{z0, z4, z3}, {z2, z1, z5}};
}

// ---------------- Miller loop / final exponentiation ----------------
struct G1 { Fp x, y; };

static inline void load_coeff(const uint64_t* co, int idx, Fp2& c0, Fp2& c1, Fp2& c2) {
    const uint64_t* b = co + 36 * idx;
    c0 = {from_raw(b), from_raw(b + 6)};
    c1 = {from_raw(b + 12), from_raw(b + 18)};
    c2 = {from_raw(b + 24), from_raw(b + 30)};
}
static inline Fp12 ell(const Fp12& f, const uint64_t* co, int idx, const G1& p) {
    Fp2 c0, c1, c2;
    load_coeff(co, idx, c0, c1, c2);
    return f12mul_by_014(f, c2, f2mul_fp(c1, p.x), f2mul_fp(c0, p.y));
}
static Fp12 multi_miller_2(const G1& p1, const uint64_t* q1, bool skip1,
                           const G1& p2, const uint64_t* q2, bool skip2) {
    Fp12 f = f12one();
    int ci = 0; bool found = false;
    for (int b = 63; b >= 0; --b) {
        bool bit = (((BLS_X >> 1) >> b) & 1) == 1;
        if (!found) { found = bit; continue; }
        if (!skip1) f = ell(f, q1, ci, p1);
        if (!skip2) f = ell(f, q2, ci, p2);
        ++ci;
        if (bit) {
            if (!skip1) f = ell(f, q1, ci, p1);
            if (!skip2) f = ell(f, q2, ci, p2);
            ++ci;
        }
        f = f12sqr(f);
    }
    if (!skip1) f = ell(f, q1, ci, p1);
    if (!skip2) f = ell(f, q2, ci, p2);
    return f12conj(f);
}
static Fp12 cyc_exp(const Fp12& f) {
    Fp12 t = f12one(); bool fd = false;
    for (int i = 63; i >= 0; --i) {
        if (fd) t = f12cyc_sqr(t);
        bool bit = ((BLS_X >> i) & 1) == 1;
        if (!fd) { fd = bit; if (!bit) continue; }
        if (bit) t = f12mul(t, f);
    }
    return f12conj(t);
}
static Fp12 final_exp(const Fp12& fi) {
    Fp12 f = fi, t0 = f12conj(f), t1 = f12inv(f), t2 = f12mul(t0, t1);
    t1 = t2; t2 = f12mul(f12frob(f12frob(t2)), t1);
    f = t2; t1 = f12conj(f12cyc_sqr(t2));
    Fp12 t3 = cyc_exp(t2), t4 = f12mul(t1, t3); t1 = cyc_exp(t4);
    t4 = f12conj(t4); f = f12mul(f, t4);
    t4 = f12cyc_sqr(t3); t0 = cyc_exp(t1); t3 = f12mul(t3, t0);
    t3 = f12frob(f12frob(t3)); f = f12mul(f, t3);
    t4 = f12mul(t4, cyc_exp(t0)); f = f12mul(f, cyc_exp(t4));
    t4 = f12mul(t4, f12conj(t2)); t2 = f12mul(t2, t1);
    t2 = f12frob(f12frob(f12frob(t2))); f = f12mul(f, t2);
    t4 = f12frob(t4); f = f12mul(f, t4);
    return f;
}
static bool f12is_one(const Fp12& r) {
    const Fp* fps = (const Fp*)&r;
    if (!feq(fps[0], fone())) return false;
    for (int i = 1; i < 12; ++i) if (!fis_zero(fps[i])) return false;
    return true;
}
static bool g1_is_identity_limbs(const uint64_t* xy) {
    Fp x = from_raw(xy), y = from_raw(xy + 6);
    return fis_zero(x) && (fis_zero(y) || feq(y, fone()));
}

// ---------------- G1 group (Jacobian) for the subgroup check ----------------
struct G1J { Fp X, Y, Z; };
static G1J g1j_dbl(const G1J& p) {
    if (fis_zero(p.Z)) return p;
    Fp A = fsqr(p.X), B = fsqr(p.Y), C = fsqr(B);
    Fp D = fsub(fsub(fsqr(fadd(p.X, B)), A), C); D = fadd(D, D);
    Fp E = fadd(fadd(A, A), A), F = fsqr(E);
    G1J r;
    r.X = fsub(F, fadd(D, D));
    Fp C8 = fadd(C, C); C8 = fadd(C8, C8); C8 = fadd(C8, C8);
    r.Y = fsub(fmul(E, fsub(D, r.X)), C8);
    r.Z = fmul(fadd(p.Y, p.Y), p.Z);
    return r;
}
static G1J g1j_add(const G1J& p, const G1J& q) {
    if (fis_zero(p.Z)) return q;
    if (fis_zero(q.Z)) return p;
    Fp Z1Z1 = fsqr(p.Z), Z2Z2 = fsqr(q.Z);
    Fp U1 = fmul(p.X, Z2Z2), U2 = fmul(q.X, Z1Z1);
    Fp S1 = fmul(fmul(p.Y, q.Z), Z2Z2), S2 = fmul(fmul(q.Y, p.Z), Z1Z1);
    if (feq(U1, U2)) {
        if (feq(S1, S2)) return g1j_dbl(p);
        G1J o; o.X = fone(); o.Y = fone(); o.Z = fzero(); return o;
    }
    Fp H = fsub(U2, U1), I = fsqr(fadd(H, H)), J = fmul(H, I);
    Fp rr = fsub(S2, S1); rr = fadd(rr, rr);
    Fp V = fmul(U1, I);
    G1J o;
    o.X = fsub(fsub(fsqr(rr), J), fadd(V, V));
    Fp S1J = fmul(S1, J);
    o.Y = fsub(fmul(rr, fsub(V, o.X)), fadd(S1J, S1J));
    o.Z = fmul(fsub(fsub(fsqr(fadd(p.Z, q.Z)), Z1Z1), Z2Z2), H);
    return o;
}
static bool g1_in_subgroup(const Fp& x, const Fp& y) {
    static const uint64_t RORD[4] = {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL,
                                     0x3339d80809a1d805ULL, 0x73eda753299d7d48ULL};
    G1J base = {x, y, fone()}, acc; acc.X = fone(); acc.Y = fone(); acc.Z = fzero();
    for (int w = 3; w >= 0; --w)
        for (int b = 63; b >= 0; --b) {
            acc = g1j_dbl(acc);
            if ((RORD[w] >> b) & 1) acc = g1j_add(acc, base);
        }
    return fis_zero(acc.Z);
}

// status codes shared with the GPU library
enum { ST_OK = 0, ST_BAD_FLAGS = 1, ST_X_NOT_CANONICAL = 2, ST_NOT_ON_CURVE = 3, ST_NOT_IN_SUBGROUP = 4 };

// 48 compressed bytes -> status, affine Montgomery (x, y); identity -> x = 0, y = R.
static int g1_decompress(const uint8_t* in, uint64_t* out_xy, bool* is_identity) {
    *is_identity = false;
    memset(out_xy, 0, 96);
    uint8_t top = in[0];
    bool comp = (top >> 7) & 1, inf = (top >> 6) & 1, sort = (top >> 5) & 1;
    uint64_t xv[6];
    for (int i = 0; i < 6; ++i) {
        uint64_t v = 0;
        for (int j = 0; j < 8; ++j) v = (v << 8) | (uint64_t)(i == 0 && j == 0 ? (in[0] & 0x1f) : in[i * 8 + j]);
        xv[5 - i] = v;
    }
    if (!comp) return ST_BAD_FLAGS;
    if (inf) {
        uint64_t o = 0;
        for (int i = 0; i < 6; ++i) o |= xv[i];
        if (sort || o) return ST_BAD_FLAGS;
        *is_identity = true;
        memcpy(out_xy + 6, ONE, 48);
        return ST_OK;
    }
    if (geq_p(xv)) return ST_X_NOT_CANONICAL;
    Fp x = to_mont(xv);
    Fp four = fadd(fadd(fone(), fone()), fadd(fone(), fone()));
    Fp y2 = fadd(fmul(fsqr(x), x), four);
    Fp y = fsqrt_cand(y2);
    if (!feq(fsqr(y), y2)) return ST_NOT_ON_CURVE;
    if (lex_largest(y) != sort) y = fneg(y);
    if (!g1_in_subgroup(x, y)) return ST_NOT_IN_SUBGROUP;
    memcpy(out_xy, x.l, 48);
    memcpy(out_xy + 6, y.l, 48);
    return ST_OK;
}

// ---------------- G2 line coefficients (cuda/test_miller_v2.cu:148-229) ----------------
struct G2P { Fp2 x, y, z; };
static void doubling_step(G2P& r, Fp2* out) {
    Fp2 tmp0 = f2sqr(r.x), tmp1 = f2sqr(r.y), tmp2 = f2sqr(tmp1);
    Fp2 tmp3 = f2sub(f2sqr(f2add(tmp1, r.x)), f2add(tmp0, tmp2));
    tmp3 = f2add(tmp3, tmp3);
    Fp2 tmp4 = f2add(f2add(tmp0, tmp0), tmp0);
    Fp2 tmp6 = f2add(r.x, tmp4);
    Fp2 tmp5 = f2sqr(tmp4);
    Fp2 zsq = f2sqr(r.z);
    r.x = f2sub(f2sub(tmp5, tmp3), tmp3);
    r.z = f2sub(f2sqr(f2add(r.z, r.y)), f2add(tmp1, zsq));
    r.y = f2mul(f2sub(tmp3, r.x), tmp4);
    tmp2 = f2add(tmp2, tmp2); tmp2 = f2add(tmp2, tmp2); tmp2 = f2add(tmp2, tmp2);
    r.y = f2sub(r.y, tmp2);
    tmp3 = f2mul(tmp4, zsq); tmp3 = f2add(tmp3, tmp3); tmp3 = f2neg(tmp3);
    tmp6 = f2sub(f2sqr(tmp6), f2add(tmp0, tmp5));
    tmp1 = f2add(tmp1, tmp1); tmp1 = f2add(tmp1, tmp1);
    tmp6 = f2sub(tmp6, tmp1);
    Fp2 t0o = f2mul(r.z, zsq); t0o = f2add(t0o, t0o);
    out[0] = t0o; out[1] = tmp3; out[2] = tmp6;
}
static void addition_step(G2P& r, const Fp2& qx, const Fp2& qy, Fp2* out) {
    Fp2 zsq = f2sqr(r.z), ysq = f2sqr(qy);
    Fp2 t0 = f2mul(zsq, qx);
    Fp2 t1 = f2mul(f2sub(f2sqr(f2add(qy, r.z)), f2add(ysq, zsq)), zsq);
    Fp2 t2 = f2sub(t0, r.x), t3 = f2sqr(t2);
    Fp2 t4 = f2add(t3, t3); t4 = f2add(t4, t4);
    Fp2 t5 = f2mul(t4, t2);
    Fp2 t6 = f2sub(f2sub(t1, r.y), r.y);
    Fp2 t9 = f2mul(t6, qx), t7 = f2mul(t4, r.x);
    r.x = f2sub(f2sub(f2sub(f2sqr(t6), t5), t7), t7);
    r.z = f2sub(f2sqr(f2add(r.z, t2)), f2add(zsq, t3));
    Fp2 t10 = f2add(qy, r.z);
    Fp2 t8 = f2mul(f2sub(t7, r.x), t6);
    Fp2 t0b = f2mul(r.y, t5); t0b = f2add(t0b, t0b);
    r.y = f2sub(t8, t0b);
    t10 = f2sub(f2sqr(t10), ysq);
    t10 = f2sub(t10, f2sqr(r.z));
    t9 = f2sub(f2add(t9, t9), t10);
    Fp2 t10o = f2add(r.z, r.z);
    t6 = f2neg(t6);
    Fp2 t1o = f2add(t6, t6);
    out[0] = t10o; out[1] = t1o; out[2] = t9;
}
static void store_coeff(uint64_t* dst, const Fp2* c) {
    for (int k = 0; k < 3; ++k) {
        memcpy(dst + 12 * k, c[k].c0.l, 48);
        memcpy(dst + 12 * k + 6, c[k].c1.l, 48);
    }
}

static void verify_one(const uint64_t* sig, const uint64_t* nhm, const uint64_t* g2c, const uint64_t* pkc,
                       bool sig_inf, bool nhm_inf, bool pk_inf, int32_t* res, uint64_t* ml_out, uint64_t* gt_out) {
    G1 s = {from_raw(sig), from_raw(sig + 6)};
    G1 h = {from_raw(nhm), from_raw(nhm + 6)};
    Fp12 ml = multi_miller_2(s, g2c, sig_inf, h, pkc, nhm_inf || pk_inf);
    Fp12 gt = final_exp(ml);
    *res = f12is_one(gt) ? 1 : 0;
    if (ml_out) memcpy(ml_out, &ml, 576);
    if (gt_out) memcpy(gt_out, &gt, 576);
}

template <class F>
static void parallel_for(int n, int nthreads, F fn) {
    if (nthreads <= 1 || n <= 1) { for (int i = 0; i < n; ++i) fn(i); return; }
    std::atomic<int> next(0);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&]() {
            for (;;) {
                int i = next.fetch_add(1);
                if (i >= n) break;
                fn(i);
            }
        });
    for (auto& x : th) x.join();
}

}  // namespace oc

using namespace oc;

extern "C" {

int oc_num_threads(void) { return (int)std::thread::hardware_concurrency(); }

// Montgomery helpers for tests
void oc_fp_mul(const uint64_t* a, const uint64_t* b, uint64_t* out) {
    Fp r = fmul(from_raw(a), from_raw(b)); memcpy(out, r.l, 48);
}

// Raw-ABI semantics: per item x/y limbs; pk tables per item (pk_index == NULL)
// or shared tables indexed by pk_index[i].  pk_inf (nullable) marks identity
// public keys by table index.
int oc_verify_batch(const uint64_t* sigs, const uint64_t* nhms, const uint64_t* g2c, const uint64_t* pkc,
                    const int32_t* pk_index, const uint8_t* pk_inf, int n, int32_t* results,
                    uint64_t* ml_out, uint64_t* gt_out, int nthreads) {
    if (n < 0) return -1;
    parallel_for(n, nthreads, [&](int i) {
        int64_t pki = pk_index ? pk_index[i] : i;
        verify_one(sigs + 12 * (size_t)i, nhms + 12 * (size_t)i, g2c, pkc + 2448 * (size_t)pki,
                   g1_is_identity_limbs(sigs + 12 * (size_t)i), g1_is_identity_limbs(nhms + 12 * (size_t)i),
                   pk_inf ? pk_inf[pki] != 0 : false, results + i,
                   ml_out ? ml_out + 72 * (size_t)i : nullptr, gt_out ? gt_out + 72 * (size_t)i : nullptr);
    });
    return 0;
}

// Compressed signatures: decode (status), then verify the valid ones.
// results[i] = 1 accept, 0 reject, -status for a decode failure.
int oc_verify_compressed_batch(const uint8_t* sigs48, const uint64_t* nhms, const uint64_t* g2c,
                               const uint64_t* pkc, const int32_t* pk_index, const uint8_t* pk_inf,
                               int n, int32_t* results, int nthreads) {
    if (n < 0) return -1;
    parallel_for(n, nthreads, [&](int i) {
        uint64_t xy[12]; bool inf;
        int st = g1_decompress(sigs48 + 48 * (size_t)i, xy, &inf);
        if (st != ST_OK) { results[i] = -st; return; }
        int64_t pki = pk_index ? pk_index[i] : i;
        verify_one(xy, nhms + 12 * (size_t)i, g2c, pkc + 2448 * (size_t)pki, inf,
                   g1_is_identity_limbs(nhms + 12 * (size_t)i), pk_inf ? pk_inf[pki] != 0 : false,
                   results + i, nullptr, nullptr);
    });
    return 0;
}

int oc_g1_decompress(const uint8_t* in48, int n, uint64_t* out_xy, int32_t* status, int nthreads) {
    if (n < 0) return -1;
    parallel_for(n, nthreads, [&](int i) {
        bool inf;
        status[i] = g1_decompress(in48 + 48 * (size_t)i, out_xy + 12 * (size_t)i, &inf);
    });
    return 0;
}

// Affine Montgomery Q (x.c0, x.c1, y.c0, y.c1: 24 u64) -> 68 x 36 u64.
int oc_g2_prepare(const uint64_t* q, uint64_t* coeffs) {
    Fp2 qx = {from_raw(q), from_raw(q + 6)}, qy = {from_raw(q + 12), from_raw(q + 18)};
    G2P r = {qx, qy, f2one()};
    int ci = 0; bool found = false;
    Fp2 c[3];
    for (int b = 63; b >= 0; --b) {
        bool bit = (((BLS_X >> 1) >> b) & 1) == 1;
        if (!found) { found = bit; continue; }
        doubling_step(r, c); store_coeff(coeffs + 36 * ci++, c);
        if (bit) { addition_step(r, qx, qy, c); store_coeff(coeffs + 36 * ci++, c); }
    }
    doubling_step(r, c); store_coeff(coeffs + 36 * ci++, c);
    return ci == 68 ? 0 : -1;
}

// Miller loop and final exponentiation alone (72 u64 Montgomery in/out).
void oc_final_exp(const uint64_t* in72, uint64_t* out72) {
    Fp12 f; memcpy(&f, in72, 576);
    Fp12 r = final_exp(f);
    memcpy(out72, &r, 576);
}
void oc_cyclotomic_square(const uint64_t* in72, uint64_t* out72) {
    Fp12 f; memcpy(&f, in72, 576);
    Fp12 r = f12cyc_sqr(f);
    memcpy(out72, &r, 576);
}

}  // extern "C"
