// Seeded BLS12-381 input generator: keys, messages, hash-to-G1, signatures,
// compressed encodings and G2 line tables, on the host CPU.
//
// This plays the caller's part of the reference path: the IC replica builds
// -H(m) and a G2Prepared table per item on the CPU before calling the GPU
// (ic-integration/patches/ic-gpu-consensus.patch:444-473), and its test and
// bench harnesses make keys and signatures the same way
// (ic-integration/patches/ic-gpu-consensus.patch:476-535).  It produces inputs
// for benches and tests; the verify library never calls it.
//
// Hash to G1 follows RFC 9380's hash_to_curve: expand_message_xmd with
// SHA-256 (FIPS 180-4), hash_to_field (L = 64, two elements), map_to_curve,
// point addition, clear_cofactor by h_eff = 1 - x.  The map is the suite
// BLS12381G1_XMD:SHA-256_SSWU_RO_ (ic_bls12_381's hash_to_curve): the
// simplified SWU map of RFC 9380 section 6.6.2 on the 11-isogenous curve E'
// and the 11-isogeny to E (section 6.6.3), with the constants that
// csrc/gen_h2c.py derives (h2c.inc, host arrays here).
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

typedef unsigned __int128 u128;

#define BLS_H2C_CONST static const
#include "../csrc/h2c.inc"

namespace wl {

// ------------------------------------------------------------------ SHA-256
struct Sha256 {
    uint32_t h[8];
    uint8_t buf[64];
    uint64_t len = 0;
    size_t fill = 0;
    static constexpr uint32_t K[64] = {
        0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
        0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
        0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
        0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
        0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
        0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
        0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
        0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
    Sha256() {
        const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
        memcpy(h, iv, sizeof iv);
    }
    static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
    void block(const uint8_t* p) {
        uint32_t w[64];
        for (int i = 0; i < 16; ++i)
            w[i] = ((uint32_t)p[4 * i] << 24) | ((uint32_t)p[4 * i + 1] << 16) | ((uint32_t)p[4 * i + 2] << 8) | p[4 * i + 3];
        for (int i = 16; i < 64; ++i) {
            uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
            uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
        for (int i = 0; i < 64; ++i) {
            uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
            uint32_t ch = (e & f) ^ (~e & g);
            uint32_t t1 = hh + S1 + ch + K[i] + w[i];
            uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
            uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
            uint32_t t2 = S0 + mj;
            hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
        }
        h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
    }
    void update(const uint8_t* p, size_t n) {
        len += n;
        while (n) {
            size_t k = 64 - fill < n ? 64 - fill : n;
            memcpy(buf + fill, p, k);
            fill += k; p += k; n -= k;
            if (fill == 64) { block(buf); fill = 0; }
        }
    }
    void final(uint8_t out[32]) {
        uint64_t bits = len * 8;
        uint8_t pad = 0x80;
        update(&pad, 1);
        uint8_t z = 0;
        while (fill != 56) update(&z, 1);
        uint8_t lb[8];
        for (int i = 0; i < 8; ++i) lb[i] = (uint8_t)(bits >> (56 - 8 * i));
        update(lb, 8);
        for (int i = 0; i < 8; ++i) {
            out[4 * i] = (uint8_t)(h[i] >> 24); out[4 * i + 1] = (uint8_t)(h[i] >> 16);
            out[4 * i + 2] = (uint8_t)(h[i] >> 8); out[4 * i + 3] = (uint8_t)h[i];
        }
    }
};
constexpr uint32_t Sha256::K[64];

// ------------------------------------------------------------------ Fp (6 x u64, Montgomery)
const uint64_t P[6] = {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                       0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
const uint64_t NINV = 0x89f3fffcfffcfffdULL;
const uint64_t ONE[6] = {0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL,
                         0x77ce585370525745ULL, 0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL};
const uint64_t RR[6] = {0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL,
                        0x67eb88a9939d83c0ULL, 0x9a793e85b519952dULL, 0x11988fe592cae3aaULL};

struct F { uint64_t v[6]; };
inline F zero() { F r{}; return r; }
inline F one() { F r; memcpy(r.v, ONE, 48); return r; }
inline bool is_zero(const F& a) { uint64_t o = 0; for (int i = 0; i < 6; ++i) o |= a.v[i]; return !o; }
inline bool eq(const F& a, const F& b) { return !memcmp(a.v, b.v, 48); }
inline bool geq(const uint64_t* a, const uint64_t* b) {
    for (int i = 5; i >= 0; --i) { if (a[i] != b[i]) return a[i] > b[i]; }
    return true;
}
inline void subp(uint64_t* a) {
    uint64_t br = 0;
    for (int i = 0; i < 6; ++i) { u128 d = (u128)a[i] - P[i] - br; a[i] = (uint64_t)d; br = (uint64_t)(d >> 64) & 1; }
}
inline F add(const F& a, const F& b) {
    F r; uint64_t c = 0;
    for (int i = 0; i < 6; ++i) { u128 s = (u128)a.v[i] + b.v[i] + c; r.v[i] = (uint64_t)s; c = (uint64_t)(s >> 64); }
    if (geq(r.v, P)) subp(r.v);
    return r;
}
inline F sub(const F& a, const F& b) {
    F r; uint64_t br = 0;
    for (int i = 0; i < 6; ++i) { u128 d = (u128)a.v[i] - b.v[i] - br; r.v[i] = (uint64_t)d; br = (uint64_t)(d >> 64) & 1; }
    if (br) { uint64_t c = 0; for (int i = 0; i < 6; ++i) { u128 s = (u128)r.v[i] + P[i] + c; r.v[i] = (uint64_t)s; c = (uint64_t)(s >> 64); } }
    return r;
}
inline F neg(const F& a) { return sub(zero(), a); }
inline F mul(const F& a, const F& b) {
    uint64_t t[8] = {0};
    for (int i = 0; i < 6; ++i) {
        uint64_t c = 0;
        for (int j = 0; j < 6; ++j) { u128 s = (u128)a.v[j] * b.v[i] + t[j] + c; t[j] = (uint64_t)s; c = (uint64_t)(s >> 64); }
        u128 s = (u128)t[6] + c; t[6] = (uint64_t)s; t[7] = (uint64_t)(s >> 64);
        uint64_t m = t[0] * NINV;
        s = (u128)m * P[0] + t[0]; c = (uint64_t)(s >> 64);
        for (int j = 1; j < 6; ++j) { s = (u128)m * P[j] + t[j] + c; t[j - 1] = (uint64_t)s; c = (uint64_t)(s >> 64); }
        s = (u128)t[6] + c; t[5] = (uint64_t)s; t[6] = t[7] + (uint64_t)(s >> 64);
    }
    F r; memcpy(r.v, t, 48);
    if (t[6] || geq(r.v, P)) subp(r.v);
    return r;
}
inline F sqr(const F& a) { return mul(a, a); }
F powe(const F& a, const uint64_t* e) {
    F r = one(), b = a;
    for (int i = 0; i < 384; ++i) { if ((e[i >> 6] >> (i & 63)) & 1) r = mul(r, b); b = sqr(b); }
    return r;
}
const uint64_t E_INV[6] = {0xb9feffffffffaaa9ULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                           0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
const uint64_t E_SQRT[6] = {0xee7fbfffffffeaabULL, 0x07aaffffac54ffffULL, 0xd9cc34a83dac3d89ULL,
                            0xd91dd2e13ce144afULL, 0x92c6e9ed90d2eb35ULL, 0x0680447a8e5ff9a6ULL};
const uint64_t E_LEG[6] = {0xdcff7fffffffd555ULL, 0x0f55ffff58a9ffffULL, 0xb39869507b587b12ULL,
                           0xb23ba5c279c2895fULL, 0x258dd3db21a5d66bULL, 0x0d0088f51cbff34dULL};  // (p-1)/2
inline F inv(const F& a) { return powe(a, E_INV); }
inline bool is_square(const F& a) { return is_zero(a) || eq(powe(a, E_LEG), one()); }
inline F sqrt_cand(const F& a) { return powe(a, E_SQRT); }
F from_raw(const uint64_t* v) { F a; memcpy(a.v, v, 48); return a; }
F to_mont(const uint64_t* v) { F rr; memcpy(rr.v, RR, 48); return mul(from_raw(v), rr); }
void canon(const F& a, uint64_t* out) { F o = zero(); o.v[0] = 1; F r = mul(a, o); memcpy(out, r.v, 48); }
F small(uint64_t k) { uint64_t v[6] = {k, 0, 0, 0, 0, 0}; return to_mont(v); }
bool lex_largest(const F& a) {
    uint64_t c[6]; canon(a, c);
    for (int i = 5; i >= 0; --i) { if (c[i] != E_LEG[i]) return c[i] > E_LEG[i]; }
    return false;
}
int sgn0(const F& a) { uint64_t c[6]; canon(a, c); return (int)(c[0] & 1); }

// ------------------------------------------------------------------ Fp2
struct F2 { F c0, c1; };
inline F2 add2(const F2& a, const F2& b) { return {add(a.c0, b.c0), add(a.c1, b.c1)}; }
inline F2 sub2(const F2& a, const F2& b) { return {sub(a.c0, b.c0), sub(a.c1, b.c1)}; }
inline F2 neg2(const F2& a) { return {neg(a.c0), neg(a.c1)}; }
inline F2 mul2(const F2& a, const F2& b) {
    F t0 = mul(a.c0, b.c0), t1 = mul(a.c1, b.c1);
    return {sub(t0, t1), sub(sub(mul(add(a.c0, a.c1), add(b.c0, b.c1)), t0), t1)};
}
inline F2 sqr2(const F2& a) { F t = mul(a.c0, a.c1); return {mul(add(a.c0, a.c1), sub(a.c0, a.c1)), add(t, t)}; }
inline F2 one2() { return {one(), zero()}; }
inline bool is_zero2(const F2& a) { return is_zero(a.c0) && is_zero(a.c1); }
inline F2 inv2(const F2& a) { F n = add(sqr(a.c0), sqr(a.c1)); F i = inv(n); return {mul(a.c0, i), neg(mul(a.c1, i))}; }
bool lex_largest2(const F2& a) { return lex_largest(a.c1) || (is_zero(a.c1) && lex_largest(a.c0)); }

// ------------------------------------------------------------------ curve arithmetic (Jacobian)
template <class T> struct Ops;
template <> struct Ops<F> {
    static F add(const F& a, const F& b) { return wl::add(a, b); }
    static F sub(const F& a, const F& b) { return wl::sub(a, b); }
    static F mul(const F& a, const F& b) { return wl::mul(a, b); }
    static F sqr(const F& a) { return wl::sqr(a); }
    static F inv(const F& a) { return wl::inv(a); }
    static bool zero(const F& a) { return is_zero(a); }
    static bool eq(const F& a, const F& b) { return wl::eq(a, b); }
    static F one() { return wl::one(); }
};
template <> struct Ops<F2> {
    static F2 add(const F2& a, const F2& b) { return add2(a, b); }
    static F2 sub(const F2& a, const F2& b) { return sub2(a, b); }
    static F2 mul(const F2& a, const F2& b) { return mul2(a, b); }
    static F2 sqr(const F2& a) { return sqr2(a); }
    static F2 inv(const F2& a) { return inv2(a); }
    static bool zero(const F2& a) { return is_zero2(a); }
    static bool eq(const F2& a, const F2& b) { return wl::eq(a.c0, b.c0) && wl::eq(a.c1, b.c1); }
    static F2 one() { return one2(); }
};
template <class T> struct Jac { T X, Y, Z; };
template <class T> Jac<T> dbl(const Jac<T>& p) {
    using O = Ops<T>;
    if (O::zero(p.Z)) return p;
    T A = O::sqr(p.X), B = O::sqr(p.Y), C = O::sqr(B);
    T D = O::sub(O::sub(O::sqr(O::add(p.X, B)), A), C); D = O::add(D, D);
    T E = O::add(O::add(A, A), A), Fv = O::sqr(E);
    Jac<T> r;
    r.X = O::sub(Fv, O::add(D, D));
    T C8 = O::add(C, C); C8 = O::add(C8, C8); C8 = O::add(C8, C8);
    r.Y = O::sub(O::mul(E, O::sub(D, r.X)), C8);
    r.Z = O::mul(O::add(p.Y, p.Y), p.Z);
    return r;
}
template <class T> Jac<T> addj(const Jac<T>& p, const Jac<T>& q) {
    using O = Ops<T>;
    if (O::zero(p.Z)) return q;
    if (O::zero(q.Z)) return p;
    T Z1Z1 = O::sqr(p.Z), Z2Z2 = O::sqr(q.Z);
    T U1 = O::mul(p.X, Z2Z2), U2 = O::mul(q.X, Z1Z1);
    T S1 = O::mul(O::mul(p.Y, q.Z), Z2Z2), S2 = O::mul(O::mul(q.Y, p.Z), Z1Z1);
    if (O::eq(U1, U2)) {
        if (O::eq(S1, S2)) return dbl(p);
        Jac<T> o; o.X = O::one(); o.Y = O::one(); o.Z = O::sub(O::one(), O::one()); return o;
    }
    T H = O::sub(U2, U1), I = O::sqr(O::add(H, H)), J = O::mul(H, I);
    T r = O::sub(S2, S1); r = O::add(r, r);
    T V = O::mul(U1, I);
    Jac<T> o;
    o.X = O::sub(O::sub(O::sqr(r), J), O::add(V, V));
    T S1J = O::mul(S1, J);
    o.Y = O::sub(O::mul(r, O::sub(V, o.X)), O::add(S1J, S1J));
    o.Z = O::mul(O::sub(O::sub(O::sqr(O::add(p.Z, q.Z)), Z1Z1), Z2Z2), H);
    return o;
}
template <class T> Jac<T> smul(const Jac<T>& p, const uint64_t* k, int nlimbs) {
    Jac<T> acc; acc.X = Ops<T>::one(); acc.Y = Ops<T>::one(); acc.Z = Ops<T>::sub(Ops<T>::one(), Ops<T>::one());
    for (int w = nlimbs - 1; w >= 0; --w)
        for (int b = 63; b >= 0; --b) { acc = dbl(acc); if ((k[w] >> b) & 1) acc = addj(acc, p); }
    return acc;
}
template <class T> bool to_affine(const Jac<T>& p, T& x, T& y) {
    using O = Ops<T>;
    if (O::zero(p.Z)) return false;
    T zi = O::inv(p.Z), zi2 = O::sqr(zi);
    x = O::mul(p.X, zi2);
    y = O::mul(p.Y, O::mul(zi2, zi));
    return true;
}

// ------------------------------------------------------------------ hash to G1
inline F fconst(const uint64_t* c) { F r; memcpy(r.v, c, 48); return r; }
inline F g_of(const F& x) { return add(mul(sqr(x), x), small(4)); }   // x^3 + 4 on E
inline F g_iso(const F& x) {           // x^3 + A' x + B' on E'
    return add(mul(add(sqr(x), fconst(bls::h2c::kIsoA)), x), fconst(bls::h2c::kIsoB));
}
// coefficients c[0..len-1] by Horner, plus x^len when monic
inline F horner(const uint64_t* c, int len, bool monic, const F& x) {
    F acc = monic ? one() : fconst(c + 6 * (len - 1));
    for (int i = monic ? len - 1 : len - 2; i >= 0; --i) acc = add(mul(acc, x), fconst(c + 6 * i));
    return acc;
}

void expand_xmd(const uint8_t* msg, size_t mlen, const uint8_t* dst, size_t dlen, uint8_t* out, size_t len) {
    size_t ell = (len + 31) / 32;
    uint8_t b0[32], bi[32];
    uint8_t dlen8 = (uint8_t)dlen;
    {
        Sha256 h;
        uint8_t z[64] = {0};
        h.update(z, 64);
        h.update(msg, mlen);
        uint8_t l2[3] = {(uint8_t)(len >> 8), (uint8_t)len, 0};
        h.update(l2, 3);
        h.update(dst, dlen);
        h.update(&dlen8, 1);
        h.final(b0);
    }
    for (size_t i = 1; i <= ell; ++i) {
        Sha256 h;
        uint8_t x[32];
        for (int k = 0; k < 32; ++k) x[k] = (uint8_t)(i == 1 ? b0[k] : (b0[k] ^ bi[k]));
        h.update(x, 32);
        uint8_t ib = (uint8_t)i;
        h.update(&ib, 1);
        h.update(dst, dlen);
        h.update(&dlen8, 1);
        h.final(bi);
        size_t off = 32 * (i - 1), k = len - off < 32 ? len - off : 32;
        memcpy(out + off, bi, k);
    }
}
// 64 big-endian bytes -> Montgomery form of the integer mod p
F field_from_64(const uint8_t* b) {
    uint64_t hi[6] = {0}, lo[6];
    for (int i = 0; i < 2; ++i) {            // top 16 bytes = hi (128 bits)
        uint64_t v = 0;
        for (int j = 0; j < 8; ++j) v = (v << 8) | b[8 * i + j];
        hi[1 - i] = v;
    }
    for (int i = 0; i < 6; ++i) {            // low 48 bytes
        uint64_t v = 0;
        for (int j = 0; j < 8; ++j) v = (v << 8) | b[16 + 8 * i + j];
        lo[5 - i] = v;
    }
    while (geq(lo, P)) subp(lo);
    F rr; memcpy(rr.v, RR, 48);
    F r3 = mul(rr, rr);                      // R^3 mod p in raw limbs
    F a = mul(from_raw(hi), r3);             // mont(hi * 2^384)
    F b2 = to_mont(lo);
    return add(a, b2);
}
// simplified SWU to E' (RFC 9380 section 6.6.2), then the 11-isogeny to E
// (section 6.6.3): a Jacobian point, the identity when a denominator vanishes
Jac<F> map_to_g1(const F& u) {
    using namespace bls::h2c;
    const F zu2 = mul(fconst(kZ), sqr(u));
    const F tv1 = add(sqr(zu2), zu2);
    const F x1 = is_zero(tv1) ? fconst(kSswuC2) : mul(fconst(kSswuC1), add(one(), inv(tv1)));
    F x = x1;
    if (!is_square(g_iso(x1))) x = mul(zu2, x1);
    F y = sqrt_cand(g_iso(x));
    if (sgn0(u) != sgn0(y)) y = neg(y);
    const F xn = horner(kIsoXNum, kIsoXNumLen, false, x), xd = horner(kIsoXDen, kIsoXDenLen, true, x);
    const F yn = horner(kIsoYNum, kIsoYNumLen, false, x), yd = horner(kIsoYDen, kIsoYDenLen, true, x);
    const F den = mul(xd, yd);
    if (is_zero(den)) return Jac<F>{one(), one(), zero()};
    const F di = inv(den);
    return Jac<F>{mul(mul(xn, yd), di), mul(mul(mul(y, yn), xd), di), one()};
}
void hash_to_g1(const uint8_t* msg, size_t mlen, const uint8_t* dst, size_t dlen, uint64_t* out12) {
    uint8_t ub[128];
    expand_xmd(msg, mlen, dst, dlen, ub, 128);
    F u0 = field_from_64(ub), u1 = field_from_64(ub + 64);
    Jac<F> q = addj(map_to_g1(u0), map_to_g1(u1));
    const uint64_t heff[1] = {0xd201000000010001ULL};
    Jac<F> r = smul(q, heff, 1);
    F x, y;
    if (!to_affine(r, x, y)) { x = zero(); y = one(); }
    memcpy(out12, x.v, 48);
    memcpy(out12 + 6, y.v, 48);
}

// ------------------------------------------------------------------ G2 line coefficients
struct G2P { F2 x, y, z; };
inline F2 dbl2(const F2& a) { return add2(a, a); }
void store2(uint64_t* d, const F2& a) { memcpy(d, a.c0.v, 48); memcpy(d + 6, a.c1.v, 48); }
void dstep(G2P& r, uint64_t* out) {
    F2 t0 = sqr2(r.x), t1 = sqr2(r.y), t2 = sqr2(t1);
    F2 t3 = dbl2(sub2(sqr2(add2(t1, r.x)), add2(t0, t2)));
    F2 t4 = add2(dbl2(t0), t0), t6 = add2(r.x, t4), t5 = sqr2(t4), zs = sqr2(r.z);
    r.x = sub2(sub2(t5, t3), t3);
    r.z = sub2(sqr2(add2(r.z, r.y)), add2(t1, zs));
    r.y = sub2(mul2(sub2(t3, r.x), t4), dbl2(dbl2(dbl2(t2))));
    F2 l1 = neg2(dbl2(mul2(t4, zs)));
    F2 l2 = sub2(sub2(sqr2(t6), add2(t0, t5)), dbl2(dbl2(t1)));
    F2 l0 = dbl2(mul2(r.z, zs));
    store2(out, l0); store2(out + 12, l1); store2(out + 24, l2);
}
void astep(G2P& r, const F2& qx, const F2& qy, uint64_t* out) {
    F2 zs = sqr2(r.z), ys = sqr2(qy);
    F2 t0 = mul2(zs, qx);
    F2 t1 = mul2(sub2(sqr2(add2(qy, r.z)), add2(ys, zs)), zs);
    F2 t2 = sub2(t0, r.x), t3 = sqr2(t2), t4 = dbl2(dbl2(t3)), t5 = mul2(t4, t2);
    F2 t6 = sub2(sub2(t1, r.y), r.y), t9 = mul2(t6, qx), t7 = mul2(t4, r.x);
    r.x = sub2(sub2(sub2(sqr2(t6), t5), t7), t7);
    r.z = sub2(sqr2(add2(r.z, t2)), add2(zs, t3));
    F2 t10 = add2(qy, r.z);
    F2 t8 = mul2(sub2(t7, r.x), t6);
    r.y = sub2(t8, dbl2(mul2(r.y, t5)));
    t10 = sub2(sub2(sqr2(t10), ys), sqr2(r.z));
    t9 = sub2(dbl2(t9), t10);
    store2(out, dbl2(r.z)); store2(out + 12, dbl2(neg2(t6))); store2(out + 24, t9);
}
void g2_prepare(const uint64_t* q, uint64_t* co) {
    F2 qx = {from_raw(q), from_raw(q + 6)}, qy = {from_raw(q + 12), from_raw(q + 18)};
    G2P r = {qx, qy, one2()};
    const uint64_t X = 0xd201000000010000ULL;
    int ci = 0; bool found = false;
    for (int b = 63; b >= 0; --b) {
        bool bit = ((X >> 1) >> b) & 1;
        if (!found) { found = bit; continue; }
        dstep(r, co + 36 * ci++);
        if (bit) astep(r, qx, qy, co + 36 * ci++);
    }
    dstep(r, co + 36 * ci);
}

const uint64_t G2X0[6] = {0xf5f28fa202940a10ULL, 0xb3f5fb2687b4961aULL, 0xa1a893b53e2ae580ULL,
                          0x9894999d1a3caee9ULL, 0x6f67b7631863366bULL, 0x058191924350bcd7ULL};
const uint64_t G2X1[6] = {0xa5a9c0759e23f606ULL, 0xaaa0c59dbccd60c3ULL, 0x3bb17e18e2867806ULL,
                          0x1b1ab6cc8541b367ULL, 0xc2b6ed0ef2158547ULL, 0x11922a097360edf3ULL};
const uint64_t G2Y0[6] = {0x4c730af860494c4aULL, 0x597cfa1f5e369c5aULL, 0xe7e6856caa0a635aULL,
                          0xbbefb5e96e0d495fULL, 0x07d3a975f0ef25a2ULL, 0x0083fd8e7e80dae5ULL};
const uint64_t G2Y1[6] = {0xadc0fc92df64b05dULL, 0x18aa270a2b1461dcULL, 0x86adac6a3be4eba0ULL,
                          0x79495c4ec93da33aULL, 0xe7175850a43ccaedULL, 0x0b2bc2a163de1bf2ULL};

void be48(const uint64_t* canon6, uint8_t* out) {
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 8; ++j) out[8 * i + j] = (uint8_t)(canon6[5 - i] >> (56 - 8 * j));
}

template <class Fn>
void pfor(int n, int nthreads, Fn fn) {
    if (nthreads <= 1 || n < 2) { for (int i = 0; i < n; ++i) fn(i); return; }
    std::atomic<int> next(0);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t)
        th.emplace_back([&] { for (;;) { int i = next.fetch_add(1); if (i >= n) break; fn(i); } });
    for (auto& t : th) t.join();
}

}  // namespace wl

using namespace wl;

extern "C" {

int wl_num_threads(void) { return (int)std::thread::hardware_concurrency(); }

void wl_sha256(const uint8_t* data, size_t len, uint8_t* out32) {
    Sha256 h; h.update(data, len); h.final(out32);
}

void wl_expand_message_xmd(const uint8_t* msg, size_t mlen, const uint8_t* dst, size_t dlen, uint8_t* out, size_t len) {
    expand_xmd(msg, mlen, dst, dlen, out, len);
}

// msgs: n x msg_len bytes -> n x 12 affine Montgomery
int wl_hash_to_g1(const uint8_t* msgs, int msg_len, int n, const uint8_t* dst, int dst_len, uint64_t* out, int nthreads) {
    pfor(n, nthreads, [&](int i) { hash_to_g1(msgs + (size_t)msg_len * i, msg_len, dst, dst_len, out + 12 * (size_t)i); });
    return 0;
}

// out[i] = k[i] * P[i] (affine Montgomery; identity -> x = 0, y = R)
int wl_g1_mul(const uint64_t* pts, const uint64_t* scalars, int n, uint64_t* out, int nthreads) {
    pfor(n, nthreads, [&](int i) {
        Jac<F> p = {from_raw(pts + 12 * (size_t)i), from_raw(pts + 12 * (size_t)i + 6), one()};
        Jac<F> r = smul(p, scalars + 4 * (size_t)i, 4);
        F x, y;
        if (!to_affine(r, x, y)) { x = zero(); y = one(); }
        memcpy(out + 12 * (size_t)i, x.v, 48);
        memcpy(out + 12 * (size_t)i + 6, y.v, 48);
    });
    return 0;
}

int wl_g1_neg(const uint64_t* pts, int n, uint64_t* out) {
    for (int i = 0; i < n; ++i) {
        F y = neg(from_raw(pts + 12 * (size_t)i + 6));
        memcpy(out + 12 * (size_t)i, pts + 12 * (size_t)i, 48);
        memcpy(out + 12 * (size_t)i + 6, y.v, 48);
    }
    return 0;
}

// pk = k * G2, affine (x.c0, x.c1, y.c0, y.c1)
int wl_g2_mul_gen(const uint64_t* scalars, int n, uint64_t* out, int nthreads) {
    pfor(n, nthreads, [&](int i) {
        Jac<F2> g = {{from_raw(G2X0), from_raw(G2X1)}, {from_raw(G2Y0), from_raw(G2Y1)}, one2()};
        Jac<F2> r = smul(g, scalars + 4 * (size_t)i, 4);
        F2 x, y;
        uint64_t* o = out + 24 * (size_t)i;
        if (!to_affine(r, x, y)) { memset(o, 0, 192); return; }
        memcpy(o, x.c0.v, 48); memcpy(o + 6, x.c1.v, 48); memcpy(o + 12, y.c0.v, 48); memcpy(o + 18, y.c1.v, 48);
    });
    return 0;
}

int wl_g2_prepare(const uint64_t* q, int n, uint64_t* coeffs, int nthreads) {
    pfor(n, nthreads, [&](int i) { g2_prepare(q + 24 * (size_t)i, coeffs + 2448 * (size_t)i); });
    return 0;
}

// affine Montgomery (identity: x = 0, y in {0, R}) -> 48-byte ZCash encoding
int wl_g1_compress(const uint64_t* pts, int n, uint8_t* out) {
    for (int i = 0; i < n; ++i) {
        F x = from_raw(pts + 12 * (size_t)i), y = from_raw(pts + 12 * (size_t)i + 6);
        uint8_t* o = out + 48 * (size_t)i;
        if (is_zero(x)) { memset(o, 0, 48); o[0] = 0xc0; continue; }
        uint64_t c[6]; canon(x, c);
        be48(c, o);
        o[0] |= 0x80;
        if (lex_largest(y)) o[0] |= 0x20;
    }
    return 0;
}

int wl_g2_compress(const uint64_t* q, int n, uint8_t* out) {
    for (int i = 0; i < n; ++i) {
        const uint64_t* p = q + 24 * (size_t)i;
        uint8_t* o = out + 96 * (size_t)i;
        F2 x = {from_raw(p), from_raw(p + 6)}, y = {from_raw(p + 12), from_raw(p + 18)};
        uint64_t c1[6], c0[6];
        canon(x.c1, c1); canon(x.c0, c0);
        be48(c1, o); be48(c0, o + 48);
        o[0] |= 0x80;
        if (lex_largest2(y)) o[0] |= 0x20;
    }
    return 0;
}

// x values (canonical, < p) -> 48-byte encodings with the compression flag:
// mode 0 picks x with x^3 + 4 a non-square (not on the curve); mode 1 picks a
// curve point and encodes it (outside the subgroup with overwhelming
// probability; the caller can confirm with a decoder).  seed drives SplitMix64.
int wl_special_points(uint64_t seed, int n, int mode, uint8_t* out) {
    uint64_t s = seed;
    auto next = [&]() {
        s += 0x9E3779B97F4A7C15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    };
    for (int i = 0; i < n; ++i) {
        for (;;) {
            uint64_t v[6];
            for (int k = 0; k < 6; ++k) v[k] = next();
            v[5] &= 0x0fffffffffffffffULL;
            if (geq(v, P)) continue;
            F x = to_mont(v);
            F g = g_of(x);
            bool sq = is_square(g);
            if ((mode == 0 && sq) || (mode == 1 && !sq)) continue;
            uint8_t* o = out + 48 * (size_t)i;
            be48(v, o);
            o[0] |= 0x80;
            if (mode == 1) {
                F y = sqrt_cand(g);
                if (next() & 1) y = neg(y);
                if (lex_largest(y)) o[0] |= 0x20;
            }
            break;
        }
    }
    return 0;
}

}  // extern "C"
