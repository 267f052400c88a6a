// G2 point decoding on the device: 96-byte compressed public keys (ZCash
// BLS12-381 encoding: x = x.c1 || x.c0 big-endian, the three flag bits in the
// top of byte 0) to affine Montgomery (x, y) on the twist y^2 = x^3 + 4(1 + u),
// with every check ic_bls12_381's G2Affine::from_compressed makes: the
// compression flag set; the infinity flag only with an all-zero payload and
// no sort flag; both halves of x below p; x^3 + 4(1 + u) a square in Fp2; the
// point in the order-r subgroup (psi(P) = [x] P).  The reference has no device G2
// decoder: its callers decode keys and build their line tables on the CPU per
// item (ic-integration/patches/ic-gpu-consensus.patch:458-461).
//
// Square roots in Fp2 (p = 3 mod 4) follow Algorithm 9 of Adj and
// Rodriguez-Henriquez, "Square root computation over even extension fields"
// (IEEE Trans. Computers, 2014): a1 = a^((p-3)/4), alpha = a1^2 a,
// x0 = a1 a; x = u x0 when alpha = -1, else (1 + alpha)^((p-1)/2) x0.  The
// sign is then fixed by the sort flag ("lexicographically largest": y.c1 >
// (p-1)/2, or y.c1 = 0 and y.c0 > (p-1)/2).
#pragma once
#include "g1.cuh"
#include "tower.cuh"

namespace bls {

// a^e for an exponent given as 6 little-endian u64 words (right to left)
static __device__ __noinline__ fp2 fp2_pow_u64(const fp2& a, const uint64_t* e, int nbits) {
    fp2 r = fp2_one(), base = a;
    for (int i = 0; i < nbits; ++i) {
        if ((e[i >> 6] >> (i & 63)) & 1) r = fp2_mul(r, base);
        base = fp2_sqr(base);
    }
    return r;
}

__device__ __forceinline__ bool fp2_eq(const fp2& a, const fp2& b) { return fp_eq(a.c0, b.c0) && fp_eq(a.c1, b.c1); }

// a square root of a (any of the two) when a is a square; *ok = false otherwise
static __device__ __noinline__ fp2 fp2_sqrt(const fp2& a, bool* ok) {
    const uint64_t e1[6] = {0xee7fbfffffffeaaaULL, 0x07aaffffac54ffffULL, 0xd9cc34a83dac3d89ULL,
                            0xd91dd2e13ce144afULL, 0x92c6e9ed90d2eb35ULL, 0x0680447a8e5ff9a6ULL};  // (p-3)/4
    const uint64_t e2[6] = {0xdcff7fffffffd555ULL, 0x0f55ffff58a9ffffULL, 0xb39869507b587b12ULL,
                            0xb23ba5c279c2895fULL, 0x258dd3db21a5d66bULL, 0x0d0088f51cbff34dULL};  // (p-1)/2
    fp2 a1 = fp2_pow_u64(a, e1, 379);
    fp2 x0 = fp2_mul(a1, a);
    fp2 alpha = fp2_mul(a1, x0);
    fp2 x;
    const fp2 minus_one = fp2_neg(fp2_one());
    if (fp2_eq(alpha, minus_one)) {
        x = {fp_neg(x0.c1), x0.c0};       // u x0
    } else {
        fp2 b = fp2_pow_u64(fp2_add(fp2_one(), alpha), e2, 380);
        x = fp2_mul(b, x0);
    }
    *ok = fp2_eq(fp2_sqr(x), a);
    return x;
}

__device__ __forceinline__ bool fp2_lex_largest(const fp2& a) {
    return fp_lex_largest(a.c1) || (fp_is_zero(a.c1) && fp_lex_largest(a.c0));
}

// Jacobian coordinates on the twist (a = 0)
struct g2j { fp2 X, Y, Z; };

// dbl-2009-l
static __device__ __noinline__ g2j g2j_dbl(const g2j& p) {
    fp2 A = fp2_sqr(p.X), B = fp2_sqr(p.Y), C = fp2_sqr(B);
    fp2 D = fp2_sub(fp2_sub(fp2_sqr(fp2_add(p.X, B)), A), C);
    D = fp2_add(D, D);
    fp2 E = fp2_add(fp2_add(A, A), A);
    fp2 F = fp2_sqr(E);
    g2j r;
    r.X = fp2_sub(F, fp2_add(D, D));
    fp2 C8 = fp2_add(C, C);
    C8 = fp2_add(C8, C8);
    C8 = fp2_add(C8, C8);
    r.Y = fp2_sub(fp2_mul(E, fp2_sub(D, r.X)), C8);
    r.Z = fp2_mul(fp2_add(p.Y, p.Y), p.Z);
    return r;
}

// p + (qx, qy), q affine (madd-2007-bl), with the equal and opposite cases
static __device__ __noinline__ g2j g2j_add_affine(const g2j& p, const fp2& qx, const fp2& qy) {
    if (fp2_is_zero(p.Z)) return {qx, qy, fp2_one()};
    fp2 Z1Z1 = fp2_sqr(p.Z);
    fp2 U2 = fp2_mul(qx, Z1Z1);
    fp2 S2 = fp2_mul(fp2_mul(qy, p.Z), Z1Z1);
    fp2 H = fp2_sub(U2, p.X);
    fp2 rr = fp2_sub(S2, p.Y);
    if (fp2_is_zero(H)) {
        if (fp2_is_zero(rr)) return g2j_dbl(p);
        return {fp2_one(), fp2_one(), fp2_zero()};
    }
    rr = fp2_add(rr, rr);
    fp2 HH = fp2_sqr(H);
    fp2 I = fp2_add(HH, HH);
    I = fp2_add(I, I);
    fp2 J = fp2_mul(H, I);
    fp2 V = fp2_mul(p.X, I);
    g2j r;
    r.X = fp2_sub(fp2_sub(fp2_sqr(rr), J), fp2_add(V, V));
    fp2 YJ = fp2_mul(p.Y, J);
    r.Y = fp2_sub(fp2_mul(rr, fp2_sub(V, r.X)), fp2_add(YJ, YJ));
    r.Z = fp2_sub(fp2_sub(fp2_sqr(fp2_add(p.Z, H)), Z1Z1), HH);
    return r;
}

// psi(P) == [x] P for an affine point P on the twist (not the identity), x the
// BLS parameter -0xd201000000010000.  psi(x, y) = (conj(x) cx, conj(y) cy)
// with cx = (1 + u)^(-(p-1)/3), cy = (1 + u)^(-(p-1)/2) is the untwist-
// Frobenius-twist endomorphism; the test holds exactly for the order-r subgroup
// (Scott, eprint 2021/1130 section 4; proof El Housni, Guillevic and
// Piellard, eprint 2022/352).  63 doublings and 5 additions, against 254 and
// 133 for [r] P == O.
static __device__ __noinline__ bool g2_in_subgroup(const fp2& x, const fp2& y) {
    const uint64_t xabs = 0xd201000000010000ULL;
    g2j acc = {x, y, fp2_one()};
    for (int i = 62; i >= 0; --i) {
        acc = g2j_dbl(acc);
        if ((xabs >> i) & 1) acc = g2j_add_affine(acc, x, y);
    }
    if (fp2_is_zero(acc.Z)) return false;
    // Montgomery forms: cx = (0, cx1), cy = (cy0, cy1)
    const uint64_t cx1[6] = {0x890dc9e4867545c3ULL, 0x2af322533285a5d5ULL, 0x50880866309b7e2cULL,
                             0xa20d1b8c7e881024ULL, 0x14e4f04fe2db9068ULL, 0x14e56d3f1564853aULL};
    const uint64_t cy0[6] = {0x3e2f585da55c9ad1ULL, 0x4294213d86c18183ULL, 0x382844c88b623732ULL,
                             0x92ad2afd19103e18ULL, 0x1d794e4fac7cf0b9ULL, 0x0bd592fc7d825ec8ULL};
    const uint64_t cy1[6] = {0x7bcfa7a25aa30fdaULL, 0xdc17dec12a927e7cULL, 0x2f088dd86b4ebef1ULL,
                             0xd1ca2087da74d4a7ULL, 0x2da2596696cebc1dULL, 0x0e2b7eedbbfd87d2ULL};
    fp2 px = fp2_mul(fp2_conj(x), fp2{fp_zero(), fp_load_u64(cx1)});
    fp2 py = fp2_mul(fp2_conj(y), fp2{fp_load_u64(cy0), fp_load_u64(cy1)});
    // [x] P = -[|x|] P = (X, -Y, Z): X == px Z^2 and -Y == py Z^3
    fp2 Z2 = fp2_sqr(acc.Z), Z3 = fp2_mul(Z2, acc.Z);
    bool ex = fp2_eq(acc.X, fp2_mul(px, Z2));
    bool ey = fp2_is_zero(fp2_add(acc.Y, fp2_mul(py, Z3)));
    return ex && ey;
}

// canonical 48-byte big-endian integer -> 12 little-endian limbs
__device__ __forceinline__ fp fp_from_be48(const uint8_t* in, bool mask_flags) {
    fp raw;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const uint8_t* b = in + 44 - 4 * i;
        uint32_t b0 = b[0];
        if (i == 11 && mask_flags) b0 &= 0x1f;
        raw.w[i] = (b0 << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
    }
    return raw;
}

// Decode one 96-byte key.  On success writes Montgomery (x, y); the identity
// is reported by *identity (and x = y = 0).  Returns a status code.
__device__ __forceinline__ int32_t g2_decode(const uint8_t* in, fp2& x, fp2& y, bool& identity) {
    identity = false;
    x = fp2_zero();
    y = fp2_zero();
    const uint32_t top = in[0];
    const bool comp = (top >> 7) & 1, inf = (top >> 6) & 1, sort = (top >> 5) & 1;
    fp x1 = fp_from_be48(in, true), x0 = fp_from_be48(in + 48, false);
    if (!comp) return ST_BAD_FLAGS;
    if (inf) {
        if (sort || !fp_is_zero(x0) || !fp_is_zero(x1)) return ST_BAD_FLAGS;
        identity = true;
        return ST_OK;
    }
    if (fp_raw_geq_p(x0) || fp_raw_geq_p(x1)) return ST_X_NOT_CANONICAL;
    fp2 xm = {fp_to_mont(x0), fp_to_mont(x1)};
    fp four = fp_four();
    fp2 y2 = fp2_add(fp2_mul(fp2_sqr(xm), xm), fp2{four, four});
    bool ok = false;
    fp2 yy = fp2_sqrt(y2, &ok);
    if (!ok) return ST_NOT_ON_CURVE;
    if (fp2_lex_largest(yy) != sort) yy = fp2_neg(yy);
    if (!g2_in_subgroup(xm, yy)) return ST_NOT_IN_SUBGROUP;
    x = xm;
    y = yy;
    return ST_OK;
}

}  // namespace bls
