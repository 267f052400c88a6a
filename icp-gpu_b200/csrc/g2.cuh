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
// Square roots in Fp2 = Fp[u] / (u^2 + 1) (p = 3 mod 4) by the norm method:
// for a = a0 + a1 u with a1 != 0, x0^2 is the root d = (a0 + g) / 2 or
// (a0 - g) / 2 of 4 d^2 - 4 a0 d - a1^2 = 0 that is a square in Fp, where
// g^2 = a0^2 + a1^2 (the norm, a square in Fp whenever a is a square in
// Fp2), and x1 = a1 / (2 x0); for a1 = 0 the root is sqrt(a0) or u sqrt(-a0).
// Two exponentiations in Fp, (p + 1) / 4 for g and (p - 3) / 4 for the rest
// (which also gives d's Legendre symbol and 1 / x0 without an inverse), where
// Algorithm 9 of Adj and Rodriguez-Henriquez (two exponentiations in Fp2)
// costs about 2.5 times the multiplies.  The sign is then fixed by the sort flag
// ("lexicographically largest": y.c1 > (p-1)/2, or y.c1 = 0 and
// y.c0 > (p-1)/2), so the decoded point does not depend on which root the
// method finds.
#pragma once
#include "g1.cuh"
#include "tower.cuh"

namespace bls {

__device__ __forceinline__ bool fp2_eq(const fp2& a, const fp2& b) { return fp_eq(a.c0, b.c0) && fp_eq(a.c1, b.c1); }

// a / 2 (a canonical; also in Montgomery form): a + p when a is odd, then one
// right shift; a + p < 2p < 2^382, so nothing carries out of the twelve limbs
__device__ __forceinline__ fp fp_half(const fp& a) {
    const uint32_t m = 0u - (a.w[0] & 1u);
    uint32_t s[12];
    asm("add.cc.u32 %0, %12, %24;\n\t"
        "addc.cc.u32 %1, %13, %25;\n\t"
        "addc.cc.u32 %2, %14, %26;\n\t"
        "addc.cc.u32 %3, %15, %27;\n\t"
        "addc.cc.u32 %4, %16, %28;\n\t"
        "addc.cc.u32 %5, %17, %29;\n\t"
        "addc.cc.u32 %6, %18, %30;\n\t"
        "addc.cc.u32 %7, %19, %31;\n\t"
        "addc.cc.u32 %8, %20, %32;\n\t"
        "addc.cc.u32 %9, %21, %33;\n\t"
        "addc.cc.u32 %10, %22, %34;\n\t"
        "addc.u32 %11, %23, %35;"
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7]),
          "=r"(s[8]), "=r"(s[9]), "=r"(s[10]), "=r"(s[11])
        : BLS_A12(a.w), "r"(BLS_P0 & m), "r"(BLS_P1 & m), "r"(BLS_P2 & m), "r"(BLS_P3 & m), "r"(BLS_P4 & m),
          "r"(BLS_P5 & m), "r"(BLS_P6 & m), "r"(BLS_P7 & m), "r"(BLS_P8 & m), "r"(BLS_P9 & m), "r"(BLS_P10 & m),
          "r"(BLS_P11 & m));
    fp r;
#pragma unroll
    for (int i = 0; i < 11; ++i) r.w[i] = __funnelshift_r(s[i], s[i + 1], 1);
    r.w[11] = s[11] >> 1;
    return r;
}

// a square root of a (any of the two) when a is a square; *ok = false otherwise
static __device__ __noinline__ fp2 fp2_sqrt(const fp2& a, bool* ok) {
    fp2 x;
    if (fp_is_zero(a.c1)) {
        // a in Fp: sqrt(a0) when a0 is a square, else u sqrt(-a0) (-1 is not a square)
        const fp t = fp_sqrt_candidate(a.c0);
        if (fp_eq(fp_sqr(t), a.c0)) x = {t, fp_zero()};
        else x = {fp_zero(), fp_sqrt_candidate(fp_neg(a.c0))};
    } else {
        const fp n = fp_add(fp_sqr(a.c0), fp_sqr(a.c1));
        const fp g = fp_sqrt_candidate(n);
        if (!fp_eq(fp_sqr(g), n)) {   // the norm is not a square: neither is a
            *ok = false;
            return fp2_zero();
        }
        // d = (a0 + g) / 2 is nonzero (d (a0 - g) / 2 = -a1^2 / 4).  With
        // t = d^((p-3)/4), d t^2 = d^((p-1)/2) is d's Legendre symbol s:
        // s = 1: x = (d t, a1 t / 2), since (d t)^2 = d;
        // s = -1: the other root (a0 - g) / 2 = -a1^2 / (4 d) is the square,
        //         x = (a1 t / 2, -d t) (t^2 = -1 / d gives x0^2 - x1^2 = a0
        //         and 2 x0 x1 = a1).
        // No inverse and no branch on s: every lane of a warp runs the same code.
        const uint64_t e[6] = {0xee7fbfffffffeaaaULL, 0x07aaffffac54ffffULL, 0xd9cc34a83dac3d89ULL,
                               0xd91dd2e13ce144afULL, 0x92c6e9ed90d2eb35ULL, 0x0680447a8e5ff9a6ULL};  // (p-3)/4
        const fp d = fp_half(fp_add(a.c0, g));
        const fp t = fp_pow_ool(d, e, 379);
        const fp dt = fp_mul(d, t);
        const fp h = fp_half(fp_mul(a.c1, t));
        const bool s_one = fp_eq(fp_mul(dt, t), fp_one());
        const fp ndt = fp_neg(dt);
        x = {s_one ? dt : h, s_one ? h : ndt};
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
