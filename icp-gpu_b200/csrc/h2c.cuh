// Hash to G1 on the device: RFC 9380 hash_to_curve for BLS12-381 G1, the
// suite BLS12381G1_XMD:SHA-256_SSWU_RO_ that ic_bls12_381's hash_to_curve
// implements and the reference's callers run on the CPU per item
// (ic-integration/patches/ic-gpu-consensus.patch:454-457,
// ic-bench/src/main.rs:65-76): expand_message_xmd over SHA-256, two field
// elements, the simplified SWU map (section 6.6.2) on the 11-isogenous curve
// E' and the 11-isogeny to y^2 = x^3 + 4 (section 6.6.3), point addition,
// cofactor clearing by h_eff = 1 - x.  Constants from gen_h2c.py (h2c.inc),
// which derives the isogeny; the kernel (hash.cu) runs the two maps of a
// message on two threads.
#pragma once
#include "fp_inv.cuh"
#include "g1.cuh"
#include "h2c.inc"

namespace bls {
namespace h2c {

__device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

// SHA-256 compression of one 64-byte block given as 16 big-endian words
static __device__ __noinline__ void sha256_block(uint32_t* h, const uint32_t* blk) {
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = blk[i];
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
#pragma unroll
    for (int t = 0; t < 64; ++t) {
        uint32_t wt;
        if (t < 16) {
            wt = w[t];
        } else {
            const uint32_t w15 = w[(t - 15) & 15], w2 = w[(t - 2) & 15];
            const uint32_t s0 = rotr(w15, 7) ^ rotr(w15, 18) ^ (w15 >> 3);
            const uint32_t s1 = rotr(w2, 17) ^ rotr(w2, 19) ^ (w2 >> 10);
            wt = w[t & 15] = w[t & 15] + s0 + w[(t - 7) & 15] + s1;
        }
        const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
        const uint32_t ch = (e & f) ^ (~e & g);
        const uint32_t t1 = hh + S1 + ch + kSha256K[t] + wt;
        const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
        const uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + S0 + mj;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}

// streaming SHA-256, fed byte by byte
struct Sha256 {
    uint32_t h[8];
    uint32_t blk[16];
    uint32_t fill;    // bytes in blk
    uint64_t total;   // bytes hashed

    __device__ void init() {
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = kSha256H0[i];
#pragma unroll
        for (int i = 0; i < 16; ++i) blk[i] = 0;
        fill = 0;
        total = 0;
    }
    __device__ __noinline__ void put(uint32_t byte) {
        blk[fill >> 2] |= (byte & 0xffu) << (24 - 8 * (fill & 3));
        ++total;
        if (++fill == 64) {
            sha256_block(h, blk);
#pragma unroll
            for (int i = 0; i < 16; ++i) blk[i] = 0;
            fill = 0;
        }
    }
    __device__ void put(const uint8_t* p, uint32_t n) {
        for (uint32_t i = 0; i < n; ++i) put(p[i]);
    }
    // big-endian digest words
    __device__ void final(uint32_t* out) {
        const uint64_t bits = total * 8;
        put(0x80u);
        while (fill != 56) put(0u);
        for (int i = 7; i >= 0; --i) put((uint32_t)(bits >> (8 * i)));
#pragma unroll
        for (int i = 0; i < 8; ++i) out[i] = h[i];
    }
};

// expand_message_xmd(msg, dst, 128) (RFC 9380 section 5.3.1): 32 big-endian words
__device__ __forceinline__ void expand_xmd_128(const uint8_t* msg, uint32_t len, const uint8_t* dst,
                                               uint32_t dst_len, uint32_t* out) {
    Sha256 s;
    s.init();
    for (int i = 0; i < 64; ++i) s.put(0u);      // Z_pad
    s.put(msg, len);
    s.put(0u);                                   // I2OSP(128, 2)
    s.put(128u);
    s.put(0u);                                   // I2OSP(0, 1)
    s.put(dst, dst_len);
    s.put(dst_len);
    uint32_t b0[8], bi[8];
    s.final(b0);
    for (uint32_t i = 1; i <= 4; ++i) {
        s.init();
        for (int k = 0; k < 8; ++k) {
            const uint32_t v = i == 1 ? b0[k] : (b0[k] ^ bi[k]);
            s.put(v >> 24); s.put(v >> 16); s.put(v >> 8); s.put(v);
        }
        s.put(i);
        s.put(dst, dst_len);
        s.put(dst_len);
        s.final(bi);
#pragma unroll
        for (int k = 0; k < 8; ++k) out[8 * (i - 1) + k] = bi[k];
    }
}

// 64 big-endian bytes (16 words) mod p, Montgomery form
__device__ __forceinline__ fp field_from_be64(const uint32_t* w) {
    fp hi, lo;
#pragma unroll
    for (int i = 0; i < 12; ++i) hi.w[i] = lo.w[i] = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        hi.w[i] = w[7 - i];
        lo.w[i] = w[15 - i];
    }
    return fp_add(fp_mul(lo, fp_rr()), fp_mul(hi, fp_load_u64(kK256)));
}

__device__ __forceinline__ uint32_t sgn0(const fp& a) { return fp_from_mont(a).w[0] & 1u; }

// The hash kernel runs one warp per scheduler, so nothing hides a miss in the
// instruction cache: its long loops (the sqrt_ratio power, the isogeny's
// Horner evaluations, the 63 doublings of the cofactor clearing) use the
// out-of-line multiply of fp.cuh rather than inlining its body at every use.

// g'(x) = x^3 + A' x + B' on E'
__device__ __forceinline__ fp g_iso(const fp& x) {
    return fp_add(fp_mul(fp_add(fp_sqr(x), fp_load_u64(kIsoA)), x), fp_load_u64(kIsoB));
}

// sqrt_ratio(u, v) for p = 3 mod 4 (RFC 9380 appendix F.2.1.2): true and
// y = sqrt(u / v) when u / v is a square, else false and y = sqrt(Z u / v);
// one exponentiation
__device__ __forceinline__ bool sqrt_ratio(const fp& u, const fp& v, fp& y) {
    const fp tv2 = fp_mul(u, v);
    const fp tv1 = fp_mul(fp_sqr(v), tv2);                          // u v^3
    const fp y1 = fp_mul(fp_pow_ool(tv1, kSqrtRatioE, kSqrtRatioBits), tv2);
    const bool qr = fp_eq(fp_mul(fp_sqr(y1), v), u);
    y = qr ? y1 : fp_mul(y1, fp_load_u64(kSqrtMinusZ));
    return qr;
}

// the simplified SWU map to E' by the RFC's straight-line steps (appendix
// F.2, steps 1-24), which give the map of section 6.6.2 with one
// exponentiation: x' = xn / xd is returned as its two parts (the isogeny
// takes a fraction), y' affine, sgn0(y') = sgn0(u)
static __device__ __noinline__ void map_sswu(const fp& u, fp& xn, fp& xd, fp& y) {
    const fp A = fp_load_u64(kIsoA), B = fp_load_u64(kIsoB), Z = fp_load_u64(kZ);
    const fp tv1 = fp_mul(Z, fp_sqr(u));                            // Z u^2
    const fp tv2 = fp_add(fp_sqr(tv1), tv1);                        // Z^2 u^4 + Z u^2
    const fp tv3 = fp_mul(B, fp_add(tv2, fp_one()));
    const fp tv4 = fp_mul(A, fp_is_zero(tv2) ? Z : fp_neg(tv2));    // x1 = tv3 / tv4
    fp tv6 = fp_sqr(tv4);
    const fp gn = fp_add(fp_mul(fp_add(fp_sqr(tv3), fp_mul(A, tv6)), tv3), fp_mul(B, fp_mul(tv6, tv4)));
    tv6 = fp_mul(tv6, tv4);                                         // g'(x1) = gn / tv4^3
    fp y1;
    const bool sq = sqrt_ratio(gn, tv6, y1);
    xn = sq ? tv3 : fp_mul(tv1, tv3);                               // x1 or x2 = Z u^2 x1
    xd = tv4;
    y = sq ? y1 : fp_mul(fp_mul(tv1, u), y1);
    if (sgn0(u) != sgn0(y)) y = fp_neg(y);
}

// C(N, D) = D^deg c(N / D) for `len` coefficients of 6 u64 (Montgomery),
// plus the leading 1 when `monic` (deg = len - 1 + monic): Horner in N with
// the running power D^(deg - i) beside it
__device__ __forceinline__ fp horner_h(const uint64_t* c, int len, bool monic, const fp& N, const fp& D) {
    const int deg = len - 1 + (monic ? 1 : 0);
    fp acc = monic ? fp_one() : fp_load_u64(c + 6 * (len - 1)), dk = D;
    for (int i = deg - 1; i >= 0; --i) {
        acc = fp_add(fp_mul_ool(acc, N), fp_mul_ool(fp_load_u64(c + 6 * i), dk));
        dk = fp_mul_ool(dk, D);
    }
    return acc;
}

// the 11-isogeny E' -> E (RFC 9380 section 6.6.3 with the map of appendix
// E.2) at x' = N / D, straight to Jacobian coordinates without an inversion:
// x = x_num / x_den = XN / (XD D), y = y' YN / YD (the powers of D cancel),
// Z = x_den y_den, X = x_num x_den y_den^2, Y = y_num x_den^3 y_den^2.  A
// vanishing denominator gives Z = 0, the identity.
static __device__ __noinline__ g1j iso_map(const fp& N, const fp& D, const fp& ys) {
    const fp xnum = horner_h(kIsoXNum, kIsoXNumLen, false, N, D);                  // D^11 x_num(x')
    const fp xden = fp_mul(horner_h(kIsoXDen, kIsoXDenLen, true, N, D), D);        // D^11 x_den(x')
    const fp ynum = fp_mul(ys, horner_h(kIsoYNum, kIsoYNumLen, false, N, D));      // D^15 y' y_num(x')
    const fp yden = horner_h(kIsoYDen, kIsoYDenLen, true, N, D);                   // D^15 y_den(x')
    const fp yd2 = fp_sqr(yden);
    return {fp_mul(fp_mul(xnum, xden), yd2), fp_mul(fp_mul(ynum, fp_mul(fp_sqr(xden), xden)), yd2),
            fp_mul(xden, yden)};
}

// [h_eff] (P0 + P1) in Jacobian coordinates: Q = P0 + P1 stays Jacobian
// through the cofactor clearing.
static __device__ __noinline__ g1j clear_sum(const g1j& p0, const g1j& p1) {
    const g1j q = g1j_add(p0, p1);
    g1j r = q;
    for (int i = 62; i >= 0; --i) {
        r = g1j_dbl(r);
        if ((kHEff >> i) & 1) r = g1j_add(r, q);
    }
    return r;
}

// -H(msg) as affine Montgomery (x, y) from r = [h_eff](P0 + P1) and zi =
// 1 / r.Z (the caller's inversion); the identity (r.Z = 0) as x = 0,
// y = R mod p.
__device__ __forceinline__ void neg_affine(const g1j& r, const fp& zi, fp& ox, fp& oy) {
    if (fp_is_zero(r.Z)) {
        ox = fp_zero();
        oy = fp_one();
        return;
    }
    const fp zi2 = fp_sqr(zi);
    ox = fp_mul(r.X, zi2);
    oy = fp_neg(fp_mul(r.Y, fp_mul(zi2, zi)));
}

}  // namespace h2c
}  // namespace bls
