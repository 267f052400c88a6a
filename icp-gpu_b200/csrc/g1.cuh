// G1 point decoding on the device: 48-byte compressed points (ZCash BLS12-381
// format, big-endian x with three flag bits in the top of byte 0) to affine
// Montgomery (x, y), with every check ic_bls12_381's G1Affine::from_compressed
// makes.  The value path follows the reference decoder (cuda/decompress.cu:
// 44-187: y = (x^3 + 4)^((p+1)/4), sign chosen by "lexicographically largest");
// the reference performs none of the checks, which are added here:
//   compression flag set; infinity flag only with an all-zero payload and no
//   sort flag; x < p; x^3 + 4 a square; the point in the order-r subgroup.
// The subgroup test is phi(P) == -[x^2] P with phi(x, y) = (beta x, y),
// beta the cube root of unity whose eigenvalue on G1 is -x^2 (Scott, eprint
// 2021/1130 section 6; correctness proof eprint 2022/352).
#pragma once
#include "fp.cuh"

namespace bls {

enum : int32_t {
    ST_OK = 0,
    ST_BAD_FLAGS = 1,
    ST_X_NOT_CANONICAL = 2,
    ST_NOT_ON_CURVE = 3,
    ST_NOT_IN_SUBGROUP = 4,
    ST_BAD_KEY_INDEX = 5,     // not a decode status: a key id outside the tables
};

// a key id the verify kernels may read (VerifyArgs::check_keys, n_keys)
__device__ __forceinline__ bool key_index_ok(int64_t id, int check, int n_keys) {
    return !check || (id >= 0 && id < (int64_t)n_keys);
}

__device__ __forceinline__ fp fp_four() {
    fp one = fp_one();
    fp two = fp_add(one, one);
    return fp_add(two, two);
}

// a^((p+1)/4); a square root whenever one exists (p = 3 mod 4)
static __device__ __noinline__ fp fp_sqrt_candidate(const fp& a) {
    const uint64_t e[6] = {0xee7fbfffffffeaabULL, 0x07aaffffac54ffffULL, 0xd9cc34a83dac3d89ULL,
                           0xd91dd2e13ce144afULL, 0x92c6e9ed90d2eb35ULL, 0x0680447a8e5ff9a6ULL};
    return fp_pow_ool(a, e, 379);
}

// canonical value > (p - 1) / 2
__device__ __forceinline__ bool fp_lex_largest(const fp& a) {
    fp v = fp_from_mont(a);
    // (p-1)/2 = 0x0d0088f51cbff34d 258dd3db21a5d66b b23ba5c279c2895f b39869507b587b12 0f55ffff58a9ffff dcff7fffffffd555
    const uint32_t h[12] = {0xffffd555u, 0xdcff7fffu, 0x58a9ffffu, 0x0f55ffffu, 0x7b587b12u, 0xb3986950u,
                            0x79c2895fu, 0xb23ba5c2u, 0x21a5d66bu, 0x258dd3dbu, 0x1cbff34du, 0x0d0088f5u};
    int res = 0;  // 1 greater, -1 less, 0 equal (most significant difference wins)
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        if (v.w[i] > h[i]) res = 1;
        else if (v.w[i] < h[i]) res = -1;
    }
    return res > 0;
}

// Jacobian coordinates on y^2 = x^3 + 4
struct g1j { fp X, Y, Z; };

// The Jacobian routines run one thread per point, a few warps per scheduler:
// their products are the out-of-line multiply of fp.cuh.
// dbl-2009-l (a = 0)
static __device__ __noinline__ g1j g1j_dbl(const g1j& p) {
    fp A = fp_sqr_ool(p.X), B = fp_sqr_ool(p.Y), C = fp_sqr_ool(B);
    fp D = fp_sub(fp_sub(fp_sqr_ool(fp_add(p.X, B)), A), C);
    D = fp_add(D, D);
    fp E = fp_add(fp_add(A, A), A);
    fp F = fp_sqr_ool(E);
    g1j r;
    r.X = fp_sub(F, fp_add(D, D));
    fp C8 = fp_add(C, C);
    C8 = fp_add(C8, C8);
    C8 = fp_add(C8, C8);
    r.Y = fp_sub(fp_mul_ool(E, fp_sub(D, r.X)), C8);
    r.Z = fp_mul_ool(fp_add(p.Y, p.Y), p.Z);
    return r;
}

// p + (qx, qy) with q affine (madd-2007-bl), exceptional cases handled
static __device__ __noinline__ g1j g1j_add_affine(const g1j& p, const fp& qx, const fp& qy) {
    if (fp_is_zero(p.Z)) return {qx, qy, fp_one()};
    fp Z1Z1 = fp_sqr_ool(p.Z);
    fp U2 = fp_mul_ool(qx, Z1Z1);
    fp S2 = fp_mul_ool(fp_mul_ool(qy, p.Z), Z1Z1);
    fp H = fp_sub(U2, p.X);
    fp rr = fp_sub(S2, p.Y);
    if (fp_is_zero(H)) {
        if (fp_is_zero(rr)) return g1j_dbl(p);
        return {fp_one(), fp_one(), fp_zero()};
    }
    rr = fp_add(rr, rr);
    fp HH = fp_sqr_ool(H);
    fp I = fp_add(HH, HH);
    I = fp_add(I, I);
    fp J = fp_mul_ool(H, I);
    fp V = fp_mul_ool(p.X, I);
    g1j r;
    r.X = fp_sub(fp_sub(fp_sqr_ool(rr), J), fp_add(V, V));
    fp YJ = fp_mul_ool(p.Y, J);
    r.Y = fp_sub(fp_mul_ool(rr, fp_sub(V, r.X)), fp_add(YJ, YJ));
    r.Z = fp_sub(fp_sub(fp_sqr_ool(fp_add(p.Z, H)), Z1Z1), HH);
    return r;
}

// p + q, both Jacobian (add-2007-bl), exceptional cases handled
static __device__ __noinline__ g1j g1j_add(const g1j& p, const g1j& q) {
    if (fp_is_zero(p.Z)) return q;
    if (fp_is_zero(q.Z)) return p;
    const fp Z1Z1 = fp_sqr_ool(p.Z), Z2Z2 = fp_sqr_ool(q.Z);
    const fp U1 = fp_mul_ool(p.X, Z2Z2), U2 = fp_mul_ool(q.X, Z1Z1);
    const fp S1 = fp_mul_ool(fp_mul_ool(p.Y, q.Z), Z2Z2), S2 = fp_mul_ool(fp_mul_ool(q.Y, p.Z), Z1Z1);
    const fp H = fp_sub(U2, U1);
    fp rr = fp_sub(S2, S1);
    if (fp_is_zero(H)) {
        if (fp_is_zero(rr)) return g1j_dbl(p);
        return {fp_one(), fp_one(), fp_zero()};
    }
    fp I = fp_add(H, H);
    I = fp_sqr_ool(I);
    const fp J = fp_mul_ool(H, I);
    rr = fp_add(rr, rr);
    const fp V = fp_mul_ool(U1, I);
    g1j r;
    r.X = fp_sub(fp_sub(fp_sqr_ool(rr), J), fp_add(V, V));
    const fp SJ = fp_mul_ool(S1, J);
    r.Y = fp_sub(fp_mul_ool(rr, fp_sub(V, r.X)), fp_add(SJ, SJ));
    r.Z = fp_mul_ool(fp_sub(fp_sub(fp_sqr_ool(fp_add(p.Z, q.Z)), Z1Z1), Z2Z2), H);
    return r;
}

// phi(P) == -[x^2] P for an affine curve point P (not the identity)
static __device__ __noinline__ bool g1_in_subgroup(const fp& x, const fp& y) {
    // x^2 = 0xac45a4010001a402_0000000100000000 (128 bits, 17 set)
    const uint64_t k[2] = {0x0000000100000000ULL, 0xac45a4010001a402ULL};
    g1j acc = {x, y, fp_one()};
    for (int i = 126; i >= 0; --i) {
        acc = g1j_dbl(acc);
        if ((k[i >> 6] >> (i & 63)) & 1) acc = g1j_add_affine(acc, x, y);
    }
    if (fp_is_zero(acc.Z)) return false;
    // beta, Montgomery form
    const uint64_t bv[6] = {0x30f1361b798a64e8ULL, 0xf3b8ddab7ece5a2aULL, 0x16a8ca3ac61577f7ULL,
                            0xc26a2ff874fd029bULL, 0x3636b76660701c6eULL, 0x051ba4ab241b6160ULL};
    fp beta = fp_load_u64(bv);
    fp Z2 = fp_sqr(acc.Z), Z3 = fp_mul(Z2, acc.Z);
    // X/Z^2 == beta x  and  Y/Z^3 == -y
    bool ex = fp_eq(acc.X, fp_mul(fp_mul(beta, x), Z2));
    bool ey = fp_eq(fp_add(acc.Y, fp_mul(y, Z3)), fp_zero());
    return ex && ey;
}

// Decode one 48-byte point.  On success writes Montgomery (x, y) and sets
// *identity for the point at infinity (x = 0, y = R mod p, the ic_bls12_381
// identity limbs).  Returns a status code.
__device__ __forceinline__ int32_t g1_decode(const uint8_t* in, fp& x, fp& y, bool& identity,
                                             bool check_subgroup) {
    identity = false;
    x = fp_zero();
    y = fp_zero();
    uint32_t top = in[0];
    bool comp = (top >> 7) & 1, inf = (top >> 6) & 1, sort = (top >> 5) & 1;
    fp raw;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        // limb i (little-endian) = big-endian bytes [44 - 4i, 48 - 4i)
        const uint8_t* b = in + 44 - 4 * i;
        uint32_t b0 = b[0];
        if (i == 11) b0 &= 0x1f;
        raw.w[i] = (b0 << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
    }
    if (!comp) return ST_BAD_FLAGS;
    if (inf) {
        if (sort || !fp_is_zero(raw)) return ST_BAD_FLAGS;
        identity = true;
        y = fp_one();
        return ST_OK;
    }
    if (fp_raw_geq_p(raw)) return ST_X_NOT_CANONICAL;
    fp xm = fp_to_mont(raw);
    fp y2 = fp_add(fp_mul(fp_sqr(xm), xm), fp_four());
    fp yy = fp_sqrt_candidate(y2);
    if (!fp_eq(fp_sqr(yy), y2)) return ST_NOT_ON_CURVE;
    if (fp_lex_largest(yy) != sort) yy = fp_neg(yy);
    if (check_subgroup && !g1_in_subgroup(xm, yy)) return ST_NOT_IN_SUBGROUP;
    x = xm;
    y = yy;
    return ST_OK;
}

// the raw-ABI identity convention: x = 0 and y in {0, R mod p}
__device__ __forceinline__ bool g1_limbs_identity(const fp& x, const fp& y) {
    return fp_is_zero(x) && (fp_is_zero(y) || fp_eq(y, fp_one()));
}

}  // namespace bls
