// BLS12-381 extension tower on the device:
//   Fp2  = Fp[u]  / (u^2 + 1)
//   Fp6  = Fp2[v] / (v^3 - xi),  xi = 1 + u
//   Fp12 = Fp6[w] / (w^2 - v)
// Formulas follow the reference tower (gpu-crypto/cuda/field_sppark.cuh:52-197),
// which mirrors ic_bls12_381 0.10.1: Karatsuba Fp2/Fp6/Fp12 products, the sparse
// line product mul_by_014, Frobenius with fixed Montgomery constants, the
// inversion (binary extended Euclid, fp_inv.cuh; the reference's Fermat power
// gives the same value), and Granger-Scott squaring in the cyclotomic
// subgroup.  The tower keeps its products inline: the out-of-line multiply of
// fp.cuh made the thread-per-verification kernel 20% faster but the key
// ingest kernels (255 registers, large live state) up to 50% slower.  Every
// value is canonical, so the final limbs equal the CPU verifier's bit for bit
// whatever order the device evaluates the same formula in.
#pragma once
#include "fp.cuh"
#include "fp_inv.cuh"

namespace bls {

struct fp2 { fp c0, c1; };
struct fp6 { fp2 c0, c1, c2; };
struct fp12 { fp6 c0, c1; };

// ----------------------------------------------------------------- Fp2
__device__ __forceinline__ fp2 fp2_zero() { return {fp_zero(), fp_zero()}; }
__device__ __forceinline__ fp2 fp2_one() { return {fp_one(), fp_zero()}; }
__device__ __forceinline__ fp2 fp2_add(const fp2& a, const fp2& b) { return {fp_add(a.c0, b.c0), fp_add(a.c1, b.c1)}; }
__device__ __forceinline__ fp2 fp2_sub(const fp2& a, const fp2& b) { return {fp_sub(a.c0, b.c0), fp_sub(a.c1, b.c1)}; }
__device__ __forceinline__ fp2 fp2_neg(const fp2& a) { return {fp_neg(a.c0), fp_neg(a.c1)}; }
__device__ __forceinline__ fp2 fp2_conj(const fp2& a) { return {a.c0, fp_neg(a.c1)}; }
__device__ __forceinline__ fp2 fp2_dbl(const fp2& a) { return fp2_add(a, a); }
// times xi = 1 + u
__device__ __forceinline__ fp2 fp2_mul_nr(const fp2& a) { return {fp_sub(a.c0, a.c1), fp_add(a.c0, a.c1)}; }
__device__ __forceinline__ bool fp2_is_zero(const fp2& a) { return fp_is_zero(a.c0) && fp_is_zero(a.c1); }

static __device__ __noinline__ fp2 fp2_mul_fp(const fp2& a, const fp& s) { return {fp_mul(a.c0, s), fp_mul(a.c1, s)}; }

// (a0 + a1 u)(b0 + b1 u): three products (field_sppark.cuh:65-68)
static __device__ __noinline__ fp2 fp2_mul(const fp2& a, const fp2& b) {
    fp t0 = fp_mul(a.c0, b.c0);
    fp t1 = fp_mul(a.c1, b.c1);
    fp t2 = fp_mul(fp_add(a.c0, a.c1), fp_add(b.c0, b.c1));
    return {fp_sub(t0, t1), fp_sub(fp_sub(t2, t0), t1)};
}
// (a0 + a1)(a0 - a1) + 2 a0 a1 u (field_sppark.cuh:69-78)
static __device__ __noinline__ fp2 fp2_sqr(const fp2& a) {
    fp t = fp_mul(a.c0, a.c1);
    fp s = fp_mul(fp_add(a.c0, a.c1), fp_sub(a.c0, a.c1));
    return {s, fp_add(t, t)};
}

// a^-1, 0 for 0 (the reference's Fermat a^(p-2), field_sppark.cuh:40-50,
// gives the same value): the binary extended Euclid of fp_inv.cuh
static __device__ __noinline__ fp fp_inv(const fp& a) {
    const fp r3 = fp_mul(fp_rr(), fp_rr());              // R^3 mod p
    return fp_inverse_mont(a, r3.w);
}
static __device__ __noinline__ fp2 fp2_inv(const fp2& a) {
    fp n = fp_add(fp_sqr(a.c0), fp_sqr(a.c1));
    fp i = fp_inv(n);
    return {fp_mul(a.c0, i), fp_neg(fp_mul(a.c1, i))};
}

// ----------------------------------------------------------------- Fp6
__device__ __forceinline__ fp6 fp6_zero() { return {fp2_zero(), fp2_zero(), fp2_zero()}; }
__device__ __forceinline__ fp6 fp6_one() { return {fp2_one(), fp2_zero(), fp2_zero()}; }
__device__ __forceinline__ fp6 fp6_add(const fp6& a, const fp6& b) { return {fp2_add(a.c0, b.c0), fp2_add(a.c1, b.c1), fp2_add(a.c2, b.c2)}; }
__device__ __forceinline__ fp6 fp6_sub(const fp6& a, const fp6& b) { return {fp2_sub(a.c0, b.c0), fp2_sub(a.c1, b.c1), fp2_sub(a.c2, b.c2)}; }
__device__ __forceinline__ fp6 fp6_neg(const fp6& a) { return {fp2_neg(a.c0), fp2_neg(a.c1), fp2_neg(a.c2)}; }
__device__ __forceinline__ fp6 fp6_mul_by_v(const fp6& a) { return {fp2_mul_nr(a.c2), a.c0, a.c1}; }

// Karatsuba over Fp2 (field_sppark.cuh:95-102)
static __device__ __noinline__ fp6 fp6_mul(const fp6& a, const fp6& b) {
    fp2 aa = fp2_mul(a.c0, b.c0), bb = fp2_mul(a.c1, b.c1), cc = fp2_mul(a.c2, b.c2);
    fp2 x = fp2_mul(fp2_add(a.c1, a.c2), fp2_add(b.c1, b.c2));
    fp2 y = fp2_mul(fp2_add(a.c0, a.c1), fp2_add(b.c0, b.c1));
    fp2 z = fp2_mul(fp2_add(a.c0, a.c2), fp2_add(b.c0, b.c2));
    fp6 r;
    r.c0 = fp2_add(aa, fp2_mul_nr(fp2_sub(fp2_sub(x, bb), cc)));
    r.c1 = fp2_add(fp2_sub(fp2_sub(y, aa), bb), fp2_mul_nr(cc));
    r.c2 = fp2_add(fp2_sub(fp2_sub(z, aa), cc), bb);
    return r;
}
// field_sppark.cuh:104-111
static __device__ __noinline__ fp6 fp6_inv(const fp6& f) {
    fp2 c0s = fp2_sqr(f.c0), c1s = fp2_sqr(f.c1), c2s = fp2_sqr(f.c2);
    fp2 c01 = fp2_mul(f.c0, f.c1), c02 = fp2_mul(f.c0, f.c2), c12 = fp2_mul(f.c1, f.c2);
    fp2 t0 = fp2_sub(c0s, fp2_mul_nr(c12));
    fp2 t1 = fp2_sub(fp2_mul_nr(c2s), c01);
    fp2 t2 = fp2_sub(c1s, c02);
    fp2 sc = fp2_add(fp2_mul(f.c0, t0), fp2_mul_nr(fp2_add(fp2_mul(f.c2, t1), fp2_mul(f.c1, t2))));
    fp2 si = fp2_inv(sc);
    return {fp2_mul(t0, si), fp2_mul(t1, si), fp2_mul(t2, si)};
}

// Frobenius coefficients xi^((p-1)/3) = (0, k1), xi^(2(p-1)/3) = (k2, 0),
// xi^((p-1)/6) = (k3, k4), Montgomery limbs (field_sppark.cuh:113-123, 159-166)
__device__ __forceinline__ fp frob_k1() {
    const uint64_t v[6] = {0xcd03c9e48671f071ULL, 0x5dab22461fcda5d2ULL, 0x587042afd3851b95ULL,
                           0x8eb60ebe01bacb9eULL, 0x03f97d6e83d050d2ULL, 0x18f0206554638741ULL};
    return fp_load_u64(v);
}
__device__ __forceinline__ fp frob_k2() {
    const uint64_t v[6] = {0x890dc9e4867545c3ULL, 0x2af322533285a5d5ULL, 0x50880866309b7e2cULL,
                           0xa20d1b8c7e881024ULL, 0x14e4f04fe2db9068ULL, 0x14e56d3f1564853aULL};
    return fp_load_u64(v);
}
__device__ __forceinline__ fp2 frob_k12() {
    const uint64_t a[6] = {0x07089552b319d465ULL, 0xc6695f92b50a8313ULL, 0x97e83cccd117228fULL,
                           0xa35baecab2dc29eeULL, 0x1ce393ea5daace4dULL, 0x08f2220fb0fb66ebULL};
    const uint64_t b[6] = {0xb2f66aad4ce5d646ULL, 0x5842a06bfc497cecULL, 0xcf4895d42599d394ULL,
                           0xc11b9cba40a8e8d0ULL, 0x2e3813cbe5a0de89ULL, 0x110eefda88847fafULL};
    return {fp_load_u64(a), fp_load_u64(b)};
}
static __device__ __noinline__ fp6 fp6_frob(const fp6& f) {
    fp2 c1 = fp2_conj(f.c1), c2 = fp2_conj(f.c2);
    fp k1 = frob_k1(), k2 = frob_k2();
    // (x0 + x1 u) * (0 + k1 u) = -x1 k1 + x0 k1 u ;  (x0 + x1 u) * k2
    fp2 r1 = {fp_neg(fp_mul(c1.c1, k1)), fp_mul(c1.c0, k1)};
    fp2 r2 = {fp_mul(c2.c0, k2), fp_mul(c2.c1, k2)};
    return {fp2_conj(f.c0), r1, r2};
}

// sparse products (field_sppark.cuh:126-134)
static __device__ __noinline__ fp6 fp6_mul_by_01(const fp6& s, const fp2& c0, const fp2& c1) {
    fp2 aa = fp2_mul(s.c0, c0), bb = fp2_mul(s.c1, c1);
    fp6 r;
    r.c0 = fp2_add(fp2_mul_nr(fp2_mul(s.c2, c1)), aa);
    r.c1 = fp2_sub(fp2_sub(fp2_mul(fp2_add(c0, c1), fp2_add(s.c0, s.c1)), aa), bb);
    r.c2 = fp2_add(fp2_mul(s.c2, c0), bb);
    return r;
}
static __device__ __noinline__ fp6 fp6_mul_by_1(const fp6& s, const fp2& c1) {
    return {fp2_mul_nr(fp2_mul(s.c2, c1)), fp2_mul(s.c0, c1), fp2_mul(s.c1, c1)};
}

// ----------------------------------------------------------------- Fp12
__device__ __forceinline__ fp12 fp12_one() { return {fp6_one(), fp6_zero()}; }
__device__ __forceinline__ fp12 fp12_conj(const fp12& a) { return {a.c0, fp6_neg(a.c1)}; }

// field_sppark.cuh:142-146
static __device__ __noinline__ fp12 fp12_mul(const fp12& a, const fp12& b) {
    fp6 aa = fp6_mul(a.c0, b.c0), bb = fp6_mul(a.c1, b.c1);
    fp6 s = fp6_mul(fp6_add(a.c0, a.c1), fp6_add(b.c0, b.c1));
    return {fp6_add(aa, fp6_mul_by_v(bb)), fp6_sub(fp6_sub(s, aa), bb)};
}
// field_sppark.cuh:148-151
static __device__ __noinline__ fp12 fp12_sqr(const fp12& a) {
    fp6 ab = fp6_mul(a.c0, a.c1);
    fp6 s = fp6_mul(fp6_add(a.c0, fp6_mul_by_v(a.c1)), fp6_add(a.c0, a.c1));
    return {fp6_sub(fp6_sub(s, ab), fp6_mul_by_v(ab)), fp6_add(ab, ab)};
}
// field_sppark.cuh:153-157
static __device__ __noinline__ fp12 fp12_inv(const fp12& f) {
    fp6 t = fp6_sub(fp6_mul(f.c0, f.c0), fp6_mul_by_v(fp6_mul(f.c1, f.c1)));
    fp6 ti = fp6_inv(t);
    return {fp6_mul(f.c0, ti), fp6_neg(fp6_mul(f.c1, ti))};
}
// field_sppark.cuh:159-166
static __device__ __noinline__ fp12 fp12_frob(const fp12& f) {
    fp6 c0 = fp6_frob(f.c0), c1 = fp6_frob(f.c1);
    fp2 k = frob_k12();
    return {c0, {fp2_mul(c1.c0, k), fp2_mul(c1.c1, k), fp2_mul(c1.c2, k)}};
}
// f * (c0 + c1 v + c4 v w)  (field_sppark.cuh:168-172)
static __device__ __noinline__ fp12 fp12_mul_by_014(const fp12& f, const fp2& c0, const fp2& c1, const fp2& c4) {
    fp6 aa = fp6_mul_by_01(f.c0, c0, c1);
    fp6 bb = fp6_mul_by_1(f.c1, c4);
    fp6 t = fp6_mul_by_01(fp6_add(f.c1, f.c0), c0, fp2_add(c1, c4));
    return {fp6_add(fp6_mul_by_v(bb), aa), fp6_sub(fp6_sub(t, aa), bb)};
}

// Granger-Scott squaring on the cyclotomic subgroup (field_sppark.cuh:174-197)
__device__ __forceinline__ void fp4_square(const fp2& a, const fp2& b, fp2& o0, fp2& o1) {
    fp2 t0 = fp2_sqr(a), t1 = fp2_sqr(b);
    o0 = fp2_add(fp2_mul_nr(t1), t0);
    o1 = fp2_sub(fp2_sub(fp2_sqr(fp2_add(a, b)), t0), t1);
}
static __device__ __noinline__ fp12 fp12_cyclotomic_sqr(const fp12& f) {
    fp2 z0 = f.c0.c0, z4 = f.c0.c1, z3 = f.c0.c2, z2 = f.c1.c0, z1 = f.c1.c1, z5 = f.c1.c2;
    fp2 A0, A1, B0, B1, C0, C1;
    fp4_square(z0, z1, A0, A1);
    fp4_square(z2, z3, B0, B1);
    fp4_square(z4, z5, C0, C1);
    z0 = fp2_sub(A0, z0); z0 = fp2_add(fp2_dbl(z0), A0);
    z1 = fp2_add(A1, z1); z1 = fp2_add(fp2_dbl(z1), A1);
    z4 = fp2_sub(B0, z4); z4 = fp2_add(fp2_dbl(z4), B0);
    z5 = fp2_add(B1, z5); z5 = fp2_add(fp2_dbl(z5), B1);
    fp2 nc1 = fp2_mul_nr(C1);
    z2 = fp2_add(nc1, z2); z2 = fp2_add(fp2_dbl(z2), nc1);
    z3 = fp2_sub(C0, z3); z3 = fp2_add(fp2_dbl(z3), C0);
    return {{z0, z4, z3}, {z2, z1, z5}};
}

__device__ __forceinline__ bool fp12_is_one(const fp12& r) {
    const fp* v = (const fp*)&r;
    bool ok = fp_eq(v[0], fp_one());
#pragma unroll
    for (int i = 1; i < 12; ++i) ok = ok && fp_is_zero(v[i]);
    return ok;
}

}  // namespace bls
