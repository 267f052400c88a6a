// BLS12-381 base field Fp on sm_100a: 381-bit Montgomery arithmetic on twelve
// 32-bit limbs, R = 2^384, every stored value canonical (< p), so a value's
// limbs equal ic_bls12_381's in-memory Montgomery representation.
//
// The multiply is CIOS (Koc, Acar, Kaliski, "Analyzing and comparing Montgomery
// multiplication algorithms", 1996) written as four PTX carry chains per row:
//   A  t[0..11]  += lo(a_j * b_i),  carry into t[12]
//   B  t[1..12]  += hi(a_j * b_i)
//   m  = t[0] * (-p^-1 mod 2^32)
//   C  t[0..11]  += lo(m * p_j),    carry into t[12]
//   D  t[1..12]  += hi(m * p_j)
// then a one-limb shift.  With a, b < p the running value stays below 2p
// before each row and below 2^415 inside it, so thirteen limbs hold it and the
// B and D chains never carry out of t[12].  Each chain is one asm statement, so
// the carry flag never crosses a statement boundary.  Per multiply: 12 rows x
// (48 mad + 1 mul.lo) = 588 IMAD-pipe instructions, plus the final subtraction.
//
// This replaces the reference's vendored sppark fp_t (gpu-crypto/cuda/vendor/
// sppark/mont_t.cuh:381-422, constants bls12-381.hpp:13-33) and is written from
// the algorithm, not from that file.
#pragma once
#include <cstdint>

namespace bls {

struct fp { uint32_t w[12]; };

// p, little-endian 32-bit limbs
#define BLS_P0 0xffffaaabu
#define BLS_P1 0xb9feffffu
#define BLS_P2 0xb153ffffu
#define BLS_P3 0x1eabfffeu
#define BLS_P4 0xf6b0f624u
#define BLS_P5 0x6730d2a0u
#define BLS_P6 0xf38512bfu
#define BLS_P7 0x64774b84u
#define BLS_P8 0x434bacd7u
#define BLS_P9 0x4b1ba7b6u
#define BLS_P10 0x397fe69au
#define BLS_P11 0x1a0111eau
#define BLS_NINV 0xfffcfffdu  // -p^-1 mod 2^32

__host__ __device__ __forceinline__ fp fp_zero() {
    fp r;
    for (int i = 0; i < 12; ++i) r.w[i] = 0;
    return r;
}
// R mod p (Montgomery one)
__host__ __device__ __forceinline__ fp fp_one() {
    fp r;
    r.w[0] = 0x0002fffdu; r.w[1] = 0x76090000u; r.w[2] = 0xc40c0002u; r.w[3] = 0xebf4000bu;
    r.w[4] = 0x53c758bau; r.w[5] = 0x5f489857u; r.w[6] = 0x70525745u; r.w[7] = 0x77ce5853u;
    r.w[8] = 0xa256ec6du; r.w[9] = 0x5c071a97u; r.w[10] = 0xfa80e493u; r.w[11] = 0x15f65ec3u;
    return r;
}
// R^2 mod p
__host__ __device__ __forceinline__ fp fp_rr() {
    fp r;
    r.w[0] = 0x1c341746u; r.w[1] = 0xf4df1f34u; r.w[2] = 0x09d104f1u; r.w[3] = 0x0a76e6a6u;
    r.w[4] = 0x4c95b6d5u; r.w[5] = 0x8de5476cu; r.w[6] = 0x939d83c0u; r.w[7] = 0x67eb88a9u;
    r.w[8] = 0xb519952du; r.w[9] = 0x9a793e85u; r.w[10] = 0x92cae3aau; r.w[11] = 0x11988fe5u;
    return r;
}

__device__ __forceinline__ bool fp_is_zero(const fp& a) {
    uint32_t o = a.w[0];
#pragma unroll
    for (int i = 1; i < 12; ++i) o |= a.w[i];
    return o == 0;
}
__device__ __forceinline__ bool fp_eq(const fp& a, const fp& b) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) o |= a.w[i] ^ b.w[i];
    return o == 0;
}

// ---------------------------------------------------------------------------
// carry chains
// ---------------------------------------------------------------------------
#define BLS_T13(t) "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), \
    "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11]), "+r"(t[12])
#define BLS_T1_12(t) "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), \
    "+r"(t[7]), "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11]), "+r"(t[12])
#define BLS_A12(a) "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), \
    "r"(a[6]), "r"(a[7]), "r"(a[8]), "r"(a[9]), "r"(a[10]), "r"(a[11])

// A: t[0..11] += lo(a * b), carry into t[12]
__device__ __forceinline__ void chain_lo(uint32_t* t, const uint32_t* a, uint32_t b) {
    asm("mad.lo.cc.u32 %0, %13, %25, %0;\n\t"
        "madc.lo.cc.u32 %1, %14, %25, %1;\n\t"
        "madc.lo.cc.u32 %2, %15, %25, %2;\n\t"
        "madc.lo.cc.u32 %3, %16, %25, %3;\n\t"
        "madc.lo.cc.u32 %4, %17, %25, %4;\n\t"
        "madc.lo.cc.u32 %5, %18, %25, %5;\n\t"
        "madc.lo.cc.u32 %6, %19, %25, %6;\n\t"
        "madc.lo.cc.u32 %7, %20, %25, %7;\n\t"
        "madc.lo.cc.u32 %8, %21, %25, %8;\n\t"
        "madc.lo.cc.u32 %9, %22, %25, %9;\n\t"
        "madc.lo.cc.u32 %10, %23, %25, %10;\n\t"
        "madc.lo.cc.u32 %11, %24, %25, %11;\n\t"
        "addc.u32 %12, %12, 0;"
        : BLS_T13(t) : BLS_A12(a), "r"(b));
}
// B: t[1..12] += hi(a * b); no carry leaves t[12]
__device__ __forceinline__ void chain_hi(uint32_t* t, const uint32_t* a, uint32_t b) {
    asm("mad.hi.cc.u32 %0, %12, %24, %0;\n\t"
        "madc.hi.cc.u32 %1, %13, %24, %1;\n\t"
        "madc.hi.cc.u32 %2, %14, %24, %2;\n\t"
        "madc.hi.cc.u32 %3, %15, %24, %3;\n\t"
        "madc.hi.cc.u32 %4, %16, %24, %4;\n\t"
        "madc.hi.cc.u32 %5, %17, %24, %5;\n\t"
        "madc.hi.cc.u32 %6, %18, %24, %6;\n\t"
        "madc.hi.cc.u32 %7, %19, %24, %7;\n\t"
        "madc.hi.cc.u32 %8, %20, %24, %8;\n\t"
        "madc.hi.cc.u32 %9, %21, %24, %9;\n\t"
        "madc.hi.cc.u32 %10, %22, %24, %10;\n\t"
        "madc.hi.u32 %11, %23, %24, %11;"
        : BLS_T1_12(t) : BLS_A12(a), "r"(b));
}
// C: t[0..11] += lo(m * p), carry into t[12]
__device__ __forceinline__ void chain_lo_p(uint32_t* t, uint32_t m) {
    asm("mad.lo.cc.u32 %0, %13, 0xffffaaab, %0;\n\t"
        "madc.lo.cc.u32 %1, %13, 0xb9feffff, %1;\n\t"
        "madc.lo.cc.u32 %2, %13, 0xb153ffff, %2;\n\t"
        "madc.lo.cc.u32 %3, %13, 0x1eabfffe, %3;\n\t"
        "madc.lo.cc.u32 %4, %13, 0xf6b0f624, %4;\n\t"
        "madc.lo.cc.u32 %5, %13, 0x6730d2a0, %5;\n\t"
        "madc.lo.cc.u32 %6, %13, 0xf38512bf, %6;\n\t"
        "madc.lo.cc.u32 %7, %13, 0x64774b84, %7;\n\t"
        "madc.lo.cc.u32 %8, %13, 0x434bacd7, %8;\n\t"
        "madc.lo.cc.u32 %9, %13, 0x4b1ba7b6, %9;\n\t"
        "madc.lo.cc.u32 %10, %13, 0x397fe69a, %10;\n\t"
        "madc.lo.cc.u32 %11, %13, 0x1a0111ea, %11;\n\t"
        "addc.u32 %12, %12, 0;"
        : BLS_T13(t) : "r"(m));
}
// D: t[1..12] += hi(m * p)
__device__ __forceinline__ void chain_hi_p(uint32_t* t, uint32_t m) {
    asm("mad.hi.cc.u32 %0, %12, 0xffffaaab, %0;\n\t"
        "madc.hi.cc.u32 %1, %12, 0xb9feffff, %1;\n\t"
        "madc.hi.cc.u32 %2, %12, 0xb153ffff, %2;\n\t"
        "madc.hi.cc.u32 %3, %12, 0x1eabfffe, %3;\n\t"
        "madc.hi.cc.u32 %4, %12, 0xf6b0f624, %4;\n\t"
        "madc.hi.cc.u32 %5, %12, 0x6730d2a0, %5;\n\t"
        "madc.hi.cc.u32 %6, %12, 0xf38512bf, %6;\n\t"
        "madc.hi.cc.u32 %7, %12, 0x64774b84, %7;\n\t"
        "madc.hi.cc.u32 %8, %12, 0x434bacd7, %8;\n\t"
        "madc.hi.cc.u32 %9, %12, 0x4b1ba7b6, %9;\n\t"
        "madc.hi.cc.u32 %10, %12, 0x397fe69a, %10;\n\t"
        "madc.hi.u32 %11, %12, 0x1a0111ea, %11;"
        : BLS_T1_12(t) : "r"(m));
}
// d = a - p over 12 limbs; returns the borrow (1 when a < p)
__device__ __forceinline__ uint32_t sub_p(uint32_t* d, const uint32_t* a) {
    uint32_t br;
    asm("sub.cc.u32 %0, %13, 0xffffaaab;\n\t"
        "subc.cc.u32 %1, %14, 0xb9feffff;\n\t"
        "subc.cc.u32 %2, %15, 0xb153ffff;\n\t"
        "subc.cc.u32 %3, %16, 0x1eabfffe;\n\t"
        "subc.cc.u32 %4, %17, 0xf6b0f624;\n\t"
        "subc.cc.u32 %5, %18, 0x6730d2a0;\n\t"
        "subc.cc.u32 %6, %19, 0xf38512bf;\n\t"
        "subc.cc.u32 %7, %20, 0x64774b84;\n\t"
        "subc.cc.u32 %8, %21, 0x434bacd7;\n\t"
        "subc.cc.u32 %9, %22, 0x4b1ba7b6;\n\t"
        "subc.cc.u32 %10, %23, 0x397fe69a;\n\t"
        "subc.cc.u32 %11, %24, 0x1a0111ea;\n\t"
        "subc.u32 %12, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
          "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(br)
        : BLS_A12(a));
    return br;  // 0xffffffff on borrow, else 0
}

// keep t if t < p, else t - p
__device__ __forceinline__ void reduce_once(uint32_t* t) {
    uint32_t d[12];
    uint32_t br = sub_p(d, t);
#pragma unroll
    for (int i = 0; i < 12; ++i) t[i] = br ? t[i] : d[i];
}

// ---------------------------------------------------------------------------
// field operations
// ---------------------------------------------------------------------------
// Montgomery product without the final subtraction.  For a, b < 8p (the
// redundant range of the lane-parallel kernel) the result is below 7.5p and
// every intermediate stays below 2^416, so thirteen limbs hold it.
__device__ __forceinline__ fp fp_mul_redundant(const fp& a, const fp& b) {
    uint32_t t[13];
#pragma unroll
    for (int i = 0; i < 13; ++i) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        chain_lo(t, a.w, b.w[i]);
        chain_hi(t, a.w, b.w[i]);
        uint32_t m = t[0] * BLS_NINV;
        chain_lo_p(t, m);
        chain_hi_p(t, m);
#pragma unroll
        for (int j = 0; j < 12; ++j) t[j] = t[j + 1];
        t[12] = 0;
    }
    fp r;
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = t[i];
    return r;
}

__device__ __forceinline__ fp fp_mul(const fp& a, const fp& b) {
    uint32_t t[13];
#pragma unroll
    for (int i = 0; i < 13; ++i) t[i] = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        chain_lo(t, a.w, b.w[i]);
        chain_hi(t, a.w, b.w[i]);
        uint32_t m = t[0] * BLS_NINV;
        chain_lo_p(t, m);
        chain_hi_p(t, m);
#pragma unroll
        for (int j = 0; j < 12; ++j) t[j] = t[j + 1];
        t[12] = 0;
    }
    reduce_once(t);
    fp r;
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = t[i];
    return r;
}
__device__ __forceinline__ fp fp_sqr(const fp& a) { return fp_mul(a, a); }

__device__ __forceinline__ fp fp_add(const fp& a, const fp& b) {
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
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]),
          "=r"(s[7]), "=r"(s[8]), "=r"(s[9]), "=r"(s[10]), "=r"(s[11])
        : BLS_A12(a.w), BLS_A12(b.w));
    reduce_once(s);  // a + b < 2p < 2^382: no carry out of limb 11
    fp r;
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = s[i];
    return r;
}

__device__ __forceinline__ fp fp_sub(const fp& a, const fp& b) {
    uint32_t s[12], mask;
    asm("sub.cc.u32 %0, %13, %25;\n\t"
        "subc.cc.u32 %1, %14, %26;\n\t"
        "subc.cc.u32 %2, %15, %27;\n\t"
        "subc.cc.u32 %3, %16, %28;\n\t"
        "subc.cc.u32 %4, %17, %29;\n\t"
        "subc.cc.u32 %5, %18, %30;\n\t"
        "subc.cc.u32 %6, %19, %31;\n\t"
        "subc.cc.u32 %7, %20, %32;\n\t"
        "subc.cc.u32 %8, %21, %33;\n\t"
        "subc.cc.u32 %9, %22, %34;\n\t"
        "subc.cc.u32 %10, %23, %35;\n\t"
        "subc.cc.u32 %11, %24, %36;\n\t"
        "subc.u32 %12, 0, 0;"
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]),
          "=r"(s[7]), "=r"(s[8]), "=r"(s[9]), "=r"(s[10]), "=r"(s[11]), "=r"(mask)
        : BLS_A12(a.w), BLS_A12(b.w));
    fp r;
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
        : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3]), "=r"(r.w[4]), "=r"(r.w[5]),
          "=r"(r.w[6]), "=r"(r.w[7]), "=r"(r.w[8]), "=r"(r.w[9]), "=r"(r.w[10]), "=r"(r.w[11])
        : BLS_A12(s), "r"(BLS_P0 & mask), "r"(BLS_P1 & mask), "r"(BLS_P2 & mask), "r"(BLS_P3 & mask),
          "r"(BLS_P4 & mask), "r"(BLS_P5 & mask), "r"(BLS_P6 & mask), "r"(BLS_P7 & mask),
          "r"(BLS_P8 & mask), "r"(BLS_P9 & mask), "r"(BLS_P10 & mask), "r"(BLS_P11 & mask));
    return r;
}

__device__ __forceinline__ fp fp_neg(const fp& a) { return fp_sub(fp_zero(), a); }
__device__ __forceinline__ fp fp_dbl(const fp& a) { return fp_add(a, a); }

// ---------------------------------------------------------------------------
// conversions
// ---------------------------------------------------------------------------
__device__ __forceinline__ fp fp_load_u64(const uint64_t* v) {
    fp r;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        r.w[2 * i] = (uint32_t)v[i];
        r.w[2 * i + 1] = (uint32_t)(v[i] >> 32);
    }
    return r;
}
__device__ __forceinline__ void fp_store_u64(uint64_t* v, const fp& a) {
#pragma unroll
    for (int i = 0; i < 6; ++i) v[i] = ((uint64_t)a.w[2 * i + 1] << 32) | a.w[2 * i];
}
// Montgomery -> canonical integer limbs (multiply by 1)
__device__ __forceinline__ fp fp_from_mont(const fp& a) {
    fp one_raw = fp_zero();
    one_raw.w[0] = 1;
    return fp_mul(a, one_raw);
}
// canonical integer limbs (< p) -> Montgomery (multiply by R^2)
__device__ __forceinline__ fp fp_to_mont(const fp& a) { return fp_mul(a, fp_rr()); }

// true when the canonical limbs are >= p
__device__ __forceinline__ bool fp_raw_geq_p(const fp& a) {
    uint32_t d[12];
    return sub_p(d, a.w) == 0;
}

// a^e for a fixed exponent given as 6 little-endian u64 words (right to left)
__device__ __forceinline__ fp fp_pow_u64(const fp& a, const uint64_t* e, int nbits) {
    fp r = fp_one(), base = a;
    for (int i = 0; i < nbits; ++i) {
        if ((e[i >> 6] >> (i & 63)) & 1) r = fp_mul(r, base);
        base = fp_sqr(base);
    }
    return r;
}

// An out-of-line Montgomery multiply, and a power over it, for code that runs
// few warps per scheduler (a thread per point, per key or per message): there
// nothing hides a miss in the instruction cache, and a loop that inlines a
// multiply of several hundred instructions at every use misses on each pass.
static __device__ __noinline__ fp fp_mul_ool(const fp& a, const fp& b) { return fp_mul(a, b); }
__device__ __forceinline__ fp fp_sqr_ool(const fp& a) { return fp_mul_ool(a, a); }
__device__ __forceinline__ fp fp_pow_ool(const fp& a, const uint64_t* e, int nbits) {
    fp r = fp_one(), base = a;
    for (int i = 0; i < nbits; ++i) {
        if ((e[i >> 6] >> (i & 63)) & 1) r = fp_mul_ool(r, base);
        base = fp_mul_ool(base, base);
    }
    return r;
}

}  // namespace bls
