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
#define BLS_T24(t) "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), \
    "+r"(t[6]), "+r"(t[7]), "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11]), "+r"(t[12]), \
    "+r"(t[13]), "+r"(t[14]), "+r"(t[15]), "+r"(t[16]), "+r"(t[17]), "+r"(t[18]), "+r"(t[19]), \
    "+r"(t[20]), "+r"(t[21]), "+r"(t[22]), "+r"(t[23])

// Montgomery square a^2 R^-1 mod p for a < 2p, canonical (below p): the 66
// cross products a_i a_j (i < j) once, by rows (row i adds a_i * a[i+1..11] at
// limb 2i+1 and carries into the fresh limb i+12; the rows before it fill
// limbs up to i+11 and their sum stays below 2^(32(i+13)), so no carry leaves
// it), doubled by a one-bit shift, plus the twelve squares a_i^2 in one chain;
// then the low twelve limbs are Montgomery-reduced on their own, (t_lo + m p)
// / R <= p, and the high twelve added: a^2 / R + p < 1.5p for a < 2p, so one
// conditional subtraction ends it.  456 multiply instructions where the
// general product takes 588; the same value as fp_mul(a, a).
__device__ __forceinline__ fp fp_sqr(const fp& a) {
    uint32_t t[24];
#pragma unroll
    for (int i = 0; i < 24; ++i) t[i] = 0;
    asm(
        "mad.lo.cc.u32 %1, %24, %25, %1;\n\t"
        "madc.lo.cc.u32 %2, %24, %26, %2;\n\t"
        "madc.lo.cc.u32 %3, %24, %27, %3;\n\t"
        "madc.lo.cc.u32 %4, %24, %28, %4;\n\t"
        "madc.lo.cc.u32 %5, %24, %29, %5;\n\t"
        "madc.lo.cc.u32 %6, %24, %30, %6;\n\t"
        "madc.lo.cc.u32 %7, %24, %31, %7;\n\t"
        "madc.lo.cc.u32 %8, %24, %32, %8;\n\t"
        "madc.lo.cc.u32 %9, %24, %33, %9;\n\t"
        "madc.lo.cc.u32 %10, %24, %34, %10;\n\t"
        "madc.lo.cc.u32 %11, %24, %35, %11;\n\t"
        "addc.u32 %12, %12, 0;\n\t"
        "mad.hi.cc.u32 %2, %24, %25, %2;\n\t"
        "madc.hi.cc.u32 %3, %24, %26, %3;\n\t"
        "madc.hi.cc.u32 %4, %24, %27, %4;\n\t"
        "madc.hi.cc.u32 %5, %24, %28, %5;\n\t"
        "madc.hi.cc.u32 %6, %24, %29, %6;\n\t"
        "madc.hi.cc.u32 %7, %24, %30, %7;\n\t"
        "madc.hi.cc.u32 %8, %24, %31, %8;\n\t"
        "madc.hi.cc.u32 %9, %24, %32, %9;\n\t"
        "madc.hi.cc.u32 %10, %24, %33, %10;\n\t"
        "madc.hi.cc.u32 %11, %24, %34, %11;\n\t"
        "madc.hi.u32 %12, %24, %35, %12;\n\t"
        "mad.lo.cc.u32 %3, %25, %26, %3;\n\t"
        "madc.lo.cc.u32 %4, %25, %27, %4;\n\t"
        "madc.lo.cc.u32 %5, %25, %28, %5;\n\t"
        "madc.lo.cc.u32 %6, %25, %29, %6;\n\t"
        "madc.lo.cc.u32 %7, %25, %30, %7;\n\t"
        "madc.lo.cc.u32 %8, %25, %31, %8;\n\t"
        "madc.lo.cc.u32 %9, %25, %32, %9;\n\t"
        "madc.lo.cc.u32 %10, %25, %33, %10;\n\t"
        "madc.lo.cc.u32 %11, %25, %34, %11;\n\t"
        "madc.lo.cc.u32 %12, %25, %35, %12;\n\t"
        "addc.u32 %13, %13, 0;\n\t"
        "mad.hi.cc.u32 %4, %25, %26, %4;\n\t"
        "madc.hi.cc.u32 %5, %25, %27, %5;\n\t"
        "madc.hi.cc.u32 %6, %25, %28, %6;\n\t"
        "madc.hi.cc.u32 %7, %25, %29, %7;\n\t"
        "madc.hi.cc.u32 %8, %25, %30, %8;\n\t"
        "madc.hi.cc.u32 %9, %25, %31, %9;\n\t"
        "madc.hi.cc.u32 %10, %25, %32, %10;\n\t"
        "madc.hi.cc.u32 %11, %25, %33, %11;\n\t"
        "madc.hi.cc.u32 %12, %25, %34, %12;\n\t"
        "madc.hi.u32 %13, %25, %35, %13;\n\t"
        "mad.lo.cc.u32 %5, %26, %27, %5;\n\t"
        "madc.lo.cc.u32 %6, %26, %28, %6;\n\t"
        "madc.lo.cc.u32 %7, %26, %29, %7;\n\t"
        "madc.lo.cc.u32 %8, %26, %30, %8;\n\t"
        "madc.lo.cc.u32 %9, %26, %31, %9;\n\t"
        "madc.lo.cc.u32 %10, %26, %32, %10;\n\t"
        "madc.lo.cc.u32 %11, %26, %33, %11;\n\t"
        "madc.lo.cc.u32 %12, %26, %34, %12;\n\t"
        "madc.lo.cc.u32 %13, %26, %35, %13;\n\t"
        "addc.u32 %14, %14, 0;\n\t"
        "mad.hi.cc.u32 %6, %26, %27, %6;\n\t"
        "madc.hi.cc.u32 %7, %26, %28, %7;\n\t"
        "madc.hi.cc.u32 %8, %26, %29, %8;\n\t"
        "madc.hi.cc.u32 %9, %26, %30, %9;\n\t"
        "madc.hi.cc.u32 %10, %26, %31, %10;\n\t"
        "madc.hi.cc.u32 %11, %26, %32, %11;\n\t"
        "madc.hi.cc.u32 %12, %26, %33, %12;\n\t"
        "madc.hi.cc.u32 %13, %26, %34, %13;\n\t"
        "madc.hi.u32 %14, %26, %35, %14;\n\t"
        "mad.lo.cc.u32 %7, %27, %28, %7;\n\t"
        "madc.lo.cc.u32 %8, %27, %29, %8;\n\t"
        "madc.lo.cc.u32 %9, %27, %30, %9;\n\t"
        "madc.lo.cc.u32 %10, %27, %31, %10;\n\t"
        "madc.lo.cc.u32 %11, %27, %32, %11;\n\t"
        "madc.lo.cc.u32 %12, %27, %33, %12;\n\t"
        "madc.lo.cc.u32 %13, %27, %34, %13;\n\t"
        "madc.lo.cc.u32 %14, %27, %35, %14;\n\t"
        "addc.u32 %15, %15, 0;\n\t"
        "mad.hi.cc.u32 %8, %27, %28, %8;\n\t"
        "madc.hi.cc.u32 %9, %27, %29, %9;\n\t"
        "madc.hi.cc.u32 %10, %27, %30, %10;\n\t"
        "madc.hi.cc.u32 %11, %27, %31, %11;\n\t"
        "madc.hi.cc.u32 %12, %27, %32, %12;\n\t"
        "madc.hi.cc.u32 %13, %27, %33, %13;\n\t"
        "madc.hi.cc.u32 %14, %27, %34, %14;\n\t"
        "madc.hi.u32 %15, %27, %35, %15;\n\t"
        "mad.lo.cc.u32 %9, %28, %29, %9;\n\t"
        "madc.lo.cc.u32 %10, %28, %30, %10;\n\t"
        "madc.lo.cc.u32 %11, %28, %31, %11;\n\t"
        "madc.lo.cc.u32 %12, %28, %32, %12;\n\t"
        "madc.lo.cc.u32 %13, %28, %33, %13;\n\t"
        "madc.lo.cc.u32 %14, %28, %34, %14;\n\t"
        "madc.lo.cc.u32 %15, %28, %35, %15;\n\t"
        "addc.u32 %16, %16, 0;\n\t"
        "mad.hi.cc.u32 %10, %28, %29, %10;\n\t"
        "madc.hi.cc.u32 %11, %28, %30, %11;\n\t"
        "madc.hi.cc.u32 %12, %28, %31, %12;\n\t"
        "madc.hi.cc.u32 %13, %28, %32, %13;\n\t"
        "madc.hi.cc.u32 %14, %28, %33, %14;\n\t"
        "madc.hi.cc.u32 %15, %28, %34, %15;\n\t"
        "madc.hi.u32 %16, %28, %35, %16;\n\t"
        "mad.lo.cc.u32 %11, %29, %30, %11;\n\t"
        "madc.lo.cc.u32 %12, %29, %31, %12;\n\t"
        "madc.lo.cc.u32 %13, %29, %32, %13;\n\t"
        "madc.lo.cc.u32 %14, %29, %33, %14;\n\t"
        "madc.lo.cc.u32 %15, %29, %34, %15;\n\t"
        "madc.lo.cc.u32 %16, %29, %35, %16;\n\t"
        "addc.u32 %17, %17, 0;\n\t"
        "mad.hi.cc.u32 %12, %29, %30, %12;\n\t"
        "madc.hi.cc.u32 %13, %29, %31, %13;\n\t"
        "madc.hi.cc.u32 %14, %29, %32, %14;\n\t"
        "madc.hi.cc.u32 %15, %29, %33, %15;\n\t"
        "madc.hi.cc.u32 %16, %29, %34, %16;\n\t"
        "madc.hi.u32 %17, %29, %35, %17;\n\t"
        "mad.lo.cc.u32 %13, %30, %31, %13;\n\t"
        "madc.lo.cc.u32 %14, %30, %32, %14;\n\t"
        "madc.lo.cc.u32 %15, %30, %33, %15;\n\t"
        "madc.lo.cc.u32 %16, %30, %34, %16;\n\t"
        "madc.lo.cc.u32 %17, %30, %35, %17;\n\t"
        "addc.u32 %18, %18, 0;\n\t"
        "mad.hi.cc.u32 %14, %30, %31, %14;\n\t"
        "madc.hi.cc.u32 %15, %30, %32, %15;\n\t"
        "madc.hi.cc.u32 %16, %30, %33, %16;\n\t"
        "madc.hi.cc.u32 %17, %30, %34, %17;\n\t"
        "madc.hi.u32 %18, %30, %35, %18;\n\t"
        "mad.lo.cc.u32 %15, %31, %32, %15;\n\t"
        "madc.lo.cc.u32 %16, %31, %33, %16;\n\t"
        "madc.lo.cc.u32 %17, %31, %34, %17;\n\t"
        "madc.lo.cc.u32 %18, %31, %35, %18;\n\t"
        "addc.u32 %19, %19, 0;\n\t"
        "mad.hi.cc.u32 %16, %31, %32, %16;\n\t"
        "madc.hi.cc.u32 %17, %31, %33, %17;\n\t"
        "madc.hi.cc.u32 %18, %31, %34, %18;\n\t"
        "madc.hi.u32 %19, %31, %35, %19;\n\t"
        "mad.lo.cc.u32 %17, %32, %33, %17;\n\t"
        "madc.lo.cc.u32 %18, %32, %34, %18;\n\t"
        "madc.lo.cc.u32 %19, %32, %35, %19;\n\t"
        "addc.u32 %20, %20, 0;\n\t"
        "mad.hi.cc.u32 %18, %32, %33, %18;\n\t"
        "madc.hi.cc.u32 %19, %32, %34, %19;\n\t"
        "madc.hi.u32 %20, %32, %35, %20;\n\t"
        "mad.lo.cc.u32 %19, %33, %34, %19;\n\t"
        "madc.lo.cc.u32 %20, %33, %35, %20;\n\t"
        "addc.u32 %21, %21, 0;\n\t"
        "mad.hi.cc.u32 %20, %33, %34, %20;\n\t"
        "madc.hi.u32 %21, %33, %35, %21;\n\t"
        "mad.lo.cc.u32 %21, %34, %35, %21;\n\t"
        "addc.u32 %22, %22, 0;\n\t"
        "mad.hi.u32 %22, %34, %35, %22;"
        : BLS_T24(t) : BLS_A12(a.w));
    t[23] = t[22] >> 31;
#pragma unroll
    for (int k = 22; k >= 1; --k) t[k] = __funnelshift_l(t[k - 1], t[k], 1);
    t[0] <<= 1;
    asm(
        "mad.lo.cc.u32 %0, %24, %24, %0;\n\t"
        "madc.hi.cc.u32 %1, %24, %24, %1;\n\t"
        "madc.lo.cc.u32 %2, %25, %25, %2;\n\t"
        "madc.hi.cc.u32 %3, %25, %25, %3;\n\t"
        "madc.lo.cc.u32 %4, %26, %26, %4;\n\t"
        "madc.hi.cc.u32 %5, %26, %26, %5;\n\t"
        "madc.lo.cc.u32 %6, %27, %27, %6;\n\t"
        "madc.hi.cc.u32 %7, %27, %27, %7;\n\t"
        "madc.lo.cc.u32 %8, %28, %28, %8;\n\t"
        "madc.hi.cc.u32 %9, %28, %28, %9;\n\t"
        "madc.lo.cc.u32 %10, %29, %29, %10;\n\t"
        "madc.hi.cc.u32 %11, %29, %29, %11;\n\t"
        "madc.lo.cc.u32 %12, %30, %30, %12;\n\t"
        "madc.hi.cc.u32 %13, %30, %30, %13;\n\t"
        "madc.lo.cc.u32 %14, %31, %31, %14;\n\t"
        "madc.hi.cc.u32 %15, %31, %31, %15;\n\t"
        "madc.lo.cc.u32 %16, %32, %32, %16;\n\t"
        "madc.hi.cc.u32 %17, %32, %32, %17;\n\t"
        "madc.lo.cc.u32 %18, %33, %33, %18;\n\t"
        "madc.hi.cc.u32 %19, %33, %33, %19;\n\t"
        "madc.lo.cc.u32 %20, %34, %34, %20;\n\t"
        "madc.hi.cc.u32 %21, %34, %34, %21;\n\t"
        "madc.lo.cc.u32 %22, %35, %35, %22;\n\t"
        "madc.hi.u32 %23, %35, %35, %23;"
        : BLS_T24(t) : BLS_A12(a.w));
    uint32_t u[13];
#pragma unroll
    for (int i = 0; i < 12; ++i) u[i] = t[i];
    u[12] = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const uint32_t m = u[0] * BLS_NINV;
        chain_lo_p(u, m);
        chain_hi_p(u, m);
#pragma unroll
        for (int j = 0; j < 12; ++j) u[j] = u[j + 1];
        u[12] = 0;
    }
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
        : BLS_A12(u), "r"(t[12]), "r"(t[13]), "r"(t[14]), "r"(t[15]), "r"(t[16]), "r"(t[17]),
          "r"(t[18]), "r"(t[19]), "r"(t[20]), "r"(t[21]), "r"(t[22]), "r"(t[23]));
    reduce_once(s);
    fp r;
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = s[i];
    return r;
}

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

// An out-of-line Montgomery multiply and square, and a power over them, for
// code that runs few warps per scheduler (a thread per point, per key or per
// message): there nothing hides a miss in the instruction cache, and a loop
// that inlines a multiply of several hundred instructions at every use misses
// on each pass.
static __device__ __noinline__ fp fp_mul_ool(const fp& a, const fp& b) { return fp_mul(a, b); }
static __device__ __noinline__ fp fp_sqr_ool(const fp& a) { return fp_sqr(a); }

// a^e (e: nbits bits, little-endian u64 words, the same for every thread) by
// a left-to-right sliding window of four bits over the odd powers a, a^3, ...,
// a^15: one squaring per bit and one product per window, about nbits / 5 of
// them, where the bit-by-bit power takes one product per set bit.  a below
// 2p; the result is canonical (a^0 = 1, 0^e = 0 for e > 0).
__device__ __forceinline__ fp fp_pow_ool(const fp& a, const uint64_t* e, int nbits) {
    fp odd[8];
    odd[0] = a;
    const fp a2 = fp_sqr_ool(a);
    for (int k = 1; k < 8; ++k) odd[k] = fp_mul_ool(odd[k - 1], a2);
    auto bit = [&](int i) { return (int)((e[i >> 6] >> (i & 63)) & 1u); };
    fp r = fp_one();
    bool started = false;
    for (int i = nbits - 1; i >= 0;) {
        if (!bit(i)) {
            if (started) r = fp_sqr_ool(r);
            --i;
            continue;
        }
        int j = i >= 3 ? i - 3 : 0;                  // the window [j, i] ends on a set bit
        while (!bit(j)) ++j;
        int v = 0;
        for (int k = i; k >= j; --k) {
            v = (v << 1) | bit(k);
            if (started) r = fp_sqr_ool(r);
        }
        r = started ? fp_mul_ool(r, odd[v >> 1]) : odd[v >> 1];
        started = true;
        i = j - 1;
    }
    return r;
}

}  // namespace bls
