// Device arithmetic of the Fp2-lane verify kernel (verify_fp2.cu): products
// into double-width accumulators, one Montgomery reduction per output, and
// the QP reduction that keeps every slot below 2^381 + p.  The generator's
// emulator (gen_fp2ops.py) models each routine here bit for bit.
#pragma once
#include "fp.cuh"
#include "fp2ops.inc"
#include "fp_inv.cuh"

namespace bls {
namespace f2 {

// p[0..23] = a * b, schoolbook rows with the CIOS carry chains of fp.cuh.
// After row i the partial product is below 2^(384 + 32 (i + 1)), so the hi
// chain never carries out of p[i + 12].  Row 0 writes p[0..12] outright.
__device__ __forceinline__ void prod24(uint32_t* p, const uint32_t* a, const uint32_t* b) {
    // row 0 writes p[0..12] without reading it: lo products, then the hi chain
#pragma unroll
    for (int j = 0; j < 12; ++j) p[j] = a[j] * b[0];
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
        "madc.hi.u32 %11, %23, %24, 0;"
        : "+r"(p[1]), "+r"(p[2]), "+r"(p[3]), "+r"(p[4]), "+r"(p[5]), "+r"(p[6]), "+r"(p[7]), "+r"(p[8]),
          "+r"(p[9]), "+r"(p[10]), "+r"(p[11]), "=r"(p[12])
        : BLS_A12(a), "r"(b[0]));
#pragma unroll
    for (int i = 13; i < 24; ++i) p[i] = 0;
#pragma unroll
    for (int i = 1; i < 12; ++i) {
        chain_lo(p + i, a, b[i]);
        chain_hi(p + i, a, b[i]);
    }
}

#define BLS_SUB13_12(m, s)                                                                                 \
    asm("sub.cc.u32 %0, %0, %13;\n\t"                                                                     \
        "subc.cc.u32 %1, %1, %14;\n\t"                                                                    \
        "subc.cc.u32 %2, %2, %15;\n\t"                                                                    \
        "subc.cc.u32 %3, %3, %16;\n\t"                                                                    \
        "subc.cc.u32 %4, %4, %17;\n\t"                                                                    \
        "subc.cc.u32 %5, %5, %18;\n\t"                                                                    \
        "subc.cc.u32 %6, %6, %19;\n\t"                                                                    \
        "subc.cc.u32 %7, %7, %20;\n\t"                                                                    \
        "subc.cc.u32 %8, %8, %21;\n\t"                                                                    \
        "subc.cc.u32 %9, %9, %22;\n\t"                                                                    \
        "subc.cc.u32 %10, %10, %23;\n\t"                                                                  \
        "subc.cc.u32 %11, %11, %24;\n\t"                                                                  \
        "subc.u32 %12, %12, 0;"                                                                          \
        : "+r"(m[0]), "+r"(m[1]), "+r"(m[2]), "+r"(m[3]), "+r"(m[4]), "+r"(m[5]), "+r"(m[6]), "+r"(m[7]),  \
          "+r"(m[8]), "+r"(m[9]), "+r"(m[10]), "+r"(m[11]), "+r"(m[12])                                  \
        : "r"((s)[0]), "r"((s)[1]), "r"((s)[2]), "r"((s)[3]), "r"((s)[4]), "r"((s)[5]), "r"((s)[6]),       \
          "r"((s)[7]), "r"((s)[8]), "r"((s)[9]), "r"((s)[10]), "r"((s)[11]))
#define BLS_ADD_MID(p, m)                                                                                    \
    asm("add.cc.u32 %0, %0, %18;\n\t"                                                                     \
        "addc.cc.u32 %1, %1, %19;\n\t"                                                                    \
        "addc.cc.u32 %2, %2, %20;\n\t"                                                                    \
        "addc.cc.u32 %3, %3, %21;\n\t"                                                                    \
        "addc.cc.u32 %4, %4, %22;\n\t"                                                                    \
        "addc.cc.u32 %5, %5, %23;\n\t"                                                                    \
        "addc.cc.u32 %6, %6, %24;\n\t"                                                                    \
        "addc.cc.u32 %7, %7, %25;\n\t"                                                                    \
        "addc.cc.u32 %8, %8, %26;\n\t"                                                                    \
        "addc.cc.u32 %9, %9, %27;\n\t"                                                                    \
        "addc.cc.u32 %10, %10, %28;\n\t"                                                                  \
        "addc.cc.u32 %11, %11, %29;\n\t"                                                                  \
        "addc.cc.u32 %12, %12, %30;\n\t"                                                                  \
        "addc.cc.u32 %13, %13, 0;\n\t"                                                                    \
        "addc.cc.u32 %14, %14, 0;\n\t"                                                                    \
        "addc.cc.u32 %15, %15, 0;\n\t"                                                                    \
        "addc.cc.u32 %16, %16, 0;\n\t"                                                                    \
        "addc.u32 %17, %17, 0;"                                                                          \
        : "+r"((p)[6]), "+r"((p)[7]), "+r"((p)[8]), "+r"((p)[9]), "+r"((p)[10]), "+r"((p)[11]),            \
          "+r"((p)[12]), "+r"((p)[13]), "+r"((p)[14]), "+r"((p)[15]), "+r"((p)[16]), "+r"((p)[17]),        \
          "+r"((p)[18]), "+r"((p)[19]), "+r"((p)[20]), "+r"((p)[21]), "+r"((p)[22]), "+r"((p)[23])         \
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]),         \
          "r"(m[8]), "r"(m[9]), "r"(m[10]), "r"(m[11]), "r"(m[12]))

// t[0..5] += lo(a[0..5] * b), carry into t[6]
__device__ __forceinline__ void chain_lo6(uint32_t* t, const uint32_t* a, uint32_t b) {
    asm("mad.lo.cc.u32 %0, %7, %13, %0;\n\t"
        "madc.lo.cc.u32 %1, %8, %13, %1;\n\t"
        "madc.lo.cc.u32 %2, %9, %13, %2;\n\t"
        "madc.lo.cc.u32 %3, %10, %13, %3;\n\t"
        "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"
        "madc.lo.cc.u32 %5, %12, %13, %5;\n\t"
        "addc.u32 %6, %6, 0;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(b));
}
// t[1..6] += hi(a[0..5] * b); no carry leaves t[6]
__device__ __forceinline__ void chain_hi6(uint32_t* t, const uint32_t* a, uint32_t b) {
    asm("mad.hi.cc.u32 %0, %6, %12, %0;\n\t"
        "madc.hi.cc.u32 %1, %7, %12, %1;\n\t"
        "madc.hi.cc.u32 %2, %8, %12, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"
        "madc.hi.cc.u32 %4, %10, %12, %4;\n\t"
        "madc.hi.u32 %5, %11, %12, %5;"
        : "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(b));
}
// r[0..11] = a[0..5] * b[0..5] (rows as in prod24)
__device__ __forceinline__ void mul6(uint32_t* r, const uint32_t* a, const uint32_t* b) {
#pragma unroll
    for (int j = 0; j < 6; ++j) r[j] = a[j] * b[0];
    asm("mad.hi.cc.u32 %0, %6, %12, %0;\n\t"
        "madc.hi.cc.u32 %1, %7, %12, %1;\n\t"
        "madc.hi.cc.u32 %2, %8, %12, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"
        "madc.hi.cc.u32 %4, %10, %12, %4;\n\t"
        "madc.hi.u32 %5, %11, %12, 0;"
        : "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "=r"(r[6])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(b[0]));
#pragma unroll
    for (int i = 7; i < 12; ++i) r[i] = 0;
#pragma unroll
    for (int i = 1; i < 6; ++i) {
        chain_lo6(r + i, a, b[i]);
        chain_hi6(r + i, a, b[i]);
    }
}

// p[0..23] = a * b by one level of Karatsuba on 6-limb halves: L = a0 b0,
// H = a1 b1, M = (a0 + a1)(b0 + b1) with the halves' carry bits folded in,
// p = L + (M - L - H) 2^192 + H 2^384.  Three 6 x 6 products (216 multiply
// instructions) instead of 288, computed row by row in lockstep (mul6x3); the
// sums and corrections are plain adds.
// three 6 x 6 products r = a b, s = c d, t = e f, row by row in lockstep: the
// three rows of one step are independent carry chains
__device__ __forceinline__ void mul6x3(uint32_t* r, const uint32_t* a, const uint32_t* b, uint32_t* s,
                                       const uint32_t* c, const uint32_t* d, uint32_t* t, const uint32_t* e,
                                       const uint32_t* f) {
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        r[j] = a[j] * b[0];
        s[j] = c[j] * d[0];
        t[j] = e[j] * f[0];
    }
#pragma unroll
    for (int i = 7; i < 12; ++i) r[i] = s[i] = t[i] = 0;
    r[6] = s[6] = t[6] = 0;
    chain_hi6(r, a, b[0]);
    chain_hi6(s, c, d[0]);
    chain_hi6(t, e, f[0]);
#pragma unroll
    for (int i = 1; i < 6; ++i) {
        chain_lo6(r + i, a, b[i]);
        chain_lo6(s + i, c, d[i]);
        chain_lo6(t + i, e, f[i]);
        chain_hi6(r + i, a, b[i]);
        chain_hi6(s + i, c, d[i]);
        chain_hi6(t + i, e, f[i]);
    }
}

__device__ __forceinline__ void prod24k(uint32_t* p, const uint32_t* a, const uint32_t* b) {
    uint32_t sa[6], sb[6], ca, cb;
    asm("add.cc.u32 %0, %7, %13;\n\t"
        "addc.cc.u32 %1, %8, %14;\n\t"
        "addc.cc.u32 %2, %9, %15;\n\t"
        "addc.cc.u32 %3, %10, %16;\n\t"
        "addc.cc.u32 %4, %11, %17;\n\t"
        "addc.cc.u32 %5, %12, %18;\n\t"
        "addc.u32 %6, 0, 0;"
        : "=r"(sa[0]), "=r"(sa[1]), "=r"(sa[2]), "=r"(sa[3]), "=r"(sa[4]), "=r"(sa[5]), "=r"(ca)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]),
          "r"(a[6]), "r"(a[7]), "r"(a[8]), "r"(a[9]), "r"(a[10]), "r"(a[11]));
    asm("add.cc.u32 %0, %7, %13;\n\t"
        "addc.cc.u32 %1, %8, %14;\n\t"
        "addc.cc.u32 %2, %9, %15;\n\t"
        "addc.cc.u32 %3, %10, %16;\n\t"
        "addc.cc.u32 %4, %11, %17;\n\t"
        "addc.cc.u32 %5, %12, %18;\n\t"
        "addc.u32 %6, 0, 0;"
        : "=r"(sb[0]), "=r"(sb[1]), "=r"(sb[2]), "=r"(sb[3]), "=r"(sb[4]), "=r"(sb[5]), "=r"(cb)
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]),
          "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]));
    uint32_t m[13];
    mul6x3(p, a, b, p + 12, a + 6, b + 6, m, sa, sb);
    // + ca sb 2^192 + cb sa 2^192 + ca cb 2^384 (m stays below 2^386)
    const uint32_t ma = 0u - ca, mb = 0u - cb;
    asm("add.cc.u32 %0, %0, %7;\n\t"
        "addc.cc.u32 %1, %1, %8;\n\t"
        "addc.cc.u32 %2, %2, %9;\n\t"
        "addc.cc.u32 %3, %3, %10;\n\t"
        "addc.cc.u32 %4, %4, %11;\n\t"
        "addc.cc.u32 %5, %5, %12;\n\t"
        "addc.u32 %6, %13, 0;"
        : "+r"(m[6]), "+r"(m[7]), "+r"(m[8]), "+r"(m[9]), "+r"(m[10]), "+r"(m[11]), "=r"(m[12])
        : "r"(sb[0] & ma), "r"(sb[1] & ma), "r"(sb[2] & ma), "r"(sb[3] & ma), "r"(sb[4] & ma), "r"(sb[5] & ma),
          "r"(ca & cb));
    asm("add.cc.u32 %0, %0, %7;\n\t"
        "addc.cc.u32 %1, %1, %8;\n\t"
        "addc.cc.u32 %2, %2, %9;\n\t"
        "addc.cc.u32 %3, %3, %10;\n\t"
        "addc.cc.u32 %4, %4, %11;\n\t"
        "addc.cc.u32 %5, %5, %12;\n\t"
        "addc.u32 %6, %6, 0;"
        : "+r"(m[6]), "+r"(m[7]), "+r"(m[8]), "+r"(m[9]), "+r"(m[10]), "+r"(m[11]), "+r"(m[12])
        : "r"(sa[0] & mb), "r"(sa[1] & mb), "r"(sa[2] & mb), "r"(sa[3] & mb), "r"(sa[4] & mb), "r"(sa[5] & mb));
    // m -= L, m -= H: a0 b1 + a1 b0, below 2^385
    BLS_SUB13_12(m, p);
    BLS_SUB13_12(m, p + 12);
    // p[6..23] += m[0..12]
    BLS_ADD_MID(p, m);
}

// acc[12..25] += x (neg = 0) or -= x (neg = 1): acc += +-x 2^384, modulo 2^832
__device__ __forceinline__ void acc_add_hi(uint32_t* acc, const uint32_t* x, uint32_t neg) {
    uint32_t c = neg, m = 0u - neg;
#pragma unroll
    for (int i = 0; i < 14; ++i) {
        const uint64_t s = (uint64_t)acc[12 + i] + ((i < 12 ? x[i] : 0u) ^ m) + c;
        acc[12 + i] = (uint32_t)s;
        c = (uint32_t)(s >> 32);
    }
}

// acc[0..25] -= p (24 limbs), modulo 2^832
__device__ __forceinline__ void acc_sub(uint32_t* acc, const uint32_t* p) {
    asm("sub.cc.u32 %0, %0, %26;\n\t"
        "subc.cc.u32 %1, %1, %27;\n\t"
        "subc.cc.u32 %2, %2, %28;\n\t"
        "subc.cc.u32 %3, %3, %29;\n\t"
        "subc.cc.u32 %4, %4, %30;\n\t"
        "subc.cc.u32 %5, %5, %31;\n\t"
        "subc.cc.u32 %6, %6, %32;\n\t"
        "subc.cc.u32 %7, %7, %33;\n\t"
        "subc.cc.u32 %8, %8, %34;\n\t"
        "subc.cc.u32 %9, %9, %35;\n\t"
        "subc.cc.u32 %10, %10, %36;\n\t"
        "subc.cc.u32 %11, %11, %37;\n\t"
        "subc.cc.u32 %12, %12, %38;\n\t"
        "subc.cc.u32 %13, %13, %39;\n\t"
        "subc.cc.u32 %14, %14, %40;\n\t"
        "subc.cc.u32 %15, %15, %41;\n\t"
        "subc.cc.u32 %16, %16, %42;\n\t"
        "subc.cc.u32 %17, %17, %43;\n\t"
        "subc.cc.u32 %18, %18, %44;\n\t"
        "subc.cc.u32 %19, %19, %45;\n\t"
        "subc.cc.u32 %20, %20, %46;\n\t"
        "subc.cc.u32 %21, %21, %47;\n\t"
        "subc.cc.u32 %22, %22, %48;\n\t"
        "subc.cc.u32 %23, %23, %49;\n\t"
        "subc.cc.u32 %24, %24, 0;\n\t"
        "subc.u32 %25, %25, 0;"
        : "+r"(acc[0]), "+r"(acc[1]), "+r"(acc[2]), "+r"(acc[3]), "+r"(acc[4]), "+r"(acc[5]), "+r"(acc[6]),
          "+r"(acc[7]), "+r"(acc[8]), "+r"(acc[9]), "+r"(acc[10]), "+r"(acc[11]), "+r"(acc[12]), "+r"(acc[13]),
          "+r"(acc[14]), "+r"(acc[15]), "+r"(acc[16]), "+r"(acc[17]), "+r"(acc[18]), "+r"(acc[19]),
          "+r"(acc[20]), "+r"(acc[21]), "+r"(acc[22]), "+r"(acc[23]), "+r"(acc[24]), "+r"(acc[25])
        : "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]), "r"(p[8]),
          "r"(p[9]), "r"(p[10]), "r"(p[11]), "r"(p[12]), "r"(p[13]), "r"(p[14]), "r"(p[15]), "r"(p[16]),
          "r"(p[17]), "r"(p[18]), "r"(p[19]), "r"(p[20]), "r"(p[21]), "r"(p[22]), "r"(p[23]));
}

// acc[0..25] += p[0..25], modulo 2^832
__device__ __forceinline__ void add26(uint32_t* acc, const uint32_t* p) {
    asm("add.cc.u32 %0, %0, %26;\n\t"
        "addc.cc.u32 %1, %1, %27;\n\t"
        "addc.cc.u32 %2, %2, %28;\n\t"
        "addc.cc.u32 %3, %3, %29;\n\t"
        "addc.cc.u32 %4, %4, %30;\n\t"
        "addc.cc.u32 %5, %5, %31;\n\t"
        "addc.cc.u32 %6, %6, %32;\n\t"
        "addc.cc.u32 %7, %7, %33;\n\t"
        "addc.cc.u32 %8, %8, %34;\n\t"
        "addc.cc.u32 %9, %9, %35;\n\t"
        "addc.cc.u32 %10, %10, %36;\n\t"
        "addc.cc.u32 %11, %11, %37;\n\t"
        "addc.cc.u32 %12, %12, %38;\n\t"
        "addc.cc.u32 %13, %13, %39;\n\t"
        "addc.cc.u32 %14, %14, %40;\n\t"
        "addc.cc.u32 %15, %15, %41;\n\t"
        "addc.cc.u32 %16, %16, %42;\n\t"
        "addc.cc.u32 %17, %17, %43;\n\t"
        "addc.cc.u32 %18, %18, %44;\n\t"
        "addc.cc.u32 %19, %19, %45;\n\t"
        "addc.cc.u32 %20, %20, %46;\n\t"
        "addc.cc.u32 %21, %21, %47;\n\t"
        "addc.cc.u32 %22, %22, %48;\n\t"
        "addc.cc.u32 %23, %23, %49;\n\t"
        "addc.cc.u32 %24, %24, %50;\n\t"
        "addc.u32 %25, %25, %51;"
        : "+r"(acc[0]), "+r"(acc[1]), "+r"(acc[2]), "+r"(acc[3]), "+r"(acc[4]), "+r"(acc[5]), "+r"(acc[6]), "+r"(acc[7]), "+r"(acc[8]), "+r"(acc[9]), "+r"(acc[10]), "+r"(acc[11]), "+r"(acc[12]), "+r"(acc[13]), "+r"(acc[14]), "+r"(acc[15]), "+r"(acc[16]), "+r"(acc[17]), "+r"(acc[18]), "+r"(acc[19]), "+r"(acc[20]), "+r"(acc[21]), "+r"(acc[22]), "+r"(acc[23]), "+r"(acc[24]), "+r"(acc[25])
        : "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]), "r"(p[8]), "r"(p[9]), "r"(p[10]), "r"(p[11]), "r"(p[12]), "r"(p[13]), "r"(p[14]), "r"(p[15]), "r"(p[16]), "r"(p[17]), "r"(p[18]), "r"(p[19]), "r"(p[20]), "r"(p[21]), "r"(p[22]), "r"(p[23]), "r"(p[24]), "r"(p[25]));
}

// acc[0..25] += p (24 limbs), modulo 2^832
__device__ __forceinline__ void acc_plus(uint32_t* acc, const uint32_t* p) {
    asm("add.cc.u32 %0, %0, %26;\n\t"
        "addc.cc.u32 %1, %1, %27;\n\t"
        "addc.cc.u32 %2, %2, %28;\n\t"
        "addc.cc.u32 %3, %3, %29;\n\t"
        "addc.cc.u32 %4, %4, %30;\n\t"
        "addc.cc.u32 %5, %5, %31;\n\t"
        "addc.cc.u32 %6, %6, %32;\n\t"
        "addc.cc.u32 %7, %7, %33;\n\t"
        "addc.cc.u32 %8, %8, %34;\n\t"
        "addc.cc.u32 %9, %9, %35;\n\t"
        "addc.cc.u32 %10, %10, %36;\n\t"
        "addc.cc.u32 %11, %11, %37;\n\t"
        "addc.cc.u32 %12, %12, %38;\n\t"
        "addc.cc.u32 %13, %13, %39;\n\t"
        "addc.cc.u32 %14, %14, %40;\n\t"
        "addc.cc.u32 %15, %15, %41;\n\t"
        "addc.cc.u32 %16, %16, %42;\n\t"
        "addc.cc.u32 %17, %17, %43;\n\t"
        "addc.cc.u32 %18, %18, %44;\n\t"
        "addc.cc.u32 %19, %19, %45;\n\t"
        "addc.cc.u32 %20, %20, %46;\n\t"
        "addc.cc.u32 %21, %21, %47;\n\t"
        "addc.cc.u32 %22, %22, %48;\n\t"
        "addc.cc.u32 %23, %23, %49;\n\t"
        "addc.cc.u32 %24, %24, 0;\n\t"
        "addc.u32 %25, %25, 0;"
        : "+r"(acc[0]), "+r"(acc[1]), "+r"(acc[2]), "+r"(acc[3]), "+r"(acc[4]), "+r"(acc[5]), "+r"(acc[6]),
          "+r"(acc[7]), "+r"(acc[8]), "+r"(acc[9]), "+r"(acc[10]), "+r"(acc[11]), "+r"(acc[12]), "+r"(acc[13]),
          "+r"(acc[14]), "+r"(acc[15]), "+r"(acc[16]), "+r"(acc[17]), "+r"(acc[18]), "+r"(acc[19]),
          "+r"(acc[20]), "+r"(acc[21]), "+r"(acc[22]), "+r"(acc[23]), "+r"(acc[24]), "+r"(acc[25])
        : "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]), "r"(p[8]),
          "r"(p[9]), "r"(p[10]), "r"(p[11]), "r"(p[12]), "r"(p[13]), "r"(p[14]), "r"(p[15]), "r"(p[16]),
          "r"(p[17]), "r"(p[18]), "r"(p[19]), "r"(p[20]), "r"(p[21]), "r"(p[22]), "r"(p[23]));
}

// x = 2 x (12 limbs; x below 2^383)
__device__ __forceinline__ void dbl12(uint32_t* x) {
#pragma unroll
    for (int i = 11; i > 0; --i) x[i] = __funnelshift_l(x[i - 1], x[i], 1);
    x[0] <<= 1;
}

// t[0..12] = k * p for a small k (k < 2^32)
__device__ __forceinline__ void set_kp(uint32_t* t, uint32_t k) {
#pragma unroll
    for (int i = 0; i < 13; ++i) t[i] = 0;
    chain_lo_p(t, k);
    chain_hi_p(t, k);
}

// Montgomery reduction of a 26-limb accumulator (value below 2^771):
// r[0..12] = acc / 2^384 mod p, as acc_hi + (acc_lo + M p) / 2^384 (below 2^388).
// The low half is reduced with the CIOS rows of fp.cuh: 12 rows of
// m = t0 * (-p^-1), t += m p, shift, on a 13-limb window.
__device__ __forceinline__ void redc26(uint32_t* r, const uint32_t* acc) {
    uint32_t t[13];
#pragma unroll
    for (int i = 0; i < 12; ++i) t[i] = acc[i];
    t[12] = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint32_t m = t[0] * BLS_NINV;
        chain_lo_p(t, m);
        chain_hi_p(t, m);
#pragma unroll
        for (int j = 0; j < 12; ++j) t[j] = t[j + 1];
        t[12] = 0;
    }
    asm("add.cc.u32 %0, %13, %26;\n\t"
        "addc.cc.u32 %1, %14, %27;\n\t"
        "addc.cc.u32 %2, %15, %28;\n\t"
        "addc.cc.u32 %3, %16, %29;\n\t"
        "addc.cc.u32 %4, %17, %30;\n\t"
        "addc.cc.u32 %5, %18, %31;\n\t"
        "addc.cc.u32 %6, %19, %32;\n\t"
        "addc.cc.u32 %7, %20, %33;\n\t"
        "addc.cc.u32 %8, %21, %34;\n\t"
        "addc.cc.u32 %9, %22, %35;\n\t"
        "addc.cc.u32 %10, %23, %36;\n\t"
        "addc.cc.u32 %11, %24, %37;\n\t"
        "addc.u32 %12, %25, 0;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12])
        : "r"(acc[12]), "r"(acc[13]), "r"(acc[14]), "r"(acc[15]), "r"(acc[16]), "r"(acc[17]), "r"(acc[18]),
          "r"(acc[19]), "r"(acc[20]), "r"(acc[21]), "r"(acc[22]), "r"(acc[23]), "r"(acc[24]),
          "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]), "r"(t[8]),
          "r"(t[9]), "r"(t[10]), "r"(t[11]));
}

// out = v - q (12 limbs; q = QP[v >> 381] in four 16-byte units)
__device__ __forceinline__ void qp_subtract(uint32_t* out, const uint32_t* v, const uint4& q0, const uint4& q1,
                                            const uint4& q2, const uint4& q3) {
    uint32_t top;
    asm("sub.cc.u32 %0, %13, %26;\n\t"
        "subc.cc.u32 %1, %14, %27;\n\t"
        "subc.cc.u32 %2, %15, %28;\n\t"
        "subc.cc.u32 %3, %16, %29;\n\t"
        "subc.cc.u32 %4, %17, %30;\n\t"
        "subc.cc.u32 %5, %18, %31;\n\t"
        "subc.cc.u32 %6, %19, %32;\n\t"
        "subc.cc.u32 %7, %20, %33;\n\t"
        "subc.cc.u32 %8, %21, %34;\n\t"
        "subc.cc.u32 %9, %22, %35;\n\t"
        "subc.cc.u32 %10, %23, %36;\n\t"
        "subc.cc.u32 %11, %24, %37;\n\t"
        "subc.u32 %12, %25, %38;"
        : "=r"(out[0]), "=r"(out[1]), "=r"(out[2]), "=r"(out[3]), "=r"(out[4]), "=r"(out[5]), "=r"(out[6]),
          "=r"(out[7]), "=r"(out[8]), "=r"(out[9]), "=r"(out[10]), "=r"(out[11]), "=r"(top)
        : "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
          "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(q0.x), "r"(q0.y), "r"(q0.z), "r"(q0.w), "r"(q1.x),
          "r"(q1.y), "r"(q1.z), "r"(q1.w), "r"(q2.x), "r"(q2.y), "r"(q2.z), "r"(q2.w), "r"(q3.x));
    (void)top;  // zero: v - QP[h] < 2^384
}

// v (13 limbs, below 2^388) -> v - QP[v >> 381], below 2^381 + p (12 limbs)
__device__ __forceinline__ void qp_reduce(uint32_t* out, const uint32_t* v) {
    const uint32_t h = (v[12] << 3) | (v[11] >> 29);
    const uint4* q = reinterpret_cast<const uint4*>(kQP2[h & 127]);
    qp_subtract(out, v, __ldg(q), __ldg(q + 1), __ldg(q + 2), __ldg(q + 3));
}

// the same with the QP table copied into shared memory, unit j of entry e at
// tab[128 j + e] (lanes reading different entries then spread over the banks)
__device__ __forceinline__ void qp_reduce_tab(uint32_t* out, const uint32_t* v, const uint4* tab) {
    const uint32_t h = ((v[12] << 3) | (v[11] >> 29)) & 127u;
    qp_subtract(out, v, tab[h], tab[128 + h], tab[256 + h], tab[384 + h]);
}

// t[0..12] += c x (x: 12 limbs, |c| < 2^31), modulo 2^416: y = |c| x by
// shifts for |c| <= 2 (the common 1 and 2 of the programs' linear terms) or
// by one multiply chain, then one add chain of y or of its complement (no
// branch on the sign, which differs between lanes)
__device__ __forceinline__ void madd13(uint32_t* t, const uint32_t* x, int c) {
    const uint32_t a = (uint32_t)(c < 0 ? -c : c), m = c < 0 ? 0xffffffffu : 0u;
    uint32_t y[13];
    if (a <= 2u) {
#pragma unroll
        for (int i = 0; i < 12; ++i) y[i] = x[i];
        y[12] = 0;
        if (a == 2u) {
            y[12] = x[11] >> 31;
#pragma unroll
            for (int i = 11; i > 0; --i) y[i] = __funnelshift_l(x[i - 1], x[i], 1);
            y[0] = x[0] << 1;
        } else if (a == 0u) {
            return;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 13; ++i) y[i] = 0;
        chain_lo(y, x, a);
        chain_hi(y, x, a);
    }
    uint32_t cf;   // carry in = 1 for a subtraction: m + m carries out exactly when m is all ones
    asm("add.cc.u32 %13, %27, %27;\n\t"
        "addc.cc.u32 %0, %0, %14;\n\t"
        "addc.cc.u32 %1, %1, %15;\n\t"
        "addc.cc.u32 %2, %2, %16;\n\t"
        "addc.cc.u32 %3, %3, %17;\n\t"
        "addc.cc.u32 %4, %4, %18;\n\t"
        "addc.cc.u32 %5, %5, %19;\n\t"
        "addc.cc.u32 %6, %6, %20;\n\t"
        "addc.cc.u32 %7, %7, %21;\n\t"
        "addc.cc.u32 %8, %8, %22;\n\t"
        "addc.cc.u32 %9, %9, %23;\n\t"
        "addc.cc.u32 %10, %10, %24;\n\t"
        "addc.cc.u32 %11, %11, %25;\n\t"
        "addc.u32 %12, %12, %26;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
          "+r"(t[8]), "+r"(t[9]), "+r"(t[10]), "+r"(t[11]), "+r"(t[12]), "=r"(cf)
        : "r"(y[0] ^ m), "r"(y[1] ^ m), "r"(y[2] ^ m), "r"(y[3] ^ m), "r"(y[4] ^ m), "r"(y[5] ^ m), "r"(y[6] ^ m),
          "r"(y[7] ^ m), "r"(y[8] ^ m), "r"(y[9] ^ m), "r"(y[10] ^ m), "r"(y[11] ^ m), "r"(y[12] ^ m), "r"(m));
    (void)cf;
}

// r = a + b (12 limbs, no carry out: both below 2^383)
__device__ __forceinline__ void add12(uint32_t* r, const uint32_t* a, const uint32_t* b) {
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
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
        : BLS_A12(a), BLS_A12(b));
}

// r = a + 3p - b (12 limbs; a, b below 2^381 + p, result below 2^384)
__device__ __forceinline__ void add3p_sub(uint32_t* r, const uint32_t* a, const uint32_t* b) {
    uint32_t s[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) s[i] = k3P[i];
    add12(s, s, a);
    asm("sub.cc.u32 %0, %12, %24;\n\t"
        "subc.cc.u32 %1, %13, %25;\n\t"
        "subc.cc.u32 %2, %14, %26;\n\t"
        "subc.cc.u32 %3, %15, %27;\n\t"
        "subc.cc.u32 %4, %16, %28;\n\t"
        "subc.cc.u32 %5, %17, %29;\n\t"
        "subc.cc.u32 %6, %18, %30;\n\t"
        "subc.cc.u32 %7, %19, %31;\n\t"
        "subc.cc.u32 %8, %20, %32;\n\t"
        "subc.cc.u32 %9, %21, %33;\n\t"
        "subc.cc.u32 %10, %22, %34;\n\t"
        "subc.u32 %11, %23, %35;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
        : BLS_A12(s), BLS_A12(b));
}

}  // namespace f2
}  // namespace bls
