// Interpreter of the generated tower programs (programs.inc) for the
// lane-parallel verify kernel.
//
// T lanes own one pairing.  A program is a list of rounds; in a round each of
// the first `nops` lanes executes one operation:
//   MUL  dst = REDC(A * B), each operand one slot or a signed sum of slots
//   LIN  dst = reduced signed sum of slots
//   INV  dst = src^(p-2)
// then the pairing's lanes meet at __syncwarp.  All pairings of a warp run the
// same program, so a round is one uniform instruction stream.
//
// Slot values are integers below 8p (a redundant form of the field element,
// congruent mod p); see gen_programs.py for the bounds.  A signed sum of k
// units starts from (negative units) * (8p + 1), adds each unit's limbs,
// complemented for a negative unit, into a 13-limb accumulator, and subtracts
// QP[acc >> 381] (a multiple of p just below acc), leaving a value below 2.3p.
#pragma once
#include "fp.cuh"
#include "programs.inc"

namespace bls {
namespace vm {

constexpr int kSlotBytes = 48;
constexpr int kKSlots = 8;          // block-shared constants: 0, 1, Frobenius k1, k2, k12
constexpr int kGroups = 8;          // Fp12 groups per pairing
constexpr int kGroupSlots = 12;

// bases: 8 slot indices (16 bits each) packed in four words
struct Bases { uint32_t w01, w23, w45, w67; };

__device__ __forceinline__ uint32_t base_of(const Bases& b, uint32_t k) {
    uint32_t w = (k & 4) ? ((k & 2) ? b.w67 : b.w45) : ((k & 2) ? b.w23 : b.w01);
    return (w >> ((k & 1) << 4)) & 0xffffu;
}
__device__ __forceinline__ uint32_t slot_of(const Bases& b, uint32_t r) {
    return base_of(b, r >> 5) + (r & 31);
}

__device__ __forceinline__ fp load_slot(const uint4* sm, uint32_t s) {
    uint4 a = sm[3 * s], b = sm[3 * s + 1], c = sm[3 * s + 2];
    fp r;
    r.w[0] = a.x; r.w[1] = a.y; r.w[2] = a.z; r.w[3] = a.w;
    r.w[4] = b.x; r.w[5] = b.y; r.w[6] = b.z; r.w[7] = b.w;
    r.w[8] = c.x; r.w[9] = c.y; r.w[10] = c.z; r.w[11] = c.w;
    return r;
}
__device__ __forceinline__ void store_slot(uint4* sm, uint32_t s, const fp& v) {
    sm[3 * s] = make_uint4(v.w[0], v.w[1], v.w[2], v.w[3]);
    sm[3 * s + 1] = make_uint4(v.w[4], v.w[5], v.w[6], v.w[7]);
    sm[3 * s + 2] = make_uint4(v.w[8], v.w[9], v.w[10], v.w[11]);
}

// (8p + 1) * k for k = 0..8, 13 limbs: the offset of a sum with k negative units
__device__ __forceinline__ void sum_offset(uint32_t* acc, uint32_t k) {
    // 8p = 0xd0088f51cbff34d2 58dd3db21a5d66bb 23ba5c279c2895fb 39869507b587b120 f55ffff58a9ffffd cff7fffffffd5558
    const uint32_t e[12] = {0xfffd5558u, 0xcff7ffffu, 0x8a9ffffdu, 0xf55ffff5u, 0xb587b120u, 0x39869507u,
                            0x9c2895fbu, 0x23ba5c27u, 0x1a5d66bbu, 0x58dd3db2u, 0xcbff34d2u, 0xd0088f51u};
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint64_t v = (uint64_t)e[i] * k + c + (i == 0 ? k : 0);
        acc[i] = (uint32_t)v;
        c = (uint32_t)(v >> 32);
    }
    acc[12] = c;
}

// acc += v ^ m  (13 limbs; v's 13th limb is 0, so its complement is m)
__device__ __forceinline__ void acc_add(uint32_t* acc, const fp& v, uint32_t m) {
    asm("add.cc.u32 %0, %0, %13;\n\t"
        "addc.cc.u32 %1, %1, %14;\n\t"
        "addc.cc.u32 %2, %2, %15;\n\t"
        "addc.cc.u32 %3, %3, %16;\n\t"
        "addc.cc.u32 %4, %4, %17;\n\t"
        "addc.cc.u32 %5, %5, %18;\n\t"
        "addc.cc.u32 %6, %6, %19;\n\t"
        "addc.cc.u32 %7, %7, %20;\n\t"
        "addc.cc.u32 %8, %8, %21;\n\t"
        "addc.cc.u32 %9, %9, %22;\n\t"
        "addc.cc.u32 %10, %10, %23;\n\t"
        "addc.cc.u32 %11, %11, %24;\n\t"
        "addc.u32 %12, %12, %25;"
        : BLS_T13(acc)
        : "r"(v.w[0] ^ m), "r"(v.w[1] ^ m), "r"(v.w[2] ^ m), "r"(v.w[3] ^ m), "r"(v.w[4] ^ m),
          "r"(v.w[5] ^ m), "r"(v.w[6] ^ m), "r"(v.w[7] ^ m), "r"(v.w[8] ^ m), "r"(v.w[9] ^ m),
          "r"(v.w[10] ^ m), "r"(v.w[11] ^ m), "r"(m));
}

// acc (< 2^388) -> acc - QP[acc >> 381] (< 2.3p)
__device__ __forceinline__ fp acc_reduce(const uint32_t* acc) {
    uint32_t h = (acc[12] << 3) | (acc[11] >> 29);
    const uint4* q = reinterpret_cast<const uint4*>(prog::kQP[h]);
    uint4 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3);
    fp r;
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
        : "=r"(r.w[0]), "=r"(r.w[1]), "=r"(r.w[2]), "=r"(r.w[3]), "=r"(r.w[4]), "=r"(r.w[5]),
          "=r"(r.w[6]), "=r"(r.w[7]), "=r"(r.w[8]), "=r"(r.w[9]), "=r"(r.w[10]), "=r"(r.w[11]), "=r"(top)
        : "r"(acc[0]), "r"(acc[1]), "r"(acc[2]), "r"(acc[3]), "r"(acc[4]), "r"(acc[5]), "r"(acc[6]),
          "r"(acc[7]), "r"(acc[8]), "r"(acc[9]), "r"(acc[10]), "r"(acc[11]), "r"(acc[12]),
          "r"(q0.x), "r"(q0.y), "r"(q0.z), "r"(q0.w), "r"(q1.x), "r"(q1.y), "r"(q1.z), "r"(q1.w),
          "r"(q2.x), "r"(q2.y), "r"(q2.z), "r"(q2.w), "r"(q3.x));
    (void)top;  // zero: acc - QP[h] < 2^384
    return r;
}

// signed sum of n unit terms; refs packed 4 per word starting at term `first`
__device__ __forceinline__ fp signed_sum(const uint4* sm, const Bases& bs, uint32_t r0, uint32_t r1,
                                         uint32_t signs, int first, int n) {
    uint32_t acc[13];
    sum_offset(acc, __popc(signs & (((1u << n) - 1u) << first)));
    for (int k = 0; k < n; ++k) {
        int t = first + k;
        uint32_t r = ((t < 4 ? r0 : r1) >> ((t & 3) << 3)) & 0xffu;
        uint32_t m = ((signs >> t) & 1u) ? 0xffffffffu : 0u;
        acc_add(acc, load_slot(sm, slot_of(bs, r)), m);
    }
    return acc_reduce(acc);
}

// x^(p-2) with the redundant multiply (right-to-left over 381 exponent bits)
static __device__ __noinline__ fp inv_redundant(const fp& x) {
    const uint32_t e[12] = {0xffffaaa9u, 0xb9feffffu, 0xb153ffffu, 0x1eabfffeu, 0xf6b0f624u, 0x6730d2a0u,
                            0xf38512bfu, 0x64774b84u, 0x434bacd7u, 0x4b1ba7b6u, 0x397fe69au, 0x1a0111eau};
    fp r = fp_one(), b = x;
    for (int i = 0; i < 381; ++i) {
        if ((e[i >> 5] >> (i & 31)) & 1u) r = fp_mul_redundant(r, b);
        b = fp_mul_redundant(b, b);
    }
    return r;
}

template <int T> __device__ __forceinline__ const uint32_t* prog_table(int pid);
template <int T> __device__ __forceinline__ const uint32_t* round_table(uint32_t r);
template <int T> __device__ __forceinline__ const uint32_t* op_table(uint32_t o);
#define BLS_VM_TABLES(TT)                                                                          \
    template <> __device__ __forceinline__ const uint32_t* prog_table<TT>(int pid) {               \
        return prog::kProgT##TT[pid];                                                              \
    }                                                                                              \
    template <> __device__ __forceinline__ const uint32_t* round_table<TT>(uint32_t r) {           \
        return prog::kRoundT##TT[r];                                                               \
    }                                                                                              \
    template <> __device__ __forceinline__ const uint32_t* op_table<TT>(uint32_t o) {              \
        return prog::kOpT##TT[o];                                                                  \
    }
BLS_VM_TABLES(1)
BLS_VM_TABLES(2)
BLS_VM_TABLES(4)
BLS_VM_TABLES(8)
#undef BLS_VM_TABLES

template <int T> struct Layout;
#define BLS_VM_LAYOUT(TT)                                                                          \
    template <> struct Layout<TT> {                                                                \
        static constexpr int kTemp = (prog::kMaxTempT##TT + 1) & ~1;                               \
        static constexpr int kSlots = kGroups * kGroupSlots + kTemp;  /* per pairing */            \
    };
BLS_VM_LAYOUT(1)
BLS_VM_LAYOUT(2)
BLS_VM_LAYOUT(4)
BLS_VM_LAYOUT(8)
#undef BLS_VM_LAYOUT

// run program `pid` for the calling lane (0 <= lane < T) of its pairing
// One out-of-line copy per T: the drivers call it from some forty sites, and
// inlining a multiply into each would overflow the instruction cache.
template <int T>
__device__ __noinline__ void run(int pid, uint4* sm, Bases bs, int lane) {
    const uint32_t* pt = prog_table<T>(pid);
    uint32_t first = __ldg(pt), count = __ldg(pt + 1);
    for (uint32_t r = first; r < first + count; ++r) {
        const uint32_t* rt = round_table<T>(r);
        uint32_t hdr = __ldg(rt), op0 = __ldg(rt + 1);
        uint32_t kind = hdr & 0xffu, nops = (hdr >> 8) & 0xffu, na = (hdr >> 16) & 0xffu, nb = hdr >> 24;
        if ((uint32_t)lane < nops) {
            const uint32_t* op = op_table<T>(op0 + lane);
            uint32_t w0 = __ldg(op), r0 = __ldg(op + 1), r1 = __ldg(op + 2);
            uint32_t dst = slot_of(bs, w0 & 0xffu), signs = w0 >> 8;
            fp v;
            if (kind == 0) {
                fp x = na == 1 ? load_slot(sm, slot_of(bs, r0 & 0xffu)) : signed_sum(sm, bs, r0, r1, signs, 0, na);
                uint32_t rb = ((na < 4 ? r0 : r1) >> ((na & 3) << 3)) & 0xffu;
                fp y = nb == 1 ? load_slot(sm, slot_of(bs, rb)) : signed_sum(sm, bs, r0, r1, signs, na, nb);
                v = fp_mul_redundant(x, y);
            } else if (kind == 1) {
                v = signed_sum(sm, bs, r0, r1, signs, 0, na);
            } else {
                v = inv_redundant(load_slot(sm, slot_of(bs, r0 & 0xffu)));
            }
            store_slot(sm, dst, v);
        }
        __syncwarp();
    }
}

}  // namespace vm
}  // namespace bls
