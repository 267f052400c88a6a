// Fp2-lane verify kernel: twelve threads per verification in two halves (the
// two warps of a block), thread (k, h) working on the k-th Fp2 coefficient of
// every Fp12 result from the generated descriptors (fp2ops.inc,
// gen_fp2ops.py), with lazy reduction: all the Fp2 products that feed one
// coefficient are summed exactly in two 832-bit accumulators and reduced once.
// The products of a coefficient are split between the halves; half h sums its
// share, hands the other component's partial sum to its partner through
// shared memory, and reduces component h (0: real, 1: imaginary).  Five
// verifications per block (lanes 30 and 31 of each warp idle).
//
// Per verification (gpu-crypto/cuda/api.cu:80-91, api.cu:30-52, api.cu:65-78):
//   Miller loop   for each of the 68 line coefficients: both pairs'
//                 coefficients go to the C area, LSCALE forms c1 P.x and c0 P.y,
//                 LINE1 and LINE2 multiply f by the two lines; 62 SQR in
//                 between; CONJ at the end (x < 0)
//   final exp     the reference's chain over 7 Fp12 groups, the inverse in 8
//                 steps with an extended-Euclid Fp inverse on one thread
//   result        canonical Gt compared with 1; optional Miller / Gt outputs
//
// Shared memory: 8 block-shared constant slots (0, 1, Frobenius constants),
// then per pairing kGroups groups of 6 Fp2 slots and a 12-slot C area (lines,
// points), then the exchange area (per pairing and coefficient, one 26-word
// partial sum per half), per-pairing flags and the table of k p for the
// outputs' bias multiples.  An Fp2 slot is 24 words: re
// then im, each below 2^381 + p.  Every program accumulates, exchanges, meets,
// reduces, meets, writes and meets again, so a program may overwrite its own
// inputs.
#include <cuda_runtime.h>

#include "fp2ops.cuh"
#include "g1.cuh"
#include "internal.h"

namespace bls {
namespace {

constexpr int kLanes = 6;
constexpr int kPairsPerBlock = 5;
constexpr int kThreads = 64;                    // two halves of 32
constexpr int kGroups = f2::kGroupsUsed;
constexpr int kCOff = 6 * kGroups;              // C area after the groups
constexpr int kPairSlots = kCOff + 12;          // Fp2 slots per pairing
constexpr int kKSlots = f2::kKSlotCount;        // block-shared constants
constexpr int kSlotWords = 24;
constexpr int kSlotArea = (kKSlots + kPairsPerBlock * kPairSlots) * kSlotWords;  // words
constexpr int kXchWords = 28;                   // 26 used; 112 B keeps uint4 alignment
constexpr int kXchArea = kPairsPerBlock * kLanes * 2 * kXchWords;                 // words
constexpr int kFlagArea = kPairsPerBlock * 2 + 2;                                // words
constexpr int kKpCount = f2::kMaxBias + 1;      // k p for every bias multiple k, 16 words each
static_assert(kKpCount <= kThreads, "one thread per table entry at start-up");


struct Ctx {
    uint32_t* sm;      // shared memory (words): slots, then exchange, then flags
    uint32_t region;   // first slot of this pairing
    int pair;          // pairing within the block, 0..4 (5 for the idle lanes)
    int lane;          // coefficient 0..5; 6, 7 for the idle lanes 30, 31
    int half;          // warp of the block: 0 or 1
    bool active;       // thread belongs to a pairing
};

// D, A, B, C, K, T: absolute slot of index 0, nine bits each (every slot
// index of a block is below 512), so a reference resolves with a shift, not
// an indexed array
struct Bases { uint64_t b; };
static_assert(kKSlots + kPairsPerBlock * kPairSlots <= 512, "slot indices must fit nine bits");

__device__ __forceinline__ uint32_t grp(const Ctx& c, int g) { return c.region + 6 * g; }

__device__ __forceinline__ uint32_t slot_addr(const Bases& bs, uint32_t ref) {
    return (uint32_t)(bs.b >> (9u * (ref >> 4))) % 512u + (ref & 15u);
}

__device__ __forceinline__ void load_fp(uint32_t* x, const uint32_t* sm, uint32_t slot, int comp) {
    const uint4* s = reinterpret_cast<const uint4*>(sm + kSlotWords * slot + 12 * comp);
    uint4 a = s[0], b = s[1], c = s[2];
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    x[8] = c.x; x[9] = c.y; x[10] = c.z; x[11] = c.w;
}
__device__ __forceinline__ void store_fp(uint32_t* sm, uint32_t slot, int comp, const uint32_t* x) {
    uint4* s = reinterpret_cast<uint4*>(sm + kSlotWords * slot + 12 * comp);
    s[0] = make_uint4(x[0], x[1], x[2], x[3]);
    s[1] = make_uint4(x[4], x[5], x[6], x[7]);
    s[2] = make_uint4(x[8], x[9], x[10], x[11]);
}

// t[0..12] = k p from the block's table (16 words per entry, filled at the
// kernel's start; k <= kMaxBias for every descriptor the generator writes)
__device__ __forceinline__ void load_kp(uint32_t* t, const uint32_t* sm, uint32_t k) {
    const uint32_t* e = sm + kSlotArea + kXchArea + kFlagArea + 16 * k;
    const uint4* v = reinterpret_cast<const uint4*>(e);
    const uint4 a = v[0], b = v[1], c = v[2];
    t[0] = a.x; t[1] = a.y; t[2] = a.z; t[3] = a.w;
    t[4] = b.x; t[5] = b.y; t[6] = b.z; t[7] = b.w;
    t[8] = c.x; t[9] = c.y; t[10] = c.z; t[11] = c.w;
    t[12] = e[12];
}

__device__ __forceinline__ int sext4(uint32_t v) { return (int)(v << 28) >> 28; }

// P into the two accumulators with coefficients ca, cb (bit 0 nonzero, bit 1 negative)
__device__ __forceinline__ void acc_pair(uint32_t* acc0, uint32_t* acc1, const uint32_t* P, uint32_t ca,
                                         uint32_t cb) {
    if (ca & 1u) {
        if (ca >> 1) f2::acc_sub(acc0, P);
        else f2::acc_plus(acc0, P);
    }
    if (cb & 1u) {
        if (cb >> 1) f2::acc_sub(acc1, P);
        else f2::acc_plus(acc1, P);
    }
}

// Phase 1 of an output (product modes): this half's products into both
// accumulators, the partner's component (accX) left in the exchange slot.
__device__ __forceinline__ void accumulate(uint32_t off, uint32_t* sm, const Bases& bs, uint32_t* xch_out,
                                           int half, uint32_t* own) {
    const uint32_t hdr = f2::kDesc[off], bias = f2::kDesc[off + 1];
    const uint32_t nt = (hdr >> 2) & 15u;
    // accO: component `half` (reduced by this thread), accX: the other one (sent
    // to the partner); coefficients and biases are swapped for half 1
    uint32_t accO[26], accX[26];
    const uint32_t sw = half ? 8u : 0u, c0 = half ? 12u : 0u, c1 = half ? 0u : 12u;
#pragma unroll
    for (int i = 0; i < 12; ++i) accO[i] = accX[i] = 0;
    accO[25] = accX[25] = 0;
    load_kp(accO + 12, sm, (bias >> sw) & 0xffu);
    load_kp(accX + 12, sm, (bias >> (8u - sw)) & 0xffu);
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t w = f2::kDesc[off + 2 + t];
        const uint32_t kind = w & 7u, xi = (w >> 3) & 1u, neg = (w >> 4) & 1u, dbl = (w >> 5) & 1u,
                       yim = (w >> 6) & 1u, mask = (w >> 24) & 7u;
        const uint32_t xs = slot_addr(bs, (w >> 8) & 0x7fu), ys = slot_addr(bs, (w >> 16) & 0x7fu);
        if (kind == f2::kOne) {             // X R: X into the high half of both accumulators
            uint32_t x0[12], x1[12];
            load_fp(x0, sm, xs, half);
            load_fp(x1, sm, xs, 1 - half);
            f2::acc_add_hi(accO, x0, neg);
            f2::acc_add_hi(accX, x1, neg);
            continue;
        }
        // coefficients in {-1, 0, 1} of product j: bit 0 nonzero, bit 1 negative;
        // (cw >> 4j) for component 0, (cw >> 4(3 + j)) for component 1
        const uint32_t cw = f2::kCoef[2 * kind + xi] ^ (neg ? 0x666666u : 0u);
        // every operand is read from shared memory when its product runs, so
        // one product call site serves every kind and nothing stays live
        // beside the accumulators between products
        const uint32_t np = kind == f2::kKara ? 3u : 2u;
#pragma unroll 1
        for (uint32_t j = 0; j < np; ++j) {
            if (!((mask >> j) & 1u)) continue;
            uint32_t U[12], V[12], P[24];
            if (kind == f2::kSqr) {          // U = x0 + x1, 2 x0
                load_fp(U, sm, xs, 0);
                if (j == 0) {
                    uint32_t T[12];
                    load_fp(T, sm, xs, 1);
                    f2::add12(U, U, T);
                } else {
                    f2::dbl12(U);
                }
            } else if (kind == f2::kKara && xi) {   // xi X = (x0 - x1 + 3p, x0 + x1); sum 2 x0 + 3p
                load_fp(U, sm, xs, 0);
                if (j == 2) {
                    const uint32_t z[12] = {0};
                    f2::dbl12(U);
                    f2::add3p_sub(U, U, z);
                } else {
                    uint32_t T[12];
                    load_fp(T, sm, xs, 1);
                    if (j == 0) f2::add3p_sub(U, U, T);
                    else f2::add12(U, U, T);
                }
            } else {                         // x0, x1 (KARA: sum x0 + x1)
                load_fp(U, sm, xs, j & 1u);
                if (j == 2) {
                    uint32_t T[12];
                    load_fp(T, sm, xs, 1);
                    f2::add12(U, U, T);
                }
            }
            if (kind == f2::kKara) {        // V = y0, y1, y0 + y1 (doubled when dbl)
                load_fp(V, sm, ys, j & 1u);
                if (j == 2) {
                    uint32_t T[12];
                    load_fp(T, sm, ys, 1);
                    f2::add12(V, V, T);
                }
                if (dbl) f2::dbl12(V);
            } else if (kind == f2::kSqr) {  // V = x0 - x1 + 3p, x1
                load_fp(V, sm, xs, 1);
                if (j == 0) {
                    uint32_t T[12];
                    load_fp(T, sm, xs, 0);
                    f2::add3p_sub(V, T, V);
                }
            } else if (kind == f2::kFpMul) {
                load_fp(V, sm, ys, yim);
            } else {                        // NORM: x_j^2
                load_fp(V, sm, xs, j);
            }
            f2::prod24k(P, U, V);
            acc_pair(accO, accX, P, (cw >> (c0 + 4 * j)) & 3u, (cw >> (c1 + 4 * j)) & 3u);
        }
    }
    uint4* x = reinterpret_cast<uint4*>(xch_out);
#pragma unroll
    for (int i = 0; i < 24; i += 4) x[i / 4] = make_uint4(accX[i], accX[i + 1], accX[i + 2], accX[i + 3]);
    xch_out[24] = accX[24];
    xch_out[25] = accX[25];
#pragma unroll
    for (int i = 0; i < 26; ++i) own[i] = accO[i];
}

// Phase 2: component `half` of the output into o (12 words).  own: this
// half's accumulator of that component (product modes), xch_in: the partner's.
__device__ __forceinline__ void finish(uint32_t off, const uint32_t* sm, const Bases& bs, int half, uint32_t* own,
                                       const uint32_t* xch_in, uint32_t* o) {
    const uint32_t hdr = f2::kDesc[off], bias = f2::kDesc[off + 1];
    const uint32_t mode = hdr & 3u, nt = (hdr >> 2) & 15u, nl = (hdr >> 6) & 3u;
    const int cc = half ? sext4(hdr >> 20) : sext4(hdr >> 16);
    const uint32_t bias_lin = (bias >> (16 + 8 * half)) & 0xffu;
    const uint32_t* lin = f2::kDesc + off + 2 + nt;

    if (mode == f2::kModeInvFp) {
        if (half == 0) {
            fp z;
            load_fp(z.w, sm, slot_addr(bs, lin[0] >> 8), 0);
            fp r = fp_inverse_mont(z, f2::kR3);
#pragma unroll
            for (int i = 0; i < 12; ++i) o[i] = r.w[i];
        } else {
#pragma unroll
            for (int i = 0; i < 12; ++i) o[i] = 0;
        }
        return;
    }
    uint32_t r[13];
    if (mode == f2::kModeLin) {
        load_kp(r, sm, bias_lin);
        for (uint32_t j = 0; j < nl; ++j) {
            uint32_t z[12];
            load_fp(z, sm, slot_addr(bs, lin[j] >> 8), half);
            f2::madd13(r, z, cc * sext4(lin[j]));
        }
    } else {
        // own += partner's partial sum (26 limbs, modulo 2^832)
        uint32_t p[26];
        const uint4* x = reinterpret_cast<const uint4*>(xch_in);
#pragma unroll
        for (int i = 0; i < 24; i += 4) {
            const uint4 q = x[i / 4];
            p[i] = q.x; p[i + 1] = q.y; p[i + 2] = q.z; p[i + 3] = q.w;
        }
        p[24] = xch_in[24];
        p[25] = xch_in[25];
        f2::add26(own, p);
        uint32_t red[13];
        f2::redc26(red, own);
        if (mode == f2::kModeSimple) {
            f2::qp_reduce(o, red);
            return;
        }
        uint32_t q[12];
        f2::qp_reduce(q, red);
        load_kp(r, sm, bias_lin);
        f2::madd13(r, q, cc);
        for (uint32_t j = 0; j < nl; ++j) {
            uint32_t z[12];
            load_fp(z, sm, slot_addr(bs, lin[j] >> 8), half);
            f2::madd13(r, z, sext4(lin[j]));
        }
    }
    f2::qp_reduce(o, r);
}

// run program `pid` on the pairing: accumulate, exchange, meet, reduce,
// write, meet.  No program of the generated sequences writes a slot that it
// reads (gen_fp2ops.py places the results), so the outputs are stored as soon
// as they are reduced.  Every thread of the block takes part in every
// barrier.  It has one call site (the op loop of the kernel), so it is
// inlined there.
__device__ __forceinline__ void run(int pid, uint32_t* sm, int pair, int lane, int half, const Bases& bs) {
    const bool active = pair < kPairsPerBlock;
    const uint32_t off = active ? f2::kOutIndex[pid][8 * half + lane] : 0xffffu;
    const uint32_t mode = off != 0xffffu ? (f2::kDesc[off] & 3u) : 0u;
    const bool prod = off != 0xffffu && (mode == f2::kModeSimple || mode == f2::kModeFull);
    uint32_t* xch = sm + kSlotArea + ((active ? pair : 0) * kLanes + (active ? lane % kLanes : 0)) * 2 * kXchWords;
    uint32_t own[26];
    if (prod) accumulate(off, sm, bs, xch + kXchWords * half, half, own);
    __syncthreads();
    uint32_t o[12];
    if (off != 0xffffu) finish(off, sm, bs, half, own, xch + kXchWords * (1 - half), o);
    if (off != 0xffffu) store_fp(sm, slot_addr(bs, (f2::kDesc[off] >> 8) & 0x7fu), half, o);
    __syncthreads();
}

__device__ __forceinline__ void copy_fp_from_global(uint32_t* sm, uint32_t slot, int comp, const uint64_t* src) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(sm + kSlotWords * slot + 12 * comp);
    d[0] = __ldg(s);
    d[1] = __ldg(s + 1);
    d[2] = __ldg(s + 2);
}

// line coefficient `ci` of both pairs into the C area (thread (k, h): pair
// k / 3, coefficient k % 3, component h).  A skipped pair gets the line
// (0, 0, 1), which leaves f unchanged.
__device__ __forceinline__ void load_lines(const Ctx& c, const uint64_t* q1, bool skip1, const uint64_t* q2,
                                           bool skip2, int ci) {
    if (c.active) {
        const int pair = c.lane / 3, k = c.lane % 3;
        const uint64_t* q = pair ? q2 : q1;
        const bool skip = pair ? skip2 : skip1;
        const uint32_t slot = c.region + kCOff + 6 * pair + k;
        if (skip) {
            fp v = (k == 2 && c.half == 0) ? fp_one() : fp_zero();
            store_fp(c.sm, slot, c.half, v.w);
        } else {
            copy_fp_from_global(c.sm, slot, c.half, q + 36 * ci + 12 * k + 6 * c.half);
        }
    }
    __syncthreads();
}

// canonical form of a slot value (below 2^381 + p < 3p)
__device__ __forceinline__ fp canonical(fp v) {
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        uint32_t d[12];
        uint32_t br = sub_p(d, v.w);
#pragma unroll
        for (int i = 0; i < 12; ++i) v.w[i] = br ? v.w[i] : d[i];
    }
    return v;
}

// canonical group `g` -> out (72 u64) and the "is one" test over the
// pairing's twelve threads (a flag per pairing and half in shared memory)
__device__ __forceinline__ bool emit_group(const Ctx& c, int g, uint64_t* out) {
    bool ok = true;
    if (c.active) {
        fp v;
        load_fp(v.w, c.sm, grp(c, g) + c.lane, c.half);
        v = canonical(v);
        if (out) fp_store_u64(out + 12 * c.lane + 6 * c.half, v);
        ok = (c.lane == 0 && c.half == 0) ? fp_eq(v, fp_one()) : fp_is_zero(v);
    }
    const unsigned bad = __ballot_sync(0xffffffffu, !ok);
    uint32_t* flags = c.sm + kSlotArea + kXchArea;
    if (c.active && c.lane == 0) {
        const unsigned first = (threadIdx.x & 31u);
        flags[2 * c.pair + c.half] = (bad >> first) & 0x3fu;
    }
    __syncthreads();
    const bool one = c.active && (flags[2 * c.pair] | flags[2 * c.pair + 1]) == 0;
    __syncthreads();
    return one;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// the published count with acquire semantics at GPU scope: the ring items
// that the host's copies wrote before the count are visible to this thread's
// later loads (and, through the block barrier that follows the claim, to the
// block's other threads)
__device__ __forceinline__ uint32_t ld_acquire_gpu(const volatile uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Ring serving, thread 0 of a block: claim the next published group of five
// items (all in device memory).  False when the block should leave: the stop
// flag, serve_idle_ns in which the published count did not move (idle for the
// whole kernel, not just for this block: a block that loses claims to others
// while work keeps arriving stays), or serve_max_ns after the launch; the loop
// also has an iteration cap, so every wait ends.
__device__ bool serve_claim(const VerifyArgs& a, uint64_t t_launch, uint32_t* base) {
    uint64_t t_moved = globaltimer_ns();
    uint32_t seen = ld_acquire_gpu(a.serve_avail);
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        const uint32_t cur = *reinterpret_cast<volatile uint32_t*>(a.serve_claimed);
        const uint32_t av = ld_acquire_gpu(a.serve_avail);
        if ((int32_t)(av - cur) > 0) {
            if (atomicCAS(a.serve_claimed, cur, cur + kPairsPerBlock) == cur) {
                // order the claimed group's input loads after the count that
                // published it
                __threadfence();
                *base = cur;
                return true;
            }
            continue;
        }
        const uint64_t now = globaltimer_ns();
        if (av != seen) {
            seen = av;
            t_moved = now;
        }
        if (*a.serve_stop || now - t_moved > a.serve_idle_ns || now - t_launch > a.serve_max_ns) return false;
        __nanosleep(500);
    }
    return false;
}

// 6 x u64 read at L2 (not L1): a serving ring rewrites its slots by copies
__device__ __forceinline__ fp fp_load_u64_cg(const uint64_t* v) {
    fp r;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const unsigned long long x = __ldcg(reinterpret_cast<const unsigned long long*>(v) + i);
        r.w[2 * i] = (uint32_t)x;
        r.w[2 * i + 1] = (uint32_t)(x >> 32);
    }
    return r;
}

__global__ void __launch_bounds__(kThreads, 6) k_verify_fp2(VerifyArgs a, const uint32_t* __restrict__ in_status) {
    extern __shared__ uint4 smem4[];
    uint32_t* sm = reinterpret_cast<uint32_t*>(smem4);
    const int half = threadIdx.x >> 5, lane32 = threadIdx.x & 31;
    const int pi = lane32 / kLanes;

    for (int i = threadIdx.x; i < kKSlots * kSlotWords; i += blockDim.x) sm[i] = f2::kKSlots[i / kSlotWords][i % kSlotWords];
    if (threadIdx.x < kKpCount) {
        uint32_t t[13];
        f2::set_kp(t, threadIdx.x);
#pragma unroll
        for (int i = 0; i < 13; ++i) sm[kSlotArea + kXchArea + kFlagArea + 16 * threadIdx.x + i] = t[i];
    }
    __syncthreads();

    Ctx c;
    c.sm = sm;
    c.active = pi < kPairsPerBlock;
    c.pair = pi;
    c.half = half;
    c.lane = c.active ? lane32 % kLanes : 6 + (lane32 & 1);
    c.region = kKSlots + (c.active ? pi : 0) * kPairSlots;
    uint32_t* bcast = sm + kSlotArea + kXchArea + 2 * kPairsPerBlock;
    // normalised line tables (every row divided by its c2) when the caller has them
    const int norm = a.pk_norm != nullptr ? 1 : 0;
    const uint64_t* g2_lines = norm ? a.g2_norm : a.g2;

    int next = blockIdx.x * kPairsPerBlock;
    const int stride = gridDim.x * kPairsPerBlock;
    const bool serving = a.serve_avail != nullptr;
    const uint64_t t_launch = serving ? globaltimer_ns() : 0;
    for (;;) {
        int base;
        if (serving) {
            if (threadIdx.x == 0) {
                uint32_t b = 0;
                const bool go = serve_claim(a, t_launch, &b);
                bcast[0] = b % a.serve_cap;
                bcast[1] = go ? 1u : 0u;
            }
            __syncthreads();
            base = (int)bcast[0];
            const bool go = bcast[1] != 0;
            __syncthreads();
            if (!go) break;
        } else if (a.work_counter) {
            if (threadIdx.x == 0) bcast[0] = (uint32_t)atomicAdd(a.work_counter, kPairsPerBlock);
            __syncthreads();
            base = (int)bcast[0];
            __syncthreads();
        } else {
            base = next;
            next += stride;
        }
        if (!serving && base >= a.n) break;
        const int item = base + (c.active ? pi : 0);
        const bool have = c.active && (serving || item < a.n);
        bool skip1 = true, skip2 = true;
        const uint64_t* pk = g2_lines;
        const uint64_t* pk_cf = a.g2_corr;
        int32_t status = 0;
        if (have) {
            const uint64_t* s = a.sig_xy ? a.sig_xy + 12 * (size_t)item : (const uint64_t*)a.sigs + 12 * (size_t)item;
            const uint64_t* h = a.nhms + 12 * (size_t)item;
            if (in_status) status = (int32_t)__ldcg(in_status + item);
            fp sx = fp_load_u64_cg(s), sy = fp_load_u64_cg(s + 6);
            fp hx = fp_load_u64_cg(h), hy = fp_load_u64_cg(h + 6);
            int64_t pki = a.pk_index ? (int64_t)__ldcg(a.pk_index + item) : (int64_t)item;
            if (!key_index_ok(pki, a.check_keys, a.n_keys)) {   // no table read for it
                if (status == 0) status = ST_BAD_KEY_INDEX;
                pki = 0;
            }
            pk = (norm ? a.pk_norm : a.pk_tables) + kCoeffU64 * pki;
            if (norm) pk_cf = a.pk_corr + 12 * pki;
            skip1 = g1_limbs_identity(sx, sy) || status != 0;
            skip2 = g1_limbs_identity(hx, hy) || (a.pk_identity && a.pk_identity[pki]) || status != 0;
            if (c.lane == 0 && c.half == 0) {
                const uint32_t C = c.region + kCOff;
                store_fp(sm, C + 0 * 6 + 3, 0, skip1 ? fp_zero().w : sx.w);
                store_fp(sm, C + 0 * 6 + 3, 1, skip1 ? fp_zero().w : sy.w);
                store_fp(sm, C + 1 * 6 + 3, 0, skip2 ? fp_zero().w : hx.w);
                store_fp(sm, C + 1 * 6 + 3, 1, skip2 ? fp_zero().w : hy.w);
            }
        } else if (c.active && c.lane == 0 && c.half == 0) {
            const uint32_t C = c.region + kCOff;
            for (int pair = 0; pair < 2; ++pair) {
                store_fp(sm, C + pair * 6 + 3, 0, fp_zero().w);
                store_fp(sm, C + pair * 6 + 3, 1, fp_zero().w);
            }
        }
        // f = 1
        if (c.active) store_fp(sm, grp(c, 0) + c.lane, c.half, (c.lane == 0 && c.half == 0) ? fp_one().w : fp_zero().w);
        __syncthreads();

        // the op sequence: Miller loop over |x| >> 1 below its leading bit
        // (api.cu:30-52), then the final exponentiation (api.cu:65-78)
        const int seq_len = norm ? f2::kSeqLenNorm : f2::kSeqLenRaw;
        for (int s = 0; s < seq_len; ++s) {
            const uint32_t e = f2::kSeq[norm][s];
            const uint32_t code = e & 31u;
            if ((e & f2::kCondMl) && !a.ml_out) continue;
            if (code == f2::kOpLoadLines) {
                load_lines(c, g2_lines, skip1, pk, skip2, (int)((e >> 14) & 127u));
            } else if (code == f2::kOpLoadCorr) {
                // the generator's and the key's Miller correction factors into the c2 slots
                if (c.active && c.lane < 2) {
                    const bool skip = c.lane ? skip2 : skip1;
                    const uint64_t* cf = c.lane ? pk_cf : a.g2_corr;
                    const uint32_t slot = c.region + kCOff + 6 * c.lane + 2;
                    if (skip) store_fp(sm, slot, c.half, c.half ? fp_zero().w : fp_one().w);
                    else copy_fp_from_global(sm, slot, c.half, cf + 6 * c.half);
                }
                __syncthreads();
            } else if (code == f2::kOpMillerDone) {
                if (a.ml_out) emit_group(c, (e >> 5) & 7u, have ? a.ml_out + 72 * (size_t)item : nullptr);
            } else {
                Bases bs;
                bs.b = (uint64_t)grp(c, (e >> 5) & 7u) | (uint64_t)grp(c, (e >> 8) & 7u) << 9 |
                       (uint64_t)grp(c, (e >> 11) & 7u) << 18 | (uint64_t)(c.region + kCOff) << 27 |
                       (uint64_t)grp(c, f2::kTGroup) << 45;
                run((int)code, sm, c.pair, c.lane, c.half, bs);
            }
        }
        const bool one = emit_group(c, (int)f2::kGtGroup[norm], (have && a.gt_out) ? a.gt_out + 72 * (size_t)item : nullptr);
        if (have && c.lane == 0 && c.half == 0) a.results[item] = status != 0 ? -status : (one ? 1 : 0);
        __syncthreads();
    }
}

size_t smem_bytes() { return (size_t)(kSlotArea + kXchArea + kFlagArea + 16 * kKpCount) * 4; }

// The carry-chain ceiling the verify kernel is measured against: every thread
// runs `iters` schoolbook 12 x 12-limb products (prod24: 144 mul.lo + 144
// mul.hi chained through the carry flag, 288 IMAD-pipe instructions) and adds each into a
// 26-limb accumulator, with the verify kernel's block shape and occupancy and
// no loads, barriers or reductions; one operand changes every iteration so
// no product can be hoisted.
__global__ void __launch_bounds__(kThreads, 6) k_imad_chain(int iters, uint32_t* out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t U[12], V[12], acc[26] = {0}, P[24];
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        U[i] = 0x9e3779b9u * (t + i) + 0x7f4a7c15u;
        V[i] = 0x85ebca6bu * (t ^ (i << 8)) + 0xc2b2ae35u;
    }
#pragma unroll 1
    for (int k = 0; k < iters; ++k) {
        f2::prod24(P, U, V);
        f2::acc_plus(acc, P);
        V[0] += 1u;
    }
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 26; ++i) x ^= acc[i];
    out[t] = x;
}

// Issue rate of one multiply form, device-wide: every thread keeps eight
// independent accumulators (no dependence between consecutive multiplies of
// one chain beyond its own), `mode` 0: mul.lo (mad.lo.u32), 1: mul.hi
// (mad.hi.u32); the iteration loop is unrolled four times so its counter and
// branch cost little issue.  64 warps per SM, enough to cover every latency.
__global__ void __launch_bounds__(128) k_imad_rate(int mode, int iters, uint32_t* out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc[8], a[8], b = t * 0x9e3779b9u + 1u;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        acc[k] = k;
        a[k] = 0x85ebca6bu * (t + k) + 7u;
    }
    if (mode == 0) {
#pragma unroll 4
        for (int i = 0; i < iters; ++i) {
#pragma unroll
            for (int k = 0; k < 8; ++k) asm volatile("mad.lo.u32 %0, %1, %2, %0;" : "+r"(acc[k]) : "r"(a[k]), "r"(b));
            b += 0x1234567u;
        }
    } else {
#pragma unroll 4
        for (int i = 0; i < iters; ++i) {
#pragma unroll
            for (int k = 0; k < 8; ++k) asm volatile("mad.hi.u32 %0, %1, %2, %0;" : "+r"(acc[k]) : "r"(a[k]), "r"(b));
            b += 0x1234567u;
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) x ^= acc[k];
    out[t] = x;
}

cudaError_t configure() {
    static cudaError_t done =
        cudaFuncSetAttribute(k_verify_fp2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes());
    return done;
}

int resident() {
    if (configure() != cudaSuccess) return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_verify_fp2, kThreads, smem_bytes()) != cudaSuccess)
        return 0;
    return blocks;
}

}  // namespace

size_t verify_fp2_smem_bytes() { return smem_bytes(); }

int verify_fp2_blocks_per_sm() { return resident(); }

// IMAD-pipe instructions per second of the carry-chain product loop on the
// whole device (blocks: 6 per SM, as the verify kernel runs); `out` must hold
// 6 x sms x 64 words.  Times one warm launch with events on `s`.
cudaError_t measure_imad_chain(int sms, int iters, uint32_t* out, cudaStream_t s, double* imad_per_s) {
    const int blocks = 6 * sms;
    cudaEvent_t a, b;
    cudaError_t e;
    if ((e = cudaEventCreate(&a)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&b)) != cudaSuccess) {
        cudaEventDestroy(a);
        return e;
    }
    k_imad_chain<<<blocks, kThreads, 0, s>>>(iters / 10 + 1, out);   // warm-up
    cudaEventRecord(a, s);
    k_imad_chain<<<blocks, kThreads, 0, s>>>(iters, out);
    cudaEventRecord(b, s);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e == cudaSuccess) *imad_per_s = (double)blocks * kThreads * iters * 288.0 / (ms * 1e-3);
    return e;
}

// Thread multiply instructions per second of mul.lo and of mul.hi on the whole
// device (16 blocks of 128 threads per SM); `out` must hold 16 x sms x 128 words.
cudaError_t measure_imad_rates(int sms, int iters, uint32_t* out, cudaStream_t s, double* lo_per_s,
                               double* hi_per_s) {
    const int blocks = 16 * sms;
    cudaEvent_t a, b;
    cudaError_t e;
    if ((e = cudaEventCreate(&a)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&b)) != cudaSuccess) {
        cudaEventDestroy(a);
        return e;
    }
    for (int mode = 0; mode < 2 && e == cudaSuccess; ++mode) {
        k_imad_rate<<<blocks, 128, 0, s>>>(mode, iters / 8 * 4 + 4, out);   // warm-up
        cudaEventRecord(a, s);
        k_imad_rate<<<blocks, 128, 0, s>>>(mode, iters, out);
        cudaEventRecord(b, s);
        e = cudaEventSynchronize(b);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) *(mode ? hi_per_s : lo_per_s) = (double)blocks * 128 * iters * 8.0 / (ms * 1e-3);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return e;
}

// ring serving: `blocks` persistent blocks (at most the resident slots)
cudaError_t launch_verify_fp2_serve(const VerifyArgs& a, const uint32_t* in_status, int blocks, int sms,
                                   cudaStream_t s) {
    if (!a.serve_avail || !a.serve_stop || !a.serve_claimed || a.serve_cap == 0 || a.serve_cap % kPairsPerBlock ||
        blocks <= 0)
        return cudaErrorInvalidValue;
    cudaError_t e = configure();
    if (e != cudaSuccess) return e;
    const int res = resident();
    if (res > 0 && blocks > res * sms) blocks = res * sms;
    k_verify_fp2<<<blocks, kThreads, smem_bytes(), s>>>(a, in_status);
    return cudaGetLastError();
}

cudaError_t launch_verify_fp2(const VerifyArgs& a, const uint32_t* in_status, int blocks_per_sm, int sms,
                              cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    cudaError_t e = configure();
    if (e != cudaSuccess) return e;
    const int need = (a.n + kPairsPerBlock - 1) / kPairsPerBlock;
    const int res = resident();
    const int per_sm = blocks_per_sm > 0 ? blocks_per_sm : (res > 0 ? res : 1);
    const int cap = per_sm * sms;
    int blocks = a.work_counter ? cap : (need < cap || blocks_per_sm <= 0 ? need : cap);
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    k_verify_fp2<<<blocks, kThreads, smem_bytes(), s>>>(a, in_status);
    return cudaGetLastError();
}

}  // namespace bls
