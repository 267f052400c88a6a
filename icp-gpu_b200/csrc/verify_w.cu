// Warp-uniform Fp2-lane verify kernel.  The same generated programs as
// verify_fp2.cu (fp2ops.inc, gen_fp2ops.py), mapped the other way round: a
// block of twelve warps verifies 32 items, warp w takes one role of the
// twelve-thread decomposition (Fp2 coefficient k = w % 6 of every Fp12
// result, half h = w / 6) and lane v works on item v.  Every lane of a warp
// therefore runs the same output descriptor: descriptor reads are constant-
// memory broadcasts, control flow never diverges, and the only per-lane
// difference is which item's slots a lane reads and writes.
//
// Per verification (gpu-crypto/cuda/api.cu:80-91, api.cu:30-52, api.cu:65-78):
// the Miller loop over both pairs with the lines of the generator's and the
// key's tables, the reference's final-exponentiation chain, the canonical Gt
// compared with one; optional Miller / Gt outputs.
//
// Shared memory (16-byte units): the items' Fp2 slots interleaved by item
// (unit ((s * 2 + c) * 3 + q) * 32 + v holds words 4q..4q+3 of component c of
// slot s of item v, so a warp's load of one component is three conflict-free
// 512-byte rows), then the block-shared constant slots, the partial-sum
// exchange area (one 26-word partial per coefficient, half and item, same
// interleaving), the per-item flags and the table of k p for the outputs'
// bias multiples.
#include <cuda_runtime.h>

#include "fp2ops.cuh"
#include "g1.cuh"
#include "internal.h"

namespace bls {
namespace {

constexpr int kV = 32;                           // items per block, one per lane
constexpr int kRoles = 12;                       // warps per block
constexpr int kThreads = 32 * kRoles;
constexpr int kGroups = f2::kGroupsUsed;
constexpr int kKSlots = f2::kKSlotCount;         // block-shared constant slots (absolute 0 .. kKSlots - 1)
constexpr int kCOff = 6 * kGroups;               // C area after the groups
constexpr int kItemSlots = kCOff + 12;           // Fp2 slots per item
constexpr int kSlotU4 = kItemSlots * 6 * kV;     // 16-byte units of the item slots
constexpr int kKU4 = kKSlots * 6;                // constant slots, not interleaved
constexpr int kXchU4 = 6 * 2 * 7 * kV;           // exchange: 26 words (7 units) per coefficient, half, item
constexpr int kKpCount = f2::kMaxBias + 1;       // k p, 16 words each
constexpr int kInfoWords = 4 * kV;               // per item: key index, flags, status, result flags
constexpr int kFlagBytes = 16 * kV;              // per item and role: "not the expected value" bytes
constexpr int kQpU4 = 128 * 4;                   // the QP table (128 entries of 16 words)
constexpr size_t kSmemBytes = (size_t)(kSlotU4 + kKU4 + kXchU4 + kQpU4) * 16 + (size_t)kKpCount * 64 +
                              (size_t)kInfoWords * 4 + kFlagBytes + 16;
static_assert(kKSlots + kItemSlots <= 256, "slot indices must fit a byte");
static_assert(kKpCount <= kThreads, "one thread per table entry at start-up");
static_assert(kSmemBytes <= 227 * 1024, "one block per SM");

struct Sm {
    uint4* slots;      // item slots
    uint4* kslots;     // constant slots
    uint4* xch;        // exchange
    uint4* qp;         // QP table (qp_reduce_tab)
    uint32_t* kp;      // k p table
    uint32_t* info;    // per item: [0] key index, [1] skip bits, [2] status, [3] spare
    uint8_t* flags;    // per item, 16 bytes: role r's "not expected" byte at r
    uint32_t* bcast;   // claim broadcast (4 words)
    int v;             // this lane's item
};

// D, A, B, C, K, T: absolute slot of index 0, one byte each
struct Bases { uint64_t b; };

__device__ __forceinline__ uint32_t slot_addr(const Bases& bs, uint32_t ref) {
    return (uint32_t)(bs.b >> (8u * (ref >> 4))) % 256u + (ref & 15u);
}

// the three 16-byte units of component `comp` of absolute slot `slot` for this lane
__device__ __forceinline__ const uint4* unit_ptr(const Sm& s, uint32_t slot, int comp) {
    if (slot < (uint32_t)kKSlots) return s.kslots + (slot * 2 + comp) * 3;
    return s.slots + ((slot - kKSlots) * 2 + comp) * 3 * kV + s.v;
}
__device__ __forceinline__ uint32_t unit_stride(uint32_t slot) { return slot < (uint32_t)kKSlots ? 1u : (uint32_t)kV; }

__device__ __forceinline__ void load_fp(uint32_t* x, const Sm& s, uint32_t slot, int comp) {
    const uint4* p = unit_ptr(s, slot, comp);
    const uint32_t st = unit_stride(slot);
    const uint4 a = p[0], b = p[st], c = p[2 * st];
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    x[8] = c.x; x[9] = c.y; x[10] = c.z; x[11] = c.w;
}
// stores go to item slots only (the constant slots are written at start-up)
__device__ __forceinline__ void store_fp(const Sm& s, uint32_t slot, int comp, const uint32_t* x) {
    uint4* p = s.slots + ((slot - kKSlots) * 2 + comp) * 3 * kV + s.v;
    p[0] = make_uint4(x[0], x[1], x[2], x[3]);
    p[kV] = make_uint4(x[4], x[5], x[6], x[7]);
    p[2 * kV] = make_uint4(x[8], x[9], x[10], x[11]);
}

// t[0..12] = k p from the block's table (k <= kMaxBias for every descriptor)
__device__ __forceinline__ void load_kp(uint32_t* t, const Sm& s, uint32_t k) {
    const uint32_t* e = s.kp + 16 * k;
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

// partial sum `acc` (26 words) of this lane into exchange unit row `row`
__device__ __forceinline__ void xch_store(uint4* row, const uint32_t* acc) {
#pragma unroll
    for (int q = 0; q < 6; ++q) row[q * kV] = make_uint4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
    row[6 * kV] = make_uint4(acc[24], acc[25], 0u, 0u);
}
__device__ __forceinline__ void xch_load(uint32_t* p, const uint4* row) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const uint4 u = row[q * kV];
        p[4 * q] = u.x; p[4 * q + 1] = u.y; p[4 * q + 2] = u.z; p[4 * q + 3] = u.w;
    }
    const uint4 u = row[6 * kV];
    p[24] = u.x;
    p[25] = u.y;
}

// Phase 1 of an output (product modes): this half's products into both
// accumulators; the partner's component (accX) goes to the exchange row.
__device__ __forceinline__ void accumulate(uint32_t off, const Sm& s, const Bases& bs, uint4* xch_out, int half,
                                           uint32_t* own) {
    const uint32_t hdr = f2::kDesc[off], bias = f2::kDesc[off + 1];
    const uint32_t nt = (hdr >> 2) & 15u;
    uint32_t accO[26], accX[26];
    const uint32_t sw = half ? 8u : 0u, c0 = half ? 12u : 0u, c1 = half ? 0u : 12u;
#pragma unroll
    for (int i = 0; i < 12; ++i) accO[i] = accX[i] = 0;
    accO[25] = accX[25] = 0;
    load_kp(accO + 12, s, (bias >> sw) & 0xffu);
    load_kp(accX + 12, s, (bias >> (8u - sw)) & 0xffu);
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t w = f2::kDesc[off + 2 + t];
        const uint32_t kind = w & 7u, xi = (w >> 3) & 1u, neg = (w >> 4) & 1u, dbl = (w >> 5) & 1u,
                       yim = (w >> 6) & 1u, mask = (w >> 24) & 7u;
        const uint32_t xs = slot_addr(bs, (w >> 8) & 0x7fu), ys = slot_addr(bs, (w >> 16) & 0x7fu);
        if (kind == f2::kOne) {             // X R: X into the high half of both accumulators
            uint32_t x0[12], x1[12];
            load_fp(x0, s, xs, half);
            load_fp(x1, s, xs, 1 - half);
            f2::acc_add_hi(accO, x0, neg);
            f2::acc_add_hi(accX, x1, neg);
            continue;
        }
        const uint32_t cw = f2::kCoef[2 * kind + xi] ^ (neg ? 0x666666u : 0u);
        const uint32_t np = kind == f2::kKara ? 3u : 2u;
#pragma unroll 1
        for (uint32_t j = 0; j < np; ++j) {
            if (!((mask >> j) & 1u)) continue;
            uint32_t U[12], V[12], P[24];
            if (kind == f2::kSqr) {          // U = x0 + x1, 2 x0
                load_fp(U, s, xs, 0);
                if (j == 0) {
                    uint32_t T[12];
                    load_fp(T, s, xs, 1);
                    f2::add12(U, U, T);
                } else {
                    f2::dbl12(U);
                }
            } else if (kind == f2::kKara && xi) {   // xi X = (x0 - x1 + 3p, x0 + x1); sum 2 x0 + 3p
                load_fp(U, s, xs, 0);
                if (j == 2) {
                    const uint32_t z[12] = {0};
                    f2::dbl12(U);
                    f2::add3p_sub(U, U, z);
                } else {
                    uint32_t T[12];
                    load_fp(T, s, xs, 1);
                    if (j == 0) f2::add3p_sub(U, U, T);
                    else f2::add12(U, U, T);
                }
            } else {                         // x0, x1 (KARA: sum x0 + x1)
                load_fp(U, s, xs, j & 1u);
                if (j == 2) {
                    uint32_t T[12];
                    load_fp(T, s, xs, 1);
                    f2::add12(U, U, T);
                }
            }
            if (kind == f2::kKara) {        // V = y0, y1, y0 + y1 (doubled when dbl)
                load_fp(V, s, ys, j & 1u);
                if (j == 2) {
                    uint32_t T[12];
                    load_fp(T, s, ys, 1);
                    f2::add12(V, V, T);
                }
                if (dbl) f2::dbl12(V);
            } else if (kind == f2::kSqr) {  // V = x0 - x1 + 3p, x1
                load_fp(V, s, xs, 1);
                if (j == 0) {
                    uint32_t T[12];
                    load_fp(T, s, xs, 0);
                    f2::add3p_sub(V, T, V);
                }
            } else if (kind == f2::kFpMul) {
                load_fp(V, s, ys, yim);
            } else {                        // NORM: x_j^2
                load_fp(V, s, xs, j);
            }
            f2::prod24k(P, U, V);
            acc_pair(accO, accX, P, (cw >> (c0 + 4 * j)) & 3u, (cw >> (c1 + 4 * j)) & 3u);
        }
    }
    xch_store(xch_out, accX);
#pragma unroll
    for (int i = 0; i < 26; ++i) own[i] = accO[i];
}

// Phase 2: component `half` of the output into o (12 words).  own: this
// half's accumulator of that component (product modes), xch_in: the partner's.
__device__ __forceinline__ void finish(uint32_t off, const Sm& s, const Bases& bs, int half, uint32_t* own,
                                       const uint4* xch_in, uint32_t* o) {
    const uint32_t hdr = f2::kDesc[off], bias = f2::kDesc[off + 1];
    const uint32_t mode = hdr & 3u, nt = (hdr >> 2) & 15u, nl = (hdr >> 6) & 3u;
    const int cc = half ? sext4(hdr >> 20) : sext4(hdr >> 16);
    const uint32_t bias_lin = (bias >> (16 + 8 * half)) & 0xffu;
    const uint32_t* lin = f2::kDesc + off + 2 + nt;

    if (mode == f2::kModeInvFp) {
        if (half == 0) {
            fp z;
            load_fp(z.w, s, slot_addr(bs, lin[0] >> 8), 0);
            fp r = fp_inverse_warp(z, f2::kR3);
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
        load_kp(r, s, bias_lin);
        for (uint32_t j = 0; j < nl; ++j) {
            uint32_t z[12];
            load_fp(z, s, slot_addr(bs, lin[j] >> 8), half);
            f2::madd13(r, z, cc * sext4(lin[j]));
        }
    } else {
        uint32_t p[26];
        xch_load(p, xch_in);
        f2::add26(own, p);
        uint32_t red[13];
        f2::redc26(red, own);
        if (mode == f2::kModeSimple) {
            f2::qp_reduce_tab(o, red, s.qp);
            return;
        }
        uint32_t q[12];
        f2::qp_reduce_tab(q, red, s.qp);
        load_kp(r, s, bias_lin);
        f2::madd13(r, q, cc);
        for (uint32_t j = 0; j < nl; ++j) {
            uint32_t z[12];
            load_fp(z, s, slot_addr(bs, lin[j] >> 8), half);
            f2::madd13(r, z, sext4(lin[j]));
        }
    }
    f2::qp_reduce_tab(o, r, s.qp);
}

// program `pid` for every item of the block: accumulate, exchange (the two
// warps of coefficient k meet), reduce, meet, write, meet.  The descriptor
// index of the role is 8 half + k.  No program of the generated sequences
// writes a slot that any role of it reads (the generator places a result
// that would overwrite an operand in an unused group, and refuses to emit a
// sequence where it cannot), so a role stores its output as soon as it has
// it: one block-wide meeting per program, after the stores.
__device__ __forceinline__ void run(int pid, const Sm& s, int k, int half, const Bases& bs) {
    const uint32_t off = f2::kOutIndex[pid][8 * half + k];
    const uint32_t mode = off != 0xffffu ? (f2::kDesc[off] & 3u) : 0u;
    const bool prod = off != 0xffffu && (mode == f2::kModeSimple || mode == f2::kModeFull);
    uint4* mine = s.xch + (k * 2 + half) * 7 * kV + s.v;
    const uint4* theirs = s.xch + (k * 2 + (1 - half)) * 7 * kV + s.v;
    uint32_t own[26];
    if (prod) accumulate(off, s, bs, mine, half, own);
    // only warps k and 6 + k exchange partial sums here: a named barrier
    // (id 1 + k) over those 64 threads instead of the whole block; both warps
    // reach it on every program, whether or not their role has an output
    asm volatile("bar.sync %0, 64;" ::"r"(1 + k) : "memory");
    uint32_t o[12];
    if (off != 0xffffu) finish(off, s, bs, half, own, theirs, o);
    if (off != 0xffffu) store_fp(s, slot_addr(bs, (f2::kDesc[off] >> 8) & 0x7fu), half, o);
    __syncthreads();
}

__device__ __forceinline__ uint32_t grp(int g) { return kKSlots + 6 * g; }

__device__ __forceinline__ void copy_fp_from_global(const Sm& s, uint32_t slot, int comp, const uint64_t* src) {
    const uint4* g = reinterpret_cast<const uint4*>(src);
    uint4* p = s.slots + ((slot - kKSlots) * 2 + comp) * 3 * kV + s.v;
    p[0] = __ldg(g);
    p[kV] = __ldg(g + 1);
    p[2 * kV] = __ldg(g + 2);
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

// canonical group `g` -> out (72 u64 per item, NULL: not wanted) and the
// "is one" test of every item over the twelve roles
__device__ __forceinline__ bool emit_group(const Sm& s, int g, int k, int half, uint64_t* out) {
    fp v;
    load_fp(v.w, s, grp(g) + k, half);
    v = canonical(v);
    if (out) fp_store_u64(out + 12 * k + 6 * half, v);
    const bool ok = (k == 0 && half == 0) ? fp_eq(v, fp_one()) : fp_is_zero(v);
    s.flags[16 * s.v + 8 * half + k] = ok ? 0 : 1;
    __syncthreads();
    const uint4 f = reinterpret_cast<const uint4*>(s.flags)[s.v];
    __syncthreads();
    return (f.x | f.y | f.z | f.w) == 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t ld_acquire_gpu(const volatile uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Ring serving, thread 0 of a block: claim up to 32 published items (all in
// device memory); *count gets how many.  False when the block should leave:
// the stop flag, serve_idle_ns in which the published count did not move,
// or serve_max_ns after the launch; the loop also has an iteration cap, so
// every wait ends.  The published count is read with acquire semantics and a
// fence follows the claim, so the claimed items' loads come after the copies
// that published them.
__device__ bool serve_claim(const VerifyArgs& a, uint64_t t_launch, uint32_t* base, uint32_t* count) {
    uint64_t t_moved = globaltimer_ns();
    uint32_t seen = ld_acquire_gpu(a.serve_avail);
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        const uint32_t cur = *reinterpret_cast<volatile uint32_t*>(a.serve_claimed);
        const uint32_t av = ld_acquire_gpu(a.serve_avail);
        const int32_t ready = (int32_t)(av - cur);
        if (ready > 0) {
            const uint32_t n = ready < kV ? (uint32_t)ready : (uint32_t)kV;
            if (atomicCAS(a.serve_claimed, cur, cur + n) == cur) {
                __threadfence();
                *base = cur;
                *count = n;
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

__global__ void __launch_bounds__(kThreads, 1) k_verify_w(VerifyArgs a, const uint32_t* __restrict__ in_status) {
    extern __shared__ uint4 smem4[];
    Sm s;
    s.slots = smem4;
    s.kslots = smem4 + kSlotU4;
    s.xch = s.kslots + kKU4;
    s.qp = s.xch + kXchU4;
    s.kp = reinterpret_cast<uint32_t*>(s.qp + kQpU4);
    s.info = s.kp + 16 * kKpCount;
    s.flags = reinterpret_cast<uint8_t*>(s.info + kInfoWords);
    s.bcast = reinterpret_cast<uint32_t*>(s.flags + kFlagBytes);
    const int role = threadIdx.x >> 5;
    const int half = role / 6, k = role % 6;
    s.v = threadIdx.x & 31;

    {
        uint32_t* kw = reinterpret_cast<uint32_t*>(s.kslots);
        for (int i = threadIdx.x; i < kKSlots * 24; i += blockDim.x) kw[i] = f2::kKSlots[i / 24][i % 24];
    }
    if (threadIdx.x < kKpCount) {
        uint32_t t[13];
        f2::set_kp(t, threadIdx.x);
#pragma unroll
        for (int i = 0; i < 13; ++i) s.kp[16 * threadIdx.x + i] = t[i];
    }
    {
        // unit j of entry e at 128 j + e (qp_reduce_tab)
        uint32_t* qw = reinterpret_cast<uint32_t*>(s.qp);
        for (int i = threadIdx.x; i < 128 * 16; i += blockDim.x) {
            const int e = i / 16, w = i % 16;
            qw[4 * (128 * (w / 4) + e) + w % 4] = f2::kQP2[e][w];
        }
    }
    // the flag bytes no role writes (6, 7, 14, 15 of each item) stay zero
    for (int i = threadIdx.x; i < kFlagBytes / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(s.flags)[i] = 0;
    __syncthreads();

    const int norm = a.pk_norm != nullptr ? 1 : 0;
    const uint64_t* g2_lines = norm ? a.g2_norm : a.g2;
    const bool serving = a.serve_avail != nullptr;
    const uint64_t t_launch = serving ? globaltimer_ns() : 0;
    int next = blockIdx.x * kV;
    const int stride = gridDim.x * kV;
    uint32_t* info = s.info + 4 * s.v;

    for (;;) {
        int base, count;
        if (serving) {
            if (threadIdx.x == 0) {
                uint32_t b = 0, n = 0;
                const bool go = serve_claim(a, t_launch, &b, &n);
                s.bcast[0] = b;
                s.bcast[1] = go ? n : 0u;
            }
            __syncthreads();
            base = (int)s.bcast[0];
            count = (int)s.bcast[1];
            __syncthreads();
            if (count == 0) break;
        } else {
            if (a.work_counter) {
                if (threadIdx.x == 0) s.bcast[0] = (uint32_t)atomicAdd(a.work_counter, kV);
                __syncthreads();
                base = (int)s.bcast[0];
                __syncthreads();
            } else {
                base = next;
                next += stride;
            }
            if (base >= a.n) break;
            count = a.n - base < kV ? a.n - base : kV;
        }
        const bool have = s.v < count;
        // item = ring slot (serving) or batch index
        const uint32_t item = serving ? (uint32_t)(base + s.v) % a.serve_cap : (uint32_t)(base + s.v);

        // warp 0 reads the item's points, status and key; the others wait for its
        // per-item record
        if (role == 0) {
            uint32_t skip = 3u, pki = 0, status = 0;
            fp sx = fp_zero(), sy = fp_zero(), hx = fp_zero(), hy = fp_zero();
            if (have) {
                const uint64_t* sp = a.sig_xy ? a.sig_xy + 12 * (size_t)item : (const uint64_t*)a.sigs + 12 * (size_t)item;
                const uint64_t* hp = a.nhms + 12 * (size_t)item;
                if (in_status) status = __ldcg(in_status + item);
                sx = fp_load_u64_cg(sp);
                sy = fp_load_u64_cg(sp + 6);
                hx = fp_load_u64_cg(hp);
                hy = fp_load_u64_cg(hp + 6);
                pki = a.pk_index ? (uint32_t)__ldcg(a.pk_index + item) : item;
                if (!key_index_ok((int64_t)(int32_t)pki, a.check_keys, a.n_keys)) {   // no table read for it
                    if (status == 0) status = ST_BAD_KEY_INDEX;
                    pki = 0;
                }
                const bool s1 = status != 0 || g1_limbs_identity(sx, sy);
                const bool s2 = status != 0 || g1_limbs_identity(hx, hy) || (a.pk_identity && a.pk_identity[pki]);
                skip = (s1 ? 1u : 0u) | (s2 ? 2u : 0u);
            }
            const uint32_t C = kKSlots + kCOff;
            store_fp(s, C + 0 * 6 + 3, 0, (skip & 1u) ? fp_zero().w : sx.w);
            store_fp(s, C + 0 * 6 + 3, 1, (skip & 1u) ? fp_zero().w : sy.w);
            store_fp(s, C + 1 * 6 + 3, 0, (skip & 2u) ? fp_zero().w : hx.w);
            store_fp(s, C + 1 * 6 + 3, 1, (skip & 2u) ? fp_zero().w : hy.w);
            info[0] = pki;
            info[1] = skip;
            info[2] = status;
        }
        // f = 1
        store_fp(s, grp(0) + k, half, (k == 0 && half == 0) ? fp_one().w : fp_zero().w);
        __syncthreads();
        const uint32_t pki = info[0], skip = info[1];
        const uint64_t* pk = (norm ? a.pk_norm : a.pk_tables) + (size_t)kCoeffU64 * pki;
        const uint64_t* pk_cf = norm ? a.pk_corr + 12 * (size_t)pki : a.g2_corr;

        const int seq_len = norm ? f2::kSeqLenNorm : f2::kSeqLenRaw;
        for (int st = 0; st < seq_len; ++st) {
            const uint32_t e = f2::kSeq[norm][st];
            const uint32_t code = e & 31u;
            if ((e & f2::kCondMl) && !a.ml_out) continue;
            if (code == f2::kOpLoadLines) {
                // role (k, h): pair k / 3, coefficient k % 3, component h; a
                // skipped pair gets the line (0, 0, 1), which leaves f unchanged.
                // When the next op is LSCALE (l2 = c1 P.x, l3 = c0 P.y), the roles
                // holding c1 and c0 form their component of it here: that
                // program's every output is one product with a zero bias, so
                // QP(REDC(c_h * P coordinate)) is bit for bit its result, and the
                // program's exchange and barriers are saved.
                const bool fuse = st + 1 < seq_len && (f2::kSeq[norm][st + 1] & 31u) == (uint32_t)f2::P_LSCALE;
                const int pair = k / 3, c = k % 3;
                const uint32_t C = kKSlots + kCOff + 6 * pair;
                uint32_t x[12];
                if ((skip >> pair) & 1u) {
                    const fp v = (c == 2 && half == 0) ? fp_one() : fp_zero();
#pragma unroll
                    for (int i = 0; i < 12; ++i) x[i] = v.w[i];
                } else {
                    const uint64_t* q = pair ? pk : g2_lines;
                    const uint4* g = reinterpret_cast<const uint4*>(q + 36 * ((e >> 14) & 127u) + 12 * c + 6 * half);
                    const uint4 a0 = __ldg(g), a1 = __ldg(g + 1), a2 = __ldg(g + 2);
                    x[0] = a0.x; x[1] = a0.y; x[2] = a0.z; x[3] = a0.w;
                    x[4] = a1.x; x[5] = a1.y; x[6] = a1.z; x[7] = a1.w;
                    x[8] = a2.x; x[9] = a2.y; x[10] = a2.z; x[11] = a2.w;
                }
                store_fp(s, C + c, half, x);
                if (fuse && c < 2) {
                    uint32_t y[12], P[26], red[13], o[12];
                    load_fp(y, s, C + 3, c == 1 ? 0 : 1);   // P.x for l2, P.y for l3
                    f2::prod24k(P, x, y);
                    P[24] = P[25] = 0;
                    f2::redc26(red, P);
                    f2::qp_reduce_tab(o, red, s.qp);
                    store_fp(s, C + (c == 1 ? 4 : 5), half, o);
                }
                __syncthreads();
                if (fuse) ++st;
            } else if (code == f2::kOpLoadCorr) {
                // the generator's and the key's Miller correction factors into the c2 slots
                if (k < 2) {
                    const uint32_t slot = kKSlots + kCOff + 6 * k + 2;
                    if ((skip >> k) & 1u) store_fp(s, slot, half, half ? fp_zero().w : fp_one().w);
                    else copy_fp_from_global(s, slot, half, (k ? pk_cf : a.g2_corr) + 6 * half);
                }
                __syncthreads();
            } else if (code == f2::kOpMillerDone) {
                if (a.ml_out) emit_group(s, (e >> 5) & 7u, k, half, have ? a.ml_out + 72 * (size_t)item : nullptr);
            } else {
                Bases bs;
                bs.b = (uint64_t)grp((e >> 5) & 7u) | (uint64_t)grp((e >> 8) & 7u) << 8 |
                       (uint64_t)grp((e >> 11) & 7u) << 16 | (uint64_t)(kKSlots + kCOff) << 24 |
                       (uint64_t)grp(f2::kTGroup) << 40;
                run((int)code, s, k, half, bs);
            }
        }
        const bool one = emit_group(s, (int)f2::kGtGroup[norm], k, half,
                                    (have && a.gt_out) ? a.gt_out + 72 * (size_t)item : nullptr);
        if (have && role == 0) {
            const int32_t status = (int32_t)info[2];
            a.results[item] = status != 0 ? -status : (one ? 1 : 0);
        }
        __syncthreads();
    }
}

cudaError_t configure() {
    static cudaError_t done =
        cudaFuncSetAttribute(k_verify_w, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    return done;
}

}  // namespace

size_t verify_w_smem_bytes() { return kSmemBytes; }

int verify_w_blocks_per_sm() {
    if (configure() != cudaSuccess) return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_verify_w, kThreads, kSmemBytes) != cudaSuccess)
        return 0;
    return blocks;
}

// ring serving: `blocks` persistent blocks (at most one per SM)
cudaError_t launch_verify_w_serve(const VerifyArgs& a, const uint32_t* in_status, int blocks, int sms,
                                 cudaStream_t s) {
    if (!a.serve_avail || !a.serve_stop || !a.serve_claimed || a.serve_cap == 0 || blocks <= 0)
        return cudaErrorInvalidValue;
    cudaError_t e = configure();
    if (e != cudaSuccess) return e;
    if (blocks > sms) blocks = sms;
    k_verify_w<<<blocks, kThreads, kSmemBytes, s>>>(a, in_status);
    return cudaGetLastError();
}

cudaError_t launch_verify_w(const VerifyArgs& a, const uint32_t* in_status, int sms, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    cudaError_t e = configure();
    if (e != cudaSuccess) return e;
    const int need = (a.n + kV - 1) / kV;
    int blocks = a.work_counter ? sms : need;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    k_verify_w<<<blocks, kThreads, kSmemBytes, s>>>(a, in_status);
    return cudaGetLastError();
}

}  // namespace bls
