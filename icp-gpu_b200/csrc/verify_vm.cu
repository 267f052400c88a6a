// Lane-parallel verify kernel: T lanes (T = 1, 2, 4, 8) per verification,
// pairing state in shared memory, tower arithmetic from the generated programs
// (programs.inc via vm.cuh).
//
// Per verification (gpu-crypto/cuda/api.cu:80-91, api.cu:30-52, api.cu:65-78):
//   Miller loop   for each of the 68 line coefficients: both pairs' coefficients
//                 and points go to the C slots, LINE2 multiplies f by both lines;
//                 62 SQR programs in between; CONJ at the end (x < 0)
//   final exp     the reference's chain, each Fp12 operation one program call;
//                 Fp12 values live in 8 groups of 12 slots, renamed, never copied
//   result        canonical Gt compared with 1; optional Miller / Gt outputs
//
// Shared memory: 8 block-shared constant slots (0, 1, Frobenius constants),
// then one region per pairing: 8 groups x 12 slots followed by the program
// temporaries.  The generator's schedule guarantees no slot is written in a
// round where another lane reads it, so a __syncwarp between rounds is the only
// synchronisation.  Every pairing of a warp runs the same program sequence;
// pairings without an item run it on the identity (both pairs skipped).
#include <cuda_runtime.h>

#include "g1.cuh"
#include "internal.h"
#include "vm.cuh"

namespace bls {
namespace {

using vm::Bases;

constexpr uint64_t kXAbs = 0xd201000000010000ULL;

__device__ __forceinline__ uint32_t pack(uint32_t lo, uint32_t hi) { return lo | (hi << 16); }

struct Ctx {
    uint4* sm;
    uint32_t region;  // first slot of this pairing
    uint32_t temp;    // first temporary slot
    int lane;         // lane within the pairing, 0..T-1
};

__device__ __forceinline__ uint32_t grp(const Ctx& c, int g) { return c.region + 12 * g; }

__device__ __forceinline__ Bases bases(const Ctx& c, uint32_t d, uint32_t a, uint32_t b, uint32_t cc) {
    Bases r;
    r.w01 = pack(d, a);
    r.w23 = pack(b, cc);
    r.w45 = pack(0, c.temp);
    r.w67 = pack(c.temp + 32, c.temp + 64);
    return r;
}

template <int T>
__device__ __forceinline__ void call(const Ctx& c, int pid, int d, int a = 0, int b = 0) {
    vm::run<T>(pid, c.sm, bases(c, grp(c, d), grp(c, a), grp(c, b), grp(c, 1)), c.lane);
}

// reduce a slot value below 8p to canonical form
__device__ __forceinline__ fp canonical(fp v) {
    // 4p, 2p, p
    const uint32_t P4[12] = {0xfffeaaacu, 0xe7fbffffu, 0xc54ffffeu, 0x7aaffffau, 0xdac3d890u, 0x9cc34a83u,
                             0xce144afdu, 0x91dd2e13u, 0x0d2eb35du, 0x2c6e9ed9u, 0xe5ff9a69u, 0x680447a8u};
    const uint32_t P2[12] = {0xffff5556u, 0x73fdffffu, 0x62a7ffffu, 0x3d57fffdu, 0xed61ec48u, 0xce61a541u,
                             0xe70a257eu, 0xc8ee9709u, 0x869759aeu, 0x96374f6cu, 0x72ffcd34u, 0x340223d4u};
    const uint32_t P1[12] = {BLS_P0, BLS_P1, BLS_P2, BLS_P3, BLS_P4, BLS_P5,
                             BLS_P6, BLS_P7, BLS_P8, BLS_P9, BLS_P10, BLS_P11};
    const uint32_t* ks[3] = {P4, P2, P1};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        uint32_t d[12], br = 0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
            uint64_t t = (uint64_t)v.w[i] - ks[k][i] - br;
            d[i] = (uint32_t)t;
            br = (uint32_t)(t >> 63);
        }
#pragma unroll
        for (int i = 0; i < 12; ++i) v.w[i] = br ? v.w[i] : d[i];
    }
    return v;
}

__device__ __forceinline__ void copy_fp_from_global(uint4* sm, uint32_t slot, const uint64_t* src) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    sm[3 * slot] = __ldg(s);
    sm[3 * slot + 1] = __ldg(s + 1);
    sm[3 * slot + 2] = __ldg(s + 2);
}

// coefficient `ci` of both pairs into C (slots 0-5 and 8-13 of the C area);
// a skipped pair gets the line (1, 0, 0) so LINE2 leaves f unchanged
template <int T>
__device__ __forceinline__ void load_lines(const Ctx& c, const uint64_t* q1, bool skip1, const uint64_t* q2,
                                           bool skip2, int ci) {
    uint32_t C = grp(c, 1);
    for (int j = c.lane; j < 12; j += T) {
        int pair = j / 6, k = j % 6;
        const uint64_t* q = pair ? q2 : q1;
        bool skip = pair ? skip2 : skip1;
        uint32_t slot = C + 8 * pair + k;
        if (skip) {
            fp v = (k == 4) ? fp_one() : fp_zero();
            vm::store_slot(c.sm, slot, v);
        } else {
            copy_fp_from_global(c.sm, slot, q + 36 * ci + 6 * k);
        }
    }
    __syncwarp();
}

template <int T>
__device__ __forceinline__ void cyc_exp(const Ctx& c, int dst, int x, int spare) {
    call<T>(c, prog::P_COPY, dst, x);
    int cur = dst, oth = spare;
    for (int i = 62; i >= 0; --i) {
        call<T>(c, prog::P_CYCSQR, cur);
        if ((kXAbs >> i) & 1) {
            call<T>(c, prog::P_MUL, oth, cur, x);
            int t = cur; cur = oth; oth = t;
        }
    }
    call<T>(c, prog::P_CONJ, dst, cur);
}

// final exponentiation of group 0 into group 0 (api.cu:65-78)
template <int T>
__device__ __forceinline__ void final_exp(const Ctx& c) {
    call<T>(c, prog::P_CONJ, 1, 0);        // t0 = conj(f)           G1
    call<T>(c, prog::P_INV, 2, 0);         // t1 = f^-1              G2
    call<T>(c, prog::P_MUL, 3, 1, 2);      // t2 = t0 t1             G3
    call<T>(c, prog::P_FROB, 0, 3);        //                        (t1 = t2)
    call<T>(c, prog::P_FROB, 1, 0);        // frob^2(t2)             G1
    call<T>(c, prog::P_MUL, 2, 1, 3);      // t2 = frob^2(t2) t1     G2 (f = t2)
    call<T>(c, prog::P_COPY, 0, 2);
    call<T>(c, prog::P_CYCSQR, 0);
    call<T>(c, prog::P_CONJ, 0, 0);        // t1 = conj(cyc_sqr(t2)) G0
    cyc_exp<T>(c, 1, 2, 3);                // t3 = cyc_exp(t2)       G1
    call<T>(c, prog::P_MUL, 3, 0, 1);      // t4 = t1 t3             G3
    cyc_exp<T>(c, 0, 3, 4);                // t1 = cyc_exp(t4)       G0
    call<T>(c, prog::P_CONJ, 3, 3);        // t4 = conj(t4)
    call<T>(c, prog::P_MUL, 4, 2, 3);      // f = f t4               G4
    call<T>(c, prog::P_COPY, 3, 1);
    call<T>(c, prog::P_CYCSQR, 3);         // t4 = cyc_sqr(t3)       G3
    cyc_exp<T>(c, 5, 0, 6);                // t0 = cyc_exp(t1)       G5
    call<T>(c, prog::P_MUL, 6, 1, 5);      // t3 = t3 t0             G6
    call<T>(c, prog::P_FROB, 1, 6);
    call<T>(c, prog::P_FROB, 6, 1);        // t3 = frob^2(t3)        G6
    call<T>(c, prog::P_MUL, 1, 4, 6);      // f = f t3               G1
    cyc_exp<T>(c, 4, 5, 6);                // c = cyc_exp(t0)        G4
    call<T>(c, prog::P_MUL, 5, 3, 4);      // t4 = t4 c              G5
    cyc_exp<T>(c, 3, 5, 4);                // c = cyc_exp(t4)        G3
    call<T>(c, prog::P_MUL, 4, 1, 3);      // f = f c                G4
    call<T>(c, prog::P_CONJ, 1, 2);        // conj(t2)               G1
    call<T>(c, prog::P_MUL, 3, 5, 1);      // t4 = t4 conj(t2)       G3
    call<T>(c, prog::P_MUL, 1, 2, 0);      // t2 = t2 t1             G1
    call<T>(c, prog::P_FROB, 0, 1);
    call<T>(c, prog::P_FROB, 2, 0);
    call<T>(c, prog::P_FROB, 0, 2);        // t2 = frob^3(t2)        G0
    call<T>(c, prog::P_MUL, 1, 4, 0);      // f = f t2               G1
    call<T>(c, prog::P_FROB, 2, 3);        // t4 = frob(t4)          G2
    call<T>(c, prog::P_MUL, 0, 1, 2);      // f = f t4               G0
}

// canonical group `g` -> out (72 u64) and/or the "is one" test across the pairing's lanes
template <int T>
__device__ __forceinline__ bool emit_group(const Ctx& c, int g, uint64_t* out) {
    bool ok = true;
    for (int j = c.lane; j < 12; j += T) {
        fp v = canonical(vm::load_slot(c.sm, grp(c, g) + j));
        if (out) fp_store_u64(out + 6 * j, v);
        ok = ok && (j == 0 ? fp_eq(v, fp_one()) : fp_is_zero(v));
    }
    unsigned mask = __ballot_sync(0xffffffffu, !ok);
    unsigned gmask = (T == 32 ? 0xffffffffu : ((1u << T) - 1u)) << ((threadIdx.x & 31) & ~(T - 1));
    return (mask & gmask) == 0;
}

template <int T>
__global__ void __launch_bounds__(32 * 4) k_verify_lanes(VerifyArgs a, const uint32_t* __restrict__ in_status) {
    extern __shared__ uint4 smem[];
    constexpr int kPairsPerWarp = 32 / T;
    constexpr int kSlots = vm::Layout<T>::kSlots;
    const int warps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane32 = threadIdx.x & 31;
    const int pair_in_block = warp * kPairsPerWarp + lane32 / T;
    const int pairs_per_block = warps * kPairsPerWarp;

    // block-shared constants: 0, 1, Frobenius k1 = (0, c1), k2 = (c2, 0), k12
    if (threadIdx.x < vm::kKSlots) {
        const uint64_t f1[6] = {0xcd03c9e48671f071ULL, 0x5dab22461fcda5d2ULL, 0x587042afd3851b95ULL,
                                0x8eb60ebe01bacb9eULL, 0x03f97d6e83d050d2ULL, 0x18f0206554638741ULL};
        const uint64_t f2[6] = {0x890dc9e4867545c3ULL, 0x2af322533285a5d5ULL, 0x50880866309b7e2cULL,
                                0xa20d1b8c7e881024ULL, 0x14e4f04fe2db9068ULL, 0x14e56d3f1564853aULL};
        const uint64_t f3[6] = {0x07089552b319d465ULL, 0xc6695f92b50a8313ULL, 0x97e83cccd117228fULL,
                                0xa35baecab2dc29eeULL, 0x1ce393ea5daace4dULL, 0x08f2220fb0fb66ebULL};
        const uint64_t f4[6] = {0xb2f66aad4ce5d646ULL, 0x5842a06bfc497cecULL, 0xcf4895d42599d394ULL,
                                0xc11b9cba40a8e8d0ULL, 0x2e3813cbe5a0de89ULL, 0x110eefda88847fafULL};
        fp v = fp_zero();
        switch (threadIdx.x) {
            case 1: v = fp_one(); break;
            case 3: v = fp_load_u64(f1); break;
            case 4: v = fp_load_u64(f2); break;
            case 6: v = fp_load_u64(f3); break;
            case 7: v = fp_load_u64(f4); break;
            default: break;
        }
        vm::store_slot(smem, threadIdx.x, v);
    }
    __syncthreads();

    Ctx c;
    c.sm = smem;
    c.region = vm::kKSlots + pair_in_block * kSlots;
    c.temp = c.region + vm::kGroups * vm::kGroupSlots;
    c.lane = lane32 & (T - 1);

    // Items are taken a warp at a time (one per pairing): from a counter in
    // persistent mode, so uneven work balances across the resident warps, or
    // by a fixed stride otherwise.  The trip count is warp-uniform: every
    // pairing of the warp runs the programs, idle ones on the identity.
    int next = (blockIdx.x * warps + warp) * kPairsPerWarp;
    const int stride = gridDim.x * pairs_per_block;
    for (;;) {
        int base;
        if (a.work_counter) {
            int b = 0;
            if (lane32 == 0) b = atomicAdd(a.work_counter, kPairsPerWarp);
            base = __shfl_sync(0xffffffffu, b, 0);
        } else {
            base = next;
            next += stride;
        }
        if (base >= a.n) break;
        const int item = base + lane32 / T;
        const bool active = item < a.n;
        bool skip1 = true, skip2 = true;
        const uint64_t* pk = a.g2;
        int32_t status = 0;
        if (active) {
            const uint64_t* s = a.sig_xy ? a.sig_xy + 12 * (size_t)item : (const uint64_t*)a.sigs + 12 * (size_t)item;
            const uint64_t* h = a.nhms + 12 * (size_t)item;
            if (in_status) status = (int32_t)in_status[item];
            fp sx = fp_load_u64(s), sy = fp_load_u64(s + 6);
            fp hx = fp_load_u64(h), hy = fp_load_u64(h + 6);
            int64_t pki = a.pk_index ? (int64_t)a.pk_index[item] : (int64_t)item;
            if (!key_index_ok(pki, a.check_keys, a.n_keys)) {   // no table read for it
                if (status == 0) status = ST_BAD_KEY_INDEX;
                pki = 0;
            }
            pk = a.pk_tables + kCoeffU64 * pki;
            skip1 = g1_limbs_identity(sx, sy) || status != 0;
            skip2 = g1_limbs_identity(hx, hy) || (a.pk_identity && a.pk_identity[pki]) || status != 0;
            if (c.lane == 0) {
                uint32_t C = grp(c, 1);
                vm::store_slot(smem, C + 6, skip1 ? fp_zero() : sx);
                vm::store_slot(smem, C + 7, skip1 ? fp_zero() : sy);
                vm::store_slot(smem, C + 14, skip2 ? fp_zero() : hx);
                vm::store_slot(smem, C + 15, skip2 ? fp_zero() : hy);
            }
        } else if (c.lane == 0) {
            uint32_t C = grp(c, 1);
            vm::store_slot(smem, C + 6, fp_zero());
            vm::store_slot(smem, C + 7, fp_zero());
            vm::store_slot(smem, C + 14, fp_zero());
            vm::store_slot(smem, C + 15, fp_zero());
        }
        // f = 1
        for (int j = c.lane; j < 12; j += T) vm::store_slot(smem, grp(c, 0) + j, j == 0 ? fp_one() : fp_zero());
        __syncwarp();

        // Miller loop over |x| >> 1 below its leading bit (api.cu:30-52)
        int ci = 0;
        for (int b = 61; b >= 0; --b) {
            load_lines<T>(c, a.g2, skip1, pk, skip2, ci++);
            call<T>(c, prog::P_LINE2, 0);
            if (((kXAbs >> 1) >> b) & 1) {
                load_lines<T>(c, a.g2, skip1, pk, skip2, ci++);
                call<T>(c, prog::P_LINE2, 0);
            }
            call<T>(c, prog::P_SQR, 0);
        }
        load_lines<T>(c, a.g2, skip1, pk, skip2, ci);
        call<T>(c, prog::P_LINE2, 0);
        call<T>(c, prog::P_CONJ, 0, 0);
        if (a.ml_out) emit_group<T>(c, 0, active ? a.ml_out + 72 * (size_t)item : nullptr);

        final_exp<T>(c);
        bool one = emit_group<T>(c, 0, (active && a.gt_out) ? a.gt_out + 72 * (size_t)item : nullptr);
        if (active && c.lane == 0) a.results[item] = status != 0 ? -status : (one ? 1 : 0);
        __syncwarp();
    }
}

constexpr int kWarpsPerBlock = 1;

template <int T>
size_t smem_t() {
    return (size_t)(vm::kKSlots + kWarpsPerBlock * (32 / T) * vm::Layout<T>::kSlots) * vm::kSlotBytes;
}

template <int T>
cudaError_t configure_t() {
    static cudaError_t done = cudaFuncSetAttribute(k_verify_lanes<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem_t<T>());
    return done;
}

template <int T>
int resident_t() {
    if (configure_t<T>() != cudaSuccess) return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_verify_lanes<T>, 32 * kWarpsPerBlock, smem_t<T>()) !=
        cudaSuccess)
        return 0;
    return blocks;
}

template <int T>
cudaError_t launch_t(const VerifyArgs& a, const uint32_t* in_status, cudaStream_t s, int blocks_per_sm, int sms) {
    cudaError_t e = configure_t<T>();
    if (e != cudaSuccess) return e;
    int pairs_per_block = kWarpsPerBlock * (32 / T);
    int need = (a.n + pairs_per_block - 1) / pairs_per_block;
    int resident = resident_t<T>();
    int per_sm = blocks_per_sm > 0 ? blocks_per_sm : (resident > 0 ? resident : 1);
    int cap = per_sm * sms;
    // persistent mode: exactly the resident grid, items claimed from the counter
    int blocks = a.work_counter ? cap : (need < cap || blocks_per_sm <= 0 ? need : cap);
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    k_verify_lanes<T><<<blocks, 32 * kWarpsPerBlock, smem_t<T>(), s>>>(a, in_status);
    return cudaGetLastError();
}

}  // namespace

size_t verify_lanes_smem_bytes(int lanes, int shape) {
    switch (lanes) {
        case 6: return six_lane_shape(shape) == kShapeWide ? verify_w_smem_bytes() : verify_fp2_smem_bytes();
        case 2: return smem_t<2>();
        case 4: return smem_t<4>();
        default: return smem_t<8>();
    }
}

int verify_lanes_blocks_per_sm(int lanes, int shape) {
    switch (lanes) {
        case 6: return six_lane_shape(shape) == kShapeWide ? verify_w_blocks_per_sm() : verify_fp2_blocks_per_sm();
        case 2: return resident_t<2>();
        case 4: return resident_t<4>();
        case 8: return resident_t<8>();
        default: return 0;
    }
}

cudaError_t launch_verify_lanes(const VerifyArgs& a, const uint32_t* in_status, int lanes, int shape,
                                int blocks_per_sm, int sms, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    switch (lanes) {
        case 6:
            return six_lane_shape(shape) == kShapeWide ? launch_verify_w(a, in_status, sms, s)
                                                       : launch_verify_fp2(a, in_status, blocks_per_sm, sms, s);
        case 2: return launch_t<2>(a, in_status, s, blocks_per_sm, sms);
        case 4: return launch_t<4>(a, in_status, s, blocks_per_sm, sms);
        case 8: return launch_t<8>(a, in_status, s, blocks_per_sm, sms);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace bls
