// Product throughput of three limb layouts for 381-bit field elements, in the
// setting of the twelve-warp verify kernel (k_verify_w): one block of 384
// threads per SM, every thread computing one double-width product per
// iteration from operands it loads out of lane-interleaved shared memory, and
// accumulating it.  The layouts:
//
//   0  12 x 32-bit limbs: one level of limb Karatsuba (three 6 x 6 products
//      whose rows are mad.lo.cc / madc.hi.cc carry chains, 216 multiplies)
//      added into a 26-limb accumulator: the form every verify kernel uses
//      (fp2ops.cuh prod24k + acc_plus);
//   1  15 x 26-bit signed limbs: 225 mad.wide.s32 into 29 signed 64-bit
//      columns, no carries (the headroom of the reduced radix absorbs them);
//   2  14 x 28-bit limbs: 196 mad.wide.u32 into 27 unsigned 64-bit columns.
//
// Each value loaded is a bounded pseudo-random word; no result is used but a
// checksum, which is stored so that nothing is optimised away.  The autotuner
// reports these rates as its limb-layout points: the verify kernels are built
// for the layout with the highest rate.
#include <cuda_runtime.h>

#include "fp2ops.cuh"
#include "internal.h"

namespace bls {
namespace {

constexpr int kThreadsLF = 384;   // twelve warps, as k_verify_w
constexpr int kSlotsLF = 16;      // operand slots per lane
constexpr int kWordsLF = 16;      // words per slot (four 16-byte units)
constexpr size_t kSmemLF = (size_t)kSlotsLF * kWordsLF * 32 * 4;   // 32 KB

// unit q of slot s for lane v, as the verify kernel interleaves items
__device__ __forceinline__ const uint4* lf_unit(const uint4* sm, int s, int q, int v) {
    return sm + (s * 4 + q) * 32 + v;
}

__device__ __forceinline__ void lf_load(uint32_t* x, const uint4* sm, int s, int v, int words) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (4 * q >= words) break;
        const uint4 u = *lf_unit(sm, s, q, v);
        x[4 * q] = u.x;
        if (4 * q + 1 < words) x[4 * q + 1] = u.y;
        if (4 * q + 2 < words) x[4 * q + 2] = u.z;
        if (4 * q + 3 < words) x[4 * q + 3] = u.w;
    }
}

template <int kForm>
__global__ void __launch_bounds__(kThreadsLF, 1) k_limb_form(int iters, uint32_t* out) {
    extern __shared__ uint4 sm4[];
    const int v = threadIdx.x & 31;
    // fill: bounded words for the reduced-radix forms (signed 26-bit, or 28-bit)
    {
        uint32_t* w = reinterpret_cast<uint32_t*>(sm4);
        for (int i = threadIdx.x; i < kSlotsLF * kWordsLF * 32; i += blockDim.x) {
            uint32_t x = 0x9e3779b9u * (uint32_t)(i + 1) ^ (0x85ebca6bu * blockIdx.x);
            x ^= x >> 15;
            x *= 0x2c1b3c6du;
            x ^= x >> 12;
            if (kForm == 1) x = (uint32_t)((int32_t)(x << 6) >> 6);   // signed 26-bit
            if (kForm == 2) x &= 0x0fffffffu;                       // 28-bit
            w[i] = x;
        }
    }
    __syncthreads();
    uint32_t check = 0;
    if (kForm == 0) {
        uint32_t acc[26];
#pragma unroll
        for (int i = 0; i < 26; ++i) acc[i] = 0;
#pragma unroll 1
        for (int k = 0; k < iters; ++k) {
            uint32_t U[12], V[12], P[24];
            lf_load(U, sm4, k & (kSlotsLF - 1), v, 12);
            lf_load(V, sm4, (5 * k + 3) & (kSlotsLF - 1), v, 12);
            U[11] &= 0x3fffffffu;   // operands below 2^382, as the kernel's slots
            V[11] &= 0x3fffffffu;
            f2::prod24k(P, U, V);
            f2::acc_plus(acc, P);
        }
#pragma unroll
        for (int i = 0; i < 26; ++i) check ^= acc[i];
    } else {
        constexpr int L = kForm == 1 ? 15 : 14;
        constexpr int C = 2 * L - 1;
        uint64_t col[C];
#pragma unroll
        for (int i = 0; i < C; ++i) col[i] = 0;
#pragma unroll 1
        for (int k = 0; k < iters; ++k) {
            uint32_t U[L], V[L];
            lf_load(U, sm4, k & (kSlotsLF - 1), v, L);
            lf_load(V, sm4, (5 * k + 3) & (kSlotsLF - 1), v, L);
#pragma unroll
            for (int i = 0; i < L; ++i) {
#pragma unroll
                for (int j = 0; j < L; ++j) {
                    if (kForm == 1)
                        asm("mad.wide.s32 %0, %1, %2, %0;" : "+l"(col[i + j]) : "r"(U[i]), "r"(V[j]));
                    else
                        asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(col[i + j]) : "r"(U[i]), "r"(V[j]));
                }
            }
        }
#pragma unroll
        for (int i = 0; i < C; ++i) check ^= (uint32_t)col[i] ^ (uint32_t)(col[i] >> 32);
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = check;
}

template <int kForm>
cudaError_t time_form(int sms, int iters, uint32_t* out, cudaStream_t s, double* per_s) {
    cudaError_t e = cudaFuncSetAttribute(k_limb_form<kForm>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSmemLF);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    if ((e = cudaEventCreate(&a)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&b)) != cudaSuccess) {
        cudaEventDestroy(a);
        return e;
    }
    k_limb_form<kForm><<<sms, kThreadsLF, kSmemLF, s>>>(iters / 10 + 1, out);   // warm-up
    cudaEventRecord(a, s);
    k_limb_form<kForm><<<sms, kThreadsLF, kSmemLF, s>>>(iters, out);
    cudaEventRecord(b, s);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e == cudaSuccess) *per_s = (double)sms * kThreadsLF * iters / (ms * 1e-3);
    return e;
}

}  // namespace

// products per second of each limb layout on the whole device (one block per
// SM); `out` must hold sms x 384 words
cudaError_t measure_limb_forms(int sms, int iters, uint32_t* out, cudaStream_t s, double* per_s) {
    cudaError_t e = time_form<0>(sms, iters, out, s, per_s);
    if (e == cudaSuccess) e = time_form<1>(sms, iters, out, s, per_s + 1);
    if (e == cudaSuccess) e = time_form<2>(sms, iters, out, s, per_s + 2);
    return e;
}

}  // namespace bls
