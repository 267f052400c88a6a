// Device kernels of the verify path and their launchers.
//
//   k_verify          one verification per thread: optional G1 decode of the
//                     signature, two-pair Miller loop, final exponentiation,
//                     identity test (gpu-crypto/cuda/api.cu:80-109).  The
//                     generator's line table is read by every thread at the same
//                     address (broadcast); public-key tables are read per item.
//   k_g1_decompress   one 48-byte point per thread (cuda/decompress.cu:140-188)
//                     plus the from_compressed checks.
//   k_g2_decompress   one 96-byte compressed public key per thread, with the
//                     G2Affine::from_compressed checks (no reference kernel: the
//                     reference's callers decode keys on the CPU).
//   k_g2_prepare      one G2 line table per thread (cuda/test_miller_v2.cu:148-229).
#include <cuda_runtime.h>

#include "g1.cuh"
#include "g2.cuh"
#include "g2prep.cuh"
#include "internal.h"

namespace bls {

__global__ void __launch_bounds__(kVerifyThreads) k_verify(VerifyArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    fp sx, sy;
    bool sig_id;
    if (a.sig_compressed) {
        int32_t st = g1_decode((const uint8_t*)a.sigs + 48 * (size_t)i, sx, sy, sig_id, true);
        if (st != ST_OK) {
            a.results[i] = -st;
            if (a.ml_out) for (int k = 0; k < 72; ++k) a.ml_out[72 * (size_t)i + k] = 0;
            if (a.gt_out) for (int k = 0; k < 72; ++k) a.gt_out[72 * (size_t)i + k] = 0;
            return;
        }
    } else {
        const uint64_t* s = (const uint64_t*)a.sigs + 12 * (size_t)i;
        sx = fp_load_u64(s);
        sy = fp_load_u64(s + 6);
        sig_id = g1_limbs_identity(sx, sy);
    }
    const uint64_t* h = a.nhms + 12 * (size_t)i;
    fp hx = fp_load_u64(h), hy = fp_load_u64(h + 6);
    bool h_id = g1_limbs_identity(hx, hy);
    int64_t pk = a.pk_index ? (int64_t)a.pk_index[i] : (int64_t)i;
    if (!key_index_ok(pk, a.check_keys, a.n_keys)) {   // no table read for it
        a.results[i] = -ST_BAD_KEY_INDEX;
        if (a.ml_out) for (int k = 0; k < 72; ++k) a.ml_out[72 * (size_t)i + k] = 0;
        if (a.gt_out) for (int k = 0; k < 72; ++k) a.gt_out[72 * (size_t)i + k] = 0;
        return;
    }
    bool pk_id = a.pk_identity ? a.pk_identity[pk] != 0 : false;
    fp12 ml = miller_loop_2(sx, sy, a.g2, sig_id, hx, hy, a.pk_tables + BLS_COEFF_U64 * pk, h_id || pk_id);
    fp12 gt = final_exponentiation(ml);
    a.results[i] = fp12_is_one(gt) ? 1 : 0;
    if (a.ml_out) fp12_store_u64(a.ml_out + 72 * (size_t)i, ml);
    if (a.gt_out) fp12_store_u64(a.gt_out + 72 * (size_t)i, gt);
}

__global__ void __launch_bounds__(128) k_g1_decompress(const uint8_t* in, int n, uint64_t* xy, int32_t* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fp x, y;
    bool id;
    int32_t st = g1_decode(in + 48 * (size_t)i, x, y, id, true);
    status[i] = st;
    fp_store_u64(xy + 12 * (size_t)i, x);
    fp_store_u64(xy + 12 * (size_t)i + 6, y);
}

// The serving ring's decoder: the same decode, grid-stride, in blocks that
// each hold a whole SM.  Its dynamic shared memory (unused) is more than half
// of an SM's, so two of its blocks never share an SM and none shares one with
// a resident ring-kernel block; a launch of b blocks therefore occupies at
// most b SMs, where blocks of the plain decoder would spread over every SM
// that frees up and keep the ring kernel's whole-SM blocks from starting.
constexpr int kDecSmThreads = 384;
constexpr size_t kDecSmSmem = 116 * 1024;
// check_subgroup false: every check but the subgroup test, which
// k_g1_subgroup_sm then runs over the decoded points.
__global__ void __launch_bounds__(kDecSmThreads, 1) k_g1_decompress_sm(const uint8_t* in, int n, uint64_t* xy,
                                                                     int32_t* status, bool check_subgroup) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        fp x, y;
        bool id;
        const int32_t st = g1_decode(in + 48 * (size_t)i, x, y, id, check_subgroup);
        status[i] = st;
        fp_store_u64(xy + 12 * (size_t)i, x);
        fp_store_u64(xy + 12 * (size_t)i + 6, y);
    }
}

// The subgroup test of points decoded without it, in the same whole-SM
// blocks: sub[i] = ST_NOT_IN_SUBGROUP for a point outside G1, else 0 (also
// for a point whose decode failed, or the identity).
__global__ void __launch_bounds__(kDecSmThreads, 1) k_g1_subgroup_sm(const uint64_t* xy, const int32_t* status, int n,
                                                                   int32_t* sub) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int32_t r = 0;
        if (status[i] == ST_OK) {
            const fp x = fp_load_u64(xy + 12 * (size_t)i), y = fp_load_u64(xy + 12 * (size_t)i + 6);
            if (!g1_limbs_identity(x, y) && !g1_in_subgroup(x, y)) r = ST_NOT_IN_SUBGROUP;
        }
        sub[i] = r;
    }
}

// q: 24 x uint64 per key (x.c0, x.c1, y.c0, y.c1 Montgomery; zeros for the
// identity and for a failure); identity (optional): 1 for the identity.
__global__ void __launch_bounds__(64) k_g2_decompress(const uint8_t* in, int n, uint64_t* q, int32_t* status,
                                                      uint8_t* identity) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    fp2 x, y;
    bool id;
    int32_t st = g2_decode(in + 96 * (size_t)i, x, y, id);
    status[i] = st;
    uint64_t* qi = q + 24 * (size_t)i;
    store_fp2(qi, x);
    store_fp2(qi + 12, y);
    if (identity) identity[i] = (st == ST_OK && id) ? 1 : 0;
}

__global__ void __launch_bounds__(64) k_g2_prepare(const uint64_t* q, int n, uint64_t* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t* qi = q + 24 * (size_t)i;
    fp2 qx = {fp_load_u64(qi), fp_load_u64(qi + 6)};
    fp2 qy = {fp_load_u64(qi + 12), fp_load_u64(qi + 18)};
    g2_prepare(qx, qy, out + BLS_COEFF_U64 * (size_t)i);
}

// Small key sets: one line table per block, one row per thread, so a table's
// latency is about one row's work.  Every row (c0, c1, c2) becomes
// (c0 / c2, c1 / c2, 1), 1 / c2 = conj(c2) / |c2| with the norms of a warp's
// 32 rows inverted together (fp_inverse_warp: one binary Euclid per warp, not
// one divergent Euclid per row), and the
// Miller correction factor prod_i c2_i^(2^s_i) is formed in parallel: s_i is
// the number of squarings that follow line i in the Miller loop's order of
// lines and squarings (api.cu:30-52), each thread squares its c2 s_i times,
// and a product tree in shared memory multiplies the 68 powers.  Every
// operation returns the canonical representative, so the values do not depend
// on the order of the products.  A table with a zero c2 is copied unchanged
// and flagged.
constexpr int kNormRows = 68;
constexpr int kNormThreads = 128;

// squarings after line `row` of the Miller loop: lines taken in iteration b
// (b = 61 .. 0 over the bits of |x| >> 1 below the leading one) are squared
// b + 1 times; the last line (after the loop) none
__device__ __forceinline__ int squarings_after(int row) {
    const uint64_t xabs = 0xd201000000010000ULL;
    int ci = 0;
    for (int b = 61; b >= 0; --b) {
        if (ci++ == row) return b + 1;
        if (((xabs >> 1) >> b) & 1) {
            if (ci++ == row) return b + 1;
        }
    }
    return 0;
}

__global__ void __launch_bounds__(kNormThreads) k_lines_normalize_rows(const uint64_t* raw, int n, uint64_t* norm,
                                                                  uint64_t* corr, uint8_t* bad) {
    __shared__ uint64_t pw[kNormRows][12];
    const int t = blockIdx.x, i = threadIdx.x;
    if (t >= n) return;   // the whole block leaves together
    const uint64_t* in = raw + BLS_COEFF_U64 * (size_t)t;
    uint64_t* out = norm + BLS_COEFF_U64 * (size_t)t;
    fp2 c2 = fp2_one();
    if (i < kNormRows) c2 = fp2{fp_load_u64(in + 36 * i + 24), fp_load_u64(in + 36 * i + 30)};
    const bool zero = __syncthreads_or(i < kNormRows && fp2_is_zero(c2));
    if (zero) {
        for (int k = i; k < BLS_COEFF_U64; k += kNormThreads) out[k] = in[k];
        if (i == 0) {
            store_fp2(corr + 12 * (size_t)t, fp2_one());
            bad[t] = 1;
        }
        return;
    }
    // every thread of the block takes part in its warp's inversion (rows past
    // the table contribute a one)
    const fp c2_norm = fp_add(fp_sqr(c2.c0), fp_sqr(c2.c1));
    const fp r3 = fp_mul(fp_rr(), fp_rr());                        // R^3 mod p
    const fp ninv = fp_inverse_warp(c2_norm, r3.w);
    if (i < kNormRows) {
        const fp2 inv = {fp_mul(c2.c0, ninv), fp_neg(fp_mul(c2.c1, ninv))};
        const fp2 c0 = {fp_load_u64(in + 36 * i), fp_load_u64(in + 36 * i + 6)};
        const fp2 c1 = {fp_load_u64(in + 36 * i + 12), fp_load_u64(in + 36 * i + 18)};
        store_fp2(out + 36 * i, fp2_mul(c0, inv));
        store_fp2(out + 36 * i + 12, fp2_mul(c1, inv));
        store_fp2(out + 36 * i + 24, fp2_one());
        fp2 p = c2;
        for (int k = squarings_after(i); k > 0; --k) p = fp2_sqr(p);
        store_fp2(pw[i], p);
    }
    __syncthreads();
    for (int stride = 1; stride < kNormRows; stride *= 2) {
        if (i % (2 * stride) == 0 && i + stride < kNormRows) {
            const fp2 a = {fp_load_u64(pw[i]), fp_load_u64(pw[i] + 6)};
            const fp2 b = {fp_load_u64(pw[i + stride]), fp_load_u64(pw[i + stride] + 6)};
            store_fp2(pw[i], fp2_mul(a, b));
        }
        __syncthreads();
    }
    if (i == 0) {
        store_fp2(corr + 12 * (size_t)t, fp2{fp_load_u64(pw[0]), fp_load_u64(pw[0] + 6)});
        bad[t] = 0;
    }
}

// Large key sets: one line table per thread, every row (c0, c1, c2) becomes (c0 / c2, c1 / c2, 1)
// (inverses by Montgomery's batch trick: one Fp2 inverse per table), and the
// Miller correction factor prod_i c2_i^(2^(squarings after line i)) follows the
// Miller loop's order of lines and squarings (api.cu:30-52).  A table with a
// zero c2 is copied unchanged and flagged.
__global__ void __launch_bounds__(64) k_lines_normalize_table(const uint64_t* raw, int n, uint64_t* norm, uint64_t* corr,
                                                      uint8_t* bad) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t* in = raw + BLS_COEFF_U64 * (size_t)t;
    uint64_t* out = norm + BLS_COEFF_U64 * (size_t)t;
    constexpr int kRows = 68;
    auto c2_of = [&](int i) { return fp2{fp_load_u64(in + 36 * i + 24), fp_load_u64(in + 36 * i + 30)}; };
    // prefix products of c2 in the output's c2 slots
    fp2 pre = fp2_one();
    for (int i = 0; i < kRows; ++i) {
        pre = fp2_mul(pre, c2_of(i));
        store_fp2(out + 36 * i + 24, pre);
    }
    if (fp2_is_zero(pre)) {
        for (int i = 0; i < BLS_COEFF_U64; ++i) out[i] = in[i];
        store_fp2(corr + 12 * (size_t)t, fp2_one());
        bad[t] = 1;
        return;
    }
    fp2 inv = fp2_inv(pre);   // (c2_0 ... c2_67)^-1
    for (int i = kRows - 1; i >= 0; --i) {
        fp2 c2 = c2_of(i);
        fp2 inv_i = i ? fp2_mul(inv, fp2{fp_load_u64(out + 36 * (i - 1) + 24), fp_load_u64(out + 36 * (i - 1) + 30)})
                      : inv;
        inv = fp2_mul(inv, c2);
        fp2 c0 = {fp_load_u64(in + 36 * i), fp_load_u64(in + 36 * i + 6)};
        fp2 c1 = {fp_load_u64(in + 36 * i + 12), fp_load_u64(in + 36 * i + 18)};
        store_fp2(out + 36 * i, fp2_mul(c0, inv_i));
        store_fp2(out + 36 * i + 12, fp2_mul(c1, inv_i));
    }
    for (int i = 0; i < kRows; ++i) store_fp2(out + 36 * i + 24, fp2_one());
    // correction factor
    const uint64_t xabs = 0xd201000000010000ULL;
    fp2 cf = fp2_one();
    int ci = 0;
    for (int b = 61; b >= 0; --b) {
        cf = fp2_mul(cf, c2_of(ci++));
        if (((xabs >> 1) >> b) & 1) cf = fp2_mul(cf, c2_of(ci++));
        cf = fp2_sqr(cf);
    }
    cf = fp2_mul(cf, c2_of(ci));
    store_fp2(corr + 12 * (size_t)t, cf);
    bad[t] = 0;
}

// A key set of at most kRowsMaxTables tables takes the row-parallel form (low
// latency: one block per table); a larger one the table-per-thread form
// (least work: the whole set in one wave, where the row form would square each
// row's c2 separately and take many waves).
constexpr int kRowsMaxTables = 2048;

cudaError_t launch_lines_normalize(const uint64_t* raw, int n, uint64_t* norm, uint64_t* corr, uint8_t* bad,
                                   cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (n <= kRowsMaxTables)
        k_lines_normalize_rows<<<n, kNormThreads, 0, s>>>(raw, n, norm, corr, bad);
    else
        k_lines_normalize_table<<<(n + 63) / 64, 64, 0, s>>>(raw, n, norm, corr, bad);
    return cudaGetLastError();
}

cudaError_t launch_verify(const VerifyArgs& a, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    if (a.sig_xy) return cudaErrorInvalidValue;
    int blocks = (a.n + kVerifyThreads - 1) / kVerifyThreads;
    k_verify<<<blocks, kVerifyThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_g1_decompress(const uint8_t* in, int n, uint64_t* xy, int32_t* status, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_g1_decompress<<<(n + 127) / 128, 128, 0, s>>>(in, n, xy, status);
    return cudaGetLastError();
}

static int dec_sm_blocks(int n, int max_sms) {
    int blocks = (n + kDecSmThreads - 1) / kDecSmThreads;
    if (blocks > max_sms) blocks = max_sms;
    return blocks < 1 ? 1 : blocks;
}

cudaError_t launch_g1_decompress_sms(const uint8_t* in, int n, uint64_t* xy, int32_t* status, int max_sms,
                                     bool check_subgroup, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    static const cudaError_t attr = cudaFuncSetAttribute(
        k_g1_decompress_sm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDecSmSmem);
    if (attr != cudaSuccess) return attr;
    k_g1_decompress_sm<<<dec_sm_blocks(n, max_sms), kDecSmThreads, kDecSmSmem, s>>>(in, n, xy, status,
                                                                                  check_subgroup);
    return cudaGetLastError();
}

cudaError_t launch_g1_subgroup_sms(const uint64_t* xy, const int32_t* status, int n, int32_t* sub, int max_sms,
                                   cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    static const cudaError_t attr = cudaFuncSetAttribute(
        k_g1_subgroup_sm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDecSmSmem);
    if (attr != cudaSuccess) return attr;
    k_g1_subgroup_sm<<<dec_sm_blocks(n, max_sms), kDecSmThreads, kDecSmSmem, s>>>(xy, status, n, sub);
    return cudaGetLastError();
}

cudaError_t launch_g2_decompress(const uint8_t* in, int n, uint64_t* q, int32_t* status, uint8_t* identity,
                                 cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_g2_decompress<<<(n + 63) / 64, 64, 0, s>>>(in, n, q, status, identity);
    return cudaGetLastError();
}

cudaError_t launch_g2_prepare(const uint64_t* q, int n, uint64_t* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_g2_prepare<<<(n + 63) / 64, 64, 0, s>>>(q, n, out);
    return cudaGetLastError();
}

}  // namespace bls
