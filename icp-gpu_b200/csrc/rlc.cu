// Random-linear-combination batch verification (opt-in).  For items
// (sig_i, -H(m_i), pk_i) and random 64-bit scalars r_i, every item verifies
// iff (with probability >= 1 - 2^-64 when one does not)
//
//     e(sum_i r_i sig_i, G2) * prod_k e(sum_{i: pk_i = k} r_i (-H(m_i)), pk_k) == 1,
//
// one pair per distinct key plus one, and a single shared final
// exponentiation instead of one per item.  The reference verifies item by item
// (gpu-crypto/cuda/api.cu:94-109); this mode is the batch-verification step of
// Bellare, Garay and Rabin (EUROCRYPT 1998) as used for BLS (Boneh, Drijvers,
// Neven, ASIACRYPT 2018).  The sum is sound only for points in G1, so every
// point is checked (on the curve, canonical, in the subgroup); an item that
// fails a check sends the whole batch to the per-item path, as does a failed
// combined check.
//
//   k_rlc_scale   four threads per item: [r] sig, [r] (-H(m)) and the two
//                 points' checks, at the same time; r = a + lambda b with
//                 32-bit a, b and lambda the GLV eigenvalue (2^64 distinct r)
//   k_rlc_tiles   partial sums of up to kTile items of one key (in key order)
//   k_rlc_final   per-key sums of the tiles, the signature sum, affine points
//                 laid out as verify-kernel items (item k: pair 1 = the
//                 signature sum for k = 0, else the identity; pair 2 = key k)
//   k_gt_product  product of the items' final exponentiations, == 1?
#include <cuda_runtime.h>

#include "g1.cuh"
#include "internal.h"
#include "pairing.cuh"

namespace bls {

namespace {

constexpr int kTileThreads = 128;

__device__ __forceinline__ void store_j(uint32_t* d, const g1j& p) {
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        d[i] = p.X.w[i];
        d[12 + i] = p.Y.w[i];
        d[24 + i] = p.Z.w[i];
    }
}

__device__ __forceinline__ g1j load_j(const uint32_t* s) {
    g1j p;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        p.X.w[i] = s[i];
        p.Y.w[i] = s[12 + i];
        p.Z.w[i] = s[24 + i];
    }
    return p;
}

__device__ __forceinline__ g1j g1j_identity() { return {fp_one(), fp_one(), fp_zero()}; }

// [a + lambda b] (x, y) for an affine point of G1 and 32-bit a, b, where
// phi(x, y) = (beta x, y) = [lambda] (x, y) (lambda = -x^2 mod r, the
// eigenvalue g1_in_subgroup tests).  Shamir's trick over the table
// (x, y), phi = (beta x, y) and (x, y) + phi = (beta^2 x, -y) (the two points
// share y, so their sum is -phi^2): 32 doublings and at most 32 mixed additions,
// against 63 and up to 63 for a plain 64-bit scalar.
static __device__ __noinline__ g1j g1_mul_glv(const fp& x, const fp& y, uint32_t a, uint32_t b) {
    const uint64_t bv[6] = {0x30f1361b798a64e8ULL, 0xf3b8ddab7ece5a2aULL, 0x16a8ca3ac61577f7ULL,
                            0xc26a2ff874fd029bULL, 0x3636b76660701c6eULL, 0x051ba4ab241b6160ULL};  // beta
    const fp beta = fp_load_u64(bv);
    const fp bx = fp_mul(beta, x), b2x = fp_mul(beta, bx), ny = fp_neg(y);
    g1j r = g1j_identity();
    for (int i = 31; i >= 0; --i) {
        r = g1j_dbl(r);
        const uint32_t sel = ((a >> i) & 1u) | (((b >> i) & 1u) << 1);
        if (sel) {
            const fp tx = sel == 1 ? x : (sel == 2 ? bx : b2x);
            const fp ty = sel == 3 ? ny : y;
            r = g1j_add_affine(r, tx, ty);
        }
    }
    return r;
}

// canonical limbs, on y^2 = x^3 + 4, in the order-r subgroup
static __device__ __noinline__ bool g1_point_ok(const fp& x, const fp& y) {
    if (fp_raw_geq_p(x) || fp_raw_geq_p(y)) return false;
    if (!fp_eq(fp_sqr(y), fp_add(fp_mul(fp_sqr(x), x), fp_four()))) return false;
    return g1_in_subgroup(x, y);
}

// A block of four warps takes 32 items; warp w has role w for all of them
// (0: [r] sig, 1: [r] nhm, 2: sig checks, 3: nhm checks), so a warp never
// splits between the scalar multiplication and the checks.
__global__ void __launch_bounds__(128) k_rlc_scale(const uint64_t* sig_xy, const int32_t* status,
                                                   const uint64_t* nhms, const uint64_t* r, int n, int check_sig,
                                                   uint32_t* pts, uint8_t* bad, int* counters) {
    const int role = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    if (i >= n) return;
    const bool dead = status && status[i] != 0;
    const bool nhm_side = role & 1;
    const uint64_t* src = nhm_side ? nhms + 12 * (size_t)i : sig_xy + 12 * (size_t)i;
    const fp x = fp_load_u64(src), y = fp_load_u64(src + 6);
    const bool id = g1_limbs_identity(x, y);
    if (role < 2) {
        const uint64_t k = r[i];
        const g1j p = (dead || id) ? g1j_identity() : g1_mul_glv(x, y, (uint32_t)k, (uint32_t)(k >> 32));
        store_j(pts + 72 * (size_t)i + 36 * role, p);
    } else {
        bool ok = true;
        if (!dead && !id && (nhm_side || check_sig)) ok = g1_point_ok(x, y);
        bad[2 * (size_t)i + (role & 1)] = ok ? 0 : 1;
        if (!ok) atomicAdd(counters + 1, 1);
    }
}

// tile t: items order[tile[3t] .. tile[3t + 1]) (one key); partials: signature
// sum then key sum, 72 words per tile
__global__ void __launch_bounds__(kTileThreads) k_rlc_tiles(const uint32_t* pts, const int32_t* order,
                                                            const int32_t* tiles, uint32_t* partials) {
    __shared__ uint32_t sm[kTileThreads][36];
    const int a = tiles[3 * blockIdx.x], b = tiles[3 * blockIdx.x + 1];
    g1j acc[2];
    for (int s = 0; s < 2; ++s) {
        acc[s] = g1j_identity();
        for (int k = a + threadIdx.x; k < b; k += kTileThreads)
            acc[s] = g1j_add(acc[s], load_j(pts + 72 * (size_t)order[k] + 36 * s));
        store_j(sm[threadIdx.x], acc[s]);
        __syncthreads();
        for (int w = kTileThreads / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) {
                acc[s] = g1j_add(acc[s], load_j(sm[threadIdx.x + w]));
                store_j(sm[threadIdx.x], acc[s]);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) store_j(partials + 72 * (size_t)blockIdx.x + 36 * s, acc[s]);
        __syncthreads();
    }
}

__device__ __forceinline__ void store_affine(uint64_t* d, const g1j& p) {
    fp x = fp_zero(), y = fp_one();   // the identity: x = 0, y = R mod p
    if (!fp_is_zero(p.Z)) {
        const uint64_t pm2[6] = {0xb9feffffffffaaa9ULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                                 0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};  // p - 2
        const fp zi = fp_pow_u64(p.Z, pm2, 381), zi2 = fp_sqr(zi);
        x = fp_mul(p.X, zi2);
        y = fp_mul(p.Y, fp_mul(zi2, zi));
    }
    fp_store_u64(d, x);
    fp_store_u64(d + 6, y);
}

// key k's tiles are key_tile[k] .. key_tile[k + 1]; out_sigs / out_nhms: K items
__global__ void __launch_bounds__(256) k_rlc_final(const uint32_t* partials, int ntiles, const int32_t* key_tile,
                                                   int nkeys, uint64_t* out_sigs, uint64_t* out_nhms) {
    __shared__ uint32_t sm[256][36];
    g1j s = g1j_identity();
    for (int t = threadIdx.x; t < ntiles; t += 256) s = g1j_add(s, load_j(partials + 72 * (size_t)t));
    store_j(sm[threadIdx.x], s);
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s = g1j_add(s, load_j(sm[threadIdx.x + w]));
            store_j(sm[threadIdx.x], s);
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < nkeys; k += 256) {
        g1j h = g1j_identity();
        for (int t = key_tile[k]; t < key_tile[k + 1]; ++t) h = g1j_add(h, load_j(partials + 72 * (size_t)t + 36));
        store_affine(out_nhms + 12 * (size_t)k, h);
        if (k == 0) store_affine(out_sigs, s);
        else store_affine(out_sigs + 12 * (size_t)k, g1j_identity());
    }
}

// product of n Gt values (in place), counters[0] = 1 when it is one
__global__ void __launch_bounds__(128) k_gt_product(uint64_t* gt, int n, int* counters) {
    for (int w = 1; w < n; w <<= 1) {
        for (int i = 2 * w * threadIdx.x; i + w < n; i += 2 * w * blockDim.x)
            fp12_store_u64(gt + 72 * (size_t)i, fp12_mul(fp12_load_u64(gt + 72 * (size_t)i),
                                                         fp12_load_u64(gt + 72 * (size_t)(i + w))));
        __syncthreads();
    }
    if (threadIdx.x == 0) counters[0] = fp12_is_one(fp12_load_u64(gt)) ? 1 : 0;
}

}  // namespace

cudaError_t launch_rlc(const RlcArgs& a, cudaStream_t s) {
    if (a.n <= 0 || a.ntiles <= 0 || a.nkeys <= 0) return cudaErrorInvalidValue;
    k_rlc_scale<<<(unsigned)((a.n + 31) / 32), 128, 0, s>>>(a.sig_xy, a.status, a.nhms, a.r, a.n, a.check_sig,
                                                                 a.pts, a.bad, a.counters);
    k_rlc_tiles<<<a.ntiles, kTileThreads, 0, s>>>(a.pts, a.order, a.tiles, a.partials);
    k_rlc_final<<<1, 256, 0, s>>>(a.partials, a.ntiles, a.key_tile, a.nkeys, a.agg_sigs, a.agg_nhms);
    return cudaGetLastError();
}

cudaError_t launch_gt_product(uint64_t* gt, int n, int* counters, cudaStream_t s) {
    if (n <= 0) return cudaErrorInvalidValue;
    k_gt_product<<<1, 128, 0, s>>>(gt, n, counters);
    return cudaGetLastError();
}

}  // namespace bls
