// Fp inverse by the binary extended Euclidean algorithm, shared by the verify
// kernels (the final exponentiation's one inversion) and the hash to G1 (the
// affine result): a few hundred shift-and-subtract passes on 12-limb values
// instead of the ~570 Montgomery multiplications of a Fermat power; and its
// warp-wide form, the inverses of a whole warp's values for one Euclid.  The
// caller passes R^3 mod p (12 limbs, from its generated constants).
#pragma once
#include "fp.cuh"

namespace bls {

// ---------------------------------------------------------------------------
// Fp inverse by the binary extended Euclidean algorithm (Knuth, TAOCP vol. 2,
// 4.5.2; Menezes et al., Handbook of Applied Cryptography, Alg. 14.61 in its
// modular form).  Variable time: the inputs are public.  x: Montgomery form
// of a (any value below 2^381 + p); returns a^-1 in Montgomery form (0 for 0).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool u_is_one(const uint32_t* u) {
    uint32_t o = u[0] ^ 1u;
#pragma unroll
    for (int i = 1; i < 12; ++i) o |= u[i];
    return o == 0;
}
__device__ __forceinline__ bool geq12(const uint32_t* a, const uint32_t* b) {
    uint32_t br = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) br = (uint32_t)(((uint64_t)a[i] - b[i] - br) >> 63);
    return br == 0;
}
__device__ __forceinline__ void sub12(uint32_t* a, const uint32_t* b) {
    uint32_t br = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint64_t t = (uint64_t)a[i] - b[i] - br;
        a[i] = (uint32_t)t;
        br = (uint32_t)(t >> 63);
    }
}
// x = x / 2 mod p for x < p
__device__ __forceinline__ void half_mod(uint32_t* x) {
    const uint32_t P_[12] = {BLS_P0, BLS_P1, BLS_P2, BLS_P3, BLS_P4, BLS_P5,
                             BLS_P6, BLS_P7, BLS_P8, BLS_P9, BLS_P10, BLS_P11};
    const uint32_t odd = 0u - (x[0] & 1u);
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint64_t t = (uint64_t)x[i] + (P_[i] & odd) + c;
        x[i] = (uint32_t)t;
        c = (uint32_t)(t >> 32);
    }
#pragma unroll
    for (int i = 0; i < 11; ++i) x[i] = __funnelshift_r(x[i], x[i + 1], 1);
    x[11] = (x[11] >> 1) | (c << 31);
}
__device__ __forceinline__ void shr1(uint32_t* u) {
#pragma unroll
    for (int i = 0; i < 11; ++i) u[i] = __funnelshift_r(u[i], u[i + 1], 1);
    u[11] >>= 1;
}
// x1 = x1 - x2 mod p (both < p)
__device__ __forceinline__ void sub_mod(uint32_t* x1, const uint32_t* x2) {
    const uint32_t P_[12] = {BLS_P0, BLS_P1, BLS_P2, BLS_P3, BLS_P4, BLS_P5,
                             BLS_P6, BLS_P7, BLS_P8, BLS_P9, BLS_P10, BLS_P11};
    uint32_t br = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint64_t t = (uint64_t)x1[i] - x2[i] - br;
        x1[i] = (uint32_t)t;
        br = (uint32_t)(t >> 63);
    }
    const uint32_t m = 0u - br;
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint64_t t = (uint64_t)x1[i] + (P_[i] & m) + c;
        x1[i] = (uint32_t)t;
        c = (uint32_t)(t >> 32);
    }
}

static __device__ __noinline__ fp fp_inverse_mont(fp x, const uint32_t* kR3) {
    // canonical representative (x < 2^381 + p < 3p)
    uint32_t d[12];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        uint32_t br = sub_p(d, x.w);
#pragma unroll
        for (int i = 0; i < 12; ++i) x.w[i] = br ? x.w[i] : d[i];
    }
    if (fp_is_zero(x)) return x;
    uint32_t u[12], v[12], x1[12], x2[12];
    const uint32_t P_[12] = {BLS_P0, BLS_P1, BLS_P2, BLS_P3, BLS_P4, BLS_P5,
                             BLS_P6, BLS_P7, BLS_P8, BLS_P9, BLS_P10, BLS_P11};
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        u[i] = x.w[i];
        v[i] = P_[i];
        x1[i] = 0;
        x2[i] = 0;
    }
    x1[0] = 1;
    // u, v stay odd-or-positive and gcd(u, v) = 1; every pass of the outer
    // loop removes at least one bit from u or v, so 2 * 381 + 2 passes end it
    for (int iter = 0; iter < 800 && !u_is_one(u) && !u_is_one(v); ++iter) {
        for (int k = 0; k < 384 && (u[0] & 1u) == 0; ++k) {
            shr1(u);
            half_mod(x1);
        }
        for (int k = 0; k < 384 && (v[0] & 1u) == 0; ++k) {
            shr1(v);
            half_mod(x2);
        }
        if (geq12(u, v)) {
            sub12(u, v);
            sub_mod(x1, x2);
        } else {
            sub12(v, u);
            sub_mod(x2, x1);
        }
    }
    fp r;
    const bool uone = u_is_one(u);
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = uone ? x1[i] : x2[i];
    fp r3;
#pragma unroll
    for (int i = 0; i < 12; ++i) r3.w[i] = kR3[i];
    return fp_mul(r, r3);                              // r R^3 / R: Montgomery form of a^-1
}


__device__ __forceinline__ fp shfl_fp(const fp& v, int src) {
    fp r;
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = __shfl_sync(0xffffffffu, v.w[i], src);
    return r;
}
__device__ __forceinline__ fp shfl_up_fp(const fp& v, int d) {
    fp r;
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = __shfl_up_sync(0xffffffffu, v.w[i], d);
    return r;
}
__device__ __forceinline__ fp shfl_down_fp(const fp& v, int d) {
    fp r;
#pragma unroll
    for (int i = 0; i < 12; ++i) r.w[i] = __shfl_down_sync(0xffffffffu, v.w[i], d);
    return r;
}

// The Fp inverses of the 32 lanes' values by Montgomery's simultaneous-
// inversion trick over the warp: prefix and suffix products by shuffles (five
// multiplications each), one inverse of the whole product, which every lane
// computes from the same value so the binary Euclid's data-dependent branches
// never split the warp, and two multiplications per lane.  Each lane's own
// binary Euclid on its own value would diverge and serialise the warp's 32
// paths.  Every lane of the warp must call it together (full-mask shuffles).
// z: any value below 2^381 + p; 0 gives 0, as fp_inverse_mont does (a zero
// stands in as one in the products); kR3: R^3 mod p.
static __device__ __noinline__ fp fp_inverse_warp(fp z, const uint32_t* kR3) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 2; ++k) {          // canonical: fp_mul wants inputs below p
        uint32_t d[12];
        const uint32_t br = sub_p(d, z.w);
#pragma unroll
        for (int i = 0; i < 12; ++i) z.w[i] = br ? z.w[i] : d[i];
    }
    const bool zero = fp_is_zero(z);
    const fp x = zero ? fp_one() : z;
    fp pre = x, suf = x;                    // inclusive prefix and suffix products
    for (int d = 1; d < 32; d <<= 1) {
        const fp y = shfl_up_fp(pre, d);
        if (lane >= d) pre = fp_mul_ool(y, pre);
    }
    for (int d = 1; d < 32; d <<= 1) {
        const fp y = shfl_down_fp(suf, d);
        if (lane + d < 32) suf = fp_mul_ool(suf, y);
    }
    const fp total = shfl_fp(pre, 31);
    fp before = shfl_up_fp(pre, 1), after = shfl_down_fp(suf, 1);
    if (lane == 0) before = fp_one();
    if (lane == 31) after = fp_one();
    const fp t = fp_inverse_mont(total, kR3);
    const fp r = fp_mul_ool(fp_mul_ool(t, before), after);
    return zero ? fp_zero() : r;
}

}  // namespace bls
