// Fp inverse by the binary extended Euclidean algorithm, shared by the verify
// kernels (the final exponentiation's one inversion) and the hash to G1 (the
// affine result): a few hundred shift-and-subtract passes on 12-limb values
// instead of the ~570 Montgomery multiplications of a Fermat power.  The
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
    uint32_t d[12], br = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        uint64_t t = (uint64_t)a[i] - b[i] - br;
        d[i] = (uint32_t)t;
        br = (uint32_t)(t >> 63);
    }
    (void)d;
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

}  // namespace bls
