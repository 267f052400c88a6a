// Two-pair optimal-ate Miller loop over precomputed G2 line coefficients and
// the final exponentiation, as the reference verifier evaluates them
// (gpu-crypto/cuda/api.cu:22-91, itself mirroring ic_bls12_381 0.10.1).
//
// Line-coefficient table layout (ic_bls12_381 G2Prepared): 68 coefficients,
// coefficient i at u64 offset 36*i holding three Fp2 (c0, c1, c2), each Fp2 as
// (c0[6], c1[6]) little-endian Montgomery limbs.  63 doubling and 5 addition
// lines in loop order for |x| = 0xd201000000010000.
#pragma once
#include "tower.cuh"

namespace bls {

#define BLS_X_ABS 0xd201000000010000ULL
#define BLS_NCOEFFS 68
#define BLS_COEFF_U64 2448

__device__ __forceinline__ fp2 load_fp2(const uint64_t* p) {
    return {fp_load_u64(p), fp_load_u64(p + 6)};
}

// f <- f * line(P) for coefficient `idx` of table `co` (api.cu:22-27, 37-38)
__device__ __forceinline__ void line_eval(fp12& f, const uint64_t* __restrict__ co, int idx,
                                          const fp& px, const fp& py) {
    const uint64_t* b = co + 36 * idx;
    fp2 c0 = load_fp2(b), c1 = load_fp2(b + 12), c2 = load_fp2(b + 24);
    f = fp12_mul_by_014(f, c2, fp2_mul_fp(c1, px), fp2_mul_fp(c0, py));
}

// prod over both pairs of the Miller function, then conjugate (x < 0).
// A pair whose `skip` is set contributes nothing, the ic_bls12_381 rule for
// an identity point on either side.
static __device__ __noinline__ fp12 miller_loop_2(const fp& p1x, const fp& p1y, const uint64_t* q1, bool skip1,
                                           const fp& p2x, const fp& p2y, const uint64_t* q2, bool skip2) {
    fp12 f = fp12_one();
    int ci = 0;
    bool found = false;
    for (int b = 63; b >= 0; --b) {
        bool bit = (((BLS_X_ABS >> 1) >> b) & 1) == 1;
        if (!found) { found = bit; continue; }
        if (!skip1) line_eval(f, q1, ci, p1x, p1y);
        if (!skip2) line_eval(f, q2, ci, p2x, p2y);
        ++ci;
        if (bit) {
            if (!skip1) line_eval(f, q1, ci, p1x, p1y);
            if (!skip2) line_eval(f, q2, ci, p2x, p2y);
            ++ci;
        }
        f = fp12_sqr(f);
    }
    if (!skip1) line_eval(f, q1, ci, p1x, p1y);
    if (!skip2) line_eval(f, q2, ci, p2x, p2y);
    return fp12_conj(f);
}

// f^x (x negative): square-and-multiply over |x| with the cyclotomic square,
// then conjugate (api.cu:54-63).  The leading 1 bit starts from t = f instead
// of multiplying 1 by f; both give the same value.
static __device__ __noinline__ fp12 cyc_exp(const fp12& f) {
    fp12 t = f;
    for (int i = 62; i >= 0; --i) {
        t = fp12_cyclotomic_sqr(t);
        if ((BLS_X_ABS >> i) & 1) t = fp12_mul(t, f);
    }
    return fp12_conj(t);
}

// api.cu:65-78: easy part f^((p^6-1)(p^2+1)), then the hard-part chain of
// ic_bls12_381 (same exponent, so the same Gt element bit for bit).
static __device__ __noinline__ fp12 final_exponentiation(const fp12& fi) {
    fp12 f = fi;
    fp12 t0 = fp12_conj(f);
    fp12 t1 = fp12_inv(f);
    fp12 t2 = fp12_mul(t0, t1);
    t1 = t2;
    t2 = fp12_mul(fp12_frob(fp12_frob(t2)), t1);
    f = t2;
    t1 = fp12_conj(fp12_cyclotomic_sqr(t2));
    fp12 t3 = cyc_exp(t2);
    fp12 t4 = fp12_mul(t1, t3);
    t1 = cyc_exp(t4);
    t4 = fp12_conj(t4);
    f = fp12_mul(f, t4);
    t4 = fp12_cyclotomic_sqr(t3);
    t0 = cyc_exp(t1);
    t3 = fp12_mul(t3, t0);
    t3 = fp12_frob(fp12_frob(t3));
    f = fp12_mul(f, t3);
    t4 = fp12_mul(t4, cyc_exp(t0));
    f = fp12_mul(f, cyc_exp(t4));
    t4 = fp12_mul(t4, fp12_conj(t2));
    t2 = fp12_mul(t2, t1);
    t2 = fp12_frob(fp12_frob(fp12_frob(t2)));
    f = fp12_mul(f, t2);
    t4 = fp12_frob(t4);
    f = fp12_mul(f, t4);
    return f;
}

__device__ __forceinline__ void fp12_store_u64(uint64_t* out, const fp12& f) {
    const fp* v = (const fp*)&f;
#pragma unroll
    for (int i = 0; i < 12; ++i) fp_store_u64(out + 6 * i, v[i]);
}
__device__ __forceinline__ fp12 fp12_load_u64(const uint64_t* in) {
    fp12 f;
    fp* v = (fp*)&f;
#pragma unroll
    for (int i = 0; i < 12; ++i) v[i] = fp_load_u64(in + 6 * i);
    return f;
}

}  // namespace bls
