// G2 line coefficients on the device: the ic_bls12_381 G2Prepared table for an
// affine point Q in homogeneous projective coordinates, Algorithms 26
// (doubling) and 27 (addition) of Costello, Lange, Naehrig, eprint 2010/354,
// in the operation order the reference restates at cuda/test_miller_v2.cu:
// 148-229.  The table is what the reference's callers build on the CPU for
// every item (ic-integration/patches/ic-gpu-consensus.patch:458-461); here it
// is built once per distinct key and kept on the device.
#pragma once
#include "pairing.cuh"

namespace bls {

struct g2proj { fp2 x, y, z; };

__device__ __forceinline__ void store_fp2(uint64_t* p, const fp2& a) {
    fp_store_u64(p, a.c0);
    fp_store_u64(p + 6, a.c1);
}

static __device__ __noinline__ void g2_doubling_step(g2proj& r, uint64_t* out) {
    fp2 tmp0 = fp2_sqr(r.x);
    fp2 tmp1 = fp2_sqr(r.y);
    fp2 tmp2 = fp2_sqr(tmp1);
    fp2 tmp3 = fp2_sub(fp2_sqr(fp2_add(tmp1, r.x)), fp2_add(tmp0, tmp2));
    tmp3 = fp2_dbl(tmp3);
    fp2 tmp4 = fp2_add(fp2_dbl(tmp0), tmp0);
    fp2 tmp6 = fp2_add(r.x, tmp4);
    fp2 tmp5 = fp2_sqr(tmp4);
    fp2 zsq = fp2_sqr(r.z);
    r.x = fp2_sub(fp2_sub(tmp5, tmp3), tmp3);
    r.z = fp2_sub(fp2_sqr(fp2_add(r.z, r.y)), fp2_add(tmp1, zsq));
    r.y = fp2_mul(fp2_sub(tmp3, r.x), tmp4);
    tmp2 = fp2_dbl(fp2_dbl(fp2_dbl(tmp2)));
    r.y = fp2_sub(r.y, tmp2);
    tmp3 = fp2_neg(fp2_dbl(fp2_mul(tmp4, zsq)));
    tmp6 = fp2_sub(fp2_sub(fp2_sqr(tmp6), fp2_add(tmp0, tmp5)), fp2_dbl(fp2_dbl(tmp1)));
    fp2 c0 = fp2_dbl(fp2_mul(r.z, zsq));
    store_fp2(out, c0);
    store_fp2(out + 12, tmp3);
    store_fp2(out + 24, tmp6);
}

static __device__ __noinline__ void g2_addition_step(g2proj& r, const fp2& qx, const fp2& qy, uint64_t* out) {
    fp2 zsq = fp2_sqr(r.z);
    fp2 ysq = fp2_sqr(qy);
    fp2 t0 = fp2_mul(zsq, qx);
    fp2 t1 = fp2_mul(fp2_sub(fp2_sqr(fp2_add(qy, r.z)), fp2_add(ysq, zsq)), zsq);
    fp2 t2 = fp2_sub(t0, r.x);
    fp2 t3 = fp2_sqr(t2);
    fp2 t4 = fp2_dbl(fp2_dbl(t3));
    fp2 t5 = fp2_mul(t4, t2);
    fp2 t6 = fp2_sub(fp2_sub(t1, r.y), r.y);
    fp2 t9 = fp2_mul(t6, qx);
    fp2 t7 = fp2_mul(t4, r.x);
    r.x = fp2_sub(fp2_sub(fp2_sub(fp2_sqr(t6), t5), t7), t7);
    r.z = fp2_sub(fp2_sqr(fp2_add(r.z, t2)), fp2_add(zsq, t3));
    fp2 t10 = fp2_add(qy, r.z);
    fp2 t8 = fp2_mul(fp2_sub(t7, r.x), t6);
    fp2 t0b = fp2_dbl(fp2_mul(r.y, t5));
    r.y = fp2_sub(t8, t0b);
    t10 = fp2_sub(fp2_sub(fp2_sqr(t10), ysq), fp2_sqr(r.z));
    t9 = fp2_sub(fp2_dbl(t9), t10);
    store_fp2(out, fp2_dbl(r.z));
    store_fp2(out + 12, fp2_dbl(fp2_neg(t6)));
    store_fp2(out + 24, t9);
}

// 68 coefficients of Q = (qx, qy) into out[0..2447]
static __device__ __noinline__ void g2_prepare(const fp2& qx, const fp2& qy, uint64_t* out) {
    g2proj r = {qx, qy, fp2_one()};
    int ci = 0;
    bool found = false;
    for (int b = 63; b >= 0; --b) {
        bool bit = (((BLS_X_ABS >> 1) >> b) & 1) == 1;
        if (!found) { found = bit; continue; }
        g2_doubling_step(r, out + 36 * ci++);
        if (bit) g2_addition_step(r, qx, qy, out + 36 * ci++);
    }
    g2_doubling_step(r, out + 36 * ci);
}

}  // namespace bls
