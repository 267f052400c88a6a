// k_neg_hash_to_g1: -H(m) for a batch of messages (h2c.cuh), two threads per
// message: both expand the message (SHA-256 is cheap next to the field work),
// thread 2i maps u0 and thread 2i + 1 maps u1 at the same time (SSWU to E',
// then the isogeny to E), then thread 2i adds the two points, clears the
// cofactor and writes the result.  The output
// is the verify kernels' neg_hms layout, so a verify from message bytes hashes
// straight into the verify launch's input buffer.
#include <cuda_runtime.h>

#include "h2c.cuh"
#include "internal.h"

namespace bls {

constexpr int kHashThreads = 64;

__global__ void __launch_bounds__(kHashThreads) k_neg_hash_to_g1(const uint8_t* msgs, const uint32_t* offsets,
                                                                 int n, const uint8_t* dst, int dst_len,
                                                                 uint64_t* out) {
    __shared__ uint4 xch[kHashThreads / 2][9];   // the odd thread's mapped point (Jacobian X, Y, Z)
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t >> 1, which = t & 1;
    const bool live = i < n;
    g1j pt;
    if (live) {
        const uint32_t a = offsets[i], b = offsets[i + 1];
        uint32_t ub[32];
        h2c::expand_xmd_128(msgs + a, b - a, dst, (uint32_t)dst_len, ub);
        fp xn, xd, ys;
        h2c::map_sswu(h2c::field_from_be64(ub + 16 * which), xn, xd, ys);
        pt = h2c::iso_map(xn, xd, ys);
        if (which) {
            uint4* d = xch[threadIdx.x >> 1];
            const fp* c[3] = {&pt.X, &pt.Y, &pt.Z};
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    d[3 * k + j] = make_uint4(c[k]->w[4 * j], c[k]->w[4 * j + 1], c[k]->w[4 * j + 2], c[k]->w[4 * j + 3]);
        }
    }
    __syncthreads();
    // the even thread of a live message adds the points and clears the
    // cofactor; then every thread of the warp takes part in one simultaneous
    // inversion of the results' Z (the others contribute a one), so the
    // warp's 16 inverses cost one binary Euclid that does not diverge
    const bool owner = live && !which;
    g1j r;
    r.Z = fp_one();
    if (owner) {
        const uint4* d = xch[threadIdx.x >> 1];
        g1j p1;
        fp* c[3] = {&p1.X, &p1.Y, &p1.Z};
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const uint4 q = d[3 * k + j];
                c[k]->w[4 * j] = q.x; c[k]->w[4 * j + 1] = q.y; c[k]->w[4 * j + 2] = q.z; c[k]->w[4 * j + 3] = q.w;
            }
        r = h2c::clear_sum(pt, p1);
    }
    const fp zi = fp_inverse_warp(owner ? r.Z : fp_one(), h2c::kR3);
    if (!owner) return;
    fp ox, oy;
    h2c::neg_affine(r, zi, ox, oy);
    fp_store_u64(out + 12 * (size_t)i, ox);
    fp_store_u64(out + 12 * (size_t)i + 6, oy);
}

cudaError_t launch_neg_hash_to_g1(const uint8_t* msgs, const uint32_t* offsets, int n, const uint8_t* dst,
                                  int dst_len, uint64_t* out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const long long threads = 2LL * n;
    k_neg_hash_to_g1<<<(unsigned)((threads + kHashThreads - 1) / kHashThreads), kHashThreads, 0, s>>>(
        msgs, offsets, n, dst, dst_len, out);
    return cudaGetLastError();
}

}  // namespace bls
