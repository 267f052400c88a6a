// k_neg_hash_to_g1: -H(m) for a batch of messages (h2c.cuh), two threads per
// message: both expand the message (SHA-256 is cheap next to the field work),
// thread 2i maps u0 and thread 2i + 1 maps u1 at the same time, then thread 2i
// adds the two points, clears the cofactor and writes the result.  The output
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
    __shared__ uint4 xch[kHashThreads / 2][6];   // the odd thread's mapped point (x, y)
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t >> 1, which = t & 1;
    const bool live = i < n;
    fp x, y;
    if (live) {
        const uint32_t a = offsets[i], b = offsets[i + 1];
        uint32_t ub[32];
        h2c::expand_xmd_128(msgs + a, b - a, dst, (uint32_t)dst_len, ub);
        h2c::map_svdw(h2c::field_from_be64(ub + 16 * which), x, y);
        if (which) {
            uint4* d = xch[threadIdx.x >> 1];
            d[0] = make_uint4(x.w[0], x.w[1], x.w[2], x.w[3]);
            d[1] = make_uint4(x.w[4], x.w[5], x.w[6], x.w[7]);
            d[2] = make_uint4(x.w[8], x.w[9], x.w[10], x.w[11]);
            d[3] = make_uint4(y.w[0], y.w[1], y.w[2], y.w[3]);
            d[4] = make_uint4(y.w[4], y.w[5], y.w[6], y.w[7]);
            d[5] = make_uint4(y.w[8], y.w[9], y.w[10], y.w[11]);
        }
    }
    __syncthreads();
    if (!live || which) return;
    const uint4* d = xch[threadIdx.x >> 1];
    fp x1, y1;
    const uint4 q[6] = {d[0], d[1], d[2], d[3], d[4], d[5]};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        x1.w[4 * k] = q[k].x; x1.w[4 * k + 1] = q[k].y; x1.w[4 * k + 2] = q[k].z; x1.w[4 * k + 3] = q[k].w;
        y1.w[4 * k] = q[3 + k].x; y1.w[4 * k + 1] = q[3 + k].y; y1.w[4 * k + 2] = q[3 + k].z;
        y1.w[4 * k + 3] = q[3 + k].w;
    }
    fp ox, oy;
    h2c::neg_clear(x, y, x1, y1, ox, oy);
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
