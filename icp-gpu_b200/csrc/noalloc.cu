// bls_verify_compressed_noalloc: verification of compressed signatures for
// callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc when they verify: code running while a
// stream is being captured into a CUDA graph (allocation is not a stream
// operation and breaks the capture), plugins whose host process has handed the
// whole device memory to its own pool allocator (a framework's caching
// allocator, a fixed per-tenant budget), and latency-critical paths where
// cudaMalloc's implicit device-wide synchronisation would stall every other
// stream.  This entry point takes only caller-owned device buffers and keeps
// its scratch -- the decoded signatures, their decode statuses and the work
// counter of the persistent launch -- in one file-scope device array of fixed
// size, so a call allocates nothing.
//
// Limits and sharing, which the caller must respect:
//   * at most kMaxItems signatures per call; larger batches are rejected
//     with BLS_ERR_INVALID before anything is launched;
//   * every GPU that loads the library holds the array (kScratchBytes) until
//     the process exits;
//   * all calls on one device share the array and it keeps the previous call's
//     contents: the work counter is cleared on the stream at the start of each
//     call, and two calls whose work overlaps on the GPU (different streams, no
//     ordering between them) race on the array and produce wrong results;
//   * the first call on a device resolves the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before starting any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/bls_gpu.h"
#include "internal.h"

namespace bls {
namespace {

constexpr int kMaxItems = BLS_NOALLOC_MAX_ITEMS;
constexpr size_t kXyBytes = (size_t)kMaxItems * 96;                 // decoded signatures
constexpr size_t kStatusBytes = (size_t)kMaxItems * 4;              // decode statuses
constexpr size_t kCounterBytes = 256;                               // work counter, padded
constexpr size_t kScratchBytes = kXyBytes + kStatusBytes + kCounterBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};

// device address of the scratch array on the current device (set up once)
cudaError_t scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace bls

extern "C" int bls_verify_compressed_noalloc(const uint8_t* sigs48, const uint64_t* neg_hms,
                                             const uint64_t* g2_coeffs, const uint64_t* pk_tables,
                                             const int32_t* pk_index, int32_t* results, int n,
                                             int lanes_per_pairing, void* stream) {
    if (n < 0 || n > bls::kMaxItems) return BLS_ERR_INVALID;
    if (n == 0) return BLS_OK;
    if (!sigs48 || !neg_hms || !g2_coeffs || !pk_tables || !pk_index || !results) return BLS_ERR_INVALID;
    if (lanes_per_pairing != 2 && lanes_per_pairing != 4 && lanes_per_pairing != 6 && lanes_per_pairing != 8)
        return BLS_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    if (bls::scratch_address(&base) != cudaSuccess) return BLS_ERR_CUDA;
    uint64_t* xy = reinterpret_cast<uint64_t*>(base);
    int32_t* status = reinterpret_cast<int32_t*>(base + bls::kXyBytes);
    int* counter = reinterpret_cast<int*>(base + bls::kXyBytes + bls::kStatusBytes);
    if (cudaMemsetAsync(counter, 0, sizeof(int), s) != cudaSuccess) return BLS_ERR_CUDA;
    if (bls::launch_g1_decompress(sigs48, n, xy, status, s) != cudaSuccess) return BLS_ERR_CUDA;
    bls::VerifyArgs a{};
    a.sigs = sigs48;
    a.sig_compressed = 1;
    a.sig_xy = xy;
    a.nhms = neg_hms;
    a.g2 = g2_coeffs;
    a.pk_tables = pk_tables;
    a.pk_index = pk_index;
    a.pk_identity = nullptr;
    a.n = n;
    a.results = results;
    a.work_counter = counter;
    int sms = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return BLS_ERR_CUDA;
    if (bls::launch_verify_lanes(a, reinterpret_cast<const uint32_t*>(status), lanes_per_pairing, 0, sms, s) !=
        cudaSuccess)
        return BLS_ERR_CUDA;
    return BLS_OK;
}
