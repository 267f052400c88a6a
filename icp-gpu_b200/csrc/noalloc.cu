// bls_verify_compressed_noalloc: verification of compressed signatures for
// callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc when they verify: plugins whose host
// process has handed the whole device memory to its own pool allocator (a
// framework's caching allocator, a fixed per-tenant budget), and
// latency-critical paths where cudaMalloc's implicit device-wide
// synchronisation would stall every other stream.  This entry point takes
// only caller-owned device buffers and keeps its scratch -- the decoded
// signatures, their decode statuses, the checked key indices and the work
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
//     call and every other word a call reads is written earlier in that call;
//     two calls whose work overlaps on the GPU (different streams, no ordering
//     between them) race on the array and produce wrong results;
//   * the first call on a device does the set-up: it resolves the array's
//     device address (cudaGetSymbolAddress, with that device current) and
//     sets the verify kernel's shared-memory attribute; make that first call
//     before starting any stream capture.  The address is cached per device
//     ordinal for the life of the process; after cudaDeviceReset the module is
//     loaded again and the cached address is stale, so this entry point must
//     not be used across a device reset.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/bls_gpu.h"
#include "internal.h"

namespace bls {
namespace {

constexpr int kMaxItems = BLS_NOALLOC_MAX_ITEMS;
constexpr size_t kXyBytes = (size_t)kMaxItems * 96;                 // decoded signatures
constexpr size_t kStatusBytes = (size_t)kMaxItems * 4;              // decode statuses
constexpr size_t kIndexBytes = (size_t)kMaxItems * 4;               // key indices, checked
constexpr size_t kCounterBytes = 256;                               // work counter, padded
constexpr size_t kScratchBytes = kXyBytes + kStatusBytes + kIndexBytes + kCounterBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};

// device address of the scratch array on the current device (set up once)
cudaError_t scratch_address(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

// Item i's key index into the scratch copy: the caller's index when it names
// one of the n_tables tables, else 0 with BLS_ST_BAD_KEY_INDEX as the item's
// status (a decode failure already recorded there is kept), so the verify
// kernel never reads outside the caller's tables and reports the item as
// -BLS_ST_BAD_KEY_INDEX.
__global__ void k_check_key_index(const int32_t* __restrict__ pk_index, int n, int n_tables, int32_t* idx,
                                  int32_t* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t k = pk_index[i];
    const bool ok = k >= 0 && k < n_tables;
    idx[i] = ok ? k : 0;
    if (!ok && status[i] == BLS_ST_OK) status[i] = BLS_ST_BAD_KEY_INDEX;
}

}  // namespace
}  // namespace bls

extern "C" int bls_verify_compressed_noalloc(const uint8_t* sigs48, const uint64_t* neg_hms,
                                             const uint64_t* g2_coeffs, const uint64_t* pk_tables,
                                             const uint8_t* pk_identity, int n_tables, const int32_t* pk_index,
                                             int32_t* results, int n, int lanes_per_pairing, void* stream) {
    if (n < 0 || n > bls::kMaxItems) return BLS_ERR_INVALID;
    if (n == 0) return BLS_OK;
    if (!sigs48 || !neg_hms || !g2_coeffs || !pk_tables || !pk_index || !results || n_tables <= 0)
        return BLS_ERR_INVALID;
    if (lanes_per_pairing != 2 && lanes_per_pairing != 4 && lanes_per_pairing != 6 && lanes_per_pairing != 8)
        return BLS_ERR_INVALID;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return BLS_ERR_CUDA;
    unsigned char* base = nullptr;
    if (bls::scratch_address(dev, &base) != cudaSuccess) return BLS_ERR_CUDA;
    uint64_t* xy = reinterpret_cast<uint64_t*>(base);
    int32_t* status = reinterpret_cast<int32_t*>(base + bls::kXyBytes);
    int32_t* idx = reinterpret_cast<int32_t*>(base + bls::kXyBytes + bls::kStatusBytes);
    int* counter = reinterpret_cast<int*>(base + bls::kXyBytes + bls::kStatusBytes + bls::kIndexBytes);
    if (cudaMemsetAsync(counter, 0, sizeof(int), s) != cudaSuccess) return BLS_ERR_CUDA;
    if (bls::launch_g1_decompress(sigs48, n, xy, status, s) != cudaSuccess) return BLS_ERR_CUDA;
    bls::k_check_key_index<<<(n + 255) / 256, 256, 0, s>>>(pk_index, n, n_tables, idx, status);
    if (cudaGetLastError() != cudaSuccess) return BLS_ERR_CUDA;
    bls::VerifyArgs a{};
    a.sigs = sigs48;
    a.sig_compressed = 1;
    a.sig_xy = xy;
    a.nhms = neg_hms;
    a.g2 = g2_coeffs;
    a.pk_tables = pk_tables;
    a.pk_index = idx;
    a.pk_identity = pk_identity;
    a.n = n;
    a.results = results;
    a.work_counter = counter;
    if (bls::launch_verify_lanes(a, reinterpret_cast<const uint32_t*>(status), lanes_per_pairing, 0, 0, sms, s) !=
        cudaSuccess)
        return BLS_ERR_CUDA;
    return BLS_OK;
}
