// Internal interface between the host library (bls_gpu.cpp) and the kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bls {

constexpr int kVerifyThreads = 64;
constexpr int kCoeffU64 = 2448;

struct VerifyArgs {
    const void* sigs;            // n x 12 u64 (affine) or n x 48 B (compressed), device
    int sig_compressed;
    const uint64_t* nhms;        // n x 12 u64, device
    const uint64_t* g2;          // generator line table, device
    const uint64_t* pk_tables;   // k x 2448 u64, device
    const int32_t* pk_index;     // n table ids, device; NULL = table i for item i
    // check_keys != 0: an id outside [0, n_keys) reads no table and the item's
    // result is -BLS_ST_BAD_KEY_INDEX (a decode failure already recorded is
    // kept); check_keys == 0: ids are not checked (the caller validated them)
    int check_keys;
    int n_keys;
    const uint8_t* pk_identity;  // per table, device; NULL = none is the identity
    int n;
    int32_t* results;            // n, device
    uint64_t* ml_out;            // n x 72 or NULL, device
    uint64_t* gt_out;            // n x 72 or NULL, device
    const uint64_t* sig_xy;      // decoded signatures (n x 12 u64) when sigs were compressed, device
    int* work_counter;           // persistent mode: items are claimed from this zeroed counter, device
    // Normalised line tables (every row divided by its c2) and the Miller
    // correction factors (Fp2, 12 u64) of the generator and the keys, device;
    // pk_norm NULL = use the raw tables.  Read by the Fp2-lane kernel only.
    const uint64_t* g2_norm;
    const uint64_t* pk_norm;
    const uint64_t* g2_corr;
    const uint64_t* pk_corr;
    // Ring serving (Fp2-lane kernel only): sigs / nhms / pk_index / results are
    // rings of serve_cap slots (a multiple of 5) in device memory, filled by the
    // host's copies; the host publishes whole groups of 5 by raising
    // *serve_avail (items since the start, device memory, written by a copy
    // after the items' own copies); blocks claim published groups from
    // *serve_claimed and leave after serve_idle_ns without a claimable group,
    // when *serve_stop is set, or serve_max_ns after the launch.
    const volatile uint32_t* serve_avail;
    const volatile uint32_t* serve_stop;
    uint32_t* serve_claimed;
    uint32_t serve_cap;
    uint64_t serve_idle_ns;
    uint64_t serve_max_ns;
};

cudaError_t launch_verify(const VerifyArgs& a, cudaStream_t s);

// random-linear-combination batch check (rlc.cu), device pointers
struct RlcArgs {
    const uint64_t* sig_xy;   // n x 12 u64 affine signatures (decoded when the input was compressed)
    const int32_t* status;    // n decode statuses, or NULL
    const uint64_t* nhms;     // n x 12 u64
    const uint64_t* r;        // n nonzero scalars
    int n;
    int check_sig;            // check the signatures too (affine input; the decoder checked compressed ones)
    uint32_t* pts;            // n x 72 words scratch: [r] sig, [r] nhm (Jacobian)
    uint8_t* bad;             // n x 2: a signature / nhm that failed its checks
    int* counters;            // [0] combined check is one, [1] points that failed their checks (zeroed)
    const int32_t* order;     // n item ids, grouped by key
    const int32_t* tiles;     // ntiles x 3: [start, end) in order, key slot
    int ntiles;
    uint32_t* partials;       // ntiles x 72 words scratch
    const int32_t* key_tile;  // nkeys + 1: first tile of each key slot
    int nkeys;
    uint64_t* agg_sigs;       // nkeys x 12 u64: verify items, pair 1
    uint64_t* agg_nhms;       // nkeys x 12 u64: verify items, pair 2
};
cudaError_t launch_rlc(const RlcArgs& a, cudaStream_t s);
cudaError_t launch_gt_product(uint64_t* gt, int n, int* counters, cudaStream_t s);
cudaError_t launch_g1_decompress(const uint8_t* in, int n, uint64_t* xy, int32_t* status, cudaStream_t s);
// the same decode in whole-SM blocks, at most max_sms of them (grid-stride):
// the serving ring's decoder, which must stay within the SMs left to it;
// check_subgroup false leaves the subgroup test to launch_g1_subgroup_sms
cudaError_t launch_g1_decompress_sms(const uint8_t* in, int n, uint64_t* xy, int32_t* status, int max_sms,
                                     bool check_subgroup, cudaStream_t s);
// sub[i] = ST_NOT_IN_SUBGROUP (4) for a decoded point (status 0, not the
// identity) outside G1, else 0; whole-SM blocks, at most max_sms
cudaError_t launch_g1_subgroup_sms(const uint64_t* xy, const int32_t* status, int n, int32_t* sub, int max_sms,
                                   cudaStream_t s);
cudaError_t launch_neg_hash_to_g1(const uint8_t* msgs, const uint32_t* offsets, int n, const uint8_t* dst,
                                  int dst_len, uint64_t* out, cudaStream_t s);
cudaError_t launch_g2_decompress(const uint8_t* in, int n, uint64_t* q, int32_t* status, uint8_t* identity,
                                 cudaStream_t s);
cudaError_t launch_g2_prepare(const uint64_t* q, int n, uint64_t* out, cudaStream_t s);
// n line tables divided row by row by their c2, with each table's Miller
// correction factor (12 u64) and a flag set when a c2 is zero (table copied)
cudaError_t launch_lines_normalize(const uint64_t* raw, int n, uint64_t* norm, uint64_t* corr, uint8_t* bad,
                                   cudaStream_t s);
// Block shapes of the six-lane (Fp2-lane) kernels, by threads per block:
// kShapeFive (64 threads, two warps, five items per block: k_verify_fp2) and
// kShapeWide (384 threads, twelve warps, 32 items per block, one per lane:
// k_verify_w).  0 selects kDefaultShape.
constexpr int kShapeFive = 64, kShapeWide = 384;
constexpr int kDefaultShape = kShapeWide;
inline int six_lane_shape(int threads_per_block) { return threads_per_block > 0 ? threads_per_block : kDefaultShape; }

// lane-parallel verify; in_status: per-item decode status or NULL.  lanes 6
// runs an Fp2-lane kernel of block shape `shape` (verify_fp2.cu or
// verify_w.cu), 2, 4 and 8 the interpreter of per-Fp programs (verify_vm.cu).
cudaError_t launch_verify_lanes(const VerifyArgs& a, const uint32_t* in_status, int lanes, int shape,
                                int blocks_per_sm, int sms, cudaStream_t s);
cudaError_t launch_verify_fp2_serve(const VerifyArgs& a, const uint32_t* in_status, int blocks, int sms,
                                   cudaStream_t s);
cudaError_t launch_verify_fp2(const VerifyArgs& a, const uint32_t* in_status, int blocks_per_sm, int sms,
                              cudaStream_t s);
size_t verify_fp2_smem_bytes();
int verify_fp2_blocks_per_sm();
// the twelve-warp form: one block per SM; ring serving claims up to 32 items
cudaError_t launch_verify_w(const VerifyArgs& a, const uint32_t* in_status, int sms, cudaStream_t s);
cudaError_t launch_verify_w_serve(const VerifyArgs& a, const uint32_t* in_status, int blocks, int sms,
                                 cudaStream_t s);
size_t verify_w_smem_bytes();
int verify_w_blocks_per_sm();
cudaError_t measure_imad_chain(int sms, int iters, uint32_t* out, cudaStream_t s, double* imad_per_s);
// products per second of the three limb layouts (limb_forms.cu); out: sms x 384 words
cudaError_t measure_limb_forms(int sms, int iters, uint32_t* out, cudaStream_t s, double* per_s);
cudaError_t measure_imad_rates(int sms, int iters, uint32_t* out, cudaStream_t s, double* lo_per_s,
                               double* hi_per_s);
size_t verify_lanes_smem_bytes(int lanes, int shape = 0);
// blocks of the lane-parallel kernel resident per SM (occupancy calculator)
int verify_lanes_blocks_per_sm(int lanes, int shape = 0);

// what the serving loop (server.cpp) needs from a context
struct CtxView {
    int device, sms, lanes, shape, blocks_per_sm;
    const uint64_t* g2;
    const uint64_t* pk_tables;
    const uint8_t* pk_identity;
    int n_pks;
    const uint64_t* g2_norm;     // NULL: raw lines only
    const uint64_t* pk_norm;
    const uint64_t* g2_corr;
    const uint64_t* pk_corr;
    // Ring serving (Fp2-lane kernel only): sigs / nhms / pk_index / results are
    // rings of serve_cap slots (a multiple of 5) in device memory, filled by the
    // host's copies; the host publishes whole groups of 5 by raising
    // *serve_avail (items since the start, device memory, written by a copy
    // after the items' own copies); blocks claim published groups from
    // *serve_claimed and leave after serve_idle_ns without a claimable group,
    // when *serve_stop is set, or serve_max_ns after the launch.
    const volatile uint32_t* serve_avail;
    const volatile uint32_t* serve_stop;
    uint32_t* serve_claimed;
    uint32_t serve_cap;
    uint64_t serve_idle_ns;
    uint64_t serve_max_ns;
};

}  // namespace bls
