/*
 * libbls_gpu.so - BLS12-381 batch signature verification on NVIDIA B200 (sm_100a).
 *
 * Part 1 is the reference's C ABI, symbol for symbol, so the reference's Rust
 * FFI crates link or dlopen this library unchanged.  Part 2 is the extended
 * API: device-resident public-key line tables, compressed signatures with
 * per-item decode status, Miller-loop / Gt values for parity checks, batched
 * persistent launches and a serving loop.
 *
 * Data formats (same as the reference):
 *   Fp      6 x uint64 little-endian limbs of a*R mod p, R = 2^384 (the
 *           in-memory form of ic_bls12_381's Fp), always < p.
 *   G1      12 x uint64: x[6], y[6] affine, Montgomery.  The identity is
 *           x = 0 with y = 0 or y = R mod p (no curve point has x = 0); a pair
 *           holding an identity contributes nothing to the Miller loop, as in
 *           ic_bls12_381's multi_miller_loop.
 *   G2 line table  2448 x uint64: ic_bls12_381 G2Prepared coefficients,
 *           68 x (c0, c1, c2), each an Fp2 (c0[6], c1[6]).
 *   Gt / Miller values  72 x uint64: 12 Fp in tower order
 *           c0.c0.c0, c0.c0.c1, c0.c1.c0, ..., c1.c2.c1.
 *   Compressed G1  48 bytes, ZCash BLS12-381 encoding (big-endian x, flags
 *           0x80 compressed, 0x40 infinity, 0x20 y lexicographically largest).
 *   Compressed G2  96 bytes, the same encoding of x = x.c1 || x.c0 (flags in
 *           the top bits of x.c1's first byte).
 *
 * All pointers are host memory owned by the caller unless a name says
 * "device".  Every entry point is thread-safe.
 */
#ifndef BLS_GPU_H
#define BLS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================
 * Part 1: the reference ABI
 * ==================================================================== */

/* Replaces gpu_crypto_init, gpu-crypto/cuda/api.cu:118-124.
 * 0 when a CUDA device is present (device 0 is selected), -1 otherwise. */
int gpu_crypto_init(void);

/* Replaces gpu_batch_bls_verify, gpu-crypto/cuda/api.cu:128-160
 * (Rust binding gpu-crypto/src/lib.rs:18-25).
 * results[i] = 1 when e(sigs[i], G2) * e(neg_hms[i], pk_i) == 1, else 0, where
 * pk_i's line table is pk_coeffs + 2448*i and g2_coeffs is the generator's.
 * M == 0 returns 0; M < 0, a NULL pointer or a CUDA error returns -1. */
int gpu_batch_bls_verify(const uint64_t* sigs, const uint64_t* neg_hms, const uint64_t* g2_coeffs,
                         const uint64_t* pk_coeffs, int32_t* results, int M);

/* Replaces gpu_batch_sha256, gpu-crypto/cuda/api.cu:165-186.  SHA-256 is not
 * on the verify path this library implements: always returns -1, which the
 * reference's callers treat as "use the CPU". */
int gpu_batch_sha256(const uint8_t* chunks, uint8_t* hashes, int N, int chunk_size);

/* Replaces gpu_g1_decompress_batch, cuda/decompress.cu:198-226 (dlopen'd by
 * ic-integration/gpu_crypto/lib.rs:92-122).  out: n x 96 bytes, Montgomery x
 * then y.  Unlike the reference, every point is validated exactly as
 * G1Affine::from_compressed does; 0 when all n points decode to non-identity
 * points, -1 when n <= 0, a pointer is NULL, any point is invalid or is the
 * identity (the 96-byte output cannot carry the infinity flag, so the caller
 * falls back to its CPU decoder, which reports the precise error), or on a
 * CUDA error.  Per-item reasons: bls_g1_decompress_status. */
int gpu_g1_decompress_batch(const unsigned char* compressed, unsigned char* out_points, int n);

/* Replaces gpu_g1_decompress, cuda/decompress.cu:229-231 (n = 1). */
int gpu_g1_decompress(const unsigned char* compressed, unsigned char* out_point);

/* Replace gpu_msm_g1 / gpu_jacobian_to_affine (ic-integration/gpu_crypto/cuda/
 * msm.cu:32; resolved together at ic-integration/gpu_crypto/lib.rs:103-107).
 * Multi-scalar multiplication is not on the verify path: both return -1 so
 * the caller keeps its CPU MSM.  They exist so the dlopen symbol check passes. */
int gpu_msm_g1(const uint8_t* points, const uint8_t* scalars, size_t n, uint8_t* result_jacobian);
int gpu_jacobian_to_affine(const uint8_t* jacobian, uint8_t* affine);

/* ======================================================================
 * Part 2: extended API (no counterpart in the reference; it extends the
 * reference's verify path above)
 * ==================================================================== */

/* The reference entry point's table cache: gpu_batch_bls_verify keeps the
 * distinct key line tables of earlier calls on device 0 as registered,
 * normalised keys, found again by exact content, so repeat calls send only an
 * item -> table index.  When a call's new tables do not fit beside the cached
 * ones, the cache is emptied and that call's tables are registered afresh.
 * Capacity: the environment variable BLS_REF_TABLE_CACHE when the first
 * reference call creates the context (1 .. 65536 tables), else 1,024.
 * resident: tables held now; capacity: the most it holds; flushes: times it
 * was emptied.  Any pointer may be NULL.  0, or -1 without a device. */
int bls_ref_cache_stats(int* resident, int* capacity, uint64_t* flushes);

/* return codes */
#define BLS_OK 0
#define BLS_ERR_NODEV (-1)
#define BLS_ERR_INVALID (-2)
#define BLS_ERR_CUDA (-3)
#define BLS_ERR_NOMEM (-4)
#define BLS_ERR_TIMEOUT (-5)
#define BLS_ERR_FULL (-6)

/* per-item results of the extended verify calls */
#define BLS_ACCEPT 1
#define BLS_REJECT 0
/* decode failures are reported as the negated status below */
#define BLS_ST_OK 0
#define BLS_ST_BAD_FLAGS 1         /* compression bit clear, or infinity with payload / sort bit */
#define BLS_ST_X_NOT_CANONICAL 2   /* x >= p */
#define BLS_ST_NOT_ON_CURVE 3      /* x^3 + 4 (G2: x^3 + 4(1 + u)) is not a square */
#define BLS_ST_NOT_IN_SUBGROUP 4   /* on the curve, outside the order-r subgroup */
#define BLS_ST_BAD_KEY_INDEX 5     /* not a decode status: a key id outside the tables, where the kernel
                                      checks ids (device-resident ids, bls_verify_compressed_noalloc) */

/* signature input formats */
#define BLS_SIG_AFFINE 0      /* 12 x uint64 Montgomery x, y */
#define BLS_SIG_COMPRESSED 1  /* 48-byte ZCash encoding, decoded and validated on the GPU */

typedef struct bls_ctx bls_ctx;

typedef struct {
    int device;             /* CUDA device ordinal */
    int max_batch;          /* items per launch preallocated (grown on demand; 0 = 65536) */
    int max_pks;            /* public-key table slots (0 = 1024) */
    size_t mem_cap_bytes;   /* device-memory budget for this context (0 = none) */
    int threads_per_block;  /* block shape of the six-lane kernel: 0 = library default (384),
                               384: twelve warps verify 32 items (one per lane, every warp
                               one Fp2 coefficient and half), 64: two warps verify five
                               items; must be 0 for other lane counts */
    int blocks_per_sm;      /* persistent launches: 0 = occupancy maximum */
    int lanes_per_pairing;  /* 6 (default, 0): six lanes per verification, one per Fp2
                               coefficient, lazy reduction (the fastest kernel);
                               2, 4, 8: lanes share per-Fp operations of one
                               verification; 1: one thread per verification */
} bls_config;

typedef struct {
    int n;                     /* items */
    int sig_format;            /* BLS_SIG_AFFINE or BLS_SIG_COMPRESSED */
    const void* sigs;          /* n x 12 uint64, or n x 48 bytes */
    const uint64_t* neg_hms;   /* n x 12 uint64: -H(m_i), affine Montgomery */
    const int32_t* pk_ids;     /* n ids from bls_pk_register_* */
    uint64_t* miller_out;      /* optional n x 72: Miller-loop value (NULL = skip) */
    uint64_t* gt_out;          /* optional n x 72: final exponentiation (NULL = skip) */
} bls_batch;

/* fill *cfg with defaults for `device` */
void bls_config_default(bls_config* cfg, int device);

/* create / destroy a context: its own stream, device buffers, pk tables */
int bls_ctx_create(const bls_config* cfg, bls_ctx** out);
void bls_ctx_destroy(bls_ctx* ctx);

/* last error message of the calling thread ("" when none) */
const char* bls_last_error(void);

/* Register a public key; its line table stays on the device for the life of
 * the context.  From a caller-computed table (reference layout): */
int bls_pk_register_coeffs(bls_ctx* ctx, const uint64_t* coeffs2448, int is_identity, int32_t* pk_id);
/* From an affine point (x.c0, x.c1, y.c0, y.c1: 24 x uint64 Montgomery); the
 * line table is computed on the GPU.  The caller vouches that the point is in G2. */
int bls_pk_register_affine(bls_ctx* ctx, const uint64_t* q24, int32_t* pk_id);
/* From n affine points at once (n x 24 uint64, each as for
 * bls_pk_register_affine); pk_ids[i] gets key i's id.  One launch builds all n
 * line tables and one normalises them, so registering a key set costs about
 * what one key costs.  The caller vouches that every point is in G2. */
int bls_pk_register_affine_batch(bls_ctx* ctx, const uint64_t* q24, int n, int32_t* pk_ids);
/* From n 96-byte compressed keys (ZCash encoding: x.c1 || x.c0 big-endian,
 * flags in byte 0 as for G1; x^3 + 4(1 + u) must be a square in Fp2 and the
 * point in G2).  Decoding, every G2Affine::from_compressed check, the line
 * tables and their normalisation all run on the GPU; this replaces the
 * per-item CPU G2Prepared::from of the reference's callers
 * (ic-integration/patches/ic-gpu-consensus.patch:458-461).  pk_ids[i] gets
 * key i's id; status (optional, n entries) gets each key's BLS_ST_* code.
 * All or nothing: when any key fails to decode, none is registered and the
 * call returns BLS_ERR_INVALID.  The identity encoding (0xc0, zeros)
 * registers an identity key, as bls_pk_register_coeffs with is_identity. */
int bls_pk_register_compressed(bls_ctx* ctx, const uint8_t* pks96, int n, int32_t* pk_ids, int32_t* status);
/* Decode n compressed G2 points: status[i] (BLS_ST_*), q24[i] 24 x uint64
 * x.c0, x.c1, y.c0, y.c1 Montgomery (identity and failures: zeros). */
int bls_g2_decompress_status(bls_ctx* ctx, const uint8_t* compressed96, int n, uint64_t* q24, int32_t* status);
/* copy a registered table back (tests) */
int bls_pk_table(bls_ctx* ctx, int32_t pk_id, uint64_t* coeffs2448);

/* Verify one batch, synchronously.  results[i] = BLS_ACCEPT, BLS_REJECT or
 * -(decode status) for a compressed signature that fails to decode. */
int bls_verify_batch(bls_ctx* ctx, const bls_batch* batch, int32_t* results);

/* Same with every pointer in device memory (inputs already resident); the
 * call enqueues on the context stream and returns without synchronising.
 * bls_ctx_sync waits for it.  The host cannot read the key ids here, so the
 * kernel checks them: an item whose id names no registered table reads no
 * table and gets -BLS_ST_BAD_KEY_INDEX (a compressed signature that failed to
 * decode keeps its own status). */
int bls_verify_batch_device(bls_ctx* ctx, const bls_batch* batch_device, int32_t* results_device);
int bls_ctx_sync(bls_ctx* ctx);
/* the context's CUDA stream (cudaStream_t) */
void* bls_ctx_stream(bls_ctx* ctx);

/* ---- batching (many requests, one launch) ---- */
typedef struct {
    int n;                     /* items in this request */
    const void* sigs;          /* n x 12 uint64 or n x 48 bytes (format given per call) */
    const uint64_t* neg_hms;   /* n x 12 uint64 */
    const int32_t* pk_ids;     /* n registered key ids */
    int32_t* results;          /* n results, as bls_verify_batch */
} bls_request;

#define BLS_MODE_PLAIN 0       /* one launch (copy in, verify, copy out) per request */
#define BLS_MODE_PERSISTENT 1  /* all requests in one persistent launch whose warps claim
                                  items from a device counter, captured once in a CUDA
                                  graph and replayed while the request shapes repeat */

/* Verify nreq requests (all with signatures in `sig_format`), synchronously. */
int bls_verify_requests(bls_ctx* ctx, const bls_request* reqs, int nreq, int sig_format, int mode);

/* ---- autotuning ---- */
typedef struct {
    int lanes_per_pairing;
    int threads_per_block;      /* block shape (six lanes: 64 or 384; else 0) */
    int blocks_per_sm;          /* 0 = occupancy maximum */
    float ms;                   /* kernel time on the sample, best of the repeats */
} bls_tune_point;

/* Time the verify kernel on a device-resident sample batch for every
 * (lanes_per_pairing, threads_per_block, blocks_per_sm) candidate, keep the
 * fastest in the context, and report up to max_points measurements. */
int bls_autotune(bls_ctx* ctx, const bls_batch* sample_device, int repeats, bls_tune_point* points,
                 int max_points, int* n_points);

/* Measured ceiling for the roofline: IMAD-pipe instructions per second of a
 * loop of 12 x 12-limb carry-chain products (the verify kernel's multiply
 * form: mul.lo / mul.hi chained through the carry flag) with the verify
 * kernel's block shape and occupancy, on the whole device. */
int bls_imad_chain_rate(bls_ctx* ctx, double* imad_per_s);
/* Measured issue rates of the two halves of a 32 x 32-bit product on the
 * whole device, in thread instructions per second: mul.lo (the low word) and
 * mul.hi (the high word), each from independent multiply-adds with every
 * latency covered.  Their ratio shows how far a multiprecision multiply, half
 * of whose multiplies are high words, can go toward the nominal IMAD peak. */
int bls_imad_pipe_rates(bls_ctx* ctx, double* lo_per_s, double* hi_per_s);
/* The autotuner's limb-layout dimension: products per second on the whole
 * device of three layouts of a 381-bit element, each in the twelve-warp verify
 * kernel's setting (one block of 384 threads per SM, operands loaded from
 * lane-interleaved shared memory, every product accumulated):
 *   [0] 12 x 32-bit limbs, limb Karatsuba with carry-chain rows into a
 *       26-limb accumulator (the layout every verify kernel is built for),
 *   [1] 15 x 26-bit signed limbs, 225 mad.wide.s32 into 64-bit columns,
 *   [2] 14 x 28-bit limbs, 196 mad.wide.u32 into 64-bit columns.
 * n_layouts must be at least BLS_LIMB_LAYOUTS. */
#define BLS_LIMB_LAYOUTS 3
int bls_limb_layout_rates(bls_ctx* ctx, double* products_per_s, int n_layouts);

/* ---- serving: continuous batching of arriving requests ----
 * A server owns a dispatcher thread and `slots` launch slots (each a stream
 * with its own pinned and device buffers).  Submitted requests queue; when a
 * slot is free the dispatcher takes every queued request that fits the slot's
 * item capacity, stages them and launches them as one persistent verify on the
 * slot's stream, so batches formed while others run overlap on the device.
 * Device memory for the slots is admitted against mem_cap_bytes. */
typedef struct bls_server bls_server;

typedef struct {
    int sig_format;            /* of every request submitted */
    int slots;                 /* launches in flight (0 = 3) */
    int max_batch_items;       /* items per launch / largest request (0 = 16384) */
    size_t mem_cap_bytes;      /* device memory for the slots or the ring (0 = 4 GiB) */
    int mode;                  /* BLS_SERVE_SLOTS (0) or BLS_SERVE_RING */
    int ring_items;            /* ring mode: ring slots, rounded up to a multiple of 5 (0 = 65535) */
    int ring_blocks_per_sm;    /* ring mode: resident blocks of the kernel per SM (0 = 4); fewer
                                  verifications share an SM, so each finishes sooner */
    int ring_blocks;           /* ring mode: total resident blocks, overriding ring_blocks_per_sm
                                  when > 0 (capped at what the device holds) */
} bls_server_config;

/* Serving modes.  SLOTS: the launch slots above.  RING (affine signatures,
 * six-lane kernel): one persistent verify kernel claims items five at a time
 * from a ring in device memory as the dispatcher publishes them, so a request
 * starts as soon as a block is free instead of waiting for a launch slot.  The
 * dispatcher copies requests in, publishes them with one more small copy and
 * polls the results back.  The kernel leaves after 20 ms without work (the
 * next request relaunches it), when the server is destroyed, or 60 s after
 * its launch; every wait in it is bounded.  Admission is by ring space
 * (ring_items x 200 bytes, counted against mem_cap_bytes). */
#define BLS_SERVE_SLOTS 0
#define BLS_SERVE_RING 1

int bls_server_create(bls_ctx* ctx, const bls_server_config* cfg, bls_server** out);
/* waits for in-flight work, then frees the server */
void bls_server_destroy(bls_server* srv);
/* Queue one request (inputs are copied; results are written to req->results
 * when it completes).  *ticket identifies it; *submit_ns is the submit time
 * (steady clock).  Requests larger than max_batch_items are rejected. */
int bls_server_submit(bls_server* srv, const bls_request* req, uint64_t* ticket, int64_t* submit_ns);
/* Wait up to timeout_ms (negative: forever) for a ticket; *done_ns is its
 * completion time.  BLS_ERR_TIMEOUT when it has not completed. */
int bls_server_wait(bls_server* srv, uint64_t ticket, int timeout_ms, int64_t* done_ns);
/* counters: launches, items completed, largest batch */
int bls_server_stats(bls_server* srv, uint64_t* launches, uint64_t* items, uint64_t* max_batch);

/* ---- verification without device allocation ----
 * No counterpart in the reference: its wrapper allocates and frees device
 * memory on every call (gpu-crypto/cuda/api.cu:137-159).  For callers that
 * cannot call cudaMalloc while they verify: plugins whose host process hands
 * all device memory to its own allocator (a framework's caching allocator, a
 * fixed per-tenant budget), and latency-critical paths that cannot afford
 * cudaMalloc's device-wide synchronisation.  Every pointer is device memory
 * owned by the caller: sigs48 (n x 48 B), neg_hms (n x 12 u64), g2_coeffs
 * (2448 u64), pk_tables (n_tables x 2448 u64), pk_identity (optional,
 * n_tables bytes, nonzero marks an identity key, which contributes nothing to
 * the Miller loop as in bls_pk_register_coeffs; NULL = no identity key),
 * pk_index (n), results (n, as bls_verify_batch, and
 * -BLS_ST_BAD_KEY_INDEX for an item whose pk_index is outside
 * [0, n_tables); no table is read for it).  The work is enqueued on `stream`
 * (a cudaStream_t) and not synchronised.  Scratch lives in a fixed device
 * array inside the library (about 0.85 MB on each GPU that loads it, held
 * until exit), so at most BLS_NOALLOC_MAX_ITEMS items per call (more returns
 * BLS_ERR_INVALID).  All calls on a device share that array: calls whose work
 * overlaps on the GPU race and must be ordered by the caller.  The first call
 * on a device does the set-up (looks up the array's address, sets the verify
 * kernel's shared-memory attribute); make it before any stream capture, and
 * do not use this entry point across a cudaDeviceReset (the cached address
 * goes stale).  lanes_per_pairing: 2, 4, 6 or 8. */
#define BLS_NOALLOC_MAX_ITEMS 8192
int bls_verify_compressed_noalloc(const uint8_t* sigs48, const uint64_t* neg_hms, const uint64_t* g2_coeffs,
                                  const uint64_t* pk_tables, const uint8_t* pk_identity, int n_tables,
                                  const int32_t* pk_index, int32_t* results, int n, int lanes_per_pairing,
                                  void* stream);

/* Random-linear-combination batch verification (opt-in): one combined check
 *   e(sum r_i sig_i, G2) * prod_k e(sum_{pk_i = k} r_i (-H(m_i)), pk_k) == 1
 * over random nonzero r_i, with one final exponentiation for the whole
 * batch.  When it holds, every item is accepted (results[i] = BLS_ACCEPT, or
 * -status for a compressed signature that failed to decode); the chance that
 * it holds while some item is invalid is at most 2^-64.  When it fails, or any
 * point is off the curve, non-canonical or outside G1 (the combination is
 * sound only in G1), the batch is verified item by item, so results always
 * equal bls_verify_batch's up to that chance.  scalars: n nonzero 64-bit
 * values s_i (tests), or NULL to draw them from the operating system; the
 * scalar of item i is r_i = (s_i mod 2^32) + lambda (s_i >> 32) mod r, lambda
 * = -x^2 the eigenvalue of the G1 endomorphism (x, y) -> (beta x, y), so a
 * multiplication needs 32 doublings and 2^64 scalars remain distinct.  combined (optional): 1 when
 * the combined check accepted the batch.  agg_out (optional, 12 x (1 + K)
 * uint64, K = distinct keys): the signature sum, then each key's sum in
 * increasing key id, affine (identity: x = 0, y = R mod p).  batch->miller_out
 * and gt_out must be NULL. */
int bls_verify_batch_rlc(bls_ctx* ctx, const bls_batch* batch, const uint64_t* scalars, int32_t* results,
                         int* combined, uint64_t* agg_out);

/* -H(m_i) for n messages on the GPU, in the neg_hms layout (12 x uint64 each,
 * affine Montgomery).  H is RFC 9380 hash_to_curve to G1 with
 * expand_message_xmd over SHA-256 and domain `dst` (0..255 bytes): the suite
 * BLS12381G1_XMD:SHA-256_SSWU_RO_ (simplified SWU map on the 11-isogenous
 * curve, the 11-isogeny to E, h_eff = 1 - x), the suite ic_bls12_381's
 * hash_to_curve implements, so with the caller's domain string the points
 * are the ones its CPU hash gives.
 * msgs: the messages back to back; offsets: n + 1 byte offsets, offsets[0] = 0,
 * non-decreasing (message i is msgs[offsets[i] .. offsets[i+1])). */
int bls_neg_hash_to_g1(bls_ctx* ctx, const uint8_t* msgs, const uint32_t* offsets, int n, const uint8_t* dst,
                       int dst_len, uint64_t* out);
/* Verify n signatures against messages: -H(m_i) as bls_neg_hash_to_g1 computes
 * it on the GPU, straight into the verify launch's input.  sig_format and
 * results as in bls_verify_batch. */
int bls_verify_messages(bls_ctx* ctx, int sig_format, const void* sigs, const uint8_t* msgs,
                        const uint32_t* offsets, const int32_t* pk_ids, int n, const uint8_t* dst, int dst_len,
                        int32_t* results);

/* Decode n compressed G1 points: status[i] (BLS_ST_*), xy[i] 12 x uint64
 * (identity: x = 0, y = R mod p; failures: zeros). */
int bls_g1_decompress_status(bls_ctx* ctx, const uint8_t* compressed, int n, uint64_t* xy, int32_t* status);

#ifdef __cplusplus
}
#endif

#endif /* BLS_GPU_H */
