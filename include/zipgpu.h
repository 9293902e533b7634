/*
 * zipgpu.h -- C ABI of the B200 (sm_100a) Zip+ commit/prove/verify backend.
 *
 * The reference (NethermindEth/zinc-plus) is a Rust workspace with no FFI; its
 * boundary for this path is a set of Rust traits and associated functions.
 * Each entry point below names the reference item it stands in for, so a Rust
 * host can bind this header with `extern "C"` declarations and keep its call
 * sites:
 *
 *   LinearCode::{row_len, codeword_len, encode, encode_wide}
 *                                   zip-plus/src/code.rs:10-72
 *   IprsCode::{new, new_with_optimal_depth}   zip-plus/src/code/iprs.rs:30-51
 *   RaaCode::new                    zip-plus/src/code/raa.rs:38-90
 *   ZipPlus::setup                  zip-plus/src/pcs/structs.rs:74-88
 *   ZipPlus::{commit, commit_single, encode_rows}
 *                                   zip-plus/src/pcs/phase_commit.rs:61,135,159
 *   ZipPlus::{prove, prove_f}       zip-plus/src/pcs/phase_prove.rs:85,119
 *   ZipPlus::verify                 zip-plus/src/pcs/phase_verify.rs:100
 *   MerkleTree::{new, root}         zip-plus/src/merkle.rs:74-103
 *   PcsProverTranscript / Blake3Transcript
 *                                   zip-plus/src/pcs_transcript.rs:44-222,
 *                                   transcript/src/lib.rs:12-77
 *
 * Conventions
 *  - Every function returns a zg_status (0 = ZG_OK).  No exception or panic
 *    crosses the ABI.  zg_last_error() gives a message for the calling thread.
 *  - Host buffers are owned by the caller.  Device hints (codewords and Merkle
 *    layers, the reference's ZipPlusHint) are owned by the library until
 *    zg_hint_free.  "_d" entry points take device pointers and a cudaStream_t
 *    passed as void*.
 *  - Evaluations: ZG_EVAL_I32 is one int32 per evaluation (Zip, Eval = i32);
 *    ZG_EVAL_I64 is one int64 per evaluation (the integer trace columns of
 *    Zinc+, IntZt of protocol/benches/e2e.rs:215-227: Eval = i64, Cw = i128);
 *    ZG_EVAL_BINPOLY is one uint64 per evaluation holding the {0,1}
 *    coefficients of a BinaryPoly<D> (bit i = coefficient of X^i, bits >= D
 *    must be zero), as the reference's `simd` feature stores it
 *    (poly/src/univariate/binary_u64.rs:28).
 *  - Codewords are laid out like the reference's DenseRowMatrix (row-major
 *    num_rows x codeword_len) when copied to the host; Cw is i128 (I32, I64 evals),
 *    DensePolynomial<i64, D> (BINPOLY + IPRS) or DensePolynomial<i32, D>
 *    (BINPOLY + RAA), little-endian, coefficient 0 first.
 *  - Field elements (MontyField<field_limbs>) are exchanged as their
 *    Montgomery-form inner value, 8*field_limbs little-endian bytes.
 *  - i128 values (challenges, points) are exchanged as little-endian 16-byte
 *    two's complement.
 */
#ifndef ZIPGPU_H
#define ZIPGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; the first four mirror ZipError (zip-plus/src/lib.rs:13-29). */
typedef enum {
    ZG_OK = 0,
    ZG_ERR_INVALID_PARAM = 1,   /* ZipError::InvalidPcsParam, setup asserts   */
    ZG_ERR_INVALID_OPEN = 2,    /* ZipError::InvalidPcsOpen: verifier rejects */
    ZG_ERR_SERIALIZATION = 3,   /* ZipError::Transcript: truncated proof      */
    ZG_ERR_OVERFLOW = 4,        /* validate_input bit budget exceeded         */
    ZG_ERR_CUDA = 5,            /* CUDA runtime error                          */
    ZG_ERR_OOM = 6,             /* device or host allocation failed            */
    ZG_ERR_TIMEOUT = 7,         /* a bounded device wait gave up               */
    ZG_ERR_NO_DEVICE = 8,       /* no CUDA device / extension unusable         */
    ZG_ERR_BUFFER_TOO_SMALL = 9 /* caller buffer shorter than required         */
} zg_status;

typedef enum { ZG_EVAL_I32 = 0, ZG_EVAL_BINPOLY = 1, ZG_EVAL_I64 = 2 } zg_eval_kind;
/* ZG_CODE_RAA_SIGN_FLIP: RaaSignFlippingCode (zip-plus/src/code/raa_sign_flip.rs:
 * 14-69), the RAA code with entries 1, 3, 5, ... negated after the repetition
 * and after the first accumulation; same permutations and width check. */
typedef enum { ZG_CODE_IPRS = 0, ZG_CODE_RAA = 1, ZG_CODE_RAA_SIGN_FLIP = 2 } zg_code_kind;

/* One ZipTypes instantiation plus its linear code and matrix shape.
 * The reference fixes these through type parameters (pcs/structs.rs:15-60):
 *   Zip    (zip-plus/benches/zip_benches.rs:25-40): I32, comb_limbs 3, field_limbs 4
 *   Zip+   (zip-plus/benches/zip_plus_benches.rs:37-65): BINPOLY D=32|64,
 *          comb_limbs 5, field_limbs 4; Cw coefficients i64 (IPRS) / i32 (RAA)
 * Chal and Pt are i128 in both. */
typedef struct {
    uint32_t eval_kind;       /* zg_eval_kind                                   */
    uint32_t degree_plus_one; /* D of BinaryPoly<D> (1..64); 1 for I32          */
    uint32_t code_kind;       /* zg_code_kind                                   */
    uint32_t rep;             /* repetition factor (inverse rate), 4            */
    uint32_t num_vars;        /* poly_size = 2^num_vars                         */
    uint32_t row_len;         /* power of two dividing poly_size                */
    uint32_t iprs_depth;      /* 0 => IprsCode::new_with_optimal_depth          */
    uint32_t comb_limbs;      /* CombR = Int<comb_limbs> (64-bit limbs)          */
    uint32_t field_limbs;     /* F = MontyField<field_limbs>, 3 or 4            */
    uint32_t num_openings;    /* NUM_COLUMN_OPENINGS (147 in the reference)     */
} zg_params_desc;

/* Derived dimensions of a parameter set. */
typedef struct {
    uint32_t num_rows, row_len, codeword_len;
    uint32_t depth, base_len, base_dim; /* IPRS only */
    uint32_t eval_bytes, cw_bytes, comb_bytes, field_bytes;
} zg_params_info;

typedef struct zg_ctx zg_ctx;
typedef struct zg_params zg_params;
typedef struct zg_hint zg_hint;
typedef struct zg_transcript zg_transcript;
typedef struct zg_server zg_server;

/* ---- library / context --------------------------------------------------- */
const char *zg_last_error(void);
const char *zg_version(void);
/* Creates a context on a CUDA device (one stream, scratch arenas). */
zg_status zg_ctx_create(int device, zg_ctx **out);
zg_status zg_ctx_destroy(zg_ctx *ctx);
/* Number of kernels this context launched so far (for measurement). */
uint64_t zg_ctx_kernel_launches(const zg_ctx *ctx);
/* Stream used by the context (a cudaStream_t). */
void *zg_ctx_stream(zg_ctx *ctx);
/* Measurement (no counterpart in the reference): when enabled, CUDA events are
 * recorded on the launching stream around every kernel launch.  The report
 * (synchronizes the stream) writes "name,launches,total_ms\n" lines and resets
 * the totals; *len receives the length needed. */
zg_status zg_ctx_set_kernel_timing(zg_ctx *ctx, int enable);
zg_status zg_ctx_kernel_timing_report(zg_ctx *ctx, char *buf, size_t cap, size_t *len);
/* Failure detection self-test (no counterpart in the reference).  The
 * tensor-core kernels bound every wait on an mbarrier (about a second); a wait
 * that runs out makes the kernel skip its work, free its tensor memory, return,
 * and write a code into the device's status word, which every later
 * synchronisation reports as ZG_ERR_CUDA.  This call runs a one-block probe
 * whose wait can never complete (nothing arrives on its barrier), waits for
 * it, writes the status word it left (4 = the probe's timeout code) to
 * *status_seen, and clears the word.  It takes about a second; the context
 * stays usable.  Run it while no other work is in flight on the device: it
 * clears the device's word. */
zg_status zg_selftest_bounded_wait(zg_ctx *ctx, uint32_t *status_seen);
/* Host-side fault injection for tests of the error paths (no counterpart in the
 * reference): the n-th device allocation made from now on by any context of
 * the process (n >= 1; n = 0 disarms) fails as if the device were out of
 * memory, without calling CUDA or touching the GPU.  The call that made it
 * returns ZG_ERR_OOM ("injected allocation failure"); a server request whose
 * lane allocation fails completes with that status. */
zg_status zg_debug_fail_allocation(uint32_t n);

/* ---- setup: ZipPlus::setup + IprsCode::new / RaaCode::new -----------------
 * ctx may be NULL for host-only parameters (tables, encode_wide, verify);
 * device entry points then return ZG_ERR_NO_DEVICE. */
zg_status zg_params_create(zg_ctx *ctx, const zg_params_desc *desc, zg_params **out);
zg_status zg_params_destroy(zg_params *p);
zg_status zg_params_get_info(const zg_params *p, zg_params_info *info);
/* Twiddle tables exactly as Radix8PnttParams holds them (params.rs:31-57):
 * base_matrix base_dim x base_len, butterfly twiddles per stage k
 * (base_dim*8^k x 7 x 8), all int64.  Either pointer may be NULL. */
zg_status zg_params_iprs_tables(const zg_params *p, int64_t *base_matrix, int64_t *twiddles);
/* The two RAA permutations (raa.rs:76-80), codeword_len uint32 each. */
zg_status zg_params_raa_perms(const zg_params *p, uint32_t *perm1, uint32_t *perm2);

/* ---- LinearCode::encode via ZipPlus::encode_rows (phase_commit.rs:159) ----
 * evals: num_rows*row_len evaluations; cw_out: num_rows x codeword_len Cw. */
zg_status zg_encode_rows(zg_params *p, const void *evals, void *cw_out);
zg_status zg_encode_rows_d(zg_params *p, const void *evals_d, void *cw_out_d, void *stream);
/* LinearCode::encode_wide on Int<limbs> rows (iprs.rs:148-150): row is
 * row_len x limbs uint64, out codeword_len x limbs. */
zg_status zg_encode_wide(zg_params *p, const uint64_t *row, uint32_t limbs, uint64_t *out);

/* LinearCode::encode_f (code.rs:69-71; iprs.rs:88-106, raa.rs:155-160,
 * raa_sign_flip.rs:101-106): row_len prime-field elements (Montgomery inners of
 * `limbs` u64 of the odd prime `modulus`, limbs 1..4) encoded over the field
 * into codeword_len elements, on the parameters' device.  zg_encode_f takes
 * host buffers; zg_encode_f_d device buffers and a cudaStream_t (NULL = the
 * context's stream, asynchronous). */
zg_status zg_encode_f(zg_params *p, const uint8_t *modulus, uint32_t limbs, const uint64_t *row, uint64_t *out);
zg_status zg_encode_f_d(zg_params *p, const uint8_t *modulus, uint32_t limbs, const uint64_t *row_d,
                        uint64_t *out_d, void *stream);

/* ---- MerkleTree::new(rows).root() (merkle.rs:74-103) ----------------------
 * rows: n_rows x (width*elem_bytes) bytes, row-major; width a power of two. */
zg_status zg_merkle_root(zg_ctx *ctx, const void *rows, uint32_t n_rows, uint32_t width,
                         uint32_t elem_bytes, uint8_t root[32]);

/* MillerRabin::test to base 2 (primality/src/lib.rs:12-19, crypto-primes'
 * strong probable-prime test; the test get_random_field_cfg applies to each
 * transcript candidate): out[c] = 1 when candidate c (limbs u64 LE, 1..4 limbs)
 * is a base-2 strong probable prime.  Host only (eight candidates at a time
 * with AVX-512 IFMA when the CPU has it). */
zg_status zg_is_probable_prime_base2(const uint64_t *n, uint32_t limbs, uint32_t count, uint8_t *out);

/* ---- Allocation-free Merkle root ---------------------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory on their request path (a serving loop that reserves its device-memory
 * budget up front, or a host whose device buffers all come from its own pool):
 * cudaMalloc/cudaFree synchronize the device and can fail under memory
 * pressure, and this entry point calls neither, nor any other allocating
 * routine.  It computes the same root as zg_merkle_root over `width` leaves
 * whose preimages are consecutive `leaf_bytes`-byte ranges at leaves_d (device
 * memory, leaf-major, 4-byte aligned; leaf_bytes a multiple of 4), and writes the 32-byte root to root_d (device memory),
 * asynchronously on `stream` (a cudaStream_t; NULL = legacy default stream).
 * Its scratch is a fixed 4 MiB device array inside the library, held by every
 * GPU that loads it until the process exits: (2*width - 1) * 32 bytes of nodes
 * plus width * ceil(leaf_bytes / 1024) * 32 bytes of chunk chaining values for
 * leaves longer than 1024 bytes must fit (e.g. 65536 leaves of at most 1024
 * bytes); larger inputs return ZG_ERR_INVALID_PARAM.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress, with that
 * device current); make that first call before any stream capture.  That
 * address belongs to the device's primary context: after cudaDeviceReset the
 * entry point must not be called again in the same process.  All calls on a
 * device share the array: calls that overlap on the GPU race. */
zg_status zg_merkle_root_noalloc_d(const void *leaves_d, uint32_t width, uint32_t leaf_bytes,
                                   uint8_t *root_d, void *stream);

/* ---- ZipPlus::commit (phase_commit.rs:61-101) ------------------------------
 * polys[i] points at poly i's 2^num_vars evaluations.  The hint (codewords and
 * Merkle layers) stays on the device.  commit_single == batch 1. */
zg_status zg_commit(zg_params *p, const void *const *polys, uint32_t batch, zg_hint **hint,
                    uint8_t root[32]);
/* Same with device-resident evaluations: polys_d holds batch polys back to back. */
zg_status zg_commit_d(zg_params *p, const void *polys_d, uint32_t batch, zg_hint **hint,
                      uint8_t root[32]);
zg_status zg_hint_free(zg_hint *hint);
uint32_t zg_hint_batch(const zg_hint *hint);
/* Copies the hint's codeword of poly `poly` to the host, row-major. */
zg_status zg_hint_codeword(const zg_hint *hint, uint32_t poly, void *cw_out);

/* ---- PcsProverTranscript (pcs_transcript.rs:44-222) ------------------------ */
/* new_from_commitments: absorbs each root as a slice. */
zg_status zg_transcript_new(const uint8_t *roots, uint32_t n_roots, zg_transcript **out);
zg_status zg_transcript_free(zg_transcript *t);
zg_status zg_transcript_absorb(zg_transcript *t, const uint8_t *buf, size_t n);
zg_status zg_transcript_absorb_slice(zg_transcript *t, const uint8_t *buf, size_t n);
/* get_challenge::<T>() for a T of n bytes (traits.rs:329-335). */
zg_status zg_transcript_challenge(zg_transcript *t, uint8_t *out, size_t n);
/* get_random_field_cfg::<MontyField<limbs>, Uint<limbs>, MillerRabin>
 * (traits.rs:364-374): samples and remembers the prime; modulus_out may be
 * NULL (else 8*limbs bytes). */
zg_status zg_transcript_sample_field(zg_transcript *t, uint32_t limbs, uint8_t *modulus_out);
/* Proof bytes written so far (the reference's `stream`). */
zg_status zg_transcript_proof(const zg_transcript *t, const uint8_t **data, size_t *len);

/* ---- ZipPlus::prove (phase_prove.rs:85-253) --------------------------------
 * Requires zg_transcript_sample_field first.  polys as for zg_commit (host);
 * point: num_vars i128 coordinates (Pt = i128).  eval_out: 8*field_limbs
 * bytes (Montgomery inner of the returned F).  Appends the proof to t. */
zg_status zg_prove(zg_params *p, zg_transcript *t, const void *const *polys, uint32_t batch,
                   const uint8_t *point, const zg_hint *hint, uint8_t *eval_out);
zg_status zg_prove_d(zg_params *p, zg_transcript *t, const void *polys_d, uint32_t batch,
                     const uint8_t *point, const zg_hint *hint, uint8_t *eval_out);
/* ZipPlus::prove_f (phase_prove.rs:119-253): as zg_prove with the point already
 * in the field (Zinc+ step 7 opens the witness columns at r_0 this way):
 * point_f is num_vars Montgomery inners of field_limbs u64 each, reduced mod the
 * transcript's prime.  zg_prove_f_d takes the polynomials in device memory. */
zg_status zg_prove_f(zg_params *p, zg_transcript *t, const void *const *polys, uint32_t batch,
                     const uint64_t *point_f, const zg_hint *hint, uint8_t *eval_out);
zg_status zg_prove_f_d(zg_params *p, zg_transcript *t, const void *polys_d, uint32_t batch,
                       const uint64_t *point_f, const zg_hint *hint, uint8_t *eval_out);

/* Whole-request convenience: commit, new_from_commitment, sample field, prove.
 * Writes root, eval and the proof (proof_len in/out: capacity/size). */
zg_status zg_commit_prove(zg_params *p, const void *const *polys, uint32_t batch,
                          const uint8_t *point, uint8_t root[32], uint8_t *eval_out,
                          uint8_t *proof, size_t *proof_len);
zg_status zg_commit_prove_d(zg_params *p, const void *polys_d, uint32_t batch,
                            const uint8_t *point, uint8_t root[32], uint8_t *eval_out,
                            uint8_t *proof, size_t *proof_len);
/* Batched form: n independent requests, each one commit_single +
 * new_from_commitment + get_random_field_cfg + prove of one polynomial at its
 * own point, spread over `lanes` concurrent lanes (each a CUDA stream with its
 * own scratch, driven by its own host thread, so one lane's Fiat-Shamir work
 * overlaps the others' kernels).  Every output is byte-identical to a
 * sequential zg_commit_prove of the same request.  polys[i]: 2^num_vars
 * evaluations in host memory, or in device memory when polys_on_device != 0.
 * points: n x num_vars i128.  roots: n x 32; evals: n x 8*field_limbs bytes;
 * proofs[i]: buffer of proof_lens[i] bytes (in: capacity, out: size).
 * latency_ms (may be NULL): per-request service time. */
zg_status zg_commit_prove_many(zg_params *p, uint32_t n, const void *const *polys,
                               int polys_on_device, const uint8_t *points, uint8_t *roots,
                               uint8_t *evals, uint8_t *const *proofs, size_t *proof_lens,
                               uint32_t lanes, double *latency_ms);
/* ---- Batched commit of independent polynomials of mixed shapes ---------------
 * n calls of ZipPlus::commit_single (phase_commit.rs:61-101, batch of one, one
 * Merkle tree each), polynomial i under params[i] (all created on ctx;
 * destroying a parameter set drops the plans that use it).  Polynomials sharing a params handle are encoded and hashed in one
 * launch chain; the chains run on `lanes` concurrent streams.  Roots-only calls
 * (hints == NULL) keep a plan per batch shape (the sequence of params handles):
 * the first call times the kernel variants of each group shape (autotune),
 * then captures every launch of the batch as one CUDA graph, which later calls
 * replay.  Results are identical to n sequential zg_commit calls.
 * polys[i]: host memory, or device memory when polys_on_device != 0.  Device
 * inputs, and host inputs that are all page-locked, are copied by DMA from the
 * caller's buffers, whose addresses the captured graph holds (it is captured
 * again when they change); other host inputs go through a pinned staging copy.  roots: n x 32 (may
 * be NULL when hints are requested); hints (may be NULL): n handles, each freed
 * with zg_hint_free; their device memory is shared per group and released with
 * the group's last hint.  The library keeps at most 8 plans per context, each
 * with its own lanes and device arena (released by zg_ctx_destroy). */
typedef struct {
    uint32_t lanes;    /* concurrent streams, 0 = 4 (max 16) */
    int use_graph;     /* roots-only calls: capture and replay a CUDA graph */
    int autotune;      /* time the kernel variants of each group shape once */
    int base_variant;  /* -1 = tuned/heuristic; binary IPRS base layer: 6 / 7 tcgen05
                          persistent (128 / 64 base rows per tile, accumulators
                          in tensor memory), 8 / 9 tcgen05 one tile per block,
                          0 mma.sync (8 chunk rows per block), 4 / 5 mma.sync
                          with 4 / 16, 1 shared-memory staged, 2 packed-lane,
                          3 plain */
    int leaf_variant;  /* -1 = tuned/heuristic; one-chunk leaves: 0 warp-coalesced, 1 per-thread */
} zg_batch_opts;
zg_status zg_commit_batch(zg_ctx *ctx, uint32_t n, zg_params *const *params,
                          const void *const *polys, int polys_on_device, const zg_batch_opts *opts,
                          uint8_t *roots, zg_hint **hints);

/* ---- Request server: continuous batching of commit+prove jobs --------------
 * Each request is zg_commit_prove of one polynomial (commit_single,
 * new_from_commitment, get_random_field_cfg, prove; byte-identical outputs).
 * `workers` threads, each with its own stream and scratch, take requests as
 * soon as they are free: the oldest request whose device footprint (input,
 * codeword, Merkle layers, kernel scratch) fits the HBM budget is admitted
 * together with queued requests of the same params handle (committed in one
 * launch chain); codewords and Merkle layers stay on the device until the
 * request's proof is done.  A request that does not fit may be passed by later
 * ones for at most max_skip_ms, after which it blocks admission until memory
 * frees up.  Requests arriving while others run join at the next free worker,
 * so their kernels overlap with the running ones.  Between groups an idle
 * worker keeps at most a quarter of the budget (of free memory when the budget
 * is 0), split over the workers, as scratch and cached blocks. */
typedef struct {
    uint32_t workers;      /* concurrent lanes, 0 = 4 (max 32) */
    uint64_t hbm_budget;   /* device bytes in flight, 0 = 60% of free memory at creation */
    uint32_t max_group;    /* most requests per launch chain, 0 = 16 */
    uint32_t max_skip_ms;  /* how long the oldest request may be passed by smaller ones */
    uint64_t group_max_bytes; /* only requests whose footprint is at most this share a
                                 launch chain, 0 = 1 GiB */
} zg_server_opts;
typedef struct {
    zg_status status;
    size_t proof_len;
    double latency_ms;  /* submit -> proof written */
    double queue_ms;    /* submit -> admitted */
    uint32_t group_size;
} zg_server_result;
typedef struct {
    uint64_t completed, queued, in_flight, groups, grouped_requests;
    uint64_t budget, reserved, peak_reserved;
    /* wall time summed over workers: input copies, group commits, prime
     * sampling (get_random_field_cfg), proves */
    double ms_input, ms_commit, ms_prime, ms_prove;
} zg_server_stats;
zg_status zg_server_create(zg_ctx *ctx, const zg_server_opts *opts, zg_server **out);
/* poly (2^num_vars evaluations, host memory), root (32 B), eval (8 * field_limbs B)
 * and proof (proof_cap >= zg_proof_size(p, 1)) must stay valid until the request
 * is waited for; point: num_vars i128 (copied).  ZG_ERR_OOM if the request can
 * never fit the budget. */
zg_status zg_server_submit(zg_server *s, zg_params *p, const void *poly, const uint8_t *point,
                           uint8_t *root, uint8_t *eval, uint8_t *proof, size_t proof_cap,
                           uint64_t *id);
/* Waits for request `id` (timeout_ms < 0: no limit; ZG_ERR_TIMEOUT if still
 * running) and releases it; returns the request's own status. */
zg_status zg_server_wait(zg_server *s, uint64_t id, int timeout_ms, zg_server_result *res);
zg_status zg_server_get_stats(zg_server *s, zg_server_stats *out);
/* Finishes every submitted request, then stops the workers. */
zg_status zg_server_destroy(zg_server *s);

/* Exact proof length for a batch (phase_commit.rs:739-805 formula). */
size_t zg_proof_size(const zg_params *p, uint32_t batch);

/* ---- ZipPlus::verify (phase_verify.rs:100-304) ------------------------------
 * Fresh verifier transcript: absorbs root, samples the field, samples alphas,
 * then runs the four checks.  ZG_OK accepts; ZG_ERR_INVALID_OPEN rejects;
 * ZG_ERR_SERIALIZATION for a truncated/malformed proof. */
zg_status zg_verify(zg_params *p, const uint8_t root[32], uint32_t batch, const uint8_t *point,
                    const uint8_t *eval, const uint8_t *proof, size_t proof_len);

/* ---- PIOP sumcheck prover ----------------------------------------------------
 * One group of MLEs with the combination function
 *   comb(v) = (sum_k coeffs[k] * prod_{q in [offsets[k], offsets[k+1])} v[indices[q]])
 *             * prod_f (factor_a[f] + factor_b[f] * v[factor_mles[f]]),
 * i.e. the `comb_fn: Fn(&[F]) -> F` of MLSumcheck::prove_as_subprotocol
 * (piop/src/sumcheck.rs:163-215) and of MultiDegreeSumcheckGroup
 * (piop/src/sumcheck/multi_degree.rs:44-67) written as a sum of products
 * times affine factors (n_factors = 0: no factor).  The combined-polynomial
 * resolver's comb_fn of a linear UAIR is folded(v) * (1 - sel) * eq_r
 * (combined_poly_resolver.rs:158-172): a sum of one-MLE products and two factors.
 * mles: n_mles x 2^nvars field elements, Montgomery inner values of `limbs`
 * u64 each (DenseMultilinearExtension<F::Inner>), MLE-major; coeffs:
 * n_products Montgomery inners; offsets: n_products + 1 entries; factor_a,
 * factor_b: n_factors Montgomery inners each. */
typedef struct {
    uint32_t degree;     /* the group's degree (longest product + n_factors), <= 8 */
    uint32_t n_mles;
    uint32_t n_products;
    const void *mles;    /* host, or device memory when mles_on_device != 0 */
    const uint64_t *coeffs;
    const uint32_t *offsets;
    const uint32_t *indices;
    uint32_t n_factors;
    const uint32_t *factor_mles;
    const uint64_t *factor_a;
    const uint64_t *factor_b;
} zg_sumcheck_group;

/* multi == 0: MLSumcheck::prove_as_subprotocol with one group; the proof is the
 * transcription of SumcheckProof (piop/src/sumcheck.rs:35-111).
 * multi != 0: MultiDegreeSumcheck::prove_as_subprotocol
 * (piop/src/sumcheck/multi_degree.rs:259-355), one shared challenge per round;
 * the proof is the transcription of MultiDegreeSumcheckProof
 * (multi_degree.rs:86-190).  modulus: `limbs` u64 LE (3 or 4), odd.  The round
 * messages and challenges go through `t` (the reference's Blake3Transcript).
 * proof_len: in capacity, out size (ZG_ERR_BUFFER_TOO_SMALL sets the size).
 * point_out (may be NULL): nvars challenges; finals_out (may be NULL): every
 * MLE of every group evaluated at the point (ProverState::randomness and the
 * final fold of prover.rs:95-247), in group order. */
zg_status zg_sumcheck_prove(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                            uint32_t nvars, int multi, const zg_sumcheck_group *groups,
                            uint32_t ngroups, int mles_on_device, uint8_t *proof,
                            size_t *proof_len, uint64_t *point_out, uint64_t *finals_out);

/* sum_x mle[x] * eq(x, point) (mle_eval_with_eq_table, poly/src/utils.rs:267-284):
 * the MLE (2^nvars Montgomery inners, host memory) at `point` (nvars inners,
 * bit k of x pairs with point[k]). */
zg_status zg_mle_evaluate(zg_ctx *ctx, const uint8_t *modulus, uint32_t limbs, const uint64_t *mle,
                          uint32_t nvars, const uint64_t *point, uint64_t *out);

/* ---- Zinc+ prover steps on the trace columns ----------------------------------
 * The step functions below keep their intermediate MLEs in the context's
 * arenas between phases (steps 4 and 5 prepare them, then run the sumcheck):
 * run one of them at a time per context. */
/* ---- Zinc+ prover steps 3 and 6 on the trace columns -------------------------
 * (protocol/src/prover.rs:385-415 step3_eval_projection and 497-532
 * step6_lift_and_project.)  Columns: n_bin binary-polynomial columns of
 * 2^nvars BinaryPoly<degree_plus_one> u64 words (bit l = coefficient l), column
 * after column, then n_int integer columns of 2^nvars i64.  Field: `limbs` u64
 * LE modulus, 3 or 4 limbs, odd; every field element is a Montgomery inner
 * (F::Inner of MontyField).
 *
 * zg_piop_eval_projection: project_trace_coeffs (piop/src/projections.rs:140-220:
 * binary coefficients become one or zero, integers F::from_with_cfg) followed by
 * evaluate_trace_to_column_mles at the projecting element a (projections.rs:
 * 227-301).  mles_out: (n_bin + n_int) MLEs of 2^nvars elements, MLE-major, the
 * layout zg_sumcheck_prove takes.  on_device != 0: the columns and mles_out are
 * device pointers (the MLEs can go straight into zg_sumcheck_prove with
 * mles_on_device); else host memory. */
zg_status zg_piop_eval_projection(zg_ctx *ctx, const uint8_t *modulus, uint32_t limbs,
                                  const uint64_t *bin_cols, uint32_t n_bin, uint32_t degree_plus_one,
                                  const int64_t *int_cols, uint32_t n_int, uint32_t nvars,
                                  const uint64_t *a, int on_device, uint64_t *mles_out);
/* zg_piop_lifted_evals: compute_lifted_evals (protocol/src/lib.rs:327-395) at
 * `point` (nvars elements, bit k of b pairs with point[k]): for binary column c,
 * coefficient l = sum_b eq(b, point) [bit l of c[b]]; for an integer column the
 * single coefficient sum_b eq(b, point) F(c[b]).  coeffs_out (host): n_bin x
 * degree_plus_one then n_int elements, untrimmed (DynamicPolynomialF::
 * new_trimmed drops trailing zero coefficients).  cols_on_device: the columns
 * are device pointers. */
zg_status zg_piop_lifted_evals(zg_ctx *ctx, const uint8_t *modulus, uint32_t limbs,
                               const uint64_t *bin_cols, uint32_t n_bin, uint32_t degree_plus_one,
                               const int64_t *int_cols, uint32_t n_int, uint32_t nvars,
                               const uint64_t *point, int cols_on_device, uint64_t *coeffs_out);
/* zg_piop_multipoint_eval: step 5, MultipointEval::prove_as_subprotocol
 * (piop/src/multipoint_eval.rs:119-231).  Samples n_shifts alphas then num_cols
 * gammas from `t` (get_field_challenges), builds eq(., r') and the shift selectors
 * next_c(r', .) (build_next_c_r_mle, poly/src/utils.rs:207-236), precombines the
 * columns as sum_j gamma_j v_j, and runs MLSumcheck of degree 2 over
 * eq * precombined + sum_k alpha_k next_k * v_{src_k}.  trace_mles: num_cols MLEs of
 * 2^nvars Montgomery inners (device memory when mles_on_device != 0, e.g. from
 * zg_piop_eval_projection); eval_point: r' (nvars inners); shift k: source column
 * shift_src[k] and shift shift_amount[k] < 2^nvars (ShiftSpec).  proof: the
 * SumcheckProof transcription (proof_len as for zg_sumcheck_prove); r0_out
 * (may be NULL): the sumcheck point r_0 (nvars inners). */
/* zg_piop_cpr_linear_prove: step 4 for a linear UAIR whose constraints are
 * homogeneous linear forms over the up and down (shifted) columns:
 * CombinedPolyResolver::prepare_sumcheck_group, MultiDegreeSumcheck with that
 * one group, and finalize_prover (piop/src/combined_poly_resolver.rs:71-247).
 * Draws the folding challenge alpha from `t`, builds the last-row selector,
 * eq(., r) at eval_point (the ideal check's point) and the down columns (source
 * column shifted up by the shift, zero padded), proves
 * sum_b (sum_k alpha^k g_k(b)) (1 - sel(b)) eq_r(b) (degree 3), then absorbs the
 * up and down columns' values at the sumcheck point.  coeffs: n_constraints x
 * (num_cols + n_shifts) Montgomery inners (constraint k's coefficients over the
 * up columns, then the down columns; projected scalars may appear here).
 * proof: the MultiDegreeSumcheckProof transcription; point_out (may be NULL):
 * the point r*; evals_out (may be NULL): up_evals then down_evals (CprProof). */
/* zg_piop_ideal_check_linear: step 2 for a linear UAIR, MLE first
 * (IdealCheckProtocol::prove_linear, piop/src/ideal_check.rs:137-176 with
 * combined_poly_builder::evaluate_combined_polynomials).  Draws nvars field
 * challenges from `t` as the point r (point_out), evaluates every up column (the
 * projected trace: binary columns as 0/1-coefficient polynomials, integer columns
 * as constants) and every shifted down column coefficient-wise at r, applies each
 * constraint's coefficients (n_constraints x (n_bin + n_int + n_shifts) Montgomery
 * inners over [binary up, integer up, down in shift order]) to those polynomial
 * values, and absorbs each constraint's combined value trimmed of trailing zero
 * coefficients (DynamicPolynomialF::new_trimmed).  combined_out: n_constraints x
 * degree_plus_one inners (zero padded); lengths_out: the trimmed lengths.  Shift
 * sources index the up columns (binary first).  cols_on_device: the columns are
 * device pointers. */
zg_status zg_piop_ideal_check_linear(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                                     const uint64_t *bin_cols, uint32_t n_bin, uint32_t degree_plus_one,
                                     const int64_t *int_cols, uint32_t n_int, uint32_t nvars,
                                     const uint32_t *shift_src, const uint32_t *shift_amount, uint32_t n_shifts,
                                     uint32_t n_constraints, const uint64_t *coeffs, int cols_on_device,
                                     uint64_t *point_out, uint64_t *combined_out, uint32_t *lengths_out);
zg_status zg_piop_cpr_linear_prove(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                                   const uint64_t *trace_mles, uint32_t num_cols, uint32_t nvars,
                                   const uint64_t *eval_point, const uint32_t *shift_src,
                                   const uint32_t *shift_amount, uint32_t n_shifts, uint32_t n_constraints,
                                   const uint64_t *coeffs, int mles_on_device, uint8_t *proof,
                                   size_t *proof_len, uint64_t *point_out, uint64_t *evals_out);
zg_status zg_piop_multipoint_eval(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                                  const uint64_t *trace_mles, uint32_t num_cols, uint32_t nvars,
                                  const uint64_t *eval_point, const uint32_t *shift_src,
                                  const uint32_t *shift_amount, uint32_t n_shifts, int mles_on_device,
                                  uint8_t *proof, size_t *proof_len, uint64_t *r0_out);

/* ---- Zinc+ prover, MLE first (ZincPlusPiop::prove::<MLE_FIRST = true>,
 * protocol/src/prover.rs:677-706) ------------------------------------------
 * A linear UAIR over binary-polynomial and integer columns (no arbitrary-
 * polynomial columns; lookups are a placeholder in the reference), e.g.
 * BigLinearUair (test-uair/src/lib.rs:325-382: 16 BinaryPoly<32> columns, 1
 * integer column, 16 shifts by 1, 17 constraints) or
 * BigLinearUairWithPublicInput (:458-489, its first 4 binary columns public).
 * The first n_pub_bin binary and the first n_pub_int integer columns are
 * public (UairTrace::public, uair/src/lib.rs:328-346): they are not committed
 * or opened, each of their entries is absorbed as 8 LE bytes after the roots
 * (absorb_public_columns, protocol/src/lib.rs:305-320), and their lifted
 * evaluations stay out of the proof.
 * Constraint k is sum_j coeffs[k][j] * col_j over [binary up, integer up, down
 * (shifted) columns in shift order]; shift sources index the up columns, binary
 * first.  Runs step 0 (commit both tables, absorb the roots of the binary, the
 * empty arbitrary and the integer table), step 1 (random prime of pp's
 * field_limbs), steps 2-6 on the GPU (zg_piop_* above), step 7 (prove_f of each
 * table at r_0) and writes the Proof transcription (protocol/src/lib.rs:87-189:
 * three commitments, the PCS stream, ideal check, resolver, multi-degree
 * sumcheck, multipoint evaluation, witness lifted evaluations).
 * pp_bin: BINPOLY parameters of num_vars (NULL when no binary column is a
 * witness); pp_int: ZG_EVAL_I64 parameters of num_vars (NULL when no integer
 * column is a witness), both with a device
 * and one context.  bin_cols: n_bin columns of 2^num_vars u64, column after
 * column; int_cols: n_int columns of 2^num_vars i64 (device pointers when
 * cols_on_device != 0).  proof_len: in capacity, out size. */
typedef struct {
    uint32_t n_bin;
    uint32_t n_int;
    uint32_t degree_plus_one;
    uint32_t n_shifts;
    const uint32_t *shift_src;
    const uint32_t *shift_amount;
    uint32_t n_constraints;
    const int64_t *coeffs; /* n_constraints x (n_bin + n_int + n_shifts) */
    uint32_t n_pub_bin;    /* public binary columns (the first ones), <= n_bin */
    uint32_t n_pub_int;    /* public integer columns (the first ones), <= n_int */
} zg_linear_uair;

zg_status zg_zinc_prove_mle_first(zg_params *pp_bin, zg_params *pp_int, const zg_linear_uair *uair,
                                  uint32_t num_vars, const uint64_t *bin_cols, const int64_t *int_cols,
                                  int cols_on_device, uint8_t *proof, size_t *proof_len);

/* ---- ZincPlusPiop::prove, both paths (protocol/src/prover.rs:677-706) --------
 * mle_first != 0: step1_mle_first + prove_linear, as zg_zinc_prove_mle_first
 * (linear constraints only); mle_first == 0: step1_combined + prove_combined
 * (the path the reference's Verify bench proves with, protocol/benches/
 * e2e.rs:346-354), which takes constraints of degree two and sends an empty
 * ideal-check value for each constraint in the zero ideal (ideal_check.rs:
 * 178-240).  The UAIR is a list of terms: constraint k is the sum over its
 * terms t in [term_offsets[k], term_offsets[k+1]) of term_coeffs[t] times the
 * product of the columns factor_cols[factor_offsets[t] .. factor_offsets[t+1])
 * (indices into [binary up, integer up, down in shift order]); a term has one
 * or two columns (constant terms are not taken).  zero_ideal[k] != 0 when
 * constraint k lies in the zero ideal (IdealOrZero::Zero).  Everything else
 * (tables, columns, public columns, proof buffer) is as for
 * zg_zinc_prove_mle_first. */
typedef struct {
    uint32_t n_bin;
    uint32_t n_int;
    uint32_t degree_plus_one;
    uint32_t n_shifts;
    const uint32_t *shift_src;
    const uint32_t *shift_amount;
    uint32_t n_constraints;
    const uint32_t *term_offsets;   /* n_constraints + 1, starting at 0 */
    const int64_t *term_coeffs;     /* one per term */
    const uint32_t *factor_offsets; /* n_terms + 1 */
    const uint32_t *factor_cols;
    const uint8_t *zero_ideal;      /* one per constraint */
    uint32_t n_pub_bin;
    uint32_t n_pub_int;
} zg_uair;

zg_status zg_zinc_prove(zg_params *pp_bin, zg_params *pp_int, const zg_uair *uair, uint32_t num_vars,
                        const uint64_t *bin_cols, const int64_t *int_cols, int cols_on_device, int mle_first,
                        uint8_t *proof, size_t *proof_len);

/* ---- Proof::read_transcription_bytes_exact (protocol/src/lib.rs:93-127) ------
 * Parses the Proof transcription that zg_zinc_prove writes (field of `limbs`
 * u64, num_vars rounds) into the places of its parts, checking every nested
 * length: the three commitments, the PCS stream, the ideal check values
 * (DynamicPolyVecF), the resolver's up and down evaluations (two Vec<F>), the
 * MultiDegreeSumcheckProof, the multipoint SumcheckProof and the witness lifted
 * evaluations.  Offsets are from the start of `proof`.  ZG_ERR_SERIALIZATION
 * when the bytes are not a Proof. */
typedef struct {
    uint8_t roots[3][32];
    uint64_t batch_sizes[3];
    uint8_t modulus[32]; /* the prime, `limbs` u64 LE */
    size_t zip_offset, zip_len;
    size_t ideal_check_offset, ideal_check_len;
    size_t resolver_offset, resolver_len;
    size_t multi_degree_offset, multi_degree_len;
    size_t multipoint_offset, multipoint_len;
    size_t lifted_offset, lifted_len;
    uint32_t n_ideal_values;      /* polynomials in the ideal check */
    uint32_t n_up_evals, n_down_evals;
    uint32_t multi_degree_groups; /* 1: the CPR group */
    uint32_t cpr_degree;          /* the CPR group's degree (max constraint degree + 2) */
    uint32_t n_lifted;            /* witness lifted evaluations */
} zg_proof_layout;

zg_status zg_proof_read(const uint8_t *proof, size_t len, uint32_t limbs, uint32_t num_vars, zg_proof_layout *out);

#ifdef __cplusplus
}
#endif
#endif /* ZIPGPU_H */
