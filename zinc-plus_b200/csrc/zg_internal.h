// Internal declarations shared by the zipgpu translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdarg>
#include <map>
#include <memory>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/zipgpu.h"
#include "zg_blake3.cuh"
#include "zg_field.cuh"

namespace zg {

// ----------------------------------------------------------------- errors
void set_error(const char *fmt, ...);

#define ZG_TRY(expr)                                                                              \
    do {                                                                                          \
        zg_status _s = (expr);                                                                    \
        if (_s != ZG_OK) return _s;                                                               \
    } while (0)

#define ZG_CUDA(call)                                                                             \
    do {                                                                                          \
        cudaError_t _e = (call);                                                                  \
        if (_e != cudaSuccess) {                                                                  \
            ::zg::set_error("CUDA error %s (%s) at %s:%d", cudaGetErrorName(_e),                  \
                            cudaGetErrorString(_e), __FILE__, __LINE__);                          \
            return _e == cudaErrorMemoryAllocation ? ZG_ERR_OOM : ZG_ERR_CUDA;                   \
        }                                                                                         \
    } while (0)

#define ZG_CHECK_LAUNCH(ctx)                                                                      \
    do {                                                                                          \
        (ctx)->launches++;                                                                        \
        ZG_CUDA(cudaGetLastError());                                                              \
    } while (0)

// Optional per-kernel CUDA-event timing (zg_ctx_set_kernel_timing): events are
// recorded on the launching stream around each launch.
#define ZG_KBEGIN(ctx, s, name) ::zg::ktimer_begin((ctx), (s), (name))
#define ZG_KEND(ctx, s)                                                                           \
    do {                                                                                          \
        ::zg::ktimer_end((ctx), (s));                                                             \
        ZG_CHECK_LAUNCH(ctx);                                                                     \
    } while (0)

// Raises a kernel's dynamic shared-memory limit to the device's opt-in maximum.
// Each launch passes its own size; setting the limit to that size per launch
// would race between threads launching the same kernel with different sizes.
int max_smem_optin();
template <class F>
inline cudaError_t allow_max_smem(F *func) {
    return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem_optin());
}

// ------------------------------------------------------- device buffers
// A growable device allocation owned by a context and reused across calls.
// With a memory pool set, allocation and release are stream-ordered on
// pool_stream (cudaMallocFromPoolAsync / cudaFreeAsync) and never synchronize
// the device.
struct DevBuf {
    void *ptr = nullptr;
    size_t cap = 0;
    cudaMemPool_t pool = nullptr;
    cudaStream_t pool_stream = nullptr;
    zg_status ensure(size_t bytes);
    void release();
    template <class T>
    T *as() const {
        return static_cast<T *>(ptr);
    }
};

// A growable pinned host allocation.
struct HostBuf {
    void *ptr = nullptr;
    size_t cap = 0;
    zg_status ensure(size_t bytes);
    void release();
    template <class T>
    T *as() const {
        return static_cast<T *>(ptr);
    }
};

struct zg_ctx_timer;
void ktimer_begin(zg_ctx *ctx, cudaStream_t s, const char *name);
void ktimer_end(zg_ctx *ctx, cudaStream_t s);
void ktimer_collect(zg_ctx *ctx);
// Host phase wall time since the previous mark, reported as "host:<name>".
void hphase_start(zg_ctx *ctx);
void hphase(zg_ctx *ctx, const char *name);
// Host-side fault injection: true when this device allocation is the one
// zg_debug_fail_allocation armed (the error message is set).
bool injected_allocation_failure();
void debug_fail_allocation(uint32_t n);
// Device block cache of a context.
void *ctx_alloc(zg_ctx *ctx, size_t bytes, size_t *got);
void ctx_release(zg_ctx *ctx, void *p, size_t bytes);
void ctx_cache_clear(zg_ctx *ctx);
// Frees cached blocks, largest first, until at most max_bytes stay cached.
void ctx_cache_trim(zg_ctx *ctx, size_t max_bytes);
// Waits until all work queued on ctx's stream is done (spinning, or sleeping
// when the context has a blocking-sync event).
cudaError_t ctx_sync(zg_ctx *ctx);
// Status word of a device, in mapped pinned host memory: a kernel whose
// bounded wait ran out writes a code into it (umma::kStatus*), skips its work and
// returns.  device_status reports a set word as cudaErrorLaunchTimeout.
uint32_t *device_status_word(int device);
cudaError_t device_status(int device);
// Current value of a device's status word, and its reset to 0 (both with the
// device's work drained).
uint32_t device_status_value(int device);
void device_status_clear(int device);
// One-block kernel whose mbarrier wait runs out and sets kStatusProbeTimeout.
zg_status launch_wait_probe(zg_ctx *ctx, cudaStream_t s);
// Routes a fresh context's hint blocks and scratch through a memory pool.
void ctx_use_pool(zg_ctx *ctx, cudaMemPool_t pool);
// Device bytes held by a context's scratch arenas, and their release.
size_t ctx_scratch_bytes(const zg_ctx *ctx);
void ctx_scratch_release(zg_ctx *ctx);

struct BatchPlan;
// Drops the cached batch plans that use parameter set p (before p is freed).
void drop_plans_of(zg_ctx *ctx, const zg_params *p);
// Creates child contexts of ctx until it has n lanes.
zg_status ensure_lanes(zg_ctx *ctx, uint32_t n);
// validate_input's bit budget for linear combinations (pcs/utils.rs:24-54).
zg_status validate_budget(const zg_params *p, uint32_t batch);

// One pending timed launch.
struct KernelEvent {
    const char *name;
    cudaEvent_t start, stop;
};

}  // namespace zg

struct zg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t launches = 0;
    int num_sms = 0;
    std::mutex mu;  // one call at a time per context
    // scratch arenas
    zg::DevBuf evals;     // staged evaluations
    zg::DevBuf stage_a;   // pNTT intermediates
    zg::DevBuf stage_b;
    zg::DevBuf stage_c;   // third pNTT buffer (depth >= 3)
    zg::DevBuf chunk_cv;  // per-chunk BLAKE3 chaining values for long leaves
    zg::DevBuf wprime;    // alpha-projected rows (CombR)
    zg::DevBuf prove_in;  // small per-prove inputs (alphas, points, coeffs, indices)
    zg::DevBuf prove_out; // b partials, combined row + openings
    zg::DevBuf sc_arena;  // sumcheck: staged MLEs, fold buffers, comb tables, partials
    zg::DevBuf piop_arena;  // PIOP step 5: the packed MLEs handed to the sumcheck
    zg::DevBuf trace_arena; // Zinc+ prover: the trace columns copied from the host
    zg::DevBuf mle_arena;   // Zinc+ prover: the projected column MLEs (steps 3-5)
    zg::HostBuf pin_in, pin_out;
    // kernel timing
    bool timing = false;
    std::vector<zg::KernelEvent> pending;
    std::vector<cudaEvent_t> event_pool;
    std::vector<std::pair<std::string, std::pair<double, uint64_t>>> totals;  // name -> (ms, n)
    std::chrono::steady_clock::time_point hmark;
    // device block cache: freed hint blocks are kept for reuse (no cudaFree on
    // the request path); released by zg_ctx_destroy.
    std::mutex cache_mu;
    std::multimap<size_t, void *> cache;
    // child contexts (same device) used as concurrent lanes by batched calls
    std::vector<zg_ctx *> lanes;
    // batched commit: captured plans by batch shape, autotuned kernel choices
    // by group shape ((base, leaf) variant), launch count correction for
    // graph capture and replay
    std::vector<std::pair<std::string, std::shared_ptr<zg::BatchPlan>>> plans;
    std::map<std::string, std::pair<int, int>> tune_cache;
    int64_t launch_adjust = 0;
    // stream-ordered pool for hint blocks and scratch (request-server lanes);
    // NULL: blocks come from the context's cache, scratch from cudaMalloc
    cudaMemPool_t pool = nullptr;
    // Waits for the stream by sleeping on a blocking-sync event instead of
    // spinning (lanes on which several host threads wait at once).
    cudaEvent_t sync_event = nullptr;
    // device pointer of this device's status word (device_status_word)
    uint32_t *status = nullptr;
};

namespace zg {
// Base rows per tile of the tcgen05 base-layer operand image.
constexpr uint32_t kUmmaImgRows = 128;
}  // namespace zg

struct zg_params {
    zg_ctx *ctx = nullptr;
    uint64_t uid = 0;  // unique per parameter set in the process (addresses get reused)
    zg_params_desc d{};
    zg_params_info info{};
    uint32_t D = 1;  // lanes per evaluation (coefficients of BinaryPoly)
    // IPRS tables (host: exactly the reference's layout; device: int32 copies)
    std::vector<int64_t> bm;  // base_dim x base_len
    std::vector<int64_t> tw;  // stage k: (base_dim*8^k) x 7 x 8, stages back to back
    int32_t *d_bmT = nullptr; // base_len x base_dim (transposed)
    int32_t *d_bmP = nullptr; // base_len x round_up(base_dim, 8) (transposed, zero padded)
    uint8_t *d_bmL = nullptr; // [3][base_dim][round_up(base_len, 32)] u8 limbs of the base matrix
    // Operand image of the tcgen05 base layer: per tile of kUmmaImgRows base
    // rows, two limbs (u8 low byte, s8 high byte) of bm[r][c] + bm_off[r], each
    // [round_up(base_len, 128) / 128][kUmmaImgRows][128] in the 128-byte
    // swizzle; bm_off[r] puts row r in [-2^15, 2^15).  NULL when a row spans
    // more than 2^16 values.  d_bmOff holds -bm_off, padded to whole tiles.
    uint8_t *d_bmU = nullptr;
    int32_t *d_bmOff = nullptr;
    uint32_t umma_kp = 0;  // round_up(base_len, 128)
    int32_t *d_tw = nullptr;  // stage k: [56][sub_k], stages back to back
    // depth 2 only: per base position rb, 576 int32 twiddles in use order:
    // [r0][j] for stage 0 (64), then [r0][r1][j] for stage 1 (512); j = 0 unused
    int32_t *d_tw2r = nullptr;
    std::vector<size_t> tw_off;      // offset of each stage in tw (host, [i][j-1][t])
    std::vector<size_t> tw_dev_off;  // offset of each stage in d_tw (device, [56][sub])
    // RAA permutations
    std::vector<uint32_t> perm1, perm2;
    uint32_t *d_perm = nullptr;  // perm1 then perm2
};

namespace zg {
// A device block shared by the hints of polynomials committed in one launch
// chain; it returns to the owning context's cache with the last hint.
struct SharedBlock {
    zg_ctx *lane = nullptr;
    void *ptr = nullptr;
    size_t bytes = 0;
    ~SharedBlock();
};
}  // namespace zg

struct zg_hint {
    std::shared_ptr<zg::SharedBlock> shared;  // set instead of `block` for group commits
    zg_params *params = nullptr;
    zg_ctx *lane = nullptr;    // context whose block cache owns `block`
    uint32_t batch = 0;
    uint32_t nrows = 0;        // batch * num_rows
    void *block = nullptr;     // one cached device block holding both arrays
    size_t block_bytes = 0;
    uint8_t *d_cw = nullptr;   // leaf-major: codeword_len x nrows x cw_bytes
    uint8_t *d_tree = nullptr; // Merkle layers, leaves first, root last, 32 B nodes;
                               // layer k starts at node 2C - 2(C >> k)
    uint32_t depth = 0;        // log2(codeword_len)
    uint8_t root[32];
};

struct zg_transcript {
    zg::b3::Hasher h;
    std::vector<uint8_t> stream;
    bool has_field = false;
    zg::FieldCfg f{};
};

namespace zg {

// ------------------------------------------------------- host utilities
void tr_absorb(zg_transcript *t, const void *buf, size_t n);
void tr_absorb_slice(zg_transcript *t, const void *buf, size_t n);
void tr_challenge(zg_transcript *t, uint8_t *out, size_t n);
i128 tr_challenge_i128(zg_transcript *t);
uint32_t tr_challenge_u32(zg_transcript *t);
void tr_absorb_field(zg_transcript *t, const uint64_t *inner);
// get_prime::<Uint<L>, MillerRabin> (transcript/src/lib.rs:58-72).
// threads: 0 = the OpenMP default team.
// One factor of a product of two trace columns (device memory): a binary
// column (2^nv BinaryPoly words) or an integer column (2^nv i64), read at row
// b + shift (zero past the last row: the zero padding of shifted columns).
struct IcFactor {
    const uint64_t *bin;
    const int64_t *ints;
    uint32_t shift;
};
// Combined-path ideal check of one product term: sum over the rows b < 2^nv - 1
// of eq(b, point) times each coefficient of a(b) * b(b); coefficients_out gets
// len_out = (a's length) + (b's length) - 1 Montgomery inners (binary: D, integer: 1).
zg_status ic_product_sums(zg_ctx *ctx, const FieldCfg &f, const uint64_t *point, uint32_t nv, const IcFactor &a,
                          const IcFactor &b, uint32_t D, std::vector<uint64_t> &coefficients_out, uint32_t &len_out);

// zg_piop_ideal_check_linear with absorb == false: the point is drawn and the
// values computed (untrimmed), nothing is absorbed.
zg_status ideal_check_linear_impl(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                                  const uint64_t *bin_cols, uint32_t n_bin, uint32_t degree_plus_one,
                                  const int64_t *int_cols, uint32_t n_int, uint32_t nvars, const uint32_t *shift_src,
                                  const uint32_t *shift_amount, uint32_t n_shifts, uint32_t n_constraints,
                                  const uint64_t *coeffs, int cols_on_device, uint64_t *point_out,
                                  uint64_t *combined_out, uint32_t *lengths_out, bool absorb);
// A product term of the CPR comb: coefficient (an integer) times the columns
// cols (indices into [up..., down...]) of constraint k.
struct CprProduct {
    uint32_t constraint;
    int64_t coeff;
    std::vector<uint32_t> cols;
};
// zg_piop_cpr_linear_prove with product terms added to the comb
// (sum_k alpha^k (linear_k + sum_t c_t prod cols_t)) (1 - sel) eq_r.
zg_status cpr_prove_impl(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus, uint32_t limbs,
                         const uint64_t *trace_mles, uint32_t num_cols, uint32_t nvars, const uint64_t *eval_point,
                         const uint32_t *shift_src, const uint32_t *shift_amount, uint32_t n_shifts,
                         uint32_t n_constraints, const uint64_t *coeffs, const std::vector<CprProduct> &products,
                         int mles_on_device, uint8_t *proof, size_t *proof_len, uint64_t *point_out,
                         uint64_t *evals_out);

void tr_get_prime(zg_transcript *t, int L, uint64_t *prime_out, int threads);
// Base-2 Miller-Rabin on up to eight odd candidates above one at once, with
// AVX-512 IFMA (mr_ifma.cpp); only when mr_ifma_available().
bool mr_ifma_available();
void mr_base2_x8(const uint64_t *cand, int L, int count, uint8_t *ok);
// The same search with the candidate tests of each round run by run_all(n, test).
void tr_get_prime_batched(zg_transcript *t, int L, uint64_t *prime_out, int group,
                          const std::function<void(int, const std::function<void(int)> &)> &run_all);
bool is_probable_prime_base2(const uint64_t *n, int L);

// IPRS parameters (params.rs:59-196); returns false if the reference rejects.
bool iprs_build_tables(uint32_t row_len, uint32_t depth, uint32_t rep, zg_params *p);
uint32_t iprs_optimal_depth(uint32_t row_len);
// rand 0.9 StdRng::seed_from_u64(seed) shuffle of 0..n (zip-plus/src/utils.rs:7-10).
void stdrng_shuffle_identity(uint64_t seed, uint32_t n, uint32_t *perm);

// ---------------------------------------------------------- pipelines
// `lane` supplies the stream, scratch and pinned buffers (a zg_ctx on p's device).
zg_status commit_device(zg_params *p, zg_ctx *lane, const void *polys_d, uint32_t batch,
                        zg_hint **out);
// tail_out: when not NULL, the proof after the b rows (combined row and column
// openings) is written there instead of being appended to t->stream.
// Kernel choices of a commit launch chain (-1: the built-in heuristic).
struct CommitTuning {
    int base_variant = -1;  // binary IPRS base layer: 0 tensor-core (4 / 5: 4 / 16 pairs per
                            // block), 1 smem-staged, 2 packed, 3 plain
    int leaf_variant = -1;  // one-chunk leaves: 0 warp-coalesced, 1 one thread per leaf
};
// Bytes of one polynomial's codeword (leaf-major) and Merkle tree in a group.
size_t group_cw_stride(const zg_params *p);
size_t group_tree_stride(const zg_params *p);
// True when m polynomials of p can share one launch chain.
bool group_fits(const zg_params *p, uint32_t m);
// Launches only: the segmented encode of m polynomials (consecutive in
// polys_d), the leaves of their m trees and all tree levels.  Polynomial k's
// codeword is at cw_d + k * group_cw_stride(p), its tree at
// tree_d + k * group_tree_stride(p) (root at node 2C - 2).
zg_status launch_commit_group(zg_params *p, zg_ctx *lane, const void *polys_d, uint32_t m,
                              uint8_t *cw_d, uint8_t *tree_d, cudaStream_t s,
                              const CommitTuning &tune);
// commit_single of m polynomials in one launch chain: hints[k] (may be NULL to
// drop the hints) and roots (m x 32, host).
zg_status commit_group_device(zg_params *p, zg_ctx *lane, const void *polys_d, uint32_t m,
                              zg_hint **hints, uint8_t *roots, const CommitTuning &tune);
// point: num_vars i128 coordinates (prove), or with point_is_field num_vars
// Montgomery inners of field_limbs u64 each (prove_f).
zg_status prove_device(zg_params *p, zg_ctx *lane, zg_transcript *t, const void *polys_d,
                       uint32_t batch, const uint8_t *point, const zg_hint *hint, uint8_t *eval_out,
                       uint8_t *tail_out, bool point_is_field = false);
zg_status verify_host(zg_params *p, const uint8_t root[32], uint32_t batch, const uint8_t *point,
                      const uint8_t *eval, const uint8_t *proof, size_t proof_len);

// ------------------------------------------------------------- kernels
// (defined in the .cu files; all launched on the given stream)
// seg_rows (leaf-major only): the rows are consecutive polynomials of seg_rows
// rows each, and each gets its own C x seg_rows codeword block; 0 = one block.
zg_status launch_encode(zg_params *p, zg_ctx *lane, const void *evals_d, uint32_t nrows,
                        uint8_t *out_d, bool leaf_major, cudaStream_t s, uint32_t seg_rows = 0,
                        int base_variant = -1);
// encode_wide (CL-limb wrapping integers) at n selected codeword positions
// (IPRS, depth <= 3): out is n x CL limbs.
zg_status launch_encode_wide_at(zg_params *p, zg_ctx *ctx, const uint64_t *row_d, uint32_t CL,
                                const uint32_t *pos_d, uint32_t n, uint64_t *out_d, cudaStream_t s);
// tree_width: the `width` leaves belong to width / tree_width trees, stored in
// consecutive blocks of 2 tree_width - 1 nodes; 0 = one tree.
// levels_done (may be NULL: none): set to the tree levels the leaf kernel
// already built (7 when it reduced each block's 128 leaves, else 0).
zg_status launch_leaf_hash(zg_ctx *ctx, const uint8_t *cw_d, uint32_t width, uint32_t leaf_bytes,
                           uint8_t *leaves_d, cudaStream_t s, uint32_t tree_width = 0,
                           int leaf_variant = -1, uint32_t *levels_done = nullptr);
// Levels k_start + 1 .. depth of ntrees trees of `width` leaves each (blocks of
// 2 width - 1 nodes), layer k_start already built.
zg_status launch_merkle_levels(zg_ctx *ctx, uint8_t *tree_d, uint32_t width, cudaStream_t s,
                               uint32_t ntrees = 1, uint32_t k_start = 0);

// Node offset of Merkle layer k for `width` leaves (layers stored leaves first).
inline size_t merkle_layer_off(size_t width, uint32_t k) { return 2 * width - 2 * (width >> k); }

}  // namespace zg
