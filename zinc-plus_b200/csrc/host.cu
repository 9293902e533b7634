// Host-side pieces of the backend: error reporting, buffers, the Fiat-Shamir
// transcript, Miller-Rabin prime sampling, IPRS parameter tables and the RAA
// permutations.
#include <omp.h>

#include <algorithm>
#include <cstring>

#include <functional>

#include "zg_internal.h"

namespace zg {

// ------------------------------------------------------------------ errors
static thread_local std::string g_err;

void set_error(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

const char *last_error() { return g_err.c_str(); }

// ----------------------------------------------------------------- buffers
// Host-side fault injection (zg_debug_fail_allocation): a countdown of device
// allocations; the one that brings it to zero fails as out of memory before
// any CUDA call is made.
static std::atomic<int64_t> g_fail_countdown{0};

bool injected_allocation_failure() {
    int64_t v = g_fail_countdown.load(std::memory_order_relaxed);
    while (v > 0) {
        if (g_fail_countdown.compare_exchange_weak(v, v - 1)) {
            if (v == 1) {
                set_error("injected allocation failure (zg_debug_fail_allocation)");
                return true;
            }
            return false;
        }
    }
    return false;
}

void debug_fail_allocation(uint32_t n) { g_fail_countdown.store((int64_t)n); }

zg_status DevBuf::ensure(size_t bytes) {
    if (bytes <= cap) return ZG_OK;
    if (injected_allocation_failure()) return ZG_ERR_OOM;
    release();
    size_t want = std::max(bytes, (size_t)256);
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&ptr, want, pool, pool_stream) : cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cap = 0;
        set_error("cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        return ZG_ERR_OOM;
    }
    cap = want;
    return ZG_OK;
}
void DevBuf::release() {
    if (ptr) {
        if (pool) cudaFreeAsync(ptr, pool_stream);
        else cudaFree(ptr);
    }
    ptr = nullptr;
    cap = 0;
}
zg_status HostBuf::ensure(size_t bytes) {
    if (bytes <= cap) return ZG_OK;
    release();
    size_t want = std::max(bytes, (size_t)4096);
    cudaError_t e = cudaMallocHost(&ptr, want);
    if (e != cudaSuccess) {
        ptr = nullptr;
        cap = 0;
        set_error("cudaMallocHost(%zu) failed: %s", want, cudaGetErrorString(e));
        return ZG_ERR_OOM;
    }
    cap = want;
    return ZG_OK;
}
void HostBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
}

// ------------------------------------------------------------ kernel timing
static void add_total(zg_ctx *ctx, const std::string &name, double ms);
static cudaEvent_t pool_get(zg_ctx *ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void ktimer_begin(zg_ctx *ctx, cudaStream_t s, const char *name) {
    if (!ctx || !ctx->timing) return;
    KernelEvent k{name, pool_get(ctx), pool_get(ctx)};
    cudaEventRecord(k.start, s);
    ctx->pending.push_back(k);
}

void ktimer_end(zg_ctx *ctx, cudaStream_t s) {
    if (!ctx || !ctx->timing || ctx->pending.empty()) return;
    cudaEventRecord(ctx->pending.back().stop, s);
}

// Folds completed launches into the per-kernel totals (synchronizes).
void ktimer_collect(zg_ctx *ctx) {
    if (ctx->pending.empty()) return;
    cudaStreamSynchronize(ctx->stream);
    for (KernelEvent &k : ctx->pending) {
        cudaEventSynchronize(k.stop);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, k.start, k.stop);
        add_total(ctx, k.name, ms);
        ctx->event_pool.push_back(k.start);
        ctx->event_pool.push_back(k.stop);
    }
    ctx->pending.clear();
}

static void add_total(zg_ctx *ctx, const std::string &name, double ms) {
    for (auto &t : ctx->totals)
        if (t.first == name) {
            t.second.first += ms;
            t.second.second += 1;
            return;
        }
    ctx->totals.push_back({name, {ms, 1}});
}

void hphase_start(zg_ctx *ctx) {
    if (ctx && ctx->timing) ctx->hmark = std::chrono::steady_clock::now();
}

void hphase(zg_ctx *ctx, const char *name) {
    if (!ctx || !ctx->timing) return;
    auto now = std::chrono::steady_clock::now();
    add_total(ctx, std::string("host:") + name,
              std::chrono::duration<double, std::milli>(now - ctx->hmark).count());
    ctx->hmark = now;
}

int max_smem_optin() {
    static std::atomic<int> cached{0};
    int v = cached.load();
    if (v == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
            cudaGetLastError();
            v = 48 * 1024;
        }
        cached.store(v);
    }
    return v;
}

// ------------------------------------------------------------ block cache
static size_t cache_round(size_t bytes) {
    const size_t g = bytes >= (2u << 20) ? (2u << 20) : 4096;
    return (bytes + g - 1) / g * g;
}

void *ctx_alloc(zg_ctx *ctx, size_t bytes, size_t *got) {
    if (injected_allocation_failure()) return nullptr;
    if (ctx->pool) {
        void *p = nullptr;
        if (cudaMallocFromPoolAsync(&p, bytes, ctx->pool, ctx->stream) != cudaSuccess) {
            cudaGetLastError();
            set_error("pool allocation of %zu bytes failed", bytes);
            return nullptr;
        }
        *got = bytes;
        return p;
    }
    const size_t want = cache_round(bytes);
    {
        std::lock_guard<std::mutex> lk(ctx->cache_mu);
        auto it = ctx->cache.lower_bound(want);
        if (it != ctx->cache.end() && it->first <= want + want / 2) {
            void *p = it->second;
            *got = it->first;
            ctx->cache.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaMalloc(&p, want) != cudaSuccess) {
        cudaGetLastError();
        ctx_cache_clear(ctx);  // give cached blocks back and retry once
        if (cudaMalloc(&p, want) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc(%zu) failed", want);
            return nullptr;
        }
    }
    *got = want;
    return p;
}

void ctx_release(zg_ctx *ctx, void *p, size_t bytes) {
    if (!p) return;
    if (ctx->pool) {
        cudaFreeAsync(p, ctx->stream);
        return;
    }
    std::lock_guard<std::mutex> lk(ctx->cache_mu);
    ctx->cache.insert({bytes, p});
}

SharedBlock::~SharedBlock() {
    if (ptr) ctx_release(lane, ptr, bytes);
}

void ctx_cache_trim(zg_ctx *ctx, size_t max_bytes) {
    std::lock_guard<std::mutex> lk(ctx->cache_mu);
    size_t total = 0;
    for (auto &kv : ctx->cache) total += kv.first;
    // drop the largest blocks first
    while (total > max_bytes && !ctx->cache.empty()) {
        auto it = std::prev(ctx->cache.end());
        total -= it->first;
        cudaFree(it->second);
        ctx->cache.erase(it);
    }
}

cudaError_t ctx_sync(zg_ctx *ctx) {
    cudaError_t e;
    if (!ctx->sync_event) {
        e = cudaStreamSynchronize(ctx->stream);
    } else {
        e = cudaEventRecord(ctx->sync_event, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(ctx->sync_event);
    }
    return e == cudaSuccess ? device_status(ctx->device) : e;
}

namespace {
constexpr int kMaxDevices = 64;
std::once_flag status_once;
uint32_t *status_host = nullptr;  // kMaxDevices words, mapped and portable
}  // namespace

uint32_t *device_status_word(int device) {
    std::call_once(status_once, [] {
        void *h = nullptr;
        if (cudaHostAlloc(&h, kMaxDevices * sizeof(uint32_t), cudaHostAllocMapped | cudaHostAllocPortable) ==
            cudaSuccess) {
            std::memset(h, 0, kMaxDevices * sizeof(uint32_t));
            status_host = static_cast<uint32_t *>(h);
        } else {
            cudaGetLastError();
        }
    });
    if (!status_host || device < 0 || device >= kMaxDevices) return nullptr;
    void *d = nullptr;
    if (cudaHostGetDevicePointer(&d, status_host + device, 0) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return static_cast<uint32_t *>(d);
}

uint32_t device_status_value(int device) {
    if (!status_host || device < 0 || device >= kMaxDevices) return 0;
    return reinterpret_cast<volatile uint32_t *>(status_host)[device];
}

void device_status_clear(int device) {
    if (!status_host || device < 0 || device >= kMaxDevices) return;
    reinterpret_cast<volatile uint32_t *>(status_host)[device] = 0;
}

cudaError_t device_status(int device) {
    if (!status_host || device < 0 || device >= kMaxDevices) return cudaSuccess;
    const uint32_t v = reinterpret_cast<volatile uint32_t *>(status_host)[device];
    if (v == 0) return cudaSuccess;
    set_error("a kernel's bounded wait ran out on device %d (status %u)", device, v);
    return cudaErrorLaunchTimeout;
}

void ctx_use_pool(zg_ctx *ctx, cudaMemPool_t pool) {
    ctx->pool = pool;
    for (DevBuf *b : {&ctx->evals, &ctx->stage_a, &ctx->stage_b, &ctx->stage_c, &ctx->chunk_cv,
                      &ctx->wprime, &ctx->prove_in, &ctx->prove_out, &ctx->sc_arena, &ctx->piop_arena,
                      &ctx->trace_arena, &ctx->mle_arena}) {
        b->pool = pool;
        b->pool_stream = ctx->stream;
    }
}

size_t ctx_scratch_bytes(const zg_ctx *ctx) {
    size_t n = 0;
    for (const DevBuf *b : {&ctx->evals, &ctx->stage_a, &ctx->stage_b, &ctx->stage_c, &ctx->chunk_cv,
                            &ctx->wprime, &ctx->prove_in, &ctx->prove_out, &ctx->sc_arena, &ctx->piop_arena,
                      &ctx->trace_arena, &ctx->mle_arena})
        n += b->cap;
    return n;
}

void ctx_scratch_release(zg_ctx *ctx) {
    for (DevBuf *b : {&ctx->evals, &ctx->stage_a, &ctx->stage_b, &ctx->stage_c, &ctx->chunk_cv,
                      &ctx->wprime, &ctx->prove_in, &ctx->prove_out, &ctx->sc_arena, &ctx->piop_arena,
                      &ctx->trace_arena, &ctx->mle_arena})
        b->release();
}

void ctx_cache_clear(zg_ctx *ctx) {
    std::lock_guard<std::mutex> lk(ctx->cache_mu);
    for (auto &kv : ctx->cache) cudaFree(kv.second);
    ctx->cache.clear();
}

// -------------------------------------------------------------- transcript
// Blake3Transcript (transcript/src/lib.rs:12-77; traits.rs:329-426).
void tr_absorb(zg_transcript *t, const void *buf, size_t n) {
    t->h.update(static_cast<const uint8_t *>(buf), n);
}
void tr_absorb_slice(zg_transcript *t, const void *buf, size_t n) {
    const uint8_t open = 0x06, close = 0x07;
    t->h.update(&open, 1);
    t->h.update(static_cast<const uint8_t *>(buf), n);
    t->h.update(&close, 1);
}
void tr_challenge(zg_transcript *t, uint8_t *out, size_t n) {
    t->h.xof(out, n);
    const uint8_t open = 0x12, close = 0x34;
    t->h.update(&open, 1);
    t->h.update(out, n);
    t->h.update(&close, 1);
}
i128 tr_challenge_i128(zg_transcript *t) {
    uint8_t b[16];
    tr_challenge(t, b, 16);
    u128 v = 0;
    for (int i = 15; i >= 0; i--) v = (v << 8) | b[i];
    return (i128)v;
}
uint32_t tr_challenge_u32(zg_transcript *t) {
    uint8_t b[4];
    tr_challenge(t, b, 4);
    return b3::load_le32(b);
}
// absorb_random_field: 0x03 | modulus | 0x05 | 0x01 | inner | 0x03
void tr_absorb_field(zg_transcript *t, const uint64_t *inner) {
    const uint8_t c3 = 3, c5 = 5, c1 = 1;
    const size_t nb = 8 * t->f.L;
    t->h.update(&c3, 1);
    t->h.update(reinterpret_cast<const uint8_t *>(t->f.p), nb);
    t->h.update(&c5, 1);
    t->h.update(&c1, 1);
    t->h.update(reinterpret_cast<const uint8_t *>(inner), nb);
    t->h.update(&c3, 1);
}

// Strong probable-prime test to base 2 (crypto-primes MillerRabin::test_base_two,
// called from primality/src/lib.rs:12-19).
template <int L>
static bool mr_base2(const uint64_t *n) {
    if (!(n[0] & 1)) return false;
    bool is_one = n[0] == 1;
    for (int i = 1; i < L; i++) is_one = is_one && n[i] == 0;
    if (is_one) return false;
    // Only n0 and R mod n are needed (field_cfg_init also builds R^2 and more by
    // 512 modular doublings, most of a test's time).  R mod n: from 2^(b-1) < n,
    // b = bit length of n, double 64L - b + 1 times modulo n.
    FieldCfg f;
    std::memset(&f, 0, sizeof f);
    f.L = L;
    for (int i = 0; i < L; i++) f.p[i] = n[i];
    {
        uint64_t inv = n[0];
        for (int i = 0; i < 6; i++) inv *= 2 - n[0] * inv;
        f.n0 = (uint64_t)0 - inv;
        int b = 64 * L;
        while (b > 0 && !((n[(b - 1) / 64] >> ((b - 1) % 64)) & 1)) b--;
        uint64_t y[L];
        for (int i = 0; i < L; i++) y[i] = 0;
        y[(b - 1) / 64] = 1ull << ((b - 1) % 64);
        for (int k = 0; k < 64 * L - b + 1; k++) {
            uint64_t c = 0;
            for (int i = 0; i < L; i++) {
                const uint64_t nc = y[i] >> 63;
                y[i] = (y[i] << 1) | c;
                c = nc;
            }
            if (c || ucmp<L>(y, n) >= 0) usub<L>(y, n);
        }
        for (int i = 0; i < L; i++) f.one[i] = y[i];
    }
    uint64_t nm1[L];
    for (int i = 0; i < L; i++) nm1[i] = n[i];
    nm1[0] -= 1;
    int s = 0;
    while (!((nm1[s / 64] >> (s % 64)) & 1)) s++;
    uint64_t d[L];
    for (int i = 0; i < L; i++) d[i] = 0;
    for (int i = 0; i + s < 64 * L; i++)
        if ((nm1[(i + s) / 64] >> ((i + s) % 64)) & 1) d[i / 64] |= 1ull << (i % 64);
    int top = 64 * L - 1;
    while (top >= 0 && !((d[top / 64] >> (top % 64)) & 1)) top--;
    uint64_t x[L], t[L];
    for (int i = 0; i < L; i++) x[i] = f.one[i];
    for (int b = top; b >= 0; b--) {
        fmul<L>(x, x, f.p, f.n0, t);
        for (int i = 0; i < L; i++) x[i] = t[i];
        if ((d[b / 64] >> (b % 64)) & 1) fadd<L>(x, x, f.p);
    }
    uint64_t mone[L];
    for (int i = 0; i < L; i++) mone[i] = f.one[i];
    fneg<L>(mone, f.p);
    if (ucmp<L>(x, f.one) == 0 || ucmp<L>(x, mone) == 0) return true;
    for (int i = 1; i < s; i++) {
        fmul<L>(x, x, f.p, f.n0, t);
        for (int k = 0; k < L; k++) x[k] = t[k];
        if (ucmp<L>(x, f.one) == 0) return false;
        if (ucmp<L>(x, mone) == 0) return true;
    }
    return false;
}

bool is_probable_prime_base2(const uint64_t *n, int L) {
    switch (L) {
        case 1: return mr_base2<1>(n);
        case 2: return mr_base2<2>(n);
        case 3: return mr_base2<3>(n);
        default: return mr_base2<4>(n);
    }
}

// get_prime: candidates are drawn one after another from the transcript
// (each absorbed raw); the first that passes Miller-Rabin is kept.  Candidates
// are generated ahead in groups and tested in parallel (run_all(n, test) runs
// test(0..n-1), possibly on several threads); the transcript is then rewound to
// the state right after the accepted candidate, so the result and the
// transcript state equal the sequential loop's.
void tr_get_prime_batched(zg_transcript *t, int L, uint64_t *prime_out, int group,
                          const std::function<void(int, const std::function<void(int)> &)> &run_all) {
    const int nb = 8 * L;
    group = std::max(1, group);
    std::vector<b3::Hasher> states(group);
    std::vector<uint64_t> cand((size_t)group * 4);
    std::vector<char> ok(group);
    // one task per eight candidates: with AVX-512 IFMA the eight odd candidates
    // above one are tested together, one per vector lane (mr_base2_x8)
    const bool vec = mr_ifma_available();
    const std::function<void(int)> test = [&](int q) {
        const int g0 = 8 * q, g1 = std::min(group, g0 + 8);
        uint64_t packed[8 * 4];
        int idx[8], np = 0;
        for (int g = g0; g < g1; g++) {
            uint64_t *c = &cand[(size_t)g * 4];
            bool zero = true;
            for (int i = 0; i < L; i++) zero = zero && c[i] == 0;
            if (zero) {
                ok[g] = 0;
                continue;
            }
            if (!(c[0] & 1)) {  // even: subtract one (full-width borrow)
                for (int i = 0; i < L; i++)
                    if (c[i]-- != 0) break;
            }
            bool one = c[0] == 1;
            for (int i = 1; i < L; i++) one = one && c[i] == 0;
            if (!vec || one) {
                ok[g] = is_probable_prime_base2(c, L) ? 1 : 0;
                continue;
            }
            for (int i = 0; i < L; i++) packed[(size_t)np * L + i] = c[i];
            idx[np++] = g;
        }
        if (np) {
            uint8_t res[8];
            mr_base2_x8(packed, L, np, res);
            for (int e = 0; e < np; e++) ok[idx[e]] = (char)res[e];
        }
    };
    for (;;) {
        b3::Hasher h = t->h;
        for (int g = 0; g < group; g++) {
            uint8_t buf[32];
            h.xof(buf, nb);
            h.update(buf, nb);
            states[g] = h;
            uint64_t *c = &cand[(size_t)g * 4];
            std::memset(c, 0, 32);
            std::memcpy(c, buf, nb);
        }
        run_all((group + 7) / 8, test);
        for (int g = 0; g < group; g++) {
            if (ok[g]) {
                t->h = states[g];
                std::memcpy(prime_out, &cand[(size_t)g * 4], nb);
                return;
            }
        }
        t->h = states[group - 1];
    }
}

void tr_get_prime(zg_transcript *t, int L, uint64_t *prime_out, int threads) {
    const int team = threads > 0 ? threads : omp_get_max_threads();
    // candidates generated ahead per round (speculative): eight per thread with
    // the vector test; without it one per thread (a single thread, one at a time)
    const int group = mr_ifma_available() ? 8 * team : team == 1 ? 1 : std::max(8, 2 * team);
    tr_get_prime_batched(t, L, prime_out, group, [team](int n, const std::function<void(int)> &fn) {
        if (team == 1) {
            for (int g = 0; g < n; g++) fn(g);
            return;
        }
#pragma omp parallel for schedule(dynamic, 1) num_threads(team)
        for (int g = 0; g < n; g++) fn(g);
    });
}

// ------------------------------------------------------------ IPRS tables
static uint64_t pow65537(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    b %= 65537;
    while (e) {
        if (e & 1) r = r * b % 65537;
        b = b * b % 65537;
        e >>= 1;
    }
    return r;
}
// normalize_field_element (params.rs:173-181): x >= (p-1)/2 maps to x - p.
static int64_t lift65537(uint64_t x) {
    int64_t v = (int64_t)x;
    return v >= 32768 ? v - 65537 : v;
}

uint32_t iprs_optimal_depth(uint32_t row_len) {
    // iprs.rs:43-51: depth = max(1, ceil(ilog2(max(1, row_len / 256)) / 3))
    uint32_t q = std::max<uint32_t>(1, row_len / 256);
    uint32_t lg = 31 - __builtin_clz(q);
    return std::max<uint32_t>(1, (lg + 2) / 3);
}

bool iprs_build_tables(uint32_t row_len, uint32_t depth, uint32_t rep, zg_params *p) {
    // Radix8PnttParams::new (params.rs:59-108)
    uint64_t cw = (uint64_t)row_len * rep;
    if (cw >= 65537 || 3 * depth >= 31) return false;
    uint64_t coeff = 1ull << (3 * depth);
    if (row_len % coeff) return false;
    uint64_t base_len = row_len / coeff, base_dim = base_len * rep;
    if (base_dim == 0 || (base_dim & (base_dim - 1))) return false;
    p->info.codeword_len = (uint32_t)cw;
    p->info.depth = depth;
    p->info.base_len = (uint32_t)base_len;
    p->info.base_dim = (uint32_t)base_dim;
    // base_matrix[r][c] = lift(w_bd^(r c)), w_n = 3^(65536/n) (generator 3, 2-adicity 16)
    p->bm.assign(base_dim * base_len, 0);
    uint64_t wbd = pow65537(3, 65536 / base_dim);
    for (uint64_t r = 0; r < base_dim; r++) {
        uint64_t wr = pow65537(wbd, r), x = 1;
        for (uint64_t c = 0; c < base_len; c++) {
            p->bm[r * base_len + c] = lift65537(x);
            x = x * wr % 65537;
        }
    }
    // butterfly_twiddles[k][i][j-1][t] = lift(BASE_TW[t] * w_C^(8^(depth-1-k) * i * j))
    static const int64_t base_tw[8] = {1, 4096, -256, 16, -1, -4096, 256, -16};
    uint64_t wc = pow65537(3, 65536 / cw);
    std::vector<uint64_t> roots(cw);
    roots[0] = 1;
    for (uint64_t i = 1; i < cw; i++) roots[i] = roots[i - 1] * wc % 65537;
    p->tw.clear();
    p->tw_off.clear();
    for (uint32_t k = 0; k < depth; k++) {
        uint64_t sub = base_dim << (3 * k), pw = 1ull << (3 * (depth - 1 - k));
        p->tw_off.push_back(p->tw.size());
        for (uint64_t i = 0; i < sub; i++)
            for (uint64_t j = 1; j <= 7; j++) {
                // the reference lifts the root first, then multiplies by the
                // lifted base twiddle mod p: the field value is the same.
                uint64_t rt = roots[(pw * i * j) % cw];
                for (int t = 0; t < 8; t++) {
                    uint64_t bt = (uint64_t)((base_tw[t] % 65537 + 65537) % 65537);
                    p->tw.push_back(lift65537(bt * rt % 65537));
                }
            }
    }
    return true;
}

// ------------------------------------------------------ rand 0.9 StdRng
// StdRng = ChaCha12 (rand_chacha 0.9: 64-bit block counter, stream 0), seeded
// by rand_core's seed_from_u64 (PCG32 output filling the 32-byte key).
namespace {
struct ChaCha12 {
    uint32_t key[8];
    uint64_t counter = 0;
    uint32_t block[16];
    int pos = 16;
    explicit ChaCha12(uint64_t seed) {
        for (int i = 0; i < 8; i++) {
            seed = seed * 6364136223846793005ull + 11634580027462260723ull;
            uint32_t xs = (uint32_t)(((seed >> 18) ^ seed) >> 27);
            uint32_t rot = (uint32_t)(seed >> 59);
            key[i] = (xs >> rot) | (xs << ((32 - rot) & 31));
        }
    }
    static uint32_t rl(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }
    void refill() {
        uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                          key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                          (uint32_t)counter, (uint32_t)(counter >> 32), 0u, 0u};
        uint32_t x[16];
        std::memcpy(x, s, sizeof x);
        auto qr = [&](int a, int b, int c, int d) {
            x[a] += x[b]; x[d] = rl(x[d] ^ x[a], 16);
            x[c] += x[d]; x[b] = rl(x[b] ^ x[c], 12);
            x[a] += x[b]; x[d] = rl(x[d] ^ x[a], 8);
            x[c] += x[d]; x[b] = rl(x[b] ^ x[c], 7);
        };
        for (int r = 0; r < 6; r++) {
            qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15);
            qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14);
        }
        for (int i = 0; i < 16; i++) block[i] = x[i] + s[i];
        counter++;
        pos = 0;
    }
    uint32_t next_u32() {
        if (pos == 16) refill();
        return block[pos++];
    }
    // Uniform u32 in [0, bound): widening multiply, with one extra draw when
    // the low half lands in the biased zone.
    uint32_t below(uint32_t bound) {
        uint64_t m = (uint64_t)next_u32() * bound;
        uint32_t hi = (uint32_t)(m >> 32), lo = (uint32_t)m;
        if (lo > (uint32_t)(0u - bound)) {
            uint32_t hi2 = (uint32_t)(((uint64_t)next_u32() * bound) >> 32);
            if ((uint64_t)lo + hi2 > 0xFFFFFFFFull) hi++;
        }
        return hi;
    }
};
}  // namespace

// SliceRandom::shuffle (rand 0.9): forward Fisher-Yates where the index for
// position i is drawn from [0, i], several indices being decoded from one
// draw in the mixed radix (n+1)(n+2)... that still fits in a u32.
void stdrng_shuffle_identity(uint64_t seed, uint32_t n, uint32_t *perm) {
    for (uint32_t i = 0; i < n; i++) perm[i] = i;
    if (n <= 1) return;
    ChaCha12 rng(seed);
    uint32_t seen = 0, chunk = 0, left = 1;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t radix = seen + 1, rem;
        if (left == 0) {
            uint64_t prod = radix, next = (uint64_t)radix + 1;
            while (prod * next <= 0xFFFFFFFFull) prod *= next++;
            chunk = rng.below((uint32_t)prod);
            rem = (uint32_t)(next - radix) - 1;
        } else {
            rem = left - 1;
        }
        uint32_t pick;
        if (rem == 0) {
            pick = chunk;
        } else {
            pick = chunk % radix;
            chunk /= radix;
        }
        left = rem;
        seen = radix;
        std::swap(perm[i], perm[pick]);
    }
}

}  // namespace zg

// MillerRabin::test to base 2 (primality/src/lib.rs:12-19) of `count`
// candidates of `limbs` u64 each: the vector path for odd candidates above one
// when the CPU has it, the scalar test otherwise.
extern "C" zg_status zg_is_probable_prime_base2(const uint64_t *n, uint32_t limbs, uint32_t count, uint8_t *out) {
    using namespace zg;
    if (!n || !out || limbs < 1 || limbs > MAX_FIELD_LIMBS) {
        set_error("is_probable_prime: null argument or %u limbs (1 to %d)", limbs, MAX_FIELD_LIMBS);
        return ZG_ERR_INVALID_PARAM;
    }
    const int L = (int)limbs;
    const bool vec = mr_ifma_available();
    uint64_t packed[8 * 4];
    uint32_t idx[8];
    int np = 0;
    auto flush = [&]() {
        uint8_t res[8];
        mr_base2_x8(packed, L, np, res);
        for (int e = 0; e < np; e++) out[idx[e]] = res[e];
        np = 0;
    };
    for (uint32_t c = 0; c < count; c++) {
        const uint64_t *x = n + (size_t)c * L;
        bool one = x[0] == 1;
        for (int i = 1; i < L; i++) one = one && x[i] == 0;
        if (!vec || one || !(x[0] & 1)) {
            out[c] = is_probable_prime_base2(x, L) ? 1 : 0;
            continue;
        }
        for (int i = 0; i < L; i++) packed[(size_t)np * L + i] = x[i];
        idx[np++] = c;
        if (np == 8) flush();
    }
    if (np) flush();
    return ZG_OK;
}
