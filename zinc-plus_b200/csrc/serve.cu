// Request server for commit+prove jobs of mixed sizes (continuous batching).
//
// Each request is ZipPlus::commit_single + PcsProverTranscript::
// new_from_commitment + get_random_field_cfg + ZipPlus::prove of one
// polynomial at its point (phase_commit.rs:61-101, pcs_transcript.rs:58-73,
// phase_prove.rs:85-304), and its outputs are byte-identical to zg_commit_prove.
//
// Workers, each with its own lane (stream + scratch), take requests from one
// queue as soon as they are free.  A worker admits the oldest request whose
// device footprint fits the HBM budget, together with queued requests of the
// same parameters (one launch chain commits them all), keeps their codewords
// and Merkle layers on the device, proves each one, and returns the memory.
// Requests that arrive while others are on the GPU join at the next free
// worker, so their work overlaps on the device with the running ones.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <thread>
#include <unordered_map>

#include "zg_internal.h"

namespace zg {
const char *last_error();
}

using namespace zg;
using Clock = std::chrono::steady_clock;

namespace {

struct Request {
    uint64_t id = 0;
    zg_params *p = nullptr;
    const void *poly = nullptr;
    std::vector<uint8_t> point;
    uint8_t *root = nullptr, *eval = nullptr, *proof = nullptr;
    size_t proof_cap = 0, proof_len = 0;
    size_t footprint = 0;
    Clock::time_point t_submit, t_admit, t_done;
    uint32_t group = 0;
    zg_status status = ZG_OK;
    std::string error;
    bool done = false;
};

// Device bytes a request holds while it is in flight: its input, codeword,
// Merkle layers and its share of the kernel scratch (pNTT intermediates, leaf
// chunk chaining values, projected rows).
size_t request_footprint(const zg_params *p) {
    const zg_params_info &I = p->info;
    const size_t input = (size_t)I.num_rows * I.row_len * I.eval_bytes;
    const size_t leaf = (size_t)I.num_rows * I.cw_bytes;
    const size_t cw = (size_t)I.codeword_len * leaf;
    const size_t tree = (2 * (size_t)I.codeword_len - 1) * 32;
    const size_t stage = (size_t)I.num_rows * I.codeword_len * p->D * 12;
    const size_t chunks = leaf > 1024 ? (size_t)I.codeword_len * ((leaf + 1023) / 1024) * 32 : 0;
    const size_t wprime = (size_t)I.num_rows * I.row_len * p->d.comb_limbs * 8;
    return input + cw + tree + stage + chunks + wprime + (1u << 20);
}

// Host threads that test prime candidates for every worker.  Between rounds
// they sleep on a condition variable (threads spinning between parallel
// regions starved the workers' kernel launches), and the worker that posts a
// round tests candidates too, so a round ends as soon as its tests do.
class TestPool {
  public:
    explicit TestPool(int threads) {
        for (int i = 0; i < threads; i++) th_.emplace_back([this] { loop(); });
    }
    ~TestPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    // Runs fn(0..n-1) on the pool and the calling thread; returns when all ran.
    void run_all(int n, const std::function<void(int)> &fn) {
        auto job = std::make_shared<Job>();
        job->n = n;
        job->fn = &fn;
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(job);
        }
        cv_.notify_all();
        for (int i; (i = job->next.fetch_add(1)) < n;) {
            fn(i);
            finish(*job);
        }
        std::unique_lock<std::mutex> lk(job->m);
        job->cv.wait(lk, [&] { return job->done == job->n; });
    }

  private:
    struct Job {
        int n = 0;
        const std::function<void(int)> *fn = nullptr;
        std::atomic<int> next{0};
        int done = 0;
        std::mutex m;
        std::condition_variable cv;
    };
    static void finish(Job &j) {
        std::lock_guard<std::mutex> lk(j.m);
        if (++j.done == j.n) j.cv.notify_all();
    }
    void loop() {
        for (;;) {
            std::shared_ptr<Job> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;  // stopping
                job = q_.front();
                if (job->next.load() >= job->n) {  // every test claimed
                    q_.pop_front();
                    continue;
                }
            }
            const int i = job->next.fetch_add(1);
            if (i >= job->n) continue;
            (*job->fn)(i);
            finish(*job);
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::shared_ptr<Job>> q_;
    bool stop_ = false;
};

}  // namespace

struct zg_server {
    zg_ctx *ctx = nullptr;
    zg_server_opts opts{};
    std::vector<zg_ctx *> lanes;  // owned
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<uint64_t, Request *> reqs;
    uint64_t next_id = 1;
    size_t budget = 0, reserved = 0, peak_reserved = 0;
    cudaMemPool_t pool = nullptr;  // all lanes allocate hint blocks and scratch here
    uint64_t completed = 0, groups = 0, grouped_requests = 0, in_flight = 0;
    double ms_input = 0, ms_commit = 0, ms_prime = 0, ms_prove = 0;  // summed over workers
    bool stop = false;
    std::unique_ptr<TestPool> tests;  // prime candidate tests, shared by the workers
    int prime_group = 1;              // candidates drawn ahead per round
    ~zg_server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        for (auto &t : workers)
            if (t.joinable()) t.join();
        tests.reset();
        for (auto &kv : reqs) delete kv.second;
        for (zg_ctx *l : lanes) zg_ctx_destroy(l);
        if (pool) cudaMemPoolDestroy(pool);
    }
};

namespace {

// Picks the requests of the next group (called with s->mu held).  Returns
// false if nothing can be admitted now.
bool pick_group(zg_server *s, std::vector<Request *> &out) {
    out.clear();
    if (s->queue.empty()) return false;
    const auto now = Clock::now();
    size_t start = s->queue.size();
    for (size_t i = 0; i < s->queue.size(); i++) {
        Request *r = s->queue[i];
        if (s->reserved + r->footprint <= s->budget) {
            start = i;
            break;
        }
        // the oldest request blocks later ones once it has waited too long
        if (i == 0 && std::chrono::duration<double, std::milli>(now - r->t_submit).count() >
                          (double)s->opts.max_skip_ms)
            return false;
    }
    if (start == s->queue.size()) return false;
    Request *head = s->queue[start];
    size_t used = head->footprint;
    out.push_back(head);
    // only small requests share a launch chain: large ones fill the GPU alone,
    // and grouping them would hold m times their memory until the last proof
    const size_t gmax = s->opts.group_max_bytes;
    for (size_t i = start + 1;
         head->footprint <= gmax && i < s->queue.size() && out.size() < s->opts.max_group; i++) {
        Request *r = s->queue[i];
        if (r->p != head->p) continue;
        if (!group_fits(head->p, (uint32_t)out.size() + 1)) break;
        if (s->reserved + used + r->footprint > s->budget) break;
        used += r->footprint;
        out.push_back(r);
    }
    for (Request *r : out) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
    s->reserved += used;
    s->peak_reserved = std::max(s->peak_reserved, s->reserved);
    s->in_flight += out.size();
    return true;
}

// Commit the group in one launch chain, then prove each request.  A request
// is handed back (done, and possibly released by its waiter) as soon as its
// proof is written; fin[k] records which ones were, so that the caller never
// touches those again.
void run_group(zg_server *s, zg_ctx *lane, std::vector<Request *> &g, std::vector<char> &fin) {
    zg_params *p = g.front()->p;
    const uint32_t m = (uint32_t)g.size();
    const size_t pb = (size_t)p->info.num_rows * p->info.row_len * p->info.eval_bytes;
    const auto t_admit = Clock::now();
    for (Request *r : g) {
        r->t_admit = t_admit;
        r->group = m;
    }
    auto fail_all = [&](zg_status st) {
        const std::string msg = last_error();
        for (size_t k = 0; k < g.size(); k++)
            if (!fin[k]) {
                g[k]->status = st;
                g[k]->error = msg;
            }
    };
    auto ms_since = [](Clock::time_point a) {
        return std::chrono::duration<double, std::milli>(Clock::now() - a).count();
    };
    double t_in = 0, t_commit = 0, t_prime = 0, t_prove = 0;
    auto tick = Clock::now();
    zg_status st = lane->evals.ensure(pb * m);
    for (uint32_t k = 0; k < m && st == ZG_OK; k++)
        if (cudaMemcpyAsync(lane->evals.as<uint8_t>() + pb * k, g[k]->poly, pb, cudaMemcpyHostToDevice,
                            lane->stream) != cudaSuccess) {
            set_error("input copy failed: %s", cudaGetErrorString(cudaGetLastError()));
            st = ZG_ERR_CUDA;
        }
    // no wait here: the commit kernels follow the copies on the lane's stream
    t_in = ms_since(tick);
    tick = Clock::now();
    std::vector<zg_hint *> hints(m, nullptr);
    std::vector<uint8_t> roots((size_t)m * 32);
    if (st == ZG_OK) {
        CommitTuning tune;
        st = commit_group_device(p, lane, lane->evals.ptr, m, hints.data(), roots.data(), tune);
    }
    t_commit = ms_since(tick);
    if (st != ZG_OK) {
        fail_all(st);
        return;
    }
    const size_t head = (size_t)p->info.num_rows * 2 * p->info.field_bytes;
    const size_t need = zg_proof_size(p, 1);
    for (uint32_t k = 0; k < m; k++) {
        Request *r = g[k];
        std::memcpy(r->root, roots.data() + 32 * (size_t)k, 32);
        zg_transcript t;
        tr_absorb_slice(&t, r->root, 32);
        uint64_t prime[MAX_FIELD_LIMBS] = {0, 0, 0, 0};
        tick = Clock::now();
        tr_get_prime_batched(&t, (int)p->d.field_limbs, prime, s->prime_group,
                             [s](int n, const std::function<void(int)> &fn) { s->tests->run_all(n, fn); });
        field_cfg_init(t.f, prime, (int)p->d.field_limbs);
        t.has_field = true;
        t_prime += ms_since(tick);
        tick = Clock::now();
        zg_status ps = prove_device(p, lane, &t, lane->evals.as<uint8_t>() + pb * k, 1, r->point.data(),
                                    hints[k], r->eval, r->proof + head);
        t_prove += ms_since(tick);
        if (ps == ZG_OK && t.stream.size() != head) {
            set_error("internal: unexpected proof head size %zu", t.stream.size());
            ps = ZG_ERR_INVALID_PARAM;
        }
        if (ps == ZG_OK) {
            std::memcpy(r->proof, t.stream.data(), head);
            r->proof_len = need;
        } else {
            r->status = ps;
            r->error = last_error();
        }
        zg_hint_free(hints[k]);
        hints[k] = nullptr;
        r->t_done = Clock::now();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->done = true;
            fin[k] = 1;
            s->completed++;
            s->in_flight--;
        }
        s->cv_done.notify_all();
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->ms_input += t_in;
    s->ms_commit += t_commit;
    s->ms_prime += t_prime;
    s->ms_prove += t_prove;
}

void worker_main(zg_server *s, uint32_t wi) {
    zg_ctx *lane = s->lanes[wi];
    cudaSetDevice(lane->device);
    std::vector<Request *> g;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            g.clear();
            s->cv_work.wait(lk, [&] { return s->stop || pick_group(s, g); });
            if (g.empty()) return;  // stopping with nothing admitted
            s->groups++;
            s->grouped_requests += g.size();
        }
        size_t freed = 0;
        for (Request *r : g) freed += r->footprint;
        std::vector<char> fin(g.size(), 0);
        try {
            std::lock_guard<std::mutex> lane_lk(lane->mu);
            run_group(s, lane, g, fin);
        } catch (const std::exception &e) {
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t k = 0; k < g.size(); k++)
                if (!fin[k]) {
                    g[k]->status = ZG_ERR_OOM;
                    g[k]->error = std::string("host failure: ") + e.what();
                }
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->reserved -= freed;
            for (size_t k = 0; k < g.size(); k++)
                if (!fin[k]) {  // failed before its proof was written
                    g[k]->done = true;
                    g[k]->t_done = Clock::now();
                    s->completed++;
                    s->in_flight--;
                }
        }
        // Scratch goes back to the shared pool (stream-ordered, no device sync),
        // so idle lanes hold no memory outside the budget.
        ctx_scratch_release(lane);
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

zg_status zg_server_create(zg_ctx *ctx, const zg_server_opts *opts, zg_server **out) {
    if (!ctx || !out) return ZG_ERR_INVALID_PARAM;
    *out = nullptr;
    try {
        std::unique_ptr<zg_server> s(new zg_server());
        s->ctx = ctx;
        zg_server_opts o{4, 0, 16, 50, 0};
        if (opts) o = *opts;
        if (o.group_max_bytes == 0) o.group_max_bytes = 1ull << 30;
        if (o.workers == 0) o.workers = 4;
        o.workers = std::min<uint32_t>(o.workers, 32);
        if (o.max_group == 0) o.max_group = 16;
        s->opts = o;
        ZG_CUDA(cudaSetDevice(ctx->device));
        size_t free_b = 0, total_b = 0;
        ZG_CUDA(cudaMemGetInfo(&free_b, &total_b));
        s->budget = o.hbm_budget ? (size_t)o.hbm_budget : free_b / 10 * 7;
        // One stream-ordered pool for every lane: freed blocks are reused by any
        // lane without cudaFree/cudaMalloc (which would synchronize the device).
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        ZG_CUDA(cudaMemPoolCreate(&s->pool, &props));
        uint64_t keep = UINT64_MAX;
        ZG_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
        // a block freed by one lane is reused by another only once its free has
        // completed, never by making that lane wait on the other's stream
        int no = 0;
        ZG_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowInternalDependencies, &no));
        // Reserve the budget in the pool once: growing the pool while several
        // lanes allocate serialized them (measured: 4 workers slower than 1).
        {
            void *r = nullptr;
            if (cudaMallocFromPoolAsync(&r, s->budget, s->pool, ctx->stream) == cudaSuccess) {
                cudaFreeAsync(r, ctx->stream);
                cudaStreamSynchronize(ctx->stream);
            }
            cudaGetLastError();
        }
        for (uint32_t i = 0; i < o.workers; i++) {
            zg_ctx *l = nullptr;
            ZG_TRY(zg_ctx_create(ctx->device, &l));
            ctx_use_pool(l, s->pool);
            // several workers wait at once: sleep on events instead of spinning
            ZG_CUDA(cudaEventCreateWithFlags(&l->sync_event,
                                             cudaEventBlockingSync | cudaEventDisableTiming));
            s->lanes.push_back(l);
        }
        // Prime candidates are tested by one pool of sleeping threads shared by
        // the workers (OpenMP teams per worker spin-waited between regions and
        // starved the other workers' launches on a shared host).
        {
            const int hw = (int)std::max(2u, std::thread::hardware_concurrency());
            const int nt = std::max(1, std::min(16, hw / 2));
            s->tests.reset(new TestPool(nt));
            s->prime_group = mr_ifma_available() ? 8 * (nt + 1) : std::max(8, 2 * (nt + 1));
        }
        zg_server *raw = s.get();
        for (uint32_t i = 0; i < o.workers; i++) raw->workers.emplace_back(worker_main, raw, i);
        *out = s.release();
        return ZG_OK;
    } catch (const std::exception &e) {
        set_error("server creation failed: %s", e.what());
        return ZG_ERR_OOM;
    }
}

zg_status zg_server_submit(zg_server *s, zg_params *p, const void *poly, const uint8_t *point,
                           uint8_t *root, uint8_t *eval, uint8_t *proof, size_t proof_cap,
                           uint64_t *id) {
    if (!s || !p || !poly || !point || !root || !eval || !proof || !id) return ZG_ERR_INVALID_PARAM;
    if (!p->ctx || p->ctx->device != s->ctx->device) {
        set_error("parameters belong to another device");
        return ZG_ERR_INVALID_PARAM;
    }
    ZG_TRY(validate_budget(p, 1));
    const size_t need = zg_proof_size(p, 1);
    if (proof_cap < need) {
        set_error("proof buffer too small (%zu bytes needed)", need);
        return ZG_ERR_BUFFER_TOO_SMALL;
    }
    try {
        std::unique_ptr<Request> r(new Request());
        r->p = p;
        r->poly = poly;
        r->point.assign(point, point + 16 * (size_t)p->d.num_vars);
        r->root = root;
        r->eval = eval;
        r->proof = proof;
        r->proof_cap = proof_cap;
        r->footprint = request_footprint(p);
        if (r->footprint > s->budget) {
            set_error("request needs %zu device bytes, above the server budget of %zu", r->footprint,
                      s->budget);
            return ZG_ERR_OOM;
        }
        r->t_submit = Clock::now();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->stop) {
                set_error("server is stopping");
                return ZG_ERR_INVALID_PARAM;
            }
            Request *raw = r.release();
            raw->id = s->next_id++;
            *id = raw->id;
            s->queue.push_back(raw);
            s->reqs[raw->id] = raw;
        }
        s->cv_work.notify_one();
        return ZG_OK;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return ZG_ERR_OOM;
    }
}

zg_status zg_server_wait(zg_server *s, uint64_t id, int timeout_ms, zg_server_result *res) {
    if (!s || !res) return ZG_ERR_INVALID_PARAM;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) {
        set_error("unknown request %llu", (unsigned long long)id);
        return ZG_ERR_INVALID_PARAM;
    }
    Request *r = it->second;
    auto ready = [&] { return r->done; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        set_error("request %llu still running", (unsigned long long)id);
        return ZG_ERR_TIMEOUT;
    }
    res->status = r->status;
    res->proof_len = r->proof_len;
    res->latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    res->queue_ms = std::chrono::duration<double, std::milli>(r->t_admit - r->t_submit).count();
    res->group_size = r->group;
    const zg_status st = r->status;
    if (st != ZG_OK) set_error("%s", r->error.c_str());
    s->reqs.erase(it);
    delete r;
    return st;
}

zg_status zg_server_get_stats(zg_server *s, zg_server_stats *out) {
    if (!s || !out) return ZG_ERR_INVALID_PARAM;
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->completed;
    out->queued = s->queue.size();
    out->in_flight = s->in_flight;
    out->groups = s->groups;
    out->grouped_requests = s->grouped_requests;
    out->budget = s->budget;
    out->reserved = s->reserved;
    out->peak_reserved = s->peak_reserved;
    out->ms_input = s->ms_input;
    out->ms_commit = s->ms_commit;
    out->ms_prime = s->ms_prime;
    out->ms_prove = s->ms_prove;
    return ZG_OK;
}

zg_status zg_server_destroy(zg_server *s) {
    if (!s) return ZG_OK;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // finish everything queued, then stop the workers
        s->cv_done.wait(lk, [&] { return s->queue.empty() && s->in_flight == 0; });
        s->stop = true;
    }
    delete s;  // joins the workers, frees the lanes and the pool
    return ZG_OK;
}

}  // extern "C"
