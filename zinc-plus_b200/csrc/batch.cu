// Batched commit of many independent polynomials of mixed shapes
// (commit_single, zip-plus/src/pcs/phase_commit.rs:61-101, once per
// polynomial, each with its own Merkle tree).
//
// Polynomials that share parameters form a group and go through ONE launch
// chain (segmented encode, the leaves of all their trees, all tree levels).
// Groups are spread over concurrent lanes (streams).  For roots-only calls the
// whole multi-stream launch sequence is captured once per batch shape as a
// CUDA graph and replayed; the kernel variant of every group is chosen by
// timing the candidates the first time a shape is seen.
#include <omp.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>

#include "zg_internal.h"

namespace zg {

zg_status ensure_lanes(zg_ctx *ctx, uint32_t n) {
    while (ctx->lanes.size() < n) {
        zg_ctx *l = nullptr;
        ZG_TRY(zg_ctx_create(ctx->device, &l));
        ctx->lanes.push_back(l);
    }
    return ZG_OK;
}

namespace {

size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t poly_bytes(const zg_params *p) {
    return (size_t)p->info.num_rows * p->info.row_len * p->info.eval_bytes;
}

struct Group {
    zg_params *p = nullptr;
    std::vector<uint32_t> members;  // indices into the caller's arrays
    uint32_t lane = 0;
    CommitTuning tune;
    size_t in_off = 0, cw_off = 0, tree_off = 0, roots_off = 0;
    double cost = 0;  // codeword bytes, for lane balancing
};

// Kernel-variant candidates of one group shape.
std::vector<CommitTuning> candidates(const zg_params *p) {
    std::vector<CommitTuning> out;
    std::vector<int> bases = {-1};
    if (p->d.code_kind == ZG_CODE_IPRS && p->d.eval_kind == ZG_EVAL_BINPOLY && p->info.depth >= 1)
        bases = {6, 7, 8, 0, 4, 5, 1, 2};
    std::vector<int> leaves = {-1};
    const size_t lb = (size_t)p->info.num_rows * p->info.cw_bytes;
    if (lb % 16 == 0) leaves = {0, 1};
    for (int b : bases)
        for (int l : leaves) {
            CommitTuning t;
            t.base_variant = b;
            t.leaf_variant = l;
            out.push_back(t);
        }
    return out;
}

std::string tune_key(const zg_params *p, uint32_t m) {
    char buf[160];
    snprintf(buf, sizeof buf, "%u/%u/%u/%u/%u/%u/%u", p->d.eval_kind, p->D, p->d.code_kind,
             p->info.row_len, p->info.num_rows, p->info.depth, m);
    return buf;
}

}  // namespace

// A batch shape: its groups, device arena, pinned staging and captured graph.
struct BatchPlan {
    std::string key;
    bool on_device = false;
    bool pinned = false;  // host inputs in page-locked memory: copied by DMA, no staging
    uint32_t n = 0, nlanes = 0;
    std::vector<Group> groups;
    std::vector<const void *> dev_inputs;  // for device inputs: the pointers baked into the graph
    DevBuf arena;
    HostBuf pin_in, pin_roots;
    size_t in_bytes = 0, roots_base = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches_per_run = 0;
    std::vector<cudaEvent_t> events;
    // Lanes owned by the plan: a captured graph holds their scratch addresses,
    // so no other call may grow (reallocate) them.
    std::vector<zg_ctx *> lanes;
    ~BatchPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        for (zg_ctx *l : lanes) zg_ctx_destroy(l);
        arena.release();
        pin_in.release();
        pin_roots.release();
    }
    uint64_t launches() const {
        uint64_t n = 0;
        for (const zg_ctx *l : lanes) n += l->launches;
        return n;
    }
};

void drop_plans_of(zg_ctx *ctx, const zg_params *p) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto &plans = ctx->plans;
    plans.erase(std::remove_if(plans.begin(), plans.end(),
                               [&](const std::pair<std::string, std::shared_ptr<BatchPlan>> &kv) {
                                   for (const Group &g : kv.second->groups)
                                       if (g.p == p) return true;
                                   return false;
                               }),
                plans.end());
}

namespace {

// Issues every group of the plan on its lane, forked from and joined back to
// the context stream.  inputs[i]: device address of polynomial i when the
// group reads it in place (single-member groups of device inputs), else NULL.
zg_status issue_plan(zg_ctx *ctx, BatchPlan &pl, const void *const *dev_polys) {
    uint8_t *arena = pl.arena.as<uint8_t>();
    ZG_CUDA(cudaEventRecord(pl.events[0], ctx->stream));
    for (uint32_t l = 0; l < pl.nlanes; l++) ZG_CUDA(cudaStreamWaitEvent(pl.lanes[l]->stream, pl.events[0], 0));
    for (Group &g : pl.groups) {
        zg_ctx *lane = pl.lanes[g.lane];
        cudaStream_t s = lane->stream;
        const size_t pb = poly_bytes(g.p);
        const uint32_t m = (uint32_t)g.members.size();
        const void *in = nullptr;
        if (pl.pinned) {
            for (uint32_t k = 0; k < m; k++)
                ZG_CUDA(cudaMemcpyAsync(arena + g.in_off + pb * k, dev_polys[g.members[k]], pb,
                                        cudaMemcpyHostToDevice, s));
            in = arena + g.in_off;
        } else if (!pl.on_device) {
            ZG_CUDA(cudaMemcpyAsync(arena + g.in_off, pl.pin_in.as<uint8_t>() + g.in_off, pb * m,
                                    cudaMemcpyHostToDevice, s));
            in = arena + g.in_off;
        } else if (m == 1) {
            in = dev_polys[g.members[0]];
        } else {
            for (uint32_t k = 0; k < m; k++)
                ZG_CUDA(cudaMemcpyAsync(arena + g.in_off + pb * k, dev_polys[g.members[k]], pb,
                                        cudaMemcpyDeviceToDevice, s));
            in = arena + g.in_off;
        }
        ZG_TRY(launch_commit_group(g.p, lane, in, m, arena + g.cw_off, arena + g.tree_off, s, g.tune));
        const size_t C = g.p->info.codeword_len;
        ZG_CUDA(cudaMemcpy2DAsync(arena + g.roots_off, 32, arena + g.tree_off + (2 * C - 2) * 32,
                                  group_tree_stride(g.p), 32, m, cudaMemcpyDeviceToDevice, s));
    }
    for (uint32_t l = 0; l < pl.nlanes; l++) {
        ZG_CUDA(cudaEventRecord(pl.events[1 + l], pl.lanes[l]->stream));
        ZG_CUDA(cudaStreamWaitEvent(ctx->stream, pl.events[1 + l], 0));
    }
    ZG_CUDA(cudaMemcpyAsync(pl.pin_roots.ptr, arena + pl.roots_base, (size_t)pl.n * 32,
                            cudaMemcpyDeviceToHost, ctx->stream));
    return ZG_OK;
}

// Times each candidate variant of group g (on its lane, inputs already staged).
zg_status autotune_group(zg_ctx *ctx, BatchPlan &pl, Group &g, const void *in) {
    const std::string key = tune_key(g.p, (uint32_t)g.members.size());
    auto it = ctx->tune_cache.find(key);
    if (it != ctx->tune_cache.end()) {
        g.tune.base_variant = it->second.first;
        g.tune.leaf_variant = it->second.second;
        return ZG_OK;
    }
    zg_ctx *lane = pl.lanes[g.lane];
    cudaStream_t s = lane->stream;
    uint8_t *arena = pl.arena.as<uint8_t>();
    cudaEvent_t e0 = pl.events[0], e1 = pl.events[1];
    float best = 1e30f;
    CommitTuning best_t;
    for (const CommitTuning &t : candidates(g.p)) {
        float tmin = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            ZG_CUDA(cudaEventRecord(e0, s));
            ZG_TRY(launch_commit_group(g.p, lane, in, (uint32_t)g.members.size(), arena + g.cw_off,
                                       arena + g.tree_off, s, t));
            ZG_CUDA(cudaEventRecord(e1, s));
            ZG_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            ZG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) tmin = std::min(tmin, ms);  // the first run is a warm-up
        }
        if (tmin < best) {
            best = tmin;
            best_t = t;
        }
    }
    g.tune = best_t;
    ctx->tune_cache[key] = {best_t.base_variant, best_t.leaf_variant};
    return ZG_OK;
}

zg_status build_plan(zg_ctx *ctx, uint32_t n, zg_params *const *params, int on_device,
                     bool pinned, uint32_t nlanes, BatchPlan &pl) {
    pl.n = n;
    pl.on_device = on_device != 0;
    pl.pinned = pinned;
    // groups: equal parameter handles, split where one launch chain cannot hold them
    std::vector<uint32_t> order(n);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return params[a] < params[b]; });
    for (uint32_t i = 0; i < n;) {
        uint32_t j = i;
        while (j < n && params[order[j]] == params[order[i]]) j++;
        zg_params *p = params[order[i]];
        uint32_t k = i;
        while (k < j) {
            uint32_t m = j - k;
            while (m > 1 && !group_fits(p, m)) m = group_fits(p, 2) ? std::min(m - 1, m / 2 + 1) : 1;
            Group g;
            g.p = p;
            for (uint32_t q = k; q < k + m; q++) g.members.push_back(order[q]);
            g.cost = (double)group_cw_stride(p) * m;
            pl.groups.push_back(std::move(g));
            k += m;
        }
        i = j;
    }
    // largest groups first, each to the least-loaded lane
    std::sort(pl.groups.begin(), pl.groups.end(),
              [](const Group &a, const Group &b) { return a.cost > b.cost; });
    pl.nlanes = std::max<uint32_t>(1, std::min<uint32_t>(nlanes, (uint32_t)pl.groups.size()));
    while (pl.lanes.size() < pl.nlanes) {
        zg_ctx *l = nullptr;
        ZG_TRY(zg_ctx_create(ctx->device, &l));
        pl.lanes.push_back(l);
    }
    std::vector<double> load(pl.nlanes, 0.0);
    for (Group &g : pl.groups) {
        const uint32_t l = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
        g.lane = l;
        load[l] += g.cost;
    }
    // arena layout
    size_t off = 0;
    for (Group &g : pl.groups) {
        const uint32_t m = (uint32_t)g.members.size();
        if (!pl.on_device || m > 1) {
            g.in_off = off;
            off = round256(off + poly_bytes(g.p) * m);
        }
    }
    pl.in_bytes = off;
    for (Group &g : pl.groups) {
        g.cw_off = off;
        off = round256(off + group_cw_stride(g.p) * g.members.size());
        g.tree_off = off;
        off = round256(off + group_tree_stride(g.p) * g.members.size());
    }
    pl.roots_base = off;
    for (Group &g : pl.groups) {
        g.roots_off = off;
        off += 32 * g.members.size();
    }
    ZG_TRY(pl.arena.ensure(round256(off)));
    if (!pl.on_device && !pl.pinned) ZG_TRY(pl.pin_in.ensure(std::max<size_t>(pl.in_bytes, 256)));
    ZG_TRY(pl.pin_roots.ensure((size_t)n * 32));
    pl.events.resize(1 + std::max<uint32_t>(pl.nlanes, 1));
    for (cudaEvent_t &e : pl.events) ZG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDefault));
    return ZG_OK;
}

// Keyed by the parameter sets' unique ids: their addresses can be reused by a
// later set of another shape once freed.
std::string plan_key(uint32_t n, zg_params *const *params, int on_device, bool pinned,
                     uint32_t nlanes) {
    std::string k = std::to_string(n) + ":" + std::to_string(on_device) + ":" +
                    std::to_string((int)pinned) + ":" + std::to_string(nlanes);
    for (uint32_t i = 0; i < n; i++) k += ":" + std::to_string(params[i]->uid);
    return k;
}

// Copies the host inputs of every multi-row group into the pinned staging area.
void stage_host_inputs(BatchPlan &pl, const void *const *polys) {
    std::vector<std::pair<uint8_t *, const void *>> jobs;
    std::vector<size_t> sizes;
    for (Group &g : pl.groups) {
        const size_t pb = poly_bytes(g.p);
        for (size_t k = 0; k < g.members.size(); k++) {
            jobs.push_back({pl.pin_in.as<uint8_t>() + g.in_off + pb * k, polys[g.members[k]]});
            sizes.push_back(pb);
        }
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (long i = 0; i < (long)jobs.size(); i++) std::memcpy(jobs[i].first, jobs[i].second, sizes[i]);
}

}  // namespace

// Direct path (hints requested): every group gets its own shared device
// block, launched on its lane without a graph; roots come back in one pass.
zg_status commit_batch_hints(zg_ctx *ctx, uint32_t n, zg_params *const *params,
                             const void *const *polys, int on_device, uint32_t nlanes,
                             const CommitTuning *force, uint8_t *roots, zg_hint **hints) {
    BatchPlan pl;  // groups and lanes only; no arena
    pl.n = n;
    pl.on_device = on_device != 0;
    {
        std::vector<uint32_t> order(n);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t a, uint32_t b) { return params[a] < params[b]; });
        for (uint32_t i = 0; i < n;) {
            uint32_t j = i;
            while (j < n && params[order[j]] == params[order[i]]) j++;
            zg_params *p = params[order[i]];
            for (uint32_t k = i; k < j;) {
                uint32_t m = j - k;
                while (m > 1 && !group_fits(p, m)) m--;
                Group g;
                g.p = p;
                for (uint32_t q = k; q < k + m; q++) g.members.push_back(order[q]);
                g.cost = (double)group_cw_stride(p) * m;
                pl.groups.push_back(std::move(g));
                k += m;
            }
            i = j;
        }
    }
    std::sort(pl.groups.begin(), pl.groups.end(),
              [](const Group &a, const Group &b) { return a.cost > b.cost; });
    pl.nlanes = std::max<uint32_t>(1, std::min<uint32_t>(nlanes, (uint32_t)pl.groups.size()));
    ZG_TRY(ensure_lanes(ctx, pl.nlanes));
    std::vector<double> load(pl.nlanes, 0.0);
    for (Group &g : pl.groups) {
        const uint32_t l = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
        g.lane = l;
        load[l] += g.cost;
    }
    ZG_TRY(ctx->pin_out.ensure((size_t)n * 32));
    uint8_t *hr = ctx->pin_out.as<uint8_t>();
    std::vector<std::shared_ptr<SharedBlock>> blocks(pl.groups.size());
    std::vector<DevBuf> inputs(pl.groups.size());
    size_t slot = 0;
    zg_status st = ZG_OK;
    for (size_t gi = 0; gi < pl.groups.size() && st == ZG_OK; gi++) {
        Group &g = pl.groups[gi];
        zg_ctx *lane = ctx->lanes[g.lane];
        cudaStream_t s = lane->stream;
        const uint32_t m = (uint32_t)g.members.size();
        const size_t pb = poly_bytes(g.p);
        const void *in = on_device && m == 1 ? polys[g.members[0]] : nullptr;
        if (!in) {
            if ((st = inputs[gi].ensure(pb * m)) != ZG_OK) break;
            for (uint32_t k = 0; k < m && st == ZG_OK; k++)
                if (cudaMemcpyAsync(inputs[gi].as<uint8_t>() + pb * k, polys[g.members[k]], pb,
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    s) != cudaSuccess)
                    st = ZG_ERR_CUDA;
            in = inputs[gi].ptr;
        }
        if (st != ZG_OK) break;
        auto blk = std::make_shared<SharedBlock>();
        blk->lane = lane;
        const size_t cwb = round256(group_cw_stride(g.p) * m);
        blk->ptr = ctx_alloc(lane, cwb + group_tree_stride(g.p) * m, &blk->bytes);
        if (!blk->ptr) {
            st = ZG_ERR_OOM;
            break;
        }
        blocks[gi] = blk;
        uint8_t *cw = static_cast<uint8_t *>(blk->ptr), *tree = cw + cwb;
        CommitTuning t = force ? *force : g.tune;
        auto it = ctx->tune_cache.find(tune_key(g.p, m));
        if (!force && it != ctx->tune_cache.end()) {
            t.base_variant = it->second.first;
            t.leaf_variant = it->second.second;
        }
        if ((st = launch_commit_group(g.p, lane, in, m, cw, tree, s, t)) != ZG_OK) break;
        const size_t C = g.p->info.codeword_len;
        g.roots_off = slot;
        if (cudaMemcpy2DAsync(hr + slot, 32, tree + (2 * C - 2) * 32, group_tree_stride(g.p), 32, m,
                              cudaMemcpyDeviceToHost, s) != cudaSuccess)
            st = ZG_ERR_CUDA;
        slot += 32 * (size_t)m;
    }
    for (uint32_t l = 0; l < pl.nlanes; l++)
        if (cudaStreamSynchronize(ctx->lanes[l]->stream) != cudaSuccess && st == ZG_OK) st = ZG_ERR_CUDA;
    for (DevBuf &b : inputs) b.release();
    if (st != ZG_OK) {
        if (st == ZG_ERR_CUDA) set_error("batched commit failed: %s", cudaGetErrorString(cudaGetLastError()));
        return st;
    }
    for (size_t gi = 0; gi < pl.groups.size(); gi++) {
        Group &g = pl.groups[gi];
        const uint32_t C = g.p->info.codeword_len;
        uint8_t *cw = static_cast<uint8_t *>(blocks[gi]->ptr);
        uint8_t *tree = cw + round256(group_cw_stride(g.p) * g.members.size());
        for (size_t k = 0; k < g.members.size(); k++) {
            const uint32_t idx = g.members[k];
            const uint8_t *r = hr + g.roots_off + 32 * k;
            if (roots) std::memcpy(roots + 32 * (size_t)idx, r, 32);
            zg_hint *h = new zg_hint();
            h->shared = blocks[gi];
            h->params = g.p;
            h->lane = ctx->lanes[g.lane];
            h->batch = 1;
            h->nrows = g.p->info.num_rows;
            h->depth = 31 - __builtin_clz(C);
            h->d_cw = cw + group_cw_stride(g.p) * k;
            h->d_tree = tree + group_tree_stride(g.p) * k;
            std::memcpy(h->root, r, 32);
            hints[idx] = h;
        }
    }
    return ZG_OK;
}

zg_status commit_batch_impl(zg_ctx *ctx, uint32_t n, zg_params *const *params,
                            const void *const *polys, int on_device, const zg_batch_opts *opts,
                            uint8_t *roots, zg_hint **hints) {
    if (!ctx || !params || !polys || n == 0 || (!roots && !hints)) {
        set_error("batched commit: null argument or empty batch");
        return ZG_ERR_INVALID_PARAM;
    }
    for (uint32_t i = 0; i < n; i++) {
        if (!params[i] || !polys[i]) {
            set_error("batched commit: polynomial %u has no parameters or data", i);
            return ZG_ERR_INVALID_PARAM;
        }
        if (params[i]->ctx != ctx) {
            set_error("batched commit: parameters %u were created on another context", i);
            return ZG_ERR_INVALID_PARAM;
        }
        ZG_TRY(validate_budget(params[i], 1));
    }
    zg_batch_opts o{4, 1, 1, -1, -1};
    if (opts) o = *opts;
    const uint32_t nlanes = std::max<uint32_t>(1, std::min<uint32_t>(o.lanes ? o.lanes : 4, 16));
    const bool forced = o.base_variant >= 0 || o.leaf_variant >= 0;
    CommitTuning force;
    force.base_variant = o.base_variant;
    force.leaf_variant = o.leaf_variant;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    if (hints) {
        for (uint32_t i = 0; i < n; i++) hints[i] = nullptr;
        return commit_batch_hints(ctx, n, params, polys, on_device, nlanes, forced ? &force : nullptr,
                                  roots, hints);
    }
    // roots only: a cached plan, replayed as one graph
    // host inputs that are all page-locked are copied by DMA straight from the
    // caller's buffers (their addresses are baked into the graph, like device inputs)
    bool pinned = false;
    if (!on_device) {
        pinned = true;
        for (uint32_t i = 0; i < n && pinned; i++) {
            cudaPointerAttributes at{};
            if (cudaPointerGetAttributes(&at, polys[i]) != cudaSuccess || at.type != cudaMemoryTypeHost)
                pinned = false;
            cudaGetLastError();
        }
    }
    const std::string key = plan_key(n, params, on_device, pinned, nlanes) +
                            (forced ? ":f" + std::to_string(o.base_variant) + "," + std::to_string(o.leaf_variant) : "");
    std::shared_ptr<BatchPlan> pl;
    for (auto &kv : ctx->plans)
        if (kv.first == key) pl = kv.second;
    bool fresh = false;
    if (!pl) {
        pl = std::make_shared<BatchPlan>();
        pl->key = key;
        ZG_TRY(build_plan(ctx, n, params, on_device, pinned, nlanes, *pl));
        fresh = true;
    }
    if (!on_device && !pinned) stage_host_inputs(*pl, polys);
    std::vector<const void *> dev(polys, polys + n);
    if ((on_device || pinned) && pl->dev_inputs != dev) {  // baked pointers changed: capture again
        if (pl->exec) cudaGraphExecDestroy(pl->exec);
        if (pl->graph) cudaGraphDestroy(pl->graph);
        pl->exec = nullptr;
        pl->graph = nullptr;
        pl->dev_inputs = dev;
    }
    // A new plan is cached only once its tuning and its sizing run succeeded:
    // a plan cached after a failure would later be captured without the run that
    // sizes its lanes' scratch.  On a failure the lanes' queued work is drained
    // before the plan (its arena and lanes) is dropped.
    auto setup = [&]() -> zg_status {
        // tuning: forced choice, or time the candidates of each group shape
        for (Group &g : pl->groups) {
            if (forced) {
                g.tune = force;
                continue;
            }
            if (!o.autotune) continue;
            zg_ctx *lane = pl->lanes[g.lane];
            const uint32_t m = (uint32_t)g.members.size();
            const size_t pb = poly_bytes(g.p);
            uint8_t *arena = pl->arena.as<uint8_t>();
            const void *in = nullptr;
            if (pinned) {
                for (uint32_t k = 0; k < m; k++)
                    ZG_CUDA(cudaMemcpyAsync(arena + g.in_off + pb * k, polys[g.members[k]], pb,
                                            cudaMemcpyHostToDevice, lane->stream));
                in = arena + g.in_off;
            } else if (!on_device) {
                ZG_CUDA(cudaMemcpyAsync(arena + g.in_off, pl->pin_in.as<uint8_t>() + g.in_off, pb * m,
                                        cudaMemcpyHostToDevice, lane->stream));
                in = arena + g.in_off;
            } else if (m == 1) {
                in = polys[g.members[0]];
            } else {
                for (uint32_t k = 0; k < m; k++)
                    ZG_CUDA(cudaMemcpyAsync(arena + g.in_off + pb * k, polys[g.members[k]], pb,
                                            cudaMemcpyDeviceToDevice, lane->stream));
                in = arena + g.in_off;
            }
            ZG_TRY(autotune_group(ctx, *pl, g, in));
        }
        // one plain run sizes every lane's scratch before capture
        ZG_TRY(issue_plan(ctx, *pl, polys));
        ZG_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->launch_adjust += (int64_t)pl->launches();
        return ZG_OK;
    };
    if (fresh) {
        const zg_status st = setup();
        if (st != ZG_OK) {
            for (zg_ctx *l : pl->lanes) cudaStreamSynchronize(l->stream);
            cudaStreamSynchronize(ctx->stream);
            return st;
        }
        if (ctx->plans.size() >= 8) ctx->plans.erase(ctx->plans.begin());
        ctx->plans.push_back({key, pl});
    }
    if (o.use_graph && !pl->exec) {
        const uint64_t before = pl->launches();
        zg_status st = ZG_OK;
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            st = ZG_ERR_CUDA;
        } else {
            st = issue_plan(ctx, *pl, polys);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (st == ZG_OK && e != cudaSuccess) st = ZG_ERR_CUDA;
            if (st == ZG_OK && cudaGraphInstantiate(&pl->exec, g, 0) != cudaSuccess) st = ZG_ERR_CUDA;
            pl->graph = g;
        }
        pl->launches_per_run = pl->launches() - before;  // captured launches, counted per replay
        if (st != ZG_OK) {
            set_error("batched commit: graph capture failed: %s", cudaGetErrorString(cudaGetLastError()));
            return st;
        }
    }
    if (o.use_graph) {
        ZG_CUDA(cudaGraphLaunch(pl->exec, ctx->stream));
        ctx->launch_adjust += (int64_t)pl->launches_per_run;
    } else if (!fresh) {
        const uint64_t before = pl->launches();
        ZG_TRY(issue_plan(ctx, *pl, polys));
        ctx->launch_adjust += (int64_t)(pl->launches() - before);
    }
    ZG_CUDA(cudaStreamSynchronize(ctx->stream));
    const uint8_t *hr = pl->pin_roots.as<uint8_t>();
    for (const Group &g : pl->groups)
        for (size_t k = 0; k < g.members.size(); k++)
            std::memcpy(roots + 32 * (size_t)g.members[k], hr + (g.roots_off - pl->roots_base) + 32 * k, 32);
    return ZG_OK;
}

}  // namespace zg

extern "C" zg_status zg_commit_batch(zg_ctx *ctx, uint32_t n, zg_params *const *params,
                                     const void *const *polys, int polys_on_device,
                                     const zg_batch_opts *opts, uint8_t *roots, zg_hint **hints) {
    try {
        return zg::commit_batch_impl(ctx, n, params, polys, polys_on_device, opts, roots, hints);
    } catch (const std::bad_alloc &) {
        zg::set_error("host allocation failed");
        return ZG_ERR_OOM;
    }
}
