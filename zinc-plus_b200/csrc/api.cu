// Commit / prove / verify pipelines and the extern "C" ABI of include/zipgpu.h.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <thread>

#include "zg_internal.h"
#include "zg_prove.h"
#include "zg_umma.cuh"

namespace zg {
const char *last_error();
}

using namespace zg;

#define ZG_GUARD(expr)                                                                            \
    try {                                                                                         \
        return (expr);                                                                            \
    } catch (const std::bad_alloc &) {                                                            \
        set_error("host allocation failed");                                                      \
        return ZG_ERR_OOM;                                                                        \
    } catch (...) {                                                                               \
        set_error("unexpected C++ exception");                                                    \
        return ZG_ERR_INVALID_PARAM;                                                              \
    }

namespace {

bool is_pow2(uint64_t x) { return x && !(x & (x - 1)); }
uint32_t ilog2u(uint64_t x) { return 63 - __builtin_clzll(x); }
uint32_t ilog_round_up(uint64_t x) { return is_pow2(x) ? ilog2u(x) : ilog2u(x) + 1; }

}  // namespace

// validate_input's bit budget for linear combinations (pcs/utils.rs:24-54).
zg_status zg::validate_budget(const zg_params *p, uint32_t batch) {
    if (batch == 0) {
        set_error("Batch must contain at least one polynomial");
        return ZG_ERR_INVALID_PARAM;
    }
    const uint32_t d = ilog2u(p->info.row_len);
    const uint32_t codeword_bits = ilog_round_up(std::max<uint64_t>((uint64_t)p->d.rep * d, 1));
    const uint32_t challenge_bits = p->D > 1 ? 256 : 128;  // Chal = i128; doubled with alphas
    const uint32_t eval_bits = p->d.eval_kind == ZG_EVAL_BINPOLY ? 1 : p->d.eval_kind == ZG_EVAL_I64 ? 64 : 32;
    const uint32_t actual = 2 * codeword_bits + ilog_round_up(std::max<uint32_t>(d, 1)) +
                            challenge_bits + (eval_bits - 1) + ilog_round_up(batch);
    if (actual > 64 * p->d.comb_limbs) {
        set_error("The number of bits used for linear combinations is too large: %u bits, max "
                  "allowed is %u bits",
                  actual, 64 * p->d.comb_limbs);
        return ZG_ERR_OVERFLOW;
    }
    return ZG_OK;
}

namespace {

uint64_t dmask_of(uint32_t D) { return D >= 64 ? ~0ull : ((1ull << D) - 1); }

// Per-row offsets of the tcgen05 base layer: off[r] moves row r of the base
// matrix into [-2^15, 2^15), where a u8 low byte and an s8 high byte hold it
// exactly; the kernel subtracts off[r] x (number of set input bits).  False
// when some row spans more than 2^16 values.
bool build_umma_offsets(const std::vector<int64_t> &bm, uint32_t bd, uint32_t bl, std::vector<int32_t> &off) {
    off.assign(bd, 0);
    for (uint32_t r = 0; r < bd; r++) {
        int64_t lo = INT64_MAX, hi = INT64_MIN;
        for (uint32_t c = 0; c < bl; c++) {
            lo = std::min(lo, bm[(size_t)r * bl + c]);
            hi = std::max(hi, bm[(size_t)r * bl + c]);
        }
        if (bl == 0) continue;
        if (hi - lo > 65535) return false;
        const int64_t o = lo < -32768 ? -32768 - lo : hi > 32767 ? 32767 - hi : 0;
        off[r] = (int32_t)o;
    }
    return true;
}

i128 load_i128(const uint8_t *b) {
    u128 v = 0;
    for (int i = 15; i >= 0; i--) v = (v << 8) | b[i];
    return (i128)v;
}

template <int L>
void host_eq_table(const FieldCfg &f, const uint64_t *r, uint32_t n, std::vector<uint64_t> &out) {
    // eq(x, r)[i] = prod_k (bit_k(i) ? r_k : 1 - r_k)   (poly/src/utils.rs:24-101)
    out.assign((size_t)L << n, 0);
    for (int w = 0; w < L; w++) out[w] = f.one[w];
    size_t len = 1;
    for (int k = (int)n - 1; k >= 0; k--) {
        for (long i = (long)len - 1; i >= 0; i--) {
            uint64_t b[L], t[L];
            for (int w = 0; w < L; w++) b[w] = out[(size_t)i * L + w];
            fmul<L>(r + (size_t)k * L, b, f.p, f.n0, t);
            for (int w = 0; w < L; w++) out[(size_t)(2 * i + 1) * L + w] = t[w];
            fsub<L>(b, t, f.p);
            for (int w = 0; w < L; w++) out[(size_t)(2 * i) * L + w] = b[w];
        }
        len *= 2;
    }
}

void host_eq(const FieldCfg &f, const uint64_t *r, uint32_t n, std::vector<uint64_t> &out) {
    if (f.L == 3) host_eq_table<3>(f, r, n, out);
    else host_eq_table<4>(f, r, n, out);
}

void f_from_i128(const FieldCfg &f, i128 v, uint64_t *out) {
    if (f.L == 3) from_i128<3>(v, f, out);
    else from_i128<4>(v, f, out);
}
void f_from_signed(const FieldCfg &f, const uint64_t *x, int limbs, uint64_t *out) {
    if (f.L == 3) from_signed<3>(x, limbs, f, out);
    else from_signed<4>(x, limbs, f, out);
}
void f_mul(const FieldCfg &f, const uint64_t *a, const uint64_t *b, uint64_t *out) {
    if (f.L == 3) fmul<3>(a, b, f.p, f.n0, out);
    else fmul<4>(a, b, f.p, f.n0, out);
}
void f_add(const FieldCfg &f, uint64_t *a, const uint64_t *b) {
    if (f.L == 3) fadd<3>(a, b, f.p);
    else fadd<4>(a, b, f.p);
}
void f_sub(const FieldCfg &f, uint64_t *a, const uint64_t *b) {
    if (f.L == 3) fsub<3>(a, b, f.p);
    else fsub<4>(a, b, f.p);
}

size_t leaf_bytes_of(const zg_params *p, uint32_t batch) {
    return (size_t)batch * p->info.num_rows * p->info.cw_bytes;
}

// Host encode_wide on Int<limbs> (wrapping), the verifier's re-encoding of the
// combined row (iprs.rs:148-150 -> radix8.rs:21-161; raa.rs encode_wide).
void host_encode_wide(const zg_params *p, const uint64_t *row, uint32_t limbs, uint64_t *out) {
    const zg_params_info &I = p->info;
    const uint32_t C = I.codeword_len;
    if (p->d.code_kind != ZG_CODE_IPRS) {
        // RAA (raa.rs:93-127); with sign flips (raa_sign_flip.rs:31-69) the
        // repeated row's and the first accumulation's odd entries are negated,
        // i.e. a gathered entry is negated when its source index is odd
        const bool flip = p->d.code_kind == ZG_CODE_RAA_SIGN_FLIP;
        auto negate = [limbs](uint64_t *x) {
            unsigned __int128 c = 1;
            for (uint32_t w = 0; w < limbs; w++) {
                const unsigned __int128 t = (unsigned __int128)(~x[w]) + c;
                x[w] = (uint64_t)t;
                c = t >> 64;
            }
        };
        const uint32_t Lr = I.row_len;
        std::vector<uint64_t> a((size_t)C * limbs), b((size_t)C * limbs);
        for (uint32_t i = 0; i < C; i++) {
            std::memcpy(&a[(size_t)i * limbs], row + (size_t)(p->perm1[i] % Lr) * limbs, 8 * limbs);
            if (flip && (p->perm1[i] & 1u)) negate(&a[(size_t)i * limbs]);
        }
        for (uint32_t i = 1; i < C; i++) wide_add(&a[(size_t)i * limbs], &a[(size_t)(i - 1) * limbs], limbs);
        for (uint32_t i = 0; i < C; i++) {
            std::memcpy(&b[(size_t)i * limbs], &a[(size_t)p->perm2[i] * limbs], 8 * limbs);
            if (flip && (p->perm2[i] & 1u)) negate(&b[(size_t)i * limbs]);
        }
        for (uint32_t i = 1; i < C; i++) wide_add(&b[(size_t)i * limbs], &b[(size_t)(i - 1) * limbs], limbs);
        std::memcpy(out, b.data(), 8 * (size_t)C * limbs);
        return;
    }
    const uint32_t bd = I.base_dim, bl = I.base_len, depth = I.depth;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)C; i++) {
        uint32_t ch = (uint32_t)i / bd, rb = (uint32_t)i % bd, oct = 0, x = ch;
        for (uint32_t k = 0; k < depth; k++) {
            oct = (oct << 3) | (x & 7);
            x >>= 3;
        }
        uint64_t *o = out + (size_t)i * limbs;
        std::memset(o, 0, 8 * limbs);
        for (uint32_t c = 0; c < bl; c++)
            wide_mul_i128_add(o, row + ((size_t)oct + ((size_t)c << (3 * depth))) * limbs,
                              (i128)p->bm[(size_t)rb * bl + c], (int)limbs);
    }
    std::vector<uint64_t> xs((size_t)8 * limbs);
    for (uint32_t k = 0; k < depth; k++) {
        const size_t sub = (size_t)bd << (3 * k);
        const int64_t *tw = p->tw.data() + p->tw_off[k];
        for (size_t blk = 0; blk < C; blk += 8 * sub) {
            uint64_t *chunk = out + blk * limbs;
            for (size_t i = 0; i < sub; i++) {
                for (int j = 0; j < 8; j++)
                    std::memcpy(&xs[(size_t)j * limbs], chunk + (j * sub + i) * limbs, 8 * limbs);
                for (int r = 0; r < 8; r++) {
                    uint64_t *y = chunk + (r * sub + i) * limbs;
                    std::memcpy(y, xs.data(), 8 * limbs);
                    for (int j = 1; j < 8; j++)
                        wide_mul_i128_add(y, &xs[(size_t)j * limbs],
                                          (i128)tw[(i * 7 + (j - 1)) * 8 + ((r * j) & 7)], (int)limbs);
                }
            }
        }
    }
}

// get_path_directions + MerkleProof::verify (merkle.rs:282-410).
// encode_wide at selected codeword positions (the verifier checks only the
// opened columns).  IPRS: position P = ch * bd + rb depends on the 8^depth base
// outputs at base position rb and on the radix-8 stages over the chunk index;
// RAA: the whole (cheap) codeword.  out: n x limbs.
void host_encode_wide_at(const zg_params *p, const uint64_t *row, uint32_t limbs,
                         const uint32_t *pos, uint32_t n, uint64_t *out) {
    const zg_params_info &I = p->info;
    if (p->d.code_kind != ZG_CODE_IPRS) {
        std::vector<uint64_t> all((size_t)I.codeword_len * limbs);
        host_encode_wide(p, row, limbs, all.data());
        for (uint32_t o = 0; o < n; o++) std::memcpy(out + (size_t)o * limbs, &all[(size_t)pos[o] * limbs], 8 * limbs);
        return;
    }
    const uint32_t bd = I.base_dim, bl = I.base_len, depth = I.depth, nch = 1u << (3 * depth);
#pragma omp parallel for schedule(dynamic, 1)
    for (long o = 0; o < (long)n; o++) {
        const uint32_t P = pos[o], rb = P % bd;
        std::vector<uint64_t> cur((size_t)nch * limbs, 0), nxt((size_t)nch * limbs);
        for (uint32_t ch = 0; ch < nch; ch++) {
            uint32_t oct = 0, x = ch;
            for (uint32_t k = 0; k < depth; k++) {
                oct = (oct << 3) | (x & 7);
                x >>= 3;
            }
            for (uint32_t c = 0; c < bl; c++)
                wide_mul_s64_add(&cur[(size_t)ch * limbs], row + ((size_t)oct + ((size_t)c << (3 * depth))) * limbs,
                                 p->bm[(size_t)rb * bl + c], (int)limbs);
        }
        for (uint32_t k = 0; k < depth; k++) {
            const uint32_t stride = 1u << (3 * k);
            const int64_t *tw = p->tw.data() + p->tw_off[k];
            for (uint32_t ch = 0; ch < nch; ch++) {
                const uint32_t r = (ch / stride) % 8, g0 = ch - r * stride;
                const size_t i = (size_t)(ch % stride) * bd + rb;
                uint64_t *y = &nxt[(size_t)ch * limbs];
                std::memcpy(y, &cur[(size_t)g0 * limbs], 8 * limbs);
                for (uint32_t j = 1; j < 8; j++)
                    wide_mul_s64_add(y, &cur[(size_t)(g0 + j * stride) * limbs],
                                     tw[(i * 7 + (j - 1)) * 8 + ((r * j) & 7)], (int)limbs);
            }
            cur.swap(nxt);
        }
        std::memcpy(out + (size_t)o * limbs, &cur[(size_t)(P / bd) * limbs], 8 * limbs);
    }
}

bool merkle_verify(const uint8_t root[32], const uint8_t *col, size_t col_len, uint64_t li,
                   uint64_t lc, const uint8_t *sib, uint64_t ns, uint64_t expected) {
    if (li != expected) return false;
    uint8_t cur8[32];
    b3::hash(col, col_len, cur8);
    if (lc == 1) return li == 0 && ns == 0 && std::memcmp(cur8, root, 32) == 0;
    std::vector<int> dirs;
    uint64_t size = lc, idx = li;
    while (size > 1) {
        uint64_t p2 = 1;
        while (p2 < size) p2 <<= 1;
        const uint64_t split = p2 / 2;
        if (idx < split) {
            dirs.push_back(0);
            size = split;
        } else {
            dirs.push_back(1);
            size -= split;
            idx -= split;
        }
    }
    std::reverse(dirs.begin(), dirs.end());
    if (dirs.size() != ns) return false;
    uint32_t cur[8];
    for (int i = 0; i < 8; i++) cur[i] = b3::load_le32(cur8 + 4 * i);
    for (size_t i = 0; i < dirs.size(); i++) {
        uint32_t s[8];
        for (int w = 0; w < 8; w++) s[w] = b3::load_le32(sib + 32 * i + 4 * w);
        const bool root_merge = i + 1 == dirs.size();
        if (dirs[i] == 0) b3::parent_cv(cur, s, root_merge, cur);
        else b3::parent_cv(s, cur, root_merge, cur);
    }
    uint8_t out[32];
    for (int i = 0; i < 8; i++) b3::store_le32(out + 4 * i, cur[i]);
    return std::memcmp(out, root, 32) == 0;
}

}  // namespace

namespace zg {

// ------------------------------------------------------------------- commit
zg_status commit_device(zg_params *p, zg_ctx *lane, const void *polys_d, uint32_t batch,
                        zg_hint **out) {
    ZG_TRY(validate_budget(p, batch));
    zg_ctx *ctx = lane;
    cudaStream_t s = ctx->stream;
    const uint32_t C = p->info.codeword_len;
    const uint32_t nrows = batch * p->info.num_rows;
    const size_t leaf_bytes = leaf_bytes_of(p, batch);
    if (leaf_bytes > 0xFFFFFFFFull || nrows > 65535) {
        set_error("commitment too large: %u rows, %zu-byte leaves", nrows, leaf_bytes);
        return ZG_ERR_INVALID_PARAM;
    }
    std::unique_ptr<zg_hint> h(new zg_hint());
    h->params = p;
    h->lane = ctx;
    h->batch = batch;
    h->nrows = nrows;
    h->depth = ilog2u(C);
    const size_t cw_bytes = ((size_t)C * leaf_bytes + 255) & ~(size_t)255;
    const size_t tree_bytes = (2 * (size_t)C - 1) * 32;
    h->block = ctx_alloc(ctx, cw_bytes + tree_bytes, &h->block_bytes);
    if (!h->block) return ZG_ERR_OOM;
    h->d_cw = static_cast<uint8_t *>(h->block);
    h->d_tree = h->d_cw + cw_bytes;
    hphase(ctx, "commit_alloc");
    auto fail = [&](zg_status st) {
        ctx_release(ctx, h->block, h->block_bytes);
        h->block = nullptr;
        return st;
    };
    zg_status st = launch_encode(p, ctx, polys_d, nrows, h->d_cw, true, s);
    if (st != ZG_OK) return fail(st);
    uint32_t done = 0;
    st = launch_leaf_hash(ctx, h->d_cw, C, (uint32_t)leaf_bytes, h->d_tree, s, 0, -1, &done);
    if (st != ZG_OK) return fail(st);
    st = launch_merkle_levels(ctx, h->d_tree, C, s, 1, done);
    if (st != ZG_OK) return fail(st);
    if ((st = ctx->pin_out.ensure(64)) != ZG_OK) return fail(st);
    uint8_t *hroot = ctx->pin_out.as<uint8_t>();
    if (cudaMemcpyAsync(hroot, h->d_tree + merkle_layer_off(C, h->depth) * 32, 32,
                        cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        ctx_sync(ctx) != cudaSuccess) {
        set_error("commit failed: %s", cudaGetErrorString(cudaGetLastError()));
        return fail(ZG_ERR_CUDA);
    }
    std::memcpy(h->root, hroot, 32);
    hphase(ctx, "commit_gpu");
    *out = h.release();
    return ZG_OK;
}

// ----------------------------------------------------------- group commit
size_t group_cw_stride(const zg_params *p) {
    return (size_t)p->info.codeword_len * leaf_bytes_of(p, 1);
}
size_t group_tree_stride(const zg_params *p) { return (2 * (size_t)p->info.codeword_len - 1) * 32; }

bool group_fits(const zg_params *p, uint32_t m) {
    if (m <= 1) return true;
    const uint64_t rows = (uint64_t)m * p->info.num_rows;
    return group_cw_stride(p) % 256 == 0 && rows <= 65535 && leaf_bytes_of(p, 1) <= 0xFFFFFFFFull &&
           (uint64_t)m * p->info.codeword_len <= 0xFFFFFFFFull;
}

zg_status launch_commit_group(zg_params *p, zg_ctx *lane, const void *polys_d, uint32_t m,
                              uint8_t *cw_d, uint8_t *tree_d, cudaStream_t s,
                              const CommitTuning &tune) {
    if (!group_fits(p, m)) {
        set_error("%u polynomials of this shape do not fit one launch chain", m);
        return ZG_ERR_INVALID_PARAM;
    }
    const uint32_t C = p->info.codeword_len, R = p->info.num_rows;
    ZG_TRY(launch_encode(p, lane, polys_d, m * R, cw_d, true, s, m > 1 ? R : 0, tune.base_variant));
    uint32_t done = 0;
    ZG_TRY(launch_leaf_hash(lane, cw_d, m * C, (uint32_t)leaf_bytes_of(p, 1), tree_d, s,
                            m > 1 ? C : 0, tune.leaf_variant, &done));
    return launch_merkle_levels(lane, tree_d, C, s, m, done);
}

zg_status commit_group_device(zg_params *p, zg_ctx *lane, const void *polys_d, uint32_t m,
                              zg_hint **hints, uint8_t *roots, const CommitTuning &tune) {
    ZG_TRY(validate_budget(p, 1));
    const uint32_t C = p->info.codeword_len;
    const size_t cws = group_cw_stride(p), trs = group_tree_stride(p);
    const size_t cw_bytes = ((size_t)m * cws + 255) & ~(size_t)255;
    auto blk = std::make_shared<SharedBlock>();
    blk->lane = lane;
    blk->ptr = ctx_alloc(lane, cw_bytes + (size_t)m * trs, &blk->bytes);
    if (!blk->ptr) return ZG_ERR_OOM;
    uint8_t *cw = static_cast<uint8_t *>(blk->ptr), *tree = cw + cw_bytes;
    cudaStream_t s = lane->stream;
    ZG_TRY(launch_commit_group(p, lane, polys_d, m, cw, tree, s, tune));
    ZG_TRY(lane->pin_out.ensure((size_t)m * 32));
    uint8_t *hr = lane->pin_out.as<uint8_t>();
    // roots: node 2C - 2 of every tree, one strided copy
    if (cudaMemcpy2DAsync(hr, 32, tree + (2 * (size_t)C - 2) * 32, trs, 32, m,
                          cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        ctx_sync(lane) != cudaSuccess) {
        set_error("group commit failed: %s", cudaGetErrorString(cudaGetLastError()));
        return ZG_ERR_CUDA;
    }
    if (roots) std::memcpy(roots, hr, (size_t)m * 32);
    if (hints) {
        for (uint32_t k = 0; k < m; k++) {
            zg_hint *h = new zg_hint();
            h->shared = blk;
            h->params = p;
            h->lane = lane;
            h->batch = 1;
            h->nrows = p->info.num_rows;
            h->depth = ilog2u(C);
            h->d_cw = cw + (size_t)k * cws;
            h->d_tree = tree + (size_t)k * trs;
            std::memcpy(h->root, hr + (size_t)k * 32, 32);
            hints[k] = h;
        }
    }
    return ZG_OK;
}

// -------------------------------------------------------------------- prove
zg_status prove_device(zg_params *p, zg_ctx *lane, zg_transcript *t, const void *polys_d,
                       uint32_t batch, const uint8_t *point, const zg_hint *hint, uint8_t *eval_out,
                       uint8_t *tail_out, bool point_is_field) {
    if (!t->has_field || t->f.L != (int)p->d.field_limbs) {
        set_error("transcript has no field configuration of %u limbs (sample it first)",
                  p->d.field_limbs);
        return ZG_ERR_INVALID_PARAM;
    }
    if (!hint || hint->params != p || hint->batch != batch) {
        set_error("hint does not match the parameters or batch size");
        return ZG_ERR_INVALID_PARAM;
    }
    ZG_TRY(validate_budget(p, batch));
    zg_ctx *ctx = lane;
    cudaStream_t s = ctx->stream;
    const FieldCfg &f = t->f;
    const int L = f.L;
    const uint32_t R = p->info.num_rows, RL = p->info.row_len, C = p->info.codeword_len;
    const uint32_t CL = p->d.comb_limbs, D = p->D, nv = p->d.num_vars;
    const uint32_t lr = ilog2u(R), nhi = nv - lr;
    const bool binary = p->d.eval_kind == ZG_EVAL_BINPOLY;
    hphase(ctx, "prove_enter");

    // point -> F, q0 (host), q1 (device) (point_to_tensor, pcs/utils.rs:90-114)
    std::vector<uint64_t> pf((size_t)(nv + 1) * L), omr((size_t)(nv + 1) * L);
    for (uint32_t i = 0; i < nv; i++) {
        if (point_is_field) {
            // prove_f (phase_prove.rs:119-130): the point is already in the field
            std::memcpy(&pf[(size_t)i * L], point + (size_t)8 * L * i, 8 * L);
            bool below = false;
            for (int w = L - 1; w >= 0; w--)
                if (pf[(size_t)i * L + w] != f.p[w]) {
                    below = pf[(size_t)i * L + w] < f.p[w];
                    break;
                }
            if (!below) {
                set_error("point coordinate %u is not a reduced field element", i);
                return ZG_ERR_INVALID_PARAM;
            }
        } else {
            f_from_i128(f, load_i128(point + 16 * i), &pf[(size_t)i * L]);
        }
        std::memcpy(&omr[(size_t)i * L], f.one, 8 * L);
        f_sub(f, &omr[(size_t)i * L], &pf[(size_t)i * L]);
    }
    std::vector<uint64_t> q0;
    if (lr) host_eq(f, &pf[(size_t)nhi * L], lr, q0);
    else q0.assign(f.one, f.one + L);

    // alphas (phase_prove.rs:157-161): Comb::DEGREE_BOUND + 1 = D challenges
    const uint32_t na = binary && D > 1 ? D : 0;
    std::vector<i128> alphas((size_t)batch * std::max<uint32_t>(na, 1), (i128)1);
    if (binary && D == 1) {
        for (uint32_t b = 0; b < batch; b++) alphas[b] = 1;
    }
    for (uint32_t b = 0; b < batch; b++)
        for (uint32_t i = 0; i < na; i++) alphas[(size_t)b * na + i] = tr_challenge_i128(t);
    const uint32_t Da = binary ? std::max<uint32_t>(na, 1) : 1;

    // device inputs: alphas | r_hi | omr_hi
    const size_t a_bytes = alphas.size() * 16, r_bytes = (size_t)std::max<uint32_t>(nhi, 1) * L * 8;
    const size_t in_bytes = a_bytes + 2 * r_bytes + 16 * (size_t)R + 4 * (size_t)p->d.num_openings + 256;
    ZG_TRY(ctx->prove_in.ensure(in_bytes));
    ZG_TRY(ctx->pin_in.ensure(in_bytes));
    uint8_t *hin = ctx->pin_in.as<uint8_t>();
    uint8_t *din = ctx->prove_in.as<uint8_t>();
    std::memcpy(hin, alphas.data(), a_bytes);
    std::memcpy(hin + a_bytes, pf.data(), (size_t)nhi * L * 8);
    std::memcpy(hin + a_bytes + r_bytes, omr.data(), (size_t)nhi * L * 8);
    ZG_CUDA(cudaMemcpyAsync(din, hin, a_bytes + 2 * r_bytes, cudaMemcpyHostToDevice, s));

    const uint32_t nparts = (RL + 255) / 256;
    const size_t q1_bytes = (size_t)RL * L * 8;
    const size_t part_bytes = (size_t)batch * R * nparts * L * 8;
    const size_t comb_bytes = (size_t)RL * CL * 8;
    const size_t leaf_bytes = leaf_bytes_of(p, batch);
    const size_t open_bytes = leaf_bytes + 24 + 32 * (size_t)hint->depth;
    const size_t tail_bytes = comb_bytes + open_bytes * p->d.num_openings;
    const size_t out_bytes = q1_bytes + part_bytes + tail_bytes + 64;
    ZG_TRY(ctx->prove_out.ensure(out_bytes));
    ZG_TRY(ctx->wprime.ensure((size_t)batch * R * RL * CL * 8));
    uint8_t *dout = ctx->prove_out.as<uint8_t>();
    uint64_t *q1_d = reinterpret_cast<uint64_t *>(dout);
    uint64_t *part_d = reinterpret_cast<uint64_t *>(dout + q1_bytes);
    uint8_t *tail_d = dout + q1_bytes + part_bytes;
    tail_d = reinterpret_cast<uint8_t *>(((uintptr_t)tail_d + 15) & ~(uintptr_t)15);

    if (nhi) {
        ZG_TRY(launch_eq_table(ctx, reinterpret_cast<const uint64_t *>(din + a_bytes),
                               reinterpret_cast<const uint64_t *>(din + a_bytes + r_bytes), nhi, f,
                               q1_d, s));
    } else {
        ZG_CUDA(cudaMemcpyAsync(q1_d, f.one, 8 * L, cudaMemcpyHostToDevice, s));
    }
    ProjectArgs pa{polys_d, binary ? 1 : p->d.eval_kind == ZG_EVAL_I64 ? 2 : 0, reinterpret_cast<const i128 *>(din), Da,
                   dmask_of(D), q1_d, RL, R, batch, CL, &f, ctx->wprime.as<uint64_t>(), part_d};
    ZG_TRY(launch_project_rows(ctx, pa, s));
    ZG_TRY(ctx->pin_out.ensure(std::max(part_bytes, tail_bytes) + 64));
    uint64_t *hb = ctx->pin_out.as<uint64_t>();
    ZG_CUDA(cudaMemcpyAsync(hb, part_d, part_bytes, cudaMemcpyDeviceToHost, s));
    hphase(ctx, "prove_setup");
    ZG_CUDA(ctx_sync(ctx));
    hphase(ctx, "prove_rows_gpu");
    // b[j] = sum over polys and blocks of the partials (field addition)
    std::vector<uint64_t> bv((size_t)R * L, 0);
    for (uint32_t b = 0; b < batch; b++)
        for (uint32_t j = 0; j < R; j++)
            for (uint32_t q = 0; q < nparts; q++)
                f_add(f, &bv[(size_t)j * L], hb + (((size_t)b * R + j) * nparts + q) * L);
    hphase(ctx, "prove_b_reduce");

    // write_field_elements(b) (pcs_transcript.rs:99-142): no length prefix for
    // Uint<L>; modulus | inner per element, each absorbed.  The stream grows
    // by this proof at most once.
    const size_t fb = 8 * (size_t)L;
    if (t->stream.capacity() < t->stream.size() + zg_proof_size(p, batch))
        t->stream.reserve(std::max(t->stream.size() + zg_proof_size(p, batch), 2 * t->stream.capacity()));
    for (uint32_t j = 0; j < R; j++) {
        tr_absorb_field(t, &bv[(size_t)j * L]);
        const uint8_t *mod = reinterpret_cast<const uint8_t *>(f.p);
        const uint8_t *inr = reinterpret_cast<const uint8_t *>(&bv[(size_t)j * L]);
        t->stream.insert(t->stream.end(), mod, mod + fb);
        t->stream.insert(t->stream.end(), inr, inr + fb);
    }
    hphase(ctx, "prove_b_absorb");
    uint64_t ev[MAX_FIELD_LIMBS] = {0, 0, 0, 0};
    for (uint32_t j = 0; j < R; j++) {
        uint64_t tmp[MAX_FIELD_LIMBS];
        f_mul(f, &q0[(size_t)j * L], &bv[(size_t)j * L], tmp);
        f_add(f, ev, tmp);
    }
    std::vector<i128> coeffs(R, (i128)1);
    if (R > 1)
        for (uint32_t j = 0; j < R; j++) coeffs[j] = tr_challenge_i128(t);
    std::vector<uint32_t> idxs(p->d.num_openings);
    for (uint32_t o = 0; o < p->d.num_openings; o++) idxs[o] = tr_challenge_u32(t) % C;
    hphase(ctx, "prove_fs");

    // second upload: coeffs | indices
    const size_t c_off = 0, i_off = 16 * (size_t)R;
    uint8_t *hin2 = hin + ((a_bytes + 2 * r_bytes + 15) & ~(size_t)15);
    uint8_t *din2 = din + ((a_bytes + 2 * r_bytes + 15) & ~(size_t)15);
    std::memcpy(hin2 + c_off, coeffs.data(), 16 * (size_t)R);
    std::memcpy(hin2 + i_off, idxs.data(), 4 * idxs.size());
    ZG_CUDA(cudaMemcpyAsync(din2, hin2, i_off + 4 * idxs.size(), cudaMemcpyHostToDevice, s));
    CombineArgs ca{ctx->wprime.as<uint64_t>(), reinterpret_cast<const i128 *>(din2 + c_off),
                   batch, R, RL, CL, reinterpret_cast<uint64_t *>(tail_d), hint->d_cw,
                   (uint32_t)leaf_bytes, hint->d_tree, hint->depth, C,
                   p->d.num_openings, reinterpret_cast<const uint32_t *>(din2 + i_off),
                   tail_d + comb_bytes};
    ZG_TRY(launch_combined_and_openings(ctx, ca, s));
    // The proof tail (combined row + openings) goes straight to tail_out when
    // the caller gave one that is page-locked; otherwise through pinned staging.
    bool direct = false;
    if (tail_out) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, tail_out) == cudaSuccess && at.type == cudaMemoryTypeHost)
            direct = true;
        cudaGetLastError();
    }
    uint8_t *htail = direct ? tail_out : ctx->pin_out.as<uint8_t>();
    ZG_CUDA(cudaMemcpyAsync(htail, tail_d, tail_bytes, cudaMemcpyDeviceToHost, s));
    ZG_CUDA(ctx_sync(ctx));
    hphase(ctx, "prove_tail_gpu");
    if (tail_out) {
        if (!direct) std::memcpy(tail_out, htail, tail_bytes);
    } else {
        t->stream.insert(t->stream.end(), htail, htail + tail_bytes);
    }
    if (eval_out) std::memcpy(eval_out, ev, fb);
    hphase(ctx, "prove_stream");
    return ZG_OK;
}

// ------------------------------------------------------------------- verify
// encode_wide at the opened positions: on the parameters' device when they
// have one (one block per position), else on the host.
static zg_status encode_wide_at(zg_params *p, const uint64_t *row, uint32_t CL, const uint32_t *pos,
                                uint32_t n, uint64_t *out) {
    if (!p->ctx || p->d.code_kind != ZG_CODE_IPRS || p->info.depth > 3) {
        host_encode_wide_at(p, row, CL, pos, n, out);
        return ZG_OK;
    }
    zg_ctx *ctx = p->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    const size_t row_b = (size_t)p->info.row_len * CL * 8, pos_b = ((size_t)n * 4 + 255) & ~(size_t)255;
    const size_t out_b = (size_t)n * CL * 8;
    const size_t row_off = 0, pos_off = (row_b + 255) & ~(size_t)255, out_off = pos_off + pos_b;
    ZG_TRY(ctx->prove_in.ensure(out_off + out_b));
    uint8_t *base = ctx->prove_in.as<uint8_t>();
    cudaStream_t s = ctx->stream;
    ZG_CUDA(cudaMemcpyAsync(base + row_off, row, row_b, cudaMemcpyHostToDevice, s));
    ZG_CUDA(cudaMemcpyAsync(base + pos_off, pos, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    ZG_TRY(launch_encode_wide_at(p, ctx, reinterpret_cast<const uint64_t *>(base + row_off), CL,
                                 reinterpret_cast<const uint32_t *>(base + pos_off), n,
                                 reinterpret_cast<uint64_t *>(base + out_off), s));
    ZG_CUDA(cudaMemcpyAsync(out, base + out_off, out_b, cudaMemcpyDeviceToHost, s));
    ZG_CUDA(ctx_sync(ctx));
    return ZG_OK;
}

zg_status verify_host(zg_params *p, const uint8_t root[32], uint32_t batch, const uint8_t *point,
                      const uint8_t *eval, const uint8_t *proof, size_t proof_len) {
    ZG_TRY(validate_budget(p, batch));
    zg_transcript tr;
    tr_absorb_slice(&tr, root, 32);
    const int L = (int)p->d.field_limbs;
    uint64_t prime[MAX_FIELD_LIMBS] = {0, 0, 0, 0};
    tr_get_prime(&tr, L, prime, 0);
    field_cfg_init(tr.f, prime, L);
    tr.has_field = true;
    const FieldCfg &f = tr.f;
    const uint32_t R = p->info.num_rows, RL = p->info.row_len, C = p->info.codeword_len;
    const uint32_t CL = p->d.comb_limbs, D = p->D, nv = p->d.num_vars;
    const uint32_t lr = ilog2u(R), nhi = nv - lr;
    const bool binary = p->d.eval_kind == ZG_EVAL_BINPOLY;
    // sample_alphas (phase_verify.rs:247-261)
    const uint32_t na = binary && D > 1 ? D : 1;
    std::vector<i128> alphas((size_t)batch * na, (i128)1);
    if (binary && D > 1)
        for (auto &a : alphas) a = tr_challenge_i128(&tr);
    std::vector<uint64_t> pf((size_t)(nv + 1) * L);
    for (uint32_t i = 0; i < nv; i++) f_from_i128(f, load_i128(point + 16 * i), &pf[(size_t)i * L]);
    std::vector<uint64_t> q0, q1;
    if (lr) host_eq(f, &pf[(size_t)nhi * L], lr, q0);
    else q0.assign(f.one, f.one + L);
    if (nhi) host_eq(f, pf.data(), nhi, q1);
    else q1.assign(f.one, f.one + L);

    size_t pos = 0;
    auto take = [&](size_t n) -> const uint8_t * {
        if (pos + n > proof_len) return nullptr;
        const uint8_t *r = proof + pos;
        pos += n;
        return r;
    };
    const size_t fb = 8 * (size_t)L;
    std::vector<uint64_t> bv((size_t)R * L);
    for (uint32_t j = 0; j < R; j++) {
        const uint8_t *mod = take(fb), *inr = take(fb);
        if (!mod || !inr) {
            set_error("proof truncated while reading b");
            return ZG_ERR_SERIALIZATION;
        }
        if (std::memcmp(mod, f.p, fb) != 0) {
            set_error("field element modulus differs from the sampled field");
            return ZG_ERR_INVALID_OPEN;
        }
        std::memcpy(&bv[(size_t)j * L], inr, fb);
        tr_absorb_field(&tr, &bv[(size_t)j * L]);
    }
    // check 1: <q0, b> == eval
    uint64_t acc[MAX_FIELD_LIMBS] = {0, 0, 0, 0}, tmp[MAX_FIELD_LIMBS];
    for (uint32_t j = 0; j < R; j++) {
        f_mul(f, &q0[(size_t)j * L], &bv[(size_t)j * L], tmp);
        f_add(f, acc, tmp);
    }
    if (std::memcmp(acc, eval, fb) != 0) {
        set_error("Evaluation consistency failure");
        return ZG_ERR_INVALID_OPEN;
    }
    std::vector<i128> coeffs(R, (i128)1);
    if (R > 1)
        for (auto &c : coeffs) c = tr_challenge_i128(&tr);
    const uint8_t *cr = take((size_t)RL * CL * 8);
    if (!cr) {
        set_error("proof truncated while reading the combined row");
        return ZG_ERR_SERIALIZATION;
    }
    std::vector<uint64_t> comb((size_t)RL * CL);
    std::memcpy(comb.data(), cr, comb.size() * 8);
    // The opened columns are the next num_openings challenges (nothing is
    // absorbed in between), so draw them first and encode only those positions.
    const uint32_t nop = p->d.num_openings;
    std::vector<uint32_t> opened(nop);
    for (uint32_t o = 0; o < nop; o++) opened[o] = tr_challenge_u32(&tr) % C;
    std::vector<uint64_t> enc((size_t)nop * CL);
    ZG_TRY(encode_wide_at(p, comb.data(), CL, opened.data(), nop, enc.data()));
    // check 2: <F(comb), q1> == <F(coeffs), b>
    uint64_t lhs[MAX_FIELD_LIMBS] = {0, 0, 0, 0}, rhs[MAX_FIELD_LIMBS] = {0, 0, 0, 0};
    for (uint32_t c = 0; c < RL; c++) {
        uint64_t fe[MAX_FIELD_LIMBS];
        f_from_signed(f, &comb[(size_t)c * CL], (int)CL, fe);
        f_mul(f, fe, &q1[(size_t)c * L], tmp);
        f_add(f, lhs, tmp);
    }
    for (uint32_t j = 0; j < R; j++) {
        uint64_t fe[MAX_FIELD_LIMBS];
        f_from_i128(f, coeffs[j], fe);
        f_mul(f, fe, &bv[(size_t)j * L], tmp);
        f_add(f, rhs, tmp);
    }
    if (std::memcmp(lhs, rhs, fb) != 0) {
        set_error("Coherence failure");
        return ZG_ERR_INVALID_OPEN;
    }
    const size_t cwb = p->info.cw_bytes, colbytes = (size_t)batch * R * cwb;
    // Parse the openings in order up to the first framing error, check the
    // parsed ones in parallel, and report whichever failure comes first in
    // opening order (what the sequential verifier reports).
    struct Opening {
        const uint8_t *col, *sib;
        uint64_t li, lc, np;
    };
    std::vector<Opening> ops;
    ops.reserve(nop);
    zg_status parse_st = ZG_OK;
    std::string parse_msg;
    for (uint32_t o = 0; o < nop && parse_st == ZG_OK; o++) {
        const uint8_t *col = take(colbytes), *hdr = take(24);
        if (!col || !hdr) {
            parse_st = ZG_ERR_SERIALIZATION;
            parse_msg = "proof truncated in column opening " + std::to_string(o);
            break;
        }
        uint64_t li, lc, np;
        std::memcpy(&li, hdr, 8);
        std::memcpy(&lc, hdr + 8, 8);
        std::memcpy(&np, hdr + 16, 8);
        if (np == 0 || li >= lc || np > 64) {
            parse_st = ZG_ERR_SERIALIZATION;
            parse_msg = "malformed Merkle proof in opening " + std::to_string(o);
            break;
        }
        const uint8_t *sib = take(32 * np);
        if (!sib) {
            parse_st = ZG_ERR_SERIALIZATION;
            parse_msg = "proof truncated in Merkle path " + std::to_string(o);
            break;
        }
        ops.push_back(Opening{col, sib, li, lc, np});
    }
    const uint32_t nparsed = (uint32_t)ops.size();
    // 0 = passes, 1 = proximity failure, 2 = Merkle failure
    std::vector<int> bad(nparsed, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (long oo = 0; oo < (long)nparsed; oo++) {
        const uint32_t o = (uint32_t)oo;
        const Opening &op = ops[o];
        // check 3 (verify_column_testing_batched, phase_verify.rs:267-304)
        uint64_t sum[MAX_COMB_LIMBS] = {0};
        for (uint32_t b = 0; b < batch; b++)
            for (uint32_t j = 0; j < R; j++) {
                const uint8_t *e = op.col + ((size_t)b * R + j) * cwb;
                uint64_t v[MAX_COMB_LIMBS] = {0};
                if (!binary) {
                    uint64_t x[2];
                    std::memcpy(x, e, 16);
                    wide_sext(x, 2, v, (int)CL);
                } else {
                    for (uint32_t i = 0; i < D; i++) {
                        int64_t c64;
                        if (cwb == 8 * (size_t)D) {
                            std::memcpy(&c64, e + 8 * i, 8);
                        } else {
                            int32_t c32;
                            std::memcpy(&c32, e + 4 * i, 4);
                            c64 = c32;
                        }
                        uint64_t x[MAX_COMB_LIMBS], one = (uint64_t)c64;
                        wide_sext(&one, 1, x, (int)CL);
                        wide_mul_i128_add(v, x, alphas[(size_t)b * na + (na > 1 ? i : 0)], (int)CL);
                    }
                }
                wide_mul_i128_add(sum, v, coeffs[j], (int)CL);
            }
        if (std::memcmp(sum, &enc[(size_t)o * CL], 8 * CL) != 0) bad[o] = 1;
        else if (!merkle_verify(root, op.col, colbytes, op.li, op.lc, op.sib, op.np, opened[o])) bad[o] = 2;
    }
    for (uint32_t o = 0; o < nparsed; o++) {
        if (bad[o] == 1) {
            set_error("Proximity failure");
            return ZG_ERR_INVALID_OPEN;
        }
        if (bad[o] == 2) {
            set_error("Column opening verification failed");
            return ZG_ERR_INVALID_OPEN;
        }
    }
    if (parse_st != ZG_OK) {
        set_error("%s", parse_msg.c_str());
        return parse_st;
    }
    return ZG_OK;
}

}  // namespace zg

// ======================================================================= ABI
extern "C" {

const char *zg_last_error(void) { return zg::last_error(); }
const char *zg_version(void) { return "zipgpu 0.1 (sm_100a)"; }

zg_status zg_ctx_create(int device, zg_ctx **out) {
    if (!out) return ZG_ERR_INVALID_PARAM;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_error("no CUDA device available");
        return ZG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        set_error("device %d out of range (%d devices)", device, n);
        return ZG_ERR_INVALID_PARAM;
    }
    ZG_CUDA(cudaSetDevice(device));
    std::unique_ptr<zg_ctx> c(new zg_ctx());
    c->device = device;
    ZG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    ZG_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    c->status = device_status_word(device);
    if (!c->status) {
        set_error("could not map the device status word");
        return ZG_ERR_CUDA;
    }
    *out = c.release();
    return ZG_OK;
}

zg_status zg_ctx_destroy(zg_ctx *ctx) {
    if (!ctx) return ZG_OK;
    cudaSetDevice(ctx->device);
    ctx->plans.clear();
    for (zg_ctx *l : ctx->lanes) zg_ctx_destroy(l);
    ctx->lanes.clear();
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (DevBuf *b : {&ctx->evals, &ctx->stage_a, &ctx->stage_b, &ctx->stage_c, &ctx->chunk_cv,
                      &ctx->wprime, &ctx->prove_in, &ctx->prove_out, &ctx->sc_arena, &ctx->piop_arena,
                      &ctx->trace_arena, &ctx->mle_arena})
        b->release();
    cudaStreamSynchronize(ctx->stream);  // stream-ordered frees of pooled buffers
    if (ctx->sync_event) cudaEventDestroy(ctx->sync_event);
    ctx->pin_in.release();
    ctx->pin_out.release();
    ktimer_collect(ctx);
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    ctx_cache_clear(ctx);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return ZG_OK;
}

uint64_t zg_ctx_kernel_launches(const zg_ctx *ctx) {
    if (!ctx) return 0;
    uint64_t n = ctx->launches + (uint64_t)ctx->launch_adjust;
    for (const zg_ctx *l : ctx->lanes) n += l->launches;
    return n;
}

zg_status zg_selftest_bounded_wait(zg_ctx *ctx, uint32_t *status_seen) {
    if (!ctx || !status_seen) return ZG_ERR_INVALID_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    ZG_CUDA(cudaDeviceSynchronize());
    *status_seen = 0;
    if (device_status_value(ctx->device) != 0) {
        set_error("device %d already reported a timed-out wait (status %u)", ctx->device,
                  device_status_value(ctx->device));
        return ZG_ERR_CUDA;
    }
    ZG_TRY(launch_wait_probe(ctx, ctx->stream));
    ZG_CUDA(cudaStreamSynchronize(ctx->stream));
    *status_seen = device_status_value(ctx->device);
    device_status_clear(ctx->device);
    return ZG_OK;
}

zg_status zg_ctx_set_kernel_timing(zg_ctx *ctx, int enable) {
    if (!ctx) return ZG_ERR_INVALID_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    ktimer_collect(ctx);
    ctx->timing = enable != 0;
    return ZG_OK;
}

zg_status zg_ctx_kernel_timing_report(zg_ctx *ctx, char *buf, size_t cap, size_t *len) {
    if (!ctx || !len) return ZG_ERR_INVALID_PARAM;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    ktimer_collect(ctx);
    std::string out;
    for (auto &t : ctx->totals) {
        char line[256];
        snprintf(line, sizeof line, "%s,%llu,%.6f\n", t.first.c_str(),
                 (unsigned long long)t.second.second, t.second.first);
        out += line;
    }
    *len = out.size();
    if (buf && cap) {
        size_t n = std::min(cap - 1, out.size());
        std::memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    ctx->totals.clear();
    return ZG_OK;
}
void *zg_ctx_stream(zg_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// ctx may be NULL: the parameters are then host-only (tables, encode_wide,
// verify) and the device entry points report ZG_ERR_NO_DEVICE.
static zg_status params_create_impl(zg_ctx *ctx, const zg_params_desc *desc, zg_params **out) {
    if (!desc || !out) return ZG_ERR_INVALID_PARAM;
    *out = nullptr;
    zg_params_desc d = *desc;
    if (d.eval_kind > ZG_EVAL_I64 || d.code_kind > ZG_CODE_RAA_SIGN_FLIP) {
        set_error("unknown evaluation or code kind");
        return ZG_ERR_INVALID_PARAM;
    }
    if (d.eval_kind != ZG_EVAL_BINPOLY) d.degree_plus_one = 1;
    if (d.eval_kind == ZG_EVAL_BINPOLY && (d.degree_plus_one < 1 || d.degree_plus_one > 64)) {
        set_error("BinaryPoly coefficient count must be in 1..64");
        return ZG_ERR_INVALID_PARAM;
    }
    if (!is_pow2(d.rep)) {
        set_error("Repetition factor must be a power of two");
        return ZG_ERR_INVALID_PARAM;
    }
    if (d.num_vars > 30 || !is_pow2(d.row_len) || ((1ull << d.num_vars) % d.row_len) != 0) {
        set_error("poly_size (2^%u) must be divisible by row_len (%u)", d.num_vars, d.row_len);
        return ZG_ERR_INVALID_PARAM;
    }
    if (d.comb_limbs < 1 || d.comb_limbs > MAX_COMB_LIMBS || (d.field_limbs != 3 && d.field_limbs != 4)) {
        set_error("comb_limbs must be 1..8 and field_limbs 3 or 4");
        return ZG_ERR_INVALID_PARAM;
    }
    if (d.num_openings == 0) d.num_openings = 147;
    std::unique_ptr<zg_params> p(new zg_params());
    static std::atomic<uint64_t> next_uid{1};
    p->uid = next_uid.fetch_add(1);
    p->ctx = ctx;
    p->d = d;
    p->D = d.eval_kind == ZG_EVAL_BINPOLY ? d.degree_plus_one : 1;
    zg_params_info &I = p->info;
    I.row_len = d.row_len;
    I.num_rows = (uint32_t)((1ull << d.num_vars) / d.row_len);
    I.eval_bytes = d.eval_kind == ZG_EVAL_I32 ? 4 : 8;
    I.comb_bytes = 8 * d.comb_limbs;
    I.field_bytes = 8 * d.field_limbs;
    if (ctx) ZG_CUDA(cudaSetDevice(ctx->device));
    if (d.code_kind == ZG_CODE_IPRS) {
        const uint32_t depth = d.iprs_depth ? d.iprs_depth : iprs_optimal_depth(d.row_len);
        if (!iprs_build_tables(d.row_len, depth, d.rep, p.get())) {
            set_error("invalid IPRS parameters: row_len %u, depth %u, rate 1/%u", d.row_len,
                      depth, d.rep);
            return ZG_ERR_INVALID_PARAM;
        }
        I.cw_bytes = d.eval_kind == ZG_EVAL_BINPOLY ? 8 * p->D : 16;
        const uint32_t bd = I.base_dim, bl = I.base_len;
        std::vector<int32_t> bmT((size_t)bd * bl);
        for (uint32_t r = 0; r < bd; r++)
            for (uint32_t c = 0; c < bl; c++) bmT[(size_t)c * bd + r] = (int32_t)p->bm[(size_t)r * bl + c];
        std::vector<int32_t> tw32(p->tw.size());
        std::vector<size_t> offs;
        size_t o = 0;
        for (uint32_t k = 0; k < depth; k++) {
            const size_t sub = (size_t)bd << (3 * k);
            offs.push_back(o);
            for (size_t i = 0; i < sub; i++)
                for (int e = 0; e < 56; e++) tw32[o + (size_t)e * sub + i] = (int32_t)p->tw[p->tw_off[k] + i * 56 + e];
            o += sub * 56;
        }
        p->tw_dev_off = offs;
        if (ctx) {
            ZG_CUDA(cudaMalloc(&p->d_bmT, bmT.size() * 4));
            ZG_CUDA(cudaMemcpy(p->d_bmT, bmT.data(), bmT.size() * 4, cudaMemcpyHostToDevice));
            const uint32_t bdp = (bd + 7) / 8 * 8;
            std::vector<int32_t> bmP((size_t)bdp * bl, 0);
            for (uint32_t c = 0; c < bl; c++)
                for (uint32_t r = 0; r < bd; r++) bmP[(size_t)c * bdp + r] = (int32_t)p->bm[(size_t)r * bl + c];
            ZG_CUDA(cudaMalloc(&p->d_bmP, bmP.size() * 4));
            ZG_CUDA(cudaMemcpy(p->d_bmP, bmP.data(), bmP.size() * 4, cudaMemcpyHostToDevice));
            // u8 limbs: bm = l0 + 256 l1 - 65536 [bm < 0]
            const uint32_t blp = (bl + 31) / 32 * 32;
            std::vector<uint8_t> bmL((size_t)3 * bd * blp, 0);
            for (uint32_t r = 0; r < bd; r++)
                for (uint32_t c = 0; c < bl; c++) {
                    const int64_t v = p->bm[(size_t)r * bl + c];
                    const uint32_t u = (uint32_t)(v & 0xFFFF);
                    bmL[((size_t)0 * bd + r) * blp + c] = (uint8_t)(u & 0xFF);
                    bmL[((size_t)1 * bd + r) * blp + c] = (uint8_t)(u >> 8);
                    bmL[((size_t)2 * bd + r) * blp + c] = v < 0 ? 1 : 0;
                }
            ZG_CUDA(cudaMalloc(&p->d_bmL, bmL.size()));
            ZG_CUDA(cudaMemcpy(p->d_bmL, bmL.data(), bmL.size(), cudaMemcpyHostToDevice));
            // tcgen05 operand image: row offsets that bring every row into
            // [-2^15, 2^15), then two byte limbs in the swizzled tile layout
            std::vector<int32_t> off;
            if (build_umma_offsets(p->bm, bd, bl, off)) {
                const uint32_t kp = (bl + 127) / 128 * 128, atoms = kp / 128;
                const uint32_t tiles = (bd + kUmmaImgRows - 1) / kUmmaImgRows;
                std::vector<uint8_t> img((size_t)tiles * 2 * kp * kUmmaImgRows, 0);
                off.resize((size_t)tiles * kUmmaImgRows, 0);
                for (uint32_t r = 0; r < bd; r++) {
                    const uint32_t t = r / kUmmaImgRows, rr = r % kUmmaImgRows;
                    for (uint32_t c = 0; c < bl; c++) {
                        const int32_t v = (int32_t)p->bm[(size_t)r * bl + c] + off[r];
                        const uint8_t limb[2] = {(uint8_t)(v & 0xFF), (uint8_t)((v >> 8) & 0xFF)};
                        for (uint32_t l = 0; l < 2; l++)
                            img[((size_t)t * 2 + l) * atoms * kUmmaImgRows * 128 +
                                umma::sw128_offset(rr, c, kUmmaImgRows)] = limb[l];
                    }
                }
                ZG_CUDA(cudaMalloc(&p->d_bmU, img.size()));
                ZG_CUDA(cudaMemcpy(p->d_bmU, img.data(), img.size(), cudaMemcpyHostToDevice));
                std::vector<int32_t> noff(off.size());  // the kernels add -off[r] x popcount
                for (size_t i = 0; i < off.size(); i++) noff[i] = -off[i];
                ZG_CUDA(cudaMalloc(&p->d_bmOff, noff.size() * 4));
                ZG_CUDA(cudaMemcpy(p->d_bmOff, noff.data(), noff.size() * 4, cudaMemcpyHostToDevice));
                p->umma_kp = kp;
            }
            ZG_CUDA(cudaMalloc(&p->d_tw, std::max<size_t>(tw32.size(), 1) * 4));
            if (!tw32.empty())
                ZG_CUDA(cudaMemcpy(p->d_tw, tw32.data(), tw32.size() * 4, cudaMemcpyHostToDevice));
            if (depth == 2) {
                // twiddles of both stages per base position, in the order the
                // fused stage kernel uses them (tw[e] with e = (j-1)*8 + ((r*j) & 7))
                std::vector<int32_t> t2((size_t)bd * 576, 0);
                for (uint32_t rb = 0; rb < bd; rb++) {
                    int32_t *dst = t2.data() + (size_t)rb * 576;
                    for (uint32_t r0 = 0; r0 < 8; r0++)
                        for (uint32_t j = 1; j < 8; j++)
                            dst[r0 * 8 + j] = (int32_t)p->tw[p->tw_off[0] + (size_t)rb * 56 + (j - 1) * 8 + ((r0 * j) & 7)];
                    for (uint32_t r0 = 0; r0 < 8; r0++)
                        for (uint32_t r1 = 0; r1 < 8; r1++)
                            for (uint32_t j = 1; j < 8; j++)
                                dst[64 + (r0 * 8 + r1) * 8 + j] =
                                    (int32_t)p->tw[p->tw_off[1] + ((size_t)r0 * bd + rb) * 56 + (j - 1) * 8 + ((r1 * j) & 7)];
                }
                ZG_CUDA(cudaMalloc(&p->d_tw2r, t2.size() * 4));
                ZG_CUDA(cudaMemcpy(p->d_tw2r, t2.data(), t2.size() * 4, cudaMemcpyHostToDevice));
            }
        }
    } else {
        const uint64_t n = (uint64_t)d.row_len * d.rep;
        if (n > (1u << 24)) {
            set_error("RAA codeword too long");
            return ZG_ERR_INVALID_PARAM;
        }
        // RaaCode::new width check (raa.rs:54-74): Cw coefficients are i32.
        const uint32_t eval_bits = d.eval_kind == ZG_EVAL_BINPOLY ? 1 : d.eval_kind == ZG_EVAL_I64 ? 64 : 32;
        const uint32_t need = eval_bits + 2 * ilog2u(d.row_len) + 2 * ilog2u(d.rep);
        if (need > 32) {
            set_error("Cannot fit %u-bit wide codeword entries in 32 bits entries", need);
            return ZG_ERR_INVALID_PARAM;
        }
        I.codeword_len = (uint32_t)n;
        I.cw_bytes = 4 * p->D;
        p->perm1.resize(n);
        p->perm2.resize(n);
        stdrng_shuffle_identity(1, (uint32_t)n, p->perm1.data());
        stdrng_shuffle_identity(2, (uint32_t)n, p->perm2.data());
        if (ctx) {
            ZG_CUDA(cudaMalloc(&p->d_perm, n * 8));
            ZG_CUDA(cudaMemcpy(p->d_perm, p->perm1.data(), n * 4, cudaMemcpyHostToDevice));
            ZG_CUDA(cudaMemcpy(p->d_perm + n, p->perm2.data(), n * 4, cudaMemcpyHostToDevice));
        }
    }
    *out = p.release();
    return ZG_OK;
}

zg_status zg_params_create(zg_ctx *ctx, const zg_params_desc *desc, zg_params **out) {
    ZG_GUARD(params_create_impl(ctx, desc, out));
}

zg_status zg_params_destroy(zg_params *p) {
    if (!p) return ZG_OK;
    if (p->ctx) {
        cudaSetDevice(p->ctx->device);
        drop_plans_of(p->ctx, p);  // their graphs point at this set's device tables
        cudaFree(p->d_bmT);
        cudaFree(p->d_bmP);
        cudaFree(p->d_bmL);
        cudaFree(p->d_bmU);
        cudaFree(p->d_bmOff);
        cudaFree(p->d_tw);
        cudaFree(p->d_tw2r);
        cudaFree(p->d_perm);
    }
    delete p;
    return ZG_OK;
}

zg_status zg_params_get_info(const zg_params *p, zg_params_info *info) {
    if (!p || !info) return ZG_ERR_INVALID_PARAM;
    *info = p->info;
    return ZG_OK;
}

zg_status zg_params_iprs_tables(const zg_params *p, int64_t *base_matrix, int64_t *twiddles) {
    if (!p || p->d.code_kind != ZG_CODE_IPRS) return ZG_ERR_INVALID_PARAM;
    if (base_matrix) std::memcpy(base_matrix, p->bm.data(), p->bm.size() * 8);
    if (twiddles && !p->tw.empty()) std::memcpy(twiddles, p->tw.data(), p->tw.size() * 8);
    return ZG_OK;
}

zg_status zg_params_raa_perms(const zg_params *p, uint32_t *perm1, uint32_t *perm2) {
    if (!p || p->d.code_kind == ZG_CODE_IPRS) return ZG_ERR_INVALID_PARAM;
    if (perm1) std::memcpy(perm1, p->perm1.data(), p->perm1.size() * 4);
    if (perm2) std::memcpy(perm2, p->perm2.data(), p->perm2.size() * 4);
    return ZG_OK;
}

static zg_status need_device(const zg_params *p) {
    if (!p->ctx) {
        set_error("parameters were created without a device context");
        return ZG_ERR_NO_DEVICE;
    }
    return ZG_OK;
}

static zg_status encode_rows_impl(zg_params *p, const void *evals, void *cw_out) {
    if (!p || !evals || !cw_out) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    zg_ctx *ctx = p->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    const zg_params_info &I = p->info;
    const size_t in_bytes = (size_t)I.num_rows * I.row_len * I.eval_bytes;
    const size_t out_bytes = (size_t)I.num_rows * I.codeword_len * I.cw_bytes;
    ZG_TRY(ctx->evals.ensure(in_bytes));
    DevBuf outb;
    ZG_TRY(outb.ensure(out_bytes));
    ZG_CUDA(cudaMemcpyAsync(ctx->evals.ptr, evals, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    zg_status st = launch_encode(p, ctx, ctx->evals.ptr, I.num_rows, outb.as<uint8_t>(), false, ctx->stream);
    if (st == ZG_OK) {
        cudaError_t e = cudaMemcpyAsync(cw_out, outb.ptr, out_bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            set_error("encode failed: %s", cudaGetErrorString(e));
            st = ZG_ERR_CUDA;
        }
    }
    outb.release();
    return st;
}

zg_status zg_encode_rows(zg_params *p, const void *evals, void *cw_out) {
    ZG_GUARD(encode_rows_impl(p, evals, cw_out));
}

zg_status zg_encode_rows_d(zg_params *p, const void *evals_d, void *cw_out_d, void *stream) {
    if (!p || !evals_d || !cw_out_d) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : p->ctx->stream;
    ZG_GUARD(launch_encode(p, p->ctx, evals_d, p->info.num_rows, static_cast<uint8_t *>(cw_out_d), false, s));
}

zg_status zg_encode_wide(zg_params *p, const uint64_t *row, uint32_t limbs, uint64_t *out) {
    if (!p || !row || !out || limbs < 1 || limbs > MAX_COMB_LIMBS) return ZG_ERR_INVALID_PARAM;
    try {
        host_encode_wide(p, row, limbs, out);
    } catch (...) {
        set_error("encode_wide failed");
        return ZG_ERR_OOM;
    }
    return ZG_OK;
}

static zg_status merkle_root_impl(zg_ctx *ctx, const void *rows, uint32_t n_rows, uint32_t width,
                                  uint32_t eb, uint8_t root[32]) {
    if (!ctx || !rows || !root || n_rows == 0 || width == 0) {
        set_error("MerkleTree::new needs a non-empty matrix");
        return ZG_ERR_INVALID_PARAM;
    }
    if (!is_pow2(width)) {
        set_error("row_width.is_power_of_two()");
        return ZG_ERR_INVALID_PARAM;
    }
    if (((size_t)n_rows * eb) % 4 != 0) {
        set_error("leaf size must be a multiple of 4 bytes");
        return ZG_ERR_INVALID_PARAM;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    const size_t leaf = (size_t)n_rows * eb, total = leaf * width;
    // row-major to leaf-major on the host (a utility entry point)
    std::vector<uint8_t> lm(total);
    const uint8_t *src = static_cast<const uint8_t *>(rows);
    for (uint32_t r = 0; r < n_rows; r++)
        for (uint32_t j = 0; j < width; j++)
            std::memcpy(&lm[(size_t)j * leaf + (size_t)r * eb], src + ((size_t)r * width + j) * eb, eb);
    const size_t o = 2 * (size_t)width - 1;
    DevBuf cw, tree;
    ZG_TRY(cw.ensure(total));
    zg_status st = tree.ensure(o * 32);
    if (st != ZG_OK) {
        cw.release();
        return st;
    }
    cudaStream_t s = ctx->stream;
    st = ZG_OK;
    if (cudaMemcpyAsync(cw.ptr, lm.data(), total, cudaMemcpyHostToDevice, s) != cudaSuccess) st = ZG_ERR_CUDA;
    uint32_t done = 0;
    if (st == ZG_OK)
        st = launch_leaf_hash(ctx, cw.as<uint8_t>(), width, (uint32_t)leaf, tree.as<uint8_t>(), s, 0, -1, &done);
    if (st == ZG_OK) st = launch_merkle_levels(ctx, tree.as<uint8_t>(), width, s, 1, done);
    if (st == ZG_OK) {
        if (cudaMemcpyAsync(root, tree.as<uint8_t>() + (o - 1) * 32, 32, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            ctx_sync(ctx) != cudaSuccess) {
            set_error("merkle root failed");
            st = ZG_ERR_CUDA;
        }
    }
    cw.release();
    tree.release();
    return st;
}

zg_status zg_merkle_root(zg_ctx *ctx, const void *rows, uint32_t n_rows, uint32_t width,
                         uint32_t elem_bytes, uint8_t root[32]) {
    ZG_GUARD(merkle_root_impl(ctx, rows, n_rows, width, elem_bytes, root));
}

static zg_status stage_polys(zg_params *p, zg_ctx *ctx, const void *const *polys, uint32_t batch) {
    if (!polys) return ZG_ERR_INVALID_PARAM;
    const size_t pb = (size_t)p->info.num_rows * p->info.row_len * p->info.eval_bytes;
    ZG_TRY(ctx->evals.ensure(pb * batch));
    for (uint32_t b = 0; b < batch; b++) {
        if (!polys[b]) return ZG_ERR_INVALID_PARAM;
        ZG_CUDA(cudaMemcpyAsync(ctx->evals.as<uint8_t>() + pb * b, polys[b], pb,
                                cudaMemcpyHostToDevice, ctx->stream));
    }
    return ZG_OK;
}

static zg_status commit_impl(zg_params *p, const void *const *polys, uint32_t batch,
                             zg_hint **hint, uint8_t root[32]) {
    if (!p || !hint || !root) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    if (batch == 0) {
        set_error("Batch must contain at least one polynomial");
        return ZG_ERR_INVALID_PARAM;
    }
    ZG_TRY(stage_polys(p, p->ctx, polys, batch));
    ZG_TRY(commit_device(p, p->ctx, p->ctx->evals.ptr, batch, hint));
    std::memcpy(root, (*hint)->root, 32);
    return ZG_OK;
}

zg_status zg_commit(zg_params *p, const void *const *polys, uint32_t batch, zg_hint **hint,
                    uint8_t root[32]) {
    ZG_GUARD(commit_impl(p, polys, batch, hint, root));
}

static zg_status commit_d_impl(zg_params *p, const void *polys_d, uint32_t batch, zg_hint **hint,
                               uint8_t root[32]) {
    if (!p || !polys_d || !hint || !root) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    ZG_TRY(commit_device(p, p->ctx, polys_d, batch, hint));
    std::memcpy(root, (*hint)->root, 32);
    return ZG_OK;
}

zg_status zg_commit_d(zg_params *p, const void *polys_d, uint32_t batch, zg_hint **hint,
                      uint8_t root[32]) {
    ZG_GUARD(commit_d_impl(p, polys_d, batch, hint, root));
}

zg_status zg_hint_free(zg_hint *h) {
    if (!h) return ZG_OK;
    // the block returns to the context's cache (freed by zg_ctx_destroy)
    if (h->block) ctx_release(h->lane, h->block, h->block_bytes);
    delete h;
    return ZG_OK;
}

uint32_t zg_hint_batch(const zg_hint *h) { return h ? h->batch : 0; }

zg_status zg_hint_codeword(const zg_hint *h, uint32_t poly, void *cw_out) {
    if (!h || !cw_out || poly >= h->batch) return ZG_ERR_INVALID_PARAM;
    zg_params *p = h->params;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    const uint32_t C = p->info.codeword_len, R = p->info.num_rows;
    const size_t cwb = p->info.cw_bytes, leaf = (size_t)h->nrows * cwb;
    std::vector<uint8_t> all((size_t)C * leaf);
    ZG_CUDA(cudaMemcpy(all.data(), h->d_cw, all.size(), cudaMemcpyDeviceToHost));
    uint8_t *out = static_cast<uint8_t *>(cw_out);
    for (uint32_t r = 0; r < R; r++)
        for (uint32_t j = 0; j < C; j++)
            std::memcpy(out + ((size_t)r * C + j) * cwb, &all[(size_t)j * leaf + ((size_t)poly * R + r) * cwb], cwb);
    return ZG_OK;
}

zg_status zg_transcript_new(const uint8_t *roots, uint32_t n_roots, zg_transcript **out) {
    if (!out || (n_roots && !roots)) return ZG_ERR_INVALID_PARAM;
    try {
        zg_transcript *t = new zg_transcript();
        for (uint32_t i = 0; i < n_roots; i++) tr_absorb_slice(t, roots + 32 * (size_t)i, 32);
        *out = t;
    } catch (...) {
        set_error("host allocation failed");
        return ZG_ERR_OOM;
    }
    return ZG_OK;
}

zg_status zg_transcript_free(zg_transcript *t) {
    delete t;
    return ZG_OK;
}

zg_status zg_transcript_absorb(zg_transcript *t, const uint8_t *buf, size_t n) {
    if (!t || (n && !buf)) return ZG_ERR_INVALID_PARAM;
    tr_absorb(t, buf, n);
    return ZG_OK;
}

zg_status zg_transcript_absorb_slice(zg_transcript *t, const uint8_t *buf, size_t n) {
    if (!t || (n && !buf)) return ZG_ERR_INVALID_PARAM;
    tr_absorb_slice(t, buf, n);
    return ZG_OK;
}

zg_status zg_transcript_challenge(zg_transcript *t, uint8_t *out, size_t n) {
    if (!t || (n && !out)) return ZG_ERR_INVALID_PARAM;
    tr_challenge(t, out, n);
    return ZG_OK;
}

zg_status zg_transcript_sample_field(zg_transcript *t, uint32_t limbs, uint8_t *modulus_out) {
    if (!t || (limbs != 3 && limbs != 4)) return ZG_ERR_INVALID_PARAM;
    uint64_t prime[MAX_FIELD_LIMBS] = {0, 0, 0, 0};
    tr_get_prime(t, (int)limbs, prime, 0);
    field_cfg_init(t->f, prime, (int)limbs);
    t->has_field = true;
    if (modulus_out) std::memcpy(modulus_out, prime, 8 * limbs);
    return ZG_OK;
}

zg_status zg_transcript_proof(const zg_transcript *t, const uint8_t **data, size_t *len) {
    if (!t || !data || !len) return ZG_ERR_INVALID_PARAM;
    *data = t->stream.data();
    *len = t->stream.size();
    return ZG_OK;
}

static zg_status prove_impl(zg_params *p, zg_transcript *t, const void *const *polys,
                            uint32_t batch, const uint8_t *point, const zg_hint *hint,
                            uint8_t *eval_out) {
    if (!p || !t || !point) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    if (batch == 0) {
        set_error("Batch must contain at least one polynomial");
        return ZG_ERR_INVALID_PARAM;
    }
    ZG_TRY(stage_polys(p, p->ctx, polys, batch));
    return prove_device(p, p->ctx, t, p->ctx->evals.ptr, batch, point, hint, eval_out, nullptr);
}

zg_status zg_prove(zg_params *p, zg_transcript *t, const void *const *polys, uint32_t batch,
                   const uint8_t *point, const zg_hint *hint, uint8_t *eval_out) {
    ZG_GUARD(prove_impl(p, t, polys, batch, point, hint, eval_out));
}

static zg_status prove_f_impl(zg_params *p, zg_transcript *t, const void *polys, uint32_t batch,
                              const uint64_t *point_f, const zg_hint *hint, uint8_t *eval_out, bool on_device) {
    if (!p || !t || !point_f || !polys) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    if (batch == 0) {
        set_error("Batch must contain at least one polynomial");
        return ZG_ERR_INVALID_PARAM;
    }
    const void *d = polys;
    if (!on_device) {
        ZG_TRY(stage_polys(p, p->ctx, static_cast<const void *const *>(polys), batch));
        d = p->ctx->evals.ptr;
    }
    return prove_device(p, p->ctx, t, d, batch, reinterpret_cast<const uint8_t *>(point_f), hint, eval_out, nullptr,
                        true);
}

zg_status zg_prove_f(zg_params *p, zg_transcript *t, const void *const *polys, uint32_t batch,
                     const uint64_t *point_f, const zg_hint *hint, uint8_t *eval_out) {
    ZG_GUARD(prove_f_impl(p, t, polys, batch, point_f, hint, eval_out, false));
}

zg_status zg_prove_f_d(zg_params *p, zg_transcript *t, const void *polys_d, uint32_t batch,
                       const uint64_t *point_f, const zg_hint *hint, uint8_t *eval_out) {
    ZG_GUARD(prove_f_impl(p, t, polys_d, batch, point_f, hint, eval_out, true));
}

static zg_status prove_d_impl(zg_params *p, zg_transcript *t, const void *polys_d, uint32_t batch,
                              const uint8_t *point, const zg_hint *hint, uint8_t *eval_out) {
    if (!p || !t || !polys_d || !point) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    return prove_device(p, p->ctx, t, polys_d, batch, point, hint, eval_out, nullptr);
}

zg_status zg_prove_d(zg_params *p, zg_transcript *t, const void *polys_d, uint32_t batch,
                     const uint8_t *point, const zg_hint *hint, uint8_t *eval_out) {
    ZG_GUARD(prove_d_impl(p, t, polys_d, batch, point, hint, eval_out));
}

size_t zg_proof_size(const zg_params *p, uint32_t batch) {
    if (!p) return 0;
    const zg_params_info &I = p->info;
    const size_t depth = ilog2u(I.codeword_len);
    return (size_t)I.num_rows * 2 * I.field_bytes + (size_t)I.row_len * I.comb_bytes +
           (size_t)p->d.num_openings * ((size_t)batch * I.num_rows * I.cw_bytes + 24 + 32 * depth);
}

static zg_status commit_prove_common(zg_params *p, zg_ctx *lane, const void *polys_d,
                                     uint32_t batch, const uint8_t *point, uint8_t root[32],
                                     uint8_t *eval_out, uint8_t *proof, size_t *proof_len,
                                     int prime_threads) {
    const size_t need = zg_proof_size(p, batch);
    if (*proof_len < need) {
        *proof_len = need;
        set_error("proof buffer too small (%zu bytes needed)", need);
        return ZG_ERR_BUFFER_TOO_SMALL;
    }
    zg_hint *h = nullptr;
    hphase_start(lane);
    ZG_TRY(commit_device(p, lane, polys_d, batch, &h));
    std::memcpy(root, h->root, 32);
    zg_transcript t;
    tr_absorb_slice(&t, h->root, 32);
    uint64_t prime[MAX_FIELD_LIMBS] = {0, 0, 0, 0};
    tr_get_prime(&t, (int)p->d.field_limbs, prime, prime_threads);
    field_cfg_init(t.f, prime, (int)p->d.field_limbs);
    t.has_field = true;
    hphase(lane, "prime");
    // The b rows are written to the transcript stream; the rest of the proof
    // lands directly after them in the caller's buffer.
    const size_t head = (size_t)p->info.num_rows * 2 * p->info.field_bytes;
    zg_status st = prove_device(p, lane, &t, polys_d, batch, point, h, eval_out, proof + head);
    zg_hint_free(h);
    if (st != ZG_OK) return st;
    if (t.stream.size() != head) {
        set_error("internal: unexpected proof head size %zu", t.stream.size());
        return ZG_ERR_INVALID_PARAM;
    }
    std::memcpy(proof, t.stream.data(), head);
    *proof_len = need;
    hphase(lane, "proof_copy");
    return ZG_OK;
}

static zg_status commit_prove_impl(zg_params *p, const void *const *polys, uint32_t batch,
                                   const uint8_t *point, uint8_t root[32], uint8_t *eval_out,
                                   uint8_t *proof, size_t *proof_len) {
    if (!p || !polys || !point || !root || !proof || !proof_len) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    if (batch == 0) {
        set_error("Batch must contain at least one polynomial");
        return ZG_ERR_INVALID_PARAM;
    }
    ZG_TRY(stage_polys(p, p->ctx, polys, batch));
    return commit_prove_common(p, p->ctx, p->ctx->evals.ptr, batch, point, root, eval_out, proof,
                               proof_len, 0);
}

zg_status zg_commit_prove(zg_params *p, const void *const *polys, uint32_t batch,
                          const uint8_t *point, uint8_t root[32], uint8_t *eval_out,
                          uint8_t *proof, size_t *proof_len) {
    ZG_GUARD(commit_prove_impl(p, polys, batch, point, root, eval_out, proof, proof_len));
}

static zg_status commit_prove_d_impl(zg_params *p, const void *polys_d, uint32_t batch,
                                     const uint8_t *point, uint8_t root[32], uint8_t *eval_out,
                                     uint8_t *proof, size_t *proof_len) {
    if (!p || !polys_d || !point || !root || !proof || !proof_len) return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    std::lock_guard<std::mutex> lk(p->ctx->mu);
    ZG_CUDA(cudaSetDevice(p->ctx->device));
    return commit_prove_common(p, p->ctx, polys_d, batch, point, root, eval_out, proof, proof_len,
                               0);
}

zg_status zg_commit_prove_d(zg_params *p, const void *polys_d, uint32_t batch,
                            const uint8_t *point, uint8_t root[32], uint8_t *eval_out,
                            uint8_t *proof, size_t *proof_len) {
    ZG_GUARD(commit_prove_d_impl(p, polys_d, batch, point, root, eval_out, proof, proof_len));
}

static zg_status commit_prove_many_impl(zg_params *p, uint32_t n, const void *const *polys,
                                        int on_device, const uint8_t *points, uint8_t *roots,
                                        uint8_t *evals, uint8_t *const *proofs, size_t *proof_lens,
                                        uint32_t nlanes, double *latency_ms) {
    if (!p || !polys || !points || !roots || !evals || !proofs || !proof_lens || n == 0)
        return ZG_ERR_INVALID_PARAM;
    ZG_TRY(need_device(p));
    zg_ctx *ctx = p->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    nlanes = std::max<uint32_t>(1, std::min<uint32_t>({nlanes, n, 16}));
    ZG_TRY(ensure_lanes(ctx, nlanes));
    const int cores = std::max(1, omp_get_num_procs());
    const int per_lane = std::max(1, cores / (int)nlanes);
    const size_t pt_bytes = 16 * (size_t)p->d.num_vars, fb = 8 * (size_t)p->d.field_limbs;
    std::atomic<uint32_t> next{0};
    std::atomic<bool> failed{false};
    std::mutex err_mu;
    zg_status first_st = ZG_OK;
    std::string first_msg;
    auto worker = [&](uint32_t li) {
        cudaSetDevice(ctx->device);
        zg_ctx *lane = ctx->lanes[li];
        for (;;) {
            const uint32_t i = next.fetch_add(1);
            if (i >= n || failed.load()) break;
            const auto t0 = std::chrono::steady_clock::now();
            zg_status st = ZG_OK;
            const void *pd = polys[i];
            if (!on_device) {
                st = stage_polys(p, lane, &polys[i], 1);
                pd = lane->evals.ptr;
            }
            if (st == ZG_OK) {
                size_t plen = proof_lens[i];
                st = commit_prove_common(p, lane, pd, 1, points + pt_bytes * i, roots + 32 * (size_t)i,
                                         evals + fb * i, proofs[i], &plen, per_lane);
                proof_lens[i] = plen;
            }
            if (st != ZG_OK) {
                std::lock_guard<std::mutex> g(err_mu);
                if (first_st == ZG_OK) {
                    first_st = st;
                    first_msg = last_error();
                }
                failed.store(true);
                break;
            }
            if (latency_ms)
                latency_ms[i] = std::chrono::duration<double, std::milli>(
                                    std::chrono::steady_clock::now() - t0).count();
        }
    };
    std::vector<std::thread> th;
    for (uint32_t li = 0; li < nlanes; li++) th.emplace_back(worker, li);
    for (auto &t : th) t.join();
    if (first_st != ZG_OK) set_error("%s", first_msg.c_str());
    return first_st;
}

zg_status zg_commit_prove_many(zg_params *p, uint32_t n, const void *const *polys,
                               int polys_on_device, const uint8_t *points, uint8_t *roots,
                               uint8_t *evals, uint8_t *const *proofs, size_t *proof_lens,
                               uint32_t lanes, double *latency_ms) {
    ZG_GUARD(commit_prove_many_impl(p, n, polys, polys_on_device, points, roots, evals, proofs,
                                    proof_lens, lanes, latency_ms));
}

zg_status zg_verify(zg_params *p, const uint8_t root[32], uint32_t batch, const uint8_t *point,
                    const uint8_t *eval, const uint8_t *proof, size_t proof_len) {
    if (!p || !root || !point || !eval || (proof_len && !proof)) return ZG_ERR_INVALID_PARAM;
    ZG_GUARD(verify_host(p, root, batch, point, eval, proof, proof_len));
}

}  // extern "C"
