// PIOP sumcheck prover on the GPU (piop/src/sumcheck.rs:163-215,
// sumcheck/prover.rs:95-247, sumcheck/multi_degree.rs:259-355) for
// combination functions of the form
//   comb(v) = (sum_k coeff_k * prod_{i in S_k} v_i) * prod_f (a_f + b_f * v_{m_f}),
// a sum of products (the reference's test comb functions, sumcheck/tests/
// utils.rs:60-80) times affine factors (the combined-polynomial resolver's
// (1 - selector) * eq_r, combined_poly_resolver.rs:158-172).  MLE values are
// field elements in Montgomery form (DenseMultilinearExtension<F::Inner>),
// layout [mle][x][limb].
//
// Round i evaluates P_i(t) = sum_b comb(v_b + t (w_b - v_b)) at t = 0..deg
// over the pairs (v_b, w_b) = (m[2b], m[2b+1]) of the MLEs folded at the
// previous challenge, m'[b] = m[2b] + r (m[2b+1] - m[2b]).  One kernel per
// round does both: each thread folds its four entries of the previous round
// into its pair, writes the pair, and evaluates the comb on it.  Field
// addition is exact, so the order of the sums is free.
#include <algorithm>
#include <cstring>
#include <memory>

#include "zg_internal.h"

namespace zg {
namespace {

constexpr int kScThreads = 256;
// threads per pair: 1 when pairs fill the GPU, more when they do not (each
// thread's share of a pair is a long chain of dependent field products).  The
// thresholds are measured (CPR group at 2^18 points, 2.18 -> 1.90 ms, from
// 2^19 / 2^15): splitting a pair costs shuffles and idle threads, worth it
// only once a round has fewer than 2^16 pairs.
constexpr int kScSubMid = 4, kScSubMax = 16;
constexpr size_t kScSplitBelow = 1u << 16, kScSplitMore = 1u << 13;
constexpr int kScMaxDeg = 8;

// fix_variables_with_config (poly/src/mle/dense.rs:243-279), one variable.
template <int L>
__global__ void k_sc_fold(const uint64_t *__restrict__ in, uint64_t *__restrict__ out,
                          uint32_t K, size_t n_out, const uint64_t *__restrict__ r, FieldCfg f) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)K * n_out) return;
    const size_t j = t / n_out, b = t % n_out;
    const uint64_t *v0 = in + (j * 2 * n_out + 2 * b) * L, *v1 = v0 + L;
    uint64_t a[L], rr[L], prod[L], o[L];
    for (int w = 0; w < L; w++) {
        a[w] = v1[w];
        rr[w] = r[w];
        o[w] = v0[w];
    }
    fsub<L>(a, v0, f.p);
    fmul<L>(rr, a, f.p, f.n0, prod);
    fadd<L>(o, prod, f.p);
    uint64_t *d = out + (j * n_out + b) * L;
    for (int w = 0; w < L; w++) d[w] = o[w];
}

// The combination function of one group, in device memory.
struct ScComb {
    const uint64_t *coeffs;   // [n_products][L]
    const uint32_t *offsets;  // [n_products + 1]
    const uint32_t *indices;
    const uint32_t *fmles;    // [n_factors]
    const uint64_t *fa, *fb;  // [n_factors][L]
    uint32_t n_products, n_factors;
};

// A field element passed by value (in registers across calls).
template <int L>
struct Fe {
    uint64_t w[L];
};

// Out-of-line Montgomery product: one copy of its code for all the call sites
// of the round kernel.  Inlined at every site, the round kernel is thousands of
// straight-line instructions that a small round runs once per warp, so its time
// was instruction-cache misses, not arithmetic.
template <int L>
__device__ __noinline__ Fe<L> fmul_nl(Fe<L> a, Fe<L> b, Fe<L> p, uint64_t n0) {
    Fe<L> o;
    fmul<L>(a.w, b.w, p.w, n0, o.w);
    return o;
}

// OUTLINE: the out-of-line product (small rounds, bound by instruction fetch),
// else inlined (large rounds, where independent products must overlap).
template <int L, bool OUTLINE>
__device__ __forceinline__ void fmul_c(const uint64_t *a, const uint64_t *b, const Fe<L> &p,
                                       uint64_t n0, uint64_t *out) {
    if (!OUTLINE) {
        fmul<L>(a, b, p.w, n0, out);
        return;
    }
    Fe<L> x, y;
#pragma unroll
    for (int w = 0; w < L; w++) {
        x.w[w] = a[w];
        y.w[w] = b[w];
    }
    const Fe<L> o = fmul_nl<L>(x, y, p, n0);
#pragma unroll
    for (int w = 0; w < L; w++) out[w] = o.w[w];
}

template <int L>
__device__ __forceinline__ void load_el(const uint64_t *p, uint64_t (&v)[L]) {
#pragma unroll
    for (int w = 0; w < L; w++) v[w] = p[w];
}

// One thread's part of one pair in a round: with fold, the pair's MLEs are
// folded at r and written to dst first (each of the pair's kScSub threads folds
// every kScSub-th MLE); then the thread's share of the sum of products at
// t = 0..D, combined over the pair's threads by shuffles, times the affine
// factors.  Summing ev over every thread of every pair gives P(t).  All 32
// lanes of the warp must call it together (the shuffles take the full warp).
// OUTLINE selects the out-of-line field product.
template <int L, int D, int kScSub, bool OUTLINE>
__device__ __forceinline__ void sc_pair(const uint64_t *__restrict__ src, size_t src_len,
                                        uint64_t *__restrict__ dst, int fold,
                                        const uint64_t *__restrict__ r, uint32_t K, const ScComb &c,
                                        const FieldCfg &f, const Fe<L> &pf, size_t b, bool active,
                                        uint32_t sub, uint64_t (&ev)[D + 1][L]) {
    // the out-of-line form also keeps its loops over t rolled: it serves the
    // small rounds, whose time is the cold fetch of the kernel's code
    constexpr int kUT = OUTLINE ? 1 : 32;
    const size_t len = fold ? src_len / 2 : src_len;
#pragma unroll kUT
    for (int t = 0; t <= D; t++)
#pragma unroll
        for (int w = 0; w < L; w++) ev[t][w] = 0;
    if (active && fold) {
        uint64_t rr[L];
        load_el<L>(r, rr);
        for (uint32_t j = sub; j < K; j += kScSub) {
                const uint64_t *q = src + ((size_t)j * src_len + 4 * b) * L;
                uint64_t *o = dst + ((size_t)j * len + 2 * b) * L;
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    uint64_t a0[L], a1[L], pr[L];
                    load_el<L>(q + 2 * e * L, a0);
                    load_el<L>(q + (2 * e + 1) * L, a1);
                    fsub<L>(a1, a0, f.p);
                    fmul_c<L, OUTLINE>(rr, a1, pf, f.n0, pr);
                    fadd<L>(a0, pr, f.p);
#pragma unroll
                for (int w = 0; w < L; w++) o[e * L + w] = a0[w];
            }
        }
    }
    __syncwarp();  // the pair's folded MLEs, written by its kScSub threads, are visible
    const uint64_t *m = fold ? dst : src;
    if (active) {
        // this thread's share of the sum of products at t = 0..D.  Products of
        // one MLE are linear in t: their sum is kept at t = 0 and t = 1 only
        // (lin0, lin1) and extended to t = 2..D at the end (exact field values).
        uint64_t lin0[L], lin1[L];
#pragma unroll
        for (int w = 0; w < L; w++) lin0[w] = lin1[w] = 0;
        bool any_lin = false;
        for (uint32_t k = sub; k < c.n_products; k += kScSub) {
            uint64_t pr[D + 1][L];
            uint64_t cf[L];
            load_el<L>(c.coeffs + (size_t)k * L, cf);
            // (degrees 2..6: at 1 it saves nothing, above 6 its registers spill)
            if (D >= 2 && D <= 6 && c.offsets[k + 1] - c.offsets[k] == 1) {
                const uint64_t *v = m + ((size_t)c.indices[c.offsets[k]] * len + 2 * b) * L;
                uint64_t v0[L], v1[L], o[L];
                load_el<L>(v, v0);
                load_el<L>(v + L, v1);
                fmul_c<L, OUTLINE>(cf, v0, pf, f.n0, o);
                fadd<L>(lin0, o, f.p);
                fmul_c<L, OUTLINE>(cf, v1, pf, f.n0, o);
                fadd<L>(lin1, o, f.p);
                any_lin = true;
                continue;
            }
#pragma unroll kUT
            for (int t = 0; t <= D; t++)
#pragma unroll
                for (int w = 0; w < L; w++) pr[t][w] = cf[w];
            for (uint32_t q = c.offsets[k]; q < c.offsets[k + 1]; q++) {
                uint64_t cur[L], st[L];
                const uint64_t *v = m + ((size_t)c.indices[q] * len + 2 * b) * L;
                load_el<L>(v, cur);
                load_el<L>(v + L, st);
                fsub<L>(st, cur, f.p);
#pragma unroll kUT
                for (int t = 0; t <= D; t++) {
                    uint64_t o[L];
                    fmul_c<L, OUTLINE>(pr[t], cur, pf, f.n0, o);
#pragma unroll
                    for (int w = 0; w < L; w++) pr[t][w] = o[w];
                    if (t < D) fadd<L>(cur, st, f.p);
                }
            }
#pragma unroll kUT
            for (int t = 0; t <= D; t++) fadd<L>(ev[t], pr[t], f.p);
        }
        if (D >= 2 && D <= 6 && any_lin) {
            uint64_t d[L], cur[L];
#pragma unroll
            for (int w = 0; w < L; w++) {
                d[w] = lin1[w];
                cur[w] = lin1[w];
            }
            fsub<L>(d, lin0, f.p);
            fadd<L>(ev[0], lin0, f.p);
#pragma unroll kUT
            for (int t = 1; t <= D; t++) {
                if (t > 1) fadd<L>(cur, d, f.p);
                fadd<L>(ev[t], cur, f.p);
            }
        }
    }
    // the pair's full sum of products, in all its threads
#pragma unroll kUT
    for (int off = 1; off < kScSub; off <<= 1) {
#pragma unroll kUT
        for (int t = 0; t <= D; t++) {
            uint64_t o[L];
#pragma unroll
            for (int w = 0; w < L; w++) o[w] = __shfl_xor_sync(0xffffffffu, ev[t][w], off);
            fadd<L>(ev[t], o, f.p);
        }
    }
    if (kScSub > D) {
        // affine factors a + b * v, one evaluation point per thread of the pair:
        // thread `sub` <= D multiplies the pair's sum at t = sub by the factors
        // there and keeps only that entry (all threads hold the full sums)
        uint64_t keep[L];
#pragma unroll
        for (int w = 0; w < L; w++) keep[w] = 0;
        if (active && (int)sub <= D) {
#pragma unroll kUT
            for (int t = 0; t <= D; t++)
                if (t == (int)sub)
#pragma unroll
                    for (int w = 0; w < L; w++) keep[w] = ev[t][w];
            for (uint32_t q = 0; q < c.n_factors; q++) {
                uint64_t cur[L], st[L], fa[L], fbv[L], fv[L], o[L];
                const uint64_t *v = m + ((size_t)c.fmles[q] * len + 2 * b) * L;
                load_el<L>(v, cur);
                load_el<L>(v + L, st);
                fsub<L>(st, cur, f.p);
                for (uint32_t i = 0; i < sub; i++) fadd<L>(cur, st, f.p);  // v(sub)
                load_el<L>(c.fa + (size_t)q * L, fa);
                load_el<L>(c.fb + (size_t)q * L, fbv);
                fmul_c<L, OUTLINE>(fbv, cur, pf, f.n0, fv);
                fadd<L>(fv, fa, f.p);
                fmul_c<L, OUTLINE>(keep, fv, pf, f.n0, o);
#pragma unroll
                for (int w = 0; w < L; w++) keep[w] = o[w];
            }
        }
#pragma unroll kUT
        for (int t = 0; t <= D; t++)
#pragma unroll
            for (int w = 0; w < L; w++) ev[t][w] = t == (int)sub ? keep[w] : 0;
    } else if (sub != 0) {
#pragma unroll kUT
        for (int t = 0; t <= D; t++)
#pragma unroll
            for (int w = 0; w < L; w++) ev[t][w] = 0;
    } else if (active) {
        // affine factors a + b * v
        for (uint32_t q = 0; q < c.n_factors; q++) {
            uint64_t cur[L], st[L], fa[L], fbv[L];
            const uint64_t *v = m + ((size_t)c.fmles[q] * len + 2 * b) * L;
            load_el<L>(v, cur);
            load_el<L>(v + L, st);
            fsub<L>(st, cur, f.p);
            load_el<L>(c.fa + (size_t)q * L, fa);
            load_el<L>(c.fb + (size_t)q * L, fbv);
#pragma unroll kUT
            for (int t = 0; t <= D; t++) {
                uint64_t fv[L], o[L];
                fmul_c<L, OUTLINE>(fbv, cur, pf, f.n0, fv);
                fadd<L>(fv, fa, f.p);
                fmul_c<L, OUTLINE>(ev[t], fv, pf, f.n0, o);
#pragma unroll
                for (int w = 0; w < L; w++) ev[t][w] = o[w];
                if (t < D) fadd<L>(cur, st, f.p);
            }
        }
    }
}

// One round for one group: (fold) and the block's partial sums of P(t),
// t = 0..D.  src: K MLEs of src_len entries; with fold, the round's MLEs (half
// as long) are written to dst first.  kScSub consecutive threads share a pair.
template <int L, int D, int kScSub>
__global__ void __launch_bounds__(kScThreads, 2) k_sc_round(const uint64_t *__restrict__ src,
                                                         size_t src_len, uint64_t *__restrict__ dst,
                                                         int fold, const uint64_t *__restrict__ r,
                                                         uint32_t K, ScComb c, FieldCfg f,
                                                         uint64_t *__restrict__ partials) {
    __shared__ uint64_t red[kScThreads / 32][(D + 1) * L];
    constexpr int kUT = kScSub == kScSubMax ? 1 : 32;  // rolled in the small rounds' form
    Fe<L> pf;
#pragma unroll
    for (int w = 0; w < L; w++) pf.w[w] = f.p[w];
    const size_t len = fold ? src_len / 2 : src_len, half = len / 2;
    const uint32_t sub = threadIdx.x % kScSub;
    const size_t b = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) / kScSub;
    uint64_t ev[D + 1][L];
    sc_pair<L, D, kScSub, kScSub == kScSubMax>(src, src_len, dst, fold, r, K, c, f, pf, b, b < half,
                                                sub, ev);
    // warp tree reduction, then across the block's warps
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll kUT
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll kUT
        for (int t = 0; t <= D; t++) {
            uint64_t o[L];
#pragma unroll
            for (int w = 0; w < L; w++) o[w] = __shfl_down_sync(0xffffffffu, ev[t][w], off);
            fadd<L>(ev[t], o, f.p);
        }
    }
    if (lane == 0)
#pragma unroll kUT
        for (int t = 0; t <= D; t++)
#pragma unroll
            for (int w = 0; w < L; w++) red[warp][t * L + w] = ev[t][w];
    __syncthreads();
    if (warp == 0) {
        const uint32_t nw = blockDim.x / 32;
#pragma unroll kUT
        for (int t = 0; t <= D; t++)
#pragma unroll
            for (int w = 0; w < L; w++) ev[t][w] = lane < nw ? red[lane][t * L + w] : 0;
#pragma unroll kUT
        for (int off = 16; off > 0; off >>= 1) {
#pragma unroll kUT
            for (int t = 0; t <= D; t++) {
                uint64_t o[L];
#pragma unroll
                for (int w = 0; w < L; w++) o[w] = __shfl_down_sync(0xffffffffu, ev[t][w], off);
                fadd<L>(ev[t], o, f.p);
            }
        }
        if (lane == 0)
#pragma unroll kUT
            for (int t = 0; t <= D; t++)
#pragma unroll
                for (int w = 0; w < L; w++) partials[((size_t)blockIdx.x * (D + 1) + t) * L + w] = ev[t][w];
    }
}

template <int L>
zg_status launch_round(zg_ctx *ctx, int D, int sub, const uint64_t *src, size_t src_len,
                       uint64_t *dst, bool fold, const uint64_t *r, uint32_t K, const ScComb &c,
                       const FieldCfg &f, uint64_t *partials, unsigned blocks, cudaStream_t s) {
    ZG_KBEGIN(ctx, s, "k_sc_round");
#define ZG_SC_CASE(DV)                                                                            \
    case DV:                                                                                      \
        if (sub == 1)                                                                             \
            k_sc_round<L, DV, 1><<<blocks, kScThreads, 0, s>>>(src, src_len, dst, fold ? 1 : 0, r, \
                                                               K, c, f, partials);                \
        else if (sub == kScSubMid)                                                                \
            k_sc_round<L, DV, kScSubMid><<<blocks, kScThreads, 0, s>>>(src, src_len, dst,         \
                                                                       fold ? 1 : 0, r, K, c, f,  \
                                                                       partials);                 \
        else                                                                                      \
            k_sc_round<L, DV, kScSubMax><<<blocks, kScThreads, 0, s>>>(src, src_len, dst,         \
                                                                       fold ? 1 : 0, r, K, c, f,  \
                                                                       partials);                 \
        break;
    switch (D) {
        ZG_SC_CASE(0)
        ZG_SC_CASE(1)
        ZG_SC_CASE(2)
        ZG_SC_CASE(3)
        ZG_SC_CASE(4)
        ZG_SC_CASE(5)
        ZG_SC_CASE(6)
        ZG_SC_CASE(7)
        ZG_SC_CASE(8)
        default:
            set_error("sumcheck degree %d above %d", D, kScMaxDeg);
            return ZG_ERR_INVALID_PARAM;
    }
#undef ZG_SC_CASE
    ZG_KEND(ctx, s);
    return ZG_OK;
}

template <int L>
zg_status launch_fold(zg_ctx *ctx, const uint64_t *in, uint64_t *out, uint32_t K, size_t n_out,
                      const uint64_t *r, const FieldCfg &f, cudaStream_t s) {
    const size_t total = (size_t)K * n_out;
    ZG_KBEGIN(ctx, s, "k_sc_fold");
    k_sc_fold<L><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(in, out, K, n_out, r, f);
    ZG_KEND(ctx, s);
    return ZG_OK;
}

// Fiat-Shamir on the device: after each round's kernels, one block sums the
// block partials of every group into the round's evaluations and its first
// thread runs the transcript step on a device copy of the Blake3 hasher (the
// reference's order, piop/src/sumcheck.rs:180-199 and multi_degree.rs:300-340:
// absorb the round messages, squeeze the challenge, absorb it).  The challenge
// stays in device memory for the next round's fold, so the rounds run back to
// back with no host round trip; the hasher state, messages and point come back
// once at the end.
constexpr uint32_t kScMaxGroups = 8;
struct FsArgs {
    b3::Hasher *h;
    const uint64_t *partials[kScMaxGroups];
    uint32_t degree[kScMaxGroups];
    uint32_t ng, multi, blocks, rd, maxd, nvars;
    uint64_t *msgs;     // [g][round][maxd + 1][L]: evaluations 1..deg of each round
    uint64_t *claimed;  // [g][L]: P_0(0) + P_0(1)
    uint64_t *r;        // this round's challenge, read by the next fold
    uint64_t *point;    // [round][L]
};

// Byte j of absorb_random_field's encoding of `inner` (transcript/src/
// traits.rs:393-413): 0x03 | modulus | 0x05 | 0x01 | inner | 0x03, 16L + 4 bytes.
template <int L>
__device__ __forceinline__ uint8_t field_byte(const FieldCfg &f, const uint64_t *inner, uint32_t j) {
    if (j == 0 || j == 16 * L + 3) return 3;
    if (j <= 8 * L) {
        const uint32_t k = j - 1;
        return (uint8_t)(f.p[k >> 3] >> (8 * (k & 7)));
    }
    if (j == 8 * L + 1) return 5;
    if (j == 8 * L + 2) return 1;
    const uint32_t k = j - 8 * L - 3;
    return (uint8_t)(inner[k >> 3] >> (8 * (k & 7)));
}

// Hasher::update by one warp on a hasher in shared memory: lane 0 takes the
// block and chunk boundaries (the compressions), the lanes copy the bytes.  The
// same state changes as the one-thread update, so the same transcript; one
// thread copying byte by byte was most of a round's transcript time.
__device__ void warp_update(b3::Hasher *h, const uint8_t *in, uint32_t n) {
    const uint32_t lane = threadIdx.x & 31;
    while (n) {
        if (lane == 0) {
            if (h->chunk_len() == b3::CHUNK_LEN) h->finish_chunk_and_push();
            if (h->block_len == 64) {
                uint32_t m[16];
                h->block_words(m);
                b3::compress_cv_h(h->cv, m, h->chunk_counter, 64, h->start_flag());
                h->blocks_compressed++;
                h->block_len = 0;
                h->clear_block();
            }
        }
        __syncwarp();
        const uint32_t bl = h->block_len;
        const uint32_t take = n < 64 - bl ? n : 64 - bl;
        for (uint32_t i = lane; i < take; i += 32) h->block[bl + i] = in[i];
        __syncwarp();
        if (lane == 0) h->block_len = bl + take;
        __syncwarp();
        in += take;
        n -= take;
    }
}

// Hasher::xof for the first 8L output bytes, as L little-endian words.
template <int L>
__device__ void xof_words(const b3::Hasher *h, uint64_t *x) {
    uint32_t ocv[8], m[16];
    uint32_t blen = h->block_len, flags = h->start_flag() | b3::CHUNK_END;
    uint64_t counter = h->chunk_counter;
    for (int i = 0; i < 8; i++) ocv[i] = h->cv[i];
    h->block_words(m);
    for (int s = (int)h->stack_len - 1; s >= 0; s--) {
        uint32_t c[8];
        for (int i = 0; i < 8; i++) c[i] = ocv[i];
        b3::compress_cv_h(c, m, counter, blen, flags);
        for (int i = 0; i < 8; i++) {
            m[i] = h->stack[s][i];
            m[8 + i] = c[i];
            ocv[i] = b3::iv(i);
        }
        counter = 0;
        blen = 64;
        flags = b3::PARENT;
    }
    uint32_t w[16];
    b3::compress_h(ocv, m, 0, blen, flags | b3::ROOT, w);
    for (int j = 0; j < L; j++) x[j] = (uint64_t)w[2 * j] | ((uint64_t)w[2 * j + 1] << 32);
}

// Bytes of the transcript step of one round: every round message, the squeeze
// and the challenge, at most kScMaxGroups x kScMaxDeg field elements.
constexpr uint32_t kFsBufBytes = kScMaxGroups * kScMaxDeg * (16 * 4 + 4) + 128;

// Block-cooperative copy of a hasher (global <-> shared memory).  The
// transcript step runs on a shared-memory copy.
__device__ __forceinline__ void hasher_copy(b3::Hasher *dst, const b3::Hasher *src) {
    static_assert(sizeof(b3::Hasher) % 8 == 0, "hasher size");
    const uint64_t *s = reinterpret_cast<const uint64_t *>(src);
    uint64_t *d = reinterpret_cast<uint64_t *>(dst);
    for (uint32_t i = threadIdx.x; i < sizeof(b3::Hasher) / 8; i += blockDim.x) d[i] = s[i];
}

// One round's transcript step, by one warp (all 32 lanes call it), in the
// reference's order (piop/src/sumcheck.rs:180-199, multi_degree.rs:300-340):
// the round-0 claimed sums are kept, the round messages P(1..deg) stored and
// absorbed (MLSumcheck: its one group's; MultiDegreeSumcheck: every group's in
// group order, the same byte sequence), the challenge squeezed
// (get_field_challenge: XOF of 8L bytes absorbed as 0x12 | bytes | 0x34, read
// as an integer and put into Montgomery form) and absorbed.  The challenge goes
// to r_out[0..L) and point[rd].  buf: kFsBufBytes of shared memory.
template <int L>
__device__ void fs_round(b3::Hasher *h, const FieldCfg &f, const uint64_t (*ev)[kScMaxDeg + 1][L],
                         const uint32_t *degree, uint32_t ng, uint32_t multi, uint32_t rd,
                         uint32_t maxd, uint32_t nvars, uint64_t *msgs, uint64_t *claimed,
                         uint64_t *point, uint64_t *r_out, uint8_t *buf) {
    const uint32_t lane = threadIdx.x & 31;
    constexpr uint32_t FB = 16 * L + 4;
    (void)multi;
    if (lane == 0)
        for (uint32_t g = 0; g < ng; g++) {
            const uint32_t D = degree[g];
            if (rd == 0) {
                uint64_t c[L];
#pragma unroll
                for (int w = 0; w < L; w++) c[w] = ev[g][0][w];
                if (D > 0) fadd<L>(c, ev[g][1], f.p);
#pragma unroll
                for (int w = 0; w < L; w++) claimed[(size_t)g * L + w] = c[w];
            }
            uint64_t *m = msgs + (((size_t)g * nvars + rd) * (maxd + 1)) * L;
            for (uint32_t e = 1; e <= D; e++)
#pragma unroll
                for (int w = 0; w < L; w++) m[(size_t)(e - 1) * L + w] = ev[g][e][w];
        }
    uint32_t n = 0;
    for (uint32_t g = 0; g < ng; g++)
        for (uint32_t e = 1; e <= degree[g]; e++) {
            for (uint32_t j = lane; j < FB; j += 32) buf[n + j] = field_byte<L>(f, ev[g][e], j);
            n += FB;
        }
    __syncwarp();
    warp_update(h, buf, n);
    uint64_t *xs = reinterpret_cast<uint64_t *>(buf + kFsBufBytes - 128), *rs = xs + 4;
    if (lane == 0) xof_words<L>(h, xs);
    __syncwarp();
    for (uint32_t j = lane; j < 8 * L + 2; j += 32)
        buf[j] = j == 0 ? 0x12 : j == 8 * L + 1 ? 0x34 : (uint8_t)(xs[(j - 1) >> 3] >> (8 * ((j - 1) & 7)));
    __syncwarp();
    warp_update(h, buf, 8 * L + 2);
    if (lane == 0) {
        uint64_t x[L], r[L];
#pragma unroll
        for (int w = 0; w < L; w++) x[w] = xs[w];
        fmul<L>(x, f.r2, f.p, f.n0, r);
#pragma unroll
        for (int w = 0; w < L; w++) {
            rs[w] = r[w];
            r_out[w] = r[w];
            point[(size_t)rd * L + w] = r[w];
        }
    }
    __syncwarp();
    for (uint32_t j = lane; j < FB; j += 32) buf[j] = field_byte<L>(f, rs, j);
    __syncwarp();
    warp_update(h, buf, FB);
}

template <int L>
__global__ void __launch_bounds__(256) k_sc_fs(FsArgs a, FieldCfg f) {
    __shared__ uint64_t ev[kScMaxGroups][kScMaxDeg + 1][L];
    __shared__ __align__(16) uint8_t hbuf[sizeof(b3::Hasher)];
    __shared__ __align__(16) uint8_t fsbuf[kFsBufBytes];
    b3::Hasher *h = reinterpret_cast<b3::Hasher *>(hbuf);
    hasher_copy(h, a.h);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x / 32;
    // warp w sums the block partials of evaluations t = w, w + nwarps, ...
    for (uint32_t g = 0; g < a.ng; g++) {
        const uint32_t D = a.degree[g];
        for (uint32_t t = warp; t <= D; t += nwarps) {
            uint64_t acc[L] = {};
            for (uint32_t bk = lane; bk < a.blocks; bk += 32)
                fadd<L>(acc, a.partials[g] + ((size_t)bk * (D + 1) + t) * L, f.p);
            for (int off = 16; off > 0; off >>= 1) {
                uint64_t o[L];
#pragma unroll
                for (int w = 0; w < L; w++) o[w] = __shfl_down_sync(0xffffffffu, acc[w], off);
                fadd<L>(acc, o, f.p);
            }
            if (lane == 0)
#pragma unroll
                for (int w = 0; w < L; w++) ev[g][t][w] = acc[w];
        }
    }
    __syncthreads();
    if (warp == 0)
        fs_round<L>(h, f, ev, a.degree, a.ng, a.multi, a.rd, a.maxd, a.nvars, a.msgs, a.claimed,
                    a.point, a.r, fsbuf);
    __syncthreads();
    hasher_copy(a.h, h);
}

// Per-group device state, carved out of the context's sumcheck arena.
struct GroupDev {
    uint32_t degree = 0, K = 0;
    const uint64_t *in = nullptr;  // round-0 MLEs (the caller's device memory, or a staged copy)
    uint64_t *buf[2] = {nullptr, nullptr};  // folded MLEs, alternating by round parity
    uint64_t *partials = nullptr;
    ScComb comb{};
};

// get_field_challenge (transcript/src/traits.rs:337-341): XOF of the inner's
// byte length read as an integer and converted to Montgomery form.
template <int L>
void field_challenge(zg_transcript *t, uint64_t *out) {
    const FieldCfg &f = t->f;
    uint8_t b[8 * L];
    tr_challenge(t, b, 8 * L);
    uint64_t x[L];
    std::memcpy(x, b, 8 * L);
    fmul<L>(x, f.r2, f.p, f.n0, out);
}

template <int L>
void f_from_u64_host(const FieldCfg &f, uint64_t v, uint64_t *out) {
    const uint64_t x[2] = {v, 0};
    from_signed<L>(x, 2, f, out);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }


template <int L>
zg_status sumcheck_prove_t(zg_ctx *ctx, zg_transcript *t, uint32_t nvars, int multi,
                           const zg_sumcheck_group *groups, uint32_t ng, int on_device,
                           uint8_t *proof, size_t *proof_len, uint64_t *point_out,
                           uint64_t *finals_out) {
    const FieldCfg &f = t->f;
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << nvars;
    const size_t fb = 8 * L;
    // proof size and validation
    size_t need = fb + (multi ? 8 + 4 * (size_t)ng : 4) + fb * ng;
    uint32_t maxd = 0;
    for (uint32_t g = 0; g < ng; g++) {
        const zg_sumcheck_group &G = groups[g];
        if (G.degree > kScMaxDeg || G.n_mles == 0 || (G.n_products && (!G.coeffs || !G.offsets ||
                                                                     !G.indices)) ||
            (G.n_factors && (!G.factor_mles || !G.factor_a || !G.factor_b)) || !G.mles) {
            set_error("sumcheck group %u: degree %u (max %d), no MLEs or missing arrays", g, G.degree,
                      kScMaxDeg);
            return ZG_ERR_INVALID_PARAM;
        }
        for (uint32_t k = 0; k < G.n_products; k++)
            for (uint32_t q = G.offsets[k]; q < G.offsets[k + 1]; q++)
                if (G.indices[q] >= G.n_mles) {
                    set_error("sumcheck group %u: product %u uses MLE %u of %u", g, k, G.indices[q],
                              G.n_mles);
                    return ZG_ERR_INVALID_PARAM;
                }
        for (uint32_t q = 0; q < G.n_factors; q++)
            if (G.factor_mles[q] >= G.n_mles) {
                set_error("sumcheck group %u: factor %u uses MLE %u of %u", g, q, G.factor_mles[q],
                          G.n_mles);
                return ZG_ERR_INVALID_PARAM;
            }
        need += (size_t)nvars * (fb * G.degree + (multi ? 0 : 4));
        maxd = std::max(maxd, G.degree);
    }
    if (*proof_len < need) {
        *proof_len = need;
        set_error("sumcheck proof buffer too small (%zu bytes needed)", need);
        return ZG_ERR_BUFFER_TOO_SMALL;
    }
    // arena: per group [staged input][fold buffers][comb][partials], then r
    // threads per pair in a round with `pairs` pairs, and that round's blocks
    auto sub_of = [](size_t pairs) {
        return pairs >= kScSplitBelow ? 1 : pairs >= kScSplitMore ? kScSubMid : kScSubMax;
    };
    auto blocks_of = [&](size_t pairs) {
        return (unsigned)std::max<size_t>(1, (pairs * sub_of(pairs) + kScThreads - 1) / kScThreads);
    };
    unsigned max_blocks = 1;
    for (size_t pairs = n / 2; pairs >= 1; pairs /= 2) max_blocks = std::max(max_blocks, blocks_of(pairs));
    std::vector<size_t> off_in(ng), off_b0(ng), off_b1(ng), off_meta(ng), off_part(ng);
    size_t total = 0;
    for (uint32_t g = 0; g < ng; g++) {
        const zg_sumcheck_group &G = groups[g];
        const size_t nidx = G.n_products ? G.offsets[G.n_products] : 0;
        off_in[g] = total;
        if (!on_device) total = align256(total + (size_t)G.n_mles * n * fb);
        off_b1[g] = total;  // rounds 1, 3, ...: K x n/2
        total = align256(total + (size_t)G.n_mles * std::max<size_t>(n / 2, 1) * fb);
        off_b0[g] = total;  // rounds 2, 4, ... and the final fold: K x max(n/4, 1)
        total = align256(total + (size_t)G.n_mles * std::max<size_t>(n / 4, 1) * fb);
        off_meta[g] = total;
        total = align256(total + (size_t)G.n_products * fb + 4 * ((size_t)G.n_products + 1) +
                         4 * nidx + 4 * (size_t)G.n_factors + 2 * fb * G.n_factors + 64);
        off_part[g] = total;
        total = align256(total + (size_t)max_blocks * (G.degree + 1) * fb);
    }
    const size_t off_r = total;
    total += 256;
    if (ng > kScMaxGroups) {
        set_error("sumcheck: %u groups (at most %u)", ng, kScMaxGroups);
        return ZG_ERR_INVALID_PARAM;
    }
    // device Fiat-Shamir state: the hasher, the round messages, claimed sums, point
    const size_t off_h = total;
    total = align256(total + sizeof(b3::Hasher));
    const size_t off_msgs = total;
    total = align256(total + (size_t)ng * nvars * (maxd + 1) * fb);
    const size_t off_claimed = total;
    total = align256(total + (size_t)ng * fb);
    const size_t off_point = total;
    total = align256(total + (size_t)nvars * fb);
    ZG_TRY(ctx->sc_arena.ensure(total));
    ZG_TRY(ctx->pin_in.ensure(256));
    ZG_TRY(ctx->pin_out.ensure((size_t)ng * max_blocks * (maxd + 1) * fb));
    uint8_t *arena = ctx->sc_arena.as<uint8_t>();
    uint64_t *r_d = reinterpret_cast<uint64_t *>(arena + off_r);
    std::vector<GroupDev> gd(ng);
    for (uint32_t g = 0; g < ng; g++) {
        const zg_sumcheck_group &G = groups[g];
        GroupDev &D = gd[g];
        D.degree = G.degree;
        D.K = G.n_mles;
        if (on_device) {
            D.in = static_cast<const uint64_t *>(G.mles);
        } else {
            uint64_t *in = reinterpret_cast<uint64_t *>(arena + off_in[g]);
            ZG_CUDA(cudaMemcpyAsync(in, G.mles, (size_t)G.n_mles * n * fb, cudaMemcpyHostToDevice, s));
            D.in = in;
        }
        D.buf[1] = reinterpret_cast<uint64_t *>(arena + off_b1[g]);
        D.buf[0] = reinterpret_cast<uint64_t *>(arena + off_b0[g]);
        D.partials = reinterpret_cast<uint64_t *>(arena + off_part[g]);
        // comb metadata: coeffs | fa | fb | offsets | indices | fmles
        uint8_t *m = arena + off_meta[g];
        const size_t nidx = G.n_products ? G.offsets[G.n_products] : 0;
        uint64_t *cf = reinterpret_cast<uint64_t *>(m);
        uint64_t *fa = cf + (size_t)G.n_products * L, *fbv = fa + (size_t)G.n_factors * L;
        uint32_t *offs = reinterpret_cast<uint32_t *>(fbv + (size_t)G.n_factors * L);
        uint32_t *idx = offs + G.n_products + 1, *fm = idx + nidx;
        if (G.n_products) {
            ZG_CUDA(cudaMemcpyAsync(cf, G.coeffs, (size_t)G.n_products * fb, cudaMemcpyHostToDevice, s));
            ZG_CUDA(cudaMemcpyAsync(offs, G.offsets, 4 * ((size_t)G.n_products + 1), cudaMemcpyHostToDevice, s));
            ZG_CUDA(cudaMemcpyAsync(idx, G.indices, 4 * nidx, cudaMemcpyHostToDevice, s));
        }
        if (G.n_factors) {
            ZG_CUDA(cudaMemcpyAsync(fa, G.factor_a, (size_t)G.n_factors * fb, cudaMemcpyHostToDevice, s));
            ZG_CUDA(cudaMemcpyAsync(fbv, G.factor_b, (size_t)G.n_factors * fb, cudaMemcpyHostToDevice, s));
            ZG_CUDA(cudaMemcpyAsync(fm, G.factor_mles, 4 * (size_t)G.n_factors, cudaMemcpyHostToDevice, s));
        }
        D.comb = ScComb{cf, offs, idx, fm, fa, fbv, G.n_products, G.n_factors};
    }
    // transcript header
    uint64_t fe[4];
    f_from_u64_host<L>(f, nvars, fe);
    tr_absorb_field(t, fe);
    f_from_u64_host<L>(f, multi ? ng : groups[0].degree, fe);
    tr_absorb_field(t, fe);
    if (multi)
        for (uint32_t g = 0; g < ng; g++) {
            f_from_u64_host<L>(f, groups[g].degree, fe);
            tr_absorb_field(t, fe);
        }
    std::vector<uint64_t> msgs((size_t)ng * nvars * (maxd + 1) * L, 0), claimed((size_t)ng * L, 0);
    b3::Hasher *h_d = reinterpret_cast<b3::Hasher *>(arena + off_h);
    uint64_t *msgs_d = reinterpret_cast<uint64_t *>(arena + off_msgs);
    uint64_t *claimed_d = reinterpret_cast<uint64_t *>(arena + off_claimed);
    uint64_t *point_d = reinterpret_cast<uint64_t *>(arena + off_point);
    // the transcript moves to the device for the rounds (its state is a plain struct)
    ZG_TRY(ctx->pin_in.ensure(sizeof(b3::Hasher) + 256));
    std::memcpy(ctx->pin_in.as<uint8_t>(), &t->h, sizeof(b3::Hasher));
    ZG_CUDA(cudaMemcpyAsync(h_d, ctx->pin_in.as<uint8_t>(), sizeof(b3::Hasher), cudaMemcpyHostToDevice, s));
    std::vector<const uint64_t *> cur(ng);
    for (uint32_t g = 0; g < ng; g++) cur[g] = gd[g].in;
    size_t src_len = n;
    FsArgs fa{};
    fa.h = h_d;
    fa.ng = ng;
    fa.multi = multi ? 1 : 0;
    fa.maxd = maxd;
    fa.nvars = nvars;
    fa.msgs = msgs_d;
    fa.claimed = claimed_d;
    fa.r = r_d;
    fa.point = point_d;
    for (uint32_t g = 0; g < ng; g++) {
        fa.partials[g] = gd[g].partials;
        fa.degree[g] = gd[g].degree;
    }
    for (uint32_t rd = 0; rd < nvars; rd++) {
        const bool fold = rd > 0;
        const size_t len = fold ? src_len / 2 : src_len;
        const unsigned blocks = blocks_of(len / 2);
        for (uint32_t g = 0; g < ng; g++) {
            uint64_t *dst = gd[g].buf[rd & 1];
            ZG_TRY(launch_round<L>(ctx, (int)gd[g].degree, sub_of(len / 2), cur[g], src_len, dst, fold,
                                   r_d, gd[g].K, gd[g].comb, f, gd[g].partials, blocks, s));
            if (fold) cur[g] = dst;
        }
        fa.blocks = blocks;
        fa.rd = rd;
        ZG_KBEGIN(ctx, s, "k_sc_fs");
        k_sc_fs<L><<<1, 256, 0, s>>>(fa, f);
        ZG_KEND(ctx, s);
        src_len = len;
    }
    {
        // the transcript state, messages, claimed sums and point back to the host
        uint8_t *hp = ctx->pin_out.as<uint8_t>();
        const size_t mb = msgs.size() * 8, cb = claimed.size() * 8, pb = (size_t)nvars * fb;
        ZG_TRY(ctx->pin_out.ensure(sizeof(b3::Hasher) + mb + cb + pb + 256));
        hp = ctx->pin_out.as<uint8_t>();
        ZG_CUDA(cudaMemcpyAsync(hp, h_d, sizeof(b3::Hasher), cudaMemcpyDeviceToHost, s));
        ZG_CUDA(cudaMemcpyAsync(hp + sizeof(b3::Hasher), msgs_d, mb, cudaMemcpyDeviceToHost, s));
        ZG_CUDA(cudaMemcpyAsync(hp + sizeof(b3::Hasher) + mb, claimed_d, cb, cudaMemcpyDeviceToHost, s));
        ZG_CUDA(cudaMemcpyAsync(hp + sizeof(b3::Hasher) + mb + cb, point_d, pb, cudaMemcpyDeviceToHost, s));
        if (ctx_sync(ctx) != cudaSuccess) {
            set_error("sumcheck rounds failed: %s", cudaGetErrorString(cudaGetLastError()));
            return ZG_ERR_CUDA;
        }
        std::memcpy(&t->h, hp, sizeof(b3::Hasher));
        std::memcpy(msgs.data(), hp + sizeof(b3::Hasher), mb);
        std::memcpy(claimed.data(), hp + sizeof(b3::Hasher) + mb, cb);
        if (point_out) std::memcpy(point_out, hp + sizeof(b3::Hasher) + mb + cb, pb);
    }
    // final evaluations of every MLE at the point (the last fold)
    if (finals_out) {
        size_t fo = 0;
        for (uint32_t g = 0; g < ng; g++) {
            uint64_t *out = gd[g].buf[nvars & 1];
            ZG_TRY(launch_fold<L>(ctx, cur[g], out, gd[g].K, 1, r_d, f, s));
            ZG_CUDA(cudaMemcpyAsync(finals_out + fo * L, out, (size_t)gd[g].K * fb,
                                    cudaMemcpyDeviceToHost, s));
            fo += gd[g].K;
        }
    }
    if (ctx_sync(ctx) != cudaSuccess) {
        set_error("sumcheck final fold failed");
        return ZG_ERR_CUDA;
    }
    // transcription (SumcheckProof, sumcheck.rs:35-111; MultiDegreeSumcheckProof,
    // multi_degree.rs:86-190)
    size_t pos = 0;
    auto put = [&](const void *src, size_t nb) {
        std::memcpy(proof + pos, src, nb);
        pos += nb;
    };
    put(f.p, fb);
    if (!multi) {
        const uint32_t nm = nvars, Dg = groups[0].degree;
        put(&nm, 4);
        for (uint32_t rd = 0; rd < nvars; rd++) {
            put(&Dg, 4);
            put(&msgs[(size_t)rd * (maxd + 1) * L], fb * Dg);
        }
        put(&claimed[0], fb);
    } else {
        const uint32_t g32 = ng, nv32 = nvars;
        put(&g32, 4);
        put(&nv32, 4);
        for (uint32_t g = 0; g < ng; g++) put(&groups[g].degree, 4);
        for (uint32_t g = 0; g < ng; g++)
            for (uint32_t rd = 0; rd < nvars; rd++)
                put(&msgs[((size_t)g * nvars + rd) * (maxd + 1) * L], fb * groups[g].degree);
        put(claimed.data(), fb * ng);
    }
    *proof_len = pos;
    return ZG_OK;
}

// sum_x mle[x] * eq(x, point) (mle_eval_with_eq_table, poly/src/utils.rs:267-284)
template <int L>
__global__ void __launch_bounds__(256) k_mle_dot_eq(const uint64_t *__restrict__ mle,
                                                    const uint64_t *__restrict__ r,
                                                    const uint64_t *__restrict__ omr, uint32_t nv,
                                                    FieldCfg f, uint64_t *__restrict__ partials) {
    __shared__ uint64_t red[256][L];
    const size_t x = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t acc[L];
    for (int w = 0; w < L; w++) acc[w] = 0;
    if (x < ((size_t)1 << nv)) {
        uint64_t e[L];
        for (int w = 0; w < L; w++) e[w] = f.one[w];
        for (uint32_t k = 0; k < nv; k++) {
            const uint64_t *sel = ((x >> k) & 1) ? r + (size_t)k * L : omr + (size_t)k * L;
            uint64_t o[L];
            fmul<L>(e, sel, f.p, f.n0, o);
            for (int w = 0; w < L; w++) e[w] = o[w];
        }
        fmul<L>(e, mle + x * L, f.p, f.n0, acc);
    }
    for (int w = 0; w < L; w++) red[threadIdx.x][w] = acc[w];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) fadd<L>(red[threadIdx.x], red[threadIdx.x + h], f.p);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int w = 0; w < L; w++) partials[(size_t)blockIdx.x * L + w] = red[0][w];
}

template <int L>
zg_status mle_evaluate_t(zg_ctx *ctx, const FieldCfg &f, const uint64_t *mle, uint32_t nv,
                         const uint64_t *point, uint64_t *out) {
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)1 << nv, fb = 8 * L;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    std::vector<uint64_t> omr((size_t)std::max<uint32_t>(nv, 1) * L);
    for (uint32_t k = 0; k < nv; k++) {
        std::memcpy(&omr[(size_t)k * L], f.one, fb);
        fsub<L>(&omr[(size_t)k * L], point + (size_t)k * L, f.p);
    }
    DevBuf buf;
    const size_t bytes = n * fb + 2 * std::max<uint32_t>(nv, 1) * fb + blocks * fb;
    ZG_TRY(buf.ensure(bytes));
    uint64_t *m_d = buf.as<uint64_t>(), *r_d = m_d + n * L, *o_d = r_d + std::max<uint32_t>(nv, 1) * L;
    uint64_t *p_d = o_d + std::max<uint32_t>(nv, 1) * L;
    zg_status st = ZG_OK;
    if (cudaMemcpyAsync(m_d, mle, n * fb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(r_d, point, nv * fb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(o_d, omr.data(), nv * fb, cudaMemcpyHostToDevice, s) != cudaSuccess)
        st = ZG_ERR_CUDA;
    std::vector<uint64_t> hp((size_t)blocks * L);
    if (st == ZG_OK) {
        ZG_KBEGIN(ctx, s, "k_mle_dot_eq");
        k_mle_dot_eq<L><<<blocks, 256, 0, s>>>(m_d, r_d, o_d, nv, f, p_d);
        ktimer_end(ctx, s);
        ctx->launches++;
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(hp.data(), p_d, blocks * fb, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            st = ZG_ERR_CUDA;
    }
    buf.release();
    if (st != ZG_OK) {
        set_error("MLE evaluation failed");
        return st;
    }
    uint64_t acc[L];
    for (int w = 0; w < L; w++) acc[w] = 0;
    for (unsigned bk = 0; bk < blocks; bk++) fadd<L>(acc, &hp[(size_t)bk * L], f.p);
    std::memcpy(out, acc, fb);
    return ZG_OK;
}

}  // namespace
}  // namespace zg

using namespace zg;

static zg_status sumcheck_prove_impl(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus,
                                     uint32_t limbs, uint32_t nvars, int multi,
                                     const zg_sumcheck_group *groups, uint32_t ngroups,
                                     int on_device, uint8_t *proof, size_t *proof_len,
                                     uint64_t *point_out, uint64_t *finals_out) {
    if (!ctx || !t || !modulus || !groups || !proof || !proof_len || ngroups == 0 || limbs < 1 ||
        limbs > 4) {
        set_error("sumcheck: null argument, no groups or field limbs not in 1..4");
        return ZG_ERR_INVALID_PARAM;
    }
    if (nvars == 0 || nvars > 30) {
        // MLSumcheck::prove_as_subprotocol asserts num_vars > 0 ("Attempt to prove a constant.")
        set_error("Attempt to prove a constant (or more than 30 variables: %u)", nvars);
        return ZG_ERR_INVALID_PARAM;
    }
    if (!multi && ngroups != 1) {
        set_error("MLSumcheck takes exactly one group");
        return ZG_ERR_INVALID_PARAM;
    }
    uint64_t p[4] = {0, 0, 0, 0};
    std::memcpy(p, modulus, 8 * limbs);
    if (!(p[0] & 1)) {
        set_error("sumcheck: the modulus must be odd");
        return ZG_ERR_INVALID_PARAM;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    // Field elements absorbed from here on carry this modulus.
    field_cfg_init(t->f, p, (int)limbs);
    t->has_field = true;
    switch (limbs) {
        case 1:
            return sumcheck_prove_t<1>(ctx, t, nvars, multi, groups, ngroups, on_device, proof,
                                       proof_len, point_out, finals_out);
        case 2:
            return sumcheck_prove_t<2>(ctx, t, nvars, multi, groups, ngroups, on_device, proof,
                                       proof_len, point_out, finals_out);
        case 3:
            return sumcheck_prove_t<3>(ctx, t, nvars, multi, groups, ngroups, on_device, proof,
                                       proof_len, point_out, finals_out);
        default:
            return sumcheck_prove_t<4>(ctx, t, nvars, multi, groups, ngroups, on_device, proof,
                                       proof_len, point_out, finals_out);
    }
}

extern "C" zg_status zg_sumcheck_prove(zg_ctx *ctx, zg_transcript *t, const uint8_t *modulus,
                                       uint32_t limbs, uint32_t nvars, int multi,
                                       const zg_sumcheck_group *groups, uint32_t ngroups,
                                       int mles_on_device, uint8_t *proof, size_t *proof_len,
                                       uint64_t *point_out, uint64_t *finals_out) {
    try {
        return sumcheck_prove_impl(ctx, t, modulus, limbs, nvars, multi, groups, ngroups,
                                   mles_on_device, proof, proof_len, point_out, finals_out);
    } catch (...) {
        set_error("sumcheck: host allocation failed");
        return ZG_ERR_OOM;
    }
}

extern "C" zg_status zg_mle_evaluate(zg_ctx *ctx, const uint8_t *modulus, uint32_t limbs,
                                     const uint64_t *mle, uint32_t nvars, const uint64_t *point,
                                     uint64_t *out) {
    if (!ctx || !modulus || !mle || !point || !out || limbs < 1 || limbs > 4 || nvars > 30 ||
        !(modulus[0] & 1)) {
        set_error("MLE evaluation: null argument, field limbs not in 1..4, odd modulus required");
        return ZG_ERR_INVALID_PARAM;
    }
    try {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ZG_CUDA(cudaSetDevice(ctx->device));
        uint64_t p[4] = {0, 0, 0, 0};
        std::memcpy(p, modulus, 8 * limbs);
        FieldCfg f;
        field_cfg_init(f, p, (int)limbs);
        switch (limbs) {
            case 1: return mle_evaluate_t<1>(ctx, f, mle, nvars, point, out);
            case 2: return mle_evaluate_t<2>(ctx, f, mle, nvars, point, out);
            case 3: return mle_evaluate_t<3>(ctx, f, mle, nvars, point, out);
            default: return mle_evaluate_t<4>(ctx, f, mle, nvars, point, out);
        }
    } catch (...) {
        set_error("MLE evaluation: host allocation failed");
        return ZG_ERR_OOM;
    }
}
