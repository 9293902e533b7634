// PIOP sumcheck prover on the GPU (piop/src/sumcheck.rs:163-215,
// sumcheck/prover.rs:95-247, sumcheck/multi_degree.rs:259-355) for
// combination functions of the form
//   comb(v) = sum_k coeff_k * prod_{i in S_k} v_i,
// the form of the reference's test comb functions (sumcheck/tests/utils.rs:60-80);
// the BigLinear combined-polynomial comb_fn and the multipoint-evaluation
// product expand into it.  MLE values are field elements in Montgomery form
// (the reference's DenseMultilinearExtension<F::Inner>), layout [mle][x][limb].
//
// Round i evaluates P_i(t) = sum_b comb(v_b + t (w_b - v_b)) at t = 0..deg
// over the pairs (v_b, w_b) = (m[2b], m[2b+1]), then every MLE is folded at
// the challenge: m'[b] = m[2b] + r (m[2b+1] - m[2b]).  Field addition is exact,
// so the order of the sums is free.
#include <algorithm>
#include <cstring>
#include <memory>

#include "zg_internal.h"

namespace zg {
namespace {

constexpr int kScThreads = 128;
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

// One round polynomial: block-level partial sums of P(t), t = 0..D.
// Products: coeffs [n_products][L], offsets [n_products+1], indices.
template <int L, int D>
__global__ void __launch_bounds__(kScThreads) k_sc_eval(const uint64_t *__restrict__ m, size_t n,
                                                        const uint64_t *__restrict__ coeffs,
                                                        const uint32_t *__restrict__ offsets,
                                                        const uint32_t *__restrict__ indices,
                                                        uint32_t n_products, FieldCfg f,
                                                        uint64_t *__restrict__ partials) {
    __shared__ uint64_t red[kScThreads][(D + 1) * L];
    const size_t half = n / 2;
    const size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t ev[D + 1][L];
    for (int t = 0; t <= D; t++)
        for (int w = 0; w < L; w++) ev[t][w] = 0;
    if (b < half) {
        for (uint32_t k = 0; k < n_products; k++) {
            uint64_t pr[D + 1][L];
            for (int t = 0; t <= D; t++)
                for (int w = 0; w < L; w++) pr[t][w] = coeffs[(size_t)k * L + w];
            for (uint32_t q = offsets[k]; q < offsets[k + 1]; q++) {
                const uint64_t *v0 = m + ((size_t)indices[q] * n + 2 * b) * L, *v1 = v0 + L;
                uint64_t cur[L], st[L];
                for (int w = 0; w < L; w++) {
                    cur[w] = v0[w];
                    st[w] = v1[w];
                }
                fsub<L>(st, v0, f.p);
                for (int t = 0; t <= D; t++) {
                    uint64_t o[L];
                    fmul<L>(pr[t], cur, f.p, f.n0, o);
                    for (int w = 0; w < L; w++) pr[t][w] = o[w];
                    fadd<L>(cur, st, f.p);
                }
            }
            for (int t = 0; t <= D; t++) fadd<L>(ev[t], pr[t], f.p);
        }
    }
    for (int t = 0; t <= D; t++)
        for (int w = 0; w < L; w++) red[threadIdx.x][t * L + w] = ev[t][w];
    __syncthreads();
    for (int h = kScThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h)
            for (int t = 0; t <= D; t++) fadd<L>(&red[threadIdx.x][t * L], &red[threadIdx.x + h][t * L], f.p);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int e = 0; e < (D + 1) * L; e++) partials[(size_t)blockIdx.x * (D + 1) * L + e] = red[0][e];
}

template <int L>
zg_status launch_eval_d(zg_ctx *ctx, int D, const uint64_t *m, size_t n, const uint64_t *coeffs,
                        const uint32_t *offsets, const uint32_t *indices, uint32_t np,
                        const FieldCfg &f, uint64_t *partials, unsigned blocks, cudaStream_t s) {
    ZG_KBEGIN(ctx, s, "k_sc_eval");
#define ZG_SC_CASE(DV)                                                                            \
    case DV:                                                                                      \
        k_sc_eval<L, DV><<<blocks, kScThreads, 0, s>>>(m, n, coeffs, offsets, indices, np, f,     \
                                                       partials);                                 \
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

// Device allocations of one proof, released together.
struct DevAllocs {
    std::vector<void *> v;
    void *get(size_t bytes) {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
        v.push_back(p);
        return p;
    }
    ~DevAllocs() {
        for (void *p : v) cudaFree(p);
    }
};

struct GroupDev {
    uint32_t degree = 0, K = 0, np = 0;
    uint64_t *buf[2] = {nullptr, nullptr};  // ping-pong MLE arrays
    uint64_t *coeffs = nullptr;
    uint32_t *offsets = nullptr, *indices = nullptr;
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
    for (uint32_t g = 0; g < ng; g++) {
        if (groups[g].degree > kScMaxDeg || groups[g].n_mles == 0) {
            set_error("sumcheck group %u: degree %u (max %d) or no MLEs", g, groups[g].degree, kScMaxDeg);
            return ZG_ERR_INVALID_PARAM;
        }
        for (uint32_t k = 0; k < groups[g].n_products; k++)
            for (uint32_t q = groups[g].offsets[k]; q < groups[g].offsets[k + 1]; q++)
                if (groups[g].indices[q] >= groups[g].n_mles) {
                    set_error("sumcheck group %u: product %u uses MLE %u of %u", g, k,
                              groups[g].indices[q], groups[g].n_mles);
                    return ZG_ERR_INVALID_PARAM;
                }
        need += (size_t)nvars * (fb * groups[g].degree + (multi ? 0 : 4));
    }
    if (*proof_len < need) {
        *proof_len = need;
        set_error("sumcheck proof buffer too small (%zu bytes needed)", need);
        return ZG_ERR_BUFFER_TOO_SMALL;
    }
    // device state
    std::vector<GroupDev> gd(ng);
    DevAllocs allocs;
    auto dalloc = [&](size_t bytes) { return allocs.get(bytes); };
    uint32_t maxd = 0;
    for (uint32_t g = 0; g < ng; g++) {
        const zg_sumcheck_group &G = groups[g];
        GroupDev &D = gd[g];
        D.degree = G.degree;
        D.K = G.n_mles;
        D.np = G.n_products;
        maxd = std::max(maxd, G.degree);
        const size_t mbytes = (size_t)G.n_mles * n * fb;
        D.buf[0] = static_cast<uint64_t *>(dalloc(mbytes));
        D.buf[1] = static_cast<uint64_t *>(dalloc(mbytes / 2 + fb * G.n_mles));
        D.coeffs = static_cast<uint64_t *>(dalloc((size_t)G.n_products * fb));
        D.offsets = static_cast<uint32_t *>(dalloc(4 * ((size_t)G.n_products + 1)));
        const size_t nidx = G.n_products ? G.offsets[G.n_products] : 0;
        D.indices = static_cast<uint32_t *>(dalloc(4 * std::max<size_t>(nidx, 1)));
        if (!D.buf[0] || !D.buf[1] || !D.coeffs || !D.offsets || !D.indices) {
            set_error("sumcheck: device allocation failed");
            return ZG_ERR_OOM;
        }
        cudaMemcpyAsync(D.buf[0], G.mles, mbytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
        if (G.n_products) {
            cudaMemcpyAsync(D.coeffs, G.coeffs, (size_t)G.n_products * fb, cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(D.offsets, G.offsets, 4 * ((size_t)G.n_products + 1), cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(D.indices, G.indices, 4 * nidx, cudaMemcpyHostToDevice, s);
        }
    }
    const unsigned max_blocks = (unsigned)std::max<size_t>(1, (n / 2 + kScThreads - 1) / kScThreads);
    uint64_t *partials = static_cast<uint64_t *>(dalloc((size_t)ng * max_blocks * (maxd + 1) * fb));
    uint64_t *r_d = static_cast<uint64_t *>(dalloc(fb));
    if (!partials || !r_d) {
        set_error("sumcheck: device allocation failed");
        return ZG_ERR_OOM;
    }
    if (cudaGetLastError() != cudaSuccess) {
        set_error("sumcheck: upload failed");
        return ZG_ERR_CUDA;
    }
    std::vector<uint64_t> hpart((size_t)ng * max_blocks * (maxd + 1) * L);
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
    uint64_t r[4] = {0, 0, 0, 0};
    size_t len = n;
    int cur = 0;
    for (uint32_t rd = 0; rd < nvars; rd++) {
        if (rd > 0) {
            for (uint32_t g = 0; g < ng; g++) {
                zg_status st = launch_fold<L>(ctx, gd[g].buf[cur], gd[g].buf[cur ^ 1], gd[g].K, len / 2, r_d, f, s);
                if (st != ZG_OK) return st;
            }
            cur ^= 1;
            len /= 2;
        }
        const unsigned blocks = (unsigned)std::max<size_t>(1, (len / 2 + kScThreads - 1) / kScThreads);
        for (uint32_t g = 0; g < ng; g++) {
            zg_status st = launch_eval_d<L>(ctx, (int)gd[g].degree, gd[g].buf[cur], len, gd[g].coeffs,
                                            gd[g].offsets, gd[g].indices, gd[g].np, f,
                                            partials + (size_t)g * max_blocks * (maxd + 1) * L, blocks, s);
            if (st != ZG_OK) return st;
        }
        for (uint32_t g = 0; g < ng; g++)
            cudaMemcpyAsync(hpart.data() + (size_t)g * max_blocks * (maxd + 1) * L,
                            partials + (size_t)g * max_blocks * (maxd + 1) * L,
                            (size_t)blocks * (gd[g].degree + 1) * fb, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            set_error("sumcheck round %u failed: %s", rd, cudaGetErrorString(cudaGetLastError()));
            return ZG_ERR_CUDA;
        }
        for (uint32_t g = 0; g < ng; g++) {
            const uint32_t Dg = gd[g].degree;
            std::vector<uint64_t> ev((size_t)(Dg + 1) * L, 0);
            const uint64_t *hp = hpart.data() + (size_t)g * max_blocks * (maxd + 1) * L;
            for (unsigned bk = 0; bk < blocks; bk++)
                for (uint32_t tt = 0; tt <= Dg; tt++)
                    fadd<L>(&ev[(size_t)tt * L], hp + ((size_t)bk * (Dg + 1) + tt) * L, f.p);
            if (rd == 0) {
                std::memcpy(&claimed[(size_t)g * L], &ev[0], fb);
                if (Dg > 0) fadd<L>(&claimed[(size_t)g * L], &ev[L], f.p);
            }
            std::memcpy(&msgs[((size_t)g * nvars + rd) * (maxd + 1) * L], &ev[L], fb * Dg);
            if (!multi)
                for (uint32_t e = 1; e <= Dg; e++) tr_absorb_field(t, &ev[(size_t)e * L]);
        }
        if (multi)
            for (uint32_t g = 0; g < ng; g++)
                for (uint32_t e = 0; e < gd[g].degree; e++)
                    tr_absorb_field(t, &msgs[(((size_t)g * nvars + rd) * (maxd + 1) + e) * L]);
        field_challenge<L>(t, r);
        tr_absorb_field(t, r);
        if (point_out) std::memcpy(point_out + (size_t)rd * L, r, fb);
        cudaMemcpyAsync(r_d, r, fb, cudaMemcpyHostToDevice, s);
    }
    // final evaluations of every MLE at the point (the last fold)
    if (finals_out) {
        size_t fo = 0;
        for (uint32_t g = 0; g < ng; g++) {
            zg_status st = launch_fold<L>(ctx, gd[g].buf[cur], gd[g].buf[cur ^ 1], gd[g].K, 1, r_d, f, s);
            if (st != ZG_OK) return st;
            cudaMemcpyAsync(finals_out + fo * L, gd[g].buf[cur ^ 1], (size_t)gd[g].K * fb,
                            cudaMemcpyDeviceToHost, s);
            fo += gd[g].K;
        }
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) {
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
