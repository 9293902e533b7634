// LinearCode::encode_f (zip-plus/src/code.rs:69-71): a row of prime-field
// elements encoded over the field.
//
// IPRS (iprs.rs:88-106, encode_inner_f): the radix-8 pNTT of radix8.rs:21-161
// with every base-matrix entry and twiddle taken as F::from_with_cfg of its
// i64 value.  The two tables are converted to Montgomery form once per call
// (k_tab_to_field), then the base layer is one thread per codeword position
// (base_len products each) and each radix-8 stage one thread per butterfly
// column (its 8 outputs from 8 inputs, 7 products per output).
//
// RAA and sign-flipping RAA (raa.rs:93-127, raa_sign_flip.rs:31-69): repeat,
// permute, prefix sums, permute, prefix sums, with the sign flips of the
// sign-flipping code.  A gathered entry is negated when its source position is
// odd (the flip of the repeated row, then of the first accumulation, applied
// before the gather that reads them).  One block runs the whole codeword: each
// thread sums a contiguous chunk, the chunk totals are scanned in shared memory,
// and each chunk adds its offset.
#include "zg_internal.h"

namespace zg {
namespace {

// out[e] = F(src[e]) for n int32 table entries
template <int L>
__global__ void k_tab_to_field(const int32_t *__restrict__ src, size_t n, FieldCfg f, uint64_t *__restrict__ out) {
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        uint64_t v[L];
        from_i128<L>((i128)src[e], f, v);
#pragma unroll
        for (int w = 0; w < L; w++) out[e * L + w] = v[w];
    }
}

// Base layer: out[i] = row[o] + sum_{c >= 1} row[o + c 8^depth] * F(bm[i mod bd][c]),
// o = octet_reversal(i / bd).  fbm: [base_len][base_dim] (transposed, as d_bmT).
template <int L>
__global__ void __launch_bounds__(256) k_encode_f_base(const uint64_t *__restrict__ row,
                                                       const uint64_t *__restrict__ fbm, uint32_t bd, uint32_t bl,
                                                       uint32_t depth, uint32_t C, FieldCfg f,
                                                       uint64_t *__restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
        const uint32_t ch = i / bd, rb = i % bd;
        uint32_t oct = 0, x = ch;
        for (uint32_t k = 0; k < depth; k++) {
            oct = (oct << 3) | (x & 7u);
            x >>= 3;
        }
        uint64_t acc[L];
#pragma unroll
        for (int w = 0; w < L; w++) acc[w] = row[(size_t)oct * L + w];
        for (uint32_t c = 1; c < bl; c++) {
            uint64_t t[L];
            fmul<L>(row + ((size_t)oct + ((size_t)c << (3 * depth))) * L, fbm + ((size_t)c * bd + rb) * L, f.p,
                    f.n0, t);
            fadd<L>(acc, t, f.p);
        }
#pragma unroll
        for (int w = 0; w < L; w++) out[(size_t)i * L + w] = acc[w];
    }
}

// One radix-8 stage (combine_stages, radix8.rs:58-113): butterfly column i of
// every chunk of 8 * sub positions, y_r = x_0 + sum_{j >= 1} x_j F(tw[j - 1][(r j) mod 8][i]).
// ftw: this stage's [56][sub] twiddles, [(j - 1) * 8 + t][i] (as d_tw).
template <int L>
__global__ void __launch_bounds__(256) k_encode_f_stage(uint64_t *__restrict__ v, const uint64_t *__restrict__ ftw,
                                                        size_t sub, uint32_t C, FieldCfg f) {
    const size_t cols = (size_t)C / 8;  // (chunk, i) pairs
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < cols; e += (size_t)gridDim.x * blockDim.x) {
        const size_t blk = (e / sub) * 8 * sub, i = e % sub;
        uint64_t xs[8][L];
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
            for (int w = 0; w < L; w++) xs[j][w] = v[(blk + j * sub + i) * L + w];
        for (int r = 0; r < 8; r++) {
            uint64_t y[L];
#pragma unroll
            for (int w = 0; w < L; w++) y[w] = xs[0][w];
            for (int j = 1; j < 8; j++) {
                uint64_t t[L];
                fmul<L>(xs[j], ftw + ((size_t)((j - 1) * 8 + ((r * j) & 7)) * sub + i) * L, f.p, f.n0, t);
                fadd<L>(y, t, f.p);
            }
#pragma unroll
            for (int w = 0; w < L; w++) v[(blk + r * sub + i) * L + w] = y[w];
        }
    }
}

// In-place prefix sums of n field elements by one block (blockDim = 1024).
template <int L>
__device__ void block_prefix_sums(uint64_t *v, uint32_t n, const FieldCfg &f, uint64_t (*tot)[L]) {
    const uint32_t T = blockDim.x, t = threadIdx.x;
    const uint32_t per = (n + T - 1) / T, a = min(n, t * per), b = min(n, a + per);
    uint64_t run[L] = {};
    for (uint32_t i = a; i < b; i++) {
        fadd<L>(run, v + (size_t)i * L, f.p);
#pragma unroll
        for (int w = 0; w < L; w++) v[(size_t)i * L + w] = run[w];
    }
#pragma unroll
    for (int w = 0; w < L; w++) tot[t][w] = run[w];
    __syncthreads();
    // inclusive scan of the chunk totals (Hillis-Steele)
    for (uint32_t d = 1; d < T; d <<= 1) {
        uint64_t add[L] = {};
        if (t >= d)
#pragma unroll
            for (int w = 0; w < L; w++) add[w] = tot[t - d][w];
        __syncthreads();
        if (t >= d) fadd<L>(tot[t], add, f.p);
        __syncthreads();
    }
    if (t > 0)
        for (uint32_t i = a; i < b; i++) fadd<L>(v + (size_t)i * L, tot[t - 1], f.p);
    __syncthreads();
}

template <int L>
__global__ void __launch_bounds__(1024) k_raa_f(const uint64_t *__restrict__ row, const uint32_t *__restrict__ perm,
                                                uint32_t row_len, uint32_t C, int flip, FieldCfg f,
                                                uint64_t *__restrict__ tmp, uint64_t *__restrict__ out) {
    __shared__ uint64_t tot[1024][L];
    const uint32_t *p1 = perm, *p2 = perm + C;
    for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
        const uint32_t s = p1[i];
        uint64_t x[L];
#pragma unroll
        for (int w = 0; w < L; w++) x[w] = row[(size_t)(s % row_len) * L + w];
        if (flip && (s & 1u)) fneg<L>(x, f.p);
#pragma unroll
        for (int w = 0; w < L; w++) tmp[(size_t)i * L + w] = x[w];
    }
    __syncthreads();
    block_prefix_sums<L>(tmp, C, f, tot);
    for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
        const uint32_t s = p2[i];
        uint64_t x[L];
#pragma unroll
        for (int w = 0; w < L; w++) x[w] = tmp[(size_t)s * L + w];
        if (flip && (s & 1u)) fneg<L>(x, f.p);
#pragma unroll
        for (int w = 0; w < L; w++) out[(size_t)i * L + w] = x[w];
    }
    __syncthreads();
    block_prefix_sums<L>(out, C, f, tot);
}

template <int L>
zg_status encode_f_t(zg_params *p, zg_ctx *ctx, const FieldCfg &f, const uint64_t *row_d, uint64_t *out_d,
                     cudaStream_t s) {
    const zg_params_info &I = p->info;
    const uint32_t C = I.codeword_len;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((C + 255) / 256, (size_t)ctx->num_sms * 8));
    if (p->d.code_kind != ZG_CODE_IPRS) {
        ZG_TRY(ctx->piop_arena.ensure((size_t)C * L * 8 + 256));
        ZG_KBEGIN(ctx, s, "k_raa_f");
        k_raa_f<L><<<1, 1024, 0, s>>>(row_d, p->d_perm, I.row_len, C,
                                      p->d.code_kind == ZG_CODE_RAA_SIGN_FLIP ? 1 : 0, f,
                                      ctx->piop_arena.as<uint64_t>(), out_d);
        ZG_KEND(ctx, s);
        return ZG_OK;
    }
    const size_t nbm = (size_t)I.base_len * I.base_dim;
    size_t ntw = 0;
    for (uint32_t k = 0; k < I.depth; k++) ntw += (size_t)56 * ((size_t)I.base_dim << (3 * k));
    ZG_TRY(ctx->piop_arena.ensure((nbm + ntw) * L * 8 + 256));
    uint64_t *fbm = ctx->piop_arena.as<uint64_t>(), *ftw = fbm + nbm * L;
    ZG_KBEGIN(ctx, s, "k_tab_to_field");
    k_tab_to_field<L><<<grid, 256, 0, s>>>(p->d_bmT, nbm, f, fbm);
    k_tab_to_field<L><<<grid, 256, 0, s>>>(p->d_tw, ntw, f, ftw);
    ZG_KEND(ctx, s);
    ZG_KBEGIN(ctx, s, "k_encode_f_base");
    k_encode_f_base<L><<<grid, 256, 0, s>>>(row_d, fbm, I.base_dim, I.base_len, I.depth, C, f, out_d);
    ZG_KEND(ctx, s);
    for (uint32_t k = 0; k < I.depth; k++) {
        const size_t sub = (size_t)I.base_dim << (3 * k);
        ZG_KBEGIN(ctx, s, "k_encode_f_stage");
        k_encode_f_stage<L><<<grid, 256, 0, s>>>(out_d, ftw + p->tw_dev_off[k] * L, sub, C, f);
        ZG_KEND(ctx, s);
    }
    return ZG_OK;
}

zg_status encode_f_impl(zg_params *p, const uint8_t *modulus, uint32_t limbs, const uint64_t *row, uint64_t *out,
                        bool on_device, cudaStream_t stream) {
    if (!p || !modulus || !row || !out) {
        set_error("encode_f: null argument");
        return ZG_ERR_INVALID_PARAM;
    }
    if (limbs < 1 || limbs > MAX_FIELD_LIMBS) {
        set_error("encode_f: field of %u limbs (1 to %d)", limbs, MAX_FIELD_LIMBS);
        return ZG_ERR_INVALID_PARAM;
    }
    uint64_t pm[MAX_FIELD_LIMBS] = {};
    std::memcpy(pm, modulus, 8 * limbs);
    if (!(pm[0] & 1) || (limbs > 1 && pm[limbs - 1] == 0)) {
        set_error("encode_f: the modulus must be odd and use its top limb");
        return ZG_ERR_INVALID_PARAM;
    }
    if (!p->ctx) {
        set_error("parameters were created without a device context");
        return ZG_ERR_NO_DEVICE;
    }
    if (p->d.code_kind == ZG_CODE_IPRS && (!p->d_bmT || !p->d_tw)) {
        set_error("encode_f: the parameters have no device tables");
        return ZG_ERR_INVALID_PARAM;
    }
    zg_ctx *ctx = p->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ZG_CUDA(cudaSetDevice(ctx->device));
    FieldCfg f;
    field_cfg_init(f, pm, (int)limbs);
    const zg_params_info &I = p->info;
    const size_t in_b = (size_t)I.row_len * limbs * 8, out_b = (size_t)I.codeword_len * limbs * 8;
    cudaStream_t s = stream ? stream : ctx->stream;
    const uint64_t *row_d = row;
    uint64_t *out_d = out;
    if (!on_device) {
        ZG_TRY(ctx->prove_in.ensure(in_b + out_b + 256));
        uint64_t *base = ctx->prove_in.as<uint64_t>();
        ZG_CUDA(cudaMemcpyAsync(base, row, in_b, cudaMemcpyHostToDevice, s));
        row_d = base;
        out_d = base + in_b / 8;
    }
    zg_status st;
    switch (limbs) {
        case 1: st = encode_f_t<1>(p, ctx, f, row_d, out_d, s); break;
        case 2: st = encode_f_t<2>(p, ctx, f, row_d, out_d, s); break;
        case 3: st = encode_f_t<3>(p, ctx, f, row_d, out_d, s); break;
        default: st = encode_f_t<4>(p, ctx, f, row_d, out_d, s); break;
    }
    ZG_TRY(st);
    if (!on_device) {
        ZG_CUDA(cudaMemcpyAsync(out, out_d, out_b, cudaMemcpyDeviceToHost, s));
        ZG_CUDA(cudaStreamSynchronize(s));
    }
    ZG_CUDA(cudaGetLastError());
    return ZG_OK;
}

}  // namespace
}  // namespace zg

using namespace zg;

extern "C" zg_status zg_encode_f(zg_params *p, const uint8_t *modulus, uint32_t limbs, const uint64_t *row,
                                 uint64_t *out) {
    try {
        return encode_f_impl(p, modulus, limbs, row, out, false, nullptr);
    } catch (const std::exception &e) {
        set_error("encode_f: %s", e.what());
        return ZG_ERR_OOM;
    }
}

extern "C" zg_status zg_encode_f_d(zg_params *p, const uint8_t *modulus, uint32_t limbs, const uint64_t *row_d,
                                   uint64_t *out_d, void *stream) {
    try {
        return encode_f_impl(p, modulus, limbs, row_d, out_d, true, static_cast<cudaStream_t>(stream));
    } catch (const std::exception &e) {
        set_error("encode_f: %s", e.what());
        return ZG_ERR_OOM;
    }
}
