// Zinc+ prover, MLE-first, for linear UAIRs: steps 0-7 on one transcript and
// the Proof wire format (protocol/src/prover.rs:218-706, protocol/src/lib.rs:
// 62-189).  Every step runs on the GPU through the entry points of api.cu and
// piop.cu; this file holds the sequencing, the host-side Fiat-Shamir glue
// between the steps and the byte layout of the proof.
#include <algorithm>
#include <cstring>
#include <vector>

#include "zg_internal.h"

using namespace zg;

namespace {

// F::from_with_cfg(i128) into a Montgomery inner
void f_from_i128(const FieldCfg &f, i128 v, uint64_t *out) {
    if (f.L == 3) from_i128<3>(v, f, out);
    else from_i128<4>(v, f, out);
}

// Growable little-endian byte writer for the proof transcription.
struct Bytes {
    std::vector<uint8_t> b;
    void put(const void *p, size_t n) {
        const uint8_t *q = static_cast<const uint8_t *>(p);
        b.insert(b.end(), q, q + n);
    }
    void u32(uint32_t v) { put(&v, 4); }
    // write_transcription_bytes_subset of a Transcribable with a u32 length
    // prefix (transcript/src/traits.rs:48-75): the byte length, then the bytes.
    void sub(const Bytes &x) {
        u32((uint32_t)x.b.size());
        put(x.b.data(), x.b.size());
    }
};

// DynamicPolyVecF (poly/src/univariate/dynamic/over_field.rs:409-476): nothing
// for an empty vector; else a flag byte (1 when some polynomial has a
// coefficient, followed by the modulus), then per polynomial its u32 length and
// its coefficients' inners.  Polynomials arrive trimmed.
Bytes poly_vec(const std::vector<std::vector<uint64_t>> &polys, const uint64_t *p, int L) {
    Bytes o;
    if (polys.empty()) return o;
    bool any = false;
    for (const auto &q : polys) any |= !q.empty();
    o.b.push_back(any ? 1 : 0);
    if (any) o.put(p, 8 * (size_t)L);
    for (const auto &q : polys) {
        o.u32((uint32_t)(q.size() / L));
        o.put(q.data(), q.size() * 8);
    }
    return o;
}

// Vec<F> (transcript/src/traits.rs:566-607): nothing when empty, else the
// modulus and the inners.
Bytes field_vec(const uint64_t *v, size_t n, const uint64_t *p, int L) {
    Bytes o;
    if (n == 0) return o;
    o.put(p, 8 * (size_t)L);
    o.put(v, n * 8 * (size_t)L);
    return o;
}

// new_trimmed: drop trailing zero coefficients.
std::vector<uint64_t> trimmed(const uint64_t *c, size_t n, int L) {
    while (n > 0) {
        bool zero = true;
        for (int w = 0; w < L; w++) zero &= c[(n - 1) * L + w] == 0;
        if (!zero) break;
        n--;
    }
    return std::vector<uint64_t>(c, c + n * L);
}

struct HintGuard {
    zg_hint *h = nullptr;
    ~HintGuard() {
        if (h) zg_hint_free(h);
    }
};
// The PCS stream of a proof is megabytes; the transcript borrows one buffer per
// thread across calls so that its pages stay mapped (no first-touch faults).
thread_local std::vector<uint8_t> t_stream_store;

struct TranscriptGuard {
    zg_transcript *t = nullptr;
    ~TranscriptGuard() {
        if (!t) return;
        t->stream.clear();
        t_stream_store.swap(t->stream);
        zg_transcript_free(t);
    }
};

// A UAIR as the driver takes it: the linear part of every constraint as a
// coefficient matrix over [binary up, integer up, down] (single-column terms),
// the terms that multiply two columns, and which constraints lie in the zero
// ideal (the combined path skips those in the ideal check).
struct UairRep {
    uint32_t n_bin = 0, n_int = 0, degree_plus_one = 0, n_shifts = 0;
    const uint32_t *shift_src = nullptr, *shift_amount = nullptr;
    uint32_t n_constraints = 0;
    const int64_t *coeffs = nullptr;  // n_constraints x (n_bin + n_int + n_shifts)
    uint32_t n_pub_bin = 0, n_pub_int = 0;
    std::vector<int64_t> coeff_store;
    std::vector<CprProduct> products;
    std::vector<uint8_t> zero_ideal;
};

UairRep rep_of(const zg_linear_uair *u) {
    UairRep r;
    r.n_bin = u->n_bin;
    r.n_int = u->n_int;
    r.degree_plus_one = u->degree_plus_one;
    r.n_shifts = u->n_shifts;
    r.shift_src = u->shift_src;
    r.shift_amount = u->shift_amount;
    r.n_constraints = u->n_constraints;
    r.coeffs = u->coeffs;
    r.n_pub_bin = u->n_pub_bin;
    r.n_pub_int = u->n_pub_int;
    r.zero_ideal.assign(u->n_constraints, 0);
    return r;
}

// The term form (zg_uair) split into the linear matrix and the products.
zg_status rep_of(const zg_uair *u, UairRep &r) {
    if (!u->term_offsets || !u->term_coeffs || !u->factor_offsets || (u->n_constraints && !u->zero_ideal)) {
        set_error("zinc prove: null term arrays");
        return ZG_ERR_INVALID_PARAM;
    }
    r.n_bin = u->n_bin;
    r.n_int = u->n_int;
    r.degree_plus_one = u->degree_plus_one;
    r.n_shifts = u->n_shifts;
    r.shift_src = u->shift_src;
    r.shift_amount = u->shift_amount;
    r.n_constraints = u->n_constraints;
    r.n_pub_bin = u->n_pub_bin;
    r.n_pub_int = u->n_pub_int;
    const uint32_t W = u->n_bin + u->n_int + u->n_shifts;
    r.coeff_store.assign((size_t)u->n_constraints * W, 0);
    r.zero_ideal.assign(u->zero_ideal, u->zero_ideal + u->n_constraints);
    if (u->term_offsets[0] != 0) {
        set_error("zinc prove: term offsets must start at 0");
        return ZG_ERR_INVALID_PARAM;
    }
    for (uint32_t k = 0; k < u->n_constraints; k++) {
        if (u->term_offsets[k + 1] < u->term_offsets[k]) {
            set_error("zinc prove: term offsets of constraint %u decrease", k);
            return ZG_ERR_INVALID_PARAM;
        }
        for (uint32_t t = u->term_offsets[k]; t < u->term_offsets[k + 1]; t++) {
            const uint32_t f0 = u->factor_offsets[t], f1 = u->factor_offsets[t + 1];
            if (f1 < f0 || (f1 > f0 && !u->factor_cols)) {
                set_error("zinc prove: factor offsets of term %u", t);
                return ZG_ERR_INVALID_PARAM;
            }
            for (uint32_t q = f0; q < f1; q++)
                if (u->factor_cols[q] >= W) {
                    set_error("zinc prove: term %u names column %u of %u", t, u->factor_cols[q], W);
                    return ZG_ERR_INVALID_PARAM;
                }
            if (f1 == f0) {
                set_error("zinc prove: constant terms (constraint %u) are not supported", k);
                return ZG_ERR_INVALID_PARAM;
            }
            if (f1 - f0 == 1) {
                r.coeff_store[(size_t)k * W + u->factor_cols[f0]] += u->term_coeffs[t];
            } else if (f1 - f0 == 2) {
                r.products.push_back({k, u->term_coeffs[t], {u->factor_cols[f0], u->factor_cols[f0 + 1]}});
            } else {
                set_error("zinc prove: term %u multiplies %u columns (at most 2 supported)", t, f1 - f0);
                return ZG_ERR_INVALID_PARAM;
            }
        }
    }
    r.coeffs = r.coeff_store.data();
    return ZG_OK;
}

zg_status check_uair(const zg_params *pb, const zg_params *pi, const UairRep *u, uint32_t nv) {
    if (!u || (u->n_bin == 0 && u->n_int == 0) || u->n_constraints == 0 || !u->coeffs ||
        (u->n_shifts && (!u->shift_src || !u->shift_amount))) {
        set_error("zinc prove: empty UAIR or null constraint/shift arrays");
        return ZG_ERR_INVALID_PARAM;
    }
    if (u->n_pub_bin > u->n_bin || u->n_pub_int > u->n_int) {
        set_error("zinc prove: more public than total columns");
        return ZG_ERR_INVALID_PARAM;
    }
    if ((u->n_bin > u->n_pub_bin && !pb) || (u->n_int > u->n_pub_int && !pi)) {
        set_error("zinc prove: parameters missing for a table with witness columns");
        return ZG_ERR_INVALID_PARAM;
    }
    if (!pb && !pi) {
        set_error("zinc prove: no parameters (every column is public)");
        return ZG_ERR_INVALID_PARAM;
    }
    const zg_params *any = pb ? pb : pi;
    if (pb && pi && (pb->ctx != pi->ctx || pb->d.field_limbs != pi->d.field_limbs)) {
        set_error("zinc prove: the two tables need one context and one field size");
        return ZG_ERR_INVALID_PARAM;
    }
    if (!any->ctx) {
        set_error("zinc prove: the parameters have no device");
        return ZG_ERR_NO_DEVICE;
    }
    if (any->d.field_limbs != 3 && any->d.field_limbs != 4) {
        set_error("zinc prove: field of %u limbs (3 or 4 supported)", any->d.field_limbs);
        return ZG_ERR_INVALID_PARAM;
    }
    if (pb && (pb->d.eval_kind != ZG_EVAL_BINPOLY || pb->d.num_vars != nv ||
               pb->d.degree_plus_one != u->degree_plus_one)) {
        set_error("zinc prove: binary table parameters do not match the trace");
        return ZG_ERR_INVALID_PARAM;
    }
    if (pi && (pi->d.eval_kind != ZG_EVAL_I64 || pi->d.num_vars != nv)) {
        set_error("zinc prove: integer table parameters must take i64 evaluations of the trace size");
        return ZG_ERR_INVALID_PARAM;
    }
    const uint32_t ncols = u->n_bin + u->n_int;
    for (uint32_t k = 0; k < u->n_shifts; k++)
        if (u->shift_src[k] >= ncols || u->shift_amount[k] == 0 || u->shift_amount[k] >= (1u << nv)) {
            set_error("zinc prove: shift %u out of range", k);
            return ZG_ERR_INVALID_PARAM;
        }
    return ZG_OK;
}

zg_status prove_impl(zg_params *pb, zg_params *pi, const UairRep *u, uint32_t nv, const uint64_t *bin,
                     const int64_t *ints, int on_device, bool mle_first, uint8_t *proof, size_t *proof_len) {
    ZG_TRY(check_uair(pb, pi, u, nv));
    if (mle_first && !u->products.empty()) {
        // prove_linear evaluates the columns first: constraints of degree above
        // one are not supported there (combined_poly_builder.rs:201-206)
        set_error("zinc prove: the MLE-first path takes linear constraints only");
        return ZG_ERR_INVALID_PARAM;
    }
    zg_params *any = pb ? pb : pi;
    zg_ctx *ctx = any->ctx;
    const int L = (int)any->d.field_limbs;
    const uint32_t nb = u->n_bin, ni = u->n_int, ncols = nb + ni, S = u->n_shifts, D = u->degree_plus_one;
    const uint32_t nc = u->n_constraints;
    const uint32_t pbn = u->n_pub_bin, pin = u->n_pub_int;  // public columns
    const uint32_t wb = nb - pbn, wi = ni - pin;             // witness columns
    const size_t n = (size_t)1 << nv;
    hphase_start(ctx);

    // the trace in device memory: binary columns, then integer columns
    const uint64_t *bin_d = bin;
    const int64_t *int_d = ints;
    if (!on_device) {
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            ZG_CUDA(cudaSetDevice(ctx->device));
            ZG_TRY(ctx->trace_arena.ensure(n * 8 * ncols + 16));
            uint64_t *dst = ctx->trace_arena.as<uint64_t>();
            // through page-locked staging: chunk k is copied on all host threads
            // while chunk k - 1 is in flight to the device
            const size_t bin_bytes = n * 8 * nb, total = n * 8 * ncols, chunk = (size_t)4 << 20;
            ZG_TRY(ctx->pin_in.ensure(total));
            uint8_t *stage = ctx->pin_in.as<uint8_t>();
            for (size_t off = 0; off < total; off += chunk) {
                const size_t len = std::min(chunk, total - off);
                const long parts = (long)((len + 65535) / 65536);
#pragma omp parallel for schedule(static)
                for (long q = 0; q < parts; q++) {
                    const size_t a = off + (size_t)q * 65536, e = std::min(a + 65536, off + len);
                    for (size_t x = a; x < e;) {  // the span may cross from the binary to the integer columns
                        const bool in_bin = x < bin_bytes;
                        const size_t stop = in_bin ? std::min(e, bin_bytes) : e;
                        const uint8_t *src = in_bin ? reinterpret_cast<const uint8_t *>(bin) + x
                                                    : reinterpret_cast<const uint8_t *>(ints) + (x - bin_bytes);
                        std::memcpy(stage + x, src, stop - x);
                        x = stop;
                    }
                }
                ZG_CUDA(cudaMemcpyAsync(reinterpret_cast<uint8_t *>(dst) + off, stage + off, len,
                                        cudaMemcpyHostToDevice, ctx->stream));
            }
            ZG_CUDA(ctx_sync(ctx));
            bin_d = dst;
            int_d = reinterpret_cast<const int64_t *>(dst + n * nb);
        }
        hphase(ctx, "zinc:h2d");
    }

    // step 0 (prover.rs:218-267): commit the witness columns of each table
    // (commit_optionally: an empty table has the default root and batch 0; the
    // arbitrary polynomial table is empty), absorb the three roots, then every
    // entry of the public columns (absorb_public_columns, lib.rs:305-320)
    const uint64_t *wbin_d = bin_d + n * pbn;
    const int64_t *wint_d = int_d + n * pin;
    HintGuard hb, hi;
    uint8_t roots[3][32];
    std::memset(roots, 0, sizeof roots);
    if (wb) ZG_TRY(zg_commit_d(pb, wbin_d, wb, &hb.h, roots[0]));
    if (wi) ZG_TRY(zg_commit_d(pi, wint_d, wi, &hi.h, roots[2]));
    TranscriptGuard tg;
    ZG_TRY(zg_transcript_new(&roots[0][0], 3, &tg.t));
    zg_transcript *t = tg.t;
    t_stream_store.clear();
    t->stream.swap(t_stream_store);
    if (pbn + pin) {
        std::vector<uint64_t> pub;
        const uint64_t *hb_pub = bin, *hi_pub = reinterpret_cast<const uint64_t *>(ints);
        if (on_device) {
            pub.resize(n * (pbn + pin));
            std::lock_guard<std::mutex> lk(ctx->mu);
            ZG_CUDA(cudaSetDevice(ctx->device));
            if (pbn) ZG_CUDA(cudaMemcpy(pub.data(), bin_d, n * 8 * pbn, cudaMemcpyDeviceToHost));
            if (pin) ZG_CUDA(cudaMemcpy(pub.data() + n * pbn, int_d, n * 8 * pin, cudaMemcpyDeviceToHost));
            hb_pub = pub.data();
            hi_pub = pub.data() + n * pbn;
        }
        for (size_t k = 0; k < n * pbn; k++) tr_absorb_slice(t, &hb_pub[k], 8);
        for (size_t k = 0; k < n * pin; k++) tr_absorb_slice(t, &hi_pub[k], 8);
    }
    // only the PCS proofs' heads (the b rows) land in t->stream
    hphase(ctx, "zinc:commit");

    // step 1 (prover.rs:285-300): the random prime; projection happens inside
    // the steps that read the columns
    uint8_t mod_b[32];
    ZG_TRY(zg_transcript_sample_field(t, (uint32_t)L, mod_b));
    const FieldCfg &f = t->f;
    std::vector<uint64_t> coeffs((size_t)nc * (ncols + S) * L);
    for (size_t k = 0; k < (size_t)nc * (ncols + S); k++) f_from_i128(f, (i128)u->coeffs[k], &coeffs[k * L]);
    hphase(ctx, "zinc:prime");

    // step 2 (prover.rs:330-380): ideal check.  The linear part of every
    // constraint is the columns evaluated at the point first, each column's
    // last row read as zero (prove_linear, ideal_check.rs:137-176).  On the
    // combined path (prove_combined, ideal_check.rs:178-240) the row-by-row
    // constraint polynomials give the same linear part (the MLE evaluation is
    // linear); their product terms are summed row by row on the GPU, and the
    // constraints in the zero ideal are sent empty.
    std::vector<uint64_t> ic_point((size_t)nv * L), combined((size_t)nc * D * L);
    std::vector<uint32_t> lens(nc);
    ZG_TRY(ideal_check_linear_impl(ctx, t, mod_b, (uint32_t)L, bin_d, nb, D, int_d, ni, nv, u->shift_src,
                                   u->shift_amount, S, nc, coeffs.data(), 1, ic_point.data(), combined.data(),
                                   lens.data(), false));
    uint32_t maxlen = D;
    for (const CprProduct &q : u->products) {
        const bool b0 = (q.cols[0] < ncols ? q.cols[0] : u->shift_src[q.cols[0] - ncols]) < nb;
        const bool b1 = (q.cols[1] < ncols ? q.cols[1] : u->shift_src[q.cols[1] - ncols]) < nb;
        maxlen = std::max(maxlen, (b0 ? D : 1) + (b1 ? D : 1) - 1);
    }
    std::vector<uint64_t> full((size_t)nc * maxlen * L, 0);
    for (uint32_t k = 0; k < nc; k++)
        std::memcpy(&full[(size_t)k * maxlen * L], &combined[(size_t)k * D * L], (size_t)D * L * 8);
    for (const CprProduct &q : u->products) {
        IcFactor fac[2];
        for (int e = 0; e < 2; e++) {
            const uint32_t j = q.cols[e];
            const uint32_t src = j < ncols ? j : u->shift_src[j - ncols];
            fac[e].shift = j < ncols ? 0 : u->shift_amount[j - ncols];
            fac[e].bin = src < nb ? bin_d + (size_t)src * n : nullptr;
            fac[e].ints = src < nb ? nullptr : int_d + (size_t)(src - nb) * n;
        }
        std::vector<uint64_t> sums;
        uint32_t plen = 0;
        ZG_TRY(ic_product_sums(ctx, f, ic_point.data(), nv, fac[0], fac[1], D, sums, plen));
        uint64_t c[4];
        f_from_i128(f, (i128)q.coeff, c);
        for (uint32_t m = 0; m < plen; m++) {
            uint64_t tm[4];
            if (L == 3) {
                fmul<3>(c, &sums[(size_t)m * L], f.p, f.n0, tm);
                fadd<3>(&full[((size_t)q.constraint * maxlen + m) * L], tm, f.p);
            } else {
                fmul<4>(c, &sums[(size_t)m * L], f.p, f.n0, tm);
                fadd<4>(&full[((size_t)q.constraint * maxlen + m) * L], tm, f.p);
            }
        }
    }
    std::vector<std::vector<uint64_t>> ic_vals(nc);
    for (uint32_t k = 0; k < nc; k++) {
        if (!mle_first && u->zero_ideal[k]) continue;  // is_zero_ideal: DynamicPolynomialF::ZERO
        ic_vals[k] = trimmed(&full[(size_t)k * maxlen * L], maxlen, L);
        for (size_t e = 0; e < ic_vals[k].size() / L; e++) tr_absorb_field(t, &ic_vals[k][e * L]);
    }
    hphase(ctx, "zinc:ideal_check");

    // step 3 (prover.rs:385-415): the projecting element a = Chal (i128) in F,
    // the columns evaluated at a, kept on the device for steps 4 and 5
    uint64_t a[4];
    f_from_i128(f, tr_challenge_i128(t), a);
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ZG_CUDA(cudaSetDevice(ctx->device));
        ZG_TRY(ctx->mle_arena.ensure(n * 8 * L * ncols + 16));
    }
    uint64_t *mles = ctx->mle_arena.as<uint64_t>();
    ZG_TRY(zg_piop_eval_projection(ctx, mod_b, (uint32_t)L, bin_d, nb, D, int_d, ni, nv, a, 1, mles));
    hphase(ctx, "zinc:eval_projection");

    // step 4 (prover.rs:420-472): CPR group + MultiDegreeSumcheck + finalize
    // capacity: modulus, group count, rounds, one degree (3 here, at most 8),
    // the round messages, the claimed sum
    size_t md_len = 8 * (size_t)L + 12 + (size_t)nv * 8 * 8 * L + 8 * (size_t)L;
    std::vector<uint8_t> md_proof(md_len);
    std::vector<uint64_t> cpr_point((size_t)nv * L), cpr_evals((size_t)(ncols + S) * L);
    ZG_TRY(cpr_prove_impl(ctx, t, mod_b, (uint32_t)L, mles, ncols, nv, ic_point.data(), u->shift_src,
                          u->shift_amount, S, nc, coeffs.data(), u->products, 1, md_proof.data(), &md_len,
                          cpr_point.data(), cpr_evals.data()));
    md_proof.resize(md_len);
    hphase(ctx, "zinc:cpr");

    // step 5 (prover.rs:478-492): multipoint evaluation down to r_0
    // capacity: modulus, message count, per round a length and 2 evaluations,
    // the claimed sum
    size_t mp_len = 8 * (size_t)L + 4 + (size_t)nv * (4 + 2 * 8 * L) + 8 * (size_t)L;
    std::vector<uint8_t> mp_proof(mp_len);
    std::vector<uint64_t> r0((size_t)nv * L);
    ZG_TRY(zg_piop_multipoint_eval(ctx, t, mod_b, (uint32_t)L, mles, ncols, nv, cpr_point.data(), u->shift_src,
                                   u->shift_amount, S, 1, mp_proof.data(), &mp_len, r0.data()));
    mp_proof.resize(mp_len);
    hphase(ctx, "zinc:multipoint");

    // step 6 (prover.rs:497-532): lifted evaluations at r_0, trimmed, every
    // coefficient absorbed (absorb_random_field_slice)
    std::vector<uint64_t> lifted(((size_t)nb * D + ni) * L);
    ZG_TRY(zg_piop_lifted_evals(ctx, mod_b, (uint32_t)L, bin_d, nb, D, int_d, ni, nv, r0.data(), 1, lifted.data()));
    std::vector<std::vector<uint64_t>> lifted_polys(ncols);
    for (uint32_t c = 0; c < ncols; c++) {
        const uint64_t *src = c < nb ? &lifted[(size_t)c * D * L] : &lifted[((size_t)nb * D + (c - nb)) * L];
        lifted_polys[c] = trimmed(src, c < nb ? D : 1, L);
        for (size_t k = 0; k < lifted_polys[c].size() / L; k++) tr_absorb_field(t, &lifted_polys[c][k * L]);
    }
    hphase(ctx, "zinc:lifted");

    // finish (prover.rs:603-650) and the transcription (lib.rs:129-160).  Every
    // part but the PCS stream is known now, so the proof is laid out in the
    // caller's buffer first and step 7 writes each table's openings (the bulk of
    // the proof) straight into their place: the PCS stream is never copied
    const uint64_t *p = f.p;
    // witness lifted evaluations: public columns come first in each table
    std::vector<std::vector<uint64_t>> witness_lifted(lifted_polys.begin() + pbn, lifted_polys.begin() + nb);
    witness_lifted.insert(witness_lifted.end(), lifted_polys.begin() + nb + pin, lifted_polys.end());
    const Bytes ic_b = poly_vec(ic_vals, p, L), lifted_b = poly_vec(witness_lifted, p, L);
    Bytes cpr;
    cpr.sub(field_vec(cpr_evals.data(), ncols, p, L));
    cpr.sub(field_vec(cpr_evals.data() + (size_t)ncols * L, S, p, L));
    const size_t size_b = wb ? zg_proof_size(pb, wb) : 0, size_i = wi ? zg_proof_size(pi, wi) : 0;
    const size_t head_b = wb ? (size_t)pb->info.num_rows * 2 * pb->info.field_bytes : 0;
    const size_t head_i = wi ? (size_t)pi->info.num_rows * 2 * pi->info.field_bytes : 0;
    const size_t zip_len = size_b + size_i;
    const size_t total = 3 * 40 + 4 + zip_len + 4 + ic_b.b.size() + 4 + cpr.b.size() + 4 + md_proof.size() + 4 +
                         mp_proof.size() + 4 + lifted_b.b.size();
    const size_t cap = *proof_len;
    *proof_len = total;
    if (cap < total) {
        set_error("zinc prove: proof needs %zu bytes, buffer holds %zu", total, cap);
        return ZG_ERR_BUFFER_TOO_SMALL;
    }
    uint8_t *w = proof;
    auto put = [&](const void *src, size_t len) {
        if (len) std::memcpy(w, src, len);
        w += len;
    };
    auto put_u32 = [&](uint32_t v) { put(&v, 4); };
    auto put_sub = [&](const uint8_t *src, size_t len) {
        put_u32((uint32_t)len);
        put(src, len);
    };
    const uint64_t batches[3] = {wb, 0, wi};
    for (int k = 0; k < 3; k++) {
        put(roots[k], 32);
        put(&batches[k], 8);
    }
    put_u32((uint32_t)zip_len);
    uint8_t *zip = w;
    w += zip_len;
    put_sub(ic_b.b.data(), ic_b.b.size());
    put_sub(cpr.b.data(), cpr.b.size());
    put_sub(md_proof.data(), md_proof.size());
    put_sub(mp_proof.data(), mp_proof.size());
    put_sub(lifted_b.b.data(), lifted_b.b.size());

    // step 7 (prover.rs:552-597): PCS openings at r_0, binary table first.  Each
    // table's b rows (the head of its PCS proof) go to the transcript stream; the
    // combined row and the openings (its tail) go to their place in `proof`
    uint8_t ev[32];
    auto prove_f_into = [&](zg_params *pp, const void *polys_d, uint32_t batch, const zg_hint *h,
                            uint8_t *tail) -> zg_status {
        std::lock_guard<std::mutex> lk(pp->ctx->mu);
        ZG_CUDA(cudaSetDevice(pp->ctx->device));
        return prove_device(pp, pp->ctx, t, polys_d, batch, reinterpret_cast<const uint8_t *>(r0.data()), h, ev,
                            tail, true);
    };
    if (wb) ZG_TRY(prove_f_into(pb, wbin_d, wb, hb.h, zip + head_b));
    if (wi) ZG_TRY(prove_f_into(pi, wint_d, wi, hi.h, zip + size_b + head_i));
    if (t->stream.size() != head_b + head_i) {
        set_error("internal: PCS proof heads of %zu bytes, %zu expected", t->stream.size(), head_b + head_i);
        return ZG_ERR_INVALID_PARAM;
    }
    if (head_b) std::memcpy(zip, t->stream.data(), head_b);
    if (head_i) std::memcpy(zip + size_b, t->stream.data() + head_b, head_i);
    hphase(ctx, "zinc:prove_f");
    hphase(ctx, "zinc:finish");
    return ZG_OK;
}

}  // namespace

extern "C" zg_status zg_zinc_prove_mle_first(zg_params *pp_bin, zg_params *pp_int, const zg_linear_uair *uair,
                                             uint32_t num_vars, const uint64_t *bin_cols, const int64_t *int_cols,
                                             int cols_on_device, uint8_t *proof, size_t *proof_len) {
    try {
        if (!uair || !proof_len || (*proof_len && !proof) || (uair->n_bin && !bin_cols) ||
            (uair->n_int && !int_cols) || num_vars == 0 || num_vars > 30) {
            set_error("zinc prove: null argument or num_vars out of range");
            return ZG_ERR_INVALID_PARAM;
        }
        const UairRep rep = rep_of(uair);
        return prove_impl(pp_bin, pp_int, &rep, num_vars, bin_cols, int_cols, cols_on_device, true, proof,
                          proof_len);
    } catch (const std::exception &e) {
        set_error("zinc prove: %s", e.what());
        return ZG_ERR_OOM;
    }
}

extern "C" zg_status zg_zinc_prove(zg_params *pp_bin, zg_params *pp_int, const zg_uair *uair, uint32_t num_vars,
                                   const uint64_t *bin_cols, const int64_t *int_cols, int cols_on_device,
                                   int mle_first, uint8_t *proof, size_t *proof_len) {
    try {
        if (!uair || !proof_len || (*proof_len && !proof) || (uair->n_bin && !bin_cols) ||
            (uair->n_int && !int_cols) || num_vars == 0 || num_vars > 30) {
            set_error("zinc prove: null argument or num_vars out of range");
            return ZG_ERR_INVALID_PARAM;
        }
        UairRep rep;
        ZG_TRY(rep_of(uair, rep));
        return prove_impl(pp_bin, pp_int, &rep, num_vars, bin_cols, int_cols, cols_on_device, mle_first != 0, proof,
                          proof_len);
    } catch (const std::exception &e) {
        set_error("zinc prove: %s", e.what());
        return ZG_ERR_OOM;
    }
}

namespace {

// Little-endian reader over a byte range; every read is bounds checked.
struct Reader {
    const uint8_t *p = nullptr;
    size_t len = 0, pos = 0;
    bool take(size_t n, const uint8_t **out) {
        if (n > len - pos) return false;
        if (out) *out = p + pos;
        pos += n;
        return true;
    }
    bool u32(uint32_t *v) {
        const uint8_t *b;
        if (!take(4, &b)) return false;
        std::memcpy(v, b, 4);
        return true;
    }
    bool u64(uint64_t *v) {
        const uint8_t *b;
        if (!take(8, &b)) return false;
        std::memcpy(v, b, 8);
        return true;
    }
    // a u32 length prefix, then that many bytes as a sub-reader
    bool sub(Reader *r, size_t *off) {
        uint32_t n;
        if (!u32(&n)) return false;
        *off = pos;
        const uint8_t *b;
        if (!take(n, &b)) return false;
        *r = Reader{b, n, 0};
        return true;
    }
    bool done() const { return pos == len; }
};

zg_status malformed(const char *what) {
    set_error("Proof: malformed %s", what);
    return ZG_ERR_SERIALIZATION;
}

// DynamicPolyVecF (over_field.rs:409-476): empty, or a flag byte, the modulus
// when the flag is set, then u32 length + inners per polynomial.
bool read_poly_vec(Reader r, size_t fb, const uint8_t *modulus, uint32_t *count) {
    *count = 0;
    if (r.done()) return true;
    const uint8_t *flag, *m;
    if (!r.take(1, &flag) || *flag > 1) return false;
    if (*flag && (!r.take(fb, &m) || std::memcmp(m, modulus, fb) != 0)) return false;
    while (!r.done()) {
        uint32_t n;
        if (!r.u32(&n) || (!*flag && n) || !r.take((size_t)n * fb, nullptr)) return false;
        (*count)++;
    }
    return true;
}

// Vec<F> (traits.rs:566-607): empty, or the modulus and whole field elements.
bool read_field_vec(Reader r, size_t fb, const uint8_t *modulus, uint32_t *count) {
    *count = 0;
    if (r.done()) return true;
    const uint8_t *m;
    if (!r.take(fb, &m) || std::memcmp(m, modulus, fb) != 0 || (r.len - r.pos) % fb != 0) return false;
    *count = (uint32_t)((r.len - r.pos) / fb);
    return true;
}

}  // namespace

// Proof::read_transcription_bytes_exact (protocol/src/lib.rs:93-127): the
// parts' places in the bytes, with every nested length checked.
extern "C" zg_status zg_proof_read(const uint8_t *proof, size_t len, uint32_t limbs, uint32_t num_vars,
                                   zg_proof_layout *out) {
    if (!proof || !out || limbs < 1 || limbs > MAX_FIELD_LIMBS || num_vars == 0 || num_vars > 64) {
        set_error("Proof: null argument, field of %u limbs or num_vars %u", limbs, num_vars);
        return ZG_ERR_INVALID_PARAM;
    }
    std::memset(out, 0, sizeof *out);
    const size_t fb = 8 * (size_t)limbs;
    Reader r{proof, len, 0};
    for (int k = 0; k < 3; k++) {
        const uint8_t *root;
        if (!r.take(32, &root) || !r.u64(&out->batch_sizes[k])) return malformed("commitments");
        std::memcpy(out->roots[k], root, 32);
    }
    uint32_t zl;
    if (!r.u32(&zl)) return malformed("PCS stream length");
    out->zip_offset = r.pos;
    out->zip_len = zl;
    if (!r.take(zl, nullptr)) return malformed("PCS stream");
    Reader ic, res, md, mp, lifted;
    if (!r.sub(&ic, &out->ideal_check_offset) || !r.sub(&res, &out->resolver_offset) ||
        !r.sub(&md, &out->multi_degree_offset) || !r.sub(&mp, &out->multipoint_offset) ||
        !r.sub(&lifted, &out->lifted_offset) || !r.done())
        return malformed("part lengths");
    out->ideal_check_len = ic.len;
    out->resolver_len = res.len;
    out->multi_degree_len = md.len;
    out->multipoint_len = mp.len;
    out->lifted_len = lifted.len;
    // MultiDegreeSumcheckProof (multi_degree.rs:86-190): modulus, group count,
    // num_vars, one degree per group, the messages, one claimed sum per group
    const uint8_t *modulus;
    uint32_t ng, nv;
    if (!md.take(fb, &modulus) || !md.u32(&ng) || !md.u32(&nv) || ng == 0 || ng > 64 || nv != num_vars)
        return malformed("multi-degree sumcheck header");
    size_t msgs = 0;
    for (uint32_t g = 0; g < ng; g++) {
        uint32_t d;
        if (!md.u32(&d) || d > 64) return malformed("multi-degree sumcheck degree");
        if (g == 0) out->cpr_degree = d;
        msgs += (size_t)d * nv;
    }
    if (!md.take((msgs + ng) * fb, nullptr) || !md.done()) return malformed("multi-degree sumcheck body");
    out->multi_degree_groups = ng;
    std::memcpy(out->modulus, modulus, fb);
    // SumcheckProof (sumcheck.rs:35-111): modulus, round count, per round a
    // u32 length and that many elements, the claimed sum
    const uint8_t *m2;
    uint32_t rounds;
    if (!mp.take(fb, &m2) || std::memcmp(m2, modulus, fb) != 0 || !mp.u32(&rounds) || rounds != num_vars)
        return malformed("multipoint sumcheck header");
    for (uint32_t k = 0; k < rounds; k++) {
        uint32_t n;
        if (!mp.u32(&n) || n > 64 || !mp.take((size_t)n * fb, nullptr)) return malformed("multipoint round");
    }
    if (!mp.take(fb, nullptr) || !mp.done()) return malformed("multipoint claimed sum");
    // the resolver: up evaluations then down evaluations, each a sub-buffer
    Reader up, down;
    size_t o1, o2;
    if (!res.sub(&up, &o1) || !res.sub(&down, &o2) || !res.done()) return malformed("resolver");
    if (!read_field_vec(up, fb, modulus, &out->n_up_evals) || !read_field_vec(down, fb, modulus, &out->n_down_evals))
        return malformed("resolver evaluations");
    if (!read_poly_vec(ic, fb, modulus, &out->n_ideal_values)) return malformed("ideal check values");
    if (!read_poly_vec(lifted, fb, modulus, &out->n_lifted)) return malformed("lifted evaluations");
    return ZG_OK;
}
