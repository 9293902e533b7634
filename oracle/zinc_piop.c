/*
 * zinc_piop.c -- CPU restatement (oracle) of the Zinc+ PIOP prover and
 * verifier (protocol/src/prover.rs, protocol/src/verifier.rs and the piop crate).
 * TEST INFRASTRUCTURE ONLY: the checker of the product's Zinc+ prover and the
 * timed CPU baseline of that prover.  Included at the end of zipref.c, whose
 * field, transcript, sumcheck and Zip+ helpers it uses.
 *
 * A UAIR here is a constraint system over the trace columns
 * [binary up..., integer up..., down (one per shift, in shift order)]: each
 * constraint is a sum of terms `coeff * prod(factors)` with an integer
 * coefficient and zero or more column factors, and lies in the zero ideal or
 * in (X - root) (RotationIdeal<_, 1>, uair/src/ideal/rotation.rs).  Binary
 * columns are BinaryPoly<D> (bit l = coefficient l), integer columns i64.
 * The first n_pub_bin / n_pub_int columns of each kind are public.
 */

static uint32_t uair_ncols(const zr_uair *u) { return u->n_bin + u->n_int; }

/* The polynomial (over F, little-endian coefficients) of column j at row b,
 * j indexing [up..., down...]: len coefficients written to out (len = D for
 * a binary column, 1 for an integer column); rows past the end read as zero
 * (the reference's zero padding of shifted columns). */
static uint32_t col_poly_at(const fcfg *f, const zr_uair *u, const uint64_t *bin, const int64_t *ints,
                            uint32_t nvars, uint32_t j, size_t b, uint64_t *out) {
    const size_t n = (size_t)1 << nvars;
    const uint32_t J = uair_ncols(u), L = f->L;
    uint32_t src = j;
    size_t row = b;
    if (j >= J) {
        src = u->shift_src[j - J];
        row = b + u->shift_amt[j - J];
    }
    if (src < u->n_bin) {
        const uint64_t x = row < n ? bin[(size_t)src * n + row] : 0;
        for (uint32_t l = 0; l < u->D; l++) {
            if ((x >> l) & 1) memcpy(out + (size_t)l * L, f->one, 8 * L);
            else memset(out + (size_t)l * L, 0, 8 * L);
        }
        return u->D;
    }
    if (row < n) f_from_i64(f, ints[(size_t)(src - u->n_bin) * n + row], out);
    else memset(out, 0, 8 * L);
    return 1;
}

static uint32_t col_len(const zr_uair *u, uint32_t j) {
    const uint32_t J = uair_ncols(u);
    const uint32_t src = j < J ? j : u->shift_src[j - J];
    return src < u->n_bin ? u->D : 1;
}

/* Coefficient count of constraint k's polynomial (a bound: the longest term). */
static uint32_t cons_len(const zr_uair *u, uint32_t k) {
    uint32_t best = 1;
    for (uint32_t t = u->term_off[k]; t < u->term_off[k + 1]; t++) {
        uint32_t len = 1;
        for (uint32_t q = u->fac_off[t]; q < u->fac_off[t + 1]; q++) len += col_len(u, u->fac_col[q]) - 1;
        if (len > best) best = len;
    }
    return best;
}

static uint32_t uair_max_degree(const zr_uair *u) {
    uint32_t m = 0;
    for (uint32_t t = 0; t < u->term_off[u->n_cons]; t++) {
        const uint32_t d = u->fac_off[t + 1] - u->fac_off[t];
        if (d > m) m = d;
    }
    return m;
}

/* acc (len coefficients) += c * a (alen) * b (blen): polynomial product */
static void poly_mul_into(const fcfg *f, const uint64_t *a, uint32_t alen, const uint64_t *b, uint32_t blen,
                          uint64_t *out) {
    const uint32_t L = f->L;
    memset(out, 0, 8 * L * (size_t)(alen + blen - 1));
    for (uint32_t i = 0; i < alen; i++) {
        if (uiszero(a + (size_t)i * L, L)) continue;
        for (uint32_t j = 0; j < blen; j++) {
            uint64_t t[4];
            fmul(f, a + (size_t)i * L, b + (size_t)j * L, t);
            fadd(f, out + (size_t)(i + j) * L, t);
        }
    }
}

/* Constraint k at one row as a polynomial over F: sum_t c_t prod_f col_f(row),
 * from the per-column polynomials vals[j] (len col_len(j) each, stride D). */
static void cons_eval_poly(const fcfg *f, const zr_uair *u, uint32_t k, const uint64_t *vals, uint32_t stride,
                           uint64_t *out, uint32_t out_len) {
    const uint32_t L = f->L;
    uint64_t *prod = (uint64_t *)malloc(8 * L * (size_t)out_len), *tmp = (uint64_t *)malloc(8 * L * (size_t)out_len);
    memset(out, 0, 8 * L * (size_t)out_len);
    for (uint32_t t = u->term_off[k]; t < u->term_off[k + 1]; t++) {
        uint32_t plen = 1;
        f_from_i64(f, u->term_coeff[t], prod);
        for (uint32_t q = u->fac_off[t]; q < u->fac_off[t + 1]; q++) {
            const uint32_t j = u->fac_col[q], cl = col_len(u, j);
            poly_mul_into(f, prod, plen, vals + (size_t)j * stride * L, cl, tmp);
            plen += cl - 1;
            memcpy(prod, tmp, 8 * L * (size_t)plen);
        }
        for (uint32_t l = 0; l < plen && l < out_len; l++) fadd(f, out + (size_t)l * L, prod + (size_t)l * L);
    }
    free(prod);
    free(tmp);
}

static uint32_t trim_len(const fcfg *f, const uint64_t *v, uint32_t len) {
    while (len && uiszero(v + (size_t)(len - 1) * f->L, f->L)) len--;
    return len;
}

/* Step 2, MLE first (IdealCheckProtocol::prove_linear, piop/src/ideal_check.rs:
 * 137-176; evaluate_combined_polynomials, ideal_check/combined_poly_builder.rs:
 * 181-300): every up and down column evaluated coefficient-wise at the point,
 * reading row i + shift for i < 2^nvars - 1 and zero on the last row, then the
 * (linear) constraints applied to those values.  values: n_cons x maxlen inners,
 * lens: trimmed lengths. */
static void ideal_values_mle_first(const fcfg *f, const zr_uair *u, const uint64_t *bin, const int64_t *ints,
                                   uint32_t nvars, const uint64_t *point, uint32_t maxlen, uint64_t *values,
                                   uint32_t *lens) {
    const size_t n = (size_t)1 << nvars;
    const uint32_t L = f->L, J = uair_ncols(u), JS = J + u->n_shifts, D = u->D;
    uint64_t *eq = (uint64_t *)malloc(8 * L * n);
    build_eq(f, point, nvars, eq);
    memset(eq + (n - 1) * L, 0, 8 * L); /* the last row is zero for every column */
    uint64_t *vals = (uint64_t *)calloc((size_t)JS * D, 8 * L);
    int nt = zr_get_threads();
    (void)nt;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (long j = 0; j < (long)JS; j++) {
        uint32_t src = (uint32_t)j;
        size_t c = 0;
        if ((uint32_t)j >= J) {
            src = u->shift_src[j - J];
            c = u->shift_amt[j - J];
        }
        uint64_t *o = vals + (size_t)j * D * L;
        for (size_t b = 0; b + c < n; b++) {
            const uint64_t *e = eq + b * L;
            if (src < u->n_bin) {
                uint64_t x = bin[(size_t)src * n + b + c];
                while (x) {
                    const uint32_t l = (uint32_t)__builtin_ctzll(x);
                    if (l < D) fadd(f, o + (size_t)l * L, e);
                    x &= x - 1;
                }
            } else {
                uint64_t v[4], t[4];
                f_from_i64(f, ints[(size_t)(src - u->n_bin) * n + b + c], v);
                fmul(f, v, e, t);
                fadd(f, o, t);
            }
        }
    }
    for (uint32_t k = 0; k < u->n_cons; k++) {
        uint64_t *o = values + (size_t)k * maxlen * L;
        cons_eval_poly(f, u, k, vals, D, o, maxlen);
        lens[k] = trim_len(f, o, maxlen);
    }
    free(vals);
    free(eq);
}

/* Step 2, combined (IdealCheckProtocol::prove_combined, ideal_check.rs:178-240;
 * compute_combined_polynomials, combined_poly_builder.rs:30-95): each row's
 * constraint polynomials over the projected trace (rows 0..2^nvars - 2, down
 * columns zero padded; the last row zero), each coefficient's MLE evaluated at
 * the point; constraints in the zero ideal are skipped (empty). */
static void ideal_values_combined(const fcfg *f, const zr_uair *u, const uint64_t *bin, const int64_t *ints,
                                  uint32_t nvars, const uint64_t *point, uint32_t maxlen, uint64_t *values,
                                  uint32_t *lens) {
    const size_t n = (size_t)1 << nvars;
    const uint32_t L = f->L, J = uair_ncols(u), JS = J + u->n_shifts, D = u->D, K = u->n_cons;
    uint64_t *eq = (uint64_t *)malloc(8 * L * n);
    build_eq(f, point, nvars, eq);
    memset(values, 0, 8 * L * (size_t)K * maxlen);
    int nt = zr_get_threads();
    (void)nt;
#pragma omp parallel num_threads(nt)
    {
        uint64_t *acc = (uint64_t *)calloc((size_t)K * maxlen, 8 * L);
        uint64_t *vals = (uint64_t *)calloc((size_t)JS * D, 8 * L);
        uint64_t *cp = (uint64_t *)calloc(maxlen, 8 * L);
#pragma omp for schedule(static)
        for (long b = 0; b < (long)n - 1; b++) {
            for (uint32_t j = 0; j < JS; j++) col_poly_at(f, u, bin, ints, nvars, j, (size_t)b, vals + (size_t)j * D * L);
            for (uint32_t k = 0; k < K; k++) {
                if (u->ideal_kind[k] == 0) continue;
                cons_eval_poly(f, u, k, vals, D, cp, maxlen);
                for (uint32_t l = 0; l < maxlen; l++) {
                    uint64_t t[4];
                    if (uiszero(cp + (size_t)l * L, L)) continue;
                    fmul(f, cp + (size_t)l * L, eq + (size_t)b * L, t);
                    fadd(f, acc + ((size_t)k * maxlen + l) * L, t);
                }
            }
        }
#pragma omp critical
        for (size_t i = 0; i < (size_t)K * maxlen; i++) fadd(f, values + i * L, acc + i * L);
        free(acc);
        free(vals);
        free(cp);
    }
    for (uint32_t k = 0; k < K; k++) lens[k] = u->ideal_kind[k] == 0 ? 0 : trim_len(f, values + (size_t)k * maxlen * L, maxlen);
    free(eq);
}

/* powers 1, x, ..., x^(n-1) */
static void f_powers(const fcfg *f, const uint64_t *x, uint32_t n, uint64_t *out) {
    const uint32_t L = f->L;
    if (!n) return;
    memcpy(out, f->one, 8 * L);
    for (uint32_t i = 1; i < n; i++) fmul(f, out + (size_t)(i - 1) * L, x, out + (size_t)i * L);
}

/* The CPR comb as a sumcheck group: sum_k alpha^k sum_t c_t prod v_(2 + f), times
 * eq_r (MLE 1) and (1 - selector) (MLE 0) (combined_poly_resolver.rs:71-178).
 * Allocates the group's coefficient and index arrays into *bufs. */
typedef struct {
    uint64_t *coeffs, *fa, *fb;
    uint32_t *offsets, *indices, *fm;
} cpr_bufs;

static void cpr_group(const fcfg *f, const zr_uair *u, const uint64_t *alpha_pows, const uint64_t *mles,
                      uint32_t n_mles, zr_sc_group *g, cpr_bufs *bb) {
    const uint32_t L = f->L, T = u->term_off[u->n_cons], NF = u->fac_off[T];
    bb->coeffs = (uint64_t *)calloc(T ? T : 1, 8 * L);
    bb->offsets = (uint32_t *)calloc(T + 1, 4);
    bb->indices = (uint32_t *)calloc(NF ? NF : 1, 4);
    for (uint32_t k = 0; k < u->n_cons; k++)
        for (uint32_t t = u->term_off[k]; t < u->term_off[k + 1]; t++) {
            uint64_t c[4];
            f_from_i64(f, u->term_coeff[t], c);
            fmul(f, c, alpha_pows + (size_t)k * L, bb->coeffs + (size_t)t * L);
        }
    for (uint32_t t = 0; t <= T; t++) bb->offsets[t] = u->fac_off[t];
    for (uint32_t q = 0; q < NF; q++) bb->indices[q] = 2 + u->fac_col[q];
    bb->fm = (uint32_t *)malloc(8);
    bb->fa = (uint64_t *)calloc(2, 8 * L);
    bb->fb = (uint64_t *)calloc(2, 8 * L);
    bb->fm[0] = 1; /* 0 + 1 * eq_r */
    memcpy(bb->fb, f->one, 8 * L);
    bb->fm[1] = 0; /* 1 - selector */
    memcpy(bb->fa + L, f->one, 8 * L);
    memcpy(bb->fb + L, f->one, 8 * L);
    fneg(f, bb->fb + L);
    g->degree = uair_max_degree(u) + 2;
    g->n_mles = n_mles;
    g->n_products = T;
    g->mles = mles;
    g->coeffs = bb->coeffs;
    g->offsets = bb->offsets;
    g->indices = bb->indices;
    g->n_factors = 2;
    g->factor_mles = bb->fm;
    g->factor_a = bb->fa;
    g->factor_b = bb->fb;
}

static void cpr_bufs_free(cpr_bufs *b) {
    free(b->coeffs);
    free(b->offsets);
    free(b->indices);
    free(b->fm);
    free(b->fa);
    free(b->fb);
}

/* sum_k alpha^k g_k(vals): the folded constraints at one point (ConstraintFolder,
 * combined_poly_resolver/folder.rs:22-62) */
static void cpr_folded(const fcfg *f, const zr_uair *u, const uint64_t *alpha_pows, const uint64_t *vals,
                       uint64_t *out) {
    const uint32_t L = f->L;
    memset(out, 0, 8 * L);
    for (uint32_t k = 0; k < u->n_cons; k++) {
        uint64_t gk[4] = {0};
        for (uint32_t t = u->term_off[k]; t < u->term_off[k + 1]; t++) {
            uint64_t p[4], q[4];
            f_from_i64(f, u->term_coeff[t], p);
            for (uint32_t r = u->fac_off[t]; r < u->fac_off[t + 1]; r++) {
                fmul(f, p, vals + (size_t)u->fac_col[r] * L, q);
                memcpy(p, q, 8 * L);
            }
            fadd(f, gk, p);
        }
        uint64_t t[4];
        fmul(f, gk, alpha_pows + (size_t)k * L, t);
        fadd(f, out, t);
    }
}

/* eq(a, b) = prod_i (a_i b_i + (1 - a_i)(1 - b_i)) */
static void eq_eval_pts(const fcfg *f, const uint64_t *a, const uint64_t *b, uint32_t nv, uint64_t *out) {
    const uint32_t L = f->L;
    memcpy(out, f->one, 8 * L);
    for (uint32_t i = 0; i < nv; i++) {
        uint64_t ab[4], oa[4], ob[4], t[4], s[4];
        fmul(f, a + (size_t)i * L, b + (size_t)i * L, ab);
        memcpy(oa, f->one, 8 * L);
        fsub(f, oa, a + (size_t)i * L);
        memcpy(ob, f->one, 8 * L);
        fsub(f, ob, b + (size_t)i * L);
        fmul(f, oa, ob, t);
        fadd(f, ab, t);
        fmul(f, out, ab, s);
        memcpy(out, s, 8 * L);
    }
}

/* The MLE of next_c(x, .) at y: sum_{b >= c} eq(x, b - c) eq(y, b), the shift
 * predicate S_c(x, y) of piop/src/shift_predicate.rs evaluated from its
 * definition (build_next_c_r_mle, poly/src/utils.rs:207-236). */
static void shift_pred_eval(const fcfg *f, const uint64_t *x, const uint64_t *y, uint32_t nv, size_t c,
                            uint64_t *out) {
    const size_t n = (size_t)1 << nv;
    const uint32_t L = f->L;
    uint64_t *ex = (uint64_t *)malloc(8 * L * n), *ey = (uint64_t *)malloc(8 * L * n);
    build_eq(f, x, nv, ex);
    build_eq(f, y, nv, ey);
    uint64_t acc[4] = {0};
    for (size_t b = c; b < n; b++) {
        uint64_t t[4];
        fmul(f, ex + (b - c) * L, ey + b * L, t);
        fadd(f, acc, t);
    }
    memcpy(out, acc, 8 * L);
    free(ex);
    free(ey);
}

/* DynamicPolyVecF transcription (poly/src/univariate/dynamic/over_field.rs:409-476) */
static void put_poly_vec(wbuf *w, const fcfg *f, const uint64_t *vals, uint32_t stride, const uint32_t *lens,
                         uint32_t count) {
    if (!count) return;
    int any = 0;
    for (uint32_t k = 0; k < count; k++) any |= lens[k] != 0;
    uint8_t flag = any ? 1 : 0;
    wput(w, &flag, 1);
    if (any) wput(w, f->p, 8 * f->L);
    for (uint32_t k = 0; k < count; k++) {
        wput(w, &lens[k], 4);
        wput(w, vals + (size_t)k * stride * f->L, 8 * f->L * (size_t)lens[k]);
    }
}

/* Vec<F> transcription: modulus then the inners, nothing when empty */
static void put_field_vec(wbuf *w, const fcfg *f, const uint64_t *vals, uint32_t count) {
    if (!count) return;
    wput(w, f->p, 8 * f->L);
    wput(w, vals, 8 * f->L * (size_t)count);
}

/* u32 length, then the bytes of a sub-buffer */
static void put_sub(wbuf *w, const uint8_t *b, size_t len) {
    uint32_t l = (uint32_t)len;
    wput(w, &l, 4);
    wput(w, b, len);
}

static void absorb_public(zr_transcript *tr, const zr_uair *u, const uint64_t *bin, const int64_t *ints,
                          uint32_t nvars) {
    /* absorb_public_columns (protocol/src/lib.rs:305-320): each entry's 8 LE
     * bytes as one slice, binary public columns then integer ones */
    const size_t n = (size_t)1 << nvars;
    for (uint32_t c = 0; c < u->n_pub_bin; c++)
        for (size_t b = 0; b < n; b++) zr_tr_absorb_slice(tr, (const uint8_t *)&bin[(size_t)c * n + b], 8);
    for (uint32_t c = 0; c < u->n_pub_int; c++)
        for (size_t b = 0; b < n; b++) zr_tr_absorb_slice(tr, (const uint8_t *)&ints[(size_t)c * n + b], 8);
}

/* ZincPlusPiop::prove (protocol/src/prover.rs:218-706): steps 0-7 on one
 * transcript and the Proof transcription (protocol/src/lib.rs:129-160).
 * mle_first selects step1_mle_first / prove_linear (linear UAIRs only) or
 * step1_combined / prove_combined. */
int zr_zinc_prove(const zr_desc *db, const zr_desc *di, uint32_t nvars, const uint64_t *bin, const int64_t *ints,
                  const zr_uair *u, uint32_t L, int mle_first, uint8_t *out, size_t cap, size_t *out_len) {
    if (nvars < 2 || L < 1 || L > 4 || u->n_pub_bin > u->n_bin || u->n_pub_int > u->n_int) return -1;
    if (mle_first && uair_max_degree(u) > 1) return -1;
    const size_t n = (size_t)1 << nvars;
    const uint32_t J = uair_ncols(u), S = u->n_shifts, K = u->n_cons, D = u->D;
    const uint32_t wb = u->n_bin - u->n_pub_bin, wi = u->n_int - u->n_pub_int;
    int rc = 0;
    /* step 0: commitments (the arbitrary table is empty: default root) */
    uint8_t roots[3][32];
    memset(roots, 0, sizeof roots);
    if (wb && zr_commit(db, bin + (size_t)u->n_pub_bin * n, wb, roots[0])) return -2;
    if (wi && zr_commit(di, ints + (size_t)u->n_pub_int * n, wi, roots[2])) return -2;
    zr_transcript *tr = zr_tr_new();
    for (int r = 0; r < 3; r++) zr_tr_absorb_slice(tr, roots[r], 32);
    absorb_public(tr, u, bin, ints, nvars);
    /* step 1: the prime */
    uint64_t prime[4] = {0};
    zr_tr_get_prime(tr, L, prime);
    fcfg f;
    fcfg_init(&f, prime, L);
    /* step 2: ideal check */
    uint32_t maxlen = 1;
    for (uint32_t k = 0; k < K; k++) maxlen = cons_len(u, k) > maxlen ? cons_len(u, k) : maxlen;
    uint64_t *icpt = (uint64_t *)calloc(nvars, 8 * L);
    for (uint32_t k = 0; k < nvars; k++) tr_field_challenge(tr, &f, icpt + (size_t)k * L);
    uint64_t *icv = (uint64_t *)calloc((size_t)K * maxlen, 8 * L);
    uint32_t *icl = (uint32_t *)calloc(K ? K : 1, 4);
    if (mle_first) ideal_values_mle_first(&f, u, bin, ints, nvars, icpt, maxlen, icv, icl);
    else ideal_values_combined(&f, u, bin, ints, nvars, icpt, maxlen, icv, icl);
    for (uint32_t k = 0; k < K; k++)
        for (uint32_t l = 0; l < icl[k]; l++) tr_absorb_field(tr, &f, icv + ((size_t)k * maxlen + l) * L);
    /* step 3: the projecting element (Chal = i128) and the projected MLEs */
    uint64_t a[4];
    f_from_i128(&f, tr_i128(tr), a);
    const size_t nmle = 2 + (size_t)J + S;
    uint64_t *mles = (uint64_t *)calloc(nmle * n, 8 * L);
    uint64_t *up = mles + 2 * n * L;
    zr_piop_eval_projection(f.p, L, bin, u->n_bin, D, ints, u->n_int, nvars, a, up);
    /* step 4: CPR (combined_poly_resolver.rs:71-247) in a MultiDegreeSumcheck */
    uint64_t alpha[4];
    tr_field_challenge(tr, &f, alpha);
    uint64_t *apow = (uint64_t *)calloc(K ? K : 1, 8 * L);
    f_powers(&f, alpha, K, apow);
    memcpy(mles + (n - 1) * L, f.one, 8 * L); /* last-row selector */
    build_eq(&f, icpt, nvars, mles + n * L);
    for (uint32_t s = 0; s < S; s++) {
        uint64_t *dst = up + ((size_t)J + s) * n * L;
        const size_t c = u->shift_amt[s];
        memcpy(dst, up + ((size_t)u->shift_src[s] * n + c) * L, 8 * L * (n - c));
    }
    zr_sc_group g;
    cpr_bufs bb;
    cpr_group(&f, u, apow, mles, (uint32_t)nmle, &g, &bb);
    size_t mdcap = 1024 + (size_t)nvars * (g.degree + 1) * 8 * L, mdlen = 0;
    uint8_t *md = (uint8_t *)malloc(mdcap);
    uint64_t *rstar = (uint64_t *)calloc(nvars, 8 * L), *fin = (uint64_t *)calloc(nmle, 8 * L);
    if (zr_sumcheck_prove(tr, f.p, L, nvars, 1, &g, 1, md, mdcap, &mdlen, rstar, fin)) rc = -3;
    cpr_bufs_free(&bb);
    for (size_t j = 2; j < nmle; j++) tr_absorb_field(tr, &f, fin + j * L);
    /* step 5: multipoint evaluation (multipoint_eval.rs:119-230) */
    uint64_t *mal = (uint64_t *)calloc(S ? S : 1, 8 * L), *mga = (uint64_t *)calloc(J, 8 * L);
    for (uint32_t s = 0; s < S; s++) tr_field_challenge(tr, &f, mal + (size_t)s * L);
    for (uint32_t j = 0; j < J; j++) tr_field_challenge(tr, &f, mga + (size_t)j * L);
    const size_t nmp = 2 + 2 * (size_t)S;
    uint64_t *mp = (uint64_t *)calloc(nmp * n, 8 * L);
    build_eq(&f, rstar, nvars, mp);
    for (uint32_t s = 0; s < S; s++) {
        const size_t c = u->shift_amt[s];
        memcpy(mp + ((1 + (size_t)s) * n + c) * L, mp, 8 * L * (n - c));
        memcpy(mp + ((2 + (size_t)S + s) * n) * L, up + (size_t)u->shift_src[s] * n * L, 8 * L * n);
    }
    {
        uint64_t *pre = mp + (1 + (size_t)S) * n * L;
        int nt = zr_get_threads();
        (void)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
        for (long b = 0; b < (long)n; b++) {
            uint64_t acc[4] = {0};
            for (uint32_t j = 0; j < J; j++) {
                uint64_t t[4];
                fmul(&f, mga + (size_t)j * L, up + ((size_t)j * n + (size_t)b) * L, t);
                fadd(&f, acc, t);
            }
            memcpy(pre + (size_t)b * L, acc, 8 * L);
        }
    }
    uint64_t *pc = (uint64_t *)calloc(1 + (size_t)S, 8 * L);
    uint32_t *po = (uint32_t *)calloc(2 + (size_t)S, 4), *pi = (uint32_t *)calloc(2 + 2 * (size_t)S, 4);
    memcpy(pc, f.one, 8 * L);
    pi[0] = 0;
    pi[1] = 1 + S;
    po[1] = 2;
    for (uint32_t s = 0; s < S; s++) {
        memcpy(pc + (1 + (size_t)s) * L, mal + (size_t)s * L, 8 * L);
        pi[2 + 2 * s] = 1 + s;
        pi[3 + 2 * s] = 2 + S + s;
        po[2 + s] = 4 + 2 * s;
    }
    zr_sc_group gm = {2, (uint32_t)nmp, 1 + S, mp, pc, po, pi, 0, NULL, NULL, NULL};
    size_t mpcap = 1024 + (size_t)nvars * 3 * 8 * L, mplen = 0;
    uint8_t *mpb = (uint8_t *)malloc(mpcap);
    uint64_t *r0 = (uint64_t *)calloc(nvars, 8 * L), *fin2 = (uint64_t *)calloc(nmp, 8 * L);
    if (!rc && zr_sumcheck_prove(tr, f.p, L, nvars, 0, &gm, 1, mpb, mpcap, &mplen, r0, fin2)) rc = -3;
    free(mp);
    /* step 6: lifted evaluations at r_0 (protocol/src/lib.rs:327-397), trimmed, absorbed */
    const uint32_t nlift = u->n_bin * D + u->n_int;
    uint64_t *lift = (uint64_t *)calloc(nlift ? nlift : 1, 8 * L);
    zr_piop_lifted_evals(f.p, L, bin, u->n_bin, D, ints, u->n_int, nvars, r0, lift);
    uint32_t *llen = (uint32_t *)calloc(J, 4);
    for (uint32_t c = 0; c < u->n_bin; c++) llen[c] = trim_len(&f, lift + (size_t)c * D * L, D);
    for (uint32_t c = 0; c < u->n_int; c++) llen[u->n_bin + c] = trim_len(&f, lift + ((size_t)u->n_bin * D + c) * L, 1);
    for (uint32_t c = 0; c < J; c++) {
        const uint64_t *q = c < u->n_bin ? lift + (size_t)c * D * L : lift + ((size_t)u->n_bin * D + c - u->n_bin) * L;
        for (uint32_t l = 0; l < llen[c]; l++) tr_absorb_field(tr, &f, q + (size_t)l * L);
    }
    /* step 7: prove_f of each committed table at r_0 */
    size_t zcap = (wb ? zr_proof_size(db, wb) : 0) + (wi ? zr_proof_size(di, wi) : 0) + 64, zlen = 0, part = 0;
    uint8_t *zip = (uint8_t *)malloc(zcap);
    uint8_t evb[32];
    if (!rc && wb) {
        if (zr_prove_f_on(db, bin + (size_t)u->n_pub_bin * n, wb, tr, f.p, r0, zip, zcap, &part, evb)) rc = -4;
        zlen += part;
    }
    if (!rc && wi) {
        if (zr_prove_f_on(di, ints + (size_t)u->n_pub_int * n, wi, tr, f.p, r0, zip + zlen, zcap - zlen, &part, evb))
            rc = -4;
        zlen += part;
    }
    /* the Proof transcription */
    if (!rc) {
        wbuf w = {out, 0, cap, 0};
        const uint64_t batches[3] = {wb, 0, wi};
        for (int r = 0; r < 3; r++) {
            wput(&w, roots[r], 32);
            wput(&w, &batches[r], 8);
        }
        put_sub(&w, zip, zlen);
        size_t scap = 4096 + 8 * L * ((size_t)K * (maxlen + 1) + nmle + (size_t)nlift + 8), slen;
        uint8_t *sb = (uint8_t *)malloc(scap), *sb2 = (uint8_t *)malloc(scap);
        wbuf s = {sb, 0, scap, 0};
        put_poly_vec(&s, &f, icv, maxlen, icl, K);
        put_sub(&w, sb, s.len);
        /* resolver: up evaluations, then down evaluations, each a sub-buffer */
        wbuf s2 = {sb2, 0, scap, 0};
        s.len = 0;
        put_field_vec(&s, &f, fin + 2 * L, J);
        put_sub(&s2, sb, s.len);
        s.len = 0;
        put_field_vec(&s, &f, fin + (2 + (size_t)J) * L, S);
        put_sub(&s2, sb, s.len);
        put_sub(&w, sb2, s2.len);
        put_sub(&w, md, mdlen);
        put_sub(&w, mpb, mplen);
        /* witness lifted evaluations: witness binary columns, then witness integer ones */
        s.len = 0;
        uint32_t nw = 0;
        uint64_t *wl = (uint64_t *)calloc((size_t)(wb + wi) * D + 1, 8 * L);
        uint32_t *wll = (uint32_t *)calloc(wb + wi + 1, 4);
        for (uint32_t c = u->n_pub_bin; c < u->n_bin; c++, nw++) {
            memcpy(wl + (size_t)nw * D * L, lift + (size_t)c * D * L, 8 * L * D);
            wll[nw] = llen[c];
        }
        for (uint32_t c = u->n_pub_int; c < u->n_int; c++, nw++) {
            memcpy(wl + (size_t)nw * D * L, lift + ((size_t)u->n_bin * D + c) * L, 8 * L);
            wll[nw] = llen[u->n_bin + c];
        }
        put_poly_vec(&s, &f, wl, D, wll, nw);
        put_sub(&w, sb, s.len);
        slen = w.len;
        *out_len = slen;
        if (w.overflow || s.overflow || s2.overflow) rc = -5;
        free(wl);
        free(wll);
        free(sb);
        free(sb2);
    }
    free(zip);
    free(llen);
    free(lift);
    free(r0);
    free(fin2);
    free(mpb);
    free(pc);
    free(po);
    free(pi);
    free(mal);
    free(mga);
    free(md);
    free(rstar);
    free(fin);
    free(apow);
    free(mles);
    free(icv);
    free(icl);
    free(icpt);
    zr_tr_free(tr);
    return rc;
}

/* ---------------------------------------------------------------- verifier */

static int get_sub(rbuf *r, rbuf *sub) {
    uint32_t l;
    if (rget(r, &l, 4) || r->pos + l > r->len) return -1;
    sub->p = r->p + r->pos;
    sub->len = l;
    sub->pos = 0;
    r->pos += l;
    return 0;
}

/* DynamicPolyVecF read: count polynomials of at most maxlen coefficients */
static int get_poly_vec(rbuf *r, const fcfg *f, uint32_t count, uint32_t maxlen, uint64_t *vals, uint32_t *lens) {
    if (!count) return r->pos == r->len ? 0 : -1;
    uint8_t flag;
    if (rget(r, &flag, 1) || flag > 1) return -1;
    if (flag) {
        uint64_t m[4] = {0};
        if (rget(r, m, 8 * f->L) || memcmp(m, f->p, 8 * f->L)) return -1;
    }
    for (uint32_t k = 0; k < count; k++) {
        if (rget(r, &lens[k], 4) || lens[k] > maxlen) return -1;
        if (!flag && lens[k]) return -1;
        if (rget(r, vals + (size_t)k * maxlen * f->L, 8 * f->L * (size_t)lens[k])) return -1;
        for (uint32_t l = 0; l < lens[k]; l++)
            if (ucmp(vals + ((size_t)k * maxlen + l) * f->L, f->p, f->L) >= 0) return -1;
    }
    return r->pos == r->len ? 0 : -1;
}

static int get_field_vec(rbuf *r, const fcfg *f, uint32_t count, uint64_t *vals) {
    if (!count) return r->len == 0 ? 0 : -1;
    uint64_t m[4] = {0};
    if (rget(r, m, 8 * f->L) || memcmp(m, f->p, 8 * f->L)) return -1;
    if (rget(r, vals, 8 * f->L * (size_t)count)) return -1;
    for (uint32_t i = 0; i < count; i++)
        if (ucmp(vals + (size_t)i * f->L, f->p, f->L) >= 0) return -1;
    return r->pos == r->len ? 0 : -1;
}

/* Horner: sum_l v_l x^l */
static void poly_eval(const fcfg *f, const uint64_t *v, uint32_t len, const uint64_t *x, uint64_t *out) {
    const uint32_t L = f->L;
    uint64_t acc[4] = {0};
    for (int l = (int)len - 1; l >= 0; l--) {
        uint64_t t[4];
        fmul(f, acc, x, t);
        memcpy(acc, t, 8 * L);
        fadd(f, acc, v + (size_t)l * L);
    }
    memcpy(out, acc, 8 * L);
}

static int verify_core(const zparams *z, const uint8_t root[32], uint32_t batch, zr_transcript *tr, const fcfg *f,
                       const uint64_t *pf, const uint64_t *eval_f, const i128 *alphas, rbuf *rd);

/* ZincPlusPiop::verify (protocol/src/verifier.rs:215-771) for the UAIR u:
 * public columns given (the first n_pub_bin / n_pub_int of each kind, each
 * 2^nvars entries), the proof bytes parsed as Proof::read_transcription_bytes_exact
 * (protocol/src/lib.rs:93-133).  0 = accept; otherwise the step that failed:
 * 1 parse, 2 ideal check, 4 CPR / sumcheck, 5 multipoint, 6 lifted evaluations,
 * 7 PCS. */
int zr_zinc_verify(const zr_desc *db, const zr_desc *di, uint32_t nvars, const uint64_t *pub_bin,
                   const int64_t *pub_int, const zr_uair *u, uint32_t L, const uint8_t *proof, size_t len) {
    if (nvars < 2 || L < 1 || L > 4) return 1;
    const size_t n = (size_t)1 << nvars;
    const uint32_t J = uair_ncols(u), S = u->n_shifts, K = u->n_cons, D = u->D;
    const uint32_t wb = u->n_bin - u->n_pub_bin, wi = u->n_int - u->n_pub_int;
    rbuf rd = {proof, len, 0};
    uint8_t roots[3][32];
    uint64_t batches[3];
    for (int r = 0; r < 3; r++)
        if (rget(&rd, roots[r], 32) || rget(&rd, &batches[r], 8)) return 1;
    if (batches[0] != wb || batches[1] != 0 || batches[2] != wi) return 1;
    rbuf zip, ics, res, mds, mps, wls;
    if (get_sub(&rd, &zip) || get_sub(&rd, &ics) || get_sub(&rd, &res) || get_sub(&rd, &mds) || get_sub(&rd, &mps) ||
        get_sub(&rd, &wls) || rd.pos != rd.len)
        return 1;
    int rc = 0;
    zr_transcript *tr = zr_tr_new();
    for (int r = 0; r < 3; r++) zr_tr_absorb_slice(tr, roots[r], 32);
    /* public columns, laid out as the prover's (binary then integer) */
    absorb_public(tr, u, pub_bin, pub_int, nvars);
    uint64_t prime[4] = {0};
    zr_tr_get_prime(tr, L, prime);
    fcfg f;
    fcfg_init(&f, prime, L);
    uint32_t maxlen = 1;
    for (uint32_t k = 0; k < K; k++) maxlen = cons_len(u, k) > maxlen ? cons_len(u, k) : maxlen;
    uint64_t *icv = (uint64_t *)calloc((size_t)K * maxlen + 1, 8 * L);
    uint32_t *icl = (uint32_t *)calloc(K + 1, 4);
    uint64_t *icpt = (uint64_t *)calloc(nvars, 8 * L);
    uint64_t *ups = (uint64_t *)calloc((size_t)J + S + 1, 8 * L);
    uint64_t *apow = (uint64_t *)calloc(K + 1, 8 * L);
    uint64_t *rstar = (uint64_t *)calloc(nvars, 8 * L), *r0 = (uint64_t *)calloc(nvars, 8 * L);
    uint64_t *mal = (uint64_t *)calloc(S + 1, 8 * L), *mga = (uint64_t *)calloc(J, 8 * L);
    uint64_t *lifts = (uint64_t *)calloc((size_t)J * D, 8 * L);
    uint32_t *llen = (uint32_t *)calloc(J, 4);
    uint8_t *mdcopy = NULL;
    /* step 2: ideal check (ideal_check.rs:242-290) */
    {
        if (get_poly_vec(&ics, &f, K, maxlen, icv, icl)) { rc = 1; goto done; }
        for (uint32_t k = 0; k < nvars; k++) tr_field_challenge(tr, &f, icpt + (size_t)k * L);
        for (uint32_t k = 0; k < K; k++)
            for (uint32_t l = 0; l < icl[k]; l++) tr_absorb_field(tr, &f, icv + ((size_t)k * maxlen + l) * L);
        for (uint32_t k = 0; k < K; k++) {
            if (u->ideal_kind[k] == 0) continue; /* the zero ideal is not checked */
            uint64_t root[4], v[4];
            f_from_i64(&f, u->ideal_root[k], root);
            poly_eval(&f, icv + (size_t)k * maxlen * L, icl[k], root, v);
            if (!uiszero(v, L)) { rc = 2; goto done; }
        }
    }
    /* step 3: the projecting element */
    uint64_t a[4];
    f_from_i128(&f, tr_i128(tr), a);
    /* step 4: CPR prepare_verifier, MultiDegreeSumcheck verify, finalize_verifier
     * (combined_poly_resolver.rs:268-440) */
    {
        rbuf up_b, down_b;
        if (get_sub(&res, &up_b) || get_sub(&res, &down_b) || res.pos != res.len) { rc = 1; goto done; }
        if (get_field_vec(&up_b, &f, J, ups) || get_field_vec(&down_b, &f, S, ups + (size_t)J * L)) { rc = 1; goto done; }
        uint64_t alpha[4];
        tr_field_challenge(tr, &f, alpha);
        f_powers(&f, alpha, K, apow);
        uint64_t expected[4] = {0};
        for (uint32_t k = 0; k < K; k++) {
            uint64_t v[4], t[4];
            poly_eval(&f, icv + (size_t)k * maxlen * L, icl[k], a, v);
            fmul(&f, v, apow + (size_t)k * L, t);
            fadd(&f, expected, t);
        }
        /* the claimed sum is the last field element of the MultiDegreeSumcheckProof */
        const uint32_t deg = uair_max_degree(u) + 2;
        if (mds.len < 8 * L) { rc = 1; goto done; }
        if (memcmp(mds.p + mds.len - 8 * L, expected, 8 * L)) { rc = 4; goto done; }
        uint64_t exp_eval[4];
        if (zr_sumcheck_verify(tr, f.p, L, nvars, 1, &deg, 1, mds.p, mds.len, rstar, exp_eval)) { rc = 4; goto done; }
        uint64_t eqv[4], ones[4 * 32], sel[4], folded[4], t1[4], t2[4];
        eq_eval_pts(&f, rstar, icpt, nvars, eqv);
        for (uint32_t k = 0; k < nvars; k++) memcpy(ones + (size_t)k * L, f.one, 8 * L);
        eq_eval_pts(&f, rstar, ones, nvars, sel);
        cpr_folded(&f, u, apow, ups, folded);
        uint64_t oms[4];
        memcpy(oms, f.one, 8 * L);
        fsub(&f, oms, sel);
        fmul(&f, eqv, oms, t1);
        fmul(&f, t1, folded, t2);
        if (memcmp(t2, exp_eval, 8 * L)) { rc = 4; goto done; }
        for (uint32_t j = 0; j < J + S; j++) tr_absorb_field(tr, &f, ups + (size_t)j * L);
    }
    /* step 5: multipoint evaluation (multipoint_eval.rs:242-300) */
    uint64_t mp_exp[4];
    {
        for (uint32_t s = 0; s < S; s++) tr_field_challenge(tr, &f, mal + (size_t)s * L);
        for (uint32_t j = 0; j < J; j++) tr_field_challenge(tr, &f, mga + (size_t)j * L);
        uint64_t expected[4] = {0};
        for (uint32_t j = 0; j < J; j++) {
            uint64_t t[4];
            fmul(&f, mga + (size_t)j * L, ups + (size_t)j * L, t);
            fadd(&f, expected, t);
        }
        for (uint32_t s = 0; s < S; s++) {
            uint64_t t[4];
            fmul(&f, mal + (size_t)s * L, ups + ((size_t)J + s) * L, t);
            fadd(&f, expected, t);
        }
        if (mps.len < 8 * L || memcmp(mps.p + mps.len - 8 * L, expected, 8 * L)) { rc = 5; goto done; }
        const uint32_t deg2 = 2;
        if (zr_sumcheck_verify(tr, f.p, L, nvars, 0, &deg2, 1, mps.p, mps.len, r0, mp_exp)) { rc = 5; goto done; }
    }
    /* step 6: all lifted evaluations (public recomputed), the subclaim, absorb */
    {
        uint64_t *wl = (uint64_t *)calloc((size_t)(wb + wi) * D + 1, 8 * L);
        uint32_t *wll = (uint32_t *)calloc(wb + wi + 1, 4);
        if (get_poly_vec(&wls, &f, wb + wi, D, wl, wll)) {
            free(wl);
            free(wll);
            rc = 1;
            goto done;
        }
        for (uint32_t q = 0; q < wb + wi; q++)
            if (q >= wb && wll[q] > 1) {
                free(wl);
                free(wll);
                rc = 1;
                goto done;
            }
        if (u->n_pub_bin + u->n_pub_int) {
            uint64_t *pl = (uint64_t *)calloc((size_t)(u->n_pub_bin * D + u->n_pub_int) + 1, 8 * L);
            zr_piop_lifted_evals(f.p, L, pub_bin, u->n_pub_bin, D, pub_int, u->n_pub_int, nvars, r0, pl);
            for (uint32_t c = 0; c < u->n_pub_bin; c++) {
                memcpy(lifts + (size_t)c * D * L, pl + (size_t)c * D * L, 8 * L * D);
                llen[c] = trim_len(&f, pl + (size_t)c * D * L, D);
            }
            for (uint32_t c = 0; c < u->n_pub_int; c++) {
                memcpy(lifts + ((size_t)u->n_bin + c) * D * L, pl + ((size_t)u->n_pub_bin * D + c) * L, 8 * L);
                llen[u->n_bin + c] = trim_len(&f, pl + ((size_t)u->n_pub_bin * D + c) * L, 1);
            }
            free(pl);
        }
        for (uint32_t q = 0; q < wb; q++) {
            memcpy(lifts + ((size_t)u->n_pub_bin + q) * D * L, wl + (size_t)q * D * L, 8 * L * D);
            llen[u->n_pub_bin + q] = wll[q];
        }
        for (uint32_t q = 0; q < wi; q++) {
            memcpy(lifts + ((size_t)u->n_bin + u->n_pub_int + q) * D * L, wl + ((size_t)wb + q) * D * L, 8 * L);
            llen[u->n_bin + u->n_pub_int + q] = wll[wb + q];
        }
        free(wl);
        free(wll);
        /* verify_subclaim: eq(r0, r*) sum_j gamma_j open_j + sum_s alpha_s S_c(r*, r0) open_src */
        uint64_t *open = (uint64_t *)calloc(J, 8 * L);
        for (uint32_t c = 0; c < J; c++) poly_eval(&f, lifts + (size_t)c * D * L, llen[c], a, open + (size_t)c * L);
        uint64_t up_b[4] = {0}, eqv[4], total[4], t[4];
        for (uint32_t j = 0; j < J; j++) {
            fmul(&f, mga + (size_t)j * L, open + (size_t)j * L, t);
            fadd(&f, up_b, t);
        }
        eq_eval_pts(&f, r0, rstar, nvars, eqv);
        fmul(&f, eqv, up_b, total);
        for (uint32_t s = 0; s < S; s++) {
            uint64_t sp[4], t2[4];
            shift_pred_eval(&f, rstar, r0, nvars, u->shift_amt[s], sp);
            fmul(&f, mal + (size_t)s * L, sp, t);
            fmul(&f, t, open + (size_t)u->shift_src[s] * L, t2);
            fadd(&f, total, t2);
        }
        free(open);
        if (memcmp(total, mp_exp, 8 * L)) { rc = 6; goto done; }
        for (uint32_t c = 0; c < J; c++)
            for (uint32_t l = 0; l < llen[c]; l++) tr_absorb_field(tr, &f, lifts + ((size_t)c * D + l) * L);
    }
    /* step 7: PCS verification at r_0, witness columns only (verifier.rs:606-700) */
    {
        const zr_desc *descs[2] = {db, di};
        const uint32_t batch[2] = {wb, wi}, first[2] = {u->n_pub_bin, u->n_bin + u->n_pub_int};
        for (int tbl = 0; tbl < 2 && !rc; tbl++) {
            if (!batch[tbl]) continue;
            zparams z;
            if (zparams_build(descs[tbl], &z) || z.d.field_limbs != L) { rc = 7; break; }
            const uint32_t na = z.D > 1 ? z.D : 1;
            i128 *al = (i128 *)malloc(sizeof(i128) * batch[tbl] * na);
            for (uint32_t b = 0; b < batch[tbl]; b++) {
                if (z.D > 1)
                    for (uint32_t i = 0; i < z.D; i++) al[b * z.D + i] = tr_i128(tr);
                else al[b] = 1;
            }
            uint64_t ev[4] = {0};
            for (uint32_t b = 0; b < batch[tbl]; b++) {
                const uint32_t c = first[tbl] + b;
                for (uint32_t l = 0; l < llen[c] && l < na; l++) {
                    uint64_t fa[4], t[4];
                    f_from_i128(&f, al[b * na + l], fa);
                    fmul(&f, fa, lifts + ((size_t)c * D + l) * L, t);
                    fadd(&f, ev, t);
                }
            }
            if (verify_core(&z, tbl == 0 ? roots[0] : roots[2], batch[tbl], tr, &f, r0, ev, al, &zip)) rc = 7;
            free(al);
            zparams_free(&z);
        }
        if (!rc && zip.pos != zip.len) rc = 7;
    }
done:
    free(mdcopy);
    free(icv);
    free(icl);
    free(icpt);
    free(ups);
    free(apow);
    free(rstar);
    free(r0);
    free(mal);
    free(mga);
    free(lifts);
    free(llen);
    zr_tr_free(tr);
    (void)n;
    return rc;
}
