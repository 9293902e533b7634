/*
 * zipref: CPU restatement of the Zip+ commit/prove/verify path of
 * NethermindEth/zinc-plus, used ONLY as test infrastructure (the checker) and
 * as the timed CPU baseline.  Nothing in the product links this code.
 *
 * Parity status: pinned by the reference's own known-answer tests (octet
 * reversal, F65537 twiddles, pNTT == NTT mod 65537, RAA 16-element codeword,
 * Merkle round trip, proof-size formula) and by the `blake3` Python wheel for
 * every hash.  Montgomery-form field bytes follow crypto-bigint MontyForm
 * (R = 2^(64*LIMBS)); the reference ships no golden proof bytes, so byte
 * parity of whole proofs is anchored on those pins, not on reference output.
 */
#ifndef ZIPREF_H
#define ZIPREF_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ZR_EVAL_I32 = 0, ZR_EVAL_BINPOLY = 1, ZR_EVAL_I64 = 2 };
enum { ZR_CODE_IPRS = 0, ZR_CODE_RAA = 1, ZR_CODE_RAA_SIGN_FLIP = 2 };

/* Same meaning as the product's zg_params_desc. */
typedef struct {
    uint32_t eval_kind;
    uint32_t degree_plus_one;
    uint32_t code_kind;
    uint32_t rep;
    uint32_t num_vars;
    uint32_t row_len;
    uint32_t iprs_depth; /* 0 => optimal depth */
    uint32_t comb_limbs;
    uint32_t field_limbs;
    uint32_t num_openings;
} zr_desc;

/* BLAKE3 */
void zr_blake3(const uint8_t *in, size_t n, uint8_t out[32]);
void zr_blake3_xof(const uint8_t *in, size_t n, uint8_t *out, size_t out_len);
void zr_blake3_chunk_cv(const uint8_t *in, size_t n, uint64_t counter, uint8_t out[32]);
void zr_blake3_parent(const uint8_t l[32], const uint8_t r[32], int root, uint8_t out[32]);

/* pNTT pieces */
size_t zr_octet_reversal(size_t x, size_t num_octets);
uint32_t zr_iprs_optimal_depth(uint32_t row_len);
int zr_iprs_dims(uint32_t row_len, uint32_t depth, uint32_t rep, uint32_t out[4]);
int zr_iprs_tables(uint32_t row_len, uint32_t depth, uint32_t rep, int64_t *base_matrix,
                   int64_t *twiddles);
int zr_roots_of_unity(uint32_t n, int64_t *out);

/* rand 0.9 StdRng shuffle of 0..n */
void zr_shuffle_identity(uint64_t seed, uint32_t n, uint32_t *perm);
uint32_t zr_stdrng_u32(uint64_t seed, uint32_t index);

/* encodings (row-major rows of Cw) */
int zr_encode_rows(const zr_desc *d, const void *evals, void *cw_out);
/* encode_wide over Int<limbs> rows (verifier side) */
int zr_encode_wide(const zr_desc *d, const uint64_t *row, uint32_t limbs, uint64_t *out);

size_t zr_cw_bytes(const zr_desc *d);
size_t zr_eval_bytes(const zr_desc *d);
uint32_t zr_num_rows(const zr_desc *d);
uint32_t zr_codeword_len(const zr_desc *d);

/* Merkle */
int zr_merkle_root_rows(const uint8_t *rows, uint32_t n_rows, uint32_t width, uint32_t elem_bytes,
                        uint8_t root[32]);

/* Commit/prove/verify.  polys: batch eval arrays laid out back to back. */
int zr_commit(const zr_desc *d, const void *polys, uint32_t batch, uint8_t root[32]);
/* point: num_vars i128 values as (lo,hi) int64 pairs.  proof/eval buffers
 * sized by zr_proof_size / 8*field_limbs. */
size_t zr_proof_size(const zr_desc *d, uint32_t batch);
int zr_commit_prove(const zr_desc *d, const void *polys, uint32_t batch, const int64_t *point,
                    uint8_t root[32], uint8_t *proof, size_t proof_cap, size_t *proof_len,
                    uint8_t *eval_out, uint8_t *modulus_out);
/* The same with prove_f's field-valued point, given as unsigned 256-bit integers. */
int zr_commit_prove_f(const zr_desc *d, const void *polys, uint32_t batch, const uint64_t *point_u256,
                      uint8_t root[32], uint8_t *proof, size_t proof_cap, size_t *proof_len, uint8_t *eval_out,
                      uint8_t *modulus_out);
int zr_verify(const zr_desc *d, const uint8_t root[32], uint32_t batch, const int64_t *point,
              const uint8_t *eval_inner, const uint8_t *proof, size_t proof_len);

/* FS transcript (Blake3Transcript) for direct tests */
typedef struct zr_transcript zr_transcript;
/* ZipPlus::prove_f on a transcript already in use, point in the field of
 * `modulus` (Montgomery inners); appends nothing but writes the proof bytes. */
int zr_prove_f_on(const zr_desc *d, const void *polys, uint32_t batch, zr_transcript *tr,
                  const uint64_t *modulus, const uint64_t *point_f, uint8_t *proof, size_t proof_cap,
                  size_t *proof_len, uint8_t *eval_out);
zr_transcript *zr_tr_new(void);
void zr_tr_free(zr_transcript *t);
void zr_tr_absorb(zr_transcript *t, const uint8_t *buf, size_t n);
void zr_tr_absorb_slice(zr_transcript *t, const uint8_t *buf, size_t n);
void zr_tr_challenge(zr_transcript *t, uint8_t *out, size_t n);
void zr_tr_get_prime(zr_transcript *t, uint32_t limbs, uint64_t *prime_out);
int zr_is_probable_prime_base2(const uint64_t *n, uint32_t limbs);

/* Sumcheck with a combination function made of a sum of products times
 * affine factors:
 * comb(v) = (sum_k coeffs[k] * prod_{q in [offsets[k], offsets[k+1])} v[indices[q]])
 *           * prod_f (factor_a[f] + factor_b[f] * v[factor_mles[f]]).
 * mles: n_mles x 2^nvars field elements (Montgomery inner, L limbs). */
typedef struct {
    uint32_t degree, n_mles, n_products;
    const uint64_t *mles;
    const uint64_t *coeffs;
    const uint32_t *offsets;
    const uint32_t *indices;
    uint32_t n_factors;
    const uint32_t *factor_mles;
    const uint64_t *factor_a, *factor_b;
} zr_sc_group;
int zr_sumcheck_prove(zr_transcript *t, const uint64_t *modulus, uint32_t L, uint32_t nvars,
                      int multi, const zr_sc_group *groups, uint32_t ngroups, uint8_t *proof,
                      size_t cap, size_t *plen, uint64_t *point_out, uint64_t *finals_out);
int zr_sumcheck_verify(zr_transcript *t, const uint64_t *modulus, uint32_t L, uint32_t nvars,
                       int multi, const uint32_t *degrees, uint32_t ngroups, const uint8_t *proof,
                       size_t len, uint64_t *point_out, uint64_t *expected_out);
void zr_sumcheck_comb(const uint64_t *modulus, uint32_t L, const zr_sc_group *g,
                      const uint64_t *vals, uint64_t *out);
void zr_mle_evaluate(const uint64_t *modulus, uint32_t L, const uint64_t *mle, uint32_t nvars,
                     const uint64_t *point, uint64_t *out);
/* Zinc+ prover step 3 (evaluation projection) and step 6 (lifted evaluations)
 * on binary-polynomial and i64 trace columns; see zipref.c. */
void zr_piop_eval_projection(const uint64_t *modulus, uint32_t L, const uint64_t *bin, uint32_t n_bin,
                             uint32_t D, const int64_t *ints, uint32_t n_int, uint32_t nvars,
                             const uint64_t *a, uint64_t *out);
void zr_tr_field_challenge(zr_transcript *t, const uint64_t *modulus, uint32_t L, uint64_t *out);
void zr_tr_absorb_field(zr_transcript *t, const uint64_t *modulus, uint32_t L, const uint64_t *inner);
void zr_piop_lifted_evals(const uint64_t *modulus, uint32_t L, const uint64_t *bin, uint32_t n_bin,
                          uint32_t D, const int64_t *ints, uint32_t n_int, uint32_t nvars,
                          const uint64_t *point, uint64_t *out);

/* A UAIR as a constraint system over the columns [binary up..., integer up...,
 * down (one per shift)]: constraint k is sum over its terms t of
 * term_coeff[t] * prod_{q in [fac_off[t], fac_off[t+1])} column fac_col[q],
 * in the zero ideal (ideal_kind 0) or in (X - ideal_root[k]) (ideal_kind 1).
 * The first n_pub_bin / n_pub_int columns of each kind are public. */
typedef struct {
    uint32_t n_bin, n_int, n_pub_bin, n_pub_int, D;
    uint32_t n_shifts;
    const uint32_t *shift_src, *shift_amt;
    uint32_t n_cons;
    const uint32_t *term_off;
    const int64_t *term_coeff;
    const uint32_t *fac_off;
    const uint32_t *fac_col;
    const uint8_t *ideal_kind;
    const int64_t *ideal_root;
} zr_uair;
/* ZincPlusPiop::prove (MLE first or combined) and ZincPlusPiop::verify; see
 * zinc_piop.c.  bin: n_bin x 2^nvars BinaryPoly<D>, ints: n_int x 2^nvars. */
int zr_zinc_prove(const zr_desc *db, const zr_desc *di, uint32_t nvars, const uint64_t *bin, const int64_t *ints,
                  const zr_uair *u, uint32_t L, int mle_first, uint8_t *out, size_t cap, size_t *out_len);
int zr_zinc_verify(const zr_desc *db, const zr_desc *di, uint32_t nvars, const uint64_t *pub_bin,
                   const int64_t *pub_int, const zr_uair *u, uint32_t L, const uint8_t *proof, size_t len);

/* LinearCode::encode_f: row (row_len Montgomery inners of L limbs) -> out
 * (codeword_len inners), over the prime `modulus`; see zipref.c. */
int zr_encode_f(const zr_desc *d, const uint64_t *modulus, uint32_t L, const uint64_t *row, uint64_t *out);

/* threads used by the parallel regions */
void zr_set_threads(int n);
int zr_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
