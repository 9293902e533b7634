// Argument bundles of the prove-phase kernels.
#pragma once
#include "zg_internal.h"

namespace zg {

struct ProjectArgs {
    const void *evals;      // batch polys back to back
    int binary;             // 1: ZG_EVAL_BINPOLY, 0: ZG_EVAL_I32, 2: ZG_EVAL_I64
    const i128 *alphas;     // batch x D
    uint32_t D;
    uint64_t dmask;
    const uint64_t *q1;     // row_len field elements (Montgomery)
    uint32_t row_len, num_rows, batch, comb_limbs;
    const FieldCfg *f;
    uint64_t *wprime;       // batch x num_rows x row_len x comb_limbs
    uint64_t *partial;      // batch x num_rows x ceil(row_len/256) x L (summed on the host)
};

struct CombineArgs {
    const uint64_t *wprime;
    const i128 *coeffs;     // num_rows
    uint32_t batch, num_rows, row_len, comb_limbs;
    uint64_t *comb_out;     // row_len x comb_limbs
    const uint8_t *cw;      // leaf-major codeword
    uint32_t leaf_bytes;
    const uint8_t *tree;
    uint32_t depth, width, n_open;
    const uint32_t *idxs;
    uint8_t *open_out;
};

zg_status launch_eq_table(zg_ctx *ctx, const uint64_t *r_d, const uint64_t *omr_d, uint32_t n,
                          const FieldCfg &f, uint64_t *out_d, cudaStream_t s);
zg_status launch_project_rows(zg_ctx *ctx, const ProjectArgs &a, cudaStream_t s);
zg_status launch_combined_and_openings(zg_ctx *ctx, const CombineArgs &a, cudaStream_t s);

}  // namespace zg
