"""Shared helpers of the tests: seeded inputs and parameter construction."""
import numpy as np

from oracle import oracle as O


def binary_evals(rng, n, D):
    """n BinaryPoly<D> evaluations with Bernoulli(0.5) coefficients, u64-packed."""
    bits = rng.integers(0, 2, size=(n, D), dtype=np.uint64)
    w = np.left_shift(np.uint64(1), np.arange(D, dtype=np.uint64))
    return (bits * w).sum(axis=1, dtype=np.uint64)


def i32_evals(rng, n, lo=-(2**15), hi=2**15):
    return rng.integers(lo, hi, size=n, dtype=np.int32)


def i64_evals(rng, n):
    """n i64 evaluations over the whole range."""
    return rng.integers(-(2**63), 2**63 - 1, size=n, dtype=np.int64, endpoint=True)


def desc_for(eval_kind, D, code_kind, num_vars, row_len, depth=0, rep=4, comb=None, field=4,
             openings=147):
    return O.make_desc(eval_kind, D, code_kind, num_vars, row_len, depth=depth, rep=rep,
                       comb_limbs=comb, field_limbs=field, num_openings=openings)


def params_for(Z, eval_kind, D, code_kind, num_vars, row_len, depth=0, rep=4, device=True,
               ctx=None, comb=None, field=4, openings=147):
    zt = Z.ZipTypes(eval_kind, D if eval_kind == Z.EVAL_BINPOLY else 1,
                    comb if comb else {Z.EVAL_I32: 3, Z.EVAL_I64: 6}.get(eval_kind, 5), field, openings)
    code = (Z.IprsCode(row_len, depth, rep) if code_kind == Z.CODE_IPRS else
            Z.RaaCode(row_len, rep) if code_kind == Z.CODE_RAA else Z.RaaSignFlippingCode(row_len, rep))
    return Z.ZipPlus.setup(1 << num_vars, code, zt, ctx=ctx, device=device)
