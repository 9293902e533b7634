"""Zinc+ prover steps 3 and 6 on the trace columns (protocol/src/prover.rs:
385-415 and 497-532): the evaluation projection (project_trace_coeffs +
evaluate_trace_to_column_mles, piop/src/projections.rs:140-301) and the lifted
evaluations (compute_lifted_evals, protocol/src/lib.rs:327-395).  The oracle is
checked against the definitions written out with Python integers; the GPU is
checked against the oracle."""
import ctypes as C

import numpy as np
import pytest

from util import binary_evals


def field(oracle, L):
    t = oracle.Transcript()
    t.absorb_slice(b"piop-steps")
    return t.get_prime(L)


def inner(v, p, L):
    """Montgomery inner limbs of the standard value v."""
    x = (v % p) * (1 << (64 * L)) % p
    return [(x >> (64 * i)) & ((1 << 64) - 1) for i in range(L)]


def std(limbs, p, L):
    x = sum(int(w) << (64 * i) for i, w in enumerate(limbs))
    return x * pow(1 << (64 * L), -1, p) % p


def columns(rng, n_bin, n_int, nv, D):
    b = np.stack([binary_evals(rng, 1 << nv, D) for _ in range(n_bin)]) if n_bin else None
    i = rng.integers(-2**62, 2**62, size=(n_int, 1 << nv), dtype=np.int64) if n_int else None
    return b, i


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_eval_projection_is_the_definition(oracle, L):
    p, nv, D = field(oracle, L), 3, 5
    rng = np.random.default_rng(L)
    b, i = columns(rng, 2, 1, nv, D)
    a = int.from_bytes(rng.bytes(8 * L), "little") % p
    got = oracle.piop_eval_projection(p, L, b, D, i, nv, np.array(inner(a, p, L), np.uint64))
    for c in range(2):
        for x in range(1 << nv):
            want = sum(pow(a, l, p) for l in range(D) if (int(b[c, x]) >> l) & 1) % p
            assert std(got[c, x], p, L) == want
    for x in range(1 << nv):
        assert std(got[2, x], p, L) == int(i[0, x]) % p


@pytest.mark.parametrize("L", [3, 4])
def test_oracle_lifted_evals_is_the_definition(oracle, L):
    p, nv, D = field(oracle, L), 4, 6
    rng = np.random.default_rng(10 + L)
    b, i = columns(rng, 2, 1, nv, D)
    r = [int.from_bytes(rng.bytes(8 * L), "little") % p for _ in range(nv)]
    got = oracle.piop_lifted_evals(p, L, b, D, i, nv, np.array([inner(v, p, L) for v in r], np.uint64))

    def eq(x):
        e = 1
        for k in range(nv):
            e = e * (r[k] if (x >> k) & 1 else 1 - r[k]) % p
        return e

    for c in range(2):
        for l in range(D):
            want = sum(eq(x) for x in range(1 << nv) if (int(b[c, x]) >> l) & 1) % p
            assert std(got[c * D + l], p, L) == want
    assert std(got[2 * D], p, L) == sum(eq(x) * int(i[0, x]) for x in range(1 << nv)) % p


def test_entry_points_reject_null_context(zipgpu):
    out = np.zeros(3, np.uint64)
    mod = (7).to_bytes(24, "little")
    assert zipgpu.lib().zg_piop_eval_projection(None, mod, 3, None, 0, 32, None, 0, 4, out.ctypes.data, 0,
                                                out.ctypes.data) != 0


@pytest.mark.gpu
@pytest.mark.parametrize("L,D,n_bin,n_int,nv", [(3, 32, 4, 2, 10), (4, 64, 2, 1, 9), (3, 5, 3, 0, 12),
                                                (3, 32, 16, 1, 14), (4, 32, 0, 2, 8)])
def test_gpu_eval_projection_matches_oracle(zipgpu, oracle, ctx, L, D, n_bin, n_int, nv):
    p = field(oracle, L)
    rng = np.random.default_rng(100 + nv)
    b, i = columns(rng, n_bin, n_int, nv, D)
    a = np.array(inner(int.from_bytes(rng.bytes(8 * L), "little"), p, L), np.uint64)
    got = zipgpu.ZincPiop.eval_projection(ctx, p, L, b, D, i, nv, a)
    assert np.array_equal(got, oracle.piop_eval_projection(p, L, b, D, i, nv, a))


@pytest.mark.gpu
@pytest.mark.parametrize("L,D,n_bin,n_int,nv", [(3, 32, 4, 2, 10), (4, 64, 2, 1, 13), (3, 7, 3, 0, 12),
                                                (3, 32, 16, 1, 14), (4, 32, 0, 2, 8), (3, 32, 2, 1, 1)])
def test_gpu_lifted_evals_match_oracle(zipgpu, oracle, ctx, L, D, n_bin, n_int, nv):
    p = field(oracle, L)
    rng = np.random.default_rng(200 + nv)
    b, i = columns(rng, n_bin, n_int, nv, D)
    r = np.array([inner(int.from_bytes(rng.bytes(8 * L), "little"), p, L) for _ in range(nv)], np.uint64)
    got = zipgpu.ZincPiop.lifted_evals(ctx, p, L, b, D, i, nv, r)
    assert np.array_equal(got, oracle.piop_lifted_evals(p, L, b, D, i, nv, r))


@pytest.mark.gpu
def test_gpu_piop_argument_errors(zipgpu, oracle, ctx):
    p = field(oracle, 3)
    b = np.zeros((1, 16), np.uint64)
    with pytest.raises(zipgpu.ZipError):  # two-limb field
        zipgpu.ZincPiop.lifted_evals(ctx, p % (1 << 128) | 1, 2, b, 32, None, 4, np.zeros((4, 2), np.uint64))
    with pytest.raises(zipgpu.ZipError):  # even modulus
        zipgpu.ZincPiop.eval_projection(ctx, p - 1, 3, b, 32, None, 4, np.zeros(3, np.uint64))
    with pytest.raises(zipgpu.ZipError):  # BinaryPoly width above 64
        zipgpu.ZincPiop.eval_projection(ctx, p, 3, b, 65, None, 4, np.zeros(3, np.uint64))
