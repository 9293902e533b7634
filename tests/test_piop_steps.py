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


# ------------------------------------------------------------------ step 5
def mp_case(oracle, L, nv, ncols, seed):
    p = field(oracle, L)
    rng = np.random.default_rng(seed)
    mles = np.array([[inner(int.from_bytes(rng.bytes(8 * L), "little"), p, L) for _ in range(1 << nv)]
                     for _ in range(ncols)], np.uint64)
    r = np.array([inner(int.from_bytes(rng.bytes(8 * L), "little"), p, L) for _ in range(nv)], np.uint64)
    return p, mles, r


@pytest.mark.parametrize("L,nv,ncols,shifts", [(3, 4, 3, [(0, 1), (2, 3)]), (4, 3, 2, [(1, 1)]),
                                               (3, 5, 4, []), (3, 4, 3, [(1, 1), (1, 1), (0, 0), (2, 1)])])
def test_oracle_multipoint_claim_is_the_batched_evaluations(oracle, L, nv, ncols, shifts):
    """The proof's claimed sum is compute_expected_sum (multipoint_eval.rs:216-219):
    sum_j gamma_j v_j(r') + sum_k alpha_k down_k, down_k = sum_b next_c(r', b) v_src(b),
    and the oracle's sumcheck verifier accepts the proof at the returned point."""
    p, mles, r = mp_case(oracle, L, nv, ncols, 40 + nv)
    proof, r0 = oracle.piop_multipoint_eval(oracle.Transcript(), p, L, mles, r, shifts)
    twin = oracle.Transcript()
    alphas = [std(twin.field_challenge(p, L), p, L) for _ in shifts]
    gammas = [std(twin.field_challenge(p, L), p, L) for _ in range(ncols)]
    rs = [std(v, p, L) for v in r]
    n = 1 << nv

    def eq(b):
        e = 1
        for k in range(nv):
            e = e * (rs[k] if (b >> k) & 1 else 1 - rs[k]) % p
        return e

    col = [[std(mles[j, b], p, L) for b in range(n)] for j in range(ncols)]
    up = [sum(eq(b) * col[j][b] for b in range(n)) % p for j in range(ncols)]
    down = [sum(eq(b - c) * col[sc][b] for b in range(c, n)) % p for sc, c in shifts]
    want = (sum(g * u for g, u in zip(gammas, up)) + sum(a * d for a, d in zip(alphas, down))) % p
    claimed = int.from_bytes(proof[-8 * L:], "little") * pow(1 << (64 * L), -1, p) % p
    assert claimed == want
    t2 = oracle.Transcript()  # the verifier draws the same alphas and gammas first
    for _ in range(len(shifts) + ncols):
        t2.field_challenge(p, L)
    rc, vpt, _exp = oracle.sumcheck_verify(t2, p, L, nv, [2], proof, False)
    assert rc == 0 and (vpt == r0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("L,nv,ncols,shifts", [(3, 6, 3, [(0, 1), (2, 3)]), (4, 8, 5, [(4, 7), (0, 1), (1, 2)]),
                                               (3, 10, 17, [(k + 1, 1) for k in range(16)]), (3, 5, 2, []),
                                               # a repeated (src, amount) pair and amount 0 among others:
                                               # the shift terms' weights are summed per amount and source
                                               (3, 6, 3, [(1, 1), (1, 1), (0, 0), (2, 1)]),
                                               (4, 7, 4, [(3, 0), (0, 2), (3, 0), (0, 2), (1, 2), (2, 5)])])
def test_gpu_multipoint_eval_matches_oracle(zipgpu, oracle, ctx, L, nv, ncols, shifts):
    p, mles, r = mp_case(oracle, L, nv, ncols, 60 + nv)
    want_proof, want_r0 = oracle.piop_multipoint_eval(oracle.Transcript(), p, L, mles, r, shifts)
    t = zipgpu.PcsProverTranscript()
    proof, r0 = zipgpu.ZincPiop.multipoint_eval(ctx, t, p, L, mles, nv, r, shifts)
    t.close()
    assert proof == want_proof and np.array_equal(r0, want_r0)


@pytest.mark.gpu
def test_gpu_steps_3_and_5_chain_on_device(zipgpu, oracle, ctx):
    """Step 3's device-resident MLEs feed step 5 directly (no host copy)."""
    import torch

    L, nv, D = 3, 9, 32
    p = field(oracle, L)
    rng = np.random.default_rng(77)
    b, i = columns(rng, 4, 1, nv, D)
    a = np.array(inner(int.from_bytes(rng.bytes(8 * L), "little"), p, L), np.uint64)
    r = np.array([inner(int.from_bytes(rng.bytes(8 * L), "little"), p, L) for _ in range(nv)], np.uint64)
    shifts = [(0, 1), (3, 2)]
    mles = oracle.piop_eval_projection(p, L, b, D, i, nv, a)
    want_proof, want_r0 = oracle.piop_multipoint_eval(oracle.Transcript(), p, L, mles, r, shifts)
    bd = torch.from_numpy(b.view(np.int64)).cuda()
    idv = torch.from_numpy(i).cuda()
    out = torch.empty(mles.size, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    zipgpu.check(zipgpu.lib().zg_piop_eval_projection(ctx.handle, p.to_bytes(8 * L, "little"), L, bd.data_ptr(), 4,
                                                      D, idv.data_ptr(), 1, nv, a.ctypes.data, 1, out.data_ptr()))
    t = zipgpu.PcsProverTranscript()
    proof, r0 = zipgpu.ZincPiop.multipoint_eval(ctx, t, p, L, (out.data_ptr(), 5), nv, r, shifts)
    t.close()
    assert proof == want_proof and np.array_equal(r0, want_r0)


# ------------------------------------------------------------------ step 4
def biglinear_system():
    """BigLinear's constraints as a coefficient matrix over [up (16 binary + 1
    integer columns), down (the 16 binary columns shifted by one row)], and its
    shifts; the same constraints as test_sumcheck_cpr.constraints()."""
    from test_sumcheck_cpr import constraints, UP0
    ncols, S = 17, 16
    rows = []
    for c in constraints():
        row = [0] * (ncols + S)
        for j, k in c.items():
            row[j - UP0] = k
        rows.append(row)
    return ncols, [(k, 1) for k in range(S)], rows


@pytest.mark.parametrize("L,nv", [(3, 4), (4, 3)])
def test_oracle_cpr_claim_is_the_folded_constraints(oracle, L, nv):
    ncols, shifts, rows = biglinear_system()
    p, mles, r = mp_case(oracle, L, nv, ncols, 80 + nv)
    proof, pt, evals = oracle.piop_cpr_linear_prove(oracle.Transcript(), p, L, mles, r, shifts, rows)
    twin = oracle.Transcript()
    alpha = std(twin.field_challenge(p, L), p, L)
    rs, n = [std(v, p, L) for v in r], 1 << nv
    col = [[std(mles[j, b], p, L) for b in range(n)] for j in range(ncols)]
    up_down = col + [col[sc][c:] + [0] * c for sc, c in shifts]

    def eq(b):
        e = 1
        for k in range(nv):
            e = e * (rs[k] if (b >> k) & 1 else 1 - rs[k]) % p
        return e

    want = 0
    for b in range(n - 1):  # the selector zeroes the last row
        folded = sum(pow(alpha, k, p) * sum(cf * up_down[j][b] for j, cf in enumerate(row)) for k, row in enumerate(rows))
        want = (want + folded * eq(b)) % p
    # MultiDegreeSumcheckProof: the claimed sum is the group's last field element
    claimed = int.from_bytes(proof[-8 * L:], "little") * pow(1 << (64 * L), -1, p) % p
    assert claimed == want
    rc, vpt, _ = oracle.sumcheck_verify(twin, p, L, nv, [3], proof, True)
    assert rc == 0 and (vpt == pt).all()
    # the evaluations are the up and down MLEs at the sumcheck point
    for j in (0, ncols - 1, ncols):
        m = np.array([inner(v, p, L) for v in up_down[j]], np.uint64)
        assert (oracle.mle_evaluate(p, L, m, pt) == evals[j]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("L,nv", [(3, 8), (4, 6), (3, 11)])
def test_gpu_cpr_linear_prove_matches_oracle(zipgpu, oracle, ctx, L, nv):
    ncols, shifts, rows = biglinear_system()
    p, mles, r = mp_case(oracle, L, nv, ncols, 90 + nv)
    ot = oracle.Transcript()
    want = oracle.piop_cpr_linear_prove(ot, p, L, mles, r, shifts, rows)
    t = zipgpu.PcsProverTranscript()
    got = zipgpu.ZincPiop.cpr_linear_prove(ctx, t, p, L, mles, nv, r, shifts, rows)
    after = t.get_challenge(32)
    t.close()
    assert got[0] == want[0] and np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
    assert after == ot.challenge(32)  # the up/down evaluations were absorbed the same way


# ------------------------------------------------------------------ step 2
@pytest.mark.parametrize("L,nv", [(3, 4), (4, 3)])
def test_oracle_ideal_check_linear_is_the_definition(oracle, L, nv):
    """Combined value of constraint k = sum_j c_kj sum_b eq(b, r) col_j(b) in F[X],
    col_j the projected column (a binary cell's 0/1 coefficients, an integer as a
    constant; down columns shifted up by their shift), over the rows b < 2^nv - 1
    only (evaluate_combined_polynomials, ideal_check/combined_poly_builder.rs:
    232-252, reads zero on the last row of every column), trimmed."""
    ncols, shifts, rows = biglinear_system()
    D, n = 32, 1 << nv
    p = field(oracle, L)
    rng = np.random.default_rng(120 + nv)
    b, i = columns(rng, 16, 1, nv, D)
    pt, combined = oracle.piop_ideal_check_linear(oracle.Transcript(), p, L, b, D, i, nv, shifts, rows)
    twin = oracle.Transcript()
    r = [std(twin.field_challenge(p, L), p, L) for _ in range(nv)]
    assert [std(v, p, L) for v in pt] == r

    def eq(x):
        e = 1
        for k in range(nv):
            e = e * (r[k] if (x >> k) & 1 else 1 - r[k]) % p
        return e

    def poly(j, x):  # projected cell of up column j at row x
        if j < 16:
            return [(int(b[j, x]) >> l) & 1 for l in range(D)]
        return [int(i[0, x]) % p] + [0] * (D - 1)

    up = [[sum(eq(x) * poly(j, x)[l] for x in range(n - 1)) % p for l in range(D)] for j in range(ncols)]
    down = [[sum(eq(x) * poly(sc, x + c)[l] for x in range(min(n - c, n - 1))) % p for l in range(D)]
            for sc, c in shifts]
    vals = up + down
    for k, row in enumerate(rows):
        want = [sum(cf * vals[j][l] for j, cf in enumerate(row)) % p for l in range(D)]
        while want and want[-1] == 0:
            want.pop()
        assert [std(e, p, L) for e in combined[k]] == want


@pytest.mark.gpu
@pytest.mark.parametrize("L,nv", [(3, 9), (4, 7), (3, 12)])
def test_gpu_ideal_check_linear_matches_oracle(zipgpu, oracle, ctx, L, nv):
    ncols, shifts, rows = biglinear_system()
    D = 32
    p = field(oracle, L)
    rng = np.random.default_rng(130 + nv)
    b, i = columns(rng, 16, 1, nv, D)
    ot = oracle.Transcript()
    wpt, wcomb = oracle.piop_ideal_check_linear(ot, p, L, b, D, i, nv, shifts, rows)
    t = zipgpu.PcsProverTranscript()
    gpt, gcomb = zipgpu.ZincPiop.ideal_check_linear(ctx, t, p, L, b, D, i, nv, shifts, rows)
    after = t.get_challenge(32)
    t.close()
    assert np.array_equal(gpt, wpt)
    assert len(gcomb) == len(wcomb) and all(np.array_equal(g, w) for g, w in zip(gcomb, wcomb))
    assert after == ot.challenge(32)
