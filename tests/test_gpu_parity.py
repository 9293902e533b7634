"""GPU parity: the CUDA path (through the C ABI) against the oracle, byte for
byte: codewords, Merkle roots, commitments, proofs and evaluations.  Sizes the
oracle finishes in seconds, plus the full-size workloads of the benchmark
checked through the same equality and through the verifier."""
import numpy as np
import pytest

from util import binary_evals, desc_for, i32_evals, i64_evals, params_for

pytestmark = pytest.mark.gpu

ENCODE_CASES = [
    # (eval_kind, D, code_kind, num_vars, row_len, depth)
    (0, 1, 0, 12, 4096, 0),   # Zip flat: depth 2, base 256 x 64
    (0, 1, 0, 12, 64, 0),     # Zip square: depth 1
    (0, 1, 0, 10, 1024, 3),   # explicit depth 3 over a tiny base
    (0, 1, 0, 6, 64, 0),
    (1, 32, 0, 12, 1024, 0),  # Zip+ deg 32: depth 1
    (1, 32, 0, 14, 4096, 0),  # depth 2
    (1, 64, 0, 12, 4096, 0),
    (1, 3, 0, 10, 256, 0),    # the reference tests' BinaryPoly<3>
    (1, 32, 0, 10, 1024, 1),
    (1, 32, 0, 10, 32, 0),
    (1, 17, 0, 9, 512, 0),
    (1, 40, 0, 12, 4096, 3),  # 33..64 lanes, depth 3 (base 32 x 8)
    (1, 64, 0, 14, 1 << 14, 0),  # base 1024 x 256, two 32-lane halves
    (1, 32, 1, 12, 64, 0),    # RAA
    (1, 64, 1, 12, 64, 0),
    (1, 3, 1, 8, 16, 0),
    (1, 32, 1, 16, 256, 0),   # RAA at the Zip+ benchmark shape
    (2, 1, 0, 12, 4096, 0),   # i64 evaluations (Zinc+ integer columns): depth 2
    (2, 1, 0, 14, 1024, 0),   # depth 1
    (2, 1, 0, 10, 1024, 3),   # depth 3
    (2, 1, 0, 6, 64, 0),
]


def _evals(rng, ek, D, n):
    if ek == 2:
        return i64_evals(rng, n)
    return binary_evals(rng, n, D) if ek else i32_evals(rng, n, -(2**31), 2**31 - 1)


@pytest.mark.parametrize("case", ENCODE_CASES)
def test_encode_rows_matches_oracle(zipgpu, oracle, ctx, rng, case):
    ek, D, ck, nv, L, depth = case
    pp = params_for(zipgpu, ek, D, ck, nv, L, depth, ctx=ctx)
    ev = _evals(rng, ek, D, 1 << nv)
    got = zipgpu.ZipPlus.encode_rows(pp, ev)
    want = oracle.encode_rows(desc_for(ek, D, ck, nv, L, depth), ev)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


@pytest.mark.parametrize("rows,width,eb", [(1, 1024, 16), (4, 4096, 256), (64, 256, 16),
                                           (3, 64, 12), (256, 16, 128), (1, 1, 16)])
def test_merkle_root_matches_oracle(zipgpu, oracle, ctx, rows, width, eb):
    data = np.random.default_rng(rows * width).integers(0, 256, (rows, width * eb), dtype=np.uint8)
    assert zipgpu.MerkleTree.new(data, eb, ctx).root() == oracle.merkle_root_rows(data, eb)


COMMIT_CASES = [
    # (eval_kind, D, code_kind, num_vars, row_len, batch)
    (0, 1, 0, 12, 4096, 1), (0, 1, 0, 12, 64, 1), (0, 1, 0, 10, 256, 5),
    (1, 32, 0, 12, 1024, 1), (1, 32, 0, 12, 1024, 2), (1, 64, 0, 10, 1024, 1),
    (1, 3, 0, 10, 256, 3), (1, 32, 1, 12, 64, 1), (1, 64, 1, 12, 64, 2),
    (1, 32, 0, 3, 8, 1),
    (2, 1, 0, 12, 4096, 1), (2, 1, 0, 12, 256, 3), (2, 1, 0, 14, 1024, 1),
]


@pytest.mark.parametrize("case", COMMIT_CASES)
def test_commit_prove_matches_oracle(zipgpu, oracle, ctx, rng, case):
    ek, D, ck, nv, L, batch = case
    pp = params_for(zipgpu, ek, D, ck, nv, L, ctx=ctx)
    polys = [_evals(rng, ek, D, 1 << nv) for _ in range(batch)]
    point = [(-1) ** i * (7 * i + 2) for i in range(nv)]
    desc = desc_for(ek, D, ck, nv, L)
    root_o, proof_o, ev_o, _ = oracle.commit_prove(desc, np.concatenate(polys), batch, point)
    hint, comm = zipgpu.ZipPlus.commit(pp, polys)
    assert comm.root == root_o
    t = zipgpu.PcsProverTranscript.new_from_commitment(comm)
    t.get_random_field_cfg(4)
    ev = zipgpu.ZipPlus.prove(t, pp, polys, point, hint)
    assert ev == ev_o
    assert t.stream == proof_o
    # the hint's codewords are the encode_rows output
    for b in range(batch):
        assert np.array_equal(hint.codeword(b), oracle.encode_rows(desc, polys[b]))
    zipgpu.ZipPlus.verify(pp, comm, point, ev, t.stream)
    assert oracle.verify(desc, comm.root, batch, point, ev, t.stream) == 0
    root2, ev2, proof2 = zipgpu.ZipPlus.commit_prove(pp, polys, point)
    assert (root2, ev2, proof2) == (root_o, ev_o, proof_o)


def test_edge_value_polynomials(zipgpu, oracle, ctx):
    """Zero, all-ones, extreme i32 values (commit_succeeds_for_zero_polynomial,
    commit_succeeds_for_alternating_values, encode_rows_handles_large_integer_values)."""
    nv = 10
    for ek, D, vals in [
        (0, 1, np.zeros(1 << nv, np.int32)),
        (0, 1, np.full(1 << nv, 2**31 - 1, np.int32)),
        (0, 1, np.full(1 << nv, -(2**31), np.int32)),
        (0, 1, np.where(np.arange(1 << nv) % 2 == 0, 1, -1).astype(np.int32)),
        (1, 32, np.zeros(1 << nv, np.uint64)),
        (1, 32, np.full(1 << nv, 0xFFFFFFFF, np.uint64)),
        (1, 64, np.full(1 << nv, 0xFFFFFFFFFFFFFFFF, np.uint64)),
        (2, 1, np.full(1 << nv, 2**63 - 1, np.int64)),
        (2, 1, np.full(1 << nv, -(2**63), np.int64)),
        (2, 1, np.where(np.arange(1 << nv) % 2 == 0, 2**63 - 1, -(2**63)).astype(np.int64)),
    ]:
        L = 256
        pp = params_for(zipgpu, ek, D, 0, nv, L, ctx=ctx)
        desc = desc_for(ek, D, 0, nv, L)
        point = [1] * nv
        root, ev, proof = zipgpu.ZipPlus.commit_prove(pp, [vals], point)
        ro, po, eo, _ = oracle.commit_prove(desc, vals, 1, point)
        assert (root, ev, proof) == (ro, eo, po)


def test_commit_is_deterministic_and_input_sensitive(zipgpu, ctx, rng):
    pp = params_for(zipgpu, 1, 32, 0, 12, 1024, ctx=ctx)
    ev = binary_evals(rng, 1 << 12, 32)
    _, c1 = zipgpu.ZipPlus.commit_single(pp, ev)
    _, c2 = zipgpu.ZipPlus.commit_single(pp, ev)
    assert c1.root == c2.root
    ev2 = ev.copy()
    ev2[100] ^= np.uint64(1)
    _, c3 = zipgpu.ZipPlus.commit_single(pp, ev2)
    assert c3.root != c1.root
    _, cb = zipgpu.ZipPlus.commit(pp, [ev, ev2])
    assert cb.root not in (c1.root, c3.root) and cb.batch_size == 2


def test_batch_and_size_errors(zipgpu, ctx, rng):
    pp = params_for(zipgpu, 1, 32, 0, 10, 1024, ctx=ctx)
    with pytest.raises(ValueError):
        zipgpu.ZipPlus.commit(pp, [])
    with pytest.raises(ValueError):
        zipgpu.ZipPlus.commit(pp, [binary_evals(rng, 512, 32)])
    hint, comm = zipgpu.ZipPlus.commit(pp, [binary_evals(rng, 1024, 32)])
    t = zipgpu.PcsProverTranscript.new_from_commitment(comm)
    with pytest.raises(zipgpu.ZipError):  # field not sampled yet
        zipgpu.ZipPlus.prove(t, pp, [binary_evals(rng, 1024, 32)], [1] * 10, hint)
    t.get_random_field_cfg(4)
    with pytest.raises(zipgpu.ZipError):  # point of the wrong length
        zipgpu.ZipPlus.prove(t, pp, [binary_evals(rng, 1024, 32)], [1] * 9, hint)
    with pytest.raises(zipgpu.ZipError):  # hint for another batch size
        zipgpu.ZipPlus.prove(t, pp, [binary_evals(rng, 1024, 32)] * 2, [1] * 10, hint)


@pytest.mark.parametrize("ck,L", [(0, 1 << 14), (1, 256)])
def test_benchmark_workload_matches_oracle(zipgpu, oracle, ctx, rng, ck, L):
    """The Zip+ benchmark workload at full size: num_vars 16, BinaryPoly<32>,
    IPRS (row_len 2^14, 4 rows) and RAA (row_len 256, 256 rows)."""
    nv, D = 16, 32
    pp = params_for(zipgpu, 1, D, ck, nv, L, ctx=ctx)
    ev = binary_evals(rng, 1 << nv, D)
    point = [1] * nv
    root, inner, proof = zipgpu.ZipPlus.commit_prove(pp, [ev], point)
    ro, po, eo, _ = oracle.commit_prove(desc_for(1, D, ck, nv, L), ev, 1, point)
    assert root == ro and inner == eo and proof == po
    zipgpu.ZipPlus.verify(pp, zipgpu.ZipPlusCommitment(root, 1), point, inner, proof)


@pytest.mark.parametrize("nv", [18, 20])
def test_large_commit_prove_verifies(zipgpu, ctx, rng, nv):
    """Sizes beyond the oracle's quick range: the proof must verify (the
    verifier re-encodes the combined row and checks 147 opened columns against
    it and against the Merkle root) and have the exact size."""
    pp = params_for(zipgpu, 1, 32, 0, nv, 1 << 14, ctx=ctx)
    ev = binary_evals(rng, 1 << nv, 32)
    point = [(-1) ** i * (i + 1) for i in range(nv)]
    root, inner, proof = zipgpu.ZipPlus.commit_prove(pp, [ev], point)
    zipgpu.ZipPlus.verify(pp, zipgpu.ZipPlusCommitment(root, 1), point, inner, proof)
    assert len(proof) == pp.proof_size(1)


@pytest.mark.parametrize("lanes", [1, 3, 4])
def test_commit_prove_many_equals_sequential(zipgpu, oracle, ctx, rng, lanes):
    """The batched, multi-lane form returns for every request exactly the bytes
    of a single commit_prove of that request (and of the oracle)."""
    nv, D, L = 12, 32, 1024
    pp = params_for(zipgpu, 1, D, 0, nv, L, ctx=ctx)
    polys = [binary_evals(rng, 1 << nv, D) for _ in range(7)]
    points = [[(i + 3) * (j + 1) - 5 for j in range(nv)] for i in range(7)]
    got = zipgpu.ZipPlus.commit_prove_many(pp, polys, points, lanes=lanes)
    desc = desc_for(1, D, 0, nv, L)
    for i, (root, ev, proof) in enumerate(got):
        assert (root, ev, proof) == zipgpu.ZipPlus.commit_prove(pp, [polys[i]], points[i])
        ro, po, eo, _ = oracle.commit_prove(desc, polys[i], 1, points[i])
        assert (root, ev, proof) == (ro, eo, po)


@pytest.mark.parametrize("case", [(0, 1, 0, 12, 4096), (1, 32, 0, 14, 1 << 14),
                                  (1, 32, 1, 12, 64), (1, 64, 0, 16, 1 << 14), (2, 1, 0, 12, 1024)])
def test_device_verifier_verdicts_match_oracle(zipgpu, oracle, ctx, rng, case):
    """With device parameters the verifier encodes the opened positions on the
    GPU; its verdicts equal the oracle's and the host-only verifier's."""
    from test_host_abi import verdicts_match_oracle

    ek, D, ck, nv, L = case
    pp = params_for(zipgpu, ek, D, ck, nv, L, ctx=ctx)
    verdicts_match_oracle(zipgpu, oracle, pp, desc_for(ek, D, ck, nv, L), ek, D, nv, rng, cases=24)


@pytest.mark.parametrize("case", [(1, 32, 0, 12, 1024, 1), (1, 64, 0, 10, 256, 2), (0, 1, 0, 10, 256, 1),
                                  (2, 1, 0, 10, 256, 2)])
def test_prove_f_matches_oracle_and_prove(zipgpu, oracle, ctx, rng, case):
    """ZipPlus::prove_f (phase_prove.rs:119-253) at a field point: the oracle's
    proof and evaluation for the same field elements, and zg_prove's bytes when
    the field point is the image of an i128 point (prove maps the point and calls
    prove_f)."""
    ek, D, ck, nv, L, batch = case
    pp = params_for(zipgpu, ek, D, ck, nv, L, ctx=ctx)
    polys = [_evals(rng, ek, D, 1 << nv) for _ in range(batch)]
    desc = desc_for(ek, D, ck, nv, L)
    hint, comm = zipgpu.ZipPlus.commit(pp, polys)
    limbs = 4
    u = [int.from_bytes(rng.bytes(32), "little") for _ in range(nv)]

    def field_point(t, values):
        prime = t.get_random_field_cfg(limbs)
        R = 1 << (64 * limbs)
        return np.array([[((v % prime) * R % prime >> (64 * w)) & ((1 << 64) - 1) for w in range(limbs)]
                         for v in values], np.uint64)

    t = zipgpu.PcsProverTranscript.new_from_commitment(comm)
    ev = zipgpu.ZipPlus.prove_f(t, pp, polys, field_point(t, u), hint)
    root_o, proof_o, ev_o, _ = oracle.commit_prove_f(desc, np.concatenate(polys), batch, u)
    assert comm.root == root_o and ev == ev_o and t.stream == proof_o
    # an i128 point through prove and its field image through prove_f
    point = [(-1) ** i * (7 * i + 2) for i in range(nv)]
    t1 = zipgpu.PcsProverTranscript.new_from_commitment(comm)
    t1.get_random_field_cfg(limbs)
    ev1 = zipgpu.ZipPlus.prove(t1, pp, polys, point, hint)
    t2 = zipgpu.PcsProverTranscript.new_from_commitment(comm)
    ev2 = zipgpu.ZipPlus.prove_f(t2, pp, polys, field_point(t2, point), hint)
    assert ev1 == ev2 and t1.stream == t2.stream
    # a coordinate that is not reduced mod the prime is rejected
    t3 = zipgpu.PcsProverTranscript.new_from_commitment(comm)
    pf = field_point(t3, u)
    pf[0] = np.iinfo(np.uint64).max
    with pytest.raises(zipgpu.ZipError):
        zipgpu.ZipPlus.prove_f(t3, pp, polys, pf, hint)
