"""RaaSignFlippingCode (zip-plus/src/code/raa_sign_flip.rs:31-69): the RAA code
with every second entry negated after the repetition and again after the first
accumulation.  The reference has no tests or golden vectors for it, so the
oracle is pinned through its parts: the permutations are the RAA code's (pinned
by the RAA known-answer test, raa.rs:398-413), and the steps are restated here
with Python integers straight from raa_sign_flip.rs:31-69 (repeat = cycle,
raa.rs:185-195; clone_shuffled = gather, raa.rs:239-244; accumulate = prefix
sum, raa.rs:208-219).  The GPU path is then checked against the oracle."""
import numpy as np
import pytest

from util import binary_evals, desc_for, params_for

SIGN_FLIP = 2


def restated_encode(oracle, row, rep, mod):
    """encode_inner of raa_sign_flip.rs on a list of integers, modulo `mod`."""
    n = len(row) * rep
    p1, p2 = oracle.shuffle_identity(1, n), oracle.shuffle_identity(2, n)
    r = [row[i % len(row)] for i in range(n)]                      # repeat (cycle)
    r = [(-v if i % 2 else v) % mod for i, v in enumerate(r)]      # flip_even_signs
    r = [r[int(i)] for i in p1]                                    # clone_shuffled(perm_1)
    for i in range(1, n):                                          # accumulate
        r[i] = (r[i] + r[i - 1]) % mod
    r = [(-v if i % 2 else v) % mod for i, v in enumerate(r)]      # flip_even_signs
    r = [r[int(i)] for i in p2]                                    # clone_shuffled(perm_2)
    for i in range(1, n):                                          # accumulate
        r[i] = (r[i] + r[i - 1]) % mod
    return r


@pytest.mark.parametrize("row_len,rep", [(4, 4), (64, 2), (256, 4)])
def test_oracle_encode_wide_equals_restatement(oracle, row_len, rep):
    desc = desc_for(0, 1, SIGN_FLIP, 10, row_len, rep=rep, comb=4)
    rng = np.random.default_rng(row_len)
    row = rng.integers(0, 1 << 40, (row_len, 4), dtype=np.uint64)
    row[:, 2:] = 0
    vals = [int(a) | (int(b) << 64) for a, b in row[:, :2]]
    want = restated_encode(oracle, vals, rep, 1 << 256)
    got = oracle.encode_wide(desc, row, 4)
    assert [sum(int(w) << (64 * k) for k, w in enumerate(e)) for e in got] == want


def test_oracle_binary_encode_equals_restatement(oracle):
    row_len, D, rep = 64, 5, 4
    desc = desc_for(1, D, SIGN_FLIP, 6, row_len, rep=rep)
    ev = binary_evals(np.random.default_rng(7), row_len, D)
    cw = oracle.encode_rows(desc, ev).view(np.int32).reshape(row_len * rep, D)
    for lane in range(D):
        bits = [int(x >> np.uint64(lane)) & 1 for x in ev]
        want = [v - (1 << 32) if v >> 31 else v for v in restated_encode(oracle, bits, rep, 1 << 32)]
        assert cw[:, lane].tolist() == want


def test_sign_flip_differs_from_plain_raa_and_is_linear(oracle):
    flip, plain = desc_for(0, 1, SIGN_FLIP, 8, 256, comb=4), desc_for(0, 1, 1, 8, 256, comb=4)
    rng = np.random.default_rng(3)
    a = rng.integers(0, 1 << 20, (256, 4), dtype=np.uint64)
    b = rng.integers(0, 1 << 20, (256, 4), dtype=np.uint64)
    ea, eb, eab = ([sum(int(w) << (64 * k) for k, w in enumerate(e)) for e in oracle.encode_wide(flip, x, 4)]
                   for x in (a, b, a + b))
    assert [(x + y) % (1 << 256) for x, y in zip(ea, eb)] == eab  # wrapping Int<4> arithmetic
    assert not np.array_equal(oracle.encode_wide(flip, a, 4), oracle.encode_wide(plain, a, 4))


@pytest.mark.gpu
@pytest.mark.parametrize("D,nv,L", [(32, 12, 64), (3, 8, 16), (64, 12, 64), (32, 16, 256)])
def test_gpu_encode_and_commit_prove_match_oracle(zipgpu, oracle, ctx, rng, D, nv, L):
    pp = params_for(zipgpu, 1, D, SIGN_FLIP, nv, L, ctx=ctx)
    desc = desc_for(1, D, SIGN_FLIP, nv, L)
    ev = binary_evals(rng, 1 << nv, D)
    assert np.array_equal(zipgpu.ZipPlus.encode_rows(pp, ev), oracle.encode_rows(desc, ev))
    point = [int(x) for x in rng.integers(1, 1 << 62, size=nv)]
    root, ev_inner, proof = zipgpu.ZipPlus.commit_prove(pp, [ev], point)
    o_root, o_proof, o_eval, _mod = oracle.commit_prove(desc, ev, 1, point)
    assert root == o_root and ev_inner == o_eval and proof == o_proof
    assert oracle.verify(desc, root, 1, point, ev_inner, proof) == 0
    comm = zipgpu.ZipPlusCommitment(root, 1)
    zipgpu.ZipPlus.verify(pp, comm, point, ev_inner, proof)  # the library's verifier
    bad = bytearray(proof)
    bad[len(bad) // 2] ^= 1
    with pytest.raises(zipgpu.ZipError):
        zipgpu.ZipPlus.verify(pp, comm, point, ev_inner, bytes(bad))
