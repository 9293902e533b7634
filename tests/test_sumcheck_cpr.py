"""The combined-polynomial-resolver sumcheck group of the BigLinear UAIR
(piop/src/combined_poly_resolver.rs:71-178, constraints test-uair/src/lib.rs:
340-382) written as a sum of products, the form zg_sumcheck_prove takes.

The reference's comb_fn is folded(up, down) * (1 - sel) * eq_r with
folded = sum_k alpha^k g_k, the g_k linear in the columns.  Field arithmetic is
exact, so expanding it gives the same field value at every point:
    comb = sum_j A_j * eq * v_j - sum_j A_j * sel * eq * v_j,
    A_j = sum_k alpha^k c_kj.
zg_sumcheck_prove also takes the reference's own shape, a sum of one-MLE
products times the affine factors eq_r and (1 - sel) (about a fifth of the
field multiplies).  The tests check both forms against the reference formula
with Python integers, check that they give the same proof, and run the sumcheck
on them with the oracle and on the GPU.
"""
import numpy as np
import pytest

NUM_BIN, NUM_UP, NUM_DOWN = 16, 17, 16
# MLE order of prepare_sumcheck_group: [selector, eq_r, up (16 binary, 1 int), down (16)]
SEL, EQ, UP0 = 0, 1, 2
DOWN0 = UP0 + NUM_UP
INT = UP0 + NUM_BIN


def constraints():
    """BigLinear's 17 constraints as {mle index: integer coefficient}, in order."""
    cs = [{**{UP0 + i: 1 for i in range(NUM_BIN)}, INT: -1},  # sum of binary cols - int
          {DOWN0 + 0: 1, INT: -1}]                             # down.bin[0] - up.int
    for i in range(1, NUM_BIN):                                # up.bin[i] - down.bin[i]
        cs.append({UP0 + i: 1, DOWN0 + i: -1})
    return cs


def reference_comb(vals, alpha, p):
    """folded_constraints * (1 - selector) * eq_r with Python integers."""
    folded, power = 0, 1
    for c in constraints():
        folded = (folded + power * sum(k * vals[j] for j, k in c.items())) % p
        power = power * alpha % p
    return folded * (1 - vals[SEL]) % p * vals[EQ] % p


def expanded_products(alpha, p):
    """(coefficient value, [mle indices]) products of the expansion."""
    A = {}
    power = 1
    for c in constraints():
        for j, k in c.items():
            A[j] = (A.get(j, 0) + power * k) % p
        power = power * alpha % p
    prods = []
    for j in sorted(A):
        prods.append((A[j], [EQ, j]))
        prods.append(((-A[j]) % p, [SEL, EQ, j]))
    return prods


def factored_group(alpha, p, L, mles):
    """The same comb in the reference's own shape: folded(v) as one-MLE products,
    times the factors eq_r (0 + 1 * eq) and (1 - sel) (1 + (p - 1) * sel)."""
    A = {}
    power = 1
    for c in constraints():
        for j, k in c.items():
            A[j] = (A.get(j, 0) + power * k) % p
        power = power * alpha % p
    prods = [(to_mont(A[j], p, L), [j]) for j in sorted(A)]
    factors = [(0, to_mont(1, p, L), EQ), (to_mont(1, p, L), to_mont(p - 1, p, L), SEL)]
    return (3, mles, prods, factors)


def to_mont(v, p, L):
    return (v % p) * (1 << (64 * L)) % p


def limbs(x, L):
    return [(x >> (64 * i)) & ((1 << 64) - 1) for i in range(L)]


def field_prime(oracle, L=3):
    """A random prime of the reference's default field (MontyField<3>), drawn
    as get_random_field_cfg draws it."""
    t = oracle.Transcript()
    t.absorb_slice(b"cpr-test")
    return t.get_prime(L)


def cpr_group(rng, nv, p, L, alpha):
    """MLE values (plain integers) of the CPR group over a random trace."""
    n = 1 << nv
    up = [[int(v) for v in rng.integers(0, 2**32, size=n)] for _ in range(NUM_UP)]
    down = [up[i][1:] + [0] for i in range(NUM_BIN)]  # shift by one, zero padded
    sel = [0] * n
    sel[-1] = 1
    r = [int.from_bytes(rng.bytes(24), "little") % p for _ in range(nv)]
    eq = []
    for x in range(n):  # eq(x, r), bit k of x paired with r[k]
        e = 1
        for k in range(nv):
            e = e * (r[k] if (x >> k) & 1 else 1 - r[k]) % p
        eq.append(e)
    vals = [sel, eq] + up + down
    mles = np.array([[limbs(to_mont(v, p, L), L) for v in col] for col in vals], np.uint64)
    prods = [(to_mont(c, p, L), idx) for c, idx in expanded_products(alpha, p)]
    return vals, (3, mles, prods)


def test_cpr_expansion_equals_reference_comb(oracle):
    L = 3
    p = field_prime(oracle, L)
    rng = np.random.default_rng(21)
    alpha = int.from_bytes(rng.bytes(24), "little") % p
    prods = expanded_products(alpha, p)
    group = (3, np.zeros((35, 1, L), np.uint64), [(to_mont(c, p, L), idx) for c, idx in prods])
    for _ in range(20):
        vals = [int.from_bytes(rng.bytes(24), "little") % p for _ in range(35)]
        got = oracle.sumcheck_comb(p, L, group,
                                   np.array([limbs(to_mont(v, p, L), L) for v in vals], np.uint64))
        got_v = sum(int(w) << (64 * i) for i, w in enumerate(got)) * pow(1 << (64 * L), -1, p) % p
        assert got_v == reference_comb(vals, alpha, p)


def test_cpr_sumcheck_oracle_subclaim(oracle):
    L, nv = 3, 5
    p = field_prime(oracle, L)
    rng = np.random.default_rng(22)
    alpha = int.from_bytes(rng.bytes(24), "little") % p
    vals, group = cpr_group(rng, nv, p, L, alpha)
    proof, pt, fin = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [group], True)
    rc, vpt, exp = oracle.sumcheck_verify(oracle.Transcript(), p, L, nv, [3], proof, True)
    assert rc == 0 and (vpt == pt).all()
    assert (oracle.sumcheck_comb(p, L, group, fin) == exp[0]).all()
    # the claimed sum is the reference comb summed over the hypercube
    claimed = int.from_bytes(proof[-8 * L:], "little") * pow(1 << (64 * L), -1, p) % p
    want = sum(reference_comb([col[x] for col in vals], alpha, p) for x in range(1 << nv)) % p
    assert claimed == want


def test_cpr_factored_form_equals_expanded(oracle):
    """The factored comb has the same value everywhere, so the proofs are equal."""
    L, nv = 3, 5
    p = field_prime(oracle, L)
    rng = np.random.default_rng(24)
    alpha = int.from_bytes(rng.bytes(24), "little") % p
    vals, group = cpr_group(rng, nv, p, L, alpha)
    fgroup = factored_group(alpha, p, L, group[1])
    for _ in range(10):
        v = [int.from_bytes(rng.bytes(24), "little") % p for _ in range(35)]
        got = oracle.sumcheck_comb(p, L, fgroup,
                                   np.array([limbs(to_mont(x, p, L), L) for x in v], np.uint64))
        got_v = sum(int(w) << (64 * i) for i, w in enumerate(got)) * pow(1 << (64 * L), -1, p) % p
        assert got_v == reference_comb(v, alpha, p)
    want = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [group], True)
    got = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [fgroup], True)
    assert got[0] == want[0] and (got[2] == want[2]).all()


@pytest.mark.gpu
def test_cpr_factored_gpu_matches_oracle(oracle, zipgpu, ctx):
    L, nv = 3, 11
    p = field_prime(oracle, L)
    rng = np.random.default_rng(25)
    alpha = int.from_bytes(rng.bytes(24), "little") % p
    _vals, group = cpr_group(rng, nv, p, L, alpha)
    fgroup = factored_group(alpha, p, L, group[1])
    want = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [fgroup], True)
    t = zipgpu.PcsProverTranscript()
    got = zipgpu.MultiDegreeSumcheck.prove_as_subprotocol(
        t, p, L, nv, [zipgpu.SumcheckGroup(3, fgroup[1], fgroup[2], factors=fgroup[3])], ctx)
    t.close()
    assert got[0] == want[0]
    assert (got[1] == want[1]).all() and (got[2] == want[2]).all()


@pytest.mark.gpu
def test_cpr_sumcheck_gpu_matches_oracle(oracle, zipgpu, ctx):
    L, nv = 3, 10
    p = field_prime(oracle, L)
    rng = np.random.default_rng(23)
    alpha = int.from_bytes(rng.bytes(24), "little") % p
    _vals, group = cpr_group(rng, nv, p, L, alpha)
    want = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [group], True)
    t = zipgpu.PcsProverTranscript()
    got = zipgpu.MultiDegreeSumcheck.prove_as_subprotocol(
        t, p, L, nv, [zipgpu.SumcheckGroup(*group)], ctx)
    t.close()
    assert got[0] == want[0]
    assert (got[1] == want[1]).all() and (got[2] == want[2]).all()
