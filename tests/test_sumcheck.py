"""PIOP sumcheck: the oracle pinned to a big-integer restatement of the
reference prover (piop/src/sumcheck.rs:163-215, sumcheck/prover.rs:95-247,
sumcheck/multi_degree.rs:259-355), the reference's own sumcheck test cases
(piop/src/sumcheck/tests.rs) run against the oracle, and the GPU prover
(zg_sumcheck_prove / zg_mle_evaluate) compared byte for byte with the oracle.
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

# Moduli of 1..4 limbs.  The 2-limb one is the ConstMontyField modulus of the
# reference's sumcheck tests (piop/src/sumcheck/tests.rs:17).
MODULI = {
    1: 0xFFFFFFFF00000001,
    2: 0xB933426489189CB5B47D567F,
    3: (1 << 192) - (1 << 64) - 1,
    4: (1 << 255) - 19,
}


def limbs_of(x: int, L: int) -> list[int]:
    return [(x >> (64 * i)) & ((1 << 64) - 1) for i in range(L)]


def to_mont(v: int, p: int, L: int) -> int:
    return (v % p) * (1 << (64 * L)) % p


def from_mont(inner: int, p: int, L: int) -> int:
    return inner * pow(1 << (64 * L), -1, p) % p


def rand_poly(rng, nv, p, L, mult_range=(2, 5), num_products=7):
    """rand_poly of piop/src/sumcheck/tests/utils.rs:9-56: num_products products
    of fresh random MLEs, each with a random coefficient.  Returns values (not
    Montgomery) and the group in oracle/product form."""
    vals, products, degree = [], [], 0
    for _ in range(num_products):
        m = int(rng.integers(mult_range[0], mult_range[1]))
        degree = max(degree, m)
        idx = list(range(len(vals), len(vals) + m))
        for _ in range(m):
            vals.append([int.from_bytes(rng.bytes(8 * L + 8), "little") % p for _ in range(1 << nv)])
        coeff = int.from_bytes(rng.bytes(8 * L + 8), "little") % p
        products.append((coeff, idx))
    return degree, vals, products


def group_arrays(degree, vals, products, p, L):
    mles = np.array([[limbs_of(to_mont(v, p, L), L) for v in mle] for mle in vals], np.uint64)
    prods = [(to_mont(c, p, L), idx) for c, idx in products]
    return degree, mles.reshape(len(vals), -1, L), prods


def absorb_field(t, p, L, value):
    t.absorb(b"\x03" + p.to_bytes(8 * L, "little") + b"\x05\x01"
             + to_mont(value, p, L).to_bytes(8 * L, "little") + b"\x03")


def model_prove(oracle, p, L, nv, groups, multi):
    """Big-integer restatement of prove_as_subprotocol; returns proof bytes and
    the challenge values.  groups: (degree, vals, products) with plain values."""
    t = oracle.Transcript()
    absorb_field(t, p, L, nv)
    absorb_field(t, p, L, len(groups) if multi else groups[0][0])
    if multi:
        for g in groups:
            absorb_field(t, p, L, g[0])
    state = [[list(m) for m in g[1]] for g in groups]
    msgs = [[] for _ in groups]
    claimed = [0] * len(groups)
    point = []
    r = None
    for rd in range(nv):
        if r is not None:
            for st in state:
                for j, m in enumerate(st):
                    st[j] = [(m[2 * b] + r * (m[2 * b + 1] - m[2 * b])) % p for b in range(len(m) // 2)]
        round_msgs = []
        for gi, (deg, _, prods) in enumerate(groups):
            ev = [0] * (deg + 1)
            st = state[gi]
            for b in range(len(st[0]) // 2):
                for tt in range(deg + 1):
                    x = [(m[2 * b] + tt * (m[2 * b + 1] - m[2 * b])) % p for m in st]
                    s = 0
                    for c, idx in prods:
                        term = c
                        for i in idx:
                            term = term * x[i] % p
                        s += term
                    ev[tt] = (ev[tt] + s) % p
            if rd == 0:
                claimed[gi] = (ev[0] + ev[1]) % p if deg > 0 else ev[0]
            msgs[gi].append(ev[1:])
            round_msgs.append(ev[1:])
            if not multi:
                for e in ev[1:]:
                    absorb_field(t, p, L, e)
        if multi:
            for tail in round_msgs:
                for e in tail:
                    absorb_field(t, p, L, e)
        r = int.from_bytes(t.challenge(8 * L), "little") % p
        absorb_field(t, p, L, r)
        point.append(r)
    fb = lambda v: to_mont(v, p, L).to_bytes(8 * L, "little")  # noqa: E731
    out = p.to_bytes(8 * L, "little")
    if not multi:
        out += struct.pack("<I", nv)
        for tail in msgs[0]:
            out += struct.pack("<I", len(tail)) + b"".join(fb(e) for e in tail)
        out += fb(claimed[0])
    else:
        out += struct.pack("<II", len(groups), nv)
        out += b"".join(struct.pack("<I", g[0]) for g in groups)
        for gi in range(len(groups)):
            for tail in msgs[gi]:
                out += b"".join(fb(e) for e in tail)
        out += b"".join(fb(c) for c in claimed)
    return out, point


def point_values(point, p, L):
    return [from_mont(sum(int(w) << (64 * i) for i, w in enumerate(row)), p, L) for row in point]


# ----------------------------------------------------------------- CPU pins
@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_oracle_matches_bigint_model(oracle, L):
    p = MODULI[L]
    rng = np.random.default_rng(100 + L)
    nv = 3
    deg, vals, prods = rand_poly(rng, nv, p, L)
    proof, pt, _ = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv,
                                         [group_arrays(deg, vals, prods, p, L)], False)
    ref, ref_pt = model_prove(oracle, p, L, nv, [(deg, vals, prods)], False)
    assert proof == ref
    assert point_values(pt, p, L) == ref_pt


def test_oracle_multi_degree_matches_bigint_model(oracle):
    L, p, nv = 2, MODULI[2], 3
    rng = np.random.default_rng(7)
    groups = [rand_poly(rng, nv, p, L, (1, 3), 3), rand_poly(rng, nv, p, L, (3, 4), 2),
              rand_poly(rng, nv, p, L, (1, 2), 2)]
    proof, pt, _ = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv,
                                         [group_arrays(*g, p, L) for g in groups], True)
    ref, ref_pt = model_prove(oracle, p, L, nv, groups, True)
    assert proof == ref
    assert point_values(pt, p, L) == ref_pt


def _prove(oracle, L, nv, seed, multi=False):
    p = MODULI[L]
    rng = np.random.default_rng(seed)
    g = group_arrays(*rand_poly(rng, nv, p, L), p, L)
    proof, pt, fin = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [g], multi)
    return p, g, proof, pt, fin


@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_full_sumcheck_protocol_works_correctly(oracle, L):
    """full_sumcheck_protocol_works_correctly (tests.rs:44-57) plus the subclaim
    check: the expected evaluation equals comb at the MLE evaluations."""
    for seed in range(5):
        p, g, proof, pt, fin = _prove(oracle, L, 3, seed)
        rc, vpt, exp = oracle.sumcheck_verify(oracle.Transcript(), p, L, 3, [g[0]], proof, False)
        assert rc == 0
        assert (vpt == pt).all()
        assert (oracle.sumcheck_comb(p, L, g, fin) == exp[0]).all()
        for j in range(g[1].shape[0]):
            assert (oracle.mle_evaluate(p, L, g[1][j], pt) == fin[j]).all()


def test_prover_message_omits_constant_term(oracle):
    p, g, proof, _, _ = _prove(oracle, 2, 3, 1)
    fb = 16
    assert struct.unpack_from("<I", proof, fb + 4)[0] == g[0]


def _claimed_offset(proof, L):
    return len(proof) - 8 * L


def test_subclaim_differs_with_incorrect_claimed_sum(oracle):
    L = 2
    p, g, proof, _, _ = _prove(oracle, L, 3, 2)
    _, pt0, e0 = oracle.sumcheck_verify(oracle.Transcript(), p, L, 3, [g[0]], proof, False)
    off = _claimed_offset(proof, L)
    inner = int.from_bytes(proof[off:], "little")
    bad = proof[:off] + ((inner + to_mont(1, p, L)) % p).to_bytes(8 * L, "little")
    rc, pt1, e1 = oracle.sumcheck_verify(oracle.Transcript(), p, L, 3, [g[0]], bad, False)
    assert rc == 0
    assert (pt0 == pt1).all()
    assert not (e0 == e1).all()


def test_subclaim_changes_when_prover_message_is_tampered(oracle):
    L = 2
    p, g, proof, _, _ = _prove(oracle, L, 3, 3)
    _, pt0, e0 = oracle.sumcheck_verify(oracle.Transcript(), p, L, 3, [g[0]], proof, False)
    off = 8 * L + 4 + 4  # first evaluation of the first message
    inner = int.from_bytes(proof[off:off + 8 * L], "little")
    bad = (proof[:off] + ((inner + to_mont(1, p, L)) % p).to_bytes(8 * L, "little")
           + proof[off + 8 * L:])
    rc, pt1, e1 = oracle.sumcheck_verify(oracle.Transcript(), p, L, 3, [g[0]], bad, False)
    assert rc == 0
    assert not (pt0 == pt1).all()
    assert not (e0 == e1).all()


def test_verifier_rejects_proof_with_wrong_degree(oracle):
    L = 2
    p, g, proof, _, _ = _prove(oracle, L, 3, 4)
    rc, _, _ = oracle.sumcheck_verify(oracle.Transcript(), p, L, 3, [g[0] - 1], proof, False)
    assert rc != 0


def test_protocol_is_deterministic_and_polynomial_sensitive(oracle):
    L = 2
    _, g, proof1, _, _ = _prove(oracle, L, 3, 5)
    _, _, proof2, _, _ = _prove(oracle, L, 3, 5)
    assert proof1 == proof2
    p = MODULI[L]
    mles = g[1].copy()
    v = sum(int(w) << (64 * i) for i, w in enumerate(mles[0, 0]))
    mles[0, 0] = limbs_of((v + to_mont(1, p, L)) % p, L)
    proof3, _, _ = oracle.sumcheck_prove(oracle.Transcript(), p, L, 3, [(g[0], mles, g[2])], False)
    assert proof3 != proof1


@pytest.mark.parametrize("kind", ["zero", "constant"])
def test_sumcheck_with_zero_and_constant_polynomials(oracle, kind):
    """sumcheck_with_zero_polynomial / sumcheck_with_constant_polynomial
    (tests.rs:367-445): two MLEs, comb = their product, degree 2."""
    L, nv = 2, 3
    p = MODULI[L]
    v = 0 if kind == "zero" else to_mont(1, p, L)
    mles = np.array([[limbs_of(v, L)] * (1 << nv)] * 2, np.uint64)
    g = (2, mles, [(to_mont(1, p, L), [0, 1])])
    proof, pt, fin = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [g], False)
    claimed = int.from_bytes(proof[-8 * L:], "little")
    assert from_mont(claimed, p, L) == (0 if kind == "zero" else (1 << nv))
    rc, _, exp = oracle.sumcheck_verify(oracle.Transcript(), p, L, nv, [2], proof, False)
    assert rc == 0
    assert (oracle.sumcheck_comb(p, L, g, fin) == exp[0]).all()


def test_multi_degree_subclaims(oracle):
    L, nv = 4, 4
    p = MODULI[L]
    rng = np.random.default_rng(11)
    groups = [group_arrays(*rand_poly(rng, nv, p, L, (1, 4), 3), p, L) for _ in range(3)]
    proof, pt, fin = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, groups, True)
    rc, vpt, exp = oracle.sumcheck_verify(oracle.Transcript(), p, L, nv, [g[0] for g in groups],
                                          proof, True)
    assert rc == 0 and (vpt == pt).all()
    k = 0
    for gi, g in enumerate(groups):
        n = g[1].shape[0]
        assert (oracle.sumcheck_comb(p, L, g, fin[k:k + n]) == exp[gi]).all()
        k += n


def test_oracle_mle_evaluate_matches_bigint(oracle):
    L, nv = 3, 6
    p = MODULI[L]
    rng = np.random.default_rng(12)
    vals = [int.from_bytes(rng.bytes(32), "little") % p for _ in range(1 << nv)]
    pt = [int.from_bytes(rng.bytes(32), "little") % p for _ in range(nv)]
    want = 0
    for x, v in enumerate(vals):
        e = 1
        for k in range(nv):
            e = e * (pt[k] if (x >> k) & 1 else 1 - pt[k]) % p
        want = (want + v * e) % p
    mle = np.array([limbs_of(to_mont(v, p, L), L) for v in vals], np.uint64)
    ptm = np.array([limbs_of(to_mont(v, p, L), L) for v in pt], np.uint64)
    got = oracle.mle_evaluate(p, L, mle, ptm)
    assert from_mont(sum(int(w) << (64 * i) for i, w in enumerate(got)), p, L) == want


# ----------------------------------------------------------------- GPU parity
def _gpu_prove(zipgpu, ctx, p, L, nv, groups, multi):
    grps = [zipgpu.SumcheckGroup(g[0], g[1], g[2]) for g in groups]
    t = zipgpu.PcsProverTranscript()
    try:
        if multi:
            return zipgpu.MultiDegreeSumcheck.prove_as_subprotocol(t, p, L, nv, grps, ctx)
        return zipgpu.MLSumcheck.prove_as_subprotocol(t, p, L, nv, grps[0], ctx)
    finally:
        t.close()


@pytest.mark.gpu
@pytest.mark.parametrize("L", [1, 2, 3, 4])
@pytest.mark.parametrize("nv", [1, 3, 8, 12])
def test_gpu_sumcheck_matches_oracle(oracle, zipgpu, ctx, L, nv):
    p = MODULI[L]
    rng = np.random.default_rng(1000 * L + nv)
    g = group_arrays(*rand_poly(rng, nv, p, L), p, L) if nv <= 8 else None
    if g is None:  # larger cases: random Montgomery inners drawn directly
        n_mles, prods = 6, [(to_mont(3, p, L), [0, 1, 2]), (to_mont(5, p, L), [3, 4]),
                            (to_mont(7, p, L), [5]), (to_mont(11, p, L), [0, 5, 3, 1])]
        vals = rng.integers(0, 1 << 63, size=(n_mles, 1 << nv, L), dtype=np.uint64)
        vals[..., L - 1] %= np.uint64(max(MODULI[L] >> (64 * (L - 1)), 1))
        g = (4, vals, prods)
    want = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [g], False)
    got = _gpu_prove(zipgpu, ctx, p, L, nv, [g], False)
    assert got[0] == want[0]
    assert (got[1] == want[1]).all()
    assert (got[2] == want[2]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("L", [2, 4])
def test_gpu_multi_degree_matches_oracle(oracle, zipgpu, ctx, L):
    p, nv = MODULI[L], 7
    rng = np.random.default_rng(77 + L)
    groups = [group_arrays(*rand_poly(rng, nv, p, L, (1, 4), 3), p, L),
              group_arrays(*rand_poly(rng, nv, p, L, (4, 6), 2), p, L),
              group_arrays(*rand_poly(rng, nv, p, L, (1, 2), 2), p, L)]
    want = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, groups, True)
    got = _gpu_prove(zipgpu, ctx, p, L, nv, groups, True)
    assert got[0] == want[0]
    assert (got[1] == want[1]).all() and (got[2] == want[2]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_gpu_factored_groups_match_oracle(oracle, zipgpu, ctx, L):
    """Sums of products times 1..3 random affine factors, single and multi-degree,
    with the MLEs on the host and on the device."""
    import torch

    p, nv = MODULI[L], 9
    rng = np.random.default_rng(300 + L)
    groups = []
    for nf in (1, 2, 3):
        deg, vals, prods = rand_poly(rng, nv, p, L, (1, 3), 4)
        g = group_arrays(deg, vals, prods, p, L)
        factors = [(to_mont(int.from_bytes(rng.bytes(8 * L), "little"), p, L),
                    to_mont(int.from_bytes(rng.bytes(8 * L), "little"), p, L),
                    int(rng.integers(0, g[1].shape[0]))) for _ in range(nf)]
        groups.append((deg + nf, g[1], g[2], factors))
    for multi, gs in ((False, groups[:1]), (True, groups)):
        want = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, gs, multi)
        for on_device in (False, True):
            keep = []
            zgroups = []
            for deg, mles, prods, factors in gs:
                if on_device:
                    d = torch.from_numpy(mles.reshape(-1).view(np.uint8).copy()).cuda()
                    keep.append(d)
                    zgroups.append(zipgpu.SumcheckGroup(deg, d.data_ptr(), prods,
                                                        n_mles=mles.shape[0], factors=factors))
                else:
                    zgroups.append(zipgpu.SumcheckGroup(deg, mles, prods, factors=factors))
            torch.cuda.synchronize()
            t = zipgpu.PcsProverTranscript()
            if multi:
                got = zipgpu.MultiDegreeSumcheck.prove_as_subprotocol(t, p, L, nv, zgroups, ctx)
            else:
                got = zipgpu.MLSumcheck.prove_as_subprotocol(t, p, L, nv, zgroups[0], ctx)
            t.close()
            assert got[0] == want[0]
            assert (got[1] == want[1]).all() and (got[2] == want[2]).all()


@pytest.mark.gpu
def test_gpu_sumcheck_edge_cases(oracle, zipgpu, ctx):
    """Zero polynomial, a constant polynomial, degree 8, and inners at p - 1."""
    L, nv = 4, 5
    p = MODULI[L]
    one = to_mont(1, p, L)
    cases = [
        (2, np.zeros((2, 1 << nv, L), np.uint64), [(one, [0, 1])]),
        (2, np.array([[limbs_of(one, L)] * (1 << nv)] * 2, np.uint64), [(one, [0, 1])]),
        (8, np.array([[limbs_of(p - 1, L)] * (1 << nv)] * 8, np.uint64),
         [(p - 1, list(range(8))), (one, [0])]),
    ]
    for g in cases:
        want = oracle.sumcheck_prove(oracle.Transcript(), p, L, nv, [g], False)
        got = _gpu_prove(zipgpu, ctx, p, L, nv, [g], False)
        assert got[0] == want[0]


@pytest.mark.gpu
def test_gpu_sumcheck_large_verifies(oracle, zipgpu, ctx):
    """2^20 evaluations: the GPU proof verifies and its subclaim equals comb at
    the final MLE values, and each final value is the MLE at the point."""
    L, nv = 4, 20
    p = MODULI[L]
    rng = np.random.default_rng(99)
    vals = rng.integers(0, 1 << 63, size=(3, 1 << nv, L), dtype=np.uint64)
    vals[..., L - 1] >>= np.uint64(2)
    g = (3, vals, [(to_mont(2, p, L), [0, 1, 2]), (to_mont(9, p, L), [1])])
    proof, pt, fin = _gpu_prove(zipgpu, ctx, p, L, nv, [g], False)
    rc, vpt, exp = oracle.sumcheck_verify(oracle.Transcript(), p, L, nv, [3], proof, False)
    assert rc == 0 and (vpt == pt).all()
    assert (oracle.sumcheck_comb(p, L, g, fin) == exp[0]).all()
    assert (zipgpu.mle_evaluate(p, L, vals[1], pt, ctx) == fin[1]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_gpu_mle_evaluate_matches_oracle(oracle, zipgpu, ctx, L):
    p, nv = MODULI[L], 10
    rng = np.random.default_rng(5 + L)
    mle = np.array([limbs_of(to_mont(int(v), p, L), L) for v in rng.integers(0, 1 << 62, 1 << nv)],
                   np.uint64)
    pt = np.array([limbs_of(to_mont(int(v), p, L), L) for v in rng.integers(0, 1 << 62, nv)],
                  np.uint64)
    assert (zipgpu.mle_evaluate(p, L, mle, pt, ctx) == oracle.mle_evaluate(p, L, mle, pt)).all()


@pytest.mark.gpu
def test_gpu_sumcheck_rejects_bad_input(zipgpu, ctx):
    L, p = 2, MODULI[2]
    mles = np.zeros((2, 8, L), np.uint64)
    one = to_mont(1, p, L)
    with pytest.raises(zipgpu.ZipError):  # nvars == 0: "Attempt to prove a constant"
        _gpu_prove(zipgpu, ctx, p, L, 0, [(2, mles[:, :1], [(one, [0, 1])])], False)
    with pytest.raises(zipgpu.ZipError):  # product index out of range
        _gpu_prove(zipgpu, ctx, p, L, 3, [(2, mles, [(one, [0, 2])])], False)
    with pytest.raises(zipgpu.ZipError):  # degree above the kernel's limit
        _gpu_prove(zipgpu, ctx, p, L, 3, [(9, mles, [(one, [0, 1])])], False)
    t = zipgpu.PcsProverTranscript()
    with pytest.raises(zipgpu.ZipError):  # factor index out of range
        zipgpu.MLSumcheck.prove_as_subprotocol(
            t, p, L, 3, zipgpu.SumcheckGroup(3, mles, [(one, [0, 1])], factors=[(one, one, 2)]), ctx)
    t.close()
