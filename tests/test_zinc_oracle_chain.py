"""The oracle's C restatement of the Zinc+ prover (zr_zinc_prove: steps 0-7 and
the Proof transcription, protocol/src/prover.rs:218-706) and of the Zinc+
verifier (zr_zinc_verify, protocol/src/verifier.rs:215-771).

The C chain is pinned against the independent Python-integer restatement of the
PIOP steps (oracle.zinc_prove_mle_first), and the restated verifier is the
acceptance oracle: it accepts honest proofs of BigLinearUair and of smaller
UAIRs, and rejects proofs tampered in each part, and proofs of traces that break
a constraint.  The combined path (prove_combined, ideal_check.rs:178-240) gives
the MLE-first bytes on linear UAIRs whose constraints lie in non-zero ideals, and
proves UAIRs with products of columns, which the verifier accepts."""
import numpy as np
import pytest

from test_zinc_prove import parse_proof, small_uair


def biglinear(O, nv, seed, n_pub_bin=0):
    import zipgpu.uair as uair

    bins, ints = uair.trace(nv, seed)
    shifts, coeffs = uair.signature()
    U = O.Uair.linear(16, 1, 32, shifts, coeffs, uair.ideal_roots(), n_pub_bin=n_pub_bin)
    return bins, ints, shifts, coeffs, U


def descs(O, nv, D, rows_log=2):
    L = 1 << max(nv - rows_log, 1)
    return (O.make_desc(O.EVAL_BINPOLY, D, 0, nv, L, comb_limbs=6, field_limbs=3),
            O.make_desc(O.EVAL_I64, 1, 0, nv, L, comb_limbs=6, field_limbs=3))


@pytest.mark.parametrize("nv,seed", [(6, 11), (9, 5)])
def test_c_chain_equals_python_chain_biglinear(oracle, nv, seed):
    bins, ints, shifts, coeffs, U = biglinear(oracle, nv, seed)
    db, di = descs(oracle, nv, 32)
    c = oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=True)
    py = oracle.zinc_prove_mle_first(db, di, nv, bins, 32, ints, shifts, coeffs, 3)
    assert c == py
    P = parse_proof(c, 3, nv)
    assert (P["up"], P["down"], P["degree"]) == (17, 16, 3)


def test_c_chain_equals_python_chain_public_input(oracle):
    nv = 7
    bins, ints, shifts, coeffs, U = biglinear(oracle, nv, 21, n_pub_bin=4)
    db, di = descs(oracle, nv, 32)
    c = oracle.zinc_prove(db, di, nv, bins, ints, U, 3)
    assert c == oracle.zinc_prove_mle_first(db, di, nv, bins, 32, ints, shifts, coeffs, 3, n_pub_bin=4)
    assert oracle.zinc_verify(db, di, nv, bins[:4], None, U, 3, c) == 0
    # the verifier takes the public columns from the caller: other values break the transcript
    other = bins[:4].copy()
    other[0, 0] ^= np.uint64(1)
    assert oracle.zinc_verify(db, di, nv, other, None, U, 3, c) != 0


@pytest.mark.parametrize("nb,ni,shifts,nc,D", [(3, 2, [(0, 1), (3, 2), (4, 1)], 4, 8), (0, 2, [(0, 1), (1, 1)], 3, 8),
                                             (1, 1, [], 1, 64)])
def test_c_chain_equals_python_chain_small_uairs(oracle, nb, ni, shifts, nc, D):
    nv = 7
    rng = np.random.default_rng(nb * 100 + ni * 10 + nc)
    bins, ints, coeffs = small_uair(rng, nb, ni, shifts, nc, D, nv)
    db, di = descs(oracle, nv, D)
    U = oracle.Uair.linear(nb, ni, D, shifts, coeffs, [None] * nc)
    c = oracle.zinc_prove(db, di, nv, bins if nb else None, ints if ni else None, U, 3)
    py = oracle.zinc_prove_mle_first(db, di, nv, bins if nb else None, D, ints if ni else None, shifts, coeffs, 3)
    assert c == py
    # random traces satisfy no constraint, but the zero ideals are not checked: the
    # verifier's remaining checks (sumchecks, openings) all pass
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, c) == 0


def _tamper(proof: bytes, offset: int) -> bytes:
    b = bytearray(proof)
    b[offset] ^= 0x01
    return bytes(b)


def test_verifier_accepts_honest_and_rejects_each_tampered_part(oracle):
    nv = 8
    bins, ints, shifts, coeffs, U = biglinear(oracle, nv, 3)
    db, di = descs(oracle, nv, 32)
    proof = oracle.zinc_prove(db, di, nv, bins, ints, U, 3)
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, proof) == 0
    # offsets of each part inside the Proof layout (lib.rs:129-160)
    pos = 3 * 40
    zlen = int.from_bytes(proof[pos:pos + 4], "little")
    zip_at = pos + 4
    parts = {}
    at = zip_at + zlen
    for name in ("ideal", "resolver", "md", "mp", "lifted"):
        ln = int.from_bytes(proof[at:at + 4], "little")
        parts[name] = (at + 4, ln)
        at += 4 + ln
    assert at == len(proof)
    fb = 24
    # a flipped low byte of a field element in each part, and of an opened column
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, parts["ideal"][0] + 1 + fb + 4)) == 2
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, parts["resolver"][0] + 4 + fb)) == 4
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, parts["md"][0] + fb + 12)) == 4
    # a multipoint round message moves the subclaim, caught by verify_subclaim in step 6;
    # its claimed sum is checked in step 5
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, parts["mp"][0] + fb + 8)) == 6
    mp_end = parts["mp"][0] + parts["mp"][1]
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, mp_end - fb)) == 5
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, parts["lifted"][0] + 1 + fb + 4)) == 6
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, zip_at + zlen // 2)) == 7
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, _tamper(proof, 5)) != 0  # a root
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, proof[:-1]) == 1  # truncated


def test_verifier_rejects_a_trace_that_breaks_a_constraint(oracle):
    """The honest prover on a trace whose row 3 breaks BigLinear's first
    constraint (sum of popcounts = z, in (X - 1)) gives ideal-check values outside
    the ideal."""
    nv = 7
    bins, ints, shifts, coeffs, U = biglinear(oracle, nv, 9)
    ints = ints.copy()
    ints[0, 3] += 1
    db, di = descs(oracle, nv, 32)
    proof = oracle.zinc_prove(db, di, nv, bins, ints, U, 3)
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, proof) == 2


def test_combined_path_equals_mle_first_on_linear_uairs(oracle):
    """prove_combined builds each row's constraint polynomials (rows 0..n-2, the
    last row zero) and evaluates their coefficient MLEs; for linear constraints in
    non-zero ideals that is the MLE-first value by linearity."""
    nv = 8
    bins, ints, shifts, coeffs, U = biglinear(oracle, nv, 4)
    db, di = descs(oracle, nv, 32)
    assert oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=False) == \
        oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=True)


def test_combined_path_skips_zero_ideal_constraints(oracle):
    """A constraint in the zero ideal gets an empty combined value on the combined
    path (ideal_check.rs:218-222); the MLE-first path sends its evaluation."""
    nv = 7
    rng = np.random.default_rng(5)
    bins, ints, coeffs = small_uair(rng, 2, 1, [(0, 1)], 2, 8, nv)
    db, di = descs(oracle, nv, 8)
    U = oracle.Uair.linear(2, 1, 8, [(0, 1)], coeffs, [None, 3])
    comb = parse_proof(oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=False), 3, nv)
    mle = parse_proof(oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=True), 3, nv)
    assert comb["ic"][0] == b"" and mle["ic"][0] != b""
    assert comb["ic"][1] == mle["ic"][1]


def product_uair(oracle, nv, seed):
    """A UAIR with products of columns (degree 2): integer columns x, y, z and a
    binary column w with
      x * y - z          in the zero ideal,
      w * x - w * x      (trivially zero) in (X - 1),
      w_down - w         in (X - 1)   (w keeps its popcount down the column),
    and an honest trace."""
    n = 1 << nv
    rng = np.random.default_rng(seed)
    x = rng.integers(-(2**20), 2**20, size=n, dtype=np.int64)
    y = rng.integers(-(2**20), 2**20, size=n, dtype=np.int64)
    z = x * y
    pc = 9
    w = np.zeros(n, np.uint64)
    for r in range(n):
        pos = rng.choice(16, size=pc, replace=False)
        w[r] = np.bitwise_or.reduce(np.left_shift(np.uint64(1), pos.astype(np.uint64)))
    # columns: up [w (0), x (1), y (2), z (3)], down [w shifted by 1 (4)]
    cons = [[(1, [1, 2]), (-1, [3])], [(1, [0, 1]), (-1, [0, 1])], [(1, [4]), (-1, [0])]]
    U = oracle.Uair(1, 3, 16, [(0, 1)], cons, [None, 1, 1])
    return w.reshape(1, n), np.stack([x, y, z]), U


def test_combined_path_proves_products_and_the_verifier_accepts(oracle):
    nv = 7
    bins, ints, U = product_uair(oracle, nv, 3)
    db, di = descs(oracle, nv, 16)
    proof = oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=False)
    P = parse_proof(proof, 3, nv)
    assert P["degree"] == 4  # max constraint degree 2, plus eq and the selector
    assert P["ic"][0] == b""  # zero ideal
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, proof) == 0
    with pytest.raises(ValueError):  # MLE first takes linear UAIRs only
        oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=True)
    # z off by one in a row: the CPR sumcheck claim no longer matches
    bad = ints.copy()
    bad[2, 5] += 1
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3,
                              oracle.zinc_prove(db, di, nv, bins, bad, U, 3, mle_first=False)) == 4


def test_proof_read_entry_point_parses_oracle_proofs(oracle, zipgpu):
    """zg_proof_read (Proof::read_transcription_bytes_exact, lib.rs:93-127) on
    proofs of both paths: the parts' places agree with the layout written, and
    truncated or altered lengths are rejected."""
    nv = 7
    bins, ints, shifts, coeffs, U = biglinear(oracle, nv, 30, n_pub_bin=2)
    db, di = descs(oracle, nv, 32)
    proof = oracle.zinc_prove(db, di, nv, bins, ints, U, 3)
    lay = zipgpu.read_proof(proof, 3, nv)
    P = parse_proof(proof, 3, nv)
    assert lay["batch_sizes"] == [14, 0, 1] and lay["roots"][1] == bytes(32)
    assert lay["n_ideal_values"] == 17 and (lay["n_up_evals"], lay["n_down_evals"]) == (17, 16)
    assert lay["cpr_degree"] == 3 and lay["multi_degree_groups"] == 1 and lay["n_lifted"] == 15
    assert proof[lay["zip_offset"]:lay["zip_offset"] + lay["zip_len"]] == P["zip"]
    assert lay["modulus"] == P["modulus"]
    assert lay["lifted_offset"] + lay["lifted_len"] == len(proof)
    with pytest.raises(zipgpu.ZipError) as e:
        zipgpu.read_proof(proof[:-1], 3, nv)
    assert e.value.status == 3
    bad = bytearray(proof)
    bad[lay["multi_degree_offset"] + 24] ^= 1  # the group count
    with pytest.raises(zipgpu.ZipError):
        zipgpu.read_proof(bytes(bad), 3, nv)
    with pytest.raises(zipgpu.ZipError):
        zipgpu.read_proof(proof, 3, nv + 1)  # wrong number of rounds
    # the combined path of a degree-2 UAIR
    bins2, ints2, U2 = product_uair(oracle, nv, 4)
    db2, di2 = descs(oracle, nv, 16)
    lay2 = zipgpu.read_proof(oracle.zinc_prove(db2, di2, nv, bins2, ints2, U2, 3, mle_first=False), 3, nv)
    assert lay2["cpr_degree"] == 4 and lay2["n_ideal_values"] == 3
