"""The MLE-first Zinc+ prover (ZincPlusPiop::prove::<MLE_FIRST = true>,
protocol/src/prover.rs:677-706) on BigLinearUair and smaller linear UAIRs: the
GPU driver's Proof bytes equal the oracle's chain of the same steps; on the CPU,
the oracle's proof parses under the reference's read_transcription_bytes_exact
layout (protocol/src/lib.rs:93-127) and the generated traces satisfy the
constraints."""
import numpy as np
import pytest

from util import desc_for, params_for

N_OPEN = 147


def tables(zipgpu, nv, D, ctx, device=True):
    L = 1 << max(nv - 2, 1)
    pb = params_for(zipgpu, 1, D, 0, nv, L, ctx=ctx, comb=6, field=3, device=device)
    pi = params_for(zipgpu, 2, 1, 0, nv, L, ctx=ctx, comb=6, field=3, device=device)
    return pb, pi, desc_for(1, D, 0, nv, L, comb=6, field=3), desc_for(2, 1, 0, nv, L, comb=6, field=3)


class Reader:
    def __init__(self, b: bytes):
        self.b, self.pos = b, 0

    def take(self, n):
        assert self.pos + n <= len(self.b), "proof truncated"
        out = self.b[self.pos:self.pos + n]
        self.pos += n
        return out

    def u32(self):
        return int.from_bytes(self.take(4), "little")

    def u64(self):
        return int.from_bytes(self.take(8), "little")

    def sub(self):
        return Reader(self.take(self.u32()))

    def done(self):
        return self.pos == len(self.b)


def parse_poly_vec(r: Reader, fb: int, modulus: bytes):
    if r.done():
        return []
    flag = r.take(1)[0]
    assert flag in (0, 1)
    if flag:
        assert r.take(fb) == modulus
    polys = []
    while not r.done():
        n = r.u32()
        assert flag or n == 0
        polys.append(r.take(n * fb))
    return polys


def parse_proof(proof: bytes, L: int, nv: int):
    """The Proof layout (lib.rs:93-127) with every nested length checked."""
    fb = 8 * L
    r = Reader(proof)
    comms = [(r.take(32), r.u64()) for _ in range(3)]
    zip_ = r.take(r.u32())
    ic = r.sub()
    res = r.sub()
    md = r.sub()
    mp = r.sub()
    lifted = r.sub()
    assert r.done()
    modulus = md.take(fb)
    ic_polys = parse_poly_vec(ic, fb, modulus)
    up, down = res.sub(), res.sub()
    assert res.done()
    up_n, down_n = [(len(x.b) - fb) // fb if x.b else 0 for x in (up, down)]
    for x in (up, down):
        assert not x.b or x.b[:fb] == modulus
    assert md.u32() == 1 and md.u32() == nv
    deg = md.u32()
    md.take(deg * nv * fb + fb)
    assert md.done()
    assert mp.take(fb) == modulus and mp.u32() == nv
    for _ in range(nv):
        mp.take(mp.u32() * fb)
    mp.take(fb)
    assert mp.done()
    lifted_polys = parse_poly_vec(lifted, fb, modulus)
    return dict(comms=comms, zip=zip_, ic=ic_polys, up=up_n, down=down_n, degree=deg, lifted=lifted_polys,
                modulus=int.from_bytes(modulus, "little"))


def test_biglinear_trace_satisfies_constraints(zipgpu):
    from zipgpu import uair

    bins, ints = uair.trace(8, 3)
    shifts, coeffs = uair.signature()
    assert bins.shape == (16, 256) and ints.shape == (1, 256) and coeffs.shape == (17, 33)

    def at(x, X):  # binary polynomial values at X
        return sum(((x >> np.uint64(k)) & np.uint64(1)).astype(np.int64) * X ** k for k in range(32))

    up1 = np.stack([at(b, 1) for b in bins] + [ints[0]])
    up2 = np.stack([at(b, 2) for b in bins] + [ints[0]])
    down = lambda v: np.stack([np.concatenate([v[s][c:], np.zeros(c, np.int64)]) for s, c in shifts])
    v1, v2 = np.concatenate([up1, down(up1)]), np.concatenate([up2, down(up2)])
    rows = slice(0, 255)  # the last row has no successor
    for k, row in enumerate(coeffs):
        X_is_two = k == 1
        val = row @ (v2 if X_is_two else v1)
        assert not val[rows].any(), k


def test_oracle_proof_layout(zipgpu, oracle):
    from zipgpu import uair

    nv = 6
    bins, ints = uair.trace(nv, 11)
    shifts, coeffs = uair.signature()
    _, _, db, di = tables(zipgpu, nv, 32, None, device=False)
    proof = oracle.zinc_prove_mle_first(db, di, nv, bins, 32, ints, shifts, coeffs, 3)
    P = parse_proof(proof, 3, nv)
    assert P["comms"][0] == (oracle.commit(db, bins, 16), 16)
    assert P["comms"][1] == (bytes(32), 0)
    assert P["comms"][2] == (oracle.commit(di, ints, 1), 1)
    assert len(P["ic"]) == 17 and all(len(p) <= 32 * 24 for p in P["ic"])
    assert (P["up"], P["down"], P["degree"]) == (17, 16, 3)
    assert len(P["lifted"]) == 17 and len(P["lifted"][16]) <= 24
    assert oracle.is_probable_prime_base2(P["modulus"], 3) and P["modulus"].bit_length() <= 192
    # the PCS stream: two prove_f transcripts (binary table, then integer table)
    assert len(P["zip"]) == oracle.proof_size(db, 16) + oracle.proof_size(di, 1)
    # BigLinearUairWithPublicInput: 4 public binary columns, neither committed nor in the proof
    Q = parse_proof(oracle.zinc_prove_mle_first(db, di, nv, bins, 32, ints, shifts, coeffs, 3, n_pub_bin=4), 3, nv)
    assert Q["comms"][0] == (oracle.commit(db, bins[4:], 12), 12) and len(Q["lifted"]) == 13
    assert len(Q["zip"]) == oracle.proof_size(db, 12) + oracle.proof_size(di, 1)
    assert Q["modulus"] != P["modulus"]  # the public entries are absorbed before the prime


def test_driver_rejects_bad_arguments(zipgpu):
    from zipgpu import uair

    nv = 6
    pb, pi, _, _ = tables(zipgpu, nv, 32, None, device=False)
    bins, ints = uair.trace(nv, 1)
    shifts, coeffs = uair.signature()
    with pytest.raises(zipgpu.ZipError):  # parameters without a device
        zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs)
    with pytest.raises(ValueError):  # coefficient rows of the wrong width
        zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs[:, :-1])


def small_uair(rng, nb, ni, shifts, nc, D, nv):
    n = 1 << nv
    mask = (1 << D) - 1
    bins = rng.integers(0, 1 << 63, size=(nb, n), dtype=np.uint64) & np.uint64(mask)
    ints = rng.integers(-(2**40), 2**40, size=(ni, n), dtype=np.int64)
    coeffs = rng.integers(-3, 4, size=(nc, nb + ni + len(shifts)), dtype=np.int64)
    return bins, ints, coeffs


@pytest.mark.gpu
@pytest.mark.parametrize("nv,seed", [(6, 11), (9, 5), (10, 2)])
def test_gpu_biglinear_proof_matches_oracle(zipgpu, oracle, ctx, nv, seed):
    from zipgpu import uair

    bins, ints = uair.trace(nv, seed)
    shifts, coeffs = uair.signature()
    pb, pi, db, di = tables(zipgpu, nv, 32, ctx)
    got = zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs)
    want = oracle.zinc_prove_mle_first(db, di, nv, bins, 32, ints, shifts, coeffs, 3)
    assert len(got) == len(want)
    assert got == want
    P = parse_proof(got, 3, nv)
    assert (P["up"], P["down"]) == (17, 16)
    # deterministic
    assert zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs) == got


@pytest.mark.gpu
@pytest.mark.parametrize("nv", [6, 9])
def test_gpu_biglinear_public_input_matches_oracle(zipgpu, oracle, ctx, nv):
    """BigLinearUairWithPublicInput (test-uair/src/lib.rs:458-489): the first
    four binary columns are public."""
    from zipgpu import uair

    bins, ints = uair.trace(nv, 21)
    shifts, coeffs = uair.signature()
    pb, pi, db, di = tables(zipgpu, nv, 32, ctx)
    got = zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs, n_pub_bin=4)
    want = oracle.zinc_prove_mle_first(db, di, nv, bins, 32, ints, shifts, coeffs, 3, n_pub_bin=4)
    assert got == want
    P = parse_proof(got, 3, nv)
    assert P["comms"][0][1] == 12 and len(P["lifted"]) == 13
    # the public columns change the transcript: a different proof than without them
    assert got != zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs)


@pytest.mark.gpu
@pytest.mark.parametrize("nb,ni,shifts,nc,D", [
    (3, 2, [(0, 1), (3, 2), (4, 1)], 4, 8),
    (2, 0, [(1, 3)], 2, 32),           # binary table only
    (0, 2, [(0, 1), (1, 1)], 3, 8),    # integer table only
    (1, 1, [], 1, 64),                 # no shifts
    (2, 3, [(0, 1), (2, 1)], 3, 16),   # public: 1 binary, 2 integer columns
    (1, 2, [(1, 2)], 2, 8),            # every binary column public
])
def test_gpu_small_uairs_match_oracle(zipgpu, oracle, ctx, nb, ni, shifts, nc, D):
    nv = 7
    npb, npi = {(2, 3): (1, 2), (1, 2): (1, 0)}.get((nb, ni), (0, 0))
    rng = np.random.default_rng(nb * 100 + ni * 10 + nc)
    bins, ints, coeffs = small_uair(rng, nb, ni, shifts, nc, D, nv)
    pb, pi, db, di = tables(zipgpu, nv, D, ctx)
    got = zipgpu.ZincPlusPiop.prove_mle_first(pb if nb > npb else None, pi if ni > npi else None, nv,
                                              bins if nb else None, D, ints if ni else None, shifts, coeffs,
                                              n_pub_bin=npb, n_pub_int=npi)
    want = oracle.zinc_prove_mle_first(db, di, nv, bins if nb else None, D, ints if ni else None, shifts, coeffs, 3,
                                       n_pub_bin=npb, n_pub_int=npi)
    assert got == want
    parse_proof(got, 3, nv)


@pytest.mark.gpu
@pytest.mark.parametrize("nv", [14, 16, 18])
def test_gpu_biglinear_proof_matches_c_chain_at_size(zipgpu, oracle, ctx, nv):
    """Config 4's shape (16 rows per table, 192-bit field) at 2^14, 2^16 and
    2^18 rows: the GPU proof equals the oracle's C chain byte for byte, and the
    oracle's restated Zinc+ verifier accepts it; a tampered copy is rejected."""
    from zipgpu import uair

    bins, ints = uair.trace(nv, 0xB16 + nv)
    shifts, coeffs = uair.signature()
    L = 1 << (nv - 4)
    pb = params_for(zipgpu, 1, 32, 0, nv, L, ctx=ctx, comb=6, field=3)
    pi = params_for(zipgpu, 2, 1, 0, nv, L, ctx=ctx, comb=6, field=3)
    db, di = desc_for(1, 32, 0, nv, L, comb=6, field=3), desc_for(2, 1, 0, nv, L, comb=6, field=3)
    got = zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs)
    U = oracle.Uair.linear(16, 1, 32, shifts, coeffs, uair.ideal_roots())
    oracle.set_threads(0)
    want = oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=True)
    assert len(got) == len(want)
    assert got == want
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, got) == 0
    bad = bytearray(got)
    bad[len(bad) - 100] ^= 1  # inside the witness lifted evaluations
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, bytes(bad)) != 0
    pb.close()
    pi.close()


def _terms_of_rows(coeffs):
    """Constraint rows over [up, down] as terms (one column each)."""
    return [[(int(c), [j]) for j, c in enumerate(row) if int(c) != 0] for row in coeffs]


@pytest.mark.gpu
@pytest.mark.parametrize("nv", [10, 14])
def test_gpu_combined_path_biglinear_matches_oracle(zipgpu, oracle, ctx, nv):
    """The reference's default path (MLE_FIRST = false: step1_combined,
    prove_combined) on BigLinearUair: the GPU bytes equal the oracle's combined
    chain, and, BigLinear's ideals being non-zero, the MLE-first bytes too."""
    from zipgpu import uair

    bins, ints = uair.trace(nv, 40 + nv)
    shifts, coeffs = uair.signature()
    pb, pi, db, di = tables(zipgpu, nv, 32, ctx)
    cons = _terms_of_rows(coeffs)
    got = zipgpu.ZincPlusPiop.prove(pb, pi, nv, bins, 32, ints, shifts, cons, [False] * len(cons), mle_first=False)
    U = oracle.Uair.linear(16, 1, 32, shifts, coeffs, uair.ideal_roots())
    oracle.set_threads(0)
    want = oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=False)
    assert got == want
    assert got == zipgpu.ZincPlusPiop.prove_mle_first(pb, pi, nv, bins, 32, ints, shifts, coeffs)
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, got) == 0


@pytest.mark.gpu
def test_gpu_combined_path_skips_zero_ideals(zipgpu, oracle, ctx):
    nv, D = 8, 8
    rng = np.random.default_rng(5)
    shifts = [(0, 1), (2, 3)]
    bins, ints, coeffs = small_uair(rng, 2, 2, shifts, 3, D, nv)
    pb, pi, db, di = tables(zipgpu, nv, D, ctx)
    zero = [True, False, True]
    cons = _terms_of_rows(coeffs)
    got = zipgpu.ZincPlusPiop.prove(pb, pi, nv, bins, D, ints, shifts, cons, zero, mle_first=False)
    U = oracle.Uair.linear(2, 2, D, shifts, coeffs, [None, 1, None])
    assert got == oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=False)
    P = parse_proof(got, 3, nv)
    assert P["ic"][0] == b"" and P["ic"][2] == b""


@pytest.mark.gpu
@pytest.mark.parametrize("nv", [8, 12])
def test_gpu_combined_path_products_match_oracle_and_verify(zipgpu, oracle, ctx, nv):
    """A UAIR of degree two (integer x integer, binary x integer and binary x
    binary products, a shifted factor): the combined path's ideal check sums the
    product polynomials row by row and the CPR comb has degree four; the bytes
    equal the oracle's and its restated verifier accepts them."""
    n = 1 << nv
    rng = np.random.default_rng(nv)
    D = 16
    x = rng.integers(-(2**20), 2**20, size=n, dtype=np.int64)
    y = rng.integers(-(2**20), 2**20, size=n, dtype=np.int64)
    w = rng.integers(0, 1 << D, size=n, dtype=np.uint64)
    v = rng.integers(0, 1 << D, size=n, dtype=np.uint64)
    bins, ints = np.stack([w, v]), np.stack([x, y, x * y])
    # columns: up [w 0, v 1, x 2, y 3, z 4], down [w shifted by 1 (5), y shifted by 2 (6)]
    shifts = [(0, 1), (3, 2)]
    cons = [
        [(1, [2, 3]), (-1, [4])],                 # x * y - z = 0 (zero ideal)
        [(2, [0, 2]), (-1, [1, 3]), (3, [6])],    # 2 w x - v y + 3 y_down   in (X - 1)
        [(1, [0, 1]), (-1, [5, 5]), (1, [1])],    # w v - w_down^2 + v        in (X - 2)
    ]
    zero = [True, False, False]
    pb, pi, db, di = tables(zipgpu, nv, D, ctx)
    got = zipgpu.ZincPlusPiop.prove(pb, pi, nv, bins, D, ints, shifts, cons, zero, mle_first=False)
    U = oracle.Uair(2, 3, D, shifts, cons, [None, 1, 2])
    want = oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=False)
    assert got == want
    P = parse_proof(got, 3, nv)
    assert P["degree"] == 4 and P["ic"][0] == b""
    lay = zipgpu.read_proof(got, 3, nv)  # the library's own Proof reader agrees
    assert lay["cpr_degree"] == 4 and lay["n_ideal_values"] == 3 and lay["n_lifted"] == 5
    assert got[lay["zip_offset"]:lay["zip_offset"] + lay["zip_len"]] == P["zip"]
    # the honest x * y = z constraint passes; the other two are not in their ideals
    # for random columns, which the verifier's ideal check rejects (step 2)
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, got) == 2
    U2 = oracle.Uair(2, 3, D, shifts, cons, [None, None, None])
    got2 = zipgpu.ZincPlusPiop.prove(pb, pi, nv, bins, D, ints, shifts, cons, [True] * 3, mle_first=False)
    assert got2 == oracle.zinc_prove(db, di, nv, bins, ints, U2, 3, mle_first=False)
    assert oracle.zinc_verify(db, di, nv, None, None, U2, 3, got2) == 4  # the CPR sum is not zero
    with pytest.raises(zipgpu.ZipError):  # MLE first takes linear constraints only
        zipgpu.ZincPlusPiop.prove(pb, pi, nv, bins, D, ints, shifts, cons, zero, mle_first=True)


@pytest.mark.gpu
def test_gpu_combined_path_honest_product_uair_verifies(zipgpu, oracle, ctx):
    from test_zinc_oracle_chain import product_uair

    nv, D = 9, 16
    bins, ints, U = product_uair(oracle, nv, 3)
    pb, pi, db, di = tables(zipgpu, nv, D, ctx)
    got = zipgpu.ZincPlusPiop.prove(pb, pi, nv, bins, D, ints, U.shifts, U.constraints,
                                    [r is None for r in U.ideals], mle_first=False)
    assert got == oracle.zinc_prove(db, di, nv, bins, ints, U, 3, mle_first=False)
    assert oracle.zinc_verify(db, di, nv, None, None, U, 3, got) == 0
