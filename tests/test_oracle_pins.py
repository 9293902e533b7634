"""Pins of the oracle (the CPU restatement of the reference path) against the
reference's own known-answer and property tests, and against independent
Python implementations.  CPU only.

Reference tests restated here:
  octet_reversal.rs:35-72        octet reversal KATs and involution
  params.rs:232-242              F65537 base twiddles are the 8th roots of unity
  radix8.rs:224-284              pNTT reduced mod 65537 == radix-2 NTT
  iprs.rs:200-212                IprsCode::new / new_with_optimal_depth validity
  raa.rs:375-455                 RAA linearity, 16-element KAT, zero codeword
  phase_commit.rs:578-600        linearity of encode_rows
  phase_commit.rs:739-805        proof size formula
  phase_prove.rs:455-483         prove eval == MLE(point) for scalar evals
  phase_verify.rs:361-1385       verifier accepts honest proofs, rejects tampering
  merkle.rs:443-469              Merkle prove/verify (through the verifier)
BLAKE3 is pinned against the `blake3` wheel, Miller-Rabin against known
base-2 strong pseudoprimes.
"""
import blake3
import numpy as np
import pytest

from util import binary_evals, desc_for, i32_evals

P = 65537


# ------------------------------------------------------------------ BLAKE3
@pytest.mark.parametrize("n", [0, 1, 31, 64, 65, 1023, 1024, 1025, 2048, 3000, 4096, 70000])
def test_blake3_matches_wheel(oracle, n):
    data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
    assert oracle.blake3(data) == blake3.blake3(data).digest()
    assert oracle.blake3_xof(data, 131) == blake3.blake3(data).digest(length=131)


def test_blake3_parent_merges_are_hazmat(oracle):
    """merge_subtrees_{non_root,root} (merkle.rs:210-212) = BLAKE3 parent nodes:
    a 4-chunk input's hash is the root merge of two non-root merges."""
    data = np.random.default_rng(1).integers(0, 256, 4096, dtype=np.uint8).tobytes()
    cv = [oracle.blake3_chunk_cv(data[i * 1024:(i + 1) * 1024], i) for i in range(4)]
    left = oracle.blake3_parent(cv[0], cv[1], False)
    right = oracle.blake3_parent(cv[2], cv[3], False)
    assert oracle.blake3_parent(left, right, True) == blake3.blake3(data).digest()


# --------------------------------------------------------------- pNTT pins
def test_octet_reversal_kats(oracle):
    assert oracle.octet_reversal(0b101_111_010_000_110, 5) == 0b110_000_010_111_101
    assert oracle.octet_reversal(0b101_111_010_000_110_000, 6) == 0b000_110_000_010_111_101
    assert oracle.octet_reversal(0, 0) == 0
    for i in range(8):
        assert oracle.octet_reversal(i, 1) == i
    for n in range(0, 4):
        for x in range(8 ** n):
            assert oracle.octet_reversal(oracle.octet_reversal(x, n), n) == x


def test_base_twiddles_are_8th_roots(oracle):
    assert list(oracle.roots_of_unity(8)) == [1, 4096, -256, 16, -1, -4096, 256, -16]


def test_iprs_code_validity(oracle):
    dims = oracle.iprs_dims
    assert dims(1, 0) is not None
    assert dims(8, 0) is not None
    assert dims(1, 1) is None
    assert dims(8, 1) is not None
    opt = lambda L: dims(L, oracle.iprs_optimal_depth(L))  # noqa: E731
    assert opt(1) is None and opt(8) is not None and opt(12) is None and opt(16) is not None
    assert oracle.iprs_optimal_depth(4096) == 2 and oracle.iprs_optimal_depth(16384) == 2
    assert oracle.iprs_optimal_depth(256) == 1 and oracle.iprs_optimal_depth(64) == 1
    # codeword_len must stay below the field size (params.rs:60-66)
    assert dims(16384, 2, 4) is not None and dims(16384, 2, 8) is None


def _ntt_mod_p(values, n):
    w = pow(3, 65536 // n, P)
    a = [v % P for v in values] + [0] * (n - len(values))

    def rec(a, w):
        if len(a) == 1:
            return a
        e, o = rec(a[0::2], w * w % P), rec(a[1::2], w * w % P)
        out, x = [0] * len(a), 1
        for k in range(len(a) // 2):
            t = x * o[k] % P
            out[k], out[k + len(a) // 2] = (e[k] + t) % P, (e[k] - t) % P
            x = x * w % P
        return out

    return rec(a, w)


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_pntt_equals_ntt_mod_p(oracle, depth):
    """pntt_against_arkworks (radix8.rs:257-284): base_len 32, rate 1/2."""
    row_len = 32 * 8 ** depth
    desc = desc_for(0, 1, 0, row_len.bit_length() - 1, row_len, depth=depth, rep=2, comb=4)
    row = np.zeros((row_len, 4), np.uint64)
    row[:, 0] = np.arange(row_len)
    enc = oracle.encode_wide(desc, row, 4)
    got = []
    for limbs in enc:
        v = sum(int(x) << (64 * i) for i, x in enumerate(limbs))
        if v >> 255:
            v -= 1 << 256
        got.append(v % P)
    assert got == _ntt_mod_p(list(range(row_len)), 2 * row_len)


# ------------------------------------------------------------------ RAA
def test_raa_known_answer(oracle):
    """encoding_produces_predictable_results (raa.rs:398-413): pins rand 0.9
    StdRng(ChaCha12) seeding and SliceRandom::shuffle."""
    desc = desc_for(0, 1, 1, 2, 4, comb=4)
    row = np.zeros((4, 4), np.uint64)
    row[:, 0] = [1, 2, 3, 4]
    enc = oracle.encode_wide(desc, row, 4)
    expect = [0x1E, 0x36, 0x39, 0x5A, 0x70, 0x7E, 0xA5, 0xC1, 0xCB, 0xDC, 0xF9, 0x11E, 0x124,
              0x14C, 0x14D, 0x160]
    assert [int(x) for x in enc[:, 0]] == expect
    assert not enc[:, 1:].any()


def test_raa_linearity_and_zero(oracle):
    desc = desc_for(0, 1, 1, 10, 256, comb=4)
    rng = np.random.default_rng(5)
    a = rng.integers(0, 1 << 20, (256, 4), dtype=np.uint64)
    b = rng.integers(0, 1 << 20, (256, 4), dtype=np.uint64)
    ea, eb, eab = (oracle.encode_wide(desc, x, 4) for x in (a, b, a + b))
    assert np.array_equal(ea + eb, eab)
    assert not oracle.encode_wide(desc, np.zeros((256, 4), np.uint64), 4).any()


def test_shuffle_is_a_permutation_and_deterministic(oracle):
    p = oracle.shuffle_identity(12345, 1000)
    assert sorted(p.tolist()) == list(range(1000))
    assert np.array_equal(p, oracle.shuffle_identity(12345, 1000))
    assert not np.array_equal(p, oracle.shuffle_identity(54321, 1000))


# -------------------------------------------------------------- encoding
def test_encode_linearity_i32(oracle, rng):
    """linear_code_preserves_linearity (phase_commit.rs:578-600), i32 -> i128."""
    desc = desc_for(0, 1, 0, 12, 4096)
    a, b = i32_evals(rng, 4096), i32_evals(rng, 4096)
    ea = oracle.encode_rows(desc, a).view(np.uint64).reshape(-1, 2)
    eb = oracle.encode_rows(desc, b).view(np.uint64).reshape(-1, 2)
    eab = oracle.encode_rows(desc, (3 * a + 5 * b).astype(np.int32)).view(np.uint64).reshape(-1, 2)
    to_int = lambda x: [(int(h) << 64 | int(l)) for l, h in x]  # noqa: E731
    m = (1 << 128) - 1
    assert to_int(eab) == [(3 * x + 5 * y) & m for x, y in zip(to_int(ea), to_int(eb))]


def test_binary_encode_is_bitplane_linear(oracle, rng):
    """A binary codeword lane equals the i64 encoding of that coefficient's bit plane."""
    desc = desc_for(1, 32, 0, 10, 1024)
    ev = binary_evals(rng, 1024, 32)
    cw = oracle.encode_rows(desc, ev).view(np.int64).reshape(-1, 32)
    d_i = desc_for(0, 1, 0, 10, 1024)
    for lane in (0, 7, 31):
        plane = ((ev >> np.uint64(lane)) & np.uint64(1)).astype(np.int32)
        ref = oracle.encode_rows(d_i, plane).view(np.int64).reshape(-1, 2)[:, 0]
        assert np.array_equal(cw[:, lane], ref)


# ------------------------------------------------------------ primality
def test_miller_rabin_base2_semantics(oracle):
    # strong pseudoprimes to base 2 pass a pure base-2 test
    for n in (2047, 3277, 4033, 4681, 8321):
        assert oracle.is_probable_prime_base2(n, 1)
    for n in (2049, 9, 15, 561, 1105):
        assert not oracle.is_probable_prime_base2(n, 1)
    for n in (3, 5, 65537, (1 << 61) - 1, (1 << 127) - 1):
        assert oracle.is_probable_prime_base2(n, 2)


def test_transcript_prime_is_prime(oracle):
    t = oracle.Transcript()
    t.absorb_slice(b"\x00" * 32)
    p = t.get_prime(4)
    assert p % 2 == 1 and p < 1 << 256
    for a in (3, 5, 7, 11, 13, 17, 19, 23):
        d, s = p - 1, 0
        while d % 2 == 0:
            d, s = d // 2, s + 1
        x = pow(a, d, p)
        assert x in (1, p - 1) or any(pow(x, 2 ** r, p) == p - 1 for r in range(1, s))


# ------------------------------------------------------- commit / prove
def _mont_value(inner: bytes, p: int, limbs: int) -> int:
    return int.from_bytes(inner, "little") * pow(1 << (64 * limbs), -1, p) % p


def _mle(evals, point, p):
    vals = [int(v) % p for v in evals]
    for r in point:  # fold the lowest variable first (bit 0 of the index)
        r %= p
        vals = [(vals[2 * i] * (1 - r) + vals[2 * i + 1] * r) % p for i in range(len(vals) // 2)]
    return vals[0]


@pytest.mark.parametrize("row_len", [1024, 64, 16])
def test_prove_eval_is_mle_of_point(oracle, rng, row_len):
    """prove_returns_correct_evaluation (phase_prove.rs:455-483)."""
    nv = 10
    desc = desc_for(0, 1, 0, nv, row_len)
    ev = i32_evals(rng, 1 << nv, -(2**31), 2**31 - 1)
    point = [(-1) ** i * (i + 2) * 1234567 for i in range(nv)]
    _, proof, inner, mod = oracle.commit_prove(desc, ev, 1, point)
    p = int.from_bytes(mod, "little")
    assert _mont_value(inner, p, 4) == _mle(ev, point, p)


def _proof_size(num_rows, row_len, cw_len, cw_bytes, comb_limbs, batch, field_limbs=4):
    depth = (cw_len - 1).bit_length()
    return (num_rows * 16 * field_limbs + row_len * 8 * comb_limbs +
            147 * (batch * num_rows * cw_bytes + 24 + 32 * depth))


@pytest.mark.parametrize("case", [
    (0, 1, 0, 12, 4096, 1), (0, 1, 0, 12, 64, 1), (0, 1, 0, 10, 256, 2),
    (1, 32, 0, 12, 1024, 1), (1, 64, 0, 10, 1024, 1), (1, 32, 1, 12, 64, 1), (1, 3, 0, 10, 256, 3),
])
def test_commit_prove_verify(oracle, rng, case):
    ek, D, ck, nv, L, batch = case
    desc = desc_for(ek, D, ck, nv, L)
    n = 1 << nv
    polys = np.concatenate([binary_evals(rng, n, D) if ek else i32_evals(rng, n)
                            for _ in range(batch)])
    point = [i + 2 for i in range(nv)]
    root, proof, inner, mod = oracle.commit_prove(desc, polys, batch, point)
    R, C, cb = oracle.num_rows(desc), oracle.codeword_len(desc), oracle.cw_bytes(desc)
    assert len(proof) == _proof_size(R, L, C, cb, desc.comb_limbs, batch)
    assert oracle.verify(desc, root, batch, point, inner, proof) == 0
    # tampering (phase_verify.rs tamper tests) is rejected
    bad_eval = bytearray(inner)
    bad_eval[0] ^= 1
    assert oracle.verify(desc, root, batch, point, bytes(bad_eval), proof) != 0
    for pos in (40, R * 64 + 3, len(proof) - 40, len(proof) // 2):
        bad = bytearray(proof)
        bad[pos] ^= 0x10
        assert oracle.verify(desc, root, batch, point, inner, bytes(bad)) != 0
    bad_root = bytes([root[0] ^ 1]) + root[1:]
    assert oracle.verify(desc, bad_root, batch, point, inner, proof) != 0
    assert oracle.verify(desc, root, batch, point, inner, proof[:-1]) != 0


def test_commit_rejects_bad_shapes(oracle, rng):
    # bit budget (validate_input): 8 columns of Int<3> cannot hold binary combinations
    desc = desc_for(1, 32, 0, 10, 1024, comb=3)
    with pytest.raises(ValueError):
        oracle.commit(desc, binary_evals(rng, 1024, 32), 1)
    with pytest.raises(ValueError):  # row_len not dividing the poly size
        oracle.commit(desc_for(0, 1, 0, 4, 32), i32_evals(rng, 16), 1)
