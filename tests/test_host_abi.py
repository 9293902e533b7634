"""CPU tests of the product library: it loads, exports every symbol that
include/zipgpu.h declares, and its host-side logic (code tables, RAA
permutations, Fiat-Shamir transcript, prime sampling, encode_wide, verifier)
matches the oracle.  No GPU compute is called here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from util import binary_evals, desc_for, i32_evals, params_for

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "zipgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(zipgpu):
    names = _declared_symbols()
    assert len(names) >= 30
    lib = C.CDLL(zipgpu.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(zipgpu.EXPORTS)


def test_version_and_errors(zipgpu):
    assert b"sm_100a" in zipgpu.lib().zg_version()
    with pytest.raises(zipgpu.ZipError) as e:  # row_len does not divide poly_size
        params_for(zipgpu, 1, 32, 0, 4, 32, device=False)
    assert e.value.status == 1
    with pytest.raises(zipgpu.ZipError):  # codeword longer than F65537
        params_for(zipgpu, 1, 32, 0, 16, 1 << 15, device=False)
    with pytest.raises(zipgpu.ZipError):  # RaaCode::new width check
        params_for(zipgpu, 1, 32, 1, 30, 1 << 15, device=False)


@pytest.mark.parametrize("row_len,depth", [(4096, 0), (64, 0), (16384, 0), (256, 1), (2048, 3),
                                           (8, 0), (1024, 0)])
def test_iprs_tables_match_oracle(zipgpu, oracle, row_len, depth):
    pp = params_for(zipgpu, 1, 32, 0, 14 if row_len <= 16384 else 15, row_len, depth, device=False)
    bm, tw = pp.iprs_tables()
    bo, to = oracle.iprs_tables(row_len, pp.info.depth)
    assert np.array_equal(bm, bo) and np.array_equal(tw, to)


def test_raa_perms_match_oracle(zipgpu, oracle):
    pp = params_for(zipgpu, 1, 32, 1, 16, 256, device=False)
    p1, p2 = pp.raa_perms()
    assert np.array_equal(p1, oracle.shuffle_identity(1, 1024))
    assert np.array_equal(p2, oracle.shuffle_identity(2, 1024))


def test_transcript_and_prime_match_oracle(zipgpu, oracle):
    t = zipgpu.PcsProverTranscript([b"\x42" * 32])
    o = oracle.Transcript()
    o.absorb_slice(b"\x42" * 32)
    assert t.get_challenge(16) == o.challenge(16)
    t.absorb(b"xyz" * 1000)
    o.absorb(b"xyz" * 1000)
    assert t.get_challenge(77) == o.challenge(77)
    assert t.get_random_field_cfg(4) == o.get_prime(4)
    assert t.get_challenge(4) == o.challenge(4)
    assert t.get_random_field_cfg(3) == o.get_prime(3)
    assert t.get_challenge(32) == o.challenge(32)


def test_transcript_across_block_and_chunk_boundaries(zipgpu, oracle):
    """The library's host transcript (the incremental BLAKE3 hasher shared with
    the device's Fiat-Shamir step) against the oracle's, whose BLAKE3 is pinned
    to the blake3 package: absorbs of random sizes cross 64-byte blocks and
    1 KiB chunks many times (chunk completions, stack merges), with challenges
    read between them."""
    rng = np.random.default_rng(0xB1A)
    t = zipgpu.PcsProverTranscript()
    o = oracle.Transcript()
    for _ in range(120):
        n = int(rng.choice([0, 1, 3, 26, 52, 63, 64, 65, 127, 1023, 1024, 1025, int(rng.integers(0, 3000))]))
        b = rng.bytes(n)
        t.absorb(b)
        o.absorb(b)
        if rng.random() < 0.4:
            k = int(rng.integers(1, 80))
            assert t.get_challenge(k) == o.challenge(k)
    assert t.get_challenge(32) == o.challenge(32)


@pytest.mark.parametrize("code_kind,row_len", [(0, 1024), (0, 64), (1, 64)])
def test_encode_wide_matches_oracle(zipgpu, oracle, code_kind, row_len):
    pp = params_for(zipgpu, 1, 32, code_kind, 12, row_len, device=False)
    desc = desc_for(1, 32, code_kind, 12, row_len)
    row = np.random.default_rng(9).integers(0, 2**63, (row_len, 5), dtype=np.uint64)
    assert np.array_equal(zipgpu.ZipPlus.encode_wide(pp, row, 5), oracle.encode_wide(desc, row, 5))


@pytest.mark.parametrize("case", [(0, 1, 0, 12, 4096, 1), (0, 1, 0, 12, 64, 2),
                                  (1, 32, 0, 12, 1024, 1), (1, 32, 1, 12, 64, 1),
                                  (1, 64, 0, 10, 256, 2)])
def test_host_verifier_accepts_oracle_proofs(zipgpu, oracle, rng, case):
    ek, D, ck, nv, L, batch = case
    desc = desc_for(ek, D, ck, nv, L)
    polys = np.concatenate([binary_evals(rng, 1 << nv, D) if ek else i32_evals(rng, 1 << nv)
                            for _ in range(batch)])
    point = [(-1) ** i * (3 * i + 1) for i in range(nv)]
    root, proof, inner, _ = oracle.commit_prove(desc, polys, batch, point)
    pp = params_for(zipgpu, ek, D, ck, nv, L, device=False)
    comm = zipgpu.ZipPlusCommitment(root, batch)
    zipgpu.ZipPlus.verify(pp, comm, point, inner, proof)
    for pos in (5, len(proof) // 3, len(proof) - 3):
        bad = bytearray(proof)
        bad[pos] ^= 4
        with pytest.raises(zipgpu.ZipError) as e:
            zipgpu.ZipPlus.verify(pp, comm, point, inner, bytes(bad))
        assert e.value.status in (2, 3)
    with pytest.raises(zipgpu.ZipError) as e:
        zipgpu.ZipPlus.verify(pp, comm, point, inner, proof[: len(proof) // 2])
    assert e.value.status == 3


def _verdict(zipgpu, pp, comm, point, inner, proof):
    try:
        zipgpu.ZipPlus.verify(pp, comm, point, inner, proof)
        return 0
    except zipgpu.ZipError as e:
        return e.status


def verdicts_match_oracle(zipgpu, oracle, pp, desc, ek, D, nv, rng, cases=40):
    """Tampered and truncated proofs get the oracle's verdict (0 accept, 2 rejected
    opening, 3 malformed), including the first failure winning over a later one."""
    if ek == 2:
        poly = rng.integers(-(2**63), 2**63 - 1, size=1 << nv, dtype=np.int64, endpoint=True)
    else:
        poly = binary_evals(rng, 1 << nv, D) if ek else i32_evals(rng, 1 << nv)
    point = [(-1) ** i * (5 * i + 2) for i in range(nv)]
    root, proof, inner, _ = oracle.commit_prove(desc, poly, 1, point)
    comm = zipgpu.ZipPlusCommitment(root, 1)
    variants = [proof, proof[:-1], proof[: len(proof) // 2]]
    for pos in rng.integers(0, len(proof), size=cases):
        bad = bytearray(proof)
        bad[int(pos)] ^= 1 << int(rng.integers(0, 8))
        variants.append(bytes(bad))
    # a bad early opening together with a truncated tail: the opening wins
    head = len(proof) - zipgpu_openings_bytes(pp)
    bad = bytearray(proof[: len(proof) - 7])
    bad[head + 3] ^= 1
    variants.append(bytes(bad))
    for v in variants:
        want = oracle.verify(desc, root, 1, point, inner, v)
        assert _verdict(zipgpu, pp, comm, point, inner, v) == want


def zipgpu_openings_bytes(pp):
    """Bytes of the column openings at the end of a batch-1 proof."""
    i = pp.info
    depth = i.codeword_len.bit_length() - 1
    return pp.zt.num_openings * (i.num_rows * i.cw_bytes + 24 + 32 * depth)


@pytest.mark.parametrize("case", [(0, 1, 0, 12, 4096), (1, 32, 0, 13, 1 << 13),
                                  (1, 32, 1, 12, 64), (1, 64, 0, 11, 512), (2, 1, 0, 12, 1024)])
def test_host_verifier_verdicts_match_oracle(zipgpu, oracle, rng, case):
    ek, D, ck, nv, L = case
    pp = params_for(zipgpu, ek, D, ck, nv, L, device=False)
    verdicts_match_oracle(zipgpu, oracle, pp, desc_for(ek, D, ck, nv, L), ek, D, nv, rng)


def test_device_entry_points_need_a_context(zipgpu):
    pp = params_for(zipgpu, 1, 32, 0, 10, 1024, device=False)
    with pytest.raises(zipgpu.ZipError) as e:
        zipgpu.ZipPlus.commit(pp, [np.zeros(1024, np.uint64)])
    assert e.value.status == 8


def test_noalloc_root_rejects_misaligned_leaves_before_any_device_call(zipgpu):
    # The argument checks of zg_merkle_root_noalloc_d run before it touches the
    # device, so a misaligned leaf pointer is refused even with no GPU present.
    # The pointers are never dereferenced.
    fn = zipgpu.lib().zg_merkle_root_noalloc_d
    assert fn(0x10001, 4096, 256, 0x20000, None) == 1
    assert b"aligned" in zipgpu.lib().zg_last_error()
    assert fn(0x10002, 16, 16, 0x20000, None) == 1


def _mr(zipgpu, vals, L):
    arr = np.array([[(v >> (64 * i)) & ((1 << 64) - 1) for i in range(L)] for v in vals], np.uint64)
    out = np.zeros(len(vals), np.uint8)
    zipgpu.check(zipgpu.lib().zg_is_probable_prime_base2(arr.ctypes.data, L, len(vals), out.ctypes.data))
    return [bool(x) for x in out]


@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_miller_rabin_matches_oracle(zipgpu, oracle, L):
    """MillerRabin::test to base 2 (primality/src/lib.rs:12-19): the library's
    test (eight candidates per vector when the CPU has AVX-512 IFMA) agrees with
    the oracle's scalar test on random odd candidates, primes, the base-2 strong
    pseudoprimes of the reference's test_base_two (which pass) and small cases."""
    rng = np.random.default_rng(100 + L)
    top = 64 * L
    vals = [int.from_bytes(rng.bytes(8 * L), "little") | 1 for _ in range(1500)]
    vals += [int.from_bytes(rng.bytes(8 * L), "little") >> int(rng.integers(0, top - 3)) | 1 for _ in range(300)]
    vals += [2047, 3277, 4033, 4681, 8321, 15841, 29341, 42799, 49141, 52633, 65281, 74665, 80581, 85489,
             1, 2, 3, 4, 5, 9, 15, 17, 65537, (1 << 61) - 1, (1 << top) - 1]
    if L >= 2:
        vals += [(1 << 127) - 1, (1 << 89) - 1, 3825123056546413051]
    if L >= 4:
        vals += [2**255 - 19, 2**256 - 189]
    vals = [v % (1 << top) for v in vals]
    got = _mr(zipgpu, vals, L)
    want = [oracle.is_probable_prime_base2(v, L) for v in vals]
    assert got == want
    assert all(_mr(zipgpu, [2047, 3277, 4033], L))  # strong pseudoprimes to base 2 pass
    assert sum(got) > 0
