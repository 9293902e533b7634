"""LinearCode::encode_f (zip-plus/src/code.rs:69-71): codes over prime-field
elements.  The oracle's restatement (IPRS: the pNTT with F::from_with_cfg of each
table entry, iprs.rs:88-106; RAA and sign-flipping RAA over the field, raa.rs:
93-127, raa_sign_flip.rs:31-69) is pinned by encode_wide, whose integer codeword
reduced mod p must equal encode_f of the reduced row (the codes are linear over
Z); the GPU's zg_encode_f equals the oracle on full-range field elements."""
import numpy as np
import pytest

from util import desc_for, params_for


def prime(oracle, L, tag):
    t = oracle.Transcript()
    t.absorb_slice(tag)
    return t.get_prime(L)


def inner(v, p, L):
    x = (v % p) * (1 << (64 * L)) % p
    return [(x >> (64 * i)) & ((1 << 64) - 1) for i in range(L)]


CODES = [(0, 64, 0), (0, 1024, 0), (0, 4096, 2), (1, 256, 0), (2, 256, 0), (1, 16, 0)]


@pytest.mark.parametrize("L", [2, 3, 4])
@pytest.mark.parametrize("ck,row_len,depth", CODES)
def test_oracle_encode_f_is_encode_wide_mod_p(oracle, L, ck, row_len, depth):
    p = prime(oracle, L, b"encode_f")
    rng = np.random.default_rng(row_len + L)
    ints = [int(v) for v in rng.integers(-(2**40), 2**40, size=row_len)]
    limbs = 4
    wide = np.array([[(v >> (64 * w)) & ((1 << 64) - 1) for w in range(limbs)] for v in ints], np.uint64)
    d = desc_for(0, 1, ck, 10 if row_len <= 1024 else 12, row_len, depth=depth)
    enc = oracle.encode_wide(d, wide, limbs)
    want = np.array([inner(sum(int(x) << (64 * w) for w, x in enumerate(r)) - (1 << 256) * (int(r[-1]) >> 63), p, L)
                     for r in enc], np.uint64)
    got = oracle.encode_f(d, p, L, np.array([inner(v, p, L) for v in ints], np.uint64))
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("L", [1, 3, 4])
@pytest.mark.parametrize("ck,row_len,depth", CODES + [(0, 16384, 0)])
def test_gpu_encode_f_matches_oracle(zipgpu, oracle, ctx, L, ck, row_len, depth):
    p = prime(oracle, L, b"encode_f gpu")
    rng = np.random.default_rng(7 * row_len + L)
    row = np.array([inner(int.from_bytes(rng.bytes(8 * L + 8), "little"), p, L) for _ in range(row_len)], np.uint64)
    nv = max(12, row_len.bit_length() - 1)
    d = desc_for(0, 1, ck, nv, row_len, depth=depth)
    # encode_f does not depend on the evaluation type; RAA parameters take binary
    # evaluations (the i32 table's codewords would not fit its 32-bit entries)
    ek, D = (0, 1) if ck == 0 else (1, 32)
    pp = params_for(zipgpu, ek, D, ck, nv, row_len, depth=depth, ctx=ctx)
    got = zipgpu.ZipPlus.encode_f(pp, p, L, row)
    assert np.array_equal(got, oracle.encode_f(d, p, L, row))
    pp.close()
