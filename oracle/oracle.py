"""ctypes front end of the oracle (``zipref``), the CPU restatement of the
reference Zip+ path.  Test infrastructure only: imported by ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``.

The shared library is built by ``oracle/Makefile`` into ``oracle/_build``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libzipref.so")

EVAL_I32, EVAL_BINPOLY, EVAL_I64 = 0, 1, 2
CODE_IPRS, CODE_RAA, CODE_RAA_SIGN_FLIP = 0, 1, 2


class Desc(C.Structure):
    """Mirror of ``zr_desc`` (same fields as the product's ``zg_params_desc``)."""

    _fields_ = [
        ("eval_kind", C.c_uint32),
        ("degree_plus_one", C.c_uint32),
        ("code_kind", C.c_uint32),
        ("rep", C.c_uint32),
        ("num_vars", C.c_uint32),
        ("row_len", C.c_uint32),
        ("iprs_depth", C.c_uint32),
        ("comb_limbs", C.c_uint32),
        ("field_limbs", C.c_uint32),
        ("num_openings", C.c_uint32),
    ]


class ScGroup(C.Structure):
    """Mirror of ``zr_sc_group`` (same layout as the product's ``zg_sumcheck_group``)."""

    _fields_ = [("degree", C.c_uint32), ("n_mles", C.c_uint32), ("n_products", C.c_uint32),
                ("mles", C.c_void_p), ("coeffs", C.c_void_p), ("offsets", C.c_void_p),
                ("indices", C.c_void_p), ("n_factors", C.c_uint32), ("factor_mles", C.c_void_p),
                ("factor_a", C.c_void_p), ("factor_b", C.c_void_p)]


class UairDesc(C.Structure):
    """Mirror of ``zr_uair``: a constraint system over [binary up, integer up,
    down] columns (see zipref.h)."""

    _fields_ = [("n_bin", C.c_uint32), ("n_int", C.c_uint32), ("n_pub_bin", C.c_uint32),
                ("n_pub_int", C.c_uint32), ("D", C.c_uint32), ("n_shifts", C.c_uint32),
                ("shift_src", C.c_void_p), ("shift_amt", C.c_void_p), ("n_cons", C.c_uint32),
                ("term_off", C.c_void_p), ("term_coeff", C.c_void_p), ("fac_off", C.c_void_p),
                ("fac_col", C.c_void_p), ("ideal_kind", C.c_void_p), ("ideal_root", C.c_void_p)]


class Uair:
    """A UAIR for the oracle's Zinc+ prover and verifier: `constraints` is a list
    of constraints, each a list of terms (integer coefficient, [column indices
    into up (binary, then integer) and down (shift order)]); `ideals` one root
    c per constraint for the ideal (X - c), or None for the zero ideal."""

    def __init__(self, n_bin, n_int, D, shifts, constraints, ideals, n_pub_bin=0, n_pub_int=0):
        self.n_bin, self.n_int, self.D = n_bin, n_int, D
        self.shifts, self.constraints, self.ideals = list(shifts), constraints, ideals
        self.n_pub_bin, self.n_pub_int = n_pub_bin, n_pub_int
        toff, coef, foff, fcol = [0], [], [0], []
        for terms in constraints:
            for c, facs in terms:
                coef.append(int(c))
                fcol.extend(int(x) for x in facs)
                foff.append(len(fcol))
            toff.append(len(coef))
        self._a = dict(
            src=np.array([s for s, _ in self.shifts] or [0], np.uint32),
            amt=np.array([a for _, a in self.shifts] or [0], np.uint32),
            toff=np.array(toff, np.uint32), coef=np.array(coef or [0], np.int64),
            foff=np.array(foff, np.uint32), fcol=np.array(fcol or [0], np.uint32),
            kind=np.array([0 if r is None else 1 for r in ideals] or [0], np.uint8),
            root=np.array([0 if r is None else int(r) for r in ideals] or [0], np.int64))
        a = self._a
        self.desc = UairDesc(n_bin, n_int, n_pub_bin, n_pub_int, D, len(self.shifts), _ptr(a["src"]),
                             _ptr(a["amt"]), len(constraints), _ptr(a["toff"]), _ptr(a["coef"]),
                             _ptr(a["foff"]), _ptr(a["fcol"]), _ptr(a["kind"]), _ptr(a["root"]))

    @classmethod
    def linear(cls, n_bin, n_int, D, shifts, coeff_rows, roots, n_pub_bin=0, n_pub_int=0):
        """From integer coefficient rows over [up, down] (one term per nonzero)."""
        cons = [[(int(c), [j]) for j, c in enumerate(row) if int(c) != 0] for row in coeff_rows]
        return cls(n_bin, n_int, D, shifts, cons, roots, n_pub_bin, n_pub_int)


def encode_f(desc: Desc, modulus: int, L: int, row) -> np.ndarray:
    """LinearCode::encode_f (zip-plus/src/code.rs:69-71) of a row of Montgomery
    inners (row_len, L) over the prime `modulus`: (codeword_len, L)."""
    r = np.ascontiguousarray(row, dtype=np.uint64)
    out = np.zeros((codeword_len(desc), L), np.uint64)
    if lib().zr_encode_f(C.byref(desc), _ptr(_limbs(modulus, L)), L, _ptr(r), _ptr(out)):
        raise ValueError("encode_f failed")
    return out


def zinc_prove(desc_bin: Desc, desc_int: Desc, nvars: int, bin_cols, int_cols, uair: Uair, L: int,
               mle_first: bool = True) -> bytes:
    """ZincPlusPiop::prove::<MLE_FIRST> (protocol/src/prover.rs:677-706) in C:
    the whole chain, steps 0-7, and the Proof transcription."""
    b, i = _piop_cols(bin_cols, int_cols, nvars)
    cap = 64 << 20
    out = C.create_string_buffer(cap)
    n = C.c_size_t(0)
    rc = lib().zr_zinc_prove(C.byref(desc_bin), C.byref(desc_int), nvars, _ptr(b), _ptr(i), C.byref(uair.desc), L,
                             1 if mle_first else 0, out, cap, C.byref(n))
    if rc:
        raise ValueError(f"zinc prove failed ({rc})")
    return out.raw[: n.value]


def zinc_verify(desc_bin: Desc, desc_int: Desc, nvars: int, pub_bin, pub_int, uair: Uair, L: int,
                proof: bytes) -> int:
    """ZincPlusPiop::verify (protocol/src/verifier.rs:715-771) in C: 0 accepts;
    otherwise the failing step (1 parse, 2 ideal check, 4 CPR, 5 multipoint, 6
    lifted evaluations, 7 PCS)."""
    b, i = _piop_cols(pub_bin, pub_int, nvars)
    return lib().zr_zinc_verify(C.byref(desc_bin), C.byref(desc_int), nvars, _ptr(b), _ptr(i), C.byref(uair.desc),
                                L, _buf(proof), len(proof))


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, u8p, sz = C.c_void_p, C.c_void_p, C.c_size_t
        L.zr_blake3.argtypes = [vp, sz, vp]
        L.zr_blake3_xof.argtypes = [vp, sz, vp, sz]
        L.zr_blake3_parent.argtypes = [vp, vp, C.c_int, vp]
        L.zr_blake3_chunk_cv.argtypes = [vp, sz, C.c_uint64, vp]
        L.zr_octet_reversal.argtypes = [sz, sz]
        L.zr_octet_reversal.restype = sz
        L.zr_iprs_dims.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, vp]
        L.zr_iprs_optimal_depth.argtypes = [C.c_uint32]
        L.zr_iprs_optimal_depth.restype = C.c_uint32
        L.zr_iprs_tables.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, vp, vp]
        L.zr_roots_of_unity.argtypes = [C.c_uint32, vp]
        L.zr_shuffle_identity.argtypes = [C.c_uint64, C.c_uint32, vp]
        L.zr_stdrng_u32.argtypes = [C.c_uint64, C.c_uint32]
        L.zr_stdrng_u32.restype = C.c_uint32
        L.zr_encode_rows.argtypes = [C.POINTER(Desc), vp, vp]
        L.zr_encode_wide.argtypes = [C.POINTER(Desc), vp, C.c_uint32, vp]
        L.zr_cw_bytes.argtypes = [C.POINTER(Desc)]
        L.zr_cw_bytes.restype = sz
        L.zr_num_rows.argtypes = [C.POINTER(Desc)]
        L.zr_num_rows.restype = C.c_uint32
        L.zr_codeword_len.argtypes = [C.POINTER(Desc)]
        L.zr_codeword_len.restype = C.c_uint32
        L.zr_merkle_root_rows.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_uint32, vp]
        L.zr_commit.argtypes = [C.POINTER(Desc), vp, C.c_uint32, vp]
        L.zr_proof_size.argtypes = [C.POINTER(Desc), C.c_uint32]
        L.zr_proof_size.restype = sz
        L.zr_commit_prove.argtypes = [C.POINTER(Desc), vp, C.c_uint32, vp, vp, vp, sz,
                                      C.POINTER(C.c_size_t), vp, vp]
        L.zr_verify.argtypes = [C.POINTER(Desc), vp, C.c_uint32, vp, vp, vp, sz]
        L.zr_tr_new.restype = vp
        L.zr_tr_free.argtypes = [vp]
        L.zr_tr_absorb.argtypes = [vp, vp, sz]
        L.zr_tr_absorb_slice.argtypes = [vp, vp, sz]
        L.zr_tr_challenge.argtypes = [vp, vp, sz]
        L.zr_tr_get_prime.argtypes = [vp, C.c_uint32, vp]
        L.zr_prove_f_on.argtypes = [C.POINTER(Desc), vp, C.c_uint32, vp, vp, vp, vp, sz, C.POINTER(sz), vp]
        L.zr_is_probable_prime_base2.argtypes = [vp, C.c_uint32]
        L.zr_set_threads.argtypes = [C.c_int]
        gp = C.POINTER(ScGroup)
        L.zr_sumcheck_prove.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_int, gp, C.c_uint32,
                                        vp, sz, C.POINTER(C.c_size_t), vp, vp]
        L.zr_sumcheck_verify.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_int, vp, C.c_uint32,
                                         vp, sz, vp, vp]
        L.zr_sumcheck_comb.argtypes = [vp, C.c_uint32, gp, vp, vp]
        L.zr_mle_evaluate.argtypes = [vp, C.c_uint32, vp, C.c_uint32, vp, vp]
        u32 = C.c_uint32
        L.zr_piop_eval_projection.argtypes = [vp, u32, vp, u32, u32, vp, u32, u32, vp, vp]
        L.zr_piop_lifted_evals.argtypes = [vp, u32, vp, u32, u32, vp, u32, u32, vp, vp]
        L.zr_tr_field_challenge.argtypes = [vp, vp, u32, vp]
        L.zr_tr_absorb_field.argtypes = [vp, vp, u32, vp]
        L.zr_commit_prove_f.argtypes = [C.POINTER(Desc), vp, u32, vp, vp, vp, sz, C.POINTER(C.c_size_t), vp, vp]
        L.zr_encode_f.argtypes = [C.POINTER(Desc), vp, u32, vp, vp]
        up = C.POINTER(UairDesc)
        L.zr_zinc_prove.argtypes = [C.POINTER(Desc), C.POINTER(Desc), u32, vp, vp, up, u32, C.c_int, vp, sz,
                                    C.POINTER(sz)]
        L.zr_zinc_verify.argtypes = [C.POINTER(Desc), C.POINTER(Desc), u32, vp, vp, up, u32, vp, sz]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _buf(b: bytes):
    return C.c_char_p(b)


def make_desc(eval_kind, D, code_kind, num_vars, row_len, depth=0, comb_limbs=None,
              field_limbs=4, num_openings=147, rep=4) -> Desc:
    if comb_limbs is None:
        comb_limbs = {EVAL_I32: 3, EVAL_I64: 6}.get(eval_kind, 5)
    return Desc(eval_kind, D if eval_kind == EVAL_BINPOLY else 1, code_kind, rep, num_vars,
                row_len, depth, comb_limbs, field_limbs, num_openings)


def set_threads(n: int) -> None:
    lib().zr_set_threads(int(n))


def blake3(data: bytes) -> bytes:
    out = C.create_string_buffer(32)
    lib().zr_blake3(_buf(data), len(data), out)
    return out.raw


def blake3_xof(data: bytes, n: int) -> bytes:
    out = C.create_string_buffer(n)
    lib().zr_blake3_xof(_buf(data), len(data), out, n)
    return out.raw


def blake3_parent(left: bytes, right: bytes, root: bool) -> bytes:
    out = C.create_string_buffer(32)
    lib().zr_blake3_parent(_buf(left), _buf(right), int(root), out)
    return out.raw


def blake3_chunk_cv(data: bytes, counter: int) -> bytes:
    out = C.create_string_buffer(32)
    lib().zr_blake3_chunk_cv(_buf(data), len(data), counter, out)
    return out.raw


def octet_reversal(x: int, n: int) -> int:
    return lib().zr_octet_reversal(x, n)


def iprs_dims(row_len, depth, rep=4):
    out = np.zeros(4, np.uint32)
    if lib().zr_iprs_dims(row_len, depth, rep, _ptr(out)):
        return None
    cw, base_len, base_dim, d = (int(v) for v in out)
    return dict(codeword_len=cw, base_len=base_len, base_dim=base_dim, depth=d)


def iprs_optimal_depth(row_len: int) -> int:
    return int(lib().zr_iprs_optimal_depth(row_len))


def iprs_tables(row_len, depth, rep=4):
    dims = iprs_dims(row_len, depth, rep)
    bm = np.zeros((dims["base_dim"], dims["base_len"]), np.int64)
    ntw = sum(dims["base_dim"] * 8 ** k * 56 for k in range(depth))
    tw = np.zeros(max(ntw, 1), np.int64)
    assert lib().zr_iprs_tables(row_len, depth, rep, _ptr(bm), _ptr(tw)) == 0
    return bm, tw[:ntw]


def roots_of_unity(n):
    out = np.zeros(n, np.int64)
    assert lib().zr_roots_of_unity(n, _ptr(out)) == 0
    return out


def shuffle_identity(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    lib().zr_shuffle_identity(seed, n, _ptr(out))
    return out


def stdrng_u32(seed: int, index: int) -> int:
    return lib().zr_stdrng_u32(seed, index)


def cw_bytes(desc: Desc) -> int:
    return lib().zr_cw_bytes(C.byref(desc))


def num_rows(desc: Desc) -> int:
    return lib().zr_num_rows(C.byref(desc))


def codeword_len(desc: Desc) -> int:
    return lib().zr_codeword_len(C.byref(desc))


def encode_rows(desc: Desc, evals: np.ndarray) -> np.ndarray:
    """Row-major num_rows x codeword_len codeword matrix, as raw bytes view."""
    R, Cl, cb = num_rows(desc), codeword_len(desc), cw_bytes(desc)
    out = np.zeros(R * Cl * cb, np.uint8)
    evals = np.ascontiguousarray(evals)
    assert lib().zr_encode_rows(C.byref(desc), _ptr(evals), _ptr(out)) == 0
    return out.reshape(R, Cl, cb)


def encode_wide(desc: Desc, row: np.ndarray, limbs: int) -> np.ndarray:
    """``LinearCode::encode_wide`` over Int<limbs>: row is (row_len, limbs) u64."""
    Cl = codeword_len(desc)
    out = np.zeros((Cl, limbs), np.uint64)
    row = np.ascontiguousarray(row, dtype=np.uint64)
    assert lib().zr_encode_wide(C.byref(desc), _ptr(row), limbs, _ptr(out)) == 0
    return out


def merkle_root_rows(rows: np.ndarray, elem_bytes: int) -> bytes:
    """rows: (n_rows, width*elem_bytes) uint8."""
    rows = np.ascontiguousarray(rows, dtype=np.uint8)
    n_rows = rows.shape[0]
    width = rows.shape[1] // elem_bytes
    out = C.create_string_buffer(32)
    rc = lib().zr_merkle_root_rows(_ptr(rows), n_rows, width, elem_bytes, out)
    if rc:
        raise ValueError("invalid merkle input")
    return out.raw


def commit(desc: Desc, polys: np.ndarray, batch: int) -> bytes:
    polys = np.ascontiguousarray(polys)
    out = C.create_string_buffer(32)
    rc = lib().zr_commit(C.byref(desc), _ptr(polys), batch, out)
    if rc:
        raise ValueError(f"commit failed ({rc})")
    return out.raw


def point_array(point) -> np.ndarray:
    """i128 coordinates -> (lo, hi) int64 pairs."""
    arr = np.zeros(2 * len(point), np.int64)
    for i, v in enumerate(point):
        v = int(v) & ((1 << 128) - 1)
        lo, hi = v & ((1 << 64) - 1), v >> 64
        arr[2 * i] = np.uint64(lo).astype(np.int64)
        arr[2 * i + 1] = np.uint64(hi).astype(np.int64)
    return arr


def proof_size(desc: Desc, batch: int) -> int:
    return lib().zr_proof_size(C.byref(desc), batch)


def commit_prove(desc: Desc, polys: np.ndarray, batch: int, point):
    """Returns (root, proof bytes, eval inner bytes, modulus bytes)."""
    polys = np.ascontiguousarray(polys)
    pt = point_array(point)
    cap = proof_size(desc, batch) + 64
    proof = C.create_string_buffer(cap)
    plen = C.c_size_t(0)
    root = C.create_string_buffer(32)
    ev = C.create_string_buffer(8 * desc.field_limbs)
    mod = C.create_string_buffer(8 * desc.field_limbs)
    rc = lib().zr_commit_prove(C.byref(desc), _ptr(polys), batch, _ptr(pt), root, proof, cap,
                               C.byref(plen), ev, mod)
    if rc:
        raise ValueError(f"commit_prove failed ({rc})")
    return root.raw, proof.raw[: plen.value], ev.raw, mod.raw


def verify(desc: Desc, root: bytes, batch: int, point, eval_inner: bytes, proof: bytes) -> int:
    pt = point_array(point)
    return lib().zr_verify(C.byref(desc), _buf(root), batch, _ptr(pt), _buf(eval_inner),
                           _buf(proof), len(proof))


class Transcript:
    """``Blake3Transcript`` restated (transcript/src/lib.rs:12-77)."""

    def __init__(self):
        self._t = lib().zr_tr_new()

    def __del__(self):
        if getattr(self, "_t", None):
            lib().zr_tr_free(self._t)
            self._t = None

    def absorb(self, b: bytes):
        lib().zr_tr_absorb(self._t, _buf(b), len(b))

    def absorb_slice(self, b: bytes):
        lib().zr_tr_absorb_slice(self._t, _buf(b), len(b))

    def field_challenge(self, modulus: int, L: int) -> np.ndarray:
        """get_field_challenge: a Montgomery inner (L u64)."""
        out = np.zeros(L, np.uint64)
        lib().zr_tr_field_challenge(self._t, _ptr(_limbs(modulus, L)), L, _ptr(out))
        return out

    def absorb_field(self, modulus: int, L: int, inner) -> None:
        """absorb_random_field of a Montgomery inner (L u64)."""
        v = np.ascontiguousarray(inner, dtype=np.uint64)
        lib().zr_tr_absorb_field(self._t, _ptr(_limbs(modulus, L)), L, _ptr(v))

    def challenge(self, n: int) -> bytes:
        out = C.create_string_buffer(n)
        lib().zr_tr_challenge(self._t, out, n)
        return out.raw

    def get_prime(self, limbs: int = 4) -> int:
        out = np.zeros(limbs, np.uint64)
        lib().zr_tr_get_prime(self._t, limbs, _ptr(out))
        return sum(int(v) << (64 * i) for i, v in enumerate(out))


def is_probable_prime_base2(n: int, limbs: int = 4) -> bool:
    arr = np.array([(n >> (64 * i)) & ((1 << 64) - 1) for i in range(limbs)], np.uint64)
    return bool(lib().zr_is_probable_prime_base2(_ptr(arr), limbs))


# ------------------------------------------------------------------ sumcheck
def _limbs(x: int, L: int) -> np.ndarray:
    return np.array([(x >> (64 * i)) & ((1 << 64) - 1) for i in range(L)], np.uint64)


def _sc_groups(groups, L):
    """groups: list of (degree, mles (K, 2^n, L) uint64, [(coeff_inner, [idx...]), ...]
    [, [(a_inner, b_inner, mle index), ...] affine factors])."""
    keep, arr = [], (ScGroup * len(groups))()
    for g, grp in zip(arr, groups):
        deg, mles, prods = grp[:3]
        factors = grp[3] if len(grp) > 3 else []
        fm = np.array([int(x[2]) for x in factors] or [0], np.uint32)
        fa = np.array([_limbs(int(x[0]), L) for x in factors] or [[0] * L], np.uint64)
        fb = np.array([_limbs(int(x[1]), L) for x in factors] or [[0] * L], np.uint64)
        keep += [fm, fa, fb]
        g.n_factors = len(factors)
        g.factor_mles, g.factor_a, g.factor_b = fm.ctypes.data, fa.ctypes.data, fb.ctypes.data
        mles = np.ascontiguousarray(mles, dtype=np.uint64)
        coeffs = np.zeros((max(len(prods), 1), L), np.uint64)
        offsets = np.zeros(len(prods) + 1, np.uint32)
        idx = []
        for k, (c, ids) in enumerate(prods):
            coeffs[k] = _limbs(int(c), L)
            idx.extend(int(i) for i in ids)
            offsets[k + 1] = len(idx)
        indices = np.array(idx or [0], np.uint32)
        keep += [mles, coeffs, offsets, indices]
        g.degree, g.n_mles, g.n_products = deg, mles.shape[0], len(prods)
        g.mles, g.coeffs = mles.ctypes.data, coeffs.ctypes.data
        g.offsets, g.indices = offsets.ctypes.data, indices.ctypes.data
    return arr, keep


def sumcheck_prove(t: Transcript, modulus: int, L: int, nvars: int, groups, multi: bool):
    """MLSumcheck / MultiDegreeSumcheck prove_as_subprotocol restated; returns
    (proof bytes, point (nvars, L), finals (total MLEs, L))."""
    arr, keep = _sc_groups(groups, L)
    fb = 8 * L
    cap = fb + 8 + 4 * len(groups) + fb * len(groups) + sum(nvars * (fb * g[0] + 4) for g in groups)
    proof = C.create_string_buffer(cap)
    plen = C.c_size_t(0)
    point = np.zeros((nvars, L), np.uint64)
    nm = sum(np.asarray(g[1]).shape[0] for g in groups)
    finals = np.zeros((max(nm, 1), L), np.uint64)
    mod = _limbs(modulus, L)
    rc = lib().zr_sumcheck_prove(t._t, _ptr(mod), L, nvars, int(multi), arr, len(groups), proof,
                                 cap, C.byref(plen), _ptr(point), _ptr(finals))
    if rc != 0:
        raise ValueError(f"zr_sumcheck_prove failed ({rc})")
    return proof.raw[: plen.value], point, finals[:nm]


def sumcheck_verify(t: Transcript, modulus: int, L: int, nvars: int, degrees, proof: bytes,
                    multi: bool):
    """Returns (rc, point, expected evaluations per group); rc 0 = well formed."""
    deg = np.array(list(degrees), np.uint32)
    point = np.zeros((nvars, L), np.uint64)
    expected = np.zeros((len(deg), L), np.uint64)
    mod = _limbs(modulus, L)
    rc = lib().zr_sumcheck_verify(t._t, _ptr(mod), L, nvars, int(multi), _ptr(deg), len(deg),
                                  _buf(proof), len(proof), _ptr(point), _ptr(expected))
    return rc, point, expected


def sumcheck_comb(modulus: int, L: int, group, vals: np.ndarray) -> np.ndarray:
    arr, keep = _sc_groups([group], L)
    vals = np.ascontiguousarray(vals, dtype=np.uint64)
    out = np.zeros(L, np.uint64)
    mod = _limbs(modulus, L)
    lib().zr_sumcheck_comb(_ptr(mod), L, arr, _ptr(vals), _ptr(out))
    return out


def mle_evaluate(modulus: int, L: int, mle: np.ndarray, point: np.ndarray) -> np.ndarray:
    mle = np.ascontiguousarray(mle, dtype=np.uint64)
    point = np.ascontiguousarray(point, dtype=np.uint64)
    out = np.zeros(L, np.uint64)
    mod = _limbs(modulus, L)
    lib().zr_mle_evaluate(_ptr(mod), L, _ptr(mle), point.shape[0], _ptr(point), _ptr(out))
    return out


def _piop_cols(bin_cols, int_cols, nvars):
    n = 1 << nvars
    b = np.ascontiguousarray(bin_cols if bin_cols is not None else np.zeros((0, n)), dtype=np.uint64)
    i = np.ascontiguousarray(int_cols if int_cols is not None else np.zeros((0, n)), dtype=np.int64)
    assert b.ndim == 2 and i.ndim == 2 and (b.shape[0] == 0 or b.shape[1] == n) and (i.shape[0] == 0 or i.shape[1] == n)
    return b, i


def piop_eval_projection(modulus: int, L: int, bin_cols, D: int, int_cols, nvars: int, a) -> np.ndarray:
    """Zinc+ prover step 3 (evaluation projection): (n_bin + n_int, 2^nvars, L)
    Montgomery inners; a is the projecting element's Montgomery inner."""
    b, i = _piop_cols(bin_cols, int_cols, nvars)
    out = np.zeros((b.shape[0] + i.shape[0], 1 << nvars, L), np.uint64)
    av = np.ascontiguousarray(a, dtype=np.uint64)
    lib().zr_piop_eval_projection(_ptr(_limbs(modulus, L)), L, _ptr(b), b.shape[0], D, _ptr(i),
                                  i.shape[0], nvars, _ptr(av), _ptr(out))
    return out


def piop_lifted_evals(modulus: int, L: int, bin_cols, D: int, int_cols, nvars: int, point) -> np.ndarray:
    """Zinc+ prover step 6 (lifted evaluations): n_bin x D then n_int x 1
    Montgomery inners, shape (n_bin * D + n_int, L)."""
    b, i = _piop_cols(bin_cols, int_cols, nvars)
    out = np.zeros((b.shape[0] * D + i.shape[0], L), np.uint64)
    pt = np.ascontiguousarray(point, dtype=np.uint64)
    lib().zr_piop_lifted_evals(_ptr(_limbs(modulus, L)), L, _ptr(b), b.shape[0], D, _ptr(i),
                               i.shape[0], nvars, _ptr(pt), _ptr(out))
    return out


def piop_multipoint_eval(t: "Transcript", modulus: int, L: int, trace_mles: np.ndarray, point: np.ndarray,
                         shifts):
    """MultipointEval::prove_as_subprotocol (piop/src/multipoint_eval.rs:119-231)
    restated with Python integers around the oracle's MLSumcheck: n_shifts alphas
    then num_cols gammas from t, eq(., r'), next_c(r', .) = eq shifted up by c with
    zeros below (build_next_c_r_mle, poly/src/utils.rs:207-236), precombined =
    sum_j gamma_j v_j, and the degree-2 comb eq * precombined + sum_k alpha_k
    next_k * v_src_k.  Returns (proof bytes, r_0 (nvars, L) inners)."""
    p, R = modulus, 1 << (64 * L)
    Rinv = pow(R, -1, p)
    ncols, n, _ = trace_mles.shape
    nv = point.shape[0]

    def std(v):
        return sum(int(w) << (64 * i) for i, w in enumerate(v)) * Rinv % p

    def inner(x):
        y = x % p * R % p
        return [(y >> (64 * i)) & ((1 << 64) - 1) for i in range(L)]

    alphas = [t.field_challenge(p, L) for _ in shifts]
    gammas = [std(t.field_challenge(p, L)) for _ in range(ncols)]
    r = [std(v) for v in point]
    eq = []
    for b in range(n):
        e = 1
        for k in range(nv):
            e = e * (r[k] if (b >> k) & 1 else 1 - r[k]) % p
        eq.append(e)
    cols = [[std(trace_mles[j, b]) for b in range(n)] for j in range(ncols)]
    pre = [sum(g * cols[j][b] for j, g in enumerate(gammas)) % p for b in range(n)]
    S = len(shifts)
    mles = [eq] + [[0] * c + eq[: n - c] for _, c in shifts] + [pre] + [cols[sc] for sc, _ in shifts]
    arr = np.array([[inner(v) for v in m] for m in mles], np.uint64)
    prods = [(int(sum(int(w) << (64 * i) for i, w in enumerate(inner(1)))), [0, 1 + S])]
    for k in range(S):
        prods.append((int(sum(int(w) << (64 * i) for i, w in enumerate(alphas[k]))), [1 + k, 2 + S + k]))
    proof, pt, _fin = sumcheck_prove(t, p, L, nv, [(2, arr, prods)], False)
    return proof, pt


def piop_cpr_linear_prove(t: "Transcript", modulus: int, L: int, trace_mles: np.ndarray, point: np.ndarray,
                          shifts, coeffs):
    """CombinedPolyResolver prepare_sumcheck_group + MultiDegreeSumcheck +
    finalize_prover (piop/src/combined_poly_resolver.rs:71-247) for a linear
    homogeneous UAIR, restated with Python integers around the oracle's
    sumcheck.  coeffs: n_constraints x (num_cols + n_shifts) standard integers
    (mod p).  Returns (proof, point, evals (num_cols + n_shifts, L))."""
    p, R = modulus, 1 << (64 * L)
    Rinv = pow(R, -1, p)
    ncols, n, _ = trace_mles.shape
    nv, S = point.shape[0], len(shifts)

    def std(v):
        return sum(int(w) << (64 * i) for i, w in enumerate(v)) * Rinv % p

    def inner(x):
        y = x % p * R % p
        return [(y >> (64 * i)) & ((1 << 64) - 1) for i in range(L)]

    def as_int(v):
        return sum(int(w) << (64 * i) for i, w in enumerate(v))

    alpha = std(t.field_challenge(p, L))
    folded = [sum(pow(alpha, k, p) * int(row[j]) for k, row in enumerate(coeffs)) % p for j in range(ncols + S)]
    r = [std(v) for v in point]
    eq = []
    for b in range(n):
        e = 1
        for k in range(nv):
            e = e * (r[k] if (b >> k) & 1 else 1 - r[k]) % p
        eq.append(e)
    cols = [[std(trace_mles[j, b]) for b in range(n)] for j in range(ncols)]
    sel = [0] * (n - 1) + [1]
    down = [cols[sc][c:] + [0] * c for sc, c in shifts]
    mles = np.array([[inner(v) for v in m] for m in [sel, eq] + cols + down], np.uint64)
    prods = [(as_int(inner(folded[j])), [2 + j]) for j in range(ncols + S)]
    factors = [(0, as_int(inner(1)), 1), (as_int(inner(1)), as_int(inner(p - 1)), 0)]
    proof, pt, fin = sumcheck_prove(t, p, L, nv, [(3, mles, prods, factors)], True)
    evals = np.array(fin[2:], np.uint64)
    for e in evals:
        t.absorb_field(p, L, e)
    return proof, pt, evals


def piop_ideal_check_linear(t: "Transcript", modulus: int, L: int, bin_cols, D: int, int_cols, nvars: int,
                            shifts, coeffs):
    """IdealCheckProtocol::prove_linear (piop/src/ideal_check.rs:137-176) restated:
    nvars field challenges as the point, the up and shifted down columns evaluated
    coefficient-wise there with the last row read as zero (compute_lifted_evals on
    copies of the columns whose last entry is cleared), each constraint's
    coefficients (standard integers) applied, trimmed, absorbed.  Returns
    (point (nvars, L), [combined (len, L) per constraint])."""
    p, R = modulus, 1 << (64 * L)
    Rinv = pow(R, -1, p)
    n = 1 << nvars
    b, i = _piop_cols(bin_cols, int_cols, nvars)
    nb, ni = b.shape[0], i.shape[0]
    point = np.array([t.field_challenge(p, L) for _ in range(nvars)], np.uint64).reshape(nvars, L)

    def shifted(col, c):
        return np.concatenate([col[c:], np.zeros(c, col.dtype)])

    db = [shifted(b[sc], c) for sc, c in shifts if sc < nb]
    di = [shifted(i[sc - nb], c) for sc, c in shifts if sc >= nb]
    eb = np.stack(list(b) + db) if nb + len(db) else None
    ei = np.stack(list(i) + di) if ni + len(di) else None
    # evaluate_combined_polynomials (ideal_check/combined_poly_builder.rs:232-252)
    # reads zero on the last row of every up and down column
    if eb is not None:
        eb[:, -1] = 0
    if ei is not None:
        ei[:, -1] = 0
    vals = piop_lifted_evals(p, L, eb, D, ei, nvars, point)
    nb2 = nb + len(db)

    def std(v):
        return sum(int(w) << (64 * k) for k, w in enumerate(v)) * Rinv % p

    def value(j):  # polynomial value (D standard coefficients) of column j of [up, down]
        if j < nb:
            return [std(vals[j * D + l]) for l in range(D)]
        if j < nb + ni:
            return [std(vals[nb2 * D + j - nb])] + [0] * (D - 1)
        k = j - nb - ni
        sc = shifts[k][0]
        if sc < nb:
            q = [kk for kk in range(len(shifts)) if shifts[kk][0] < nb].index(k)
            return [std(vals[(nb + q) * D + l]) for l in range(D)]
        q = [kk for kk in range(len(shifts)) if shifts[kk][0] >= nb].index(k)
        return [std(vals[nb2 * D + ni + q])] + [0] * (D - 1)

    cols = [value(j) for j in range(nb + ni + len(shifts))]
    out = []
    for row in coeffs:
        comb = [sum(int(cf) * cols[j][l] for j, cf in enumerate(row)) % p for l in range(D)]
        while comb and comb[-1] == 0:
            comb.pop()
        arr = np.array([[((x * R % p) >> (64 * w)) & ((1 << 64) - 1) for w in range(L)] for x in comb],
                       np.uint64).reshape(len(comb), L)
        for e in arr:
            t.absorb_field(p, L, e)
        out.append(arr)
    return point, out


def commit_prove_f(desc: Desc, polys: np.ndarray, batch: int, point_u256):
    """commit + prove_f with the point given as non-negative integers (< 2^256),
    mapped into the field once the prime is drawn.  Returns (root, proof, eval
    inner bytes, modulus bytes)."""
    polys = np.ascontiguousarray(polys)
    pt = np.array([[(int(v) >> (64 * w)) & ((1 << 64) - 1) for w in range(4)] for v in point_u256], np.uint64)
    cap = proof_size(desc, batch) + 64
    proof = C.create_string_buffer(cap)
    plen = C.c_size_t(0)
    root = C.create_string_buffer(32)
    ev = C.create_string_buffer(8 * desc.field_limbs)
    mod = C.create_string_buffer(8 * desc.field_limbs)
    rc = lib().zr_commit_prove_f(C.byref(desc), _ptr(polys), batch, _ptr(pt), root, proof, cap, C.byref(plen), ev,
                                 mod)
    if rc:
        raise ValueError(f"commit_prove_f failed ({rc})")
    return root.raw, proof.raw[: plen.value], ev.raw, mod.raw


def prove_f_on(desc: Desc, polys: np.ndarray, batch: int, t: "Transcript", modulus: int, point_f) -> tuple[bytes, bytes]:
    """ZipPlus::prove_f on a transcript already in use, at a point of field
    elements (Montgomery inners, (num_vars, L)) of the prime `modulus`.
    Returns (proof bytes, eval inner bytes)."""
    polys = np.ascontiguousarray(polys)
    L = desc.field_limbs
    pt = np.ascontiguousarray(point_f, dtype=np.uint64)
    cap = proof_size(desc, batch) + 64
    proof = C.create_string_buffer(cap)
    plen = C.c_size_t(0)
    ev = C.create_string_buffer(8 * L)
    rc = lib().zr_prove_f_on(C.byref(desc), _ptr(polys), batch, t._t, _ptr(_limbs(modulus, L)), _ptr(pt), proof,
                             cap, C.byref(plen), ev)
    if rc:
        raise ValueError(f"prove_f failed ({rc})")
    return proof.raw[: plen.value], ev.raw


def _trim(rows: np.ndarray) -> np.ndarray:
    n = rows.shape[0]
    while n and not rows[n - 1].any():
        n -= 1
    return rows[:n]


def _poly_vec_bytes(polys, modulus: int, L: int) -> bytes:
    """DynamicPolyVecF transcription (poly/src/univariate/dynamic/over_field.rs:
    409-476) of trimmed (len, L) inner arrays."""
    if not polys:
        return b""
    any_ = any(q.shape[0] for q in polys)
    out = bytes([1 if any_ else 0]) + (_limbs(modulus, L).tobytes() if any_ else b"")
    for q in polys:
        out += int(q.shape[0]).to_bytes(4, "little") + np.ascontiguousarray(q, np.uint64).tobytes()
    return out


def _sub(b: bytes) -> bytes:
    return len(b).to_bytes(4, "little") + b


def zinc_prove_mle_first(desc_bin: Desc, desc_int: Desc, nvars: int, bin_cols, D: int, int_cols, shifts, coeffs,
                         L: int, n_pub_bin: int = 0, n_pub_int: int = 0) -> bytes:
    """ZincPlusPiop::prove::<MLE_FIRST = true> (protocol/src/prover.rs:677-706)
    for a linear UAIR over binary-polynomial and i64 witness columns, chaining
    the oracle's steps on one transcript: step 0 commitments (prover.rs:218-267;
    the empty arbitrary table has the default root), step 1 prime, step 2
    ideal check, step 3 the Chal (i128) projecting element and evaluation
    projection, step 4 CPR, step 5 multipoint, step 6 lifted evaluations
    (trimmed, each coefficient absorbed), step 7 prove_f per table, and the
    Proof transcription (protocol/src/lib.rs:129-160).  coeffs: integer
    constraint coefficients over [binary up, integer up, down].  The first
    n_pub_bin / n_pub_int columns of each table are public (UairTrace::public,
    uair/src/lib.rs:328-346): not committed or opened, their entries absorbed
    as 8 LE bytes each after the roots (absorb_public_columns, lib.rs:305-320),
    their lifted evaluations left out of the proof (prover.rs:614-632)."""
    b, i = _piop_cols(bin_cols, int_cols, nvars)
    nb, ni = b.shape[0], i.shape[0]
    wb, wi = nb - n_pub_bin, ni - n_pub_int
    roots = [b"\0" * 32, b"\0" * 32, b"\0" * 32]
    if wb:
        roots[0] = commit(desc_bin, b[n_pub_bin:], wb)
    if wi:
        roots[2] = commit(desc_int, i[n_pub_int:], wi)
    t = Transcript()
    for r in roots:
        t.absorb_slice(r)
    for col in list(b[:n_pub_bin]) + list(i[:n_pub_int]):
        for e in np.ascontiguousarray(col).view(np.uint8).reshape(-1, 8):
            t.absorb_slice(e.tobytes())
    p = t.get_prime(L)
    R = 1 << (64 * L)
    cf = [[int(c) % p for c in row] for row in coeffs]
    ic_point, combined = piop_ideal_check_linear(t, p, L, b if nb else None, D, i if ni else None, nvars, shifts, cf)
    a = int.from_bytes(t.challenge(16), "little", signed=True) % p * R % p
    mles = piop_eval_projection(p, L, b if nb else None, D, i if ni else None, nvars, _limbs(a, L))
    md, cpr_pt, evals = piop_cpr_linear_prove(t, p, L, mles, ic_point, shifts, cf)
    mp, r0 = piop_multipoint_eval(t, p, L, mles, cpr_pt, shifts)
    lifted = piop_lifted_evals(p, L, b if nb else None, D, i if ni else None, nvars, r0)
    polys = [_trim(lifted[c * D:(c + 1) * D]) for c in range(nb)] + \
        [_trim(lifted[nb * D + c:nb * D + c + 1]) for c in range(ni)]
    for q in polys:
        for e in q:
            t.absorb_field(p, L, e)
    zip_ = b""
    if wb:
        zip_ += prove_f_on(desc_bin, b[n_pub_bin:], wb, t, p, r0)[0]
    if wi:
        zip_ += prove_f_on(desc_int, i[n_pub_int:], wi, t, p, r0)[0]
    S = len(shifts)
    vec = lambda rows: (_limbs(p, L).tobytes() + np.ascontiguousarray(rows, np.uint64).tobytes()) if len(rows) else b""
    out = roots[0] + int(wb).to_bytes(8, "little") + roots[1] + bytes(8) + roots[2] + int(wi).to_bytes(8, "little")
    out += _sub(zip_)
    out += _sub(_poly_vec_bytes(list(combined), p, L))
    out += _sub(_sub(vec(evals[:nb + ni])) + _sub(vec(evals[nb + ni:nb + ni + S])))
    out += _sub(md) + _sub(mp)
    out += _sub(_poly_vec_bytes(polys[n_pub_bin:nb] + polys[nb + n_pub_int:], p, L))
    return out
