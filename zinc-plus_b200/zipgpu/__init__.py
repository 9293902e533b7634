"""Python front end of libzipgpu, the B200 (sm_100a) backend of the Zip+
polynomial commitment scheme of NethermindEth/zinc-plus.

The classes mirror the reference's Rust API for the commit/prove path, with
the same names and argument meaning:

  ``IprsCode.new`` / ``IprsCode.new_with_optimal_depth``  (zip-plus/src/code/iprs.rs:30-51)
  ``RaaCode.new``                                          (zip-plus/src/code/raa.rs:38-90)
  ``ZipPlus.setup`` / ``commit`` / ``commit_single`` / ``encode_rows``
                                                           (pcs/structs.rs:74, pcs/phase_commit.rs)
  ``ZipPlus.prove`` / ``ZipPlus.verify``                   (pcs/phase_prove.rs:85, pcs/phase_verify.rs:100)
  ``PcsProverTranscript.new_from_commitment(s)``           (zip-plus/src/pcs_transcript.rs:58-73)
  ``MerkleTree.new(rows).root()``                          (zip-plus/src/merkle.rs:74-103)

Every call goes through the C ABI declared in include/zipgpu.h.  There is no
CPU fallback: a missing or unloadable library raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzipgpu.so")

ZG_OK = 0
STATUS = {
    0: "ZG_OK", 1: "ZG_ERR_INVALID_PARAM", 2: "ZG_ERR_INVALID_OPEN", 3: "ZG_ERR_SERIALIZATION",
    4: "ZG_ERR_OVERFLOW", 5: "ZG_ERR_CUDA", 6: "ZG_ERR_OOM", 7: "ZG_ERR_TIMEOUT",
    8: "ZG_ERR_NO_DEVICE", 9: "ZG_ERR_BUFFER_TOO_SMALL",
}
EVAL_I32, EVAL_BINPOLY, EVAL_I64 = 0, 1, 2
CODE_IPRS, CODE_RAA, CODE_RAA_SIGN_FLIP = 0, 1, 2

# Every symbol include/zipgpu.h declares.
EXPORTS = (
    "zg_last_error", "zg_version", "zg_ctx_create", "zg_ctx_destroy", "zg_ctx_kernel_launches",
    "zg_ctx_stream", "zg_ctx_set_kernel_timing", "zg_ctx_kernel_timing_report", "zg_params_create", "zg_params_destroy", "zg_params_get_info",
    "zg_params_iprs_tables", "zg_params_raa_perms", "zg_encode_rows", "zg_encode_rows_d",
    "zg_encode_wide", "zg_merkle_root", "zg_merkle_root_noalloc_d", "zg_commit", "zg_commit_d", "zg_hint_free",
    "zg_hint_batch", "zg_hint_codeword", "zg_transcript_new", "zg_transcript_free",
    "zg_transcript_absorb", "zg_transcript_absorb_slice", "zg_transcript_challenge",
    "zg_transcript_sample_field", "zg_transcript_proof", "zg_prove", "zg_prove_d",
    "zg_commit_prove", "zg_commit_prove_d", "zg_commit_prove_many", "zg_proof_size", "zg_verify",
    "zg_sumcheck_prove", "zg_mle_evaluate", "zg_commit_batch", "zg_server_create",
    "zg_server_submit", "zg_server_wait", "zg_server_get_stats", "zg_server_destroy",
    "zg_selftest_bounded_wait", "zg_piop_eval_projection", "zg_piop_lifted_evals", "zg_piop_multipoint_eval",
    "zg_piop_cpr_linear_prove", "zg_piop_ideal_check_linear", "zg_prove_f", "zg_prove_f_d",
    "zg_zinc_prove_mle_first", "zg_zinc_prove", "zg_encode_f", "zg_encode_f_d", "zg_proof_read", "zg_debug_fail_allocation", "zg_is_probable_prime_base2",
)


class ZipError(RuntimeError):
    """Error status from libzipgpu (mirrors zip_plus::ZipError)."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class ParamsDesc(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "eval_kind", "degree_plus_one", "code_kind", "rep", "num_vars", "row_len",
        "iprs_depth", "comb_limbs", "field_limbs", "num_openings")]


class ParamsInfo(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "num_rows", "row_len", "codeword_len", "depth", "base_len", "base_dim",
        "eval_bytes", "cw_bytes", "comb_bytes", "field_bytes")]


class BatchOpts(C.Structure):
    """Mirror of ``zg_batch_opts``."""

    _fields_ = [("lanes", C.c_uint32), ("use_graph", C.c_int), ("autotune", C.c_int),
                ("base_variant", C.c_int), ("leaf_variant", C.c_int)]

    @staticmethod
    def make(lanes=4, use_graph=True, autotune=True, base_variant=-1, leaf_variant=-1):
        return BatchOpts(lanes, int(use_graph), int(autotune), base_variant, leaf_variant)


class ServerOpts(C.Structure):
    """Mirror of ``zg_server_opts``."""

    _fields_ = [("workers", C.c_uint32), ("hbm_budget", C.c_uint64), ("max_group", C.c_uint32),
                ("max_skip_ms", C.c_uint32), ("group_max_bytes", C.c_uint64)]


class ServerResult(C.Structure):
    _fields_ = [("status", C.c_int), ("proof_len", C.c_size_t), ("latency_ms", C.c_double),
                ("queue_ms", C.c_double), ("group_size", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("completed", "queued", "in_flight", "groups",
                                          "grouped_requests", "budget", "reserved",
                                          "peak_reserved")] + \
               [(n, C.c_double) for n in ("ms_input", "ms_commit", "ms_prime", "ms_prove")]


class LinearUairDesc(C.Structure):
    """Mirror of ``zg_linear_uair``."""

    _fields_ = [("n_bin", C.c_uint32), ("n_int", C.c_uint32), ("degree_plus_one", C.c_uint32),
                ("n_shifts", C.c_uint32), ("shift_src", C.c_void_p), ("shift_amount", C.c_void_p),
                ("n_constraints", C.c_uint32), ("coeffs", C.c_void_p), ("n_pub_bin", C.c_uint32),
                ("n_pub_int", C.c_uint32)]


class UairDesc(C.Structure):
    """Mirror of ``zg_uair`` (constraints as terms)."""

    _fields_ = [("n_bin", C.c_uint32), ("n_int", C.c_uint32), ("degree_plus_one", C.c_uint32),
                ("n_shifts", C.c_uint32), ("shift_src", C.c_void_p), ("shift_amount", C.c_void_p),
                ("n_constraints", C.c_uint32), ("term_offsets", C.c_void_p), ("term_coeffs", C.c_void_p),
                ("factor_offsets", C.c_void_p), ("factor_cols", C.c_void_p), ("zero_ideal", C.c_void_p),
                ("n_pub_bin", C.c_uint32), ("n_pub_int", C.c_uint32)]


class ProofLayout(C.Structure):
    """Mirror of ``zg_proof_layout``."""

    _fields_ = [("roots", (C.c_uint8 * 32) * 3), ("batch_sizes", C.c_uint64 * 3), ("modulus", C.c_uint8 * 32)] + \
               [(n, C.c_size_t) for n in ("zip_offset", "zip_len", "ideal_check_offset", "ideal_check_len",
                                          "resolver_offset", "resolver_len", "multi_degree_offset",
                                          "multi_degree_len", "multipoint_offset", "multipoint_len",
                                          "lifted_offset", "lifted_len")] + \
               [(n, C.c_uint32) for n in ("n_ideal_values", "n_up_evals", "n_down_evals", "multi_degree_groups",
                                          "cpr_degree", "n_lifted")]


class SumcheckGroupDesc(C.Structure):
    """Mirror of ``zg_sumcheck_group``."""

    _fields_ = [("degree", C.c_uint32), ("n_mles", C.c_uint32), ("n_products", C.c_uint32),
                ("mles", C.c_void_p), ("coeffs", C.c_void_p), ("offsets", C.c_void_p),
                ("indices", C.c_void_p), ("n_factors", C.c_uint32), ("factor_mles", C.c_void_p),
                ("factor_a", C.c_void_p), ("factor_b", C.c_void_p)]


_lib = None


def lib() -> C.CDLL:
    """Loads libzipgpu.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libzipgpu.so not built at {LIB_PATH}; run `make -C zinc-plus_b200`")
    L = C.CDLL(LIB_PATH)
    vp, sz, u32, st = C.c_void_p, C.c_size_t, C.c_uint32, C.c_int
    sig = {
        "zg_last_error": ([], C.c_char_p), "zg_version": ([], C.c_char_p),
        "zg_ctx_create": ([C.c_int, C.POINTER(vp)], st), "zg_ctx_destroy": ([vp], st),
        "zg_ctx_kernel_launches": ([vp], C.c_uint64), "zg_ctx_stream": ([vp], vp),
        "zg_ctx_set_kernel_timing": ([vp, C.c_int], st),
        "zg_ctx_kernel_timing_report": ([vp, C.c_char_p, sz, C.POINTER(sz)], st),
        "zg_selftest_bounded_wait": ([vp, C.POINTER(C.c_uint32)], st),
        "zg_prove_f": ([vp, vp, vp, C.c_uint32, vp, vp, vp], st),
        "zg_prove_f_d": ([vp, vp, vp, C.c_uint32, vp, vp, vp], st),
        "zg_piop_eval_projection": ([vp, C.c_char_p, C.c_uint32, vp, C.c_uint32, C.c_uint32, vp,
                                     C.c_uint32, C.c_uint32, vp, C.c_int, vp], st),
        "zg_piop_lifted_evals": ([vp, C.c_char_p, C.c_uint32, vp, C.c_uint32, C.c_uint32, vp,
                                  C.c_uint32, C.c_uint32, vp, C.c_int, vp], st),
        "zg_piop_multipoint_eval": ([vp, vp, C.c_char_p, C.c_uint32, vp, C.c_uint32, C.c_uint32, vp, vp, vp,
                                     C.c_uint32, C.c_int, vp, C.POINTER(sz), vp], st),
        "zg_piop_cpr_linear_prove": ([vp, vp, C.c_char_p, C.c_uint32, vp, C.c_uint32, C.c_uint32, vp, vp, vp,
                                      C.c_uint32, C.c_uint32, vp, C.c_int, vp, C.POINTER(sz), vp, vp], st),
        "zg_zinc_prove_mle_first": ([vp, vp, C.POINTER(LinearUairDesc), C.c_uint32, vp, vp, C.c_int, vp,
                                     C.POINTER(sz)], st),
        "zg_debug_fail_allocation": ([C.c_uint32], st),
        "zg_is_probable_prime_base2": ([vp, C.c_uint32, C.c_uint32, vp], st),
        "zg_proof_read": ([C.c_char_p, sz, C.c_uint32, C.c_uint32, C.POINTER(ProofLayout)], st),
        "zg_encode_f": ([vp, C.c_char_p, C.c_uint32, vp, vp], st),
        "zg_encode_f_d": ([vp, C.c_char_p, C.c_uint32, vp, vp, vp], st),
        "zg_zinc_prove": ([vp, vp, C.POINTER(UairDesc), C.c_uint32, vp, vp, C.c_int, C.c_int, vp, C.POINTER(sz)],
                          st),
        "zg_piop_ideal_check_linear": ([vp, vp, C.c_char_p, C.c_uint32, vp, C.c_uint32, C.c_uint32, vp,
                                        C.c_uint32, C.c_uint32, vp, vp, C.c_uint32, C.c_uint32, vp, C.c_int, vp,
                                        vp, vp], st),
        "zg_params_create": ([vp, C.POINTER(ParamsDesc), C.POINTER(vp)], st),
        "zg_params_destroy": ([vp], st),
        "zg_params_get_info": ([vp, C.POINTER(ParamsInfo)], st),
        "zg_params_iprs_tables": ([vp, vp, vp], st), "zg_params_raa_perms": ([vp, vp, vp], st),
        "zg_encode_rows": ([vp, vp, vp], st), "zg_encode_rows_d": ([vp, vp, vp, vp], st),
        "zg_encode_wide": ([vp, vp, u32, vp], st),
        "zg_merkle_root": ([vp, vp, u32, u32, u32, vp], st),
        "zg_merkle_root_noalloc_d": ([vp, u32, u32, vp, vp], st),
        "zg_commit": ([vp, vp, u32, C.POINTER(vp), vp], st),
        "zg_commit_d": ([vp, vp, u32, C.POINTER(vp), vp], st),
        "zg_hint_free": ([vp], st), "zg_hint_batch": ([vp], u32),
        "zg_hint_codeword": ([vp, u32, vp], st),
        "zg_transcript_new": ([vp, u32, C.POINTER(vp)], st), "zg_transcript_free": ([vp], st),
        "zg_transcript_absorb": ([vp, vp, sz], st), "zg_transcript_absorb_slice": ([vp, vp, sz], st),
        "zg_transcript_challenge": ([vp, vp, sz], st),
        "zg_transcript_sample_field": ([vp, u32, vp], st),
        "zg_transcript_proof": ([vp, C.POINTER(vp), C.POINTER(sz)], st),
        "zg_prove": ([vp, vp, vp, u32, vp, vp, vp], st),
        "zg_prove_d": ([vp, vp, vp, u32, vp, vp, vp], st),
        "zg_commit_prove": ([vp, vp, u32, vp, vp, vp, vp, C.POINTER(sz)], st),
        "zg_commit_prove_d": ([vp, vp, u32, vp, vp, vp, vp, C.POINTER(sz)], st),
        "zg_commit_prove_many": ([vp, u32, vp, C.c_int, vp, vp, vp, vp, vp, u32, vp], st),
        "zg_proof_size": ([vp, u32], sz),
        "zg_verify": ([vp, vp, u32, vp, vp, vp, sz], st),
        "zg_sumcheck_prove": ([vp, vp, vp, u32, u32, C.c_int, C.POINTER(SumcheckGroupDesc), u32,
                               C.c_int, vp, C.POINTER(sz), vp, vp], st),
        "zg_mle_evaluate": ([vp, vp, u32, vp, u32, vp, vp], st),
        "zg_commit_batch": ([vp, u32, vp, vp, C.c_int, C.POINTER(BatchOpts), vp, vp], st),
        "zg_server_create": ([vp, C.POINTER(ServerOpts), C.POINTER(vp)], st),
        "zg_server_submit": ([vp, vp, vp, vp, vp, vp, vp, sz, C.POINTER(C.c_uint64)], st),
        "zg_server_wait": ([vp, C.c_uint64, C.c_int, C.POINTER(ServerResult)], st),
        "zg_server_get_stats": ([vp, C.POINTER(ServerStats)], st),
        "zg_server_destroy": ([vp], st),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(status: int) -> None:
    if status != ZG_OK:
        raise ZipError(status, lib().zg_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def i128_bytes(values: Sequence[int]) -> bytes:
    return b"".join((int(v) & ((1 << 128) - 1)).to_bytes(16, "little") for v in values)


# --------------------------------------------------------------------- context
class Context:
    """A CUDA device context (stream and scratch arenas)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().zg_ctx_create(device, C.byref(h)))
        self.handle = h

    @property
    def kernel_launches(self) -> int:
        return int(lib().zg_ctx_kernel_launches(self.handle))

    @property
    def stream(self) -> int:
        return int(lib().zg_ctx_stream(self.handle) or 0)

    def set_kernel_timing(self, enable: bool) -> None:
        check(lib().zg_ctx_set_kernel_timing(self.handle, int(enable)))

    def kernel_times(self) -> dict:
        """{kernel: (launches, total_ms)} since the last report (CUDA events)."""
        n = C.c_size_t()
        buf = C.create_string_buffer(1 << 16)
        check(lib().zg_ctx_kernel_timing_report(self.handle, buf, 1 << 16, C.byref(n)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, cnt, ms = line.rsplit(",", 2)
            out[name] = (int(cnt), float(ms))
        return out

    def selftest_bounded_wait(self) -> int:
        """Runs a probe kernel whose bounded wait must run out (about a second)
        and returns the device status code it reported (4), clearing it."""
        v = C.c_uint32()
        check(lib().zg_selftest_bounded_wait(self.handle, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "handle", None):
            lib().zg_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


# ---------------------------------------------------------------------- codes
@dataclass(frozen=True)
class IprsCode:
    """IPRS code over F65537 (IprsCode<Zt, PnttConfigF65537, REP, CHECK>)."""

    row_len: int
    depth: int = 0  # 0: new_with_optimal_depth
    rep: int = 4
    kind: int = CODE_IPRS

    @staticmethod
    def new(row_len: int, depth: int, rep: int = 4) -> "IprsCode":
        return IprsCode(row_len, depth, rep)

    @staticmethod
    def new_with_optimal_depth(row_len: int, rep: int = 4) -> "IprsCode":
        return IprsCode(row_len, 0, rep)


@dataclass(frozen=True)
class RaaCode:
    """Repeat-accumulate-accumulate code (RaaCode<Zt, Config, REP>)."""

    row_len: int
    rep: int = 4
    depth: int = 0
    kind: int = CODE_RAA

    @staticmethod
    def new(row_len: int, rep: int = 4) -> "RaaCode":
        return RaaCode(row_len, rep)


@dataclass(frozen=True)
class RaaSignFlippingCode:
    """RAA with sign flips (RaaSignFlippingCode<Zt, Config, REP>,
    raa_sign_flip.rs:14-69)."""

    row_len: int
    rep: int = 4
    depth: int = 0
    kind: int = CODE_RAA_SIGN_FLIP

    @staticmethod
    def new(row_len: int, rep: int = 4) -> "RaaSignFlippingCode":
        return RaaSignFlippingCode(row_len, rep)


@dataclass(frozen=True)
class ZipTypes:
    """The ZipTypes instantiation (pcs/structs.rs:15-60)."""

    eval_kind: int = EVAL_BINPOLY
    degree_plus_one: int = 32
    comb_limbs: int = 5
    field_limbs: int = 4
    num_openings: int = 147


# The reference benches' instantiations.
ZIP_I32 = ZipTypes(EVAL_I32, 1, 3, 4, 147)  # zip_benches.rs:25-40


def zip_plus_binary(degree_plus_one: int) -> ZipTypes:  # zip_plus_benches.rs:37-65
    return ZipTypes(EVAL_BINPOLY, degree_plus_one, 5, 4, 147)


class ZipPlusParams:
    """ZipPlusParams (setup output) backed by device-resident code tables."""

    def __init__(self, zt: ZipTypes, code, num_vars: int, ctx: Context | None):
        self.zt, self.code, self.num_vars, self.ctx = zt, code, num_vars, ctx
        d = ParamsDesc(zt.eval_kind, zt.degree_plus_one, code.kind, code.rep, num_vars,
                       code.row_len, code.depth, zt.comb_limbs, zt.field_limbs, zt.num_openings)
        self.desc = d
        h = C.c_void_p()
        check(lib().zg_params_create(ctx.handle if ctx else None, C.byref(d), C.byref(h)))
        self.handle = h
        info = ParamsInfo()
        check(lib().zg_params_get_info(h, C.byref(info)))
        self.info = info
        self.num_rows = info.num_rows
        self.row_len = info.row_len
        self.codeword_len = info.codeword_len

    @property
    def eval_dtype(self):
        return {EVAL_I32: np.int32, EVAL_I64: np.int64}.get(self.zt.eval_kind, np.uint64)

    def proof_size(self, batch: int = 1) -> int:
        return int(lib().zg_proof_size(self.handle, batch))

    def iprs_tables(self):
        i = self.info
        bm = np.zeros((i.base_dim, i.base_len), np.int64)
        ntw = sum(i.base_dim * 8 ** k * 56 for k in range(i.depth))
        tw = np.zeros(max(ntw, 1), np.int64)
        check(lib().zg_params_iprs_tables(self.handle, _ptr(bm), _ptr(tw)))
        return bm, tw[:ntw]

    def raa_perms(self):
        p1 = np.zeros(self.codeword_len, np.uint32)
        p2 = np.zeros(self.codeword_len, np.uint32)
        check(lib().zg_params_raa_perms(self.handle, _ptr(p1), _ptr(p2)))
        return p1, p2

    def close(self):
        if getattr(self, "handle", None):
            lib().zg_params_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ZipPlusCommitment:
    root: bytes
    batch_size: int

    def to_bytes(self) -> bytes:  # pcs/structs.rs:140-157
        return self.root + int(self.batch_size).to_bytes(8, "little")


class ZipPlusHint:
    """Device-resident codewords and Merkle layers (ZipPlusHint)."""

    def __init__(self, handle, params: ZipPlusParams):
        self.handle, self.params = handle, params

    @property
    def batch(self) -> int:
        return int(lib().zg_hint_batch(self.handle))

    def codeword(self, poly: int = 0) -> np.ndarray:
        p = self.params
        out = np.zeros(p.num_rows * p.codeword_len * p.info.cw_bytes, np.uint8)
        check(lib().zg_hint_codeword(self.handle, poly, _ptr(out)))
        return out.reshape(p.num_rows, p.codeword_len, p.info.cw_bytes)

    def close(self):
        if getattr(self, "handle", None):
            lib().zg_hint_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PcsProverTranscript:
    """PcsProverTranscript: Blake3 Fiat-Shamir sponge plus the proof stream."""

    def __init__(self, roots: Sequence[bytes] = ()):
        h = C.c_void_p()
        buf = b"".join(roots)
        check(lib().zg_transcript_new(C.c_char_p(buf) if buf else None, len(roots), C.byref(h)))
        self.handle = h
        self.modulus: int | None = None

    @staticmethod
    def new_from_commitment(comm: ZipPlusCommitment) -> "PcsProverTranscript":
        return PcsProverTranscript([comm.root])

    @staticmethod
    def new_from_commitments(comms: Sequence[ZipPlusCommitment]) -> "PcsProverTranscript":
        return PcsProverTranscript([c.root for c in comms])

    def absorb(self, b: bytes):
        check(lib().zg_transcript_absorb(self.handle, C.c_char_p(b), len(b)))

    def absorb_slice(self, b: bytes):
        check(lib().zg_transcript_absorb_slice(self.handle, C.c_char_p(b), len(b)))

    def get_challenge(self, nbytes: int) -> bytes:
        out = C.create_string_buffer(nbytes)
        check(lib().zg_transcript_challenge(self.handle, out, nbytes))
        return out.raw

    def get_random_field_cfg(self, limbs: int = 4) -> int:
        out = C.create_string_buffer(8 * limbs)
        check(lib().zg_transcript_sample_field(self.handle, limbs, out))
        self.modulus = int.from_bytes(out.raw, "little")
        return self.modulus

    @property
    def stream(self) -> bytes:
        data, n = C.c_void_p(), C.c_size_t()
        check(lib().zg_transcript_proof(self.handle, C.byref(data), C.byref(n)))
        return C.string_at(data, n.value) if n.value else b""

    def close(self):
        if getattr(self, "handle", None):
            lib().zg_transcript_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _poly_ptrs(params: ZipPlusParams, polys):
    arrs = [np.ascontiguousarray(p, dtype=params.eval_dtype) for p in polys]
    n = params.num_rows * params.row_len
    for a in arrs:
        if a.size != n:
            raise ValueError(f"Polynomial has an incorrect number of evaluations ({a.size}) for "
                             f"the expected matrix size ({n})")
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    return arrs, ptrs


class ZipPlus:
    """ZipPlus<Zt, Lc> associated functions."""

    @staticmethod
    def setup(poly_size: int, code, zt: ZipTypes = ZipTypes(), ctx: Context | None = None,
              device: bool = True) -> ZipPlusParams:
        if poly_size <= 0 or poly_size & (poly_size - 1):
            raise ValueError("poly_size must be a power of two")
        num_vars = poly_size.bit_length() - 1
        if device and ctx is None:
            ctx = default_context()
        return ZipPlusParams(zt, code, num_vars, ctx if device else None)

    @staticmethod
    def encode_rows(pp: ZipPlusParams, evals) -> np.ndarray:
        ev = np.ascontiguousarray(evals, dtype=pp.eval_dtype)
        out = np.zeros(pp.num_rows * pp.codeword_len * pp.info.cw_bytes, np.uint8)
        check(lib().zg_encode_rows(pp.handle, _ptr(ev), _ptr(out)))
        return out.reshape(pp.num_rows, pp.codeword_len, pp.info.cw_bytes)

    @staticmethod
    def encode_wide(pp: ZipPlusParams, row: np.ndarray, limbs: int) -> np.ndarray:
        row = np.ascontiguousarray(row, dtype=np.uint64)
        out = np.zeros((pp.codeword_len, limbs), np.uint64)
        check(lib().zg_encode_wide(pp.handle, _ptr(row), limbs, _ptr(out)))
        return out

    @staticmethod
    def encode_f(pp: ZipPlusParams, modulus: int, limbs: int, row: np.ndarray) -> np.ndarray:
        """LinearCode::encode_f of (row_len, limbs) Montgomery inners over the
        prime `modulus`: (codeword_len, limbs), on the GPU."""
        row = np.ascontiguousarray(row, dtype=np.uint64)
        if row.shape != (pp.info.row_len, limbs):
            raise ValueError("row must be (row_len, limbs) Montgomery inners")
        out = np.zeros((pp.codeword_len, limbs), np.uint64)
        check(lib().zg_encode_f(pp.handle, modulus.to_bytes(8 * limbs, "little"), limbs, _ptr(row), _ptr(out)))
        return out

    @staticmethod
    def commit(pp: ZipPlusParams, polys) -> tuple[ZipPlusHint, ZipPlusCommitment]:
        if len(polys) == 0:
            raise ValueError("Batch must contain at least one polynomial")
        _keep, ptrs = _poly_ptrs(pp, polys)
        h = C.c_void_p()
        root = C.create_string_buffer(32)
        check(lib().zg_commit(pp.handle, ptrs, len(polys), C.byref(h), root))
        return ZipPlusHint(h, pp), ZipPlusCommitment(root.raw, len(polys))

    @staticmethod
    def commit_single(pp: ZipPlusParams, poly) -> tuple[ZipPlusHint, ZipPlusCommitment]:
        return ZipPlus.commit(pp, [poly])

    @staticmethod
    def commit_batch(pps: Sequence[ZipPlusParams], polys, ctx: Context | None = None,
                     opts: BatchOpts | None = None, hints: bool = False, on_device: bool = False):
        """commit_single of every polys[i] under pps[i] in one batched call
        (zg_commit_batch).  Returns the commitments, plus the hints when asked.
        With on_device, polys are device addresses (ints)."""
        n = len(polys)
        if n == 0 or len(pps) != n:
            raise ValueError("need one parameter set per polynomial")
        ctx = ctx or pps[0].ctx or default_context()
        if on_device:
            keep, ptrs = None, (C.c_void_p * n)(*[int(a) for a in polys])
        else:
            keep = []
            for pp, poly in zip(pps, polys):
                keep += _poly_ptrs(pp, [poly])[0]
            ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in keep])
        hs = (C.c_void_p * n)() if hints else None
        roots = C.create_string_buffer(32 * n)
        prm = (C.c_void_p * n)(*[pp.handle.value for pp in pps])
        check(lib().zg_commit_batch(ctx.handle, n, prm, ptrs, int(on_device),
                                    C.byref(opts) if opts is not None else None, roots, hs))
        comms = [ZipPlusCommitment(roots.raw[32 * i:32 * i + 32], 1) for i in range(n)]
        if hints:
            return comms, [ZipPlusHint(C.c_void_p(hs[i]), pps[i]) for i in range(n)]
        return comms

    @staticmethod
    def prove(transcript: PcsProverTranscript, pp: ZipPlusParams, polys, point: Sequence[int],
              hint: ZipPlusHint) -> bytes:
        """Returns the evaluation as its Montgomery inner bytes; appends the proof."""
        _keep, ptrs = _poly_ptrs(pp, polys)
        if len(point) != pp.num_vars:
            raise ZipError(1, f"Invalid point (expect point to have {pp.num_vars} variates but "
                              f"got {len(point)})")
        pt = i128_bytes(point)
        ev = C.create_string_buffer(8 * pp.zt.field_limbs)
        check(lib().zg_prove(pp.handle, transcript.handle, ptrs, len(polys), C.c_char_p(pt),
                             hint.handle, ev))
        return ev.raw

    @staticmethod
    def prove_f(transcript: PcsProverTranscript, pp: ZipPlusParams, polys, point_f, hint: ZipPlusHint) -> bytes:
        """ZipPlus::prove_f: point_f is (num_vars, field_limbs) Montgomery inners
        under the transcript's prime.  Returns the evaluation's inner bytes."""
        _keep, ptrs = _poly_ptrs(pp, polys)
        pf = np.ascontiguousarray(point_f, dtype=np.uint64)
        ev = C.create_string_buffer(8 * pp.zt.field_limbs)
        check(lib().zg_prove_f(pp.handle, transcript.handle, ptrs, len(polys), _ptr(pf), hint.handle, ev))
        return ev.raw

    @staticmethod
    def commit_prove(pp: ZipPlusParams, polys, point: Sequence[int]):
        """commit + new_from_commitment + get_random_field_cfg + prove in one call."""
        _keep, ptrs = _poly_ptrs(pp, polys)
        pt = i128_bytes(point)
        cap = C.c_size_t(pp.proof_size(len(polys)))
        proof = C.create_string_buffer(cap.value)
        root = C.create_string_buffer(32)
        ev = C.create_string_buffer(8 * pp.zt.field_limbs)
        check(lib().zg_commit_prove(pp.handle, ptrs, len(polys), C.c_char_p(pt), root, ev, proof,
                                    C.byref(cap)))
        return root.raw, ev.raw, proof.raw[: cap.value]

    @staticmethod
    def commit_prove_many(pp: ZipPlusParams, polys, points, lanes: int = 4):
        """Batched commit+prove of independent polynomials (one per request);
        returns [(root, eval, proof)] identical to sequential commit_prove."""
        n = len(polys)
        arrs = [np.ascontiguousarray(p, dtype=pp.eval_dtype) for p in polys]
        ptrs = (C.c_void_p * n)(*[a.ctypes.data for a in arrs])
        pts = b"".join(i128_bytes(pt) for pt in points)
        cap = pp.proof_size(1)
        bufs = [C.create_string_buffer(cap) for _ in range(n)]
        bptrs = (C.c_void_p * n)(*[C.addressof(b) for b in bufs])
        lens = (C.c_size_t * n)(*([cap] * n))
        roots = C.create_string_buffer(32 * n)
        fb = 8 * pp.zt.field_limbs
        evs = C.create_string_buffer(fb * n)
        check(lib().zg_commit_prove_many(pp.handle, n, ptrs, 0, C.c_char_p(pts), roots, evs, bptrs,
                                         lens, lanes, None))
        return [(roots.raw[32 * i:32 * i + 32], evs.raw[fb * i:fb * i + fb],
                 bufs[i].raw[: lens[i]]) for i in range(n)]

    @staticmethod
    def verify(pp: ZipPlusParams, comm: ZipPlusCommitment, point: Sequence[int], eval_inner: bytes,
               proof: bytes) -> None:
        """Raises ZipError unless the proof verifies."""
        pt = i128_bytes(point)
        check(lib().zg_verify(pp.handle, C.c_char_p(comm.root), comm.batch_size, C.c_char_p(pt),
                              C.c_char_p(eval_inner), C.c_char_p(proof), len(proof)))


class MerkleTree:
    """MerkleTree::new over the columns of a row-major matrix (root only)."""

    def __init__(self, root: bytes):
        self._root = root

    @staticmethod
    def new(rows: np.ndarray, elem_bytes: int, ctx: Context | None = None) -> "MerkleTree":
        rows = np.ascontiguousarray(rows, dtype=np.uint8)
        n_rows, width = rows.shape[0], rows.shape[1] // elem_bytes
        root = C.create_string_buffer(32)
        check(lib().zg_merkle_root((ctx or default_context()).handle, _ptr(rows), n_rows, width,
                                   elem_bytes, root))
        return MerkleTree(root.raw)

    def root(self) -> bytes:
        return self._root


# -------------------------------------------------------------------- sumcheck
def int_to_limbs(x: int, limbs: int) -> np.ndarray:
    return np.array([(x >> (64 * i)) & ((1 << 64) - 1) for i in range(limbs)], np.uint64)


def limbs_to_int(a) -> int:
    return sum(int(v) << (64 * i) for i, v in enumerate(np.asarray(a, np.uint64).ravel()))


def to_montgomery(x: int, modulus: int, limbs: int) -> int:
    """The Montgomery inner of x mod modulus (R = 2^(64 limbs))."""
    return (x % modulus) * (1 << (64 * limbs)) % modulus


def from_montgomery(inner: int, modulus: int, limbs: int) -> int:
    return inner * pow(1 << (64 * limbs), -1, modulus) % modulus


@dataclass
class SumcheckGroup:
    """One group of MLEs and its combination function, written as
    sum_k coeff_k * prod_{i in products[k]} mle_i (MultiDegreeSumcheckGroup,
    piop/src/sumcheck/multi_degree.rs:44-67).

    mles: (n_mles, 2^nvars, limbs) uint64 Montgomery inners, or the device address
    of that array (an int) with n_mles given; products: a list of
    (coeff_inner, [mle indices]); factors: affine factors (a_inner, b_inner,
    mle index) that multiply the sum of products; degree: the longest product
    plus the number of factors.
    """

    degree: int
    mles: object
    products: list
    n_mles: int = 0
    factors: list = None

    @property
    def on_device(self) -> bool:
        return isinstance(self.mles, int)

    def _arrays(self, limbs: int):
        mles = self.mles if self.on_device else np.ascontiguousarray(self.mles, dtype=np.uint64)
        coeffs = np.zeros((max(len(self.products), 1), limbs), np.uint64)
        offsets = np.zeros(len(self.products) + 1, np.uint32)
        idx = []
        for k, (c, ids) in enumerate(self.products):
            coeffs[k] = int_to_limbs(int(c), limbs)
            idx.extend(int(i) for i in ids)
            offsets[k + 1] = len(idx)
        indices = np.array(idx or [0], np.uint32)
        return mles, coeffs, offsets, indices

    def _factor_arrays(self, limbs: int):
        fs = self.factors or []
        fm = np.array([int(x[2]) for x in fs] or [0], np.uint32)
        fa = np.array([int_to_limbs(int(x[0]), limbs) for x in fs] or [[0] * limbs], np.uint64)
        fb = np.array([int_to_limbs(int(x[1]), limbs) for x in fs] or [[0] * limbs], np.uint64)
        return len(fs), fm, fa, fb


def _sumcheck_prove(transcript: PcsProverTranscript, modulus: int, limbs: int, nvars: int,
                    groups: Sequence[SumcheckGroup], multi: bool, ctx: Context | None):
    keep, descs = [], (SumcheckGroupDesc * len(groups))()
    n_mles = 0
    on_device = all(grp.on_device for grp in groups)
    if not on_device and any(grp.on_device for grp in groups):
        raise ValueError("MLEs of all groups must be on the device, or all on the host")
    for g, grp in zip(descs, groups):
        mles, coeffs, offsets, indices = grp._arrays(limbs)
        keep += [mles, coeffs, offsets, indices]
        k = grp.n_mles if on_device else mles.shape[0]
        g.degree, g.n_mles, g.n_products = grp.degree, k, len(grp.products)
        g.mles = mles if on_device else mles.ctypes.data
        g.coeffs = coeffs.ctypes.data
        g.offsets, g.indices = offsets.ctypes.data, indices.ctypes.data
        nf, fm, fa, fb_ = grp._factor_arrays(limbs)
        keep += [fm, fa, fb_]
        g.n_factors, g.factor_mles = nf, fm.ctypes.data
        g.factor_a, g.factor_b = fa.ctypes.data, fb_.ctypes.data
        n_mles += k
    fb = 8 * limbs
    cap = fb + 8 + 4 * len(groups) + fb * len(groups) + sum(
        nvars * (fb * g.degree + 4) for g in groups)
    proof = C.create_string_buffer(cap)
    plen = C.c_size_t(cap)
    point = np.zeros((nvars, limbs), np.uint64)
    finals = np.zeros((max(n_mles, 1), limbs), np.uint64)
    mod = int_to_limbs(modulus, limbs).tobytes()
    check(lib().zg_sumcheck_prove((ctx or default_context()).handle, transcript.handle,
                                  C.c_char_p(mod), limbs, nvars, int(multi), descs, len(groups),
                                  int(on_device),
                                  proof, C.byref(plen), _ptr(point), _ptr(finals)))
    return proof.raw[: plen.value], point, finals[:n_mles]


class MLSumcheck:
    """MLSumcheck::prove_as_subprotocol (piop/src/sumcheck.rs:163-215)."""

    @staticmethod
    def prove_as_subprotocol(transcript: PcsProverTranscript, modulus: int, limbs: int,
                             nvars: int, group: SumcheckGroup, ctx: Context | None = None):
        """Returns (SumcheckProof bytes, point inners (nvars, limbs), final MLE values)."""
        return _sumcheck_prove(transcript, modulus, limbs, nvars, [group], False, ctx)


class MultiDegreeSumcheck:
    """MultiDegreeSumcheck::prove_as_subprotocol (piop/src/sumcheck/multi_degree.rs:259-355)."""

    @staticmethod
    def prove_as_subprotocol(transcript: PcsProverTranscript, modulus: int, limbs: int,
                             nvars: int, groups: Sequence[SumcheckGroup],
                             ctx: Context | None = None):
        return _sumcheck_prove(transcript, modulus, limbs, nvars, list(groups), True, ctx)


def mle_evaluate(modulus: int, limbs: int, mle: np.ndarray, point: np.ndarray,
                 ctx: Context | None = None) -> np.ndarray:
    """sum_x mle[x] * eq(x, point) (mle_eval_with_eq_table, poly/src/utils.rs:267-284)."""
    mle = np.ascontiguousarray(mle, dtype=np.uint64)
    point = np.ascontiguousarray(point, dtype=np.uint64)
    out = np.zeros(limbs, np.uint64)
    mod = int_to_limbs(modulus, limbs).tobytes()
    check(lib().zg_mle_evaluate((ctx or default_context()).handle, C.c_char_p(mod), limbs,
                                _ptr(mle), point.shape[0], _ptr(point), _ptr(out)))
    return out


# -------------------------------------------------------------------- serving
class ZipServer:
    """Continuous-batching request server for commit+prove jobs (zg_server_*)."""

    def __init__(self, ctx: Context | None = None, workers: int = 4, hbm_budget: int = 0,
                 max_group: int = 16, max_skip_ms: int = 50, group_max_bytes: int = 0):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        opts = ServerOpts(workers, hbm_budget, max_group, max_skip_ms, group_max_bytes)
        check(lib().zg_server_create(self.ctx.handle, C.byref(opts), C.byref(h)))
        self.handle = h
        self._pending = {}

    def submit(self, pp: ZipPlusParams, poly, point: Sequence[int]) -> int:
        arr = _poly_ptrs(pp, [poly])[0][0]
        pt = C.create_string_buffer(i128_bytes(point), 16 * pp.num_vars)
        cap = pp.proof_size(1)
        root, ev = C.create_string_buffer(32), C.create_string_buffer(8 * pp.zt.field_limbs)
        proof = C.create_string_buffer(cap)
        rid = C.c_uint64()
        check(lib().zg_server_submit(self.handle, pp.handle, C.c_void_p(arr.ctypes.data), pt, root, ev,
                                     proof, cap, C.byref(rid)))
        self._pending[rid.value] = (arr, pt, root, ev, proof)
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1):
        """Returns (root, eval, proof, ServerResult) of request rid."""
        res = ServerResult()
        st = lib().zg_server_wait(self.handle, rid, timeout_ms, C.byref(res))
        if st == 7:  # still running: keep its buffers
            check(st)
        _arr, _pt, root, ev, proof = self._pending.pop(rid)
        check(st)
        return root.raw, ev.raw, proof.raw[: res.proof_len], res

    def stats(self) -> ServerStats:
        out = ServerStats()
        check(lib().zg_server_get_stats(self.handle, C.byref(out)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            check(lib().zg_server_destroy(self.handle))
            self.handle = None
            self._pending.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ZincPlusPiop:
    """ZincPlusPiop::prove::<MLE_FIRST = true> (protocol/src/prover.rs:677-706)
    for a linear UAIR over binary-polynomial and integer (i64) witness columns,
    every step on the GPU; returns the Proof transcription
    (protocol/src/lib.rs:87-189)."""

    _out = None  # output buffer reused across calls (one call at a time)

    @staticmethod
    def prove_mle_first(pp_bin, pp_int, nvars: int, bin_cols, degree_plus_one: int, int_cols, shifts,
                        coeffs, n_pub_bin: int = 0, n_pub_int: int = 0, out_buffer=None) -> bytes:
        """The first n_pub_bin binary and n_pub_int integer columns are public.
        out_buffer (optional): a uint8 array the proof is written into (a
        page-locked one receives the column openings by DMA); the proof is then
        returned as a view of it (valid until the buffer is reused), not a copy."""
        b, i = ZincPiop._cols(bin_cols, int_cols, nvars)
        src = np.array([s for s, _ in shifts] or [0], np.uint32)
        amt = np.array([a for _, a in shifts] or [0], np.uint32)
        cf = np.ascontiguousarray(coeffs, dtype=np.int64)
        ncols = b.shape[0] + i.shape[0]
        if cf.ndim != 2 or cf.shape[1] != ncols + len(shifts):
            raise ValueError("coeffs must be n_constraints x (n_bin + n_int + n_shifts)")
        u = LinearUairDesc(b.shape[0], i.shape[0], degree_plus_one, len(shifts), src.ctypes.data, amt.ctypes.data,
                           cf.shape[0], cf.ctypes.data, n_pub_bin, n_pub_int)
        pbin = pp_bin.handle if pp_bin is not None else None
        pint = pp_int.handle if pp_int is not None else None
        cap = 64 << 10
        for pp in (pp_bin, pp_int):
            if pp is not None:
                cap += pp.proof_size(max(b.shape[0], i.shape[0], 1))
        cap += (ncols * (degree_plus_one + 2) + cf.shape[0] * degree_plus_one + 64 * nvars) * 64
        buf = out_buffer if out_buffer is not None else ZincPlusPiop._out
        if buf is None or buf.size < cap:
            if out_buffer is not None:
                raise ValueError(f"out_buffer holds {out_buffer.size} bytes, {cap} needed")
            buf = ZincPlusPiop._out = np.empty(cap, np.uint8)
        n = C.c_size_t(buf.size)
        check(lib().zg_zinc_prove_mle_first(pbin, pint, C.byref(u), nvars, _ptr(b), _ptr(i), 0, _ptr(buf),
                                            C.byref(n)))
        if out_buffer is not None:
            return memoryview(buf)[: n.value]
        return buf[: n.value].tobytes()

    @staticmethod
    def prove(pp_bin, pp_int, nvars: int, bin_cols, degree_plus_one: int, int_cols, shifts, constraints,
              zero_ideal, mle_first: bool = False, n_pub_bin: int = 0, n_pub_int: int = 0) -> bytes:
        """ZincPlusPiop::prove::<MLE_FIRST> with the UAIR as terms: constraints is
        a list per constraint of (integer coefficient, [one or two column indices
        into up (binary, then integer) and down (shift order)]); zero_ideal one
        flag per constraint.  mle_first=False is the reference's default
        (combined) path."""
        b, i = ZincPiop._cols(bin_cols, int_cols, nvars)
        src = np.array([s for s, _ in shifts] or [0], np.uint32)
        amt = np.array([a for _, a in shifts] or [0], np.uint32)
        toff, coef, foff, fcol = [0], [], [0], []
        for terms in constraints:
            for c, cols in terms:
                coef.append(int(c))
                fcol.extend(int(x) for x in cols)
                foff.append(len(fcol))
            toff.append(len(coef))
        toff_a = np.array(toff, np.uint32)
        coef_a = np.array(coef or [0], np.int64)
        foff_a = np.array(foff, np.uint32)
        fcol_a = np.array(fcol or [0], np.uint32)
        zi = np.array([1 if z else 0 for z in zero_ideal] or [0], np.uint8)
        if len(zero_ideal) != len(constraints):
            raise ValueError("one zero_ideal flag per constraint")
        u = UairDesc(b.shape[0], i.shape[0], degree_plus_one, len(shifts), src.ctypes.data, amt.ctypes.data,
                     len(constraints), toff_a.ctypes.data, coef_a.ctypes.data, foff_a.ctypes.data,
                     fcol_a.ctypes.data, zi.ctypes.data, n_pub_bin, n_pub_int)
        pbin = pp_bin.handle if pp_bin is not None else None
        pint = pp_int.handle if pp_int is not None else None
        ncols = b.shape[0] + i.shape[0]
        cap = 64 << 10
        for pp in (pp_bin, pp_int):
            if pp is not None:
                cap += pp.proof_size(max(b.shape[0], i.shape[0], 1))
        cap += (ncols * (degree_plus_one + 2) + len(constraints) * 2 * degree_plus_one + 64 * nvars) * 64
        buf = ZincPlusPiop._out
        if buf is None or buf.size < cap:
            buf = ZincPlusPiop._out = np.empty(cap, np.uint8)
        n = C.c_size_t(buf.size)
        check(lib().zg_zinc_prove(pbin, pint, C.byref(u), nvars, _ptr(b), _ptr(i), 0, 1 if mle_first else 0,
                                  _ptr(buf), C.byref(n)))
        return buf[: n.value].tobytes()


def read_proof(proof: bytes, limbs: int, num_vars: int) -> dict:
    """Proof::read_transcription_bytes_exact (protocol/src/lib.rs:93-127): the
    places and counts of a Zinc+ proof's parts (raises ZipError if malformed)."""
    lay = ProofLayout()
    check(lib().zg_proof_read(proof, len(proof), limbs, num_vars, C.byref(lay)))
    out = {f: getattr(lay, f) for f, _ in ProofLayout._fields_ if f not in ("roots", "batch_sizes", "modulus")}
    out["roots"] = [bytes(r) for r in lay.roots]
    out["batch_sizes"] = list(lay.batch_sizes)
    out["modulus"] = int.from_bytes(bytes(lay.modulus)[: 8 * limbs], "little")
    return out


class ZincPiop:
    """Zinc+ prover steps 3 and 6 on the trace columns (protocol/src/prover.rs:
    385-415 and 497-532) on the GPU.  Field elements are Montgomery inners
    (uint64 arrays of `limbs` words); the modulus is a Python int."""

    @staticmethod
    def _cols(bin_cols, int_cols, nvars):
        n = 1 << nvars
        b = np.ascontiguousarray(bin_cols if bin_cols is not None else np.zeros((0, n)), dtype=np.uint64)
        i = np.ascontiguousarray(int_cols if int_cols is not None else np.zeros((0, n)), dtype=np.int64)
        for x in (b, i):
            if x.ndim != 2 or (x.shape[0] and x.shape[1] != n):
                raise ValueError("columns must be (count, 2^nvars) arrays")
        return b, i

    @staticmethod
    def eval_projection(ctx: Context, modulus: int, limbs: int, bin_cols, degree_plus_one: int, int_cols,
                        nvars: int, a) -> np.ndarray:
        """step3: (n_bin + n_int, 2^nvars, limbs) MLEs of the projected trace at a."""
        b, i = ZincPiop._cols(bin_cols, int_cols, nvars)
        out = np.zeros((b.shape[0] + i.shape[0], 1 << nvars, limbs), np.uint64)
        av = np.ascontiguousarray(a, dtype=np.uint64)
        mod = modulus.to_bytes(8 * limbs, "little")
        check(lib().zg_piop_eval_projection(ctx.handle, mod, limbs, _ptr(b), b.shape[0], degree_plus_one,
                                            _ptr(i), i.shape[0], nvars, _ptr(av), 0, _ptr(out)))
        return out

    @staticmethod
    def lifted_evals(ctx: Context, modulus: int, limbs: int, bin_cols, degree_plus_one: int, int_cols,
                     nvars: int, point) -> np.ndarray:
        """step6: (n_bin * degree_plus_one + n_int, limbs) coefficients."""
        b, i = ZincPiop._cols(bin_cols, int_cols, nvars)
        out = np.zeros((b.shape[0] * degree_plus_one + i.shape[0], limbs), np.uint64)
        pt = np.ascontiguousarray(point, dtype=np.uint64)
        mod = modulus.to_bytes(8 * limbs, "little")
        check(lib().zg_piop_lifted_evals(ctx.handle, mod, limbs, _ptr(b), b.shape[0], degree_plus_one,
                                         _ptr(i), i.shape[0], nvars, _ptr(pt), 0, _ptr(out)))
        return out

    @staticmethod
    def multipoint_eval(ctx: Context, transcript, modulus: int, limbs: int, trace_mles, nvars: int,
                        eval_point, shifts):
        """step5 (MultipointEval::prove_as_subprotocol): trace_mles (num_cols, 2^nvars,
        limbs) Montgomery inners, or a device pointer int with num_cols given as
        trace_mles=(ptr, num_cols); shifts [(source_col, shift_amount)].  Returns
        (SumcheckProof bytes, r_0 (nvars, limbs))."""
        if isinstance(trace_mles, tuple):
            ptr, ncols, on_dev = trace_mles[0], trace_mles[1], 1
        else:
            arr = np.ascontiguousarray(trace_mles, dtype=np.uint64)
            ptr, ncols, on_dev = arr.ctypes.data, arr.shape[0], 0
        r = np.ascontiguousarray(eval_point, dtype=np.uint64)
        src = np.array([sc for sc, _ in shifts] or [0], np.uint32)
        amt = np.array([c for _, c in shifts] or [0], np.uint32)
        cap = C.c_size_t(64 + 16 * limbs * (4 + 3 * nvars))
        proof = C.create_string_buffer(cap.value)
        r0 = np.zeros((nvars, limbs), np.uint64)
        mod = modulus.to_bytes(8 * limbs, "little")
        check(lib().zg_piop_multipoint_eval(ctx.handle, transcript.handle, mod, limbs, ptr, ncols, nvars,
                                            _ptr(r), _ptr(src), _ptr(amt), len(shifts), on_dev, proof,
                                            C.byref(cap), _ptr(r0)))
        return proof.raw[: cap.value], r0

    @staticmethod
    def cpr_linear_prove(ctx: Context, transcript, modulus: int, limbs: int, trace_mles, nvars: int, eval_point,
                         shifts, coeffs):
        """step4 for a linear UAIR: trace_mles (num_cols, 2^nvars, limbs) inners or
        (device pointer, num_cols); coeffs (n_constraints, num_cols + len(shifts))
        standard integers mod the modulus.  Returns (proof, point (nvars, limbs),
        evals (num_cols + len(shifts), limbs))."""
        if isinstance(trace_mles, tuple):
            ptr, ncols, on_dev = trace_mles[0], trace_mles[1], 1
        else:
            arr = np.ascontiguousarray(trace_mles, dtype=np.uint64)
            ptr, ncols, on_dev = arr.ctypes.data, arr.shape[0], 0
        R = 1 << (64 * limbs)
        cf = np.array([[[((int(c) % modulus) * R % modulus >> (64 * w)) & ((1 << 64) - 1) for w in range(limbs)]
                        for c in row] for row in coeffs], np.uint64)
        r = np.ascontiguousarray(eval_point, dtype=np.uint64)
        src = np.array([sc for sc, _ in shifts] or [0], np.uint32)
        amt = np.array([c for _, c in shifts] or [0], np.uint32)
        cap = C.c_size_t(64 + 8 * limbs * (8 + 6 * nvars))
        proof = C.create_string_buffer(cap.value)
        pt = np.zeros((nvars, limbs), np.uint64)
        ev = np.zeros((ncols + len(shifts), limbs), np.uint64)
        mod = modulus.to_bytes(8 * limbs, "little")
        check(lib().zg_piop_cpr_linear_prove(ctx.handle, transcript.handle, mod, limbs, ptr, ncols, nvars, _ptr(r),
                                             _ptr(src), _ptr(amt), len(shifts), cf.shape[0], _ptr(cf), on_dev,
                                             proof, C.byref(cap), _ptr(pt), _ptr(ev)))
        return proof.raw[: cap.value], pt, ev

    @staticmethod
    def _mont_matrix(coeffs, modulus, limbs):
        R = 1 << (64 * limbs)
        return np.array([[[((int(c) % modulus) * R % modulus >> (64 * w)) & ((1 << 64) - 1) for w in range(limbs)]
                          for c in row] for row in coeffs], np.uint64)

    @staticmethod
    def ideal_check_linear(ctx: Context, transcript, modulus: int, limbs: int, bin_cols, degree_plus_one: int,
                           int_cols, nvars: int, shifts, coeffs):
        """step2 for a linear UAIR: returns (point (nvars, limbs), [combined value
        per constraint as a (trimmed length, limbs) array])."""
        b, i = ZincPiop._cols(bin_cols, int_cols, nvars)
        cf = ZincPiop._mont_matrix(coeffs, modulus, limbs)
        src = np.array([sc for sc, _ in shifts] or [0], np.uint32)
        amt = np.array([c for _, c in shifts] or [0], np.uint32)
        pt = np.zeros((nvars, limbs), np.uint64)
        comb = np.zeros((cf.shape[0], degree_plus_one, limbs), np.uint64)
        lens = np.zeros(cf.shape[0], np.uint32)
        mod = modulus.to_bytes(8 * limbs, "little")
        check(lib().zg_piop_ideal_check_linear(ctx.handle, transcript.handle, mod, limbs, _ptr(b), b.shape[0],
                                               degree_plus_one, _ptr(i), i.shape[0], nvars, _ptr(src), _ptr(amt),
                                               len(shifts), cf.shape[0], _ptr(cf), 0, _ptr(pt), _ptr(comb),
                                               _ptr(lens)))
        return pt, [comb[k, : lens[k]] for k in range(cf.shape[0])]
