"""BigLinearUair (test-uair/src/lib.rs:325-456): its signature and constraints
in the form the MLE-first prover takes, and a seeded trace generator with the
reference generator's structure.

Columns: 16 BinaryPoly<32> columns b_0..b_15 and one integer column z; shifts
(b_k, 1) for k = 0..15, so the down columns are d_k = b_k shifted up one row.
Constraints (constrain_general, lib.rs:340-382), as coefficient rows over
[b_0..b_15, z, d_0..d_15]:
  b_0 + ... + b_15 - z    in (X - 1)
  d_0 - z                 in (X - 2)
  b_k - d_k, k = 1..15    in (X - 1)
"""
import numpy as np

N_BIN, N_INT, DEGREE_PLUS_ONE = 16, 1, 32


def signature():
    """(shifts [(source column, amount)], coefficient rows) of BigLinearUair."""
    shifts = [(k, 1) for k in range(N_BIN)]
    ncol = N_BIN + N_INT + len(shifts)
    rows = []
    r = np.zeros(ncol, np.int64)
    r[:N_BIN] = 1
    r[N_BIN] = -1
    rows.append(r)
    r = np.zeros(ncol, np.int64)
    r[N_BIN + N_INT] = 1
    r[N_BIN] = -1
    rows.append(r)
    for k in range(1, N_BIN):
        r = np.zeros(ncol, np.int64)
        r[k] = 1
        r[N_BIN + N_INT + k] = -1
        rows.append(r)
    return shifts, np.stack(rows)


def ideal_roots():
    """The root c of each constraint's ideal (X - c), in constraint order."""
    return [1, 2] + [1] * (N_BIN - 1)


def _popcount32(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    c = np.zeros(x.shape, np.int64)
    for k in range(32):
        c += ((x >> np.uint64(k)) & np.uint64(1)).astype(np.int64)
    return c


def trace(nvars: int, seed: int):
    """A BigLinear trace (generate_random_trace, lib.rs:384-456) from a seeded
    generator: row 0 of every binary column uniform; b_k (k >= 1) keeps its
    popcount down the column with a uniformly random bit pattern per row; z_i =
    sum_k popcount(b_k[i]); b_0[i + 1] = z_i as a bit pattern.  Returns (binary
    columns (16, 2^nvars) u64, integer columns (1, 2^nvars) i64)."""
    rng = np.random.default_rng(seed)
    n = 1 << nvars
    first = rng.integers(0, 1 << 32, size=N_BIN, dtype=np.uint64)
    bins = np.zeros((N_BIN, n), np.uint64)
    K = 0
    for k in range(1, N_BIN):
        pc = int(_popcount32(first[k : k + 1])[0])
        K += pc
        bins[k, 0] = first[k]
        if n > 1 and pc:
            # a uniformly random pc-subset of the 32 positions per row
            keys = rng.random((n - 1, 32))
            pos = np.argpartition(keys, pc - 1, axis=1)[:, :pc]
            bins[k, 1:] = np.bitwise_or.reduce(np.left_shift(np.uint64(1), pos.astype(np.uint64)), axis=1)
    b0 = np.zeros(n, np.uint64)
    x = int(first[0])
    for i in range(n):
        b0[i] = x
        x = bin(x).count("1") + K
    bins[0] = b0
    ints = (_popcount32(b0) + K).astype(np.int64).reshape(1, n)
    return bins, ints
