"""The allocation-free Merkle root entry point, zg_merkle_root_noalloc_d.

It serves callers that must not allocate device memory while handling a
request (a serving loop that reserved its device-memory budget up front, or a
host whose device buffers all come from its own pool): it takes the leaves and
the root buffer from the caller and keeps its node layers in a fixed 4 MiB
array inside the library.  These tests call it through the C ABI and compare
its root with the existing entry point zg_merkle_root on the same data, for
two calls in a row (the shared scratch keeps the previous call's contents, so
the second call must not depend on them).

This file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_root(zipgpu, torch, leaf_major: np.ndarray) -> bytes:
    width, leaf_bytes = leaf_major.shape
    leaves = torch.from_numpy(np.ascontiguousarray(leaf_major).reshape(-1)).cuda()
    root = torch.zeros(32, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    zipgpu.check(zipgpu.lib().zg_merkle_root_noalloc_d(
        leaves.data_ptr(), width, leaf_bytes, root.data_ptr(), stream.cuda_stream))
    stream.synchronize()
    return bytes(root.cpu().numpy())


@pytest.mark.parametrize("rows,width,eb", [
    (4, 4096, 256),   # 1 KiB leaves, one BLAKE3 chunk each
    (64, 256, 16),
    (1, 65536, 16),   # the largest tree the scratch holds
    (16, 512, 256),   # 4 KiB leaves: chunk chaining values in the scratch too
    (3, 1, 12),       # a single leaf is the root
])
def test_noalloc_root_matches_merkle_root(zipgpu, ctx, rows, width, eb):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(rows * 7919 + width)
    for _ in range(2):  # two calls in a row on the shared scratch
        data = rng.integers(0, 256, (rows, width * eb), dtype=np.uint8)
        expected = zipgpu.MerkleTree.new(data, eb, ctx).root()
        leaf_major = data.reshape(rows, width, eb).transpose(1, 0, 2).reshape(width, rows * eb)
        assert _noalloc_root(zipgpu, torch, leaf_major) == expected


def test_noalloc_rejects_sizes_beyond_its_scratch(zipgpu, ctx):
    torch = pytest.importorskip("torch")
    small = torch.zeros(64, dtype=torch.uint8, device="cuda")
    root = torch.zeros(32, dtype=torch.uint8, device="cuda")
    fn = zipgpu.lib().zg_merkle_root_noalloc_d
    # 2^17 leaves need (2^18 - 1) * 32 bytes of nodes: more than 4 MiB.  The size
    # check comes before any access, so the small buffer is never read.
    status = fn(small.data_ptr(), 1 << 17, 16, root.data_ptr(), None)
    assert status == 1
    assert b"limit" in zipgpu.lib().zg_last_error()
    assert fn(small.data_ptr(), 3, 16, root.data_ptr(), None) == 1  # not a power of two
    # A leaf pointer at an odd offset is refused before any launch: the leaf
    # kernels read 32-bit words.
    assert fn(small.data_ptr() + 1, 2, 16, root.data_ptr(), None) == 1
    assert b"aligned" in zipgpu.lib().zg_last_error()
    # The context is still usable afterwards.
    data = np.arange(2 * 16, dtype=np.uint8).reshape(1, 32)
    assert _noalloc_root(zipgpu, torch, data.reshape(2, 16)) == zipgpu.MerkleTree.new(data, 16, ctx).root()
