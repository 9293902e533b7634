"""Batched commit of independent polynomials of mixed shapes (zg_commit_batch):
every root equals the oracle's commit_single of that polynomial (and a
sequential zg_commit), across group splits, kernel variants, graph replays,
device inputs, and the hints that feed prove."""
import numpy as np
import pytest

from util import binary_evals, desc_for, i32_evals, params_for

pytestmark = pytest.mark.gpu


def layout(nv):
    """row_len = 2^min(nv, 14), num_rows = 2^max(0, nv - 14)."""
    return 1 << min(nv, 14)


def _evals(rng, ek, D, n):
    return i32_evals(rng, n) if ek == 0 else binary_evals(rng, n, D)


class Shapes:
    def __init__(self, zipgpu, ctx):
        self.z, self.ctx, self.cache = zipgpu, ctx, {}

    def get(self, ek, D, ck, nv, L=None):
        key = (ek, D, ck, nv, L)
        if key not in self.cache:
            self.cache[key] = params_for(self.z, ek, D, ck, nv, L or layout(nv), ctx=self.ctx)
        return self.cache[key]


MIXED = [  # (eval_kind, D, code_kind, num_vars, row_len or None, count)
    (1, 64, 0, 10, None, 3), (1, 64, 0, 12, None, 2), (1, 32, 0, 11, None, 4),
    (1, 64, 0, 15, None, 2), (1, 32, 0, 16, None, 1), (0, 1, 0, 12, 4096, 2),
    (0, 1, 0, 10, 64, 3), (1, 32, 1, 12, 64, 2), (1, 3, 0, 10, 256, 2),
]


def _mixed(zipgpu, ctx, rng):
    sh = Shapes(zipgpu, ctx)
    pps, polys, descs = [], [], []
    for ek, D, ck, nv, L, cnt in MIXED:
        for _ in range(cnt):
            pps.append(sh.get(ek, D, ck, nv, L))
            polys.append(_evals(rng, ek, D, 1 << nv))
            descs.append(desc_for(ek, D, ck, nv, L or layout(nv)))
    order = rng.permutation(len(pps))  # interleave the shapes
    return [pps[i] for i in order], [polys[i] for i in order], [descs[i] for i in order]


def test_batch_commit_matches_oracle(zipgpu, oracle, ctx, rng):
    pps, polys, descs = _mixed(zipgpu, ctx, rng)
    comms = zipgpu.ZipPlus.commit_batch(pps, polys, ctx)
    for c, d, p in zip(comms, descs, polys):
        assert c.root == oracle.commit(d, p, 1)
    # replay of the captured graph on new inputs of the same shapes
    polys2 = [_evals(rng, pp.zt.eval_kind, pp.zt.degree_plus_one, 1 << pp.num_vars) for pp in pps]
    comms2 = zipgpu.ZipPlus.commit_batch(pps, polys2, ctx)
    for c, d, p in zip(comms2, descs, polys2):
        assert c.root == oracle.commit(d, p, 1)


@pytest.mark.parametrize("base,leaf", [(0, 0), (1, 1), (2, 0), (3, 1), (4, 0), (5, 1), (6, 0), (7, 1),
                                       (8, 0), (9, 1), (-1, -1)])
def test_batch_commit_variants_agree(zipgpu, ctx, rng, base, leaf):
    pps, polys, _ = _mixed(zipgpu, ctx, rng)
    want = [zipgpu.ZipPlus.commit(pp, [p])[1].root for pp, p in zip(pps, polys)]
    for graph in (True, False):
        opts = zipgpu.BatchOpts.make(lanes=3, use_graph=graph, autotune=False, base_variant=base,
                                     leaf_variant=leaf)
        got = zipgpu.ZipPlus.commit_batch(pps, polys, ctx, opts)
        assert [c.root for c in got] == want


def test_batch_commit_hints_prove(zipgpu, oracle, ctx, rng):
    """Hints of a grouped commit (segmented codewords, stacked trees) give the
    same proofs as a plain commit_prove."""
    sh = Shapes(zipgpu, ctx)
    pps = [sh.get(1, 32, 0, 12), sh.get(1, 32, 0, 12), sh.get(1, 32, 0, 12), sh.get(1, 64, 0, 15),
           sh.get(1, 64, 0, 15), sh.get(0, 1, 0, 10, 64)]
    polys = [_evals(rng, pp.zt.eval_kind, pp.zt.degree_plus_one, 1 << pp.num_vars) for pp in pps]
    comms, hints = zipgpu.ZipPlus.commit_batch(pps, polys, ctx, hints=True)
    for pp, p, c, h in zip(pps, polys, comms, hints):
        point = [(-1) ** i * (3 * i + 1) for i in range(pp.num_vars)]
        root, ev, proof = zipgpu.ZipPlus.commit_prove(pp, [p], point)
        assert c.root == root
        t = zipgpu.PcsProverTranscript.new_from_commitment(c)
        t.get_random_field_cfg(4)
        assert zipgpu.ZipPlus.prove(t, pp, [p], point, h) == ev
        assert t.stream == proof
        assert np.array_equal(h.codeword(0), zipgpu.ZipPlus.encode_rows(pp, p))
    # freeing hints one by one keeps the others' shared block alive
    for h in hints[:2]:
        h.close()
    t = zipgpu.PcsProverTranscript.new_from_commitment(comms[2])
    t.get_random_field_cfg(4)
    point = [5] * pps[2].num_vars
    ev = zipgpu.ZipPlus.prove(t, pps[2], [polys[2]], point, hints[2])
    zipgpu.ZipPlus.verify(pps[2], comms[2], point, ev, t.stream)


def test_batch_commit_device_inputs(zipgpu, ctx, rng):
    import torch

    sh = Shapes(zipgpu, ctx)
    pps = [sh.get(1, 64, 0, 11)] * 3 + [sh.get(1, 32, 0, 13)] * 2 + [sh.get(0, 1, 0, 12, 4096)]
    polys = [_evals(rng, pp.zt.eval_kind, pp.zt.degree_plus_one, 1 << pp.num_vars) for pp in pps]
    want = [zipgpu.ZipPlus.commit(pp, [p])[1].root for pp, p in zip(pps, polys)]
    dev = [torch.from_numpy(p.view(np.uint8).copy()).cuda() for p in polys]
    torch.cuda.synchronize()
    for _ in range(2):
        got = zipgpu.ZipPlus.commit_batch(pps, [d.data_ptr() for d in dev], ctx, on_device=True)
        assert [c.root for c in got] == want
    # new device buffers: the plan captures again
    dev2 = [d.clone() for d in dev]
    torch.cuda.synchronize()
    got = zipgpu.ZipPlus.commit_batch(pps, [d.data_ptr() for d in dev2], ctx, on_device=True)
    assert [c.root for c in got] == want


def test_batch_commit_pinned_inputs(zipgpu, ctx, rng):
    """Page-locked host inputs are read by DMA in place; new buffers recapture."""
    import torch

    sh = Shapes(zipgpu, ctx)
    pps = [sh.get(1, 64, 0, 12)] * 2 + [sh.get(1, 32, 0, 15), sh.get(0, 1, 0, 10, 64)]
    polys = [_evals(rng, pp.zt.eval_kind, pp.zt.degree_plus_one, 1 << pp.num_vars) for pp in pps]
    want = [zipgpu.ZipPlus.commit(pp, [p])[1].root for pp, p in zip(pps, polys)]
    for _ in range(2):
        pinned = [torch.from_numpy(p.copy()).pin_memory().numpy() for p in polys]
        for _ in range(2):
            got = zipgpu.ZipPlus.commit_batch(pps, pinned, ctx)
            assert [c.root for c in got] == want
        pinned[0][:] = polys[1]  # same buffers, new contents: the replay reads them
        got = zipgpu.ZipPlus.commit_batch(pps, pinned, ctx)
        assert got[0].root == want[1]


def test_batch_commit_64_polys_nv10_20_deg64(zipgpu, oracle, ctx):
    """64 polynomials, num_vars uniform in 10..20, BinaryPoly<64> Bernoulli(0.5),
    IPRS: equal to 64 sequential commits; the smallest ones also to the oracle."""
    rng = np.random.default_rng(0x5A1F)
    sh = Shapes(zipgpu, ctx)
    nvs = rng.integers(10, 21, size=64)
    pps = [sh.get(1, 64, 0, int(nv)) for nv in nvs]
    polys = [binary_evals(rng, 1 << int(nv), 64) for nv in nvs]
    got = zipgpu.ZipPlus.commit_batch(pps, polys, ctx)
    for pp, p, c in zip(pps, polys, got):
        assert c.root == zipgpu.ZipPlus.commit(pp, [p])[1].root
    for nv, p, c in zip(nvs, polys, got):
        if nv <= 11:
            assert c.root == oracle.commit(desc_for(1, 64, 0, int(nv), layout(int(nv))), p, 1)


def test_batch_commit_after_parameters_are_freed(zipgpu, ctx, rng):
    """Plans are keyed per parameter set, not per address: freeing a set and
    creating sets of other shapes (which can reuse its address) commits right."""
    import gc

    for nv in (11, 13, 12, 14, 11, 15):
        pp = params_for(zipgpu, 1, 32, 0, nv, 1 << min(nv, 14), ctx=ctx)
        poly = binary_evals(rng, 1 << nv, 32)
        want = zipgpu.ZipPlus.commit(pp, [poly])[1].root
        for _ in range(2):
            assert zipgpu.ZipPlus.commit_batch([pp], [poly], ctx)[0].root == want
        pp.close()
        del pp
        gc.collect()


def test_batch_commit_rejects_bad_input(zipgpu, ctx, rng):
    pp = params_for(zipgpu, 1, 32, 0, 10, 1024, ctx=ctx)
    with pytest.raises(ValueError):
        zipgpu.ZipPlus.commit_batch([pp], [], ctx)
    with pytest.raises(ValueError):  # wrong size
        zipgpu.ZipPlus.commit_batch([pp], [binary_evals(rng, 512, 32)], ctx)


# (D, num_vars, row_len, depth): odd lane counts (one 32-lane half padded, or two
# halves), K padded to 128 (base_len 2..128), base dimensions below and above the
# 64 / 128-row tiles, several codeword rows
UMMA_SHAPES = [(3, 10, 256, 0), (17, 12, 1024, 0), (40, 12, 4096, 3), (64, 14, 4096, 0),
               (32, 14, 1 << 14, 0), (8, 12, 1024, 1), (32, 16, 1 << 12, 0)]


@pytest.mark.parametrize("variant", [6, 7, 8, 9])
def test_tcgen05_base_variants_match_oracle(zipgpu, oracle, ctx, rng, variant):
    """Each tcgen05 base-layer kernel (persistent / one tile per block, 128 or 64
    base rows per tile) gives the oracle's roots on every shape."""
    opts = zipgpu.BatchOpts.make(lanes=1, use_graph=False, autotune=False, base_variant=variant,
                                 leaf_variant=-1)
    for D, nv, L, depth in UMMA_SHAPES:
        pp = params_for(zipgpu, 1, D, 0, nv, L, depth, ctx=ctx)
        ev = binary_evals(rng, 1 << nv, D)
        got = zipgpu.ZipPlus.commit_batch([pp], [ev], ctx, opts)
        assert got[0].root == oracle.commit(desc_for(1, D, 0, nv, L, depth), ev, 1), (D, nv, L, depth)
