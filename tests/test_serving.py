"""Request server (zg_server_*): continuous batching of commit+prove requests of
mixed sizes.  Every result must be byte-identical to the same request run
alone through zg_commit_prove, whatever else is in flight."""
import time

import numpy as np
import pytest

from util import binary_evals, i32_evals, params_for

pytestmark = pytest.mark.gpu


def _shapes(zipgpu, ctx):
    out = {}
    for D in (32, 64):
        for nv in (10, 11, 12, 13):
            out[(1, D, nv)] = params_for(zipgpu, 1, D, 0, nv, 1 << min(nv, 14), ctx=ctx)
    out[(0, 1, 10)] = params_for(zipgpu, 0, 1, 0, 10, 1024, ctx=ctx)
    out[(1, 32, 15)] = params_for(zipgpu, 1, 32, 0, 15, 1 << 14, ctx=ctx)  # 2 rows
    return out


def _request(rng, pp):
    if pp.zt.eval_kind == 0:
        poly = i32_evals(rng, 1 << pp.num_vars)
    else:
        poly = binary_evals(rng, 1 << pp.num_vars, pp.zt.degree_plus_one)
    point = [int(v) for v in rng.integers(-(2**40), 2**40, size=pp.num_vars)]
    return poly, point


def _stream(zipgpu, ctx, rng, n, workers, budget=0, mean_gap_ms=0.5, repeat_shape=0.5):
    shapes = _shapes(zipgpu, ctx)
    keys = list(shapes)
    reqs = []
    for i in range(n):
        # runs of equal shapes, so that some requests can share a launch chain
        key = reqs[-1][0] if reqs and rng.random() < repeat_shape else keys[rng.integers(len(keys))]
        reqs.append((key,) + _request(rng, shapes[key]))
    srv = zipgpu.ZipServer(ctx, workers=workers, hbm_budget=budget)
    ids = []
    for key, poly, point in reqs:
        ids.append(srv.submit(shapes[key], poly, point))
        time.sleep(rng.exponential(mean_gap_ms) / 1000.0)
    results = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.close()
    return shapes, reqs, results, stats


def test_server_results_equal_alone(zipgpu, ctx, rng):
    shapes, reqs, results, stats = _stream(zipgpu, ctx, rng, 48, workers=4)
    assert stats.completed == 48 and stats.grouped_requests == 48
    for (key, poly, point), (root, ev, proof, res) in zip(reqs, results):
        assert res.status == 0 and res.latency_ms >= res.queue_ms >= 0
        assert (root, ev, proof) == zipgpu.ZipPlus.commit_prove(shapes[key], [poly], point)


def test_server_groups_same_shape_requests(zipgpu, ctx, rng):
    """A burst of equal-shape requests is committed in shared launch chains."""
    shapes = _shapes(zipgpu, ctx)
    pp = shapes[(1, 32, 11)]
    srv = zipgpu.ZipServer(ctx, workers=1, max_group=8)
    reqs = [_request(rng, pp) for _ in range(24)]
    ids = [srv.submit(pp, poly, point) for poly, point in reqs]
    results = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.close()
    assert stats.groups < 24
    assert max(r[3].group_size for r in results) > 1
    for (poly, point), (root, ev, proof, _res) in zip(reqs, results):
        assert (root, ev, proof) == zipgpu.ZipPlus.commit_prove(pp, [poly], point)


def test_server_respects_hbm_budget(zipgpu, ctx, rng):
    budget = 160 << 20
    shapes, reqs, results, stats = _stream(zipgpu, ctx, rng, 24, workers=6, budget=budget,
                                           mean_gap_ms=0.1)
    assert stats.budget == budget
    assert 0 < stats.peak_reserved <= budget
    for (key, poly, point), (root, ev, proof, res) in zip(reqs, results):
        assert (root, ev, proof) == zipgpu.ZipPlus.commit_prove(shapes[key], [poly], point)


def test_server_rejects_request_above_budget(zipgpu, ctx, rng):
    pp = params_for(zipgpu, 1, 64, 0, 13, 1 << 13, ctx=ctx)
    srv = zipgpu.ZipServer(ctx, workers=1, hbm_budget=1 << 20)
    poly, point = _request(rng, pp)
    with pytest.raises(zipgpu.ZipError) as e:
        srv.submit(pp, poly, point)
    assert e.value.status == 6
    srv.close()


def test_served_results_equal_the_oracle(zipgpu, oracle, ctx, rng):
    """Served proofs checked against the oracle directly (not only through the
    plain GPU path): a mixed stream of i32 and BinaryPoly shapes, with groups."""
    shapes, reqs, results, stats = _stream(zipgpu, ctx, rng, 16, workers=3)
    assert stats.completed == 16
    for (key, poly, point), (root, ev, proof, res) in zip(reqs, results):
        ek, D, nv = key
        desc = oracle.make_desc(ek, D, 0, nv, 1 << min(nv, 14) if ek else 1024)
        ro, po, eo, _ = oracle.commit_prove(desc, poly, 1, point)
        assert root == ro and proof == po and ev[:len(eo)] == eo
