"""Host-side fault injection (zg_debug_fail_allocation): a device allocation is
made to fail on the host, before any CUDA call, and the error must come back
through each entry point's status (the plain commit, the batched commit, a
server request through zg_server_wait, with the server's fail-all path for a
group) while the context and the server stay usable: the next calls give the
same bytes as the oracle or the plain path.  No GPU fault is involved."""
import numpy as np
import pytest

from util import binary_evals, params_for

OOM = 6


def test_arming_and_disarming_needs_no_device(zipgpu):
    assert zipgpu.lib().zg_debug_fail_allocation(5) == 0
    assert zipgpu.lib().zg_debug_fail_allocation(0) == 0


@pytest.mark.gpu
def test_failed_allocation_in_a_plain_commit(zipgpu, oracle):
    ctx = zipgpu.Context(0)  # fresh: its first commit allocates
    try:
        nv, D, L = 12, 32, 1 << 12
        pp = params_for(zipgpu, 1, D, 0, nv, L, ctx=ctx)
        poly = binary_evals(np.random.default_rng(3), 1 << nv, D)
        zipgpu.lib().zg_debug_fail_allocation(1)
        with pytest.raises(zipgpu.ZipError) as e:
            zipgpu.ZipPlus.commit(pp, [poly])
        assert e.value.status == OOM and "injected" in str(e.value)
        zipgpu.lib().zg_debug_fail_allocation(0)
        hint, comm = zipgpu.ZipPlus.commit(pp, [poly])
        hint.close()
        assert comm.root == oracle.commit(oracle.make_desc(1, D, 0, nv, L), poly, 1)
        pp.close()
    finally:
        zipgpu.lib().zg_debug_fail_allocation(0)
        ctx.close()


@pytest.mark.gpu
def test_failed_allocation_in_a_batched_commit(zipgpu):
    ctx = zipgpu.Context(0)
    try:
        rng = np.random.default_rng(8)
        nvs = [10, 12, 12, 11]
        pps = [params_for(zipgpu, 1, 64, 0, nv, 1 << nv, ctx=ctx) for nv in nvs]
        polys = [binary_evals(rng, 1 << nv, 64) for nv in nvs]
        zipgpu.lib().zg_debug_fail_allocation(1)
        with pytest.raises(zipgpu.ZipError) as e:
            zipgpu.ZipPlus.commit_batch(pps, polys, ctx)
        assert e.value.status == OOM
        zipgpu.lib().zg_debug_fail_allocation(0)
        comms = zipgpu.ZipPlus.commit_batch(pps, polys, ctx)
        for pp, poly, c in zip(pps, polys, comms):
            h, alone = zipgpu.ZipPlus.commit(pp, [poly])
            h.close()
            assert c.root == alone.root
        for pp in pps:
            pp.close()
    finally:
        zipgpu.lib().zg_debug_fail_allocation(0)
        ctx.close()


@pytest.mark.gpu
def test_failed_lane_allocation_in_the_server(zipgpu):
    """The worker's first allocation (its lane's input buffer) fails: every
    request of that group completes with ZG_ERR_OOM through zg_server_wait (the
    fail-all path), and the server serves the following requests correctly."""
    ctx = zipgpu.Context(0)
    try:
        nv, D = 11, 32
        pp = params_for(zipgpu, 1, D, 0, nv, 1 << nv, ctx=ctx)
        rng = np.random.default_rng(4)
        reqs = [(binary_evals(rng, 1 << nv, D), [int(v) for v in rng.integers(-(2**30), 2**30, size=nv)])
                for _ in range(6)]
        srv = zipgpu.ZipServer(ctx, workers=1)
        zipgpu.lib().zg_debug_fail_allocation(1)
        ids = [srv.submit(pp, poly, pt) for poly, pt in reqs[:3]]
        failed = 0
        for i in ids:
            try:
                srv.wait(i)
            except zipgpu.ZipError as e:
                assert e.status == OOM
                assert "injected" in str(e)
                failed += 1
        assert failed >= 1
        zipgpu.lib().zg_debug_fail_allocation(0)
        for poly, pt in reqs[3:]:
            root, ev, proof, res = srv.wait(srv.submit(pp, poly, pt))
            assert res.status == 0
            assert (root, ev, proof) == zipgpu.ZipPlus.commit_prove(pp, [poly], pt)
        srv.close()
        pp.close()
    finally:
        zipgpu.lib().zg_debug_fail_allocation(0)
        ctx.close()
