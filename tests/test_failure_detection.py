"""Failure detection of the tensor-core kernels without a GPU fault: every
mbarrier wait in them is bounded, and a wait that runs out is reported through
the device status word.  The GPU test makes a wait run out on purpose (a probe
kernel whose barrier nothing arrives on), reads the code, and checks that the
context still commits correctly afterwards."""
import ctypes as C
import time

import numpy as np
import pytest

from util import binary_evals, desc_for, params_for


def test_selftest_rejects_null_arguments(zipgpu):
    v = C.c_uint32()
    assert zipgpu.lib().zg_selftest_bounded_wait(None, C.byref(v)) != 0


@pytest.mark.gpu
def test_bounded_wait_runs_out_and_is_reported(zipgpu, oracle, ctx, rng):
    t0 = time.perf_counter()
    code = ctx.selftest_bounded_wait()
    elapsed = time.perf_counter() - t0
    assert code == 4  # the probe's timeout code
    assert 0.1 < elapsed < 60  # the wait gave up after its limit, not at once
    # the word was cleared and the context is usable: a commit still matches the oracle
    nv, D, L = 14, 32, 1 << 12
    pp = params_for(zipgpu, 1, D, 0, nv, L, ctx=ctx)
    ev = binary_evals(rng, 1 << nv, D)
    _, comm = zipgpu.ZipPlus.commit(pp, [ev])
    assert comm.root == oracle.commit(desc_for(1, D, 0, nv, L), ev, 1)
    # a second probe reports again (the word starts from zero each time)
    assert ctx.selftest_bounded_wait() == 4
