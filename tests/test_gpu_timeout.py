"""The failure path of a bounded device wait, made to happen on purpose.

Every spin wait of the device code is bounded; when one runs out, the
kernel records an error and leaves, and the host reports EPLACE_ERR_TIMEOUT
instead of hanging.  Here the step kernel's grid barrier is started with
one phantom arrival (eplace_stage_barrier_timeout), so one block waits for
an arrival that never comes and must give up after the limit.  Nothing
faults or traps: the wait simply runs out.  Checked: the status, that the
call ends within a bound of the limit, and that the same context then runs
a placement identical to the one it ran before."""

import time

import numpy as np
import pytest

import eisenjoch_b200 as E
from eisenjoch_b200 import _abi

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_the_context_recovers():
    nl, chip, cfg = E.workload("electro_5k_128")
    cfg.max_iters = 40
    opts = E.RunOptions(field_mode=1)
    L = _abi.lib()
    with E.PlacementContext(nl, chip) as ctx:
        before = ctx.run(cfg, opts)
        for limit_us in (2000, 20000):
            t0 = time.perf_counter()
            st = L.eplace_stage_barrier_timeout(ctx.handle, limit_us, 1)
            dt = time.perf_counter() - t0
            assert st == _abi.EPLACE_ERR_TIMEOUT, st
            # a few barriers of the one step can each wait up to the limit
            assert dt < 1.0 + 8 * limit_us * 1e-6, dt
        after = ctx.run(cfg, opts)
    assert after.hpwl == before.hpwl and after.iters == before.iters
    assert np.array_equal(after.bel_tile, before.bel_tile)
    assert np.array_equal(after.x, before.x)
    assert after.trajectory == before.trajectory


def test_wait_limit_option_leaves_a_normal_run_unchanged():
    """A run with a short but sufficient wait limit gives the default run's
    result (the limit only bounds waits that never end)."""
    nl, chip, cfg = E.workload("electro_5k_128")
    cfg.max_iters = 40
    a = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=1))
    b = E.place_electro(nl, chip, cfg, E.RunOptions(field_mode=1, wait_limit_us=200000))
    assert a.hpwl == b.hpwl and np.array_equal(a.bel_tile, b.bel_tile) and a.trajectory == b.trajectory


def test_barrier_timeout_entry_rejects_bad_arguments():
    nl, chip, _ = E.workload("electro_5k_128")
    L = _abi.lib()
    with E.PlacementContext(nl, chip) as ctx:
        assert L.eplace_stage_barrier_timeout(ctx.handle, 0, 1) == _abi.EPLACE_ERR_INVALID
        assert L.eplace_stage_barrier_timeout(ctx.handle, 1000, 0) == _abi.EPLACE_ERR_INVALID
        assert L.eplace_stage_barrier_timeout(ctx.handle, 1000, 1 << 30) == _abi.EPLACE_ERR_INVALID
