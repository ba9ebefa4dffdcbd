"""The job engine (eplace_server_*): jobs of uneven size run concurrently on
one GPU and each result equals the job run alone; admission respects the
device-memory budget; contexts are reused; a failing job does not disturb
the others."""

import time

import numpy as np
import pytest

import eisenjoch_b200 as E

pytestmark = pytest.mark.gpu

SPECS = [
    E.SynthSpec(seed=1001, num_cells=2000, num_nets=2200, num_pads=120, width=64, height=64),
    E.SynthSpec(seed=1002, num_cells=9000, num_nets=9900, num_pads=300, width=192, height=192, bins_x=64, bins_y=64,
                cluster_size=64, macro_fraction=0.05),
    E.SynthSpec(seed=1003, num_cells=4500, num_nets=4950, num_pads=200, width=96, height=96),
    E.SynthSpec(seed=1004, num_cells=20000, num_nets=22000, num_pads=500, width=320, height=320, bins_x=64,
                bins_y=64, cluster_size=64, macro_fraction=0.05),
    E.SynthSpec(seed=1005, num_cells=1200, num_nets=1320, num_pads=80, width=48, height=48),
    E.SynthSpec(seed=1006, num_cells=6000, num_nets=6600, num_pads=250, width=128, height=128, bins_x=64,
                bins_y=64),
    # FFT transforms of different lengths launched side by side
    E.SynthSpec(seed=1007, num_cells=12000, num_nets=13200, num_pads=400, width=256, height=256, bins_x=128,
                bins_y=128, cluster_size=64),
    E.SynthSpec(seed=1008, num_cells=30000, num_nets=33000, num_pads=600, width=512, height=512, bins_x=256,
                bins_y=256, cluster_size=64, macro_fraction=0.05),
]
CFG = E.ElectroPlaceCfg(max_iters=120)
OPTS = E.RunOptions(field_mode=1)


def same(a, b):
    assert a.hpwl == b.hpwl and a.iters == b.iters and a.best_iter == b.best_iter
    assert a.converged == b.converged
    assert np.array_equal(a.bel_tile, b.bel_tile)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
    assert a.trajectory == b.trajectory


@pytest.fixture(scope="module")
def designs():
    out = []
    for sp in SPECS:
        nl, chip = E.synth_netlist(sp)
        out.append((nl, chip, E.place_electro(nl, chip, CFG, OPTS)))
    return out


@pytest.mark.parametrize("max_jobs", [4, 1])
def test_results_in_the_mix_equal_alone(designs, max_jobs):
    with E.JobServer(max_jobs=max_jobs, opts=OPTS) as srv:
        ids = [srv.submit(nl, chip, CFG) for nl, chip, _ in designs]
        for jid, (nl, chip, alone) in zip(ids, designs):
            r, info = srv.wait(jid)
            same(r, alone)
            assert info.latency_seconds >= info.run_seconds > 0
        st = srv.stats()
        assert st["finished"] == len(designs) and st["running"] == 0 and st["queued"] == 0
        # at most twice max_jobs contexts are kept (one per bin grid of the mix)
        assert st["contexts"] <= 2 * max_jobs


def test_context_reloaded_across_bin_grids_equals_fresh(designs):
    """One context re-loaded with designs whose bin grids differ (64^2 ->
    96^2 -> 64^2 -> 48^2) gives each design the result of a fresh context.
    On 64-multiple grids the FP32 transform is a split-K cluster launch, on
    the others a plain one; the interval graph of a context must be made
    anew, not updated in place, when the grid changes."""
    order = [0, 2, 1, 4]
    with E.PlacementContext(designs[order[0]][0], designs[order[0]][1]) as c:
        for k, d in enumerate(order):
            nl, chip, _ = designs[d]
            if k:
                c.load(nl, chip)
            got = c.run(CFG, OPTS)
            with E.PlacementContext(nl, chip) as fresh:
                same(got, fresh.run(CFG, OPTS))


def test_admission_budget_runs_one_at_a_time(designs):
    # any two jobs exceed the budget; a job larger than the budget runs alone
    fp = min(E.footprint(nl, chip) for nl, chip, _ in designs)
    with E.JobServer(max_jobs=8, hbm_budget=fp + 1, opts=OPTS) as srv:
        ids = [srv.submit(nl, chip, CFG) for nl, chip, _ in designs]
        peak = 0
        pending = set(ids)
        res = {}
        while pending:
            peak = max(peak, srv.stats()["running"])
            for jid in list(pending):
                got = srv.wait(jid, timeout_ms=0)
                if got is not None:
                    res[jid] = got[0]
                    pending.discard(jid)
            time.sleep(0.001)
        assert peak <= 1
        for jid, (_, _, alone) in zip(ids, designs):
            same(res[jid], alone)


def test_failing_job_does_not_disturb_others(designs):
    nl, chip, alone = designs[0]
    full = E.Netlist(num_cells=17, net_offsets=np.array([0, 2], np.uint32), pin_cell=np.array([0, 1], np.uint32))
    with E.JobServer(max_jobs=3, opts=OPTS) as srv:
        a = srv.submit(nl, chip, CFG)
        bad = srv.submit(full, E.Chip(4, 4), E.ElectroPlaceCfg(max_iters=10))
        b = srv.submit(nl, chip, CFG)
        with pytest.raises(E.PlacerError):
            srv.wait(bad)
        same(srv.wait(a)[0], alone)
        same(srv.wait(b)[0], alone)
        with pytest.raises(E.EplaceError):
            srv.submit(E.Netlist(num_cells=2, net_offsets=np.array([0, 2], np.uint32),
                                 pin_cell=np.array([0, 9], np.uint32)), E.Chip(4, 4))
