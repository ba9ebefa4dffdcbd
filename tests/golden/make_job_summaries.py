"""Runs the FP64 CPU oracle on the benchmark workloads and records each
job's outcome in job_summaries.json (iterations, convergence, final
legalised HPWL, best checkpoint, overlap trajectory at the checkpoints).

    python tests/golden/make_job_summaries.py [workload:field_mode ...]

field_mode 0 is the reference's field formula, 1 the potential-gradient
extension.  The records pin the GPU full-run parity tests (final HPWL within
0.5%, same convergence) and give bench.py's CPU arm the iteration count of a
job.  Deterministic: same inputs, same numbers.
"""

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import eisenjoch_b200 as E  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

DEFAULT = ["electro_5k_128:0", "electro_5k_128:1", "electro_200k_1024:1"]


def main(items):
    path = os.path.join(HERE, "job_summaries.json")
    out = {}
    if os.path.exists(path):
        with open(path) as f:
            out = json.load(f)
    for item in items:
        name, mode = item.split(":")
        mode = int(mode)
        nl, chip, cfg = E.workload(name)
        t0 = time.perf_counter()
        st, r = Oracle(nl, chip).place(cfg, field_mode=mode)
        dt = time.perf_counter() - t0
        key = name if mode == 1 else name + ":reference_field"
        out[key] = dict(
            status=st, iters=r["iters"], converged=r["converged"], hpwl=r["hpwl"], best_iter=r["best_iter"],
            field_mode=mode, cpu_seconds=round(dt, 2),
            checkpoints=[dict(iter=t["iter"], hpwl=t["hpwl"], overlap=round(t["overlap"], 6))
                         for t in r["trajectory"]],
        )
        print(key, {k: v for k, v in out[key].items() if k != "checkpoints"}, flush=True)
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or DEFAULT)
