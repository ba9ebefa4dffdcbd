"""Runs the FP64 CPU oracle on the benchmark workloads and records each
job's outcome in job_summaries.json (iterations, convergence, final
legalised HPWL, best checkpoint, the overlap and HPWL at every checkpoint,
the first iteration whose WA gradient was not finite).

    python tests/golden/make_job_summaries.py [workload:field_mode[:wa_mode] ...]

field_mode 0 is the reference's field formula, 1 the potential-gradient
extension.  wa_mode 0 is the reference's WA exponent shift (the pin mean,
which overflows FP64 on nets wider than about 1,400 sites at wl_coeff 0.5),
1 the per-net max / min shift (extension: the same function; the shift the
CUDA kernel uses).  Record keys: the workload name, + ":reference_field"
for field_mode 0, + ":stable_wa" for wa_mode 1.  The inputs come from the
oracle's own copy of the generator (equal to the product's, checked by
tests/test_host_cpu.py).  Deterministic: same inputs, same numbers.
"""

import json
import math
import os
import sys
import time
from types import SimpleNamespace

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Cfg, Oracle, synth  # noqa: E402

DEFAULT = ["electro_5k_128:0", "electro_5k_128:1", "electro_200k_1024:1", "electro_200k_1024:0",
           "electro_800k_2048:1:0", "electro_800k_2048:1:1"]


def workload(name):
    with open(os.path.join(ROOT, "eisenjoch_b200", "workloads.json")) as f:
        w = json.load(f)[name]
    spec = dict(bins_x=0, bins_y=0, cluster_size=32, locality=0.6, macro_fraction=0.0, macro_min=2, macro_max=8)
    spec.update(w["spec"])
    nl, chip = synth(SimpleNamespace(**spec))
    return nl, chip, Cfg(**w["cfg"])


def key_of(name, field_mode, wa_mode):
    return name + ("" if field_mode == 1 else ":reference_field") + (":stable_wa" if wa_mode == 1 else "")


def main(items):
    path = os.path.join(HERE, "job_summaries.json")
    out = {}
    if os.path.exists(path):
        with open(path) as f:
            out = json.load(f)
    for item in items:
        parts = item.split(":")
        name, mode = parts[0], int(parts[1])
        wa = int(parts[2]) if len(parts) > 2 else 0
        nl, chip, cfg = workload(name)
        t0 = time.perf_counter()
        st, r = Oracle(nl, chip).place(cfg, field_mode=mode, wa_mode=wa, want_trace=True)
        dt = time.perf_counter() - t0
        trace = r["overlap_trace"]
        bad = [i for i, v in enumerate(trace) if not math.isfinite(v)]
        key = key_of(name, mode, wa)
        out[key] = dict(
            status=st, iters=r["iters"], converged=r["converged"], hpwl=r["hpwl"], best_iter=r["best_iter"],
            field_mode=mode, wa_mode=wa, cpu_seconds=round(dt, 2),
            first_nonfinite_overlap_iter=bad[0] if bad else None,
            first_nonfinite_grad_iter=None if r["first_nonfinite_grad_iter"] < 0 else r["first_nonfinite_grad_iter"],
            checkpoints=[dict(iter=t["iter"], hpwl=t["hpwl"], overlap=round(t["overlap"], 6))
                         for t in r["trajectory"]],
        )
        print(key, {k: v for k, v in out[key].items() if k != "checkpoints"}, flush=True)
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or DEFAULT)
