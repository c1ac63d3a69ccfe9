"""How hard hamalloc probes, launch by launch: the probe counters of an
instrumented build (-DHA_PROBE_STATS; see csrc/ha_stamp.cuh ProbeStat) over
the reference-form phase workload's 16 B x1 private row -- 1,048,576 threads,
32 iterations per launch, 16 launches, 512 MiB pool (halloc's
phase-throughput -l1 -s16 -i32 -t16) -- started the way halloc's own program
starts it: one warm-up launch of 512 threads and one iteration.

    python -m halloc_b200.build -DHA_PROBE_STATS   # replaces the library in place
    python -m halloc_b200.probestats [--runs 4] [--no-surge]
    python -m halloc_b200.build -DHA_PROBE_STATS=0 # back to the normal build (any -D forces a rebuild)

Printed per run and launch: the launch time, and per allocation the first
probes that missed, the look-ahead rounds, the reservation atomics of the
look-ahead, and the head replacements asked for; per run the size-0 surge
level reached.  A normal build has no counters and this tool says so.
"""
from __future__ import annotations

import argparse
import ctypes

import numpy as np

from . import load

NSTATS = 9  # ProbeStat entries read (kPsCount)


def run(runs: int, surge: bool) -> list:
    import torch

    import halloc_b200 as H
    from halloc_b200.workloads import group_seeds

    lib = load()
    if not hasattr(lib, "ha_probe_stats_c"):
        raise SystemExit("the loaded library has no probe counters: build it with "
                         "python -m halloc_b200.build -DHA_PROBE_STATS")
    out = (ctypes.c_ulonglong * NSTATS)()

    def counters():
        if lib.ha_probe_stats_c(out, 1) != 0:
            raise RuntimeError("ha_probe_stats_c failed")
        return list(out)

    probs = H.phase_ref_probabilities(0.95, 0.05, 0.91)
    n, size, niters, ntries, warm = 1 << 20, 16, 32, 16, 512
    H.set_surge(surge)
    results = []
    try:
        for r in range(runs):
            H.init(H.HallocOpts(memory=512 << 20))
            acc = torch.zeros(4, dtype=torch.int64, device="cuda")
            ws = torch.tensor(group_seeds(warm, 32, 0x5EED).view(np.int32), device="cuda")
            H.phase_ref_run(warm, 1, 1, 1, probs, size, size, ws,
                            torch.zeros(warm, dtype=torch.int64, device="cuda"),
                            torch.zeros(warm, dtype=torch.int32, device="cuda"), acc)
            states = torch.tensor(group_seeds(n, 32, 0x5EED).view(np.int32), device="cuda")
            slots = torch.zeros(n, dtype=torch.int64, device="cuda")
            ctrs = torch.zeros(n, dtype=torch.int32, device="cuda")
            counters()
            launches = []
            for t in range(ntries):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                H.phase_ref_step(n, 1, t, niters, probs, size, size, states, slots, ctrs, acc)
                e1.record()
                e1.synchronize()
                c = counters()
                a = max(c[0], 1)
                launches.append({"ms": e0.elapsed_time(e1), "allocs": c[0],
                                 "first_miss": c[1] / a, "rounds": c[3] / a,
                                 "reserve": c[4] / a, "head_requests": c[5]})
            H.phase_ref_step(n, 1, 0, niters, probs, size, size, states, slots, ctrs, acc,
                             rest=True)
            torch.cuda.synchronize()
            st = H.stats()
            results.append({"run": r, "surge_level": st["surge_level"][0],
                            "surge_changes": st["n_surge_changes"],
                            "status": H.status(), "launches": launches})
            H.shutdown()
    finally:
        H.set_surge(None)
    return results


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--runs", type=int, default=4)
    ap.add_argument("--no-surge", action="store_true", help="one head per size (ha_set_surge_c(0))")
    args = ap.parse_args()
    for res in run(args.runs, not args.no_surge):
        ms = [x["ms"] for x in res["launches"]]
        print(f"run {res['run']}: {sum(ms):.1f} ms over {len(ms)} launches, size-0 surge level "
              f"{res['surge_level']} ({res['surge_changes']} changes), status {res['status']}")
        for t, x in enumerate(res["launches"]):
            if t < 3 or t % 4 == 3:
                print(f"  launch {t:2d}: {x['ms']:.2f} ms  first-probe misses {x['first_miss']:.3f}"
                      f"  look-ahead rounds {x['rounds']:.3f}  reservations {x['reserve']:.3f}"
                      f"  head requests {x['head_requests']}")


if __name__ == "__main__":
    main()
