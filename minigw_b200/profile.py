"""Run a few solves of a named synthetic workload, for profilers (ncu launch lists and metrics).

    python -m minigw_b200.profile [--workload cfg3] [--precision fp64|mixed|mixed-refined]
                                  [--ingest states|block] [--warmup 1] [--solves 1]

`--ingest states` loads the system with gwb200_load_system_states (V_ph and the states' panel rows
copied from the host, as bench.py does); `--ingest block` with gwb200_load_system (the (pq|o.)
block resident, V_ph and the panel rows gathered on the device by k_gather_vph / k_gather_panel).
The load runs once, then `warmup` untimed solves and `solves` profiled ones, each one whole
gwb200_run_g0w0.  Prints one line per solve: device times of the phases and the launch count.
"""
from __future__ import annotations

import argparse


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cfg3")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "mixed-refined"])
    ap.add_argument("--ingest", default="states", choices=["states", "block"])
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--solves", type=int, default=1)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()

    from minigw_b200 import B200Backend
    from minigw_b200.synthetic import WORKLOADS, make_input_on_device

    wl = WORKLOADS[args.workload]
    inp = make_input_on_device(wl.nmo, wl.nocc, seed=args.seed, device=0, pin=True)
    states = list(wl.states)
    with B200Backend(0) as be:
        be.load_system(inp, states if args.ingest == "states" else None)
        for _ in range(args.warmup):
            be.run_g0w0(wl.nfreq, wl.npade, states, precision=args.precision)
        for i in range(args.solves):
            st = be.run_g0w0(wl.nfreq, wl.npade, states, precision=args.precision)["stats"]
            print(f"solve {i}: total {st['device_ms_total']:.3f} ms, gather {st['device_ms_gather']:.3f} ms, "
                  f"screening {st['device_ms_screening']:.3f} ms, contract {st['device_ms_contract']:.3f} ms, "
                  f"launches {st['kernel_launches']}", flush=True)


if __name__ == "__main__":
    main()
