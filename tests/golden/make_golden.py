"""Regenerate the committed golden fixtures under tests/golden/ (run in a container that has
the reference tree; the fixtures then travel with the repository).

    MINIGW_REF_ROOT=<reference tree> python tests/golden/make_golden.py [--ref-root <reference tree>]

1. h2o/: the reference's own H2O regression vectors, copied verbatim from
   regression_tests/h2o_serial/ -- gw_input.h5 (the input), E_c_before_Pade.out (200 complex
   Sigma_c(iw) of state 5), gw.out (summary row) -- and E_c.out subsampled to every 20th line.
2. cfg1_reference.npz: outputs of the reference itself (oracle/_ref/libgwref.so, the
   reference's sources compiled unmodified) on the seeded synthetic config-1 input
   (nmo=24, nocc=5, seed 0, 200 frequencies, 16 Pade parameters, state index 4):
   Sigma_c(iw) row, Sigma_x diagonal, QP energy, grid, and the screened forms q[f, k] at
   eight frequencies (reference backend).
"""
from __future__ import annotations

import argparse
import os
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("MINIGW_REF_ROOT"),
                    help="the reference tree (default: $MINIGW_REF_ROOT)")
    args = ap.parse_args()
    if not args.ref_root:
        ap.error("give --ref-root or set MINIGW_REF_ROOT")
    src = Path(args.ref_root) / "regression_tests" / "h2o_serial"
    dst = HERE / "h2o"
    dst.mkdir(exist_ok=True)
    for name in ("gw_input.h5", "E_c_before_Pade.out", "gw.out"):
        shutil.copyfile(src / name, dst / name)
    lines = (src / "E_c.out").read_text().splitlines()
    (dst / "E_c_every20.out").write_text("\n".join(lines[::20]) + "\n")

    import oracle
    from minigw_b200.synthetic import WORKLOADS, make_workload_input

    oracle.build(args.ref_root)
    ref = oracle.Ref()
    w = WORKLOADS["cfg1"]
    inp = make_workload_input(w, seed=0)
    out = ref.run_g0w0(inp, w.nfreq, w.npade, w.states[0], backend="reference")
    om, wt = ref.grid(w.nfreq)
    fsel = np.array([0, 1, 17, 50, 99, 150, 198, 199])
    q = ref.forms(inp, om[fsel], list(w.states), backend="reference")
    np.savez(HERE / "cfg1_reference.npz", sigma_row=out["sigma"][w.states[0]], qp=out["qp"][w.states[0]],
             sigma_x_diag=np.diag(out["sigma_x"]).copy(), omegas=om, weights=wt, forms_freq_index=fsel,
             forms=q[:, 0, :], seed=0, nmo=w.nmo, nocc=w.nocc, state=w.states[0])
    print("wrote", dst, HERE / "cfg1_reference.npz")


if __name__ == "__main__":
    main()
