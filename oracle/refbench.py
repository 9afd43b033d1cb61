"""ORACLE timing leg (test infrastructure; run only by bench.py's CPU-baseline
leg and by `bench.py --impl reference`).

Times the reference's own CPU path for the Gross-Pitaevskii split-operator
step (the reference's CPU sources compiled into oracle/_ref with the
project's FFTW stand-in), composed from the reference's exported primitives
exactly as the GPU path's definition states:
    FFT, K(dt/2), IFFT/N, rho = |psi|^2, V = V_ext + g rho,
    grid_wf_propagate_potential(dt), FFT, K(dt/2), IFFT/N.
Falls back to the project's C restatement (kind "port") when oracle/_ref is
absent.  Prints one JSON object.

    python -m oracle.refbench --size 256 --steps 2 --warmup 1
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args(argv)

    import numpy as np

    from libgrid_b200 import capi, workloads
    from oracle import pyoracle, refsteps

    threads = a.threads or len(os.sched_getaffinity(0))
    shape, step, g, dt = (a.size,) * 3, 0.5, 0.0025, 1.0
    mass = 4.0 / capi.GRID_AUTOAMU
    psi0, v = workloads.gp_wells(shape, step, g, seed=2)
    kind = "reference" if pyoracle.reference_available() else "port"
    if kind == "reference":
        stepper = refsteps.GPStepper(pyoracle.reference(threads), psi0, v, step, mass, g, dt)
        one_step = stepper.step_once

    else:
        os.environ.setdefault("OMP_NUM_THREADS", str(threads))
        R = pyoracle.restatement()
        state = {"psi": psi0.copy()}
        vr = workloads.padded(v)

        def one_step():
            state["psi"] = R.fft_step(state["psi"], step, mass, dt, vr=vr, g=g)

    for _ in range(a.warmup):
        one_step()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        one_step()
    dt_s = time.perf_counter() - t0
    print(
        json.dumps(
            {
                "kind": kind,
                "steps": a.steps,
                "seconds": dt_s,
                "steps_per_s": a.steps / dt_s,
                "cores": threads,
                "size": a.size,
                "sample": "%d GP split-operator steps on %d^3 after %d warm-up" % (a.steps, a.size, a.warmup),
            }
        )
    )
    return 0


if __name__ == "__main__":
    sys.exit(main())
