"""Generate the long-trajectory fixtures of the full-size workloads from the
reference itself (libgrid's CPU sources compiled unchanged into oracle/_ref
by oracle/build_ref.sh, OpenMP on all host cores).

  gp256_traj.npz  Gross-Pitaevskii FFT split operator, 256^3, step 0.5 bohr,
                  4 amu, 8 seeded wells (workloads.gp_wells seed 2), g 0.0025,
                  dt 1 au, 1000 steps
  cn192_traj.npz  Gross-Pitaevskii Crank-Nicolson, 192^3 Dirichlet, step
                  0.3 bohr, 4 amu, workloads.cn_wells seed 3, g 0.001,
                  dt 0.5 au, 500 steps

At each checkpoint the file holds psi at a fixed seeded subset of grid
points (oracle.refsteps.sample_indices), the norm, the kinetic energy
(FFT method for the split operator, finite differences for CN), <V_ext>,
the interaction energy (g/2) int |psi|^4, and sum(psi) over the full grid.
Inputs are rebuilt from libgrid_b200.workloads, so only outputs are saved.
A 1000-step 256^3 trajectory takes about 20 minutes on 8 cores.

    python tests/golden/make_baseline_traj.py [gp256] [cn192]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libgrid_b200 import capi, workloads  # noqa: E402
from oracle import pyoracle, refsteps  # noqa: E402

NSAMPLE = 16384

CASES = {
    "gp256": dict(kind="gp", shape=(256, 256, 256), step=0.5, g=0.0025, dt=1.0, seed=2, steps=1000,
                  checkpoints=(50, 500, 1000)),
    "cn192": dict(kind="cn", shape=(192, 192, 192), step=0.3, g=0.001, dt=0.5, seed=3, steps=500,
                  checkpoints=(20, 100, 500)),
}


def run_case(ref, name):
    c = CASES[name]
    mass = 4.0 / capi.GRID_AUTOAMU
    if c["kind"] == "gp":
        psi0, v = workloads.gp_wells(c["shape"], c["step"], c["g"], seed=c["seed"])
        st = refsteps.GPStepper(ref, psi0, v, c["step"], mass, c["g"], c["dt"])
    else:
        psi0, v = workloads.cn_wells(c["shape"], c["step"], c["g"], seed=c["seed"])
        st = refsteps.CNGPStepper(ref, psi0, v, c["step"], mass, c["g"], c["dt"])
    idx = refsteps.sample_indices(psi0.size, NSAMPLE)
    out = {"idx": idx}

    def record(s):
        psi = st.psi()
        ob = st.observables(psi)
        out["psi_%d" % s] = psi.ravel()[idx]
        out["sum_%d" % s] = np.sum(psi)
        for k, val in ob.items():
            out["%s_%d" % (k, s)] = val

    record(0)
    t0 = time.time()
    for s in range(1, c["steps"] + 1):
        st.step_once()
        if s in c["checkpoints"]:
            record(s)
            print("%s: step %d (%.0f s)" % (name, s, time.time() - t0), flush=True)
    meta = {"meta_" + k: np.asarray(val) for k, val in c.items() if k != "kind"}
    meta["meta_mass"] = np.asarray(mass)
    np.savez_compressed(os.path.join(HERE, name + "_traj.npz"), **out, **meta)
    print("wrote", name, flush=True)
    st.free()


def main(argv):
    ref = pyoracle.reference(len(os.sched_getaffinity(0)))
    for name in argv or list(CASES):
        run_case(ref, name)


if __name__ == "__main__":
    main(sys.argv[1:])
