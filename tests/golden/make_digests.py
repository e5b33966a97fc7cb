"""Make the committed digests of the oracle's final states at full size.

CPU only.  For every pinned workload (``tests/digests.py``: the 2D P7 line
source at 100^2 to t_final = 1 (67 steps), the 2D P39 checkerboard lattice at
350^2 to t_final = 3.2 (321 steps), the 3D P9 point source at 128^3 to
t_final = 0.75 (96 steps), eight instances of the seeded batched sweep for 200
steps each, and the 2D P15 adjoint problem at 200^2 for 400 steps with the
constant and the true sigma_a) this runs the oracle -- the numpy restatement
of starmap_solver.m for the setup and hook evaluation, its C restatement
(oracle/loop_ref.c, OpenMP, no FMA contraction) for every step -- and writes
``tests/golden/<name>.json``: the step count, the final time and the digests
of every component of the output struct (``mom_output = 'all'``) or of the
state after a fixed number of steps.

    python tests/golden/make_digests.py [name ...]     # default: all

The largest two take tens of minutes on 8 host cores.
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

import digests  # noqa: E402
from oracle import c_oracle  # noqa: E402
from starmap_b200 import starmap_init  # noqa: E402


def make(name: str) -> dict:
    prob, steps = digests.full_size_prob(name)
    par = starmap_init(prob)
    t0 = time.perf_counter()
    res = c_oracle.run(par, nthreads=0, max_steps=steps)
    secs = time.perf_counter() - t0
    if steps is None:
        comps = [o["U"] for o in res.output]
        what = "output struct U of every moment at t_final"
    else:
        comps = res.U
        what = f"state after {steps} steps"
    return {"workload": name, "what": what, "steps": res.step_count, "t": float(res.t).hex(),
            "dt": float(res.dt).hex(), "oracle": "numpy setup + C steps (oracle/loop_ref.c)",
            "oracle_seconds": round(secs, 1), "components": digests.state_digest(comps)}


def main(names):
    names = names or digests.workload_names()
    for name in names:
        out = os.path.join(HERE, name + ".json")
        rec = make(name)
        comps = rec.pop("components")
        with open(out, "w") as f:
            # one component per line
            f.write(json.dumps(rec)[:-1] + ', "components": [\n')
            f.write(",\n".join(json.dumps(c, separators=(",", ":")) for c in comps))
            f.write("\n]}\n")
        print(f"{name}: {rec['steps']} steps, {len(comps)} components, "
              f"{rec['oracle_seconds']} s -> {os.path.relpath(out, ROOT)}", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
