#!/usr/bin/env python3
"""Record golden HMC chains with the reference Qlattice library itself into
reference_chains.json.

Each chain is run by oracle/_ref/ref_chain (the reference C++ library built
from its own sources by oracle/ref/Makefile): the Python driver
run_hmc_pure_gauge of hmc.pyx:190-216, step for step, through the
reference's set_gm_force / gf_evolve / gm_hamilton_node / gf_hamilton_node /
unitarize and the Python form of metropolis_accept.  The chains are chosen so
that the Metropolis step decides both ways with probabilities well inside
(0, 1): the tests then compare every decision, delta_h and plaquette of the
CUDA library's chain with the reference's.

    python tests/golden/make_chain_goldens.py      (after oracle/_ref is built)
"""

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# name -> (lattice, beta, c1, integrator, n_step, md_time, seed, start, n_traj, n_always)
CHAINS = {
    # the small configuration's lattice and action: 8^4 Wilson beta = 5.5, leapfrog.  From a unit start the
    # first trajectories are accepted downhill; from trajectory ~14 on the decisions are random.
    "wilson_8x4_leapfrog": ((8, 8, 8, 8), 5.5, 0.0, "leapfrog", 12, 1.0, "b200-c1-8x4-wilson", "unit", 24, 0),
    # the benchmark's action and integrator on a small lattice: Iwasaki beta = 2.13, force-gradient,
    # hot start at scale 0.3; six forced acceptances, then twelve Metropolis decisions.
    "iwasaki_8x4_fg": ((8, 8, 8, 8), 2.13, -0.331, "fg", 6, 1.0, "b200-chain-8x4-iwasaki", "hot:0.3:1", 18, 6),
}


def run_chain(exe, spec, threads):
    ts, beta, c1, integ, n_step, md_time, seed, start, n_traj, n_always = spec
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), q_verbose="-1")
    out = subprocess.run([exe, *map(str, ts), repr(beta), repr(c1), integ, str(n_step), repr(md_time), seed, start,
                          str(n_traj), str(n_always)], capture_output=True, text=True, env=env, check=True).stdout
    rows = [json.loads(ln) for ln in out.splitlines() if ln.startswith("{\"")]
    head, trajs = rows[0], rows[1:]
    for r in trajs:
        r.pop("seconds", None)
    return {"total_site": list(ts), "beta": beta, "c1": c1, "integrator": integ, "n_step": n_step,
            "md_time": md_time, "seed": seed, "start": start, "n_traj": n_traj, "n_always": n_always,
            "plaq0": head["plaq0"], "rows": trajs}


def main():
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_chain")
    if not os.path.exists(exe):
        sys.exit("oracle/_ref/ref_chain is not built (oracle/ref/Makefile)")
    out = {"source": "oracle/_ref/ref_chain: the reference library's own functions, run_hmc_pure_gauge "
                     "(hmc.pyx:190-216) semantics, Python metropolis_accept (hmc.pyx:139-155)",
           "chains": {name: run_chain(exe, spec, os.cpu_count() or 1) for name, spec in CHAINS.items()}}
    with open(os.path.join(HERE, "reference_chains.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    for name, c in out["chains"].items():
        flags = "".join("A" if r["flag"] else "r" for r in c["rows"])
        print(name, flags)


if __name__ == "__main__":
    main()
