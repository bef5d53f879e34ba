"""The oracle's HMC chain against chains recorded with the reference library
itself (tests/golden/reference_chains.json, made by make_chain_goldens.py from
oracle/_ref/ref_chain): every Metropolis decision, delta_h and plaquette.

The oracle draws its Gaussian momenta with the C library's log here (log
mode 0), as the reference does, so it follows the reference's arithmetic.
To keep the CPU suite short, the force-gradient chain is replayed for its
first trajectories only; the GPU tests replay both chains in full."""

import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def chains():
    with open(os.path.join(HERE, "golden", "reference_chains.json")) as f:
        return json.load(f)["chains"]


def oracle_chain(O, c, n_traj):
    ts = tuple(c["total_site"])
    rs = O.RngState(c["seed"])
    gf = O.new_field(ts)
    if c["start"] == "unit":
        O.set_unit(gf, ts)
    else:
        _, sigma, n = c["start"].split(":")
        O.gf_set_rand(gf, ts, rs.split("gf-init"), float(sigma), int(n))
    integ = {"fg": "force-gradient", "leapfrog": "leapfrog"}[c["integrator"]]
    out = []
    for traj in range(1, n_traj + 1):
        flag, dh = O.run_hmc_pure_gauge(gf, ts, c["beta"], c["c1"], traj, rs.split("hmc"), n_step=c["n_step"],
                                        md_time=c["md_time"], is_always_accept=traj <= c["n_always"],
                                        integrator=integ)
        out.append((flag, dh, O.gf_avg_plaq(gf, ts)))
    return out


@pytest.mark.parametrize("name,n_traj", [("wilson_8x4_leapfrog", 24), ("iwasaki_8x4_fg", 3)])
def test_oracle_reproduces_reference_chain(oracle, chains, name, n_traj):
    c = chains[name]
    rows = c["rows"][:n_traj]
    got = oracle_chain(oracle, c, n_traj)
    decisions = [r["flag"] for r in c["rows"]]
    assert 0 < sum(decisions) < len(decisions)  # the recorded chain decides both ways
    for r, (flag, dh, plaq) in zip(rows, got):
        assert int(flag) == r["flag"], (name, r["traj"])
        assert abs(dh - r["delta_h"]) <= 1e-8, (name, r["traj"], dh, r["delta_h"])
        assert abs(plaq - r["plaq"]) <= 1e-14, (name, r["traj"], plaq, r["plaq"])
