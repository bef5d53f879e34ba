"""HMC chains on the GPU against chains recorded with the reference library
itself (tests/golden/reference_chains.json, made by make_chain_goldens.py from
oracle/_ref/ref_chain, the reference's own C++ functions under the Python
driver's semantics, hmc.pyx:139-216).

Both recorded chains decide both ways, with acceptance probabilities well
inside (0, 1), so identical decisions are a real check.  The FP64 form must
make every decision the reference makes, with delta_h within 1e-12 of the
Hamiltonian's size and the plaquette within 1e-12.  The GPU draws its
Gaussian momenta with a correctly rounded logarithm, which differs from the C
library's in about 0.08% of draws by one ulp: these tests bound the effect of
that on a whole chain.  The mixed form (FP32 molecular dynamics, FP64
Hamiltonians, FP64 re-unitarisation every 4 steps) is held to FP32 accuracy:
delta_h within 5e-3 (absolute, delta_h is O(1) here), the plaquette within
1e-6, and the same decisions."""

import json
import os

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
INTEG = {"fg": "force-gradient", "leapfrog": "leapfrog"}


@pytest.fixture(scope="module")
def chains():
    with open(os.path.join(HERE, "golden", "reference_chains.json")) as f:
        return json.load(f)["chains"]


def gpu_chain(q, c, precision):
    ts = tuple(c["total_site"])
    ga = q.GaugeAction(c["beta"], c["c1"])
    rs = q.RngState(c["seed"])
    gf = q.GaugeField(q.Geometry(ts))
    if c["start"] == "unit":
        q.set_unit(gf)
    else:
        _, sigma, n = c["start"].split(":")
        gf.set_rand(rs.split("gf-init"), float(sigma), int(n))
    assert abs(q.gf_avg_plaq(gf) - c["plaq0"]) <= 1e-14
    V = ts[0] * ts[1] * ts[2] * ts[3]
    out = []
    for traj in range(1, c["n_traj"] + 1):
        # the size of the Hamiltonian delta_h is a difference of: |action| + kinetic (16 per site on average)
        h_scale = abs(q.gf_hamilton_node(gf, ga)) + 16.0 * V
        flag, dh = q.run_hmc_pure_gauge(gf, ga, traj, rs.split("hmc"), n_step=c["n_step"], md_time=c["md_time"],
                                        is_always_accept=traj <= c["n_always"], integrator=INTEG[c["integrator"]],
                                        precision=precision, reunit_interval=4)
        out.append((flag, dh, q.gf_avg_plaq(gf), h_scale))
    return out


@pytest.mark.parametrize("name", ["wilson_8x4_leapfrog", "iwasaki_8x4_fg"])
def test_fp64_chain_matches_reference_library(q, chains, name):
    c = chains[name]
    got = gpu_chain(q, c, "fp64")
    assert len(got) == len(c["rows"]) >= 10
    free = [r for r in c["rows"] if r["traj"] > c["n_always"]]
    assert len(free) >= 10 and 0 < sum(r["flag"] for r in free) < len(free)
    for r, (flag, dh, plaq, h_scale) in zip(c["rows"], got):
        assert int(flag) == r["flag"], (name, r["traj"], dh, r["delta_h"])
        assert abs(dh - r["delta_h"]) <= 1e-12 * h_scale, (name, r["traj"], dh, r["delta_h"], h_scale)
        assert abs(plaq - r["plaq"]) <= 1e-12 * abs(r["plaq"]), (name, r["traj"], plaq, r["plaq"])


def test_mixed_chain_matches_reference_library(q, chains):
    c = chains["iwasaki_8x4_fg"]
    got = gpu_chain(q, c, "mixed")
    for r, (flag, dh, plaq, _) in zip(c["rows"], got):
        assert int(flag) == r["flag"], (r["traj"], dh, r["delta_h"])
        assert abs(dh - r["delta_h"]) <= 5e-3, (r["traj"], dh, r["delta_h"])
        assert abs(plaq - r["plaq"]) <= 1e-6, (r["traj"], plaq, r["plaq"])
