#!/usr/bin/env python3
"""Extract the golden values that pin the pure-gauge path from the
reference's own test logs into reference_goldens.json.

Run in a checkout that has the reference source tree, passing its path as
the first argument or in QLAT_REFERENCE_ROOT (there is no default).  Sources:
  examples-cpp/hmc/log                        C++ force-gradient HMC, plaq per trajectory
  examples-cpp/flowed-hmc/log                 C++ flowed HMC (masked invertible flows), plaq per trajectory
  examples-py/hmc-pure-gauge.log.json         Python HMC, plaq and delta_h per trajectory
  examples-py/hmc-pure-gauge-test.log.json    Python HMC from a unit start, plaq per trajectory
  examples-py/flow-and-smear.log.json         Wilson flow steps and energies
  examples-py/gf-utils.log.json               hot-start plaquette, clover and 5-loop charges along the flow
  examples-py/hmc-pure-gauge-fa-sym.log.json  field-accelerated HMC, five jobs, plaq per trajectory
  examples-py/gf-flow-topo.log.json           Wilson and plaquette-weighted flows: plaq, plaq_min, flow time, signatures
  examples-py/hmc-pure-gauge-symmetric.log.json  HMC with a dual momentum (gf_evolve + gf_evolve_dual), plaq per trajectory
  examples-py/hmc-pure-gauge-flowed.log.json  flowed HMC (add_rand_order_flow), plaq per trajectory
  examples-py/hmc-pure-gauge-flowed-test.log.json  flowed HMC, plaq and 1x1 Wilson loop per trajectory
"""

import json
import os
import re
import sys


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("QLAT_REFERENCE_ROOT")
    if not ref:
        sys.exit("usage: make_reference_goldens.py <reference source tree> (or set QLAT_REFERENCE_ROOT)")
    out = {}
    # C++ HMC log
    lines = open(os.path.join(ref, "examples-cpp/hmc/log")).read().splitlines()
    cpp = []
    for ln in lines:
        m = re.match(r"CHECK: test_hmc: traj=(\d+) ; plaq_avg=\s*(\S+) ; plaq_sum=\s*(\S+)\.", ln)
        if m:
            cpp.append([int(m.group(1)), float(m.group(2)), float(m.group(3))])
    out["cpp_hmc"] = {"source": "examples-cpp/hmc/log", "rows": cpp, "printed_digits": 13}
    lines = open(os.path.join(ref, "examples-cpp/flowed-hmc/log")).read().splitlines()
    rows = []
    for ln in lines:
        m = re.match(r"CHECK: test_hmc: traj=(\d+) ; plaq_avg=\s*(\S+) ; plaq_sum=\s*(\S+)\.", ln)
        if m:
            rows.append([int(m.group(1)), float(m.group(2)), float(m.group(3))])
    out["cpp_flowed_hmc"] = {"source": "examples-cpp/flowed-hmc/log", "rows": rows, "printed_digits": 13,
                             "beta": 2.31, "c1": -0.331, "total_site": [4, 4, 4, 8]}

    def load(name):
        d = json.load(open(os.path.join(ref, "examples-py", name)))
        return {e[0]: [e[1], e[2]] for e in d if len(e) == 3}

    g = load("hmc-pure-gauge.log.json")
    out["py_hmc"] = {"source": "examples-py/hmc-pure-gauge.log.json",
                     "plaq": [g[f"run_hmc: {t} plaq"][0] for t in range(1, 9)],
                     "delta_h": [g[f"run_hmc: {t} delta_h"][0] for t in range(1, 9)],
                     "eps_plaq": 1e-10, "eps_delta_h": 1e-4}
    g = load("hmc-pure-gauge-test.log.json")
    out["py_hmc_test"] = {"source": "examples-py/hmc-pure-gauge-test.log.json",
                          "iwasaki_plaq": [g[f"beta=2.13_c1=-0.331 traj={t} plaq"][0] for t in range(1, 5)],
                          "wilson_plaq": [g[f"beta=5.5_c1=0.0 traj={t} plaq"][0] for t in range(1, 5)],
                          "eps": 1e-10}
    g = load("flow-and-smear.log.json")
    out["flow"] = {"source": "examples-py/flow-and-smear.log.json",
                   "rk3_plaq": g["gf_wilson_flow_step runge-kutta plaq"][0],
                   "euler_plaq": g["gf_wilson_flow_step euler plaq"][0],
                   "c1_plaq": {str(c1): g[f"gf_wilson_flow_step c1={c1} plaq"][0] for c1 in (0.0, -0.331, -1.4008)},
                   "flow3_energy": g["gf_wilson_flow energy_list"][0]["value"],
                   "flow3_plaq": g["gf_wilson_flow final plaq"][0],
                   "flow_topo": {k[len("gf_flow_topo "):-len(" plaq")]: v[0] for k, v in g.items()
                                 if k.startswith("gf_flow_topo ")},
                   "eps": 1e-10}
    g = load("gf-utils.log.json")
    out["gf_utils"] = {"source": "examples-py/gf-utils.log.json",
                       "hot_plaq": g["gf_ape_list[0] plaq"][0],
                       "topo_clf": {str(t): g[f"t={t} topo_clf"][0] for t in ("0", "1.0", "2.0", "3.0", "4.0", "5.0")},
                       "topo_5li": {str(t): g[f"t={t} topo_5li"][0] for t in ("0", "1.0", "2.0", "3.0", "4.0", "5.0")},
                       "topo_5li_terms_sum": {str(t): g[f"t={t} topo_5li sum(topo_terms)"][0]
                                              for t in ("0", "1.0", "2.0", "3.0", "4.0", "5.0")},
                       "eps_topo": 1e-9}
    # field-accelerated HMC: the log holds, per job of the script's default
    # job list (in that order), the job's parameters then 'run_hmc: {traj} plaq'
    src = open(os.path.join(ref, "examples-py/hmc-pure-gauge-fa-sym.py")).read()
    tags = re.findall(r'"([^"]+)"', re.search(r"job_tag_list_default = \[(.*?)\]", src, re.S).group(1))
    jobs = []
    for e in json.load(open(os.path.join(ref, "examples-py/hmc-pure-gauge-fa-sym.log.json"))):
        if len(e) == 1:
            jobs.append({"job_tag": tags[len(jobs)], "params": json.loads(e[0]), "plaq": []})
        else:
            m = re.match(r"run_hmc: (\d+) plaq", e[0])
            assert m and int(m.group(1)) == len(jobs[-1]["plaq"]) + 1
            jobs[-1]["plaq"].append(e[1])
    out["py_hmc_fa_sym"] = {"source": "examples-py/hmc-pure-gauge-fa-sym.log.json", "jobs": jobs,
                            "reference_check_eps": 1e-5}
    # single-job HMC examples: the job's parameters, then 'run_hmc: {traj} plaq'
    for key, name in (("py_hmc_symmetric", "hmc-pure-gauge-symmetric"), ("py_hmc_flowed", "hmc-pure-gauge-flowed")):
        log = json.load(open(os.path.join(ref, "examples-py", name + ".log.json")))
        params = json.loads(log[0][0])
        plaq = []
        for e in log[1:]:
            m = re.match(r"run_hmc: (\d+) plaq", e[0])
            assert m and int(m.group(1)) == len(plaq) + 1
            plaq.append(e[1])
        out[key] = {"source": f"examples-py/{name}.log.json", "job_tag": params["job_tag"],
                    "total_site": params["total_site"], "hmc": params["hmc"], "plaq": plaq}
    g = load("hmc-pure-gauge-flowed-test.log.json")
    out["py_hmc_flowed_test"] = {"source": "examples-py/hmc-pure-gauge-flowed-test.log.json",
                                 "rows": [[t, g[f"beta=2.31_c1=-0.331 traj={t} plaq"][0],
                                           g[f"beta=2.31_c1=-0.331 traj={t} wilson_loop"][0]] for t in (1, 2, 3)],
                                 "eps": 1e-10}
    # gf_flow_topo stages: (name, value) in log order; complex signature
    # entries as [re, im] pairs
    rows = []
    for e in json.load(open(os.path.join(ref, "examples-py/gf-flow-topo.log.json"))):
        if len(e) != 3:
            continue
        v = e[1]
        if isinstance(v, dict):
            v = [[x["real"], x["imag"]] if isinstance(x, dict) else x for x in v["value"]]
        rows.append([e[0], v])
    out["gf_flow_topo"] = {"source": "examples-py/gf-flow-topo.log.json", "rows": rows, "eps": 1e-10,
                           "flow_order": [None, "Freeze", "Shrink", "Localize", "Preserve"], "n_step": 5,
                           "step_size": 0.1}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_goldens.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
