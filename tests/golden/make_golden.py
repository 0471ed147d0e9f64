"""Regenerate the golden fixtures in tests/golden/ from the reference tree.

Run in a container that has the NEST GPU source tree (default location given by
NESTGPU_REF, else ../reference next to this repository's parent):

    NESTGPU_REF=/path/to/nest-gpu python tests/golden/make_golden.py

Inputs (paths inside the reference tree):
  python/test/test_<model>_nest.txt   NEST-simulator V_m traces (t [ms], V_m [mV]) used
                                      by the reference's single-neuron tests
  python/test/test_<model>.py         the tolerance each of those tests applies
  python/test/logp3_connect.txt       golden stdout of python/test/test_connect.py

Outputs:
  nest_traces.npz     one (t, V_m) array per model, plus its tolerance
  connect_log.json    the GetStatus dictionaries of each section of logp3_connect.txt
"""
import ast
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = ["aeif_cond_beta_multisynapse", "aeif_cond_alpha_multisynapse",
          "aeif_psc_exp_multisynapse", "aeif_psc_alpha_multisynapse", "iaf_psc_exp"]


def main():
    ref = os.environ.get("NESTGPU_REF")
    if not ref:
        sys.exit("set NESTGPU_REF to the reference source tree")
    tdir = os.path.join(ref, "python", "test")
    if not os.path.isdir(tdir):
        sys.exit("reference test directory not found: " + tdir)
    arrays = {}
    for m in MODELS:
        data = np.loadtxt(os.path.join(tdir, "test_%s_nest.txt" % m), delimiter="\t")
        src = open(os.path.join(tdir, "test_%s.py" % m)).read()
        tol = float(re.search(r"^tolerance\s*=\s*([0-9.eE+-]+)", src, re.M).group(1))
        arrays[m] = data.astype(np.float64)
        arrays[m + "__tolerance"] = np.array(tol)
    np.savez_compressed(os.path.join(HERE, "nest_traces.npz"), **arrays)

    sections = {}
    cur = None
    for line in open(os.path.join(tdir, "logp3_connect.txt")):
        line = line.strip()
        if line.startswith("#####"):
            cur = None
            continue
        if cur is None and line and not line.startswith("{") and not line.startswith("--") \
                and "NEST GPU" not in line and "Copyright" not in line and "program" not in line \
                and "WARRANTY" not in line and "Homepage" not in line:
            cur = line
            sections[cur] = []
            continue
        if cur is not None and (line.startswith("{") or line.startswith("[")):
            sections[cur].append(ast.literal_eval(line))
    with open(os.path.join(HERE, "connect_log.json"), "w") as f:
        json.dump(sections, f, indent=0)
    print("wrote", sorted(arrays), "and", list(sections))


if __name__ == "__main__":
    main()
