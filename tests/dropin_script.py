"""A NEST GPU user script run unchanged against this engine's library through the
reference's own Python binding (the binding's directory is the first argument).  Prints a
JSON summary of what it built; tests/test_dropin.py compares it with the same script
through this repository's front-end.  Creation, parameters and connections only: no GPU
work is needed before calibration."""
import json
import sys

sys.path.insert(0, sys.argv[1])
import nestgpu as ngpu  # noqa: E402

ngpu.SetVerbosityLevel(0)
ngpu.SetRandomSeed(1234)
n = ngpu.Create("aeif_cond_beta_multisynapse", 20, 2)
ngpu.SetStatus(n, {"E_rev": [0.0, -85.0], "tau_decay": [20.0, 10.0], "tau_rise": [2.0, 1.0]})
m = ngpu.Create("iaf_psc_exp", 15)
ngpu.SetStatus(m, "V_m_rel", -5.0)
pg = ngpu.Create("poisson_generator")
ngpu.SetStatus(pg, "rate", 1234.0)
ngpu.Connect(n, m, {"rule": "fixed_indegree", "indegree": 4}, {"weight": 1.5, "delay": 1.0})
ngpu.Connect(m, n, {"rule": "fixed_total_number", "total_num": 40},
             {"weight": 0.25, "delay": 2.0, "receptor": 1})
ngpu.Connect(pg, n, {"rule": "all_to_all"}, {"weight": 0.1, "delay": 1.0, "receptor": 0})
conns = ngpu.GetConnections(n, m)
st = ngpu.GetStatus(conns)
out = {
    "E_rev": [list(map(float, x)) for x in ngpu.GetStatus(n, "E_rev")],
    "tau_decay": [list(map(float, x)) for x in ngpu.GetStatus(n[0:3], "tau_decay")],
    "V_m_rel": [float(x) for x in ngpu.GetStatus(m, "V_m_rel")],
    "rate": float(ngpu.GetStatus(pg, "rate")[0]),
    "n_conn_nm": len(conns),
    "targets": sorted([int(s["target"]) for s in st]),
    "sources": sorted([int(s["source"]) for s in st]),
    "weights": sorted([float(s["weight"]) for s in st]),
    "n_conn_mn": len(ngpu.GetConnections(m, n)),
    "random_int": None,
}
r = ngpu.RandomInt(5)   # the reference binding returns the C pointer itself
out["random_int"] = [int(r[i]) for i in range(5)]
print("JSON:" + json.dumps(out))
