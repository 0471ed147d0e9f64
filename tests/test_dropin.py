"""Drop-in check: the reference's own pythonlib/nestgpu.py, unchanged, loads
libnestgpu_b200.so through NESTGPU_LIB and a user script gives the same network through it as
through this repository's front-end.  Needs the reference's binding and scripts as copied
into oracle/_ref/py by oracle/Makefile.ref (skipped where they are absent)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "nest-gpu_b200", "lib", "libnestgpu_b200.so")
# the reference's binding and scripts as copied beside the reference library by
# oracle/Makefile.ref (its `py` target)
REF_PY = os.path.join(ROOT, "oracle", "_ref", "py")
SCRIPT = os.path.join(ROOT, "tests", "dropin_script.py")


def run(binding_dir):
    env = dict(os.environ, NESTGPU_LIB=LIB)
    p = subprocess.run([sys.executable, SCRIPT, binding_dir], env=env, capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads([x for x in p.stdout.splitlines() if x.startswith("JSON:")][-1][5:])


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_PY, "nestgpu.py")), reason="reference binding not copied into oracle/_ref/py")
def test_reference_binding_drives_engine():
    ref = run(REF_PY)
    own = run(os.path.join(ROOT, "nest-gpu_b200"))
    assert ref == own
    assert ref["n_conn_nm"] == 15 * 4 and ref["n_conn_mn"] == 40
    assert ref["E_rev"][0] == [0.0, -85.0]


REF_TEST = os.path.join(ROOT, "oracle", "_ref", "py", "test")


def _clean(text):
    banner = ("-- NEST GPU --", "Copyright", "This program is provided", "NO WARRANTY", "Homepage")
    return [l.rstrip() for l in text.splitlines() if l.strip() and not any(b in l for b in banner)]


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_PY, "nestgpu.py")), reason="reference binding not copied into oracle/_ref/py")
@pytest.mark.parametrize("name", ["getarr", "setvar2", "syn_group", "connect"])
def test_reference_api_scripts_reproduce_their_logs(name, tmp_path):
    """The reference's own API test scripts (python/test/test_<name>.py), run unchanged through
    its unchanged pythonlib/nestgpu.py on this library, print what their logs
    (python/test/logp3_<name>.txt) hold.  No GPU is needed: none of them calibrates.
    (logp3_setvar3.txt comes from an older library version, without den_delay among the
    scalar parameters; test_group_param.py needs iaf_psc_exp_g, outside this engine.)"""
    env = dict(os.environ, NESTGPU_LIB=LIB, PYTHONPATH=REF_PY)
    p = subprocess.run([sys.executable, os.path.join(REF_TEST, "test_%s.py" % name)], env=env,
                       capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert p.returncode == 0, p.stderr[-2000:]
    with open(os.path.join(REF_TEST, "logp3_%s.txt" % name)) as f:
        assert _clean(p.stdout) == _clean(f.read())
