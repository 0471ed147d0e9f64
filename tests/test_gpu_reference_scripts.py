"""The reference's own acceptance scripts, run unchanged on this library.

Each script of the reference's python/test directory (the list of test_all.sh that falls
on this engine's models) runs as its own process through the reference's unchanged
pythonlib/nestgpu.py, loaded with NESTGPU_LIB pointing at libnestgpu_b200.so, in a
temporary directory holding the script's data files.  Scripts that judge themselves must
exit 0 (trace tests against NEST's golden traces, Brunel rate tests, spike-time
consistency, STDP against the closed form); scripts that print must reproduce their
logp3_<name>.txt logs (lines naming the dynamic-library path filtered as test_all.sh
does, the library banner dropped).

The binding and scripts are the copies oracle/Makefile.ref places in oracle/_ref/py; the
tests are skipped where they are absent.
"""
import os
import shutil
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "nest-gpu_b200", "lib", "libnestgpu_b200.so")
REF_PY = os.path.join(ROOT, "oracle", "_ref", "py")
REF_TEST = os.path.join(REF_PY, "test")

needs_scripts = pytest.mark.skipif(not os.path.exists(os.path.join(REF_PY, "nestgpu.py")),
                                   reason="reference binding not copied into oracle/_ref/py")

SELF_JUDGING = ["test_iaf_psc_exp.py", "test_aeif_cond_beta_multisynapse.py",
                "test_aeif_cond_alpha_multisynapse.py", "test_aeif_psc_exp_multisynapse.py",
                "test_aeif_psc_alpha_multisynapse.py", "test_brunel_list.py", "test_brunel_outdegree.py",
                "test_fixed_total_number.py", "test_spike_times.py", "test_stdp.py", "test_stdp_list.py",
                "test_syn_model.py"]
LOGGED = ["connect", "syn_group", "getarr", "setvar2"]


def run_script(name, tmp_path, timeout=900):
    for f in os.listdir(REF_TEST):
        shutil.copy(os.path.join(REF_TEST, f), str(tmp_path))
    env = dict(os.environ, NESTGPU_LIB=LIB, PYTHONPATH=REF_PY)
    return subprocess.run([sys.executable, name], env=env, capture_output=True, text=True, timeout=timeout,
                          cwd=str(tmp_path))


def _clean(text):
    banner = ("-- NEST GPU --", "Copyright", "This program is provided", "NO WARRANTY", "Homepage")
    return [l.rstrip() for l in text.splitlines()
            if l.strip() and "dyl" not in l and not any(b in l for b in banner)]


@needs_scripts
@pytest.mark.parametrize("script", SELF_JUDGING)
def test_reference_script_passes(script, tmp_path):
    p = run_script(script, tmp_path)
    assert p.returncode == 0, (p.stdout[-3000:], p.stderr[-3000:])


@needs_scripts
@pytest.mark.parametrize("name", LOGGED)
def test_reference_script_reproduces_log(name, tmp_path):
    p = run_script("test_%s.py" % name, tmp_path)
    assert p.returncode == 0, p.stderr[-3000:]
    with open(os.path.join(REF_TEST, "logp3_%s.txt" % name)) as f:
        assert _clean(p.stdout) == _clean(f.read())
