"""The reference's example scripts run unchanged, as files, through this backend.

The scripts are the reference project's own sources and are not part of this
repository: set PERIODICFLOW_EXAMPLES to the examples/ directory of a
periodic-flow checkout to run them (the tests skip otherwise).  Each script
runs in a fresh process, in a scratch directory, with this package first on
PYTHONPATH -- the backend switch -- and must exit 0 and leave the
reconfigured dataset its last line asks for.

examples/tgv3d.py is not run: 256^3 for 10,000 steps writing every 50 steps
is 200 snapshots of 400 MB (80 GB).  Its call pattern runs at 16^3 against
the oracle in test_gpu_examples.py.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

EXAMPLES = os.environ.get("PERIODICFLOW_EXAMPLES")
needs_examples = pytest.mark.skipif(
    not EXAMPLES, reason="PERIODICFLOW_EXAMPLES (a periodic-flow examples/ directory) not set")


def _run(script, args, cwd, timeout):
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join(
        [os.path.join(ROOT, "periodic-flow_b200")] + env.get("PYTHONPATH", "").split(os.pathsep))
    r = subprocess.run([sys.executable, os.path.join(EXAMPLES, script)] + args, cwd=cwd, env=env,
                       capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


def _dataset(cwd, name):
    for ext in (".h5", ".npz"):
        p = os.path.join(cwd, name + ext)
        if os.path.exists(p):
            return p
    raise AssertionError(f"no reconfigured dataset {name}.h5/.npz in {cwd}")


@needs_examples
def test_correlated_noise_example_unchanged(tmp_path):
    """64^2, dt 0.01 to t = 10 (1000 steps), written every 5 steps, L = 0.2."""
    _run("fluctuating_stokes_correlated_noise.py", ["0.2"], str(tmp_path), 1800)
    z = np.load(_dataset(str(tmp_path), "correlated"))
    keys = set(z.files)
    assert {"x", "y", "t", "u/0000", "v/1000"} <= keys
    assert len([k for k in keys if k.startswith("u/")]) == 201
    assert z["u/1000"].shape == (64, 64) and np.isfinite(z["u/1000"]).all()
    # mean kinetic energy per point stays of the order of the thermal level
    e = np.mean(z["u/1000"] ** 2 + z["v/1000"] ** 2)
    assert 0.0 < e < 1e3


@needs_examples
def test_thermal_noise_example_unchanged(tmp_path):
    """256^2, dt 1e-3 to t = 10 (10,000 steps), written every 2 steps."""
    _run("fluctuating_stokes_thermal_noise.py", [], str(tmp_path), 3600)
    z = np.load(_dataset(str(tmp_path), "thermal"))
    keys = set(z.files)
    assert {"x", "y", "t", "u/00000", "v/10000"} <= keys
    assert len([k for k in keys if k.startswith("v/")]) == 5001
    assert z["v/10000"].shape == (256, 256) and np.isfinite(z["v/10000"]).all()
