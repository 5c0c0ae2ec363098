"""The bounds-checked build (MPR_B200_CHECKED=1 loads libpoisson_b200_checked.so,
compiled with -DPB_CHECKED): the reconstruction paths run to the same bits as
with the normal library, and no padded index or guarded store left its array
(the device check word stays 0).  Each library runs in its own process, since
one process loads one of them."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r'''
import hashlib, json, sys
import numpy as np
sys.path.insert(0, ROOT)
import mojo_poissonrecon_b200 as mpr
from mojo_poissonrecon_b200 import _native, workloads
from mojo_poissonrecon_b200.batch import reconstruct_many

def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()

out = {}
pts, nrm = workloads.torus(60_000, seed=5)
for prec, depth in (("fp64", 6), ("fp32_refined", 6), ("fp32_refined", 7)):
    m = mpr.reconstruct(pts, nrm, depth=depth, precision=prec, tol=1e-8)
    out[f"{prec}@{depth}"] = digest(m.vertices, m.faces, m.density)
clouds = [workloads.torus(20_000 + 7_000 * k, seed=11 + k) + (5 + k % 3,) for k in range(4)]
meshes = reconstruct_many(clouds)
out["batch"] = digest(*[a for m in meshes for a in (m.vertices, m.faces)])
out["checked"] = int(_native.lib().pb_checked_build())
out["word"] = _native.check_word()
print(json.dumps(out))
'''


def _run(checked: bool) -> dict:
    env = dict(os.environ, MPR_B200_CHECKED="1" if checked else "0")
    code = SCRIPT.replace("ROOT", repr(ROOT))
    proc = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert proc.returncode == 0, proc.stderr[-3000:]
    return json.loads(proc.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_checked_build_runs_clean_and_bit_identical():
    from mojo_poissonrecon_b200 import buildlib

    if not os.path.exists(buildlib.CHECKED_LIBRARY):
        pytest.skip("checked library not built")
    plain, checked = _run(False), _run(True)
    assert plain["checked"] == 0 and checked["checked"] == 1
    assert checked["word"] == 0, checked["word"]
    for key in ("fp64@6", "fp32_refined@6", "fp32_refined@7", "batch"):
        assert checked[key] == plain[key], key
