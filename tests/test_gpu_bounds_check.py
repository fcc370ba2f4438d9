"""GPU: the checked build (lib/libtblite_b200_check.so, index guards that skip
and record any global-memory access outside its structure's own slice; no
trap) runs the singlepoint paths in a fresh process -- plain and mixed forms,
the whole-loop graph, d shells, gradients, the nspin = 2 read-out, the
batched generalized eigensolver -- and records no violation; its results
equal the normal build's (1e-10)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from tblite_b200 import capi, geometry as g

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import json, sys
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[2])
import numpy as np
from tblite_b200 import capi
capi.load_library(capi.LIB_CHECK_PATH)
import run_cases
out = run_cases.run()
out["violations"] = list(capi.bounds_violations())
out["checked"] = int(capi.load_library().tb_bounds_check_build())
print("RESULT " + json.dumps(out))
"""


def test_checked_build_runs_clean_and_agrees():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    here = os.path.dirname(os.path.abspath(__file__))
    p = subprocess.run([sys.executable, "-c", _CHILD, os.path.join(ROOT, "tblite-cuda_b200"),
                        os.path.join(here, "golden")], capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [s for s in p.stdout.splitlines() if s.startswith("RESULT ")]
    assert line, p.stdout[-2000:] + p.stderr[-2000:]
    got = json.loads(line[-1][len("RESULT "):])
    assert got["checked"] == 1
    assert got["violations"][0] == 0, got["violations"]
    sys.path.insert(0, os.path.join(here, "golden"))
    import run_cases
    ref = run_cases.run()  # the normal build, this process
    for k, v in ref.items():
        np.testing.assert_allclose(np.asarray(got[k], float), np.asarray(v, float), atol=1e-10, err_msg=k)
