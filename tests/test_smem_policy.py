"""CPU: the eigensolver's shared-memory sizing (syev_smem_bytes, tb_kernels.h).

k_syev takes divide and conquer for a structure of kDcMin+ rows when its
dynamic shared memory holds the merge workspace.  A batch launches with
syev_smem_bytes(nmax), so the choice depends on the structure's size alone
(and a structure gives the same bits alone and in any batch) exactly when
syev_smem_bytes(n) covers 2n + dc_ws_elems(n) doubles for every n >= kDcMin
and never decreases with n.  A host-only program compiled with nvcc checks
both over every size the in-house solver accepts; it launches nothing.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "tblite-cuda_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include "tb_kernels.h"
int main() {
  int bad = 0;
  for (int n = 1; n <= tb::kSyevMaxN; ++n) {
    const size_t need = n >= tb::kDcMin ? (2 * (size_t)n + (size_t)tb::dc_ws_elems<double>(n)) * sizeof(double) : 0;
    if (tb::syev_smem_bytes(n) < need) ++bad;
    if (n > 1 && tb::syev_smem_bytes(n) < tb::syev_smem_bytes(n - 1)) ++bad;
    if (tb::syev_smem_bytes(n) < (7 + 2 * (size_t)tb::kRing) * n * sizeof(double)) ++bad;
  }
  std::printf("%d\n", bad);
  return bad != 0;
}
"""


def test_syev_smem_covers_the_merge_workspace(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "smem_policy.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "smem_policy"
    subprocess.run([nvcc, "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True,
                   capture_output=True, timeout=300)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "0", out.stdout + out.stderr
