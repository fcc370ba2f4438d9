"""One singlepoint step of a water-cluster batch for profiling (ncu):
warm-up runs, then one more run whose launches the profiler captures.

    cd tblite-cuda_b200 && python -m tblite_b200.profile_step --count 1024 --precision 0 --warmup 1
"""
import argparse
import sys

import torch

from . import Calculator, capi, geometry


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=1024)
    ap.add_argument("--nmin", type=int, default=8)
    ap.add_argument("--nmax", type=int, default=64)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--solver", type=int, default=1, help="1: in-house eigensolver only (no calibration launches)")
    ap.add_argument("--gemm-tiles", type=int, default=-1,
                    help="-1: measured tile choice (its calibration launches come first); 0: 64 x 64 tiles only")
    a = ap.parse_args(argv)
    calc = Calculator()
    calc.set_gemm_tiles(a.gemm_tiles)
    mols = geometry.water_clusters(a.count, seed=1001, nmin=a.nmin, nmax=a.nmax)
    b = capi.Batch(calc, mols, precision=a.precision, solver=a.solver)
    for _ in range(a.warmup):
        b.run()
    torch.cuda.synchronize()
    w = b.launches()
    b.run()
    torch.cuda.synchronize()
    print(f"launches per run {b.launches()} (warm-up runs launched {w} each)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
