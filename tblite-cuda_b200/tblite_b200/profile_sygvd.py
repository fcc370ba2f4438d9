"""tb_sygvd_batch on random symmetric matrices for profiling the cluster
tridiagonalisation (k_trid_smem, which tb_sygvd_batch uses from 64 AOs):
148 matrices of 200 x 200 (one CTA each, one wave on 148 SMs) and 37 of
384 x 384 (clusters of 4 CTAs); prints the largest eigenvalue error against
numpy on the first four of each.

    cd tblite-cuda_b200 && python -m tblite_b200.profile_sygvd
"""
import sys

import numpy as np

from . import capi


def main(argv=None):
    rng = np.random.default_rng(5)
    for n, cnt in ((200, 148), (384, 37)):
        Hs = []
        for _ in range(cnt):
            M = rng.normal(size=(n, n))
            Hs.append(0.5 * (M + M.T))
        st, out = capi.sygvd_batch(Hs, [np.eye(n)] * cnt)
        if st != capi.TB_OK:
            raise SystemExit(f"tb_sygvd_batch: status {st}")
        err = max(np.max(np.abs(w - np.linalg.eigvalsh(H))) for H, (w, C) in zip(Hs[:4], out[:4]))
        print(n, cnt, "max |dw|", err)
    return 0


if __name__ == "__main__":
    sys.exit(main())
