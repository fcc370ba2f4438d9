"""A fixed set of singlepoint cases through the public binding, for comparing
two builds of the library (the checked build against the normal one):
returns plain lists of energies, charges, gradients and read-outs."""
import os

import numpy as np

from tblite_b200 import capi, geometry as g

HERE = os.path.dirname(os.path.abspath(__file__))


def run():
    import make_parity_fixtures as fx
    out = {}
    calc = capi.Calculator()
    mols = g.water_clusters(6, seed=123, nmin=2, nmax=20) + [g.alkane(6, np.random.default_rng(3))]
    r = calc.singlepoint_batch(mols, use_graphs=1)
    out["plain_E"] = [x["energy"] for x in r]
    out["plain_q"] = np.concatenate([x["qat"] for x in r]).tolist()
    r = calc.singlepoint_batch(mols, precision=1)
    out["mixed_E"] = [x["energy"] for x in r]
    r = calc.singlepoint_batch(mols[:3], gradient=True, wavefunction=True, nspin=2)
    out["grad"] = np.concatenate([x["gradient"].ravel() for x in r]).tolist()
    out["dens"] = np.concatenate([x["wfn"]["density"].ravel() for x in r]).tolist()
    hcos = capi.Calculator(fx.PARAMS["hcos"])
    m = fx.rebuild(fx.load()["water_cluster_8_h2s"])
    r = hcos.singlepoint_batch([m], gradient=True)[0]
    out["d_E"] = [r["energy"]]
    out["d_grad"] = r["gradient"].ravel().tolist()
    rng = np.random.default_rng(8)
    H = rng.normal(size=(40, 40)); H = H + H.T
    R = rng.normal(size=(40, 40)); S = R @ R.T / 40 + np.eye(40)
    st, res = capi.sygvd_batch([H], [S])
    out["sygvd_w"] = res[0][0].tolist()
    return out
