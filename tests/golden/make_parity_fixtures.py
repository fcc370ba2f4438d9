#!/usr/bin/env python3
"""Write parity_singlepoints.json: FP64 oracle singlepoints of the benchmarked
configurations, at sizes the GPU parity tests compare against.

The oracle (oracle/liboracle.so, the FP64 CPU restatement of the reference's
quoted tblite routines) is run here once per structure; the GPU tests read the
committed results instead of re-running the oracle for minutes per structure.
Every structure is regenerated deterministically by the workload generators
(``tblite_b200.geometry``); each record keeps a checksum of its coordinates so a
test notices if a generator ever changes.

Structures (plain FP64 form at accuracy 1, default options):
* config-1 water clusters (1024 clusters, seed 1001): the three largest (64
  waters, 384 AOs) and five others spread over the size range;
* config-2 alkanes (256 chains, seed 1002): n = 20, 62, 120 and 199 (the
  largest of the set, 1196 AOs);
* a 210-water cluster (1260 AOs), above the in-house eigensolver bound;
* with the H/C/O/S test parameters (S has an s+p+d shell set): water clusters
  with one or two waters replaced by H2S, and dimethyl sulfide (their
  coordinates are stored in the file).
Mixed-precision records repeat the three largest clusters and the four alkanes
at accuracy 0.01, where the charges are converged tightly enough for the
mixed-form charge tolerance.

Run ``python tests/golden/make_parity_fixtures.py`` (about five minutes on eight
cores).
"""
from __future__ import annotations

import concurrent.futures as cf
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tblite-cuda_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from tblite_b200 import geometry as g  # noqa: E402

OUT = os.path.join(HERE, "parity_singlepoints.json")
PARAMS = {"hco": os.path.join(ROOT, "tblite-cuda_b200", "params", "synthetic_hco.tbp"),
          "hcos": os.path.join(ROOT, "tblite-cuda_b200", "params", "synthetic_hcos.tbp")}

CLUSTER_IDX = [1019, 44, 23]      # the three 64-water clusters of config 1 listed first
CLUSTER_SIZES = [8, 20, 32, 45, 56]
ALKANE_IDX = {20: 33, 62: 55, 120: 11, 199: 27}
SPECIES_S = 3                     # index of S in synthetic_hcos.tbp


def checksum(mol):
    x = np.asarray(mol.xyz, np.float64)
    return [float(x.sum()), float((x * x).sum()), int(np.asarray(mol.id).sum())]


def with_h2s(mol, k_list):
    """Replace waters k of a cluster (atoms 3k..3k+2 = O, H, H) by H2S:
    S at the O position, S-H 1.34 A along the former O-H directions."""
    ids = np.array(mol.id, np.int32)
    xyz = np.array(mol.xyz, np.float64)
    for k in k_list:
        o = 3 * k
        ids[o] = SPECIES_S
        for h in (o + 1, o + 2):
            v = xyz[h] - xyz[o]
            xyz[h] = xyz[o] + v / np.linalg.norm(v) * (1.34 * g.ANGSTROM)
    return g.Molecule(ids, np.ascontiguousarray(xyz), label=mol.label + f"+{len(k_list)}H2S")


def dimethyl_sulfide(rng):
    """CH3-S-CH3: C-S 1.81 A, C-S-C 99 deg, C-H 1.09 A, tetrahedral methyls; 0.02 A jitter."""
    a = math.radians(99.0) / 2
    S = np.zeros(3)
    C1 = 1.81 * np.array([math.sin(a), 0.0, math.cos(a)])
    C2 = 1.81 * np.array([-math.sin(a), 0.0, math.cos(a)])
    atoms, sp = [S, C1, C2], [SPECIES_S, 1, 1]
    for C in (C1, C2):
        u = C / np.linalg.norm(C)
        p = np.cross(u, [0.0, 1.0, 0.0])
        p /= np.linalg.norm(p)
        q = np.cross(u, p)
        for k in range(3):
            phi = 2 * math.pi * k / 3
            d = -math.cos(math.radians(109.4712)) * u + math.sin(math.radians(109.4712)) * (
                math.cos(phi) * p + math.sin(phi) * q)
            atoms.append(C + 1.09 * d)
            sp.append(0)
    xyz = np.array(atoms) + rng.normal(scale=0.02, size=(len(atoms), 3))
    return g.Molecule(np.array(sp, np.int32), np.ascontiguousarray(xyz * g.ANGSTROM), label="(CH3)2S")


def structures():
    """name -> (molecule, parameter set, generator description)."""
    out = {}
    clusters = g.water_clusters(1024, seed=1001)
    sizes = np.array([m.nat // 3 for m in clusters])
    idx = list(CLUSTER_IDX)
    for s in CLUSTER_SIZES:
        idx.append(int(np.flatnonzero(sizes == s)[0]))
    for i in idx:
        out[f"water_clusters_1024[{i}]"] = (clusters[i], "hco", {"workload": "water_clusters", "count": 1024,
                                                                 "seed": 1001, "index": i})
    alk = g.alkanes(256, seed=1002)
    for n, i in ALKANE_IDX.items():
        assert (alk[i].nat - 2) // 3 == n
        out[f"alkanes_256[{i}]"] = (alk[i], "hco", {"workload": "alkanes", "count": 256, "seed": 1002, "index": i})
    out["water_cluster_210"] = (g.water_cluster(210, np.random.default_rng(1210)), "hco",
                                {"workload": "water_cluster", "nwat": 210, "seed": 1210})
    rng = np.random.default_rng(1300)
    out["water_cluster_8_h2s"] = (with_h2s(g.water_cluster(8, rng), [0]), "hcos",
                                  {"workload": "water_cluster+h2s", "nwat": 8, "seed": 1300, "h2s": [0]})
    out["water_cluster_24_2h2s"] = (with_h2s(g.water_cluster(24, rng), [3, 17]), "hcos",
                                    {"workload": "water_cluster+h2s", "nwat": 24, "seed": 1300, "h2s": [3, 17]})
    out["dimethyl_sulfide"] = (dimethyl_sulfide(rng), "hcos", {"workload": "dimethyl_sulfide", "seed": 1300})
    return out


MIXED = [f"water_clusters_1024[{i}]" for i in CLUSTER_IDX] + [f"alkanes_256[{i}]" for i in ALKANE_IDX.values()]

_SETS = {}


def rebuild(rec):
    """The molecule of one fixture record (regenerated, or stored for the S set);
    raises if its coordinates no longer match the checksum."""
    gen = rec["generator"]
    w = gen["workload"]
    if "xyz" in rec:
        mol = g.Molecule(np.array(rec["id"], np.int32), np.ascontiguousarray(np.array(rec["xyz"], np.float64)),
                         charge=rec["charge"], uhf=rec["uhf"])
    elif w in ("water_clusters", "alkanes"):
        key = (w, gen["count"], gen["seed"])
        if key not in _SETS:
            make = g.water_clusters if w == "water_clusters" else g.alkanes
            _SETS[key] = make(gen["count"], seed=gen["seed"])
        mol = _SETS[key][gen["index"]]
    elif w == "water_cluster":
        mol = g.water_cluster(gen["nwat"], np.random.default_rng(gen["seed"]))
    else:
        raise ValueError(w)
    cs = checksum(mol)
    if cs[2] != rec["checksum"][2] or not np.allclose(cs[:2], rec["checksum"][:2], rtol=1e-14, atol=0):
        raise AssertionError(f"generator output changed: checksum {cs} != {rec['checksum']}")
    return mol


def load():
    with open(OUT) as fh:
        return json.load(fh)["structures"]


def run(job):
    import pyoracle
    name, mol, pset, acc = job
    t = time.time()
    r = pyoracle.Oracle(PARAMS[pset]).singlepoint(mol, accuracy=acc)
    rec = {k: float(r[k]) for k in ("energy", "e_rep", "e_elec", "e_band", "e_ts", "e_es2", "e_aes2", "e_es3")}
    rec.update(qat=[float(x) for x in r["qat"]], dipole=[float(x) for x in r["dipole"]],
               iterations=int(r["iterations"]), status=int(r["status"]), nao=int(len(r["emo"])))
    print(f"{name} acc={acc}: nao {rec['nao']}, E {rec['energy']:.10f}, it {rec['iterations']}, "
          f"{time.time() - t:.1f} s", flush=True)
    return name, acc, rec


def main():
    mols = structures()
    jobs = [(n, m, p, 1.0) for n, (m, p, _) in mols.items()] + [(n, mols[n][0], mols[n][1], 0.01) for n in MIXED]
    jobs.sort(key=lambda j: -j[1].nat)  # largest first
    res = {}
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:  # the oracle call releases the GIL
        for name, acc, rec in ex.map(run, jobs):
            res[(name, acc)] = rec
    doc = {"note": "FP64 oracle singlepoints (oracle/liboracle.so); generated by make_parity_fixtures.py",
           "structures": {}}
    for n, (m, p, gen) in mols.items():
        e = {"params": p, "generator": gen, "nat": int(m.nat), "checksum": checksum(m), "charge": m.charge,
             "uhf": m.uhf, "acc1": res[(n, 1.0)]}
        if (n, 0.01) in res:
            e["acc001"] = res[(n, 0.01)]
        if gen["workload"] in ("water_cluster+h2s", "dimethyl_sulfide"):
            e["xyz"] = np.asarray(m.xyz).tolist()
            e["id"] = np.asarray(m.id).tolist()
        doc["structures"][n] = e
    with open(OUT, "w") as fh:
        json.dump(doc, fh, indent=0)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
