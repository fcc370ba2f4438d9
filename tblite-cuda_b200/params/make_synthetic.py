#!/usr/bin/env python3
"""Write the synthetic, GFN2-shaped H/C/O parameter file ``synthetic_hco.tbp``.

The real GFN2-xTB parameter set, tblite's STO-nG expansion tables and the D4
reference data are not available to this project, and they are not typed in
from memory.  This script instead produces a clearly labelled *synthetic*
parameter file that has every field the GFN2 Hamiltonian needs (per-shell
self-energies, CN shifts, polynomial enhancement, reference occupations,
shell-resolved Hubbard parameters and their derivatives, repulsion, the
anisotropic-electrostatics globals) with plausible magnitudes.

Contracted Gaussians are obtained here by a numerical least-squares fit of
Slater functions r^(n-1) exp(-zeta r) with ``nprim`` Gaussians
(maximising the normalised radial overlap, exponents optimised in log space,
coefficients solved linearly).  Coefficients written to the file already
include the primitive normalisation of the Cartesian component x^l exp(-a r^2)
and the contraction normalisation, so that every spherical atomic orbital has
unit self-overlap (the d-shell factor matches the sqrt(3) spherical transform
used by the integral code).

The file format (``.tbp``) is plain text, one keyword per line:

    format tblite-b200-params 1
    name <text>
    global <key> <value>            scalar globals
    kshell <li> <lj> <value>        angular-momentum pair scaling of H0
    kpair <sym_i> <sym_j> <value>   optional element-pair scaling of H0
    d4freq <n> <n values>           optional D4 block: frequency grid (Eh) and
    d4wts <n> <n values>            quadrature weights of the Casimir-Polder integral
    element <symbol> <Z>
      <key> <value>                 element scalars (rad, rcov, en, ..., d4_r4r2)
      d4_ref <cn> <n values>        D4 reference: its CN and alpha(i w) on the grid
      shell <ang> <nprim>
        <key> <value>               shell scalars (selfenergy, kcn, ...)
        alpha <nprim values>
        coeff <nprim values>
      end
    end

Run ``python make_synthetic.py`` to regenerate the file deterministically.
"""
from __future__ import annotations

import math
import os

import numpy as np
from scipy.optimize import minimize

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "synthetic_hco.tbp")
# test file with one more element whose shell set includes a d shell, so that
# the d-shell integral, transformation and Fock paths are exercised
OUT_D = os.path.join(HERE, "synthetic_hcos.tbp")
# the H/C/O file plus a synthetic D4 dispersion block (see D4 below)
OUT_D4 = os.path.join(HERE, "synthetic_hco_d4.tbp")

# radial grid for the fits
_R = np.linspace(1e-6, 40.0, 40001)
_DR = _R[1] - _R[0]


def _radial_overlap(f, g, l):
    return float(np.sum(f * g * _R ** (2 + 2 * l)) * _DR)


def fit_sto(n: int, l: int, zeta: float, nprim: int):
    """Fit r^(n-1-l) exp(-zeta r) (times r^l Y_lm) with nprim primitives r^l exp(-a r^2).

    Returns exponents (descending) and contraction coefficients for
    *normalised primitives*, normalised so that the contraction is normalised.
    """
    sto = _R ** (n - 1 - l) * np.exp(-zeta * _R)
    sto = sto / math.sqrt(_radial_overlap(sto, sto, l))

    def prim(a):
        g = np.exp(-a * _R * _R)
        return g / math.sqrt(_radial_overlap(g, g, l))

    def solve(loga):
        a = np.exp(loga)
        G = np.stack([prim(x) for x in a])
        M = np.array([[_radial_overlap(G[i], G[j], l) for j in range(nprim)] for i in range(nprim)])
        b = np.array([_radial_overlap(G[i], sto, l) for i in range(nprim)])
        c = np.linalg.solve(M, b)
        ov = float(b @ c) / math.sqrt(float(c @ M @ c))
        return ov, c, M

    x0 = np.log(zeta * zeta * np.geomspace(0.1, 8.0, nprim))
    # keep the exponents in a physically sensible window (0.03..60 zeta^2)
    lo, hi = math.log(0.03 * zeta * zeta), math.log(60.0 * zeta * zeta)
    res = minimize(lambda x: -solve(x)[0], x0, method="Powell",
                   bounds=[(lo, hi)] * nprim,
                   options={"xtol": 1e-10, "ftol": 1e-14, "maxiter": 20000, "maxfev": 40000})
    ov, c, M = solve(res.x)
    c = c / math.sqrt(float(c @ M @ c))
    a = np.exp(res.x)
    order = np.argsort(-a)
    return a[order], c[order], ov


def cart_norm(a: float, l: int) -> float:
    """Normalisation of x^l exp(-a r^2) (the 'xx..' Cartesian component)."""
    dfac = [1.0, 1.0, 3.0, 15.0][l]  # (2l-1)!!
    return (2.0 * a / math.pi) ** 0.75 * (4.0 * a) ** (0.5 * l) / math.sqrt(dfac)


def sph_prim_factor(a: float, l: int) -> float:
    """Radial-normalised primitive -> Cartesian-normalised primitive factor.

    The fit uses radially normalised primitives; the integral code expects the
    coefficient multiplying the raw Cartesian primitive x^l exp(-a r^2), whose
    self-overlap is 1/cart_norm^2.  Both normalisations describe the same
    function up to a constant, so the contraction coefficient just becomes
    c * cart_norm(a, l).
    """
    return cart_norm(a, l)


# ---------------------------------------------------------------------------
# synthetic values (plausible magnitudes, NOT the GFN2-xTB parameters)
# ---------------------------------------------------------------------------
GLOBALS = {
    "gexp": 2.0,            # exponent of the ES2 gamma kernel
    "kdmp3": 3.0,           # AES damping exponent, inverse-cubic terms
    "kdmp5": 4.0,           # AES damping exponent, inverse-quintic terms
    "mp_shift": 1.0,        # shift of the multipole damping radii
    "mp_kexp": 4.5,         # steepness of the multipole damping radii
    "mp_rmax": 5.5,         # maximum multipole damping radius (Bohr)
    "rep_kexp": 1.5,        # repulsion exponent on R
    "rep_kexp_light": 1.0,  # repulsion exponent on R for H/He pairs
    "rep_rexp": 1.0,        # repulsion polynomial exponent
    "enscale": 0.02,        # electronegativity scaling of H0
    "wexp": 0.5,            # Slater-exponent weighting exponent of H0
    "cn_cutoff": 25.0,      # real-space cutoff of the coordination number (Bohr)
    "rep_cutoff": 25.0,     # real-space cutoff of the repulsion (Bohr)
}
KSHELL = {(0, 0): 1.90, (0, 1): 2.05, (1, 1): 2.20, (0, 2): 2.00, (1, 2): 2.10, (2, 2): 2.30}

ELEMENTS = [
    # symbol, Z, element scalars, shells (n, l, zeta, nprim, shell scalars)
    ("H", 1,
     dict(rad=1.10, rcov=0.80, en=2.20, rep_alpha=2.20, rep_zeff=1.10,
          mp_rad=1.40, mp_vcn=1.0, dkernel=0.0100, qkernel=0.0010),
     [(1, 0, 1.20, 3, dict(selfenergy=-0.4000, kcn=0.0030, shpoly=-0.050, refocc=1.0,
                           hubbard=0.4050, hubbard_deriv=0.0800))]),
    ("C", 6,
     dict(rad=1.45, rcov=1.90, en=2.55, rep_alpha=2.00, rep_zeff=4.20,
          mp_rad=3.00, mp_vcn=3.0, dkernel=0.0080, qkernel=0.0020),
     [(2, 0, 1.70, 4, dict(selfenergy=-0.5000, kcn=0.0040, shpoly=-0.020, refocc=1.0,
                           hubbard=0.5380, hubbard_deriv=0.1000)),
      (2, 1, 1.60, 4, dict(selfenergy=-0.3700, kcn=0.0020, shpoly=0.050, refocc=3.0,
                           hubbard=0.4600, hubbard_deriv=0.0500))]),
    ("O", 8,
     dict(rad=1.40, rcov=1.60, en=3.44, rep_alpha=2.30, rep_zeff=5.80,
          mp_rad=2.50, mp_vcn=2.0, dkernel=0.0150, qkernel=0.0030),
     [(2, 0, 2.20, 4, dict(selfenergy=-0.7500, kcn=0.0050, shpoly=-0.030, refocc=2.0,
                           hubbard=0.5700, hubbard_deriv=0.1200)),
      (2, 1, 2.10, 4, dict(selfenergy=-0.5000, kcn=0.0030, shpoly=0.040, refocc=4.0,
                           hubbard=0.6200, hubbard_deriv=0.0600))]),
]


# S-like element with an s+p+d valence shell set (d empty in the reference
# occupation, as for the heavier main-group elements of GFN2)
ELEMENT_S = ("S", 16,
             dict(rad=1.80, rcov=2.00, en=2.58, rep_alpha=1.80, rep_zeff=8.00,
                  mp_rad=3.20, mp_vcn=2.0, dkernel=0.0060, qkernel=0.0015),
             [(3, 0, 2.10, 4, dict(selfenergy=-0.6200, kcn=0.0040, shpoly=-0.010, refocc=2.0,
                                   hubbard=0.4400, hubbard_deriv=0.0900)),
              (3, 1, 1.85, 4, dict(selfenergy=-0.4200, kcn=0.0020, shpoly=0.030, refocc=4.0,
                                   hubbard=0.3900, hubbard_deriv=0.0500)),
              (3, 2, 1.20, 3, dict(selfenergy=-0.1200, kcn=0.0010, shpoly=0.060, refocc=0.0,
                                   hubbard=0.3000, hubbard_deriv=0.0300))])


# ---------------------------------------------------------------------------
# synthetic D4 dispersion data (plausible magnitudes, NOT the dftd4 reference
# polarizabilities).  Each reference system of an element is a single
# Lorentzian oscillator, alpha(i w) = alpha0 / (1 + (w / w0)^2), tabulated on a
# 23-point Gauss-Legendre grid mapped to [0, inf) by w = ws (1 + t) / (1 - t);
# the C6 of two such oscillators by the Casimir-Polder integral has the London
# closed form 3/2 a1 a2 w1 w2 / (w1 + w2), against which the grid is checked.
# ---------------------------------------------------------------------------
D4_NFREQ = 23
D4_WS = 0.5
D4_GLOBALS = {
    "d4_s6": 1.0,           # two-body C6 scaling
    "d4_s8": 2.5,           # two-body C8 scaling
    "d4_a1": 0.5,           # rational damping: R = a1 R0 + a2
    "d4_a2": 5.0,
    "d4_s9": 1.0,           # three-body (Axilrod-Teller-Muto) scaling
    "d4_alp": 16.0,         # three-body damping exponent
    "d4_wf": 6.0,           # Gaussian weight of the reference CNs
    "d4_k0": 7.5,           # steepness of the error-function counting
    "d4_k1": 1.0,           # covalent-radius scaling of the counting
    "d4_k4": 4.1,           # electronegativity factor k4 exp(-(|dEN| + k5)^2 / k6)
    "d4_k5": 19.1,
    "d4_k6": 254.5,
    "d4_cn_cut": 25.0,      # cutoffs (Bohr): coordination number, three-body, two-body
    "d4_atm_cut": 25.0,
    "d4_pair_cut": 60.0,
}
# per element: r4/r2 expectation-value factor Q and the references (CN, alpha0, w0)
D4_ELEMENTS = {
    "H": (2.00, [(0.0, 4.50, 0.45), (1.0, 3.00, 0.50)]),
    "C": (3.10, [(0.0, 11.9, 0.40), (2.0, 10.0, 0.42), (3.0, 9.0, 0.44), (4.0, 8.0, 0.46)]),
    "O": (2.60, [(0.0, 5.40, 0.55), (1.0, 5.00, 0.57), (2.0, 4.60, 0.60)]),
}


def d4_grid():
    t, wt = np.polynomial.legendre.leggauss(D4_NFREQ)
    w = D4_WS * (1.0 + t) / (1.0 - t)
    wts = wt * 2.0 * D4_WS / (1.0 - t) ** 2
    return w, wts


def d4_lines():
    w, wts = d4_grid()
    lines = [f"global {k} {v!r}" for k, v in D4_GLOBALS.items()]
    lines.append(f"d4freq {D4_NFREQ} " + " ".join(f"{x:.17g}" for x in w))
    lines.append(f"d4wts {D4_NFREQ} " + " ".join(f"{x:.17g}" for x in wts))
    # quadrature check against the London formula for every pair of references
    worst = 0.0
    refs = [r for _, rs in D4_ELEMENTS.values() for r in rs]
    for _, a1, w1 in refs:
        for _, a2, w2 in refs:
            quad = 3.0 / math.pi * float(np.sum(wts * a1 / (1 + (w / w1) ** 2) * a2 / (1 + (w / w2) ** 2)))
            exact = 1.5 * a1 * a2 * w1 * w2 / (w1 + w2)
            worst = max(worst, abs(quad - exact) / exact)
    print(f"D4 grid: largest relative C6 quadrature error {worst:.2e}")
    return lines


def d4_element_lines(sym):
    w, _ = d4_grid()
    q, refs = D4_ELEMENTS[sym]
    lines = [f"  d4_r4r2 {q!r}"]
    for cn, a0, w0 in refs:
        lines.append(f"  d4_ref {cn!r} " + " ".join(f"{a0 / (1 + (x / w0) ** 2):.17g}" for x in w))
    return lines


def write(path, name, title, elements, d4=False):
    lines = [
        f"# SYNTHETIC GFN2-shaped parameters for {title}.",
        "# These are NOT the GFN2-xTB parameters; they only have the same fields and",
        "# plausible magnitudes. Generated by make_synthetic.py (deterministic).",
        "format tblite-b200-params 1",
        f"name {name}",
    ]
    for k, v in GLOBALS.items():
        lines.append(f"global {k} {v!r}")
    if d4:
        lines.append("# synthetic D4 dispersion block (NOT the dftd4 reference data)")
        lines += d4_lines()
    for (li, lj), v in sorted(KSHELL.items()):
        lines.append(f"kshell {li} {lj} {v!r}")
    for sym, z, escal, shells in elements:
        lines.append(f"element {sym} {z}")
        for k, v in escal.items():
            lines.append(f"  {k} {v!r}")
        if d4:
            lines += d4_element_lines(sym)
        for n, l, zeta, nprim, sscal in shells:
            a, c, ov = fit_sto(n, l, zeta, nprim)
            coeff = [float(ci * sph_prim_factor(ai, l)) for ai, ci in zip(a, c)]
            lines.append(f"  shell {l} {nprim}")
            lines.append(f"    # fit of n={n} l={l} Slater zeta={zeta}: overlap {ov:.8f}")
            lines.append(f"    slater {zeta!r}")
            for k, v in sscal.items():
                lines.append(f"    {k} {v!r}")
            lines.append("    alpha " + " ".join(f"{x:.17g}" for x in a))
            lines.append("    coeff " + " ".join(f"{x:.17g}" for x in coeff))
            lines.append("  end")
        lines.append("end")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    print("wrote", path)


def main():
    write(OUT, "synthetic-gfn2-shaped-HCO", "H, C, O", ELEMENTS)
    write(OUT_D, "synthetic-gfn2-shaped-HCOS", "H, C, O, S (test file: S has a d shell)",
          ELEMENTS + [ELEMENT_S])
    write(OUT_D4, "synthetic-gfn2-shaped-HCO-D4", "H, C, O with a synthetic D4 dispersion block", ELEMENTS,
          d4=True)


if __name__ == "__main__":
    main()
