#!/usr/bin/env python3
"""Write kat_reference.json: the known-answer data held by the reference's own tests.

The values are transcribed from the reference project's test sources (read as
text; nothing of the reference is executed):

* src/test.old:97-150   test_multipole_grad_3d: s-s moments with given rpi, rpj,
  exponents and s1d; expected s3d, d3d, q3d (tolerance 1e-4 in the reference).
* src/test.old:152-176  test_transform0: isotropic Cartesian d block -> zero s-d
  spherical block.
* src/blas/level2.cu:14-26  gemv case 1 (cases 2 and 3 have wrong expected values
  in the reference and are not used).
* src/lapack/sygvd.cu:180-186  2x2 generalized problem (no expected values in the
  reference; A = 2 B exactly, so both eigenvalues are 2, which scipy confirms).
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))

kat = {
    "multipole_3d_ss": {
        "source": "src/test.old:97-150",
        # the reference passes (rpi, rpj, ai, aj, li, lj, s1d); the moments are taken
        # about the centre of its second vector argument (the quoted Fortran's rpi)
        "r_other": [0.083114717636212157, -0.39033516689727543, -0.25671966537784952],
        "r_moment": [-0.804297356879628, 3.7772557251143746, 2.4842645706404505],
        "a_other": 5.9405971566712825,
        "a_moment": 0.61389118221497996,
        "s1d": [1.0, 0.0, 0.076283605088381307, 0.0, 0.0, 0.0, 0.0],
        "s3d": 1.0,
        "d3d": [-0.804297356879628, 3.7772557251143746, 2.4842645706404505],
        "q3d": [0.72317784337193691, -3.0380367959679342, 14.343944417997701,
                -1.9980874279558183, 9.3837025721504457, 6.2478540620277627],
        "tol": 1e-4,
    },
    "transform0_sd": {
        "source": "src/test.old:152-176",
        "li": 0, "lj": 2,
        "cart": [0.6451174322, 0.6451174322, 0.6451174322, 0.0, 0.0, 0.0],
        "sphr": [0.0, 0.0, 0.0, 0.0, 0.0],
    },
    "gemv_case1": {
        "source": "src/blas/level2.cu:14-26",
        "A": [[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]],
        "x": [1.0, 2.0, 3.0],
        "y": [14.0, 32.0],
    },
    "sygvd_2x2": {
        "source": "src/lapack/sygvd.cu:180-186",
        "A": [[4.0, 1.0], [1.0, 3.0]],
        "B": [[2.0, 0.5], [0.5, 1.5]],
        "w": [2.0, 2.0],
    },
}

if __name__ == "__main__":
    with open(os.path.join(HERE, "kat_reference.json"), "w") as fh:
        json.dump(kat, fh, indent=1)
    print("wrote kat_reference.json")
