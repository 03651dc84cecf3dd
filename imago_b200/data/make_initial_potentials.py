"""Write initial_potentials.json: the atomic-superposition starting
potential of each element on the potential Gaussians this library's
systems use.

Imago starts its SCF from the isolated-atom potentials of its database
(src/data/atomicPDB/<element>/coeff1, column 1 the coefficient, column 2 the
exponent; read by initPotCoeffs, potential.f90:433-563, from the scfV deck
makeinput.py writes).  The systems here use other exponent ranges than the
database, so each element's database potential V(r) = sum_i c_i
exp(-a_i r^2) is projected onto the target Gaussians g_j = exp(-b_j r^2) in
the L2 metric the reference fits its potentials in (the potential alpha
overlap (pi / (b_j + b_k))^(3/2)):

    sum_k (pi/(b_j+b_k))^1.5 d_k = sum_i (pi/(b_j+a_i))^1.5 c_i.

Run where the reference is mounted:

    python imago_b200/data/make_initial_potentials.py <root of the reference checkout>

The library reads the JSON; the database itself is not needed afterwards.
"""
import io
import json
import os
import sys
import tarfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from imago_b200.system import pot_alphas  # noqa: E402

# (element symbol, Z, number of terms, smallest and largest exponent)
TARGETS = [("c", 6, 16, 0.12, 1.0e5), ("si", 14, 20, 0.10, 1.0e5), ("o", 8, 20, 0.12, 1.0e5)]


def read_db(root, element):
    with tarfile.open(os.path.join(root, "src", "data", "atomicPDB.tgz")) as tf:
        data = tf.extractfile(f"atomicPDB/{element}/coeff1").read().decode()
    lines = data.split("\n")
    n = int(lines[0])
    rows = np.array([[float(x) for x in l.split()[:2]] for l in lines[1:1 + n]])
    return rows[:, 0], rows[:, 1]


def project(c, a, b):
    S = (np.pi / (b[:, None] + b[None, :])) ** 1.5
    X = (np.pi / (b[:, None] + a[None, :])) ** 1.5
    return np.linalg.solve(S, X @ c)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_initial_potentials.py <root of the reference checkout>")
    out = []
    for el, z, n, lo, hi in TARGETS:
        c, a = read_db(sys.argv[1], el)
        b = pot_alphas(n, lo, hi)
        out.append({"element": el, "z": z, "alpha_min": lo, "alpha_max": hi,
                    "alphas": b.tolist(), "coeffs": project(c, a, b).tolist()})
    with open(os.path.join(HERE, "initial_potentials.json"), "w") as fh:
        json.dump({"potentials": out}, fh, indent=1)


if __name__ == "__main__":
    main()
