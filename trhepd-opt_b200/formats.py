"""Reader for the reference's rocking-curve output (surflf.f90:154-165).

Rows are '(E12.4,200(",",E23.15))' with format reversion for nb > 200, so a
row may span several lines; exponents beyond two digits drop the 'E'.
"""
from __future__ import annotations

import numpy as np


def _fortran_float(tok: str) -> float:
    try:
        return float(tok)
    except ValueError:
        for k in range(len(tok) - 1, 0, -1):
            if tok[k] in "+-" and tok[k - 1] not in "eE":
                return float(tok[:k] + "e" + tok[k:])
        raise


def read_rocking_curves(path) -> tuple[np.ndarray, np.ndarray, dict]:
    """Return (angles[nrows], f2[nrows, nb], header) of a single-domain .s file."""
    lines = [ln for ln in open(path).read().split("\n") if not ln.startswith("#")]
    toks = " ".join(lines).replace(",", " ").split()
    naz, ng, nb = int(toks[0]), int(toks[1]), int(toks[2])
    ihik = np.array([int(t) for t in toks[3:3 + 2 * nb]]).reshape(nb, 2)
    vals = np.array([_fortran_float(t) for t in toks[3 + 2 * nb:]])
    arr = vals.reshape(-1, nb + 1)
    return arr[:, 0], arr[:, 1:], {"naz": naz, "ng": ng, "nb": nb, "beams": ihik}
