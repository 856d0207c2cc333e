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


def read_domain_curves(path) -> tuple[list, dict]:
    """Return ([(angles, f2[nrows, nb_d]) per domain], header) of a multi-domain .md
    file (surfio.f90:276-287 header, then each domain's srfref rows)."""
    lines = [ln for ln in open(path).read().split("\n") if not ln.startswith("#")]
    toks = " ".join(lines).replace(",", " ").split()
    naz, ng, ndom, nh, nk = (int(t) for t in toks[:5])
    gam = float(toks[5])
    p = 6
    nbd, rdom, wdom = [], [], []
    for _ in range(ndom):
        nbd.append(int(toks[p]))
        rdom.append(float(toks[p + 1]))
        wdom.append(_fortran_float(toks[p + 2]))
        p += 3
    beams = []
    for nb in nbd:
        beams.append(np.array([int(t) for t in toks[p:p + 2 * nb]]).reshape(nb, 2))
        p += 2 * nb
    vals = np.array([_fortran_float(t) for t in toks[p:]])
    rows = naz * ng
    out, q = [], 0
    for nb in nbd:
        arr = vals[q:q + rows * (nb + 1)].reshape(rows, nb + 1)
        out.append((arr[:, 0], arr[:, 1:]))
        q += rows * (nb + 1)
    return out, {"naz": naz, "ng": ng, "ndom": ndom, "nh": nh, "nk": nk, "gam_deg": gam,
                 "nbd": nbd, "rdom_deg": rdom, "wdom": wdom, "beams": beams}
