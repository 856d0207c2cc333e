"""Electron scattering-factor parameters and atomic masses for the host side.

Reads the published tables compiled into csrc/scattering_tables.h (Doyle &
Turner 1968 first, Peng 1999 otherwise — the selection of
sim-trhepd-rheed/src/asf.f90:415-431) so the Python and C++ sides share one copy.
"""
from __future__ import annotations

import re
from functools import lru_cache
from pathlib import Path

HEADER = Path(__file__).resolve().parent / "csrc" / "scattering_tables.h"


@lru_cache(maxsize=1)
def _tables():
    text = HEADER.read_text()

    def block(name):
        m = re.search(r"%s\[[^\]]*\](?:\[[^\]]*\])? = \{(.*?)\n\};" % name, text, re.S)
        nums = re.findall(r"[-+]?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?", re.sub(r"//.*", "", m.group(1)))
        return [float(x) for x in nums]

    dt, pg, am = block("kDoyleTurner"), block("kPeng"), block("kAtomicMass")
    return ([dt[8 * i:8 * i + 8] for i in range(98)], [pg[8 * i:8 * i + 8] for i in range(98)], am)


def params(z: int, iabr: int = 0):
    """(a[4], b[4]) for element z (largest b first)."""
    dt, pg, _ = _tables()
    row = dt[z - 1] if (iabr == 0 and dt[z - 1][0] > 1e-5) else pg[z - 1]
    return row[:4], row[4:]


def mass(z: int) -> float:
    return _tables()[2][z - 1] if 1 <= z <= 110 else 1000.0
