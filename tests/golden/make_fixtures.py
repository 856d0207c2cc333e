"""Oracle fixtures for the synthetic benchmark structures.

The reference ships no outputs for the seeded synthetic structures the
benchmark runs on, so their parity pins come from the CPU oracle (the FP64
restatement of the sim-trhepd-rheed surface path, itself pinned to the
reference's committed outputs by ``test_oracle_golden.py``).  This script
regenerates each structure with the package's seeded generator, writes the
reference-format inputs to a scratch directory, runs the oracle and stores
per case:

* ``f2`` (angles x beams) and ``angle`` of the selected schedule rows ``idx``;
* ``renorm``: per-angle renormalisation counts;
* ``sha``: SHA-256 of bulk.txt + surf.txt + bulkP.b, so a test can tell that it
  regenerated the same inputs;
* for the growth-bound renormalisation schedule, ``f2_growth`` and
  ``interval`` (slices between renormalisations).

Cases (sizes of the benchmark configurations):

* ``batch47``   — N = 47, 121 angles x 2 azimuths, 15 A in 0.02 A slices, every row;
* ``dense521``  — N = 521, 61 angles, 20 A in 0.01 A slices (2004 slices), rows
  0, 8, 17, 25, 34, 42, 51, 60, Gershgorin and growth-bound schedules;
* ``uneven<N>`` — the first jittered candidate (sigma 0.1 A) of the uneven batch's
  base structure for N = 23, 47, 95, 191, rows 0, 20, 40, 60.

Usage: python tests/golden/make_fixtures.py [case ...]   (about 20 minutes on 8
cores, almost all of it dense521).  Test infrastructure only.
"""
from __future__ import annotations

import hashlib
import importlib.util
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "synthetic"


def _package():
    name = "trhepd_opt_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "trhepd-opt_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def input_sha(d: Path) -> str:
    h = hashlib.sha256()
    for f in ("bulk.txt", "surf.txt", "bulkP.b"):
        h.update((d / f).read_bytes())
    return h.hexdigest()


def structures():
    """name -> (structure factory, selected rows, growth-bound schedule too)."""
    _package()
    from trhepd_opt_b200 import generator
    cases = {
        "batch47": (lambda: generator.batch47(2), None, False),
        "dense521": (lambda: generator.dense(521, seed=3), [0, 8, 17, 25, 34, 42, 51, 60], True),
    }
    for n in (23, 47, 95, 191):
        base = lambda n=n: generator.dense(n, seed=20 + n, n_angles=61, region=15.0, dz=0.02)
        cases[f"uneven{n}"] = (lambda b=base, n=n: generator.jitter(b(), 0.1, 1000 * n),
                               [0, 20, 40, 60], False)
    return cases


def write_inputs(s, d: Path) -> None:
    from trhepd_opt_b200 import bulkfile
    s.write(d)
    bulkfile.write_bulkp(s, d / "bulkP.b")


def make(name: str, tmp: Path) -> None:
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    O.build()
    make_s, idx, growth = structures()[name]
    s = make_s()
    d = tmp / name
    write_inputs(s, d)
    O.set_threads()
    S = O.Surface(d / "bulkP.b", d / "surf.txt", s.surface_dz, s.int_method)
    idx = np.arange(S.n_angles) if idx is None else np.asarray(idx)
    t0 = time.time()
    O.set_renorm_every(0)
    f2, ang, ren = S.solve_list(idx)
    out = {"f2": f2, "angle": ang, "renorm": ren, "idx": idx, "sha": input_sha(d),
           "nb": S.nb, "ns": S.ns, "dz": S.dz}
    if growth:
        L = O.growth_interval(S.kappa_max(), S.dz)
        O.set_renorm_every(L)
        f2g, _, reng = S.solve_list(idx)
        O.set_renorm_every(0)
        out.update({"f2_growth": f2g, "renorm_growth": reng, "interval": L})
    S.close()
    OUT.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(f"{name}: {len(idx)} rows x {S.nb} beams, {S.ns} slices, {time.time() - t0:.0f} s",
          flush=True)


def main(names):
    names = names or list(structures())
    with tempfile.TemporaryDirectory() as t:
        for n in names:
            make(n, Path(t))


if __name__ == "__main__":
    main(sys.argv[1:])
