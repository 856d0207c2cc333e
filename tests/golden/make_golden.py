"""Extract the reference's own regression data into small fixtures.

Reads the reference checkout (its path is the required first argument) and
writes, per test case (test23 / test47 / test521):

* ``<case>/bulkP.b``, ``<case>/surf.txt``, ``<case>/bulk.txt`` — the inputs the
  reference's regression runs used (test/<case>/);
* ``<case>/perf-<method>-<dz>.npz`` — angles and intensities of the committed
  outputs test/<case>/test-results/perf-<method>-<dz>.txt (E23.15, 15 digits),
  for the integrators and slice thicknesses listed below;
* ``conv-<name>.npz`` — a sample's rocking curves (surf-bulkP.s) and the
  convolution.txt the reference's make_convolution.py wrote from them;
* ``ge001/`` — the Ge(001) sample's bulk.txt, surf.txt and the bulkP.b the
  reference wrote from them (sim-trhepd-rheed/sample/Ge_001_c4x2), the only
  reference output with a Z = 32 element;
* ``test23/accurate.npz`` — the converged curves surf-bulkP-str-accurate.s (sp4,
  dz 0.001, E23.15) and, per (method, dz) of the perf fixtures, the first
  repetition of the per-angle rows compare.py printed against them
  (test-results/perf-comp-acc.txt: angle, e0 / max n0, e0 / n0).

Run once in a container that has the reference; the fixtures travel with the
repository and nothing at test time reads the reference.
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SEL = {
    "test23": [(m, dz) for m in (4, 5, 6, 7) for dz in ("0.68", "0.1", "0.022")],
    "test47": [(m, dz) for m in (5, 6) for dz in ("0.68", "0.22")] + [(7, "0.22")],
    "test521": [(5, "0.68"), (6, "0.68"), (5, "0.33"), (6, "0.33")],
}


CONV = [("ge001", "sim-trhepd-rheed", "Ge_001_c4x2"), ("t4al", "str-lapack", "T4Al_on_Si_111")]


def parse_s(path):
    sys.path.insert(0, str(HERE.parents[1] / "trhepd-opt_b200"))
    from formats import read_rocking_curves
    return read_rocking_curves(path)


def main(ref: Path):
    for case, sel in SEL.items():
        src = ref / "test" / case
        dst = HERE / case
        dst.mkdir(parents=True, exist_ok=True)
        for f in ("bulkP.b", "surf.txt", "bulk.txt"):
            shutil.copyfile(src / f, dst / f)
        for m, dz in sel:
            p = src / "test-results" / f"perf-{m}-{dz}.txt"
            ang, f2, hdr = parse_s(p)
            np.savez_compressed(dst / f"perf-{m}-{dz}.npz", angle=ang, f2=f2,
                                beams=hdr["beams"], naz=hdr["naz"], ng=hdr["ng"])
    # the Ge(001) sample: inputs and the bulkP.b the reference wrote from them
    src = ref / "sim-trhepd-rheed" / "sample" / "Ge_001_c4x2"
    dst = HERE / "ge001"
    dst.mkdir(parents=True, exist_ok=True)
    for f in ("bulk.txt", "surf.txt"):
        shutil.copyfile(src / f, dst / f)
    shutil.copyfile(src / "output" / "bulkP.b", dst / "bulkP.b")
    # converged curves and the comparison metric printed against them
    src = ref / "test" / "test23"
    ang, f2, hdr = parse_s(src / "surf-bulkP-str-accurate.s")
    rows = {}
    for line in (src / "test-results" / "perf-comp-acc.txt").read_text().split("\n"):
        t = line.split()
        if len(t) != 7:
            continue
        key = f"comp-{t[2]}-{t[3]}"
        if (int(t[2]), t[3]) not in SEL["test23"]:
            continue
        r = rows.setdefault(key, [])
        if len(r) < len(ang):  # compare.py ran once per repetition; keep the first
            r.append([float(t[4]), float(t[5]), float(t[6])])
    np.savez_compressed(HERE / "test23" / "accurate.npz", angle=ang, f2=f2,
                        beams=hdr["beams"], **{k: np.array(v) for k, v in rows.items()})
    # rocking-curve convolution samples: the reference's surf-bulkP.s and the
    # convolution.txt its make_convolution.py wrote from it (omega 0.5 deg)
    for name, tree, samp in CONV:
        src = ref / tree / "sample" / samp / "output"
        ang, f2, hdr = parse_s(src / "surf-bulkP.s")
        conv = np.loadtxt(src / "convolution.txt")
        np.savez_compressed(HERE / f"conv-{name}.npz", angle=ang, f2=f2, beams=hdr["beams"],
                            conv=conv[:, 1:], conv_angle=conv[:, 0])
    print("fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference checkout>")
    main(Path(sys.argv[1]))
