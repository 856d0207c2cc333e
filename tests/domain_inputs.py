"""A two-domain variant of the reference's N = 23 Si(111) case (test23): the
reference ships no multi-domain inputs, so the domain-sum tests rotate the second
domain by 60 deg (the hexagonal cell allows multiples of 60, bulkio.f90:87-99) and
give it the rotated beam set, (h, k) -> (-k, h + k) in the 120-degree basis, so
that every beam of it maps onto a beam of the first domain; weights 0.6 and 0.4
follow the surface atoms in surf.txt (surfio.f90:186-190)."""
from __future__ import annotations

from pathlib import Path


def two_domain_inputs(golden: Path, out: Path, weights=(0.6, 0.4)) -> tuple[Path, Path]:
    out.mkdir(parents=True, exist_ok=True)
    lines = (golden / "test23" / "bulk.txt").read_text().split("\n")
    beams = [int(t) for t in lines[3].split("\t")[0].split(",") if t.strip()]
    pairs = list(zip(beams[0::2], beams[1::2]))
    rot = [(-k, h + k) for h, k in pairs]
    lines[0] = "7,7,2\t\t\t\t\t\t,NH,NK,NDOM"
    lines[1] = f"{len(pairs)},{len(rot)}\t\t\t\t\t,NB"
    lines[2] = "0,60\t\t\t\t\t\t,RDOM"
    lines[3] = ",".join(f"{h},{k}" for h, k in pairs) + "\t,(IH(I),IK(I)"
    lines.insert(4, ",".join(f"{h},{k}" for h, k in rot) + "\t,(IH(I),IK(I)")
    (out / "bulk.txt").write_text("\n".join(lines))
    surf = (golden / "test23" / "surf.txt").read_text().rstrip("\n").split("\n")
    natm_line = next(i for i, ln in enumerate(surf) if ",NATM" in ln)
    natm = int(surf[natm_line].split()[0])
    last = natm_line + natm
    surf.insert(last + 1, ",".join(f"{w:g}" for w in weights) + "\t\t\t,WDOM")
    (out / "surf.txt").write_text("\n".join(surf) + "\n")
    return out / "bulk.txt", out / "surf.txt"
