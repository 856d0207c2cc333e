"""The schedule tuner: every candidate runs, the chosen split schedule meets the
error bound against FP64 on its problem, and a context configured with a chosen
schedule solves to the same intensities as the tuner saw."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tune_small_and_medium(tmp_path):
    from trhepd_opt_b200 import autotune, build, native
    build.build()
    ctx = native.Context(0)
    try:
        table = autotune.tune(ctx, beam_counts=(23, 95), angles=6, region=1.0)
        assert set(table) == {23, 95}
        for n, e in table.items():
            names = {c.name for c in autotune.candidates(n)}
            assert set(e["times_ms"]) == names
            assert all(t > 0 for t in e["times_ms"].values())
            assert e["fp64"] in names and e["split"] in names
            if e["split"] != e["fp64"]:
                assert e["errors"][e["split"]] <= 1e-6
        assert "fp64-fused" in table[23]["times_ms"] and "fp64-fused" not in table[95]["times_ms"]
        autotune.save(table, tmp_path / "t.json")
        assert autotune.load(tmp_path / "t.json")[95]["split"] == table[95]["split"]
    finally:
        ctx.close()
