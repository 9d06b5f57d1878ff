"""The research bench (basements_b200.research) on the CUDA couplers: every
scene with every coupler (M0, M1, M4.5a, M4.5b, M4.5), the CSV files
written in the reference's formats, their metrics against the shipped ones
and the findings of scripts/reproduce_findings.py reaching the verdicts the
reference's own outputs reach."""
import os

import pytest

import basements_b200 as bm
from basements_b200 import research as RS
from tests.test_research import check_record, shipped, write_shipped

pytestmark = pytest.mark.gpu


def test_research_bench_reproduces_the_reference_findings(tmp_path):
    out = str(tmp_path / "gpu")
    RS.run_all(out, lambda sc, coupler: RS.GpuGrid(bm, sc, coupler))
    checked = 0
    for method in RS.METHODS:
        for scene in ("box_drop_dense", "foot_step", "tine_drag", "rover_wheel"):
            ref = shipped(scene, method)
            if ref is None:
                continue
            got = {}
            for kind in ("metrics", "summary", "roll", "rebound"):
                path = os.path.join(out, f"{scene}_{method}_{kind}.csv")
                if os.path.exists(path):
                    names, vals = [line.strip().split(",") for line in open(path)][:2]
                    got.setdefault(kind, {}).update({n: float(v) for n, v in zip(names[1:], vals[1:])})
            # the CUDA couplers sum their reactions in another order (the
            # research-scene bars: 1e-4 relative)
            checked += check_record(got, ref, (scene, method), rel_default=1e-4)
    assert checked >= 60
    ship = str(tmp_path / "shipped")
    write_shipped(ship)
    ours = RS.findings(out)
    for name, ok, msg in ours:
        print(f"{'PASS' if ok else 'FAIL'}  {name}: {msg}")
    assert [ok for _, ok, _ in ours] == [ok for _, ok, _ in RS.findings(ship)]
