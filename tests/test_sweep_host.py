"""The sweep's host side: sampling, the shocked-band refusal and the result table (no GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import pkg


def test_sampling_is_seeded_and_in_range():
    sw = pkg("sweep")
    a, b = sw.sample_points(64, 0), sw.sample_points(64, 0)
    assert a == b and a != sw.sample_points(64, 1)
    assert all(1.5 <= p.area_ratio <= 4.0 and 0.1 <= p.back_pressure_ratio <= 0.9 for p in a)
    assert {p.order for p in a} == {1, 2, 3} and {p.refine for p in a} == {1, 2, 3}
    assert {p.element for p in a} == {"tri", "quad"}


def test_shocked_points_are_refused():
    sw = pkg("sweep")
    pts = [sw.Point(2.5, 0.15, 1, 1, "tri"), sw.Point(2.5, 0.8, 1, 1, "tri")]
    insts, index, refused = sw.build_instances(pts, max_iterations=10)
    assert index == [0] and refused == [1] and len(insts) == 1


def test_result_table_and_csv(tmp_path):
    sw = pkg("sweep")
    pts = [sw.Point(2.0, 0.15, 1, 1, "tri"), sw.Point(3.0, 0.8, 2, 1, "quad")]
    values = {m: np.array([float(i + 1), np.nan]) for i, m in enumerate(sw.METRICS)}
    res = sw.SweepResult(pts, values, np.array([True, False]), ["converged", "refused"], np.array([120, 0]),
                         ["", "shock"])
    assert res.n_points == 2 and not res.all_converged
    assert list(res["area_ratio"]) == [2.0, 3.0] and res["thrust"][0] == 1.0
    assert res.failures() == [(pts[1], "shock")]
    with pytest.raises(KeyError):
        res["nope"]
    assert "thrust_coefficient" in res.table().splitlines()[0]
    path = tmp_path / "sweep.csv"
    res.to_csv(str(path))
    lines = path.read_text().splitlines()
    assert len(lines) == 3 and lines[0].startswith("area_ratio,back_pressure_ratio,order,refine,element,thrust")
    assert lines[2].endswith("False,refused,0")
