"""The pass geometry the planner reads (orot_b200/csrc/geometry_table.h),
checked through the library without a GPU: every row boundary belongs to
its own row, sizes scale with the device's SM count, and the table's rows
are ordered and hold valid tiles."""
import re
import os

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _rows():
    text = open(os.path.join(ROOT, "orot_b200", "csrc", "geometry_table.h")).read()
    rows = []
    for m in re.finditer(r"\{(\d+)ull(?: << (\d+))?, (\d+), (\d+), \{(\d+), (\d+), (\d+)\}\}", text):
        lo = int(m.group(1)) << int(m.group(2) or 0)
        rows.append((lo, int(m.group(3)), int(m.group(4))))
    return rows


@pytest.fixture(scope="module")
def deflate():
    from orot_b200 import deflate as d
    return d


def test_table_rows_are_ordered_and_valid():
    rows = _rows()
    assert rows and rows[0][0] == 0
    assert [r[0] for r in rows] == sorted(r[0] for r in rows)
    for _, t12, t14 in rows:
        for t in (t12, t14):
            assert t >= 4096 and t & (t - 1) == 0 and t % 32 == 0


def test_each_boundary_belongs_to_its_row(deflate):
    rows = _rows()
    for i, (lo, t12, t14) in enumerate(rows):
        assert deflate.geometry_tile(lo, 148, 12) == t12, lo
        assert deflate.geometry_tile(lo, 148, 14) == t14, lo
        if lo:
            prev = rows[i - 1]
            assert deflate.geometry_tile(lo - 1, 148, 12) == prev[1], lo
            assert deflate.geometry_tile(lo - 1, 148, 14) == prev[2], lo


def test_sizes_scale_with_the_sm_count(deflate):
    rows = _rows()
    for lo, t12, _ in rows[1:]:
        # half the SMs: half the bytes reach the same row
        assert deflate.geometry_tile(lo // 2, 74, 12) == t12, lo
        assert deflate.geometry_tile(lo * 2, 296, 12) == t12, lo
