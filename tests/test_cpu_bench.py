"""Host-side logic of bench.py on CPU: the split of the virtual orbitals into
ranges whose Rkab block fits on the device (the c5 job's 156 GB output)."""
import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import bench  # noqa: E402


def _check(ranges, b0, b1, nvecs, na, free, frac=0.55):
    assert ranges[0][0] == b0 and ranges[-1][1] == b1
    for (p0, p1), (q0, _) in zip(ranges, ranges[1:]):
        assert q0 == p1 + 1
    widths = [q1 - q0 + 1 for q0, q1 in ranges]
    assert min(widths) >= 1
    # every block fits, unless a single virtual orbital already does not
    assert max(widths) == 1 or 8.0 * nvecs * na * max(widths) <= frac * free


def test_c2_output_in_one_piece():
    r = bench.virtual_ranges(16285, 60, 61, 960, 160e9)
    assert r == [(61, 960)]


def test_c5_output_in_two_ranges():
    # 48,073 vectors x 150 occupied x 2700 virtual = 156 GB against ~160 GB free
    r = bench.virtual_ranges(48073, 150, 151, 2850, 160e9)
    assert r == [(151, 1500), (1501, 2850)]
    _check(r, 151, 2850, 48073, 150, 160e9)


@pytest.mark.parametrize("nvecs,na,b0,b1,free", [(1000, 10, 11, 20, 1e5), (5000, 3, 4, 1003, 2e8),
                                                  (7, 1, 2, 2, 1.0), (100, 100, 101, 5100, 3e9)])
def test_ranges_cover_and_fit(nvecs, na, b0, b1, free):
    _check(bench.virtual_ranges(nvecs, na, b0, b1, free), b0, b1, nvecs, na, free)
