"""Host-side figures of bench.py that need no GPU: the forcing spread's
roofline inputs (force tiles, list entries and touched cells of the markers'
4 x 4 stencils) on hand-checked marker sets."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


class _Params:
    def __init__(self, nx, ny):
        self.nx, self.ny = nx, ny


class _Plan:
    def __init__(self, nx, ny):
        self.params = _Params(nx, ny)


class _View:
    def __init__(self, X):
        self._X = np.asarray(X, dtype=np.float64)

    def positions(self):
        return self._X.ravel()


class _Ens:
    def __init__(self, per_channel):
        self._p = per_channel

    def capsules(self, i):
        return _View(self._p[i])


def test_single_marker_inside_one_tile():
    # stencil columns 9..12, rows 2..5: one tile (0, 0), 16 cells
    ens = _Ens([[(10.3, 3.6)]])
    assert bench.spread_geometry(ens, [_Plan(64, 16)]) == (1, 1, 16)


def test_marker_across_tile_row_and_column():
    # columns 30..33 cross x = 32, rows 6..9 cross y = 8: four tiles
    ens = _Ens([[(31.5, 7.5)]])
    assert bench.spread_geometry(ens, [_Plan(64, 16)]) == (4, 4, 16)


def test_periodic_seam_and_wall_rows():
    # columns 63, 0, 1, 2 (seam of a 64-wide channel) and rows -1..2: the
    # row below the lattice is dropped (12 cells), the stencil touches
    # tiles (1, 0) and (0, 0)
    ens = _Ens([[(0.5, 0.2)]])
    assert bench.spread_geometry(ens, [_Plan(64, 16)]) == (2, 2, 12)


def test_shared_cells_counted_once_and_channels_summed():
    # two markers in neighbouring cells share 12 of their 16 stencil cells
    # (columns 9..12 and 10..13); a second channel adds one marker of its own
    ens = _Ens([[(10.7, 3.5), (11.2, 3.5)], [(5.5, 5.5)]])
    slots, entries, touched = bench.spread_geometry(ens, [_Plan(64, 16), _Plan(32, 16)])
    assert (slots, entries) == (2, 3)
    assert touched == (16 + 4) + 16


def test_roofline_bytes():
    ens = _Ens([[(10.3, 3.6)]])
    r = bench.spread_roofline(ens, [_Plan(64, 16)], spread_ms=1.0, sweeps=3, peak=1000.0,
                              peak_kind="test")
    alg = 3 * 1 * bench.SPREAD_ENTRY_BYTES + 16 * 8 * 4 + 1 * bench.SLOT_FINAL_BYTES
    assert r["algorithmic_bytes_per_step"] == alg
    assert abs(r["achieved"] - alg / 1e-3 / 1e9) < 1e-9
