"""Host-side model of k_vp_tb2's tile layout (hm_vpipes_tb.cu), on the CPU.

The two-step vpipes kernel walks rings of width 6, 5, 4, 2, 1 and 0 around
its output tile, clipped to the grid, and indexes one shared-memory array per
field by grid coordinates.  This model repeats that arithmetic for every
tile of many grids and both tile shapes and checks that every index stays in
the field arrays and that every read is of a cell an earlier pass wrote.  It
also checks the row decode the kernel uses instead of an integer division.
"""
import numpy as np
import pytest

HX = 4             # ring of the first step's eroded sediment
H1, H2 = HX + 1, HX + 2


def _region(x0, y0, h, nx, ny, tx, ty):
    xa, xb = max(0, x0 - h), min(nx - 1, x0 + tx - 1 + h)
    ya, yb = max(0, y0 - h), min(ny - 1, y0 + ty - 1 + h)
    return [(x, y) for y in range(ya, yb + 1) for x in range(xa, xb + 1)]


def _check_grid(nx, ny, tx, ty):
    w, h = tx + 2 * H2, ty + 2 * H2
    for y0 in range(0, ny, ty):
        for x0 in range(0, nx, tx):
            ox, oy = x0 - H2, y0 - H2

            def at(x, y):
                assert 0 <= x < nx and 0 <= y < ny
                cx, cy = x - ox, y - oy
                assert 0 <= cx < w and 0 <= cy < h, (nx, ny, x0, y0, x, y)
                return cy * w + cx

            def nb(x, y):
                return {at(x, y), at(max(x - 1, 0), y), at(min(x + 1, nx - 1), y), at(x, max(y - 1, 0)),
                        at(x, min(y + 1, ny - 1))}

            zd = {at(x, y) for x, y in _region(x0, y0, H2, nx, ny, tx, ty)}          # A: z, start depth
            fs = {at(x, y) for x, y in _region(x0, y0, H1, nx, ny, tx, ty)}          # A: fluxes, sediment
            for x, y in _region(x0, y0, H1, nx, ny, tx, ty):                         # B: first flow
                assert nb(x, y) <= zd and at(x, y) in fs
            first = set()
            for x, y in _region(x0, y0, HX, nx, ny, tx, ty):                         # C: first water, erosion
                assert nb(x, y) <= fs
                first.add(at(x, y))
            d1 = set()
            for x, y in _region(x0, y0, 2, nx, ny, tx, ty):                          # D: second start depth
                assert at(x, y) in first
                d1.add(at(x, y))
            # taps of the second advection inside the first step's ring read shared memory
            for x in range(max(0, x0 - HX), min(nx, x0 + tx + HX)):
                for y in (max(0, y0 - HX), min(ny - 1, y0 + ty - 1 + HX)):
                    assert at(x, y) in first
            sed = {at(x, y) for x, y in _region(x0, y0, 1, nx, ny, tx, ty)}
            assert sed <= first
            for x, y in _region(x0, y0, 1, nx, ny, tx, ty):                          # E: second flow
                assert nb(x, y) <= d1 and nb(x, y) <= first
            for x, y in _region(x0, y0, 0, nx, ny, tx, ty):                          # F: second water, erosion
                assert nb(x, y) <= sed


@pytest.mark.parametrize("tile", [(32, 16), (16, 8)])
@pytest.mark.parametrize("grid", [(1, 1), (1, 5), (5, 1), (2, 3), (7, 9), (31, 15), (32, 16), (33, 17), (44, 28),
                                  (64, 33), (97, 131), (131, 97), (300, 5), (5, 300)])
def test_regions_stay_in_shared_memory(grid, tile):
    _check_grid(*grid, *tile)


def test_row_decode_is_exact():
    """Row of item e of a region w cells wide: (e + 0.5) * RN(1/w), each
    operation rounded to fp32, truncated; equals e // w for every w < 64 and
    e < 4096 (the kernel's regions are at most 44 wide and 1232 cells)."""
    e = np.arange(4096, dtype=np.int64)
    ef = e.astype(np.float32)
    for w in range(1, 64):
        rw = np.float32(1.0) / np.float32(w)
        q = ((ef + np.float32(0.5)) * rw).astype(np.float32).astype(np.int64)
        assert np.array_equal(q, e // w), w
