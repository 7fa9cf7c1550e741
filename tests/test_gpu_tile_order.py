"""Tile-ordered steps (mrlbm_set_tile_order): within one mrlbm_step call a
step launch may start while the one before it finishes, each tile waiting
only for the previous step's 27 tiles around it.  The arithmetic of a tile
does not change, so the moments must be bit-identical to whole-launch
ordering, for every z chunk (1 plane, 2, one chunk per column, uneven last
chunks), tile grids of one tile along an axis, periodic and walled axes,
16-bit storage, and mixes with graph replay and with a z chunk changed
between calls.
"""
import numpy as np
import pytest

import mrlbm

pytestmark = pytest.mark.gpu


def run(desc, steps, chunk=0, order=True, node_types=None, tgv=None, calls=1, graph=False):
    dom = mrlbm.Domain(desc)
    if node_types is not None:
        dom.set_node_types(node_types)
    if tgv:
        dom.init_taylor_green(*tgv)
    dom.set_z_chunk(chunk)
    dom.set_tile_order(order)
    for _ in range(calls):
        if graph:
            dom.step_graph(steps)
        else:
            dom.step(steps)
    dom.synchronize()
    m = dom.moments()
    dom.close()
    return m


def same(a, b):
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), float(np.max(np.abs(a - b)))


@pytest.mark.parametrize("lattice", [mrlbm.D3Q19, mrlbm.D3Q27])
@pytest.mark.parametrize("chunk", [0, 1, 2, 7, 36])
def test_periodic_vortex_bit_identical(lattice, chunk):
    # 70 x 20 x 36: three x tiles (the last partial), 3 or 2 y tiles, and
    # chunks of 1, 2, 7 (uneven last chunk) and 36 (one chunk a column)
    n = (70, 20, 36)
    d = mrlbm.make_desc(*n, lattice=lattice, tau=0.56)
    tg = (0.04, 36 / (2 * np.pi))
    ref = run(d, 9, chunk, order=False, tgv=tg)
    got = run(d, 9, chunk, order=True, tgv=tg)
    same(got, ref)


@pytest.mark.parametrize("lattice", [mrlbm.D3Q19, mrlbm.D3Q27])
def test_lid_cavity_bit_identical(lattice):
    # walls on every face; one x tile, so the x neighbours are the tile itself
    nx, ny, nz = 30, 26, 40
    d = mrlbm.lid_cavity_desc(nx, re=100.0, lid_u=0.05, lattice=lattice, ny=ny, nz=nz)
    nt = mrlbm.lid_cavity_node_types(nx, ny, nz, 1)
    ref = run(d, 25, 3, order=False, node_types=nt)
    got = run(d, 25, 3, order=True, node_types=nt)
    same(got, ref)


def test_fp16_and_repeated_calls_bit_identical():
    # several step calls (each starts with a whole-launch ordered step) and
    # fp16 storage
    d = mrlbm.make_desc(64, 48, 40, lattice=mrlbm.D3Q27, storage=mrlbm.F16, tau=0.6)
    tg = (0.04, 40 / (2 * np.pi))
    ref = run(d, 5, 4, order=False, tgv=tg, calls=3)
    got = run(d, 5, 4, order=True, tgv=tg, calls=3)
    same(got.astype(np.float32), ref.astype(np.float32))


def test_graph_and_chunk_change_mixed():
    """Tile-ordered eager steps, graph replays (whose captured launches order
    whole grids but keep the tile state), a z chunk change (a new tile grid:
    the state is zeroed) and eager steps again, against whole-launch eager
    steps."""
    d = mrlbm.make_desc(64, 40, 48, lattice=mrlbm.D3Q19, tau=0.58)
    tg = (0.05, 48 / (2 * np.pi))

    def seq(order):
        dom = mrlbm.Domain(d)
        dom.init_taylor_green(*tg)
        dom.set_tile_order(order)
        dom.step(7)
        dom.step_graph(33)
        dom.set_z_chunk(5)
        dom.step(6)
        dom.set_z_chunk(0)
        dom.step(4)
        dom.synchronize()
        m = dom.moments()
        dom.close()
        return m

    same(seq(True), seq(False))


def test_large_grid_matches_and_reports_no_timeout():
    """256^3 D3Q27 vortex, 40 steps in one call: the overlapped launches end
    with the same moments and no raised wait flag (synchronize checks it)."""
    n = 256
    d = mrlbm.make_desc(n, n, n, lattice=mrlbm.D3Q27, tau=0.5 + 3 * 0.04 * (n / (2 * np.pi)) / 1600)
    tg = (0.04, n / (2 * np.pi))
    ref = run(d, 40, 0, order=False, tgv=tg)
    got = run(d, 40, 0, order=True, tgv=tg)
    same(got, ref)
