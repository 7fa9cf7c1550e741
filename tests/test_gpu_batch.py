"""Batched persistent kernel: every member evolves exactly as it would alone.

Each node's update reads the same stored moments and does the same arithmetic
whichever CTA (and whichever z chunk) computes it, so a member of a batch must
be bit-identical to the same domain stepped alone by the single-domain kernel.
"""
import numpy as np
import pytest

import mrlbm
import parity_util as pu

pytestmark = pytest.mark.gpu


def cavity(n, re, storage=mrlbm.F32, ny=None, nz=None):
    d = mrlbm.lid_cavity_desc(n, re=re, lid_u=0.05, storage=storage, ny=ny, nz=nz)
    return d, mrlbm.lid_cavity_node_types(n, ny or n, nz or n, 1)


def duct(n, seed, storage=mrlbm.F32):
    rng = np.random.default_rng(seed)
    solid = np.zeros((n, n, n), dtype=np.uint8)
    solid[:, 1:-1, 1:-1] = rng.random((n, n - 2, n - 2)) < 0.05
    nt = mrlbm.voxel_node_types(solid, (0, 0, 1))
    d = mrlbm.make_desc(n, n, n, lattice=19, storage=storage, periodic=(0, 0, 1), tau=0.8, force=(0, 0, 2e-5),
                        rheology=mrlbm.POWERLAW, nnf_n=float(rng.uniform(0.6, 1.2)))
    return d, nt


def run_alone(desc, nt, steps):
    dom = mrlbm.Domain(desc)
    dom.set_node_types(nt)
    dom.init_uniform()
    dom.step(steps)
    m = dom.moments()
    dom.close()
    return m


@pytest.mark.parametrize("storage,rows", [(mrlbm.F32, 8), (mrlbm.F16, 8), (mrlbm.F32, 14), (mrlbm.F16U, 14)])
def test_batch_members_equal_alone(storage, rows):
    """Both tile heights of the batch kernel (8 rows, two CTAs an SM; 14, one)."""
    cases = [cavity(24, 100, storage), cavity(37, 400, storage, ny=29, nz=41), cavity(50, 1000, storage),
             cavity(33, 60, storage, ny=47, nz=26), duct(28, 1, storage), duct(35, 2, storage)]
    steps = 40
    b = mrlbm.Batch(mrlbm.D3Q19, storage)
    b.set_rows(rows)
    assert b.rows() == rows
    mem = []
    for d, nt in cases:
        m = b.add(d)
        m.set_node_types(nt)
        m.init_uniform()
        mem.append(m)
    b.step(steps)          # 40 = 2 graph replays of 16 + 8 eager launches
    b.synchronize()
    info = b.info()
    assert info["members"] == len(cases) and info["items"] > len(cases)
    for (d, nt), m in zip(cases, mem):
        np.testing.assert_array_equal(m.moments(), run_alone(d, nt, steps))
    b.close()


def test_batch_admission_and_removal_mid_run():
    """Members joining and leaving between steps do not disturb the others."""
    a_desc, a_nt = cavity(30, 200)
    c_desc, c_nt = cavity(26, 500)
    b = mrlbm.Batch()
    a = b.add(a_desc)
    a.set_node_types(a_nt)
    a.init_uniform()
    b.step(7)                      # odd: a's parity differs from a newcomer's
    c = b.add(c_desc)
    c.set_node_types(c_nt)
    c.init_uniform()
    b.step(20)
    b.remove(c)
    b.step(5)
    np.testing.assert_array_equal(a.moments(), run_alone(a_desc, a_nt, 32))
    b.close()


def test_batch_matches_oracle():
    d, nt = cavity(20, 150)
    b = mrlbm.Batch()
    m = b.add(d)
    m.set_node_types(nt)
    m.init_uniform()
    m0 = m.moments()
    b.step(60)
    orc = pu.oracle_for(d, nt)
    orc.set_moments(pu.gpu_to_oracle_layout(m0))
    orc.step(60)
    res = pu.compare(m.moments(), orc.moments())
    for k, (e2, einf) in res.items():
        assert e2 < (3e-4 if 4 <= k <= 9 else 5e-5), (k, e2)
    b.close()


def test_batch_autotune_keeps_results():
    cases = [cavity(n, 100 + 10 * n) for n in (24, 40, 64)]
    b = mrlbm.Batch()
    mem = []
    for d, nt in cases:
        m = b.add(d)
        m.set_node_types(nt)
        m.init_uniform()
        mem.append(m)
    b.step(6)
    before = [(m.step_count, m.moments()) for m in mem]
    b.autotune()                   # times candidate chunks and tile heights on the members, then restores them
    assert b.rows() in (8, 14)
    with pytest.raises(mrlbm.MrlbmError):
        b.set_rows(10)
    for (steps, mom), m in zip(before, mem):
        assert m.step_count == steps == 6
        np.testing.assert_array_equal(m.moments(), mom)
    b.step(10)
    for (d, nt), m in zip(cases, mem):
        np.testing.assert_array_equal(m.moments(), run_alone(d, nt, 16))
        assert 1 <= b.chunk_for(d.nx, d.ny, d.nz) <= d.nz
    b.close()
