"""mrlbm_reduce_fp64_ref_layout_noalloc: FP64 sums of a caller-owned device
field in the reference's idxMom layout, with scratch in a static device array
instead of an allocation.  Checked through the C ABI against the domain
reduction (mrlbm_reduce_fp64) on the same values, two calls in a row on each
of two fields.  The caller-owned device buffer is a torch tensor (test-side
plumbing only).  Named to be collected last; it also passes on its own in a
fresh process.
"""
import numpy as np
import pytest

import mrlbm

pytestmark = pytest.mark.gpu

KEYS = ("mass", "momentum", "kinetic_energy", "fluid_nodes", "max_speed", "nonfinite")


def field_pair(lattice, nx, ny, nz, seed):
    """A stepped F32 periodic domain and its moments in the idxMom layout on the device."""
    import torch

    d = mrlbm.make_desc(nx, ny, nz, lattice=lattice, tau=0.7)
    dom = mrlbm.Domain(d)
    rng = np.random.default_rng(seed)
    rho = 1 + 0.01 * rng.standard_normal((nz, ny, nx))
    u = 0.03 * rng.standard_normal((3, nz, ny, nx))
    dom.init_flow(rho, u[0], u[1], u[2])
    dom.step(7)
    host = np.ascontiguousarray(dom.moments_ref_layout(), dtype=np.float32)
    dev = torch.from_numpy(host).to("cuda:0")
    torch.cuda.synchronize()
    return dom, dev


def close(a, b):
    for k in KEYS:
        np.testing.assert_allclose(np.asarray(a[k], dtype=np.float64), np.asarray(b[k], dtype=np.float64),
                                   rtol=1e-12, atol=1e-12, err_msg=k)


def equal(a, b):
    for k in KEYS:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_noalloc_reduction_matches_domain_reduction_two_calls_in_a_row():
    import torch

    dom1, dev1 = field_pair(mrlbm.D3Q19, 48, 40, 32, 1)
    dom2, dev2 = field_pair(mrlbm.D3Q27, 64, 32, 40, 2)
    try:
        ref1, ref2 = dom1.sums(), dom2.sums()
        # two calls in a row on the first field, then two on the second
        a1 = mrlbm.reduce_ref_layout_noalloc(dev1.data_ptr(), 48, 40, 32, dom1.nm, 1.0)
        b1 = mrlbm.reduce_ref_layout_noalloc(dev1.data_ptr(), 48, 40, 32, dom1.nm, 1.0)
        s = torch.cuda.Stream()
        a2 = mrlbm.reduce_ref_layout_noalloc(dev2.data_ptr(), 64, 32, 40, dom2.nm, 1.0, s.cuda_stream)
        b2 = mrlbm.reduce_ref_layout_noalloc(dev2.data_ptr(), 64, 32, 40, dom2.nm, 1.0, s.cuda_stream)
        equal(a1, b1)
        equal(a2, b2)
        close(a1, ref1)
        close(a2, ref2)
        assert a1["fluid_nodes"] == 48 * 40 * 32 and a2["fluid_nodes"] == 64 * 32 * 40
        assert a1["nonfinite"] == 0 and a2["nonfinite"] == 0
        # the first field again after the second: nothing stale in the scratch
        equal(mrlbm.reduce_ref_layout_noalloc(dev1.data_ptr(), 48, 40, 32, dom1.nm, 1.0), a1)
    finally:
        dom1.close()
        dom2.close()


def test_noalloc_reduction_strides_over_fields_larger_than_its_grid():
    # 96 x 64 x 64 = 393,216 nodes: more than the 592 blocks x 256 threads
    # (151,552) the call launches, so every thread loops over several nodes
    dom, dev = field_pair(mrlbm.D3Q19, 96, 64, 64, 3)
    try:
        ref = dom.sums()
        a = mrlbm.reduce_ref_layout_noalloc(dev.data_ptr(), 96, 64, 64, dom.nm, 1.0)
        b = mrlbm.reduce_ref_layout_noalloc(dev.data_ptr(), 96, 64, 64, dom.nm, 1.0)
        equal(a, b)
        close(a, ref)
        assert a["fluid_nodes"] == 96 * 64 * 64 and a["nonfinite"] == 0
    finally:
        dom.close()


def test_noalloc_reduction_rejects_bad_arguments_before_launching():
    import torch

    host = np.zeros(8 * 8 * 8 * 10, dtype=np.float32)
    with pytest.raises(mrlbm.MrlbmError, match="not device memory"):
        mrlbm.reduce_ref_layout_noalloc(host.ctypes.data, 8, 8, 8, 10)
    dev = torch.zeros(12 * 8 * 8 * 10, dtype=torch.float32, device="cuda:0")
    with pytest.raises(mrlbm.MrlbmError, match="multiples of 8"):
        mrlbm.reduce_ref_layout_noalloc(dev.data_ptr(), 12, 8, 8, 10)
    with pytest.raises(mrlbm.MrlbmError, match="null argument"):
        mrlbm.reduce_ref_layout_noalloc(0, 8, 8, 8, 10)
