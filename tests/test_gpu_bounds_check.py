"""The bounds-check build (libmrlbm_check.so, -DMRLBM_BOUNDS_CHECK) on the
edge shapes of every step-kernel family (tests/bounds_cases.py): no kernel
skips an out-of-range shared-memory or global access (the device error word
stays clear: no MRLBM_EBOUNDS), and the moments equal the product build's bit
for bit, which they can only do if no consumption read an exchange or edge
slot that the production before it left unwritten (those are NaN-poisoned in
the check build)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import bounds_cases

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CHECK_LIB = os.path.join(os.path.dirname(HERE), "mr-lbm_b200", "libmrlbm_check.so")


def test_check_build_finds_nothing_and_matches_the_product_build(tmp_path):
    assert os.path.exists(CHECK_LIB), "bounds-check build missing (mr-lbm_b200/build.py builds it)"
    out = str(tmp_path / "check.npz")
    env = dict(os.environ, MRLBM_LIBRARY=CHECK_LIB)
    r = subprocess.run([sys.executable, os.path.join(HERE, "bounds_cases.py"), out], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "libmrlbm_check.so" in r.stdout
    checked = np.load(out)
    product = bounds_cases.run_all()
    assert sorted(checked.files) == sorted(product)
    for k, v in product.items():
        assert np.all(np.isfinite(v)), k
        assert np.array_equal(checked[k], v), k
