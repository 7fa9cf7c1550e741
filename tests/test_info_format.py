"""The simulation-information file (_info.txt) in the reference's format.

tests/golden/info_golden.json holds texts that the reference's own reader
(post/fileTreat.py getSimInfo, src/saveData.cu:469-613 writes the format) was
checked to parse into the descriptions' values when the fixture was made
(tests/golden/make_info_golden.py).  The library must still write exactly
these texts (mrlbm_info_text, the text mrlbm_save_info writes); when the
environment variable MRLBM_REFERENCE names a reference checkout, the
reference's reader parses them again here.
"""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_info_golden as mig  # noqa: E402


def golden():
    with open(os.path.join(HERE, "golden", "info_golden.json")) as f:
        return json.load(f)


def test_info_text_is_the_golden_text():
    g = golden()
    for key, d, sim_id, case_name, nsteps, mlups in mig.cases():
        assert mig.mrlbm.info_text(d, sim_id, case_name, nsteps, mlups) == g[key]["text"], key


def test_reference_reader_parses_the_info_text(tmp_path):
    ref = os.environ.get("MRLBM_REFERENCE")
    if not ref or not os.path.exists(os.path.join(ref, "post", "fileTreat.py")):
        pytest.skip("MRLBM_REFERENCE does not name a reference checkout")
    ft = mig.reference_parser(ref)
    g = golden()
    for key, d, sim_id, case_name, nsteps, mlups in mig.cases():
        text = mig.mrlbm.info_text(d, sim_id, case_name, nsteps, mlups)
        assert mig.parse_with_reference(ft, text, str(tmp_path / key), sim_id) == g[key]["parsed"], key
