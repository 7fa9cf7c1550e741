"""Golden _info.txt texts, checked with the reference's own reader.

    MRLBM_REFERENCE=<reference checkout> python tests/golden/make_info_golden.py

Formats the simulation-information file of two descriptions with the library
(mrlbm_info_text, the same text mrlbm_save_info writes), parses each with the
reference's post/fileTreat.py getSimInfo (imported from the reference
checkout; test infrastructure only), checks that every key it reads has the
description's value, and writes the texts and the parsed dictionaries to
tests/golden/info_golden.json.  tests/test_info_format.py then checks that the
library still writes exactly these texts.
"""
import importlib.util
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "mr-lbm_b200"))
import mrlbm  # noqa: E402


def cases():
    tg = mrlbm.make_desc(256, 256, 256, lattice=27, tau=0.50305577)
    pl = mrlbm.make_desc(96, 64, 48, lattice=19, periodic=(0, 0, 1), tau=0.8, force=(0.0, 0.0, 2.5e-6),
                         rheology=mrlbm.POWERLAW, nnf_n=0.7, nnf_k=0.1)
    return [("tgv", tg, "000", "taylorGreen", 1000, 51234.5), ("duct", pl, "001", "duct", 20000, 4321.0)]


def reference_parser(ref_root):
    spec = importlib.util.spec_from_file_location("fileTreat", os.path.join(ref_root, "post", "fileTreat.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def parse_with_reference(ft, text, tmpdir, sim_id):
    os.makedirs(tmpdir, exist_ok=True)
    with open(os.path.join(tmpdir, sim_id + "_info.txt"), "w") as f:
        f.write(text)
    ft.__info__.clear()
    return dict(ft.getSimInfo(tmpdir + "/"))


def main():
    import tempfile

    ref = os.environ.get("MRLBM_REFERENCE")
    if not ref:
        raise SystemExit("set MRLBM_REFERENCE to the reference checkout")
    ft = reference_parser(ref)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for key, d, sim_id, case_name, nsteps, mlups in cases():
            text = mrlbm.info_text(d, sim_id, case_name, nsteps, mlups)
            parsed = parse_with_reference(ft, text, os.path.join(tmp, key), sim_id)
            want = {"ID": sim_id, "NX": d.nx, "NY": d.ny, "NZ": d.nz, "NZ_TOTAL": d.nz, "Nsteps": nsteps,
                    "FX": d.force[0], "FY": d.force[1], "FZ": d.force[2]}
            for k, v in want.items():
                assert parsed[k] == v or abs(parsed[k] - v) <= 1e-6 * max(1.0, abs(v)), (key, k, parsed[k], v)
            assert abs(parsed["Tau"] - d.tau) < 1e-6
            out[key] = {"text": text, "parsed": parsed}
    with open(os.path.join(HERE, "info_golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "info_golden.json"))


if __name__ == "__main__":
    main()
