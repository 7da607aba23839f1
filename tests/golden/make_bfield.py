"""Write the From1dXFile fixtures of this directory with the reference's own
writer, tools/makeBfld.py:write_1d_field (header int32 n, float32 d, then
n + 1 float32 values), which EMField.mm:658-687 reads back.

Usage: python tests/golden/make_bfield.py /path/to/gample

It also runs tools/makeBfld.py itself, unmodified, in a scratch directory:
its main block writes the Hall-thruster profile of data/org_3rd.json
(data/Bx_3rd.bin, By_3rd.bin, Bz_3rd.bin for ngx = 500, ngb = 1), copied
here as Bx_3rd.bin, By_3rd.bin, Bz_3rd.bin.

Grid of the small fixtures: ngx = 48, weighting order 3 (ngb = 1), so nx = 50 and
dx = 0.005 cm; the arrays have the lengths EMField.mm:175-197 indexes: Bx
nx + 1 values, By and Bz nx + 2. The profile is a magnetic-field bump in
tesla, Bz(x) = 6 mT + 4 mT exp(-(x - 0.12 cm)^2 / (2 (0.05 cm)^2)) at the
half-shifted nodes x = (i + 0.5) dx, and a weaker, linear By.
"""
import importlib.util
import os
import sys

import numpy as np

NGX, NGB, DX = 48, 1, 0.005


def main(src):
    spec = importlib.util.spec_from_file_location("makeBfld", os.path.join(src, "tools", "makeBfld.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    here = os.path.dirname(os.path.abspath(__file__))
    nx = NGX + 2 * NGB
    x = (np.arange(nx + 2) + 0.5) * DX
    bz = 6e-3 + 4e-3 * np.exp(-0.5 * ((x - 0.12) / 0.05) ** 2)
    by = 1e-4 * x / x[-1]
    mod.write_1d_field(os.path.join(here, "Bz_1dx.bin"), nx + 1, DX, bz)
    mod.write_1d_field(os.path.join(here, "By_1dx.bin"), nx + 1, DX, by)
    mod.write_1d_field(os.path.join(here, "Bx_1dx.bin"), nx, DX, np.zeros(nx + 1))
    print("wrote Bx_1dx.bin, By_1dx.bin, Bz_1dx.bin to", here)
    import runpy
    import shutil
    import tempfile
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.makedirs(os.path.join(td, "data"))
        os.chdir(td)
        try:
            runpy.run_path(os.path.join(src, "tools", "makeBfld.py"), run_name="__main__")
        finally:
            os.chdir(cwd)
        for c in ("x", "y", "z"):
            shutil.copyfile(os.path.join(td, "data", f"B{c}_3rd.bin"), os.path.join(here, f"B{c}_3rd.bin"))
    print("wrote Bx_3rd.bin, By_3rd.bin, Bz_3rd.bin (tools/makeBfld.py) to", here)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_bfield.py /path/to/gample")
    main(sys.argv[1])
