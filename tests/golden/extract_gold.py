"""Extract the reference's gold plotfiles used to pin the oracle into .npz
fixtures (run in a checkout that has the reference tree):

    python tests/golden/extract_gold.py /path/to/ERF

Source: Tests/ERFGoldFiles/<name>/ (AMReX plotfiles written by ERF's CTest
regression runs, Tests/CTestList.cmake:177).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from plotfile import read_plotfile, read_plotfile_minmax, read_plotfile_minmax_boxes  # noqa: E402

TESTS = ["TaylorGreenAdvecting", "TaylorGreenAdvectingDiffusing", "EkmanSpiral", "IsentropicVortexAdvecting"]
# gold plotfiles stored without their FAB data: only the per-variable
# min / max of the MultiFab header travel
MINMAX_TESTS = ["ABL_MOST"]
# the same, several FABs: per-box minima and maxima
MINMAX_BOX_TESTS = ["MovingTerrain_nosub", "MovingTerrain_sub"]

if __name__ == "__main__":
    ref = sys.argv[1]
    for name in TESTS:
        pf = read_plotfile(os.path.join(ref, "Tests", "ERFGoldFiles", name))
        out = os.path.join(HERE, f"{name}_gold.npz")
        np.savez_compressed(out, data=pf["data"], names=np.array(pf["names"]), time=pf["time"],
                            header=np.array(pf["header"]))
        print(out, pf["data"].shape, pf["names"], pf["time"])
    for name in MINMAX_TESTS:
        pf = read_plotfile_minmax(os.path.join(ref, "Tests", "ERFGoldFiles", name))
        out = os.path.join(HERE, f"{name}_minmax.npz")
        np.savez_compressed(out, names=np.array(pf["names"]), time=pf["time"], vmin=pf["min"], vmax=pf["max"])
        print(out, pf["names"], pf["time"], pf["min"], pf["max"])
    for name in MINMAX_BOX_TESTS:
        pf = read_plotfile_minmax_boxes(os.path.join(ref, "Tests", "ERFGoldFiles", name))
        out = os.path.join(HERE, f"{name}_minmax.npz")
        np.savez_compressed(out, names=np.array(pf["names"]), time=pf["time"], boxes=pf["boxes"],
                            vmin=pf["min"], vmax=pf["max"])
        print(out, pf["names"], pf["time"], pf["boxes"].tolist())
