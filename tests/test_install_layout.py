"""The install layout that keeps PyHEA's `device: cpu` beside the drop-in.

The drop-in module replaces pyhea/cpp/accelerate*.so, which is also where
PyHEA's CPU engine lives (pyhea/cpp/bind.cpp:7-46).  The documented layout puts
PyHEA's own module in pyhea/cpp/ref/, this build's in pyhea/cpp/b200/, and a
three-line pyhea/cpp/accelerate.py that takes each entry point from its module.
Here that layout is assembled in a temporary directory with PyHEA's module
compiled from its own sources (oracle/build_oracle.py) and imported the way
pyhea/model/opt.py:5-9 imports it; the CPU engine runs (no GPU is needed).
"""
import glob
import os
import shutil
import subprocess
import sys

import pytest

from conftest import REPO

REF_MOD = glob.glob(os.path.join(REPO, "oracle", "_ref", "pymod", "accelerate*.so"))
OUR_MOD = glob.glob(os.path.join(REPO, "pyhea_b200", "accelerate*.so"))

SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from pyhea.cpp import accelerate as acc            # as pyhea/model/opt.py:5-9
from pyhea.cpp.ref import accelerate as ref
from pyhea.cpp.b200 import accelerate as b200
assert acc.run_local_parallel_hcs is ref.run_local_parallel_hcs
assert acc.run_local_parallel_hcs_cuda is b200.run_local_parallel_hcs_cuda
assert acc.cuda_available is b200.cuda_available
sys.path.insert(0, sys.argv[2])
from pyhea_b200 import lattice as L
nbor, sizes = L.neighbors(L.FCC, 3)
nested = [[list(map(int, shell)) for shell in site] for site in L.as_nested(nbor, sizes)]
element = [27, 27, 27, 27]
latts, fits = acc.run_local_parallel_hcs(2, 1, 8, 2, 0.001, nested, element, [4.0, 1.0, 0.5],
                                         [[0.0] * 16, [0.0] * 16, [0.0] * 16])
assert len(latts) == 2 and fits == sorted(fits)
for occ in latts:
    assert np.bincount(occ, minlength=4).tolist() == element
print("layout ok", bool(acc.cuda_available()))
"""


@pytest.mark.skipif(not REF_MOD or not OUR_MOD, reason="PyHEA's module or the drop-in is not built")
def test_cpu_engine_beside_the_dropin(tmp_path):
    cpp = tmp_path / "pyhea" / "cpp"
    for d in (cpp / "ref", cpp / "b200"):
        d.mkdir(parents=True)
        (d / "__init__.py").write_text("")
    (tmp_path / "pyhea" / "__init__.py").write_text("")
    (cpp / "__init__.py").write_text("from .accelerate import *\n")  # PyHEA's package re-exports the engine
    shutil.copy(REF_MOD[0], cpp / "ref")
    shutil.copy(OUR_MOD[0], cpp / "b200")
    shutil.copy(os.path.join(REPO, "pyhea_b200", "libhea_cuda.so"), cpp / "b200")
    (cpp / "accelerate.py").write_text(
        "from .b200.accelerate import run_local_parallel_hcs_cuda, cuda_available  # B200 engine\n"
        "from .ref.accelerate import run_local_parallel_hcs                        # reference CPU engine\n")
    r = subprocess.run([sys.executable, "-c", SCRIPT, str(tmp_path), REPO], capture_output=True, text=True,
                       timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "layout ok" in r.stdout
