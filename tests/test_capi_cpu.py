"""The C ABI library and the pybind11 drop-in module without a GPU: every
declared symbol is exported, and argument errors are reported before any
device work."""
import ctypes
import os
import re

import numpy as np
import pytest

import pyhea_b200 as hb
from conftest import REPO, opt_call_args
from pyhea_b200 import accelerate
from pyhea_b200 import lattice as L


def declared_symbols():
    text = open(os.path.join(REPO, "include", "hea_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hea_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(hb._LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 11
    for s in syms:
        assert hasattr(lib, s), s


def test_pybind_module_links_the_library():
    assert hasattr(accelerate, "run_local_parallel_hcs_cuda")
    assert hasattr(accelerate, "cuda_available")
    assert hasattr(accelerate, "run_local_parallel_hcs")
    assert accelerate.cuda_available() == hb.cuda_available()


def _problem(species=(32, 32, 32, 32), cell=4):
    nbor, sizes = L.neighbors(L.FCC, cell)
    T = len(species)
    return hb.Problem(nbor, sizes, species, [4.0, 1.0, 0.5], np.zeros((3, T * T)))


@pytest.mark.parametrize("kw,msg", [
    (dict(num_solutions=0), "nnet"),
    (dict(total_iter=-1), "step"),
    (dict(parallel_task=0), "task"),
    (dict(converge_depth=-1), "depth"),
])
def test_invalid_params_raise_value_error(kw, msg):
    args = dict(num_solutions=2, total_iter=1, parallel_task=8, converge_depth=2)
    args.update(kw)
    with pytest.raises(ValueError, match=msg):
        hb.search(_problem(), **args)


def test_invalid_problems_raise_before_device_work():
    with pytest.raises(ValueError, match="sum of element"):
        nbor, sizes = L.neighbors(L.FCC, 4)
        pb = hb.Problem(nbor, sizes, [32, 32, 32, 32], [4.0, 1.0, 0.5], np.zeros((3, 16)))
        pb._c.num_sites = 100
        hb.search(pb, 2, 1, 8, 2)
    with pytest.raises(ValueError, match="at least one"):
        hb.search(_problem(species=(64, 64, 128, 0)), 2, 1, 8, 2)
    with pytest.raises(ValueError, match="weight"):
        nbor, sizes = L.neighbors(L.FCC, 4)
        hb.search(hb.Problem(nbor, sizes, [128, 128], [1.0, -1.0], np.zeros((2, 4))), 2, 1, 8, 2)
    with pytest.raises(hb.HeaError, match="species"):
        hb.search(_problem(species=(256,)), 2, 1, 8, 2)


def test_pybind_argument_errors():
    nbor, sizes = L.neighbors(L.FCC, 3)
    nested = L.as_nested(nbor, sizes)
    tgt = np.zeros((3, 16))
    with pytest.raises(ValueError, match="sites"):
        accelerate.run_local_parallel_hcs_cuda(2, 1, 8, 2, 0.001, nested[:-1], [27] * 4, [4.0, 1.0, 0.5], tgt)
    with pytest.raises(ValueError, match="target_sro"):
        accelerate.run_local_parallel_hcs_cuda(2, 1, 8, 2, 0.001, nested, [27] * 4, [4.0, 1.0, 0.5], np.zeros((3, 9)))
    bad = [list(map(list, s)) for s in nested]
    bad[5][1] = bad[5][1][:-1]
    with pytest.raises(ValueError, match="one size"):
        accelerate.run_local_parallel_hcs_cuda(2, 1, 8, 2, 0.001, bad, [27] * 4, [4.0, 1.0, 0.5], tgt)
    with pytest.raises(RuntimeError, match="CPU engine"):
        accelerate.run_local_parallel_hcs(2, 1, 8, 2, 0.001, nested, [27] * 4, [4.0, 1.0, 0.5], tgt)


@pytest.mark.skipif(hb.cuda_available(), reason="checks argument handling on a machine without a GPU")
def test_reference_driver_call_is_accepted():
    """The exact positional call of the reference driver (recorded from pyhea/model/opt.py:89-90:
    neighbour shells as numpy arrays in nested lists, target as an ndarray) is parsed by the
    drop-in module, which fails only at the device step here."""
    args = opt_call_args()
    with pytest.raises(RuntimeError) as err:
        accelerate.run_local_parallel_hcs_cuda(*args)
    assert not isinstance(err.value, (TypeError, ValueError))


@pytest.mark.parametrize("lattice,cell,species,shell_set,msg", [
    (L.FCC, 4, (64, 64, 64, 60), L.SHELLS_REFERENCE, "does not hold"),   # 252 sites, not 4 * 4^3
    (L.BCC, 1, (1, 1), L.SHELLS_REFERENCE, "does not hold"),             # edge below 2
])
def test_implicit_lattice_must_describe_the_structure(lattice, cell, species, shell_set, msg):
    """An implicit-neighbour problem is checked against its lattice before any device work."""
    T = len(species)
    pb = hb.Problem.from_lattice(lattice, cell, species, [4.0, 1.0, 0.5], np.zeros((3, T * T)), shell_set=shell_set)
    with pytest.raises(ValueError, match=msg):
        hb.search(pb, 2, 1, 8, 2)


def test_implicit_lattice_shell_sizes_must_match():
    pb = hb.Problem.from_lattice(L.FCC, 4, (64,) * 4, [4.0, 1.0, 0.5], np.zeros((3, 16)))
    pb.shell_sizes[2] = 24  # the reference shell set's third FCC shell has 12
    with pytest.raises(ValueError, match="shell 2"):
        hb.search(pb, 2, 1, 8, 2)
