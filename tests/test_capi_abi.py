"""The C-ABI library loads and exports every entry point its header declares
(no device calls: this runs without a GPU)."""
import ctypes
import os

from meltpooldg_b200 import _capi


def test_library_exports_every_header_symbol():
    names = _capi.header_symbols()
    assert "mpdg_vmult" in names and "mpdg_solve" in names
    lib = _capi.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_built_for_sm100a():
    # the fatbin carries an sm_100a cubin: check the build flags recorded by the Makefile
    mk = open(os.path.join(os.path.dirname(_capi.HERE), "meltpooldg_b200", "csrc", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_host_only_entry_points_work_without_gpu():
    lib = _capi.lib()
    assert lib.mpdg_version() == 1
    d = _capi.SolverDesc()
    lib.mpdg_solver_desc_default(ctypes.byref(d))
    assert d.rel_tolerance == 1e-12 and d.abs_tolerance == 1e-20 and d.max_iterations == 10000
    assert d.solver == _capi.SOLVER_GMRES and d.preconditioner == _capi.PREC_JACOBI
    # argument checks fail before touching the device
    assert lib.mpdg_mesh_create(None, None) == _capi.ERR_ARG
    assert lib.mpdg_vmult(None, None, None) == _capi.ERR_ARG
