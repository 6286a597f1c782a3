"""The C++ adapter over the C ABI (include/mpdg_operator.hpp): compiles on the
CPU; on a GPU, a C++ program drives vmult / inverse diagonal / CG through it
and its results are checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "tests", "cpp", "adapter_demo.cpp")


def _compile(out):
    lib = os.path.join(ROOT, "meltpooldg_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), DEMO,
                    "-o", out, "-L", lib, "-lmpdg", f"-Wl,-rpath,{lib}"], check=True)


def test_adapter_compiles_and_links(tmp_path):
    _compile(str(tmp_path / "demo"))
    assert os.path.exists(tmp_path / "demo")


@pytest.mark.gpu
def test_adapter_drives_the_device(cuda, tmp_path):
    from oracle import oracle as O
    from meltpooldg_b200.operators import box_vertices, boundary_mask
    exe = str(tmp_path / "demo")
    _compile(exe)
    nc, p = (5, 4, 3), 2
    V = box_vertices(nc, perturb=0.1, seed=4)
    mask = boundary_mask(nc, p)
    n = int(np.prod([c * p + 1 for c in nc]))
    src = np.random.Generator(np.random.PCG64(9)).uniform(-1, 1, n)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(np.array(nc, np.int32).tobytes())
        f.write(np.array([p], np.int32).tobytes())
        f.write(np.array([n], np.int64).tobytes())
        f.write(V.tobytes())
        f.write(mask.tobytes())
        f.write(src.tobytes())
    subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], check=True)
    raw = open(tmp_path / "out.bin", "rb").read()
    out = np.frombuffer(raw[: 24 * n], dtype=np.float64).reshape(3, n)
    om = O.Mesh(3, p, nc, V)
    op = O.Operator(O.HEAT, 1e-3, rho_cp=1.0, k0=1.0, dirichlet=mask)
    ref = O.vmult(om, op, src)
    assert np.abs(out[0] - ref).max() <= 1e-12 * np.abs(ref).max()
    inv = O.inverse_diagonal(om, op)
    assert np.abs(out[1] - inv).max() <= 1e-12 * np.abs(inv).max()
    free = mask == 0
    assert np.abs(out[2][free] - src[free]).max() < 1e-8
