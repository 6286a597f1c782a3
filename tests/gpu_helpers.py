"""Shared set-up of the GPU parity tests: one vertex array feeds both the
CUDA path (through the C ABI) and the CPU oracle."""
import numpy as np

from oracle import oracle as O


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def meshes(nc, p, perturb=0.0, seed=0, mask=None, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
           geometry="auto"):
    import meltpooldg_b200 as M
    V = M.box_vertices(nc, lo, hi, perturb, seed)
    gm = M.Mesh(V, nc, p, mask, geometry=geometry)
    om = O.Mesh(3, p, nc, V)
    return gm, om


def relerr(got, ref):
    return float(np.abs(np.asarray(got) - ref).max() / max(np.abs(ref).max(), 1e-300))


def dev(a, dtype=None):
    import torch
    t = torch.tensor(np.asarray(a), device="cuda")
    return t if dtype is None else t.to(dtype)
