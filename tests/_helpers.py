"""Shared helpers for the test suite (conversion between package fields and
oracle fields, seeded cases)."""
import numpy as np

from oracle import tbfp_oracle as O


def mesh_of(g):
    return O.Mesh(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz, y_uniform=not g.y_stretched, gamma=g.gamma)


def to_oracle(f, g):
    a = f.a
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return O.FField(f.kind, f.hd, g.nx, g.ny, g.nz, a.copy())


def rel_linf(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))
