"""Field storage with the reference's Fortran layout.

A field ``f_(is-hd:ie+hd, js-hd:je+hd, ks-hd:ke+hd)`` (src/fields/field/field.f90:271-273)
is held as a C-ordered array of shape ``(nk, nj, ni)`` -- the same bytes as the
column-major Fortran array, so its base address can be handed to the C ABI
unchanged.  Index bounds per field type follow setIndexesBounds
(field.f90:1746-1789): 'cl' 1..n in all directions, 'sx' i=0..nx, 'sy'
j=0..ny, 'sz' k=0..nz.  The array may be a numpy array (host) or a torch
tensor (host or CUDA); the library's host or device entry points are chosen
from it.
"""
from __future__ import annotations

import numpy as np

KIND_LO = {"cl": (1, 1, 1), "sx": (0, 1, 1), "sy": (1, 0, 1), "sz": (1, 1, 0)}


def field_shape(kind: str, hd: int, nx: int, ny: int, nz: int):
    lo = KIND_LO[kind]
    ni = nx - lo[0] + 1 + 2 * hd
    nj = ny - lo[1] + 1 + 2 * hd
    nk = nz - lo[2] + 1 + 2 * hd
    return (nk, nj, ni)


class Field:
    """A staggered or cell field with halo ``hd``."""

    def __init__(self, kind: str, hd: int, nx: int, ny: int, nz: int, data=None):
        if kind not in KIND_LO:
            raise ValueError(f"unknown field type {kind!r}")
        self.kind, self.hd = kind, int(hd)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        lo = KIND_LO[kind]
        self.lb = (lo[0] - hd, lo[1] - hd, lo[2] - hd)
        shape = field_shape(kind, hd, nx, ny, nz)
        if data is None:
            data = np.zeros(shape, dtype=np.float64)
        if tuple(data.shape) != shape:
            raise ValueError(f"field {kind} hd={hd}: expected shape {shape}, got {tuple(data.shape)}")
        self.a = data

    @classmethod
    def like(cls, other: "Field", data=None) -> "Field":
        return cls(other.kind, other.hd, other.nx, other.ny, other.nz, data)

    def v(self, i0, i1, j0, j1, k0, k1):
        """View of the inclusive Fortran index range (i0:i1, j0:j1, k0:k1)."""
        lb = self.lb
        return self.a[k0 - lb[2] : k1 - lb[2] + 1, j0 - lb[1] : j1 - lb[1] + 1, i0 - lb[0] : i1 - lb[0] + 1]

    def interior(self):
        lo = KIND_LO[self.kind]
        return self.v(lo[0], self.nx, lo[1], self.ny, lo[2], self.nz)

    # --- placement --------------------------------------------------------
    @property
    def on_cuda(self) -> bool:
        return getattr(self.a, "is_cuda", False)

    def address(self) -> int:
        """Base address of the array (host or device), checked for the C ABI."""
        a = self.a
        if isinstance(a, np.ndarray):
            if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
                raise ValueError("fields must be C-contiguous float64 arrays")
            return a.ctypes.data
        import torch  # noqa: PLC0415 - optional dependency for device fields

        if a.dtype != torch.float64 or not a.is_contiguous():
            raise ValueError("fields must be contiguous float64 tensors")
        return a.data_ptr()

    def numpy(self) -> np.ndarray:
        a = self.a
        if isinstance(a, np.ndarray):
            return a
        return a.detach().cpu().numpy()


class VField:
    """Staggered velocity triple (ux 'sx', uy 'sy', uz 'sz'), src/fields/vfield/vfield.f90."""

    def __init__(self, ux: Field, uy: Field, uz: Field):
        if (ux.kind, uy.kind, uz.kind) != ("sx", "sy", "sz"):
            raise ValueError("VField needs components of types sx, sy, sz")
        self.ux, self.uy, self.uz = ux, uy, uz

    @classmethod
    def zeros(cls, hd: int, nx: int, ny: int, nz: int) -> "VField":
        return cls(Field("sx", hd, nx, ny, nz), Field("sy", hd, nx, ny, nz), Field("sz", hd, nx, ny, nz))

    def components(self):
        return (self.ux, self.uy, self.uz)
