"""Field, restart and parameter files in the reference's formats.

Field files (readField / readInternalField / writeField, field.f90:331-476):
one file per field and time folder, ``<n>/<name>`` (the folder name is the
integer n written with I6 and left-adjusted; the field directory constant is
empty, field.f90:35, 244-245); vector fields are three files ``<name>x``,
``<name>y``, ``<name>z`` (vfield.f90:78-80).  Each file is an unformatted
stream: one default integer (int32, native byte order) holding the number of
values, then the values (float64) of the internal box in Fortran order,
is..ie x js..je x ks..ke with the bounds of setIndexesBounds
(field.f90:1746-1789): 1..n for a cell field, 0..n in the staggered
direction of sx / sy / sz.  A size that differs from the mesh's is an error
(readInternalField aborts).

Restart (writeTimeFolder / initTimeLevel, time.f90:307-345, 409-438):
``<n>/info_restart`` holds the time (ES25.15E3) and the number of bubbles
(I6), one per line.

Parameter files (parFile.f90:60-256): lines of at most 100 characters; the
first line whose first blank-delimited token equals the name gives the
value, read from the first non-blank character after it with the formats of
formats.f90: I6 (integers), L7 (logicals), ES25.15E3 (reals), A (strings).
Fortran formatted input reads a fixed width, ignores blanks inside numeric
fields and accepts D exponents; a real without a decimal point takes the 15
implied decimals of the edit descriptor.
"""
from __future__ import annotations

import os
import re

import numpy as np

from .fields import KIND_LO, Field

_LINE = 100  # character(len=100) :: whole


def folder_name(n: int) -> str:
    """The time folder of level n (write(dirName, '(I6)') n, then adjustl)."""
    s = f"{n:6d}"
    if len(s) > 6:  # I6 overflow prints asterisks
        s = "*" * 6
    return s.strip()


def field_path(case_dir: str, n: int, name: str) -> str:
    return os.path.join(case_dir, folder_name(n), name)


def _box(kind: str, nx: int, ny: int, nz: int):
    lo = KIND_LO[kind]
    return lo, (nx, ny, nz)


def _host(a) -> np.ndarray:
    return a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)


def write_field(case_dir: str, n: int, name: str, f: Field) -> str:
    """writeField (field.f90:453-474): the internal box of f into <n>/<name>."""
    lo, hi = _box(f.kind, f.nx, f.ny, f.nz)
    view = Field(f.kind, f.hd, f.nx, f.ny, f.nz, _host(f.a)).v(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])
    path = field_path(case_dir, n, name)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "wb") as fh:
        fh.write(np.asarray([view.size], dtype=np.int32).tobytes())
        fh.write(np.ascontiguousarray(view, dtype=np.float64).tobytes())
    return path


def read_field(case_dir: str, n: int, name: str, f: Field) -> None:
    """readField / readInternalField (field.f90:331-448): <n>/<name> into the
    internal box of f (ghosts untouched; the reference updates them after)."""
    lo, hi = _box(f.kind, f.nx, f.ny, f.nz)
    size = (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1)
    path = field_path(case_dir, n, name)
    with open(path, "rb") as fh:
        head = np.frombuffer(fh.read(4), dtype=np.int32)
        if head.size != 1 or int(head[0]) != size:
            raise ValueError(f"Dimension of field {name} not equal to mesh size ({path})")
        data = np.frombuffer(fh.read(8 * size), dtype=np.float64)
    if data.size != size:
        raise ValueError(f"field file {path} is truncated")
    vals = data.reshape(hi[2] - lo[2] + 1, hi[1] - lo[1] + 1, hi[0] - lo[0] + 1)
    if hasattr(f.a, "copy_"):
        import torch  # noqa: PLC0415

        Field(f.kind, f.hd, f.nx, f.ny, f.nz, f.a).v(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]).copy_(
            torch.from_numpy(vals.copy()))
    else:
        f.v(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])[...] = vals


def write_vfield(case_dir: str, n: int, name: str, u) -> None:
    """The three component files of a vector field (vfield.f90:78-80)."""
    for c, f in zip("xyz", u.components()):
        write_field(case_dir, n, name + c, f)


def read_vfield(case_dir: str, n: int, name: str, u) -> None:
    for c, f in zip("xyz", u.components()):
        read_field(case_dir, n, name + c, f)


def _fmt_es25_15e3(x: float) -> str:
    """ES25.15E3 as gfortran writes it: d.ddddddddddddddd E+eee, right-aligned in 25."""
    m, e = f"{x:.15E}".split("E")
    ei = int(e)
    return f"{m}E{'-' if ei < 0 else '+'}{abs(ei):03d}".rjust(25)


def write_restart_info(case_dir: str, n: int, t: float, nbubbles: int) -> str:
    """writeTimeFolder (time.f90:307-345): <n>/info_restart with t and the bubble count."""
    d = os.path.join(case_dir, folder_name(n))
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, "info_restart")
    with open(path, "w") as fh:
        fh.write(_fmt_es25_15e3(t) + "\n")
        fh.write(f"{nbubbles:6d}\n")
    return path


def read_restart_time(case_dir: str, n: int) -> float:
    """initTimeLevel (time.f90:409-438): the time of input folder n (0 for n = 0)."""
    if n == 0:
        return 0.0
    with open(os.path.join(case_dir, folder_name(n), "info_restart")) as fh:
        return _read_real(fh.readline().rstrip("\n"))


# ---------------------------------------------------------------------------
# parFile (parFile.f90:48-256)
# ---------------------------------------------------------------------------
def _numeric_field(s: str, width: int) -> str:
    # fixed width; blanks inside a numeric field are ignored (BN, the default)
    return s[:width].replace(" ", "")


def _read_int(s: str) -> int:
    v = _numeric_field(s, 6)
    if not re.fullmatch(r"[+-]?\d*", v):
        raise ValueError(f"invalid integer field {s[:6]!r}")
    return int(v) if v not in ("", "+", "-") else 0


def _read_real(s: str) -> float:
    v = _numeric_field(s, 25)
    if v in ("", "+", "-"):
        return 0.0
    m = re.fullmatch(r"([+-]?)(\d*)(\.(\d*))?(?:[EeDdQq]([+-]?\d+)|([+-]\d+))?", v)
    if not m or (not m.group(2) and not m.group(4)):
        raise ValueError(f"invalid real field {s[:25]!r}")
    sign, ip, dotpart, fp, ex1, ex2 = m.groups()
    ex = int(ex1 or ex2 or 0)
    if dotpart is None:  # no decimal point: the 15 implied decimals of ES25.15
        val = float(f"{ip}e{ex - 15}")
    else:
        val = float(f"{ip or '0'}.{fp or '0'}e{ex}")
    return -val if sign == "-" else val


def _read_logical(s: str) -> bool:
    v = s[:7].strip()
    if v.startswith("."):
        v = v[1:]
    if not v or v[0] not in "TtFf":
        raise ValueError(f"invalid logical field {s[:7]!r}")
    return v[0] in "Tt"


class ParFile:
    """parFileCTOR (parFile.f90:48-56): the parameter file <dir>/<name>."""

    def __init__(self, file_name: str, file_dir: str):
        self.file_name = file_name
        self.file_path = os.path.join(file_dir, file_name)

    def _value(self, name: str) -> str:
        with open(self.file_path) as fh:
            for raw in fh:
                whole = raw.rstrip("\n")[:_LINE].ljust(_LINE)
                i1 = whole.find(" ")  # index(whole, ' '), 0-based
                if i1 < 0:  # no blank in the 100 characters: whole(1:-1) is empty
                    continue
                if whole[:i1] == name:
                    rest = whole[i1 + 1:]
                    nb = len(rest) - len(rest.lstrip(" "))
                    if nb == len(rest):
                        raise ValueError(f"Invalid entry while parsing parameter: {name}")
                    return rest[nb:]
        raise KeyError(f"Parameter {name} not found in file {self.file_name}")

    def read_int(self, name: str) -> int:
        return _read_int(self._value(name))

    def read_bool(self, name: str) -> bool:
        return _read_logical(self._value(name))

    def read_real(self, name: str) -> float:
        return _read_real(self._value(name))

    def read_string(self, name: str) -> str:
        return self._value(name).rstrip(" ")


def velocity_walls(specs_dir: str):
    """The y-wall values of u from the case's boundary file specs/fstart_bc/u
    (read by vfieldCTOR / boundaryFieldCTOR through parFile: bx1..bx6 the types
    of the six patches, bvx1..bvx6 their values; likewise y, z).  The library
    runs the channel: periodic (type 3) in x and z, fixedValue (type 1) at the
    bottom (patch 3) and top (patch 4); anything else is an error.  Returns
    ((ux, uy, uz) at the bottom, (ux, uy, uz) at the top); no file gives the
    no-slip zeros."""
    path = os.path.join(specs_dir, "fstart_bc", "u")
    if not os.path.exists(path):
        return (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)
    bc = ParFile("u", os.path.dirname(path))
    for comp in "xyz":
        types = [bc.read_int(f"b{comp}{n}") for n in range(1, 7)]
        if types != [3, 3, 1, 1, 3, 3]:
            raise ValueError(f"velocity boundaries of u{comp}: patch types {types}; the channel (periodic x "
                             "and z, fixedValue walls in y) is supported")
    return (tuple(bc.read_real(f"bv{c}3") for c in "xyz"), tuple(bc.read_real(f"bv{c}4") for c in "xyz"))
