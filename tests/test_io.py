"""Field, restart and parameter files in the reference's formats
(tbfsolver_b200.io): field.f90:331-476, time.f90:307-345/409-438 and
parFile.f90:48-256."""
import os

import numpy as np
import pytest

from tbfsolver_b200 import io
from tbfsolver_b200.fields import Field, VField

# The reference's own example case (channel_18/specs), where a checkout of the
# reference is available: TBFP_REFERENCE_DIR names its root.  Tests that read it
# are skipped without it.
_REF = os.environ.get("TBFP_REFERENCE_DIR", "")
SPECS = os.path.join(_REF, "channel_18", "specs") if _REF else ""
needs_specs = pytest.mark.skipif(not (SPECS and os.path.isdir(SPECS)),
                                 reason="set TBFP_REFERENCE_DIR to a checkout of the reference")


@pytest.mark.parametrize("kind", ["cl", "sx", "sy", "sz"])
def test_field_file_layout_and_round_trip(tmp_path, kind):
    nx, ny, nz, hd = 6, 5, 4, 2
    f = Field(kind, hd, nx, ny, nz)
    rng = np.random.default_rng(1)
    f.a[...] = rng.standard_normal(f.a.shape)
    path = io.write_field(str(tmp_path), 3, "psi", f)
    assert path == os.path.join(str(tmp_path), "3", "psi")
    raw = open(path, "rb").read()
    lo = {"cl": (1, 1, 1), "sx": (0, 1, 1), "sy": (1, 0, 1), "sz": (1, 1, 0)}[kind]
    n = (nx - lo[0] + 1) * (ny - lo[1] + 1) * (nz - lo[2] + 1)
    assert len(raw) == 4 + 8 * n
    assert np.frombuffer(raw[:4], dtype=np.int32)[0] == n
    vals = np.frombuffer(raw[4:], dtype=np.float64)
    # Fortran order over the internal box: i fastest
    assert vals[0] == f.v(lo[0], lo[0], lo[1], lo[1], lo[2], lo[2]).item()
    assert vals[1] == f.v(lo[0] + 1, lo[0] + 1, lo[1], lo[1], lo[2], lo[2]).item()
    assert vals[nx - lo[0] + 1] == f.v(lo[0], lo[0], lo[1] + 1, lo[1] + 1, lo[2], lo[2]).item()
    g = Field(kind, hd, nx, ny, nz)
    io.read_field(str(tmp_path), 3, "psi", g)
    assert np.array_equal(g.interior() if kind == "cl" else g.v(lo[0], nx, lo[1], ny, lo[2], nz),
                          f.v(lo[0], nx, lo[1], ny, lo[2], nz))
    # ghosts are not read
    assert np.count_nonzero(g.a) == n


def test_vector_field_files_and_size_check(tmp_path):
    u = VField.zeros(2, 4, 3, 2)
    for c in u.components():
        c.a[...] = np.arange(c.a.size).reshape(c.a.shape)
    io.write_vfield(str(tmp_path), 0, "u", u)
    assert sorted(os.listdir(tmp_path / "0")) == ["ux", "uy", "uz"]
    w = VField.zeros(2, 4, 3, 2)
    io.read_vfield(str(tmp_path), 0, "u", w)
    for a, b in zip(u.components(), w.components()):
        assert np.array_equal(a.interior(), b.interior())
    with pytest.raises(ValueError, match="not equal to mesh size"):
        io.read_field(str(tmp_path), 0, "ux", Field("sx", 2, 5, 3, 2))


def test_restart_info(tmp_path):
    io.write_restart_info(str(tmp_path), 12, 1.2345678901234567e-3, 200)
    lines = open(tmp_path / "12" / "info_restart").read().splitlines()
    assert len(lines[0]) == 25 and lines[0].strip() == "1.234567890123457E-003"
    assert lines[1] == "   200"
    assert io.read_restart_time(str(tmp_path), 12) == pytest.approx(1.2345678901234567e-3, rel=1e-15)
    assert io.read_restart_time(str(tmp_path), 0) == 0.0
    assert io.folder_name(0) == "0" and io.folder_name(999999) == "999999"


def test_parameter_file_reader(tmp_path):
    (tmp_path / "specs").mkdir()
    (tmp_path / "specs" / "p").write_text(
        "! comment line\n\n"
        "Lx 3.141592653589793d0\n"
        "nx 192\n"
        "big 1234567\n"
        "isYunif .TRUE.\n"
        "flag .F.\n"
        "tol 1.d-10\n"
        "plain 25\n"
        "name   channel_18   \n"
        "gamma    1.5E+000\n")
    p = io.ParFile("p", str(tmp_path / "specs"))
    assert p.read_real("Lx") == 3.141592653589793
    assert p.read_int("nx") == 192
    assert p.read_int("big") == 123456  # I6 reads six characters
    assert p.read_bool("isYunif") is True and p.read_bool("flag") is False
    assert p.read_real("tol") == 1e-10
    assert p.read_real("plain") == 25e-15  # no decimal point: 15 implied decimals
    assert p.read_string("name") == "channel_18"
    assert p.read_real("gamma") == 1.5
    with pytest.raises(KeyError):
        p.read_int("ny")


@needs_specs
def test_reads_the_reference_case_specs():
    mesh = io.ParFile("mesh", SPECS)
    assert (mesh.read_int("nx"), mesh.read_int("ny"), mesh.read_int("nz")) == (192, 160, 96)
    assert mesh.read_real("Lx") == 3.141592653589793 and mesh.read_bool("isXunif") is True
    pcg = io.ParFile("pcg_solver", SPECS)
    assert (pcg.read_int("nLevels"), pcg.read_int("nPreSweep"), pcg.read_int("nPostSweep")) == (5, 2, 4)
    assert pcg.read_real("tolMG") == 0.4 and pcg.read_real("tolPCG") == 1e-10
    par = io.ParFile("parameters", SPECS)
    assert par.read_real("rhog") == 0.1 and par.read_real("mul") == 3.33333333333333e-4


def test_velocity_walls_from_the_boundary_file(tmp_path):
    """specs/fstart_bc/u in the case's format: periodic x, z and fixedValue walls
    give the wall values; another patch type is refused; no file is no-slip."""
    from tbfsolver_b200.io import velocity_walls

    assert velocity_walls(str(tmp_path)) == ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
    d = tmp_path / "fstart_bc"
    d.mkdir()
    lines = ["! header", "gridx_type sx", "init_opt 2"]
    for c, top in zip("xyz", ("1.5d0", "0.d0", "-2.5d-1")):
        lines += [f"b{c}{n} {t}" for n, t in zip(range(1, 7), (3, 3, 1, 1, 3, 3))]
        lines += [f"bv{c}1 0.d0", f"bv{c}2 0.d0", f"bv{c}3 0.d0", f"bv{c}4 {top}", f"bv{c}5 0.d0", f"bv{c}6 0.d0"]
    (d / "u").write_text("\n".join(lines) + "\n")
    assert velocity_walls(str(tmp_path)) == ((0.0, 0.0, 0.0), (1.5, 0.0, -0.25))
    (d / "u").write_text("\n".join(lines).replace("by3 1", "by3 2") + "\n")
    with pytest.raises(ValueError):
        velocity_walls(str(tmp_path))
