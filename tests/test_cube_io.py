"""Cube files in the reference's dialect (qsb_cube_write / qsb_cube_read, host
code in the C-ABI library) against the reference's own CubeWriter::SaveCube
(source/cube_writer.h:27-90) and CubeReader3::LoadCube + GetMeshData
(source/cube_reader3.h:38-124), compiled from its sources into oracle/_ref.

Bars: written files byte-identical to the reference's; values read
bit-identical to the reference reader's; a write -> read round trip within
the %.12f rounding (5e-13); short or malformed files rejected with a message."""
import os

import numpy as np
import pytest

import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")

CASES = [((7, 5, 13), 2), ((12, 12, 12), 0), ((1, 1, 6), 1), ((16, 9, 11), 3)]


def _case(grid, n_atoms, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = grid
    field = rng.standard_normal(nx * ny * nz) * 10.0 ** rng.integers(-6, 3, nx * ny * nz)
    axis = np.diag([nx * 0.25, ny * 0.3, nz * 0.2]) + 0.01 * rng.standard_normal((3, 3))
    origin = rng.standard_normal(3)
    Z = rng.integers(1, 30, n_atoms)
    pos = rng.uniform(0, 5, (n_atoms, 3))
    return field, axis, origin, Z, pos


@needs_ref
@pytest.mark.parametrize("grid,n_atoms", CASES)
def test_written_files_are_byte_identical_to_the_reference(qsb_host, tmp_path, grid, n_atoms):
    field, axis, origin, Z, pos = _case(grid, n_atoms, 1)
    a, b = tmp_path / "ours.cube", tmp_path / "ref.cube"
    qsb_host.cube_write(a, field, grid, axis, origin, Z, pos, "rho_out step 7")
    O.ref_cube_write(str(b), field, grid, axis, origin, Z, pos, "rho_out step 7")
    assert a.read_bytes() == b.read_bytes()


@needs_ref
@pytest.mark.parametrize("grid,n_atoms", CASES)
def test_values_read_equal_the_reference_reader(qsb_host, tmp_path, grid, n_atoms):
    field, axis, origin, Z, pos = _case(grid, n_atoms, 2)
    path = tmp_path / "ref.cube"
    O.ref_cube_write(str(path), field, grid, axis, origin, Z, pos, "state 3")
    f_ref, h_ref = O.ref_cube_read(str(path))
    f, h = qsb_host.cube_read(path)
    assert h["grid"] == h_ref["grid"] == tuple(grid)
    assert np.array_equal(f, f_ref)
    assert np.array_equal(h["axis"], h_ref["axis"]) and np.array_equal(h["origin"], h_ref["origin"])
    assert np.array_equal(h["Z"], Z)
    np.testing.assert_allclose(h["pos"], pos, rtol=0, atol=5e-16 * 8)
    # the round trip keeps the values to the writer's 12 decimals
    assert np.abs(f - field).max() <= 5e-13 + 1e-15 * np.abs(field).max()


def test_large_grid_round_trip(qsb_host, tmp_path):
    grid = (96, 96, 96)
    rng = np.random.default_rng(3)
    field = rng.uniform(-1, 1, 96 ** 3)
    path = tmp_path / "big.cube"
    qsb_host.cube_write(path, field, grid, np.eye(3) * 12.0)
    f, h = qsb_host.cube_read(path)
    assert h["grid"] == grid and len(h["Z"]) == 0
    assert np.abs(f - field).max() <= 5e-13 + 2.3e-16


def test_malformed_files_are_rejected(qsb_host, tmp_path):
    field, axis, origin, Z, pos = _case((6, 6, 6), 1, 4)
    path = tmp_path / "a.cube"
    qsb_host.cube_write(path, field, (6, 6, 6), axis, origin, Z, pos)
    text = path.read_text()
    short = tmp_path / "short.cube"
    short.write_text(text[: len(text) // 2])
    with pytest.raises(qsb_host.QsbError, match="expected 216 values"):
        qsb_host.cube_read(short)
    bad = tmp_path / "bad.cube"
    lines = text.splitlines(True)
    toks = lines[-1].split("\t")
    toks[0] = "x" + toks[0]                       # same count, one token not a number
    lines[-1] = "\t".join(toks)
    bad.write_text("".join(lines))
    with pytest.raises(qsb_host.QsbError, match="not a number"):
        qsb_host.cube_read(bad)
    with pytest.raises(qsb_host.QsbError, match="cannot open"):
        qsb_host.cube_read(tmp_path / "missing.cube")
    with pytest.raises(qsb_host.QsbError, match="one line"):
        qsb_host.cube_write(tmp_path / "c.cube", field, (6, 6, 6), axis, origin, comment="two\nlines")


CUBE_DROPIN_PROGRAM = r"""
#include <cstdio>
#include <cstring>
#include <vector>
struct GridRange { int begin_x, begin_y, begin_z, end_x, end_y, end_z;
  int SizeX() const { return end_x - begin_x; } int SizeY() const { return end_y - begin_y; }
  int SizeZ() const { return end_z - begin_z; } };
struct Nucleus { int Z; double Rx; double Ry; double Rz; };
#include "qumasun_dropin.hpp"
int main(int argc, char** argv) {
  const int nx = 5, ny = 4, nz = 7;
  std::vector<double> f(nx * ny * nz);
  for (size_t i = 0; i < f.size(); ++i) f[i] = 0.001 * (double)i - 0.05;
  qsb_dropin::CubeWriter::Frame frame{};
  frame.grid_x = nx; frame.grid_y = ny; frame.grid_z = nz;
  const double ax[9] = {2.5, 0, 0, 0, 2.0, 0, 0, 0, 3.5};
  std::memcpy(frame.boxaxis, ax, sizeof ax);
  std::strcpy(frame.comment, "density");
  Nucleus nuc[2] = {{8, 0.1, 0.2, 0.3}, {1, 1.5, -0.5, 2.0}};
  if (qsb_dropin::CubeWriter::SaveCube(argv[1], frame, 2, nuc, f.data()) != 1) return 2;
  qsb_dropin::CubeReader3 r;
  const auto g = r.LoadCube(argv[1]);
  std::vector<double> back(f.size());
  r.GetMeshData(back.data());
  double err = 0;
  for (size_t i = 0; i < f.size(); ++i) err = std::max(err, std::fabs(back[i] - f[i]));
  std::printf("%d %d %d %.17g %s", g.grid_x, g.grid_y, g.grid_z, err, g.comment);
  return 0;
}
"""


@needs_ref
def test_dropin_cube_classes_match_the_reference(tmp_path):
    """The reference-shaped CubeWriter / CubeReader3 of qumasun_dropin.hpp compile
    against a caller's own Nucleus type, write the reference writer's bytes and
    read them back."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "qumasun-workshop-template_b200")
    src = tmp_path / "cube.cpp"
    src.write_text(CUBE_DROPIN_PROGRAM)
    exe = tmp_path / "cube"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(root, "include"), str(src), "-o", str(exe), "-L", libdir,
                    "-lqumasun_b200", f"-Wl,-rpath,{libdir}"], check=True, capture_output=True)
    ours = tmp_path / "ours.cube"
    out = subprocess.run([str(exe), str(ours)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    nx, ny, nz, err, comment = out.stdout.split()
    assert (int(nx), int(ny), int(nz)) == (5, 4, 7) and float(err) <= 5e-13 and comment == "density"
    f = 0.001 * np.arange(5 * 4 * 7) - 0.05
    ref = tmp_path / "ref.cube"
    O.ref_cube_write(str(ref), f, (5, 4, 7), [[2.5, 0, 0], [0, 2.0, 0], [0, 0, 3.5]], np.zeros(3), [8, 1],
                     [[0.1, 0.2, 0.3], [1.5, -0.5, 2.0]], "density")
    assert ours.read_bytes() == ref.read_bytes()


@needs_ref
def test_state_files_follow_the_reference_naming_and_round_trip(qsb_host, tmp_path):
    """write_states / read_states: the reference's state file names, list
    order and comment; its own CubeReader3 reads the values; the round trip
    keeps the bundle to the %.12f rounding and the eigenvalues to 1e-10."""
    grid = (6, 5, 7)
    N = 6 * 5 * 7
    rng = np.random.default_rng(8)
    X = rng.uniform(-1, 1, (3, 2, N))
    ev = np.array([-0.512345678912, -0.25, 0.125])
    names = qsb_host.write_states(str(tmp_path), "state", X, ev, grid, (3.0, 2.5, 3.5), [6], [[0.1, 0.2, 0.3]],
                                  sk=1, n_kpoints=4, kpoint=(1, 4, 0, 1, 0, 1), list_name="states.txt")
    assert names[:2] == ["state_up_k1_n0_re.cube", "state_up_k1_n0_im.cube"] and len(names) == 6
    f_ref, _ = O.ref_cube_read(str(tmp_path / names[3]))
    assert np.abs(f_ref - X[1, 1]).max() <= 5e-13
    line2 = (tmp_path / names[0]).read_text().splitlines()[1]
    assert line2 == "eigenvalue=-0.5123456789, kpoint=1/4,0/1,0/1"
    Y, ev2, hdr = qsb_host.read_states(str(tmp_path / "states.txt"))
    assert Y.shape == X.shape and np.abs(Y - X).max() <= 5e-13
    assert np.abs(ev2 - ev).max() <= 1e-10 and hdr["grid"] == grid
    # spin down: k index past the spin-up set
    assert qsb_host.write_states(str(tmp_path), "s", X[:1], ev, grid, (3.0, 2.5, 3.5), sk=5, n_kpoints=4)[0] == \
        "s_down_k1_n0_re.cube"
