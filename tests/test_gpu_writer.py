"""VTK output of the Writer (api/Writer.cpp) through a C++ driver written
against the reference API: file names and master list, grid, and the values
of a physical scalar, a Fourier-space scalar (written after its inverse) and
a vector, each captured at the time of its write() call."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _exe():
    from spectral_upcxx_b200 import build as B
    return B.build_cpp_program([os.path.join(HERE, "cpp", "api_writer.cpp")],
                               os.path.join(B.LIBDIR, "test_drivers", "api_writer.exe"))


def _read_vtk(path):
    toks = open(path).read().split()
    assert toks[:2] == ["#", "vtk"]
    i = toks.index("DIMENSIONS")
    dims = [int(t) for t in toks[i + 1:i + 4]]
    coords = []
    pos = i + 4
    for ax in "XYZ":
        assert toks[pos] == f"{ax}_COORDINATES" and int(toks[pos + 1]) == dims["XYZ".index(ax)]
        n = int(toks[pos + 1])
        coords.append(np.array(toks[pos + 3:pos + 3 + n], dtype=float))
        pos += 3 + n
    assert toks[pos] == "POINT_DATA"
    npts = int(toks[pos + 1])
    pos += 2
    fields = {}
    while pos < len(toks):
        kind, name = toks[pos], toks[pos + 1]
        if kind == "SCALARS":
            pos += 5  # SCALARS name float LOOKUP_TABLE default
            fields[name] = np.array(toks[pos:pos + npts], dtype=float)
            pos += npts
        else:
            pos += 3
            fields[name] = np.array(toks[pos:pos + 3 * npts], dtype=float).reshape(npts, 3)
            pos += 3 * npts
    return dims, coords, fields


def test_writer_vtk_files(cuda, tmp_path):
    prefix = str(tmp_path / "sol")
    r = subprocess.run([_exe(), prefix], stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    master = open(prefix + ".visit").read().split("\n")
    assert master[0] == "!NBLOCKS 1"
    assert master[1:4] == [prefix + f"0_{w}.vtk" for w in range(3)]
    nx, ny, nz = 8, 4, 16
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    f3 = np.sin(0.7 * i) + 0.1 * j - 0.3 * k
    f = f3.ravel()
    # g is Scalar::forward (Nyquist planes zeroed) of f, written after its inverse
    fh = np.fft.fftn(f3)
    fh[nz // 2, :, :] = 0
    fh[:, ny // 2, :] = 0
    fh[:, :, nx // 2] = 0
    g = np.fft.ifftn(fh).real.ravel()
    for w in range(3):
        dims, coords, fields = _read_vtk(prefix + f"0_{w}.vtk")
        assert dims == [nx, ny, nz]
        # coordinates as the reference sets them (y spaced by 2 pi / nx as well)
        assert np.allclose(coords[0], np.arange(nx) * 2 * np.pi / nx, rtol=1e-6)
        assert np.allclose(coords[1], np.arange(ny) * 2 * np.pi / nx, rtol=1e-6)
        assert np.allclose(coords[2], np.arange(nz) * 2 * np.pi / nz, rtol=1e-6)
        assert list(fields) == ["s", "g", "velocity"]
        assert np.allclose(fields["s"], f + 2 * w, rtol=1e-6, atol=1e-6)
        assert np.allclose(fields["g"], g, rtol=1e-6, atol=1e-6)
        vel = fields["velocity"]
        assert np.allclose(vel[:, 0], i.ravel()) and np.allclose(vel[:, 1], 10 * j.ravel())
        assert np.allclose(vel[:, 2], 100 * k.ravel())
    assert not os.path.exists(prefix + "0_3.vtk")


def test_writer_frequency_zero_writes_nothing(cuda, tmp_path):
    """exec/ns.cpp sets a write frequency of 0: no file, no fault."""
    from spectral_upcxx_b200 import build as B
    src = tmp_path / "w0.cpp"
    src.write_text(open(os.path.join(HERE, "cpp", "api_writer.cpp")).read()
                   .replace("writer.setFreq(2);", "writer.setFreq(0);"))
    exe = B.build_cpp_program([str(src)], str(tmp_path / "w0.exe"))
    prefix = str(tmp_path / "none")
    r = subprocess.run([exe, prefix], stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    assert not any(p.name.startswith("none") for p in tmp_path.iterdir())
