"""Link-level drop-in: the reference's own command-line programs (their main() unchanged,
built by `make -C oracle ref_cli` from the reference sources) linked against libsysmat.so
instead of the reference kernels.  They read Params_*.dat from the working directory and
write .sysmat files exactly as the reference CLIs do; the files must equal what the
library returns through its entry points."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, geometry, sysmat

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref")


def _exe(name):
    path = os.path.join(REF, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not built (make -C oracle ref_cli, needs the reference sources)")
    return path


def _run(exe, cwd, *args):
    r = subprocess.run([exe, *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def _fname(prefix, g):
    return f"{prefix}_shift_{g.image[8]:f}_{g.image[9]:f}_{g.image[10]:f}.sysmat"


def test_relinked_reference_pe_cli(gpu, tmp_path):
    exe = _exe("PEGen_CircularHole_sysmat")
    g = geometry.mini(seed=3, n_rot=3)
    g.write(str(tmp_path))
    _run(exe, str(tmp_path), "-cuda", "0")
    got = np.fromfile(tmp_path / _fname("PE_SysMat", g), np.float32)
    D, V = g.n_det, g.n_vox
    assert got.size == D * V * 3
    for r in range(3):
        dst = np.zeros(D * V, np.float32)
        sysmat.PESysMatGen(g.collimator, g.detector, g.with_rotation(r).image, dst)
        assert np.array_equal(got[r * D * V:(r + 1) * D * V], dst)


def test_relinked_reference_scatter_cli(gpu, tmp_path):
    pe_exe = _exe("PEGen_CircularHole_sysmat")
    sc_exe = _exe("ScatterGen_CircularHole_sysmat")
    g = geometry.mini(seed=5)
    g.write(str(tmp_path))
    _run(pe_exe, str(tmp_path), "-cuda", "0")
    _run(sc_exe, str(tmp_path), "-cuda", "0")       # computes and writes both bitmaps
    D, V = g.n_det, g.n_vox
    pe = np.fromfile(tmp_path / _fname("PE_SysMat", g), np.float32)
    sc = np.fromfile(tmp_path / _fname("Scatter_SysMat", g), np.float32)
    full = np.fromfile(tmp_path / _fname("SysMat_withScatter", g), np.float32)
    dst = np.zeros(D * V, np.float32)
    sysmat.scatter(g.collimator, g.detector, g.image, g.physics, pe,
                   str(tmp_path / "c2"), str(tmp_path / "h2"), dst)
    assert np.array_equal(sc, dst)
    assert np.array_equal(full, pe + sc)
    # the bitmap files the CLI wrote re-load through the -Geo* flags
    _run(sc_exe, str(tmp_path), "-cuda", "0", "-GeoCrystal", "GeometryRelationShip_Crystal2Crystal",
         "-GeoCollimator", "GeometryRelationShip_Collimator2Crystal")
    assert np.array_equal(np.fromfile(tmp_path / _fname("Scatter_SysMat", g), np.float32), sc)


@pytest.mark.parametrize("exe_name,key", [("ScatterGen_Collimator_sysmat", "collimator"),
                                          ("ScatterGen_Crystal_sysmat", "crystal")])
def test_relinked_reference_split_scatter_clis(gpu, tmp_path, exe_name, key):
    pe_exe = _exe("PEGen_CircularHole_sysmat")
    exe = _exe(exe_name)
    g = geometry.mini(seed=6)
    g.write(str(tmp_path))
    _run(pe_exe, str(tmp_path), "-cuda", "0")
    _run(exe, str(tmp_path), "-cuda", "0")
    pe = np.fromfile(tmp_path / _fname("PE_SysMat", g), np.float32)
    D, V = g.n_det, g.n_vox
    dst = np.zeros(D * V, np.float32)
    if key == "collimator":
        sysmat.scatter_collimator(g.collimator, g.detector, g.image, g.physics, pe, str(tmp_path / "h2"), dst)
    else:
        sysmat.scatter_crystal(g.detector, g.image, g.physics, pe, str(tmp_path / "c2"), dst)
    full = np.fromfile(tmp_path / _fname("SysMat", g), np.float32)
    assert np.array_equal(full, pe + dst)
