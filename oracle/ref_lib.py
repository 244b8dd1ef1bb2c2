"""Test infrastructure only: ctypes access to the reference's own programs.

oracle/Makefile (target `ref`) compiles the unmodified reference CUDA sources for
sm_100a into oracle/_ref/.  These wrappers call the reference host entry points
(PEGen_RayTracing_CircularHole/PESysMatGen.cu:1368, ScatterGen_RayTracing_CircularHole/
scatter.cu:2013, ScatterGen_Collimator/scatter.cu:1511, ScatterGen_Crystal/scatter.cu:1528)
exactly as the reference CLIs do: host buffers in, host buffers out.  The reference
prints progress banners on stdout; they are sent to stderr so that a caller's stdout
stays machine-readable.

Only tests, fixture scripts and the reference arm of bench.py use this module.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_fp = ctypes.POINTER(ctypes.c_float)


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_pe.so"))


@contextlib.contextmanager
def _stdout_to_stderr():
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        try:
            import ctypes.util
            libc = ctypes.CDLL(None)
            libc.fflush(None)
        except Exception:
            pass
        os.dup2(saved, 1)
        os.close(saved)


def _load(name):
    return ctypes.CDLL(os.path.join(REF_DIR, name))


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


def pe(geo, cuda_id: int = 0) -> np.ndarray:
    """Reference PESysMatGen for the rotation in geo.image[20]; returns (D, V) float32."""
    lib = _load("libref_pe.so")
    lib.ref_PESysMatGen.restype = ctypes.c_int
    c, pc = _f(geo.collimator.copy())
    d, pd = _f(geo.detector.copy())
    i, pi = _f(geo.image.copy())
    out = np.zeros(geo.n_det * geo.n_vox, dtype=np.float32)
    with _stdout_to_stderr():
        ret = lib.ref_PESysMatGen(pc, pd, pi, out.ctypes.data_as(_fp), ctypes.c_int(cuda_id))
    if ret != geo.n_vox:
        raise RuntimeError(f"reference PESysMatGen returned {ret}")
    return out.reshape(geo.n_det, geo.n_vox)


def _geo_paths(tmp):
    return (os.path.join(tmp, "GeometryRelationShip_Crystal2Crystal").encode(),
            os.path.join(tmp, "GeometryRelationShip_Collimator2Crystal").encode())


def scatter(geo, pe_matrix, variant: str = "combined", cuda_id: int = 0, workdir=None, load_bitmaps=False):
    """Reference scatter program.  variant: combined | collimator | crystal.

    The bitmaps are computed by the reference (physics[8] = physics[9] = 1) and read back
    from the files it writes; with load_bitmaps (and a workdir holding the files of an earlier
    call) the reference reads them instead (physics[8] = physics[9] = 0).  Returns
    (dst (D,V) float32, bitmaps dict of uint32 arrays)."""
    if geo.n_rot != 1 and variant == "combined":
        raise ValueError("the combined reference sums D*V*R elements on the host; use R = 1")
    phys = geo.physics.copy()
    phys[8] = 0.0 if load_bitmaps else 1.0
    phys[9] = 0.0 if load_bitmaps else 1.0
    D, V = geo.n_det, geo.n_vox
    c, pc = _f(geo.collimator.copy())
    d, pd = _f(geo.detector.copy())
    i, pi = _f(geo.image.copy())
    p, pp = _f(phys)
    m, pm = _f(np.ascontiguousarray(pe_matrix, dtype=np.float32).reshape(-1)[:D * V].copy())
    out = np.zeros(D * V, dtype=np.float32)
    po = out.ctypes.data_as(_fp)
    own = workdir is None
    tmp = tempfile.mkdtemp(prefix="refgeo_") if own else workdir
    fcry, fcol = _geo_paths(tmp)
    with _stdout_to_stderr():
        if variant == "combined":
            lib = _load("libref_scatter.so")
            ret = lib.ref_scatter(pc, pd, pi, pp, pm, fcry, fcol, po, ctypes.c_int(cuda_id))
        elif variant == "collimator":
            lib = _load("libref_scatter_collimator.so")
            ret = lib.ref_scatter_collimator(pc, pd, pi, pp, pm, fcol, po, ctypes.c_int(cuda_id))
        elif variant == "crystal":
            lib = _load("libref_scatter_crystal.so")
            ret = lib.ref_scatter_crystal(pd, pi, pp, pm, fcry, po, ctypes.c_int(cuda_id))
        else:
            raise ValueError(variant)
    bitmaps = {}
    for key, path in (("crystal", fcry), ("collimator", fcol)):
        if os.path.exists(path):
            if own or not load_bitmaps:
                bitmaps[key] = np.fromfile(path.decode(), dtype=np.uint32)
            if own:
                os.remove(path)
    if own:
        os.rmdir(tmp)
    if ret not in (V, 0, None) and variant != "combined":
        pass
    return out.reshape(D, V), bitmaps


def ell_chords(args, cuda_id: int = 0) -> np.ndarray:
    """The reference's length_ellipticalcylinder_ray on rows of 13 arguments (x_in, y_in, z_in,
    x_out, y_out, z_out, xc, y1, y2, zc, rho_x, rho_z, theta), evaluated by a test kernel
    compiled with the unmodified reference source (oracle/ref/ref_ell.cu)."""
    a, pa = _f(np.asarray(args, dtype=np.float32).reshape(-1, 13))
    n = a.shape[0]
    out = np.zeros(n, dtype=np.float32)
    rc = _load("libref_ell.so").ref_ell_chords(pa, out.ctypes.data_as(_fp), ctypes.c_int(n), ctypes.c_int(cuda_id))
    if rc != 0:
        raise RuntimeError(f"ref_ell_chords failed ({rc})")
    return out
