"""Test infrastructure only: ctypes binding of the CPU oracle (liboracle.so).

The oracle restates the reference's algorithm in C (sysmat_oracle.c, oracle_body.h) in
two precisions: 32 = the reference's float arithmetic, 64 = the same program widened to
double.  Tests, the smoke check and bench.py's CPU-baseline leg use it as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i64p = ctypes.POINTER(ctypes.c_longlong)


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_pe.argtypes = [_fp, _fp, _fp, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_longlong,
                                ctypes.c_longlong, _dp, _i64p, ctypes.c_int]
        L.oracle_pe.restype = ctypes.c_int
        L.oracle_scatter.argtypes = [_fp, _fp, _fp, _fp, _fp, _u32p, ctypes.c_int, ctypes.c_int, _ip,
                                     ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, _dp,
                                     ctypes.c_int]
        L.oracle_scatter.restype = ctypes.c_int
        L.oracle_bitmap_crystal_words.argtypes = [_fp]
        L.oracle_bitmap_crystal_words.restype = ctypes.c_longlong
        L.oracle_bitmap_collimator_words.argtypes = [_fp, _fp]
        L.oracle_bitmap_collimator_words.restype = ctypes.c_longlong
        L.oracle_bitmap_crystal.argtypes = [_fp, _u32p, ctypes.c_int]
        L.oracle_bitmap_collimator.argtypes = [_fp, _fp, _u32p, ctypes.c_int]
        L.oracle_pe_shapes.argtypes = [_fp, _fp, _fp, _fp, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_longlong,
                                       ctypes.c_longlong, _dp, _i64p, ctypes.c_int]
        L.oracle_pe_shapes.restype = ctypes.c_int
        L.oracle_pe_sampled.argtypes = [_fp, _fp, _fp, _fp, _ip, _ip, ctypes.c_int, _ip, ctypes.c_int,
                                        ctypes.c_longlong, ctypes.c_longlong, _dp, ctypes.c_int]
        L.oracle_pe_sampled.restype = ctypes.c_int
        L.oracle_pe_local.argtypes = [_fp, _fp, _fp, _ip, ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, _dp,
                                      ctypes.c_int]
        L.oracle_pe_local.restype = ctypes.c_int
        L.oracle_pe_local_sampled.argtypes = [_fp, _fp, _fp, _fp, _ip, _ip, _ip, ctypes.c_int, ctypes.c_longlong,
                                              ctypes.c_longlong, _dp, ctypes.c_int]
        L.oracle_pe_local_sampled.restype = ctypes.c_int
        L.oracle_pe_subelements.argtypes = [_fp, _fp, _fp, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, _dp]
        L.oracle_pe_subelements.restype = ctypes.c_int
        L.oracle_scatter_grid.argtypes = [_fp, _fp, _fp, _fp, _fp, ctypes.c_int, ctypes.c_double, _ip, ctypes.c_int,
                                          ctypes.c_longlong, ctypes.c_longlong, _dp, ctypes.c_int]
        L.oracle_scatter_grid.restype = ctypes.c_int
        for name in ("oracle_box_chord", "oracle_box_chord_inside", "oracle_cyl_chord", "oracle_ell_chord"):
            getattr(L, name).argtypes = [ctypes.c_int, _dp]
            getattr(L, name).restype = ctypes.c_double
        L.oracle_scatter_trace.argtypes = [_fp, _fp, _fp, _fp, _fp, _u32p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_longlong, _dp]
        L.oracle_scatter_trace.restype = ctypes.c_double
        L.oracle_kn_sum.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.oracle_kn_sum.restype = ctypes.c_double
        _lib = L
    return _lib


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


def _dets(geo, dets):
    if dets is None:
        dets = np.arange(geo.n_det)
    d = np.ascontiguousarray(np.asarray(dets, dtype=np.int32))
    return d, d.ctypes.data_as(_ip)


def pe(geo, prec=64, dets=None, v0=0, nv=None, threads=0, counts=False, shapes=None):
    """PE elements (len(dets), nv) as float64; with counts=True also the per-element work
    counts (subelements, hole hits, crystal hits, candidate crystals, candidate holes).
    shapes: optional (n_holes, 3) float32 rows (rho_x, rho_z, theta); rho_x > 0 marks an
    elliptical hole (the reference's length_ellipticalcylinder_ray)."""
    nv = geo.n_vox - v0 if nv is None else nv
    c, pc = _f32(geo.collimator)
    d, pd = _f32(geo.detector)
    i, pi = _f32(geo.image)
    dd, pdd = _dets(geo, dets)
    out = np.zeros((dd.size, nv), dtype=np.float64)
    cnt = np.zeros((dd.size, nv, 5), dtype=np.int64) if counts else None
    if shapes is not None:
        sh, psh = _f32(np.asarray(shapes, dtype=np.float32).reshape(-1))
        rc = lib().oracle_pe_shapes(pc, pd, pi, psh, prec, pdd, dd.size, v0, nv, out.ctypes.data_as(_dp),
                                    cnt.ctypes.data_as(_i64p) if counts else None, threads)
    else:
        rc = lib().oracle_pe(pc, pd, pi, prec, pdd, dd.size, v0, nv, out.ctypes.data_as(_dp),
                             cnt.ctypes.data_as(_i64p) if counts else None, threads)
    if rc:
        raise RuntimeError(f"oracle_pe failed ({rc})")
    return (out, cnt) if counts else out


def pe_local(geo, dets=None, v0=0, nv=None, threads=0, crystal_div=(8, 16, 8), voxel_sub=(1, 1, 1), shapes=None):
    """PE elements (len(dets), nv) of the local-coordinate FP32 form (oracle_local.h) with the
    given crystal division and voxel source points (the element is the mean over the source
    points), as float values widened to float64.  shapes: optional elliptical holes, as in pe."""
    nv = geo.n_vox - v0 if nv is None else nv
    c, pc = _f32(geo.collimator)
    d, pd = _f32(geo.detector)
    i, pi = _f32(geo.image)
    dd, pdd = _dets(geo, dets)
    dv = np.ascontiguousarray(crystal_div, dtype=np.int32)
    sv = np.ascontiguousarray(voxel_sub, dtype=np.int32)
    out = np.zeros((dd.size, nv), dtype=np.float64)
    psh = None
    if shapes is not None:
        sh, psh = _f32(np.asarray(shapes, dtype=np.float32).reshape(-1))
    rc = lib().oracle_pe_local_sampled(pc, pd, pi, psh, dv.ctypes.data_as(_ip), sv.ctypes.data_as(_ip), pdd,
                                       dd.size, v0, nv, out.ctypes.data_as(_dp), threads)
    if rc:
        raise RuntimeError(f"oracle_pe_local_sampled failed ({rc})")
    return out


def pe_sampled(geo, crystal_div, voxel_sub, prec=64, dets=None, v0=0, nv=None, threads=0, shapes=None):
    """PE elements of the sampled form (len(dets), nv) as float64: crystal_div sub-elements of
    each crystal along x, depth, z and voxel_sub source points per voxel along x, y, z, the
    element being the mean over the source points (see oracle_pe_sampled).  shapes as for pe()."""
    nv = geo.n_vox - v0 if nv is None else nv
    c, pc = _f32(geo.collimator)
    d, pd = _f32(geo.detector)
    i, pi = _f32(geo.image)
    dd, pdd = _dets(geo, dets)
    dv = np.ascontiguousarray(np.asarray(crystal_div, dtype=np.int32).reshape(3))
    sv = np.ascontiguousarray(np.asarray(voxel_sub, dtype=np.int32).reshape(3))
    out = np.zeros((dd.size, nv), dtype=np.float64)
    sh, psh = _f32(np.asarray(shapes, dtype=np.float32).reshape(-1)) if shapes is not None else (None, None)
    rc = lib().oracle_pe_sampled(pc, pd, pi, psh, dv.ctypes.data_as(_ip), sv.ctypes.data_as(_ip), prec, pdd, dd.size,
                                 v0, nv, out.ctypes.data_as(_dp), threads)
    if rc:
        raise RuntimeError(f"oracle_pe_sampled failed ({rc})")
    return out


def ell_chord(args, prec=64):
    """The reference's elliptical-cylinder chord on 13 arguments (see oracle_ell_chord)."""
    a = np.ascontiguousarray(np.asarray(args, dtype=np.float64))
    return lib().oracle_ell_chord(prec, a.ctypes.data_as(_dp))


def bitmap_crystal(geo, threads=0):
    d, pd = _f32(geo.detector)
    n = lib().oracle_bitmap_crystal_words(pd)
    out = np.zeros(n, dtype=np.uint32)
    lib().oracle_bitmap_crystal(pd, out.ctypes.data_as(_u32p), threads)
    return out


def bitmap_collimator(geo, threads=0):
    c, pc = _f32(geo.collimator)
    d, pd = _f32(geo.detector)
    n = lib().oracle_bitmap_collimator_words(pc, pd)
    out = np.zeros(n, dtype=np.uint32)
    lib().oracle_bitmap_collimator(pc, pd, out.ctypes.data_as(_u32p), threads)
    return out


PART = {"crystal": 1, "collimator": 2, "collimator_variant": 3, "collimator_native": 4}


def scatter(geo, pe_matrix, part, bitmap, prec=64, dets=None, v0=0, nv=None, threads=0):
    """Scatter elements for part 'crystal', 'collimator' (combined program),
    'collimator_variant' (collimator-only program) or 'collimator_native' (the library's
    native model: holes of every layer, their layer's mu, tungsten attenuation of the
    scattered photon; `bitmap` is not read); float64 (len(dets), nv)."""
    nv = geo.n_vox - v0 if nv is None else nv
    c, pc = _f32(geo.collimator)
    d, pd = _f32(geo.detector)
    i, pi = _f32(geo.image)
    p, pp = _f32(geo.physics)
    m, pm = _f32(np.asarray(pe_matrix, dtype=np.float32).reshape(-1))
    b = np.ascontiguousarray(bitmap, dtype=np.uint32)
    dd, pdd = _dets(geo, dets)
    out = np.zeros((dd.size, nv), dtype=np.float64)
    rc = lib().oracle_scatter(pc, pd, pi, pp, pm, b.ctypes.data_as(_u32p), PART[part], prec, pdd,
                              dd.size, v0, nv, out.ctypes.data_as(_dp), threads)
    if rc:
        raise RuntimeError(f"oracle_scatter failed ({rc})")
    return out


def pe_subelements(geo, d, v, which=64):
    """The 1024 sub-element contributions of element (d, v) (index (iz * 8 + ix) * 16 + iy):
    which = 64 FP64 restatement, 32 FP32 twin, 'local' the local-coordinate FP32 form."""
    c, pc = _f32(geo.collimator)
    dd, pd = _f32(geo.detector)
    i, pi = _f32(geo.image)
    out = np.zeros(1024, dtype=np.float64)
    w = 0 if which == "local" else int(which)
    rc = lib().oracle_pe_subelements(pc, pd, pi, w, int(d), int(v), out.ctypes.data_as(_dp))
    if rc:
        raise RuntimeError(f"oracle_pe_subelements failed ({rc})")
    return out


def scatter_grid(geo, parts=3, cell=0.25, dets=None, v0=0, nv=None, threads=0, shapes=None):
    """Elements (len(dets), nv) of the grid scatter model (oracle_grid.h) in double: parts 1 =
    crystal cells, 2 = septal cells; cell = grid step in mm; shapes: optional elliptical holes,
    as in pe."""
    nv = geo.n_vox - v0 if nv is None else nv
    c, pc = _f32(geo.collimator)
    d, pd = _f32(geo.detector)
    i, pi = _f32(geo.image)
    p, pp = _f32(geo.physics)
    dd, pdd = _dets(geo, dets)
    out = np.zeros((dd.size, nv), dtype=np.float64)
    psh = None
    if shapes is not None:
        sh, psh = _f32(np.asarray(shapes, dtype=np.float32).reshape(-1))
    rc = lib().oracle_scatter_grid(pc, pd, pi, pp, psh, int(parts), float(cell), pdd, dd.size, v0, nv,
                                   out.ctypes.data_as(_dp), threads)
    if rc:
        raise RuntimeError(f"oracle_scatter_grid failed ({rc})")
    return out


def box_chord(args, prec=64):
    a = np.ascontiguousarray(args, dtype=np.float64)
    return lib().oracle_box_chord(prec, a.ctypes.data_as(_dp))


def box_chord_inside(args, prec=64):
    a = np.ascontiguousarray(args, dtype=np.float64)
    return lib().oracle_box_chord_inside(prec, a.ctypes.data_as(_dp))


def cyl_chord(args, prec=64):
    a = np.ascontiguousarray(args, dtype=np.float64)
    return lib().oracle_cyl_chord(prec, a.ctypes.data_as(_dp))


def kn_sum(e0, lo, hi, prec=64):
    return lib().oracle_kn_sum(prec, e0, lo, hi)


def scatter_trace(geo, pe_matrix, part, bitmap, d, v, prec=64):
    """(element value, per-item trace array (n_items, 9)) for one scatter element."""
    c, pc = _f32(geo.collimator)
    dd, pd = _f32(geo.detector)
    i, pi = _f32(geo.image)
    p, pp = _f32(geo.physics)
    m, pm = _f32(np.asarray(pe_matrix, dtype=np.float32).reshape(-1))
    b = np.ascontiguousarray(bitmap, dtype=np.uint32)
    n = geo.n_det if part == "crystal" else (geo.n_holes if part == "collimator_native" else geo.n_holes_layer0)
    tr = np.full((n, 9), np.nan)
    val = lib().oracle_scatter_trace(pc, pd, pi, pp, pm, b.ctypes.data_as(_u32p), PART[part], prec, d, v,
                                     tr.ctypes.data_as(_dp))
    return val, tr
