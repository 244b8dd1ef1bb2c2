"""Python binding of libsysmat.so (ctypes) — the host-side mirror of the reference API.

`PESysMatGen` and the three `scatter` programs keep the reference's host-buffer calling
convention (PEGen_RayTracing_CircularHole/PESysMatGen.h:4-5 and the three scatter.h
headers).  `Context` exposes the native device API on torch CUDA tensors, which is what the
tests and the benchmark use.  The library must be built (make -C <this directory>); there
is no CPU fallback: every call fails loudly if the CUDA library is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsysmat.so")

OK = 0
ERRORS = {-1: "SYSMAT_ERR_ARG", -2: "SYSMAT_ERR_CUDA", -3: "SYSMAT_ERR_CAPACITY",
          -4: "SYSMAT_ERR_IO", -5: "SYSMAT_ERR_NOMEM", -6: "SYSMAT_ERR_TIMEOUT"}
MODE_REFERENCE = 0
MODE_PRECISE = 1
MODE_FP64 = 2
MODE_LOCAL = 3
THETA_N = 7
THETA_NAMES = ("mu_w", "mu_crystal", "radius", "dx", "dy", "dz", "tilt")
SCATTER_CRYSTAL = 1
SCATTER_COLLIMATOR = 2
HOLE_MODEL_COMBINED = 0
HOLE_MODEL_VARIANT = 1
HOLE_MODEL_NATIVE = 2

# Every symbol declared in include/sysmat.h.
EXPORTS = ("PESysMatGen", "scatter", "scatter_collimator", "scatter_crystal", "sysmat_create",
           "sysmat_destroy", "sysmat_dims", "sysmat_pe", "sysmat_bitmap_crystal_words",
           "sysmat_bitmap_collimator_words", "sysmat_bitmap_crystal", "sysmat_bitmap_collimator",
           "sysmat_scatter_prepare", "sysmat_scatter", "sysmat_pe_noalloc", "sysmat_csr_count",
           "sysmat_csr_fill", "sysmat_pe_work", "sysmat_batch_create", "sysmat_batch_set_tiles",
           "sysmat_batch_get_tiles", "sysmat_batch_tune", "sysmat_batch_run", "sysmat_batch_destroy",
           "sysmat_batch", "sysmat_scatter_prepare_native", "sysmat_set_hole_shapes", "sysmat_pe_csr_file", "sysmat_project", "sysmat_vjp", "sysmat_backproject",
           "sysmat_measure_peaks", "sysmat_ell_chords", "sysmat_pe_sampled", "sysmat_pe_sampled_mode",
           "sysmat_scatter_grid",
           "sysmat_scatter_batch_create", "sysmat_scatter_batch_run", "sysmat_scatter_batch_destroy",
           "sysmat_error_string", "sysmat_version")

_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p
_lib = None


class BatchItem(ctypes.Structure):
    """sysmat_batch_item: one (context, rotation, detector x voxel block) task of a batch."""
    _fields_ = [("ctx", ctypes.c_int), ("rotation", ctypes.c_float), ("det_begin", ctypes.c_int),
                ("det_count", ctypes.c_int), ("vox_begin", ctypes.c_longlong),
                ("vox_count", ctypes.c_longlong), ("d_out", ctypes.c_void_p), ("ld", ctypes.c_longlong)]


class SysmatError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        name = ERRORS.get(code, str(code))
        super().__init__(f"{what}: {name} ({lib().sysmat_error_string(code).decode()})")


def lib():
    """Load libsysmat.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        sigs = {
            "PESysMatGen": ([_fp, _fp, _fp, _fp, ctypes.c_int], ctypes.c_int),
            "scatter": ([_fp, _fp, _fp, _fp, _fp, ctypes.c_char_p, ctypes.c_char_p, _fp, ctypes.c_int],
                        ctypes.c_int),
            "scatter_collimator": ([_fp, _fp, _fp, _fp, _fp, ctypes.c_char_p, _fp, ctypes.c_int],
                                   ctypes.c_int),
            "scatter_crystal": ([_fp, _fp, _fp, _fp, ctypes.c_char_p, _fp, ctypes.c_int], ctypes.c_int),
            "sysmat_create": ([ctypes.POINTER(_vp), ctypes.c_int, _fp, _fp, _fp, _fp], ctypes.c_int),
            "sysmat_destroy": ([_vp], ctypes.c_int),
            "sysmat_dims": ([_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong),
                             ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                             ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
            "sysmat_pe": ([_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                           ctypes.c_longlong, _vp, ctypes.c_longlong, ctypes.c_int, _vp], ctypes.c_int),
            "sysmat_pe_sampled": ([_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                   ctypes.c_longlong, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   _vp, ctypes.c_longlong, _vp], ctypes.c_int),
            "sysmat_pe_sampled_mode": ([_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                        ctypes.c_longlong, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_int, _vp, ctypes.c_longlong, _vp],
                                       ctypes.c_int),
            "sysmat_bitmap_crystal_words": ([_vp], ctypes.c_longlong),
            "sysmat_bitmap_collimator_words": ([_vp], ctypes.c_longlong),
            "sysmat_bitmap_crystal": ([_vp, _vp, _vp], ctypes.c_int),
            "sysmat_bitmap_collimator": ([_vp, _vp, _vp], ctypes.c_int),
            "sysmat_scatter_prepare": ([_vp, ctypes.c_int, _vp, _vp, _vp], ctypes.c_int),
            "sysmat_scatter": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, _vp, ctypes.c_int,
                                ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, _vp,
                                ctypes.c_longlong, _vp], ctypes.c_int),
            "sysmat_pe_work": ([_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                ctypes.c_longlong, _vp, ctypes.c_longlong,
                                ctypes.POINTER(ctypes.c_ulonglong), _vp], ctypes.c_int),
            "sysmat_measure_peaks": ([ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
                                     ctypes.c_int),
            "sysmat_pe_noalloc": ([_fp, _fp, _fp, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_longlong, ctypes.c_longlong, _vp, ctypes.c_longlong,
                                   ctypes.c_int, _vp], ctypes.c_int),
            "sysmat_csr_count": ([_vp, ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_float,
                                  _vp, _vp, _vp], ctypes.c_int),
            "sysmat_csr_fill": ([_vp, ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_float,
                                 ctypes.c_longlong, _vp, _vp, _vp, _vp], ctypes.c_int),
            "sysmat_batch_create": ([ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.c_int,
                                     ctypes.POINTER(BatchItem), ctypes.c_int], ctypes.c_int),
            "sysmat_batch_set_tiles": ([_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int],
                                       ctypes.c_int),
            "sysmat_batch_get_tiles": ([_vp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
            "sysmat_batch_tune": ([_vp, ctypes.c_int, _vp, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
            "sysmat_batch_run": ([_vp, ctypes.c_int, _vp], ctypes.c_int),
            "sysmat_batch_destroy": ([_vp], ctypes.c_int),
            "sysmat_batch": ([ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(BatchItem), ctypes.c_int,
                              ctypes.c_int, _vp], ctypes.c_int),
            "sysmat_scatter_prepare_native": ([_vp, ctypes.c_int, _vp, _vp], ctypes.c_int),
            "sysmat_set_hole_shapes": ([_vp, _fp, _fp, _fp], ctypes.c_int),
            "sysmat_pe_csr_file": ([_vp, ctypes.c_float, ctypes.c_char_p, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_longlong), _vp], ctypes.c_int),
            "sysmat_project": ([_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp], ctypes.c_int),
            "sysmat_vjp": ([_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp], ctypes.c_int),
            "sysmat_backproject": ([_vp, ctypes.c_float, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp],
                                   ctypes.c_int),
            "sysmat_ell_chords": ([_vp, _vp, ctypes.c_int, _vp], ctypes.c_int),
            "sysmat_scatter_batch_create": ([ctypes.POINTER(_vp), _vp, ctypes.c_int, _vp, ctypes.c_int, _vp],
                                            ctypes.c_int),
            "sysmat_scatter_batch_run": ([_vp, _vp], ctypes.c_int),
            "sysmat_scatter_batch_destroy": ([_vp], ctypes.c_int),
            "sysmat_scatter_grid": ([_vp, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_longlong, ctypes.c_longlong, _vp, ctypes.c_longlong, _vp],
                                    ctypes.c_int),
            "sysmat_error_string": ([ctypes.c_int], ctypes.c_char_p),
            "sysmat_version": ([], ctypes.c_char_p),
        }
        for name, (args, res) in sigs.items():
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
        _lib = L
    return _lib


def _check(rc, what):
    if rc < 0:
        raise SysmatError(rc, what)
    return rc


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


# ---------------------------------------------------------------------------------------
# Reference-compatible entry points (host buffers).

def PESysMatGen(collimator, detector, image, dst, cuda_id=0):
    """dst: float32 numpy array of at least D*V elements (written in place).  Returns V."""
    c, pc = _f32(collimator)
    d, pd = _f32(detector)
    i, pi = _f32(image)
    if dst.dtype != np.float32 or not dst.flags.c_contiguous:
        raise ValueError("dst must be a contiguous float32 array")
    return _check(lib().PESysMatGen(pc, pd, pi, dst.ctypes.data_as(_fp), cuda_id), "PESysMatGen")


def scatter(collimator, detector, image, physics, pe, fname_crystal, fname_collimator, dst, cuda_id=0):
    c, pc = _f32(collimator)
    d, pd = _f32(detector)
    i, pi = _f32(image)
    p, pp = _f32(physics)
    m, pm = _f32(pe)
    return _check(lib().scatter(pc, pd, pi, pp, pm, fname_crystal.encode(), fname_collimator.encode(),
                                dst.ctypes.data_as(_fp), cuda_id), "scatter")


def scatter_collimator(collimator, detector, image, physics, pe, fname, dst, cuda_id=0):
    c, pc = _f32(collimator)
    d, pd = _f32(detector)
    i, pi = _f32(image)
    p, pp = _f32(physics)
    m, pm = _f32(pe)
    return _check(lib().scatter_collimator(pc, pd, pi, pp, pm, fname.encode(),
                                           dst.ctypes.data_as(_fp), cuda_id), "scatter_collimator")


def scatter_crystal(detector, image, physics, pe, fname, dst, cuda_id=0):
    d, pd = _f32(detector)
    i, pi = _f32(image)
    p, pp = _f32(physics)
    m, pm = _f32(pe)
    return _check(lib().scatter_crystal(pd, pi, pp, pm, fname.encode(), dst.ctypes.data_as(_fp),
                                        cuda_id), "scatter_crystal")


# ---------------------------------------------------------------------------------------
# Native API on torch CUDA tensors.

class Context:
    """One uploaded system on one device (sysmat_create / sysmat_destroy)."""

    def __init__(self, geo, device=0):
        import torch
        self.device = device
        torch.cuda.set_device(device)
        self._arrays = [_f32(geo.collimator), _f32(geo.detector), _f32(geo.image), _f32(geo.physics)]
        h = ctypes.c_void_p()
        (c, pc), (d, pd), (i, pi), (p, pp) = self._arrays
        _check(lib().sysmat_create(ctypes.byref(h), device, pc, pd, pi, pp), "sysmat_create")
        self.handle = h
        nd, nv, nh0, nh, nl = (ctypes.c_int(), ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int(),
                               ctypes.c_int())
        _check(lib().sysmat_dims(h, ctypes.byref(nd), ctypes.byref(nv), ctypes.byref(nh0),
                                 ctypes.byref(nh), ctypes.byref(nl)), "sysmat_dims")
        self.n_det, self.n_vox = nd.value, nv.value
        self.n_holes0, self.n_holes, self.n_layers = nh0.value, nh.value, nl.value

    def close(self):
        if self.handle:
            lib().sysmat_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pe(self, out, rotation=0.0, det_begin=0, det_count=None, vox_begin=0, vox_count=None,
           mode=MODE_REFERENCE, stream=None):
        """Fill `out` (CUDA float32, rows x >=vox_count, row-contiguous) with the PE block."""
        det_count = self.n_det - det_begin if det_count is None else det_count
        vox_count = self.n_vox - vox_begin if vox_count is None else vox_count
        ld = out.stride(0) if out.dim() == 2 else vox_count
        _check(lib().sysmat_pe(self.handle, float(rotation), det_begin, det_count, vox_begin, vox_count,
                               _ptr(out), ld, mode, _stream(stream)), "sysmat_pe")
        return out

    def pe_sampled(self, out, crystal_div=(8, 16, 8), voxel_sub=(1, 1, 1), rotation=0.0, det_begin=0,
                   det_count=None, vox_begin=0, vox_count=None, stream=None, mode=MODE_PRECISE):
        """Fill `out` with the PE block of the sampled form: crystal_div sub-elements of each
        crystal along x, depth, z and voxel_sub source points per voxel along x, y, z; each
        element is the mean over its source points (sysmat_pe_sampled_mode).  mode: MODE_PRECISE
        (the reference's float program, FP64 sums) or MODE_LOCAL (the local-coordinate FP32
        form, within 1e-5 of FP64)."""
        det_count = self.n_det - det_begin if det_count is None else det_count
        vox_count = self.n_vox - vox_begin if vox_count is None else vox_count
        ld = out.stride(0) if out.dim() == 2 else vox_count
        dv = (ctypes.c_int * 3)(*[int(x) for x in crystal_div])
        sv = (ctypes.c_int * 3)(*[int(x) for x in voxel_sub])
        _check(lib().sysmat_pe_sampled_mode(self.handle, float(rotation), det_begin, det_count, vox_begin,
                                            vox_count, dv, sv, int(mode), _ptr(out), ld, _stream(stream)),
               "sysmat_pe_sampled_mode")
        return out

    def pe_work(self, out, rotation=0.0, det_begin=0, det_count=None, vox_begin=0, vox_count=None,
                stream=None):
        """Reference-mode PE block with work counters; returns a dict of counts."""
        det_count = self.n_det - det_begin if det_count is None else det_count
        vox_count = self.n_vox - vox_begin if vox_count is None else vox_count
        ld = out.stride(0) if out.dim() == 2 else vox_count
        c = (ctypes.c_ulonglong * 12)()
        _check(lib().sysmat_pe_work(self.handle, float(rotation), det_begin, det_count, vox_begin,
                                    vox_count, _ptr(out), ld, c, _stream(stream)), "sysmat_pe_work")
        keys = ("subelements", "hole_hits", "crystal_hits", "elements", "blocked", "chunked",
                "kept", "sublist_entries", "superset_overflow", "superset_sum", "hole_evals",
                "crystal_evals")
        return dict(zip(keys, (int(x) for x in c)))

    def bitmap_crystal(self, stream=None):
        import torch
        n = lib().sysmat_bitmap_crystal_words(self.handle)
        out = torch.empty(max(n, 1), dtype=torch.int32, device=f"cuda:{self.device}")
        _check(lib().sysmat_bitmap_crystal(self.handle, _ptr(out), _stream(stream)), "bitmap_crystal")
        return out[:n]

    def bitmap_collimator(self, stream=None):
        import torch
        n = lib().sysmat_bitmap_collimator_words(self.handle)
        out = torch.empty(max(n, 1), dtype=torch.int32, device=f"cuda:{self.device}")
        _check(lib().sysmat_bitmap_collimator(self.handle, _ptr(out), _stream(stream)),
               "bitmap_collimator")
        return out[:n]

    def scatter_prepare(self, bm_crystal=None, bm_collimator=None,
                        parts=SCATTER_CRYSTAL | SCATTER_COLLIMATOR, stream=None):
        nullp = ctypes.c_void_p(0)
        _check(lib().sysmat_scatter_prepare(self.handle, parts,
                                            _ptr(bm_crystal) if bm_crystal is not None else nullp,
                                            _ptr(bm_collimator) if bm_collimator is not None else nullp,
                                            _stream(stream)), "sysmat_scatter_prepare")

    def scatter_prepare_native(self, bm_crystal=None, parts=SCATTER_CRYSTAL | SCATTER_COLLIMATOR, stream=None):
        """Pair tables of the native model (sysmat_scatter_prepare_native); then call scatter with
        hole_model=HOLE_MODEL_NATIVE."""
        nullp = ctypes.c_void_p(0)
        _check(lib().sysmat_scatter_prepare_native(self.handle, parts,
                                                   _ptr(bm_crystal) if bm_crystal is not None else nullp,
                                                   _stream(stream)), "sysmat_scatter_prepare_native")

    def scatter(self, out, pe=None, parts=SCATTER_CRYSTAL | SCATTER_COLLIMATOR,
                hole_model=HOLE_MODEL_COMBINED, rotation=0.0, det_begin=0, det_count=None,
                vox_begin=0, vox_count=None, stream=None):
        det_count = self.n_det - det_begin if det_count is None else det_count
        vox_count = self.n_vox - vox_begin if vox_count is None else vox_count
        ld = out.stride(0) if out.dim() == 2 else vox_count
        _check(lib().sysmat_scatter(self.handle, parts, hole_model, float(rotation),
                                    _ptr(pe) if pe is not None else ctypes.c_void_p(0), det_begin,
                                    det_count, vox_begin, vox_count, _ptr(out), ld, _stream(stream)),
               "sysmat_scatter")
        return out


def _context_project(self, x, p=None, rotation=0.0, det_begin=0, det_count=None, stream=None):
    """p = A x over all voxels (x: CUDA float32 of n_vox); returns a float64 CUDA tensor."""
    import torch
    det_count = self.n_det - det_begin if det_count is None else det_count
    p = torch.empty(det_count, dtype=torch.float64, device=x.device) if p is None else p
    _check(lib().sysmat_project(self.handle, float(rotation), det_begin, det_count, _ptr(x), _ptr(p),
                                _stream(stream)), "sysmat_project")
    return p


def _context_vjp(self, x, u, rotation=0.0, det_begin=0, det_count=None, stream=None):
    """d(u^T A x)/d theta (float64 CUDA tensor of THETA_N + 1; the last entry is u^T A x)."""
    import torch
    det_count = self.n_det - det_begin if det_count is None else det_count
    g = torch.empty(THETA_N + 1, dtype=torch.float64, device=x.device)
    _check(lib().sysmat_vjp(self.handle, float(rotation), det_begin, det_count, _ptr(x), _ptr(u), _ptr(g),
                            _stream(stream)), "sysmat_vjp")
    return g


def _context_backproject(self, u, rotation=0.0, det_begin=0, det_count=None, stream=None):
    """q = A^T u (u: CUDA float32 of det_count); returns a float64 CUDA tensor of n_vox."""
    import torch
    det_count = self.n_det - det_begin if det_count is None else det_count
    q = torch.empty(self.n_vox, dtype=torch.float64, device=u.device)
    _check(lib().sysmat_backproject(self.handle, float(rotation), det_begin, det_count, _ptr(u), _ptr(q),
                                    _stream(stream)), "sysmat_backproject")
    return q


def _context_pe_csr_file(self, path, rotation=0.0, threshold=1e-9, mode=MODE_REFERENCE, rows_per_block=0,
                         stream=None):
    """Whole PE matrix of one rotation to a compressed file (sysmat_pe_csr_file); returns nnz."""
    n = ctypes.c_longlong()
    _check(lib().sysmat_pe_csr_file(self.handle, float(rotation), os.fsencode(path), float(threshold), mode,
                                    int(rows_per_block), ctypes.byref(n), _stream(stream)), "sysmat_pe_csr_file")
    return n.value


def read_csr_file(path):
    """Read a sysmat_pe_csr_file file: (rows, cols, threshold, mode, row_ptr int64, col int64,
    val float32), rows assembled in order."""
    with open(path, "rb") as f:
        head = f.read(40)
        if head[:8] != b"SMCSR001":
            raise ValueError(f"{path}: not a sysmat CSR file")
        rows, cols = np.frombuffer(head[8:24], dtype=np.int64)
        threshold = float(np.frombuffer(head[24:28], dtype=np.float32)[0])
        mode = int(np.frombuffer(head[28:32], dtype=np.int32)[0])
        ptr = [np.zeros(1, dtype=np.int64)]
        cols_l, vals_l = [], []
        base = 0
        next_row = 0
        while True:
            b = f.read(24)
            if not b:
                break
            d0, n, nnz = np.frombuffer(b, dtype=np.int64)
            if d0 != next_row:
                raise ValueError(f"{path}: block starts at row {d0}, expected {next_row}")
            rp = np.frombuffer(f.read(8 * (n + 1)), dtype=np.int64)
            cols_l.append(np.frombuffer(f.read(8 * nnz), dtype=np.int64))
            vals_l.append(np.frombuffer(f.read(4 * nnz), dtype=np.float32))
            ptr.append(rp[1:] + base)
            base += int(nnz)
            next_row += int(n)
    if next_row != rows:
        raise ValueError(f"{path}: {next_row} rows of {rows}")
    cat = (lambda xs, t: np.concatenate(xs) if xs else np.zeros(0, dtype=t))
    return int(rows), int(cols), threshold, mode, np.concatenate(ptr), cat(cols_l, np.int64), cat(vals_l, np.float32)


def _context_set_hole_shapes(self, shapes=None):
    """shapes: (n_holes, 3) rows (rho_x, rho_z, theta), rho_x <= 0 for a circular hole; None
    restores circular holes (sysmat_set_hole_shapes)."""
    if shapes is None:
        _check(lib().sysmat_set_hole_shapes(self.handle, None, None, None), "sysmat_set_hole_shapes")
        return
    a = np.ascontiguousarray(np.asarray(shapes, dtype=np.float32).reshape(-1, 3))
    cols = [np.ascontiguousarray(a[:, k]) for k in range(3)]
    self._shapes = cols
    _check(lib().sysmat_set_hole_shapes(self.handle, *[c.ctypes.data_as(_fp) for c in cols]),
           "sysmat_set_hole_shapes")


def _context_scatter_columns(self, out, vox_begin, vox_count, parts=SCATTER_CRYSTAL | SCATTER_COLLIMATOR,
                             hole_model=HOLE_MODEL_COMBINED, rotation=0.0, pe=None, stream=None):
    """Scatter for every detector over voxel columns [vox_begin, vox_begin + vox_count) with the
    photoelectric columns it reads computed here (the unit a rank owns when voxels are split
    across ranks: no PE exchange).  The pair tables must be prepared.  `out`: CUDA float32,
    n_det rows x vox_count; `pe`: optional n_det x n_vox scratch (its other columns are left
    as they are).  Returns `out`."""
    import torch
    if pe is None:
        pe = torch.zeros((self.n_det, self.n_vox), dtype=torch.float32, device=out.device)
    if parts & SCATTER_CRYSTAL:
        self.pe(pe[:, vox_begin:vox_begin + vox_count], rotation=rotation, vox_begin=vox_begin, vox_count=vox_count,
                stream=stream)
    return self.scatter(out, pe, parts=parts, hole_model=hole_model, rotation=rotation, vox_begin=vox_begin,
                        vox_count=vox_count, stream=stream)


def _context_scatter_grid(self, out, parts=SCATTER_CRYSTAL | SCATTER_COLLIMATOR, cell=0.25, rotation=0.0,
                          det_begin=0, det_count=None, vox_begin=0, vox_count=None, stream=None):
    """Grid scatter model (sysmat_scatter_grid): scatter points on a `cell` mm grid inside the
    crystals (parts bit SCATTER_CRYSTAL) and the collimator's tungsten (SCATTER_COLLIMATOR),
    FP64 sums per element.  `out`: CUDA float32, det_count rows."""
    det_count = self.n_det - det_begin if det_count is None else det_count
    vox_count = self.n_vox - vox_begin if vox_count is None else vox_count
    ld = out.stride(0) if out.dim() == 2 else vox_count
    _check(lib().sysmat_scatter_grid(self.handle, int(parts), float(cell), float(rotation), det_begin, det_count,
                                     vox_begin, vox_count, _ptr(out), ld, _stream(stream)), "sysmat_scatter_grid")
    return out


Context.scatter_grid = _context_scatter_grid
Context.scatter_columns = _context_scatter_columns
Context.set_hole_shapes = _context_set_hole_shapes
Context.pe_csr_file = _context_pe_csr_file
Context.project = _context_project
Context.vjp = _context_vjp
Context.backproject = _context_backproject


class ScatterItem(ctypes.Structure):
    """sysmat_scatter_item: one scatter task (what one sysmat_scatter call takes)."""
    _fields_ = [("ctx", ctypes.c_int), ("parts", ctypes.c_int), ("hole_model", ctypes.c_int),
                ("rotation", ctypes.c_float), ("d_pe", ctypes.c_void_p), ("det_begin", ctypes.c_int),
                ("det_count", ctypes.c_int), ("vox_begin", ctypes.c_longlong), ("vox_count", ctypes.c_longlong),
                ("d_out", ctypes.c_void_p), ("ld", ctypes.c_longlong)]


class ScatterBatchPlan:
    """Many scatter tasks in one persistent launch (sysmat_scatter_batch_*).  items: tuples
    (ctx_index, parts, hole_model, rotation, pe, det_begin, det_count, vox_begin, vox_count, out)
    with `pe` a CUDA float32 PE matrix (or None without the crystal part) and `out` a CUDA
    float32 tensor of det_count rows.  Keep the contexts, PE matrices and outputs alive."""

    def __init__(self, contexts, items, stream=None):
        self._keep = (list(contexts), [(it[4], it[9]) for it in items])
        arr = (ScatterItem * max(len(items), 1))()
        for k, (c, parts, model, rot, pe, d0, nd, v0, nv, out) in enumerate(items):
            ld = out.stride(0) if out.dim() == 2 else nv
            arr[k] = ScatterItem(int(c), int(parts), int(model), float(rot), pe.data_ptr() if pe is not None else 0,
                                 int(d0), int(nd), int(v0), int(nv), out.data_ptr(), int(ld))
        ctxs = (_vp * len(contexts))(*[c.handle.value for c in contexts])
        h = ctypes.c_void_p()
        _check(lib().sysmat_scatter_batch_create(ctypes.byref(h), ctxs, len(contexts), arr, len(items),
                                                 _stream(stream)), "sysmat_scatter_batch_create")
        self.handle = h

    def run(self, stream=None):
        _check(lib().sysmat_scatter_batch_run(self.handle, _stream(stream)), "sysmat_scatter_batch_run")

    def close(self):
        if self.handle:
            lib().sysmat_scatter_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _batch_items(contexts, items):
    """items: iterables (ctx_index, rotation, det_begin, det_count, vox_begin, vox_count, out)
    with `out` a CUDA float32 tensor of det_count rows (row-contiguous)."""
    arr = (BatchItem * max(len(items), 1))()
    for k, (c, rot, d0, nd, v0, nv, out) in enumerate(items):
        ld = out.stride(0) if out.dim() == 2 else nv
        arr[k] = BatchItem(int(c), float(rot), int(d0), int(nd), int(v0), int(nv), out.data_ptr(), int(ld))
    ctxs = (_vp * len(contexts))(*[c.handle.value for c in contexts])
    return ctxs, arr


class BatchPlan:
    """Many (system, rotation, block) PE tasks in one persistent launch (sysmat_batch_*).

    The plan refers to the contexts' device tables and to the output tensors: keep them alive
    while the plan is used."""

    def __init__(self, contexts, items):
        self._keep = (list(contexts), [it[-1] for it in items])
        ctxs, arr = _batch_items(contexts, items)
        h = ctypes.c_void_p()
        _check(lib().sysmat_batch_create(ctypes.byref(h), ctxs, len(contexts), arr, len(items)),
               "sysmat_batch_create")
        self.handle = h

    def set_tiles(self, bx, by, bz, blocks_per_sm=0):
        _check(lib().sysmat_batch_set_tiles(self.handle, bx, by, bz, blocks_per_sm), "sysmat_batch_set_tiles")

    def tiles(self):
        t = (ctypes.c_int * 4)()
        _check(lib().sysmat_batch_get_tiles(self.handle, t), "sysmat_batch_get_tiles")
        return tuple(t)

    def tune(self, mode=MODE_REFERENCE, stream=None):
        t = (ctypes.c_int * 4)()
        _check(lib().sysmat_batch_tune(self.handle, mode, _stream(stream), t), "sysmat_batch_tune")
        return tuple(t)

    def run(self, mode=MODE_REFERENCE, stream=None):
        _check(lib().sysmat_batch_run(self.handle, mode, _stream(stream)), "sysmat_batch_run")

    def close(self):
        if self.handle:
            lib().sysmat_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch(contexts, items, mode=MODE_REFERENCE, stream=None):
    """One-shot batched PE (sysmat_batch): create, run, synchronise, destroy."""
    ctxs, arr = _batch_items(contexts, items)
    _check(lib().sysmat_batch(ctxs, len(contexts), arr, len(items), mode, _stream(stream)), "sysmat_batch")


def ell_chords(args, stream=None):
    """Device elliptical-cylinder chord on a CUDA float32 tensor of (n, 13) arguments."""
    import torch
    args = args.contiguous()
    out = torch.empty(args.shape[0], dtype=torch.float32, device=args.device)
    _check(lib().sysmat_ell_chords(_ptr(args), _ptr(out), args.shape[0], _stream(stream)), "sysmat_ell_chords")
    return out


def measure_peaks():
    """(FP32 TFLOP/s, MUFU Tops/s) measured on the current device."""
    f, m = ctypes.c_double(), ctypes.c_double()
    _check(lib().sysmat_measure_peaks(ctypes.byref(f), ctypes.byref(m)), "sysmat_measure_peaks")
    return f.value, m.value


def pe_noalloc(geo, out, rotation=0.0, det_begin=0, det_count=None, vox_begin=0, vox_count=None,
               mode=MODE_REFERENCE, stream=None):
    """Photoelectric block through sysmat_pe_noalloc (no device allocation; host parameter
    arrays, `out` a CUDA float32 tensor).  Returns `out`."""
    (c, pc), (d, pd), (i, pi) = _f32(geo.collimator), _f32(geo.detector), _f32(geo.image)
    # the crystal count as the library decodes it: floor(pD[0] + 1e-6) in float32
    n_det = int(np.floor(np.float32(geo.detector[0]) + np.float32(0.000001)))
    n_vox = geo.n_vox
    det_count = n_det - det_begin if det_count is None else det_count
    vox_count = n_vox - vox_begin if vox_count is None else vox_count
    ld = out.stride(0) if out.dim() == 2 else vox_count
    _check(lib().sysmat_pe_noalloc(pc, pd, pi, float(rotation), det_begin, det_count, vox_begin,
                                   vox_count, _ptr(out), ld, mode, _stream(stream)),
           "sysmat_pe_noalloc")
    return out


def to_csr(dense, threshold=1e-9, col_offset=0, stream=None):
    """CSR (row_ptr int64 [rows+1], col_idx int64, values float32) of a CUDA float32 block,
    keeping entries > threshold.  Two device passes; one small host read of the total."""
    import torch
    rows, cols = dense.shape
    ld = dense.stride(0)
    dev = dense.device
    nnz = torch.empty(rows, dtype=torch.int64, device=dev)
    ptr = torch.empty(rows + 1, dtype=torch.int64, device=dev)
    _check(lib().sysmat_csr_count(_ptr(dense), rows, cols, ld, float(threshold), _ptr(nnz), _ptr(ptr),
                                  _stream(stream)), "sysmat_csr_count")
    total = int(ptr[rows].item())
    col = torch.empty(max(total, 1), dtype=torch.int64, device=dev)
    val = torch.empty(max(total, 1), dtype=torch.float32, device=dev)
    _check(lib().sysmat_csr_fill(_ptr(dense), rows, cols, ld, float(threshold), int(col_offset), _ptr(ptr),
                                 _ptr(col), _ptr(val), _stream(stream)), "sysmat_csr_fill")
    return ptr, col[:total], val[:total]
