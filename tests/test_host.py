"""CPU tests of the host side: parameter layout and generator, the C ABI (loads, exports
every declared symbol, rejects bad input without touching a GPU), and the multi-rank
partitioning with world_size 2 over gloo."""
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import PKG_DIR, ROOT, _load, geometry, sysmat

sharding = _load("sysmat_sharding", os.path.join(PKG_DIR, "sharding.py"))


# ---- parameter files -------------------------------------------------------------------

def test_config_sizes():
    assert (geometry.config1().n_det, geometry.config1().n_vox) == (256, 1024)
    g2 = geometry.config2()
    assert (g2.n_det, g2.n_vox, g2.n_holes) == (4096, 96 * 96 * 32, 48 * 48)
    g3 = geometry.config3()
    assert (g3.n_det, g3.n_vox, g3.n_holes_layer0) == (1024, 48 * 48 * 16, 1024)


def test_layout_indices_follow_reference():
    g = geometry.mini(layers=2)
    c, d = g.collimator, g.detector
    assert c[0] == 2 and c[10] == 25 and c[20] == 25          # layer headers at (m+1)*10
    assert c[12] == 6.0 and c[22] == 6.0                      # thickness
    assert c[100 + 9 * 25 + 1] == pytest.approx(7.0 - 3.0)    # first hole of layer 1: y1
    assert d[0] == 36 and d[12 * 0 + 4] == 2.0 and d[12 * 0 + 5] == 5.0
    assert d[12 * 0 + 9] == pytest.approx(0.23 - 0.18)


def test_params_file_round_trip():
    g = geometry.mini(seed=3, rotated=True)
    with tempfile.TemporaryDirectory() as tmp:
        g.write(tmp)
        sizes = {f: os.path.getsize(os.path.join(tmp, f)) for f in os.listdir(tmp)}
        assert sizes["Params_Collimator.dat"] == 80000 * 4 and sizes["Params_Image.dat"] == 400
        h = geometry.read_params(tmp)
    for a, b in ((g.collimator, h.collimator), (g.detector, h.detector), (g.image, h.image),
                 (g.physics, h.physics)):
        assert np.array_equal(a, b)


def test_short_params_file_is_zero_padded():
    g = geometry.mini()
    with tempfile.TemporaryDirectory() as tmp:
        g.write(tmp)
        g.physics[:10].astype(np.float32).tofile(os.path.join(tmp, "Params_Physics.dat"))
        h = geometry.read_params(tmp)
    assert h.physics.size == 100 and np.all(h.physics[10:] == 0)


def _voxel_centres(img):
    nx, ny, nz = (int(np.floor(np.float32(img[i]))) for i in range(3))
    w = img[3:6].astype(np.float32)
    s = img[8:11].astype(np.float32)
    ix, iy, iz = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    f = np.float32
    x = (ix.astype(f) - f(nx) / f(2) + f(0.5)) * w[0] + s[0]
    y = (iy.astype(f) - f(ny) / f(2) + f(0.5)) * w[1] + s[1]
    z = (iz.astype(f) - f(nz) / f(2) + f(0.5)) * w[2] + s[2]
    return np.stack([x, y, z], -1)


@pytest.mark.parametrize("iz,iy0,ny", [(0, 0, None), (16, 40, 8), (31, 95, 1)])
def test_voxel_slab_reproduces_full_grid_centres(iz, iy0, ny):
    g = geometry.config2()
    full = _voxel_centres(g.image)
    sl = geometry.voxel_slab(g, iz, iy0, ny)
    sub = _voxel_centres(sl.image)
    n = sub.shape[1]
    assert np.array_equal(full[:, iy0:iy0 + n, iz], sub[:, :, 0])


# ---- C ABI -------------------------------------------------------------------------------

def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "sysmat.h")).read()
    declared = set(re.findall(r"SYSMAT_API\s+[\w\s\*]+?\b(\w+)\s*\(", hdr))
    assert declared == set(sysmat.EXPORTS)
    lib = sysmat.lib()
    for name in declared:
        assert hasattr(lib, name), name


def test_error_strings_and_version():
    lib = sysmat.lib()
    assert b"sm_100a" in lib.sysmat_version()
    for code in range(0, -7, -1):
        assert lib.sysmat_error_string(code)
    assert lib.sysmat_error_string(-99) == b"unknown error"


def _create(g):
    import ctypes
    h = ctypes.c_void_p()
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (g.collimator, g.detector, g.image, g.physics)]
    fp = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) for a in arrs]
    return sysmat.lib().sysmat_create(ctypes.byref(h), 0, *fp)


def test_create_rejects_bad_parameters_before_any_device_call():
    g = geometry.mini()
    d = g.detector.copy(); d[0] = 0
    assert _create(geometry.Geometry("x", g.collimator, d, g.image, g.physics)) == -3
    d = g.detector.copy(); d[0] = 7000            # beyond the 80000-float table
    assert _create(geometry.Geometry("x", g.collimator, d, g.image, g.physics)) == -3
    i = g.image.copy(); i[1] = 0
    assert _create(geometry.Geometry("x", g.collimator, g.detector, i, g.physics)) == -1
    d = g.detector.copy(); d[12 * 3 + 2] = np.nan
    assert _create(geometry.Geometry("x", g.collimator, d, g.image, g.physics)) == -1
    c = g.collimator.copy(); c[0] = 10            # the 10th layer header would hit the hole table
    assert _create(geometry.Geometry("x", c, g.detector, g.image, g.physics)) == -3


def test_reference_entry_points_reject_null_buffers():
    import ctypes
    lib = sysmat.lib()
    null = ctypes.POINTER(ctypes.c_float)()
    assert lib.PESysMatGen(null, null, null, null, 0) == -1
    assert lib.scatter(null, null, null, null, null, None, None, null, 0) == -1
    assert lib.scatter_crystal(null, null, null, null, None, null, 0) == -1


def test_native_entry_points_reject_a_null_context():
    """Every handle entry point answers SYSMAT_ERR_ARG for a null context or plan before any
    device call (no GPU here)."""
    import ctypes
    lib = sysmat.lib()
    div = (ctypes.c_int * 3)(4, 4, 4)
    sub = (ctypes.c_int * 3)(1, 1, 1)
    cnt = (ctypes.c_ulonglong * 12)()
    calls = {
        "sysmat_pe": lambda: lib.sysmat_pe(None, 0.0, 0, 1, 0, 1, None, 1, 0, None),
        "sysmat_pe_sampled": lambda: lib.sysmat_pe_sampled(None, 0.0, 0, 1, 0, 1, div, sub, None, 1, None),
        "sysmat_pe_work": lambda: lib.sysmat_pe_work(None, 0.0, 0, 1, 0, 1, None, 1, cnt, None),
        "sysmat_scatter": lambda: lib.sysmat_scatter(None, 3, 0, 0.0, None, 0, 1, 0, 1, None, 1, None),
        "sysmat_scatter_prepare": lambda: lib.sysmat_scatter_prepare(None, 3, None, None, None),
        "sysmat_scatter_prepare_native": lambda: lib.sysmat_scatter_prepare_native(None, 3, None, None),
        "sysmat_set_hole_shapes": lambda: lib.sysmat_set_hole_shapes(None, None, None, None),
        "sysmat_pe_csr_file": lambda: lib.sysmat_pe_csr_file(None, 0.0, b"x", 0.0, 0, 0, None, None),
        "sysmat_project": lambda: lib.sysmat_project(None, 0.0, 0, 1, None, None, None),
        "sysmat_backproject": lambda: lib.sysmat_backproject(None, 0.0, 0, 1, None, None, None),
        "sysmat_vjp": lambda: lib.sysmat_vjp(None, 0.0, 0, 1, None, None, None, None),
        "sysmat_batch_run": lambda: lib.sysmat_batch_run(None, 0, None),
    }
    for name, call in calls.items():
        assert call() == -1, name

def test_detector_slabs_cover_rows_once():
    for n, w in ((4096, 2), (4096, 8), (1023, 4), (3, 8)):
        rows = []
        for r in range(w):
            b, c = sharding.detector_slab(n, r, w)
            rows.extend(range(b, b + c))
        assert rows == list(range(n))


def test_plane_assignment_is_disjoint_within_a_step():
    for world in (1, 2, 4, 8):
        for step in range(3):
            planes = [sharding.plane_for_step(step, r, world, 32) for r in range(world)]
            assert len(set(planes)) == world


def test_planes_stay_in_the_image_for_long_runs():
    """A bench run of warm-up + timed steps longer than the image has planes (the 25 steps of
    a 5 + 20 run on 32 planes starting at plane 16, and longer) wraps around the image
    instead of running past its last plane."""
    for n_planes in (1, 16, 32):
        for first in (0, n_planes // 2, n_planes - 1):
            for world in (1, 2, 8):
                for step in range(64):
                    planes = [sharding.plane_for_step(step, r, world, n_planes, first)
                              for r in range(world)]
                    assert all(0 <= p < n_planes for p in planes)
                    if world <= n_planes:
                        assert len(set(planes)) == world
    # consecutive steps of one rank walk the image from `first`
    assert [sharding.plane_for_step(s, 0, 1, 32, 16) for s in range(18)] == \
        list(range(16, 32)) + [0, 1]


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # each rank "computes" its planes and the job reduces the step time as a max
    planes = torch.tensor([sharding.plane_for_step(s, rank, world, 32) for s in range(4)])
    gathered = [torch.zeros_like(planes) for _ in range(world)]
    dist.all_gather(gathered, planes)
    t = torch.tensor([0.5 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        q.put((torch.stack(gathered).tolist(), float(t)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_partition_and_max_timing():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    gathered, tmax = q.get()
    flat = [p for step in zip(*gathered) for p in step]
    assert len(flat) == len(set(flat)) == 8           # 2 ranks x 4 steps, all distinct
    assert tmax == 1.5
