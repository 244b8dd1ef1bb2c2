"""GPU tests of the grid scatter model (sysmat_scatter_grid), through the C ABI, against its
definition restated in FP64 (oracle.scatter_grid, oracle/oracle_grid.h).

The model has no reference counterpart: scatter points on a 0.25 mm grid inside every crystal
and inside the collimator's tungsten, FP64 sums per element.  The device evaluates each item in
FP32 with the weights and the detector-only terms formed in double or in the local-coordinate
FP32 form; its elements must stay within 1e-5 of the FP64 definition."""
import numpy as np
import pytest

from conftest import TOL, geometry, oracle, rel_err, sysmat

pytestmark = pytest.mark.gpu


def _grid(torch, geo, parts, cell=0.25, rotation=0.0, shapes=None, **blk):
    ctx = sysmat.Context(geo)
    if shapes is not None:
        ctx.set_hole_shapes(shapes)
    nd = blk.get("det_count", ctx.n_det)
    nv = blk.get("vox_count", ctx.n_vox)
    out = torch.full((nd, nv), -1.0, dtype=torch.float32, device="cuda")
    ctx.scatter_grid(out, parts=parts, cell=cell, rotation=rotation, **blk)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("parts", [1, 2, 3])
def test_grid_scatter_matches_fp64_definition(gpu, parts):
    geo = geometry.mini(seed=3, nvox=(3, 3, 1), ncry=(3, 3), nholes=3)
    a = _grid(gpu, geo, parts)
    o = oracle.scatter_grid(geo, parts=parts, cell=0.25)
    assert o.max() > 0
    r = rel_err(a, o)
    assert r.max() <= TOL, (parts, r.max(), np.median(r))


def test_grid_scatter_rotated_crystals_two_layers(gpu):
    geo = geometry.mini(seed=7, rotated=True, layers=2, n_rot=4, nvox=(3, 2, 2), ncry=(3, 3), nholes=3)
    geo = geo.with_rotation(1)
    a = _grid(gpu, geo, 3, rotation=1.0)
    o = oracle.scatter_grid(geo, parts=3, cell=0.25)
    r = rel_err(a, o)
    assert o.max() > 0 and r.max() <= TOL, (r.max(), np.median(r))


def test_grid_scatter_blocks_match_the_full_matrix(gpu):
    geo = geometry.mini(seed=3, nvox=(3, 3, 1), ncry=(3, 3), nholes=3)
    full = _grid(gpu, geo, 3)
    blk = _grid(gpu, geo, 3, det_begin=2, det_count=5, vox_begin=3, vox_count=4)
    # FP64 sums taken in another order: equal to the float output's rounding
    assert rel_err(blk, full[2:7, 3:7]).max() < 1e-6


def test_grid_scatter_config3_element(gpu):
    """Configuration 3 at full size (1024 crystals of 8 x 24 x 8 cells, 64 x 64 x 10 mm plate of
    256 x 40 x 256 cells): one crystal x two voxels of z-plane 8 against the FP64 definition."""
    geo = geometry.voxel_slab(geometry.config3(), 8, 24, 1)
    a = _grid(gpu, geo, 3, det_begin=528, det_count=1, vox_begin=22, vox_count=2)
    o = oracle.scatter_grid(geo, parts=3, cell=0.25, dets=[528], v0=22, nv=2)
    r = rel_err(a, o)
    assert o.min() > 0 and r.max() <= TOL, (a, o, r)


def test_grid_scatter_rejects_unequal_crystal_divisions(gpu):
    torch = gpu
    geo = geometry.mini(seed=3, nvox=(3, 3, 1), ncry=(3, 3), nholes=3)
    det = geo.detector.copy()
    det[12 * 1 + 4] = np.float32(det[12 * 1 + 4] * 1.5)             # crystal 1 wider: another division
    g2 = geometry.Geometry("unequal", geo.collimator, det, geo.image, geo.physics)
    ctx = sysmat.Context(g2)
    out = torch.empty((ctx.n_det, ctx.n_vox), dtype=torch.float32, device="cuda")
    with pytest.raises(sysmat.SysmatError):
        ctx.scatter_grid(out)


@pytest.mark.parametrize("parts", [1, 2, 3])
def test_grid_scatter_with_elliptical_holes(gpu, parts):
    """Elliptical holes (two thirds of them, seeded semi-axes and angles): septal cells outside
    the ellipses, exact segment overlaps with the elliptical cylinders, crystal-cell weights from
    the local form with its elliptical extents; against the FP64 definition with the same
    shapes, and different from the circular system."""
    geo = geometry.mini(seed=3, nvox=(3, 3, 1), ncry=(3, 3), nholes=3)
    H = geo.n_holes
    rng = np.random.default_rng(8)
    r = geo.collimator[100:100 + 9 * H].reshape(H, 9)[:, 4].astype(np.float64)
    shapes = np.stack([r * rng.uniform(0.5, 1.0, H), r * rng.uniform(0.4, 0.9, H),
                       rng.uniform(0.0, np.pi, H)], 1).astype(np.float32)
    shapes[::3, 0] = 0.0                                 # every third hole circular
    a = _grid(gpu, geo, parts, shapes=shapes)
    o = oracle.scatter_grid(geo, parts=parts, cell=0.25, shapes=shapes)
    r = rel_err(a, o)
    assert o.max() > 0 and r.max() <= TOL, (parts, r.max(), np.median(r))
    assert rel_err(oracle.scatter_grid(geo, parts=parts, cell=0.25), o).max() > 1e-3
