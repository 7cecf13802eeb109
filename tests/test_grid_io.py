"""hxg_upload_grid_file: grids loaded straight from the reference's binary
grid files (Grid_*::import_grid, source/grid/grid_breg.cc:48-66; B slots with
(bx, by, bz) interleaved per voxel, CRE grid with the energy fastest) hold
exactly the values an upload of the same arrays holds."""
import numpy as np
import pytest

from hammurabix_b200 import _lib, abi, units as U, workloads as W
from hammurabix_b200 import integrator as I

pytestmark = pytest.mark.gpu


def _positions(n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    p = rng.uniform(-1, 1, size=(n, 3)) * np.array([21., 21., 5.5]) * U.kpc
    return p.reshape(-1)


def test_grid_files_load_the_same_values(tmp_path):
    nx, ny, nz = 40, 36, 20          # 28 800 voxels: one partial chunk
    desc = W.grid_desc(nx)
    desc.ny, desc.nz = ny, nz
    rng = np.random.Generator(np.random.PCG64(3))
    b = [rng.standard_normal(nx * ny * nz) * U.muGauss for _ in range(3)]
    ne = rng.random(nx * ny * nz) * 0.05
    bfile, tfile = tmp_path / "brnd.bin", tmp_path / "tereg.bin"
    np.stack(b, axis=1).astype("<f8").tofile(bfile)
    ne.astype("<f8").tofile(tfile)
    pos = _positions(4000, 4)
    with I.Integrator("fp64") as a, I.Integrator("fp64") as f:
        a.set_models(W.grid_models())
        f.set_models(W.grid_models())
        a.upload_grid(abi.HXG_FIELD_BRND, desc, b)
        a.upload_grid(abi.HXG_FIELD_TEREG, desc, [ne])
        f.upload_grid_file(abi.HXG_FIELD_BRND, desc, str(bfile))
        f.upload_grid_file(abi.HXG_FIELD_TEREG, desc, str(tfile))
        for field in (abi.HXG_FIELD_BRND, abi.HXG_FIELD_TEREG):
            np.testing.assert_array_equal(a.read_grid(field, pos), f.read_grid(field, pos))


def test_multi_chunk_vector_grid(tmp_path):
    # 160^3 voxels x 3 components = 12.3 M doubles: four 3 * 2^20 chunks plus
    # a partial one, through both pinned buffers
    n = 160
    desc = W.grid_desc(n)
    rng = np.random.Generator(np.random.PCG64(5))
    b = [rng.standard_normal(n ** 3) for _ in range(3)]
    path = tmp_path / "b.bin"
    np.stack(b, axis=1).astype("<f8").tofile(path)
    pos = _positions(20000, 6)
    m = W.grid_models()
    m.tereg = abi.HXG_TEREG_NONE     # this case uploads the B grid only
    with I.Integrator("fp64") as a, I.Integrator("fp64") as f:
        a.set_models(m)
        f.set_models(m)
        a.upload_grid(abi.HXG_FIELD_BRND, desc, b)
        f.upload_grid_file(abi.HXG_FIELD_BRND, desc, str(path))
        np.testing.assert_array_equal(a.read_grid(abi.HXG_FIELD_BRND, pos),
                                      f.read_grid(abi.HXG_FIELD_BRND, pos))


def test_bad_files_are_rejected(tmp_path):
    desc = W.grid_desc(8)
    short = tmp_path / "short.bin"
    np.zeros(8 ** 3 * 3 - 1).tofile(short)
    with I.Integrator("fp64") as f:
        for path in (short, tmp_path / "missing.bin"):
            with pytest.raises(_lib.HxgError) as e:
                f.upload_grid_file(abi.HXG_FIELD_BRND, desc, str(path))
            assert e.value.status == abi.HXG_ERR_INVALID
