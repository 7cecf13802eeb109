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


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_fp32_host_grids_match_their_fp64_values(precision, fields32):
    """hxg_upload_grid_f32 widens FP32 host grids on the device: the slots
    and the maps equal those of hxg_upload_grid given the same values as
    FP64 (bit for bit), in both forms."""
    n = 32
    desc = W.grid_desc(n)
    b32 = [np.asarray(a, dtype=np.float32).reshape(-1) for a in fields32[:3]]
    t32 = [np.asarray(fields32[3], dtype=np.float32).reshape(-1)]
    o = W.make_obs([8, 16, 32], 20.0, 0.05, freq_ghz=1.4)
    with I.Integrator(precision) as a, I.Integrator(precision) as f:
        for ig, conv in ((a, lambda v: [x.astype(np.float64) for x in v]), (f, lambda v: v)):
            ig.set_models(W.grid_models())
            ig.upload_grid(abi.HXG_FIELD_BRND, desc, conv(b32))
            ig.upload_grid(abi.HXG_FIELD_TEREG, desc, conv(t32))
        for field in (abi.HXG_FIELD_BRND, abi.HXG_FIELD_TEREG):
            for x, y in zip(a.download_grid(field, desc), f.download_grid(field, desc)):
                np.testing.assert_array_equal(x, y)
        ma, mf = a.write_grid(o), f.write_grid(o)
        for k in ("dm", "fd", "is", "qs", "us"):
            assert np.abs(ma[k]).max() > 0, k
            np.testing.assert_array_equal(ma[k], mf[k])


def test_fp32_host_grid_in_several_chunks():
    # 420^3 = 74.1 M values: one full 2^26-value chunk and a partial one
    n = 420
    desc = W.grid_desc(n)
    rng = np.random.Generator(np.random.PCG64(9))
    t32 = rng.random(n ** 3, dtype=np.float32)
    m = W.grid_models()
    m.brnd = abi.HXG_BRND_NONE
    with I.Integrator("fp32c") as f:
        f.set_models(m)
        f.upload_grid(abi.HXG_FIELD_TEREG, desc, [t32])
        (got,) = f.download_grid(abi.HXG_FIELD_TEREG, desc)
    np.testing.assert_array_equal(got.reshape(-1), t32.astype(np.float64))
