"""VDB export: the library's OpenVDB writer (lbm_vdb_write_vec3 /
lbm_vdb_export) read back by the independent format reader in oracle/.

The reference writes vdb_export/velocity_%06u.vdb through OpenVDB
(src/main.cpp:1767-1790 -> common/common-cpp/src/vdb_writer.cpp:96-141): a
Vec3SGrid "velocity", class staggered, voxel size 1, every voxel of the box
set (active), values = half_to_float of the rgba16f velocity.  OpenVDB is not
installed here, so the file is checked against a restatement of the format:
values bit-exact, every box voxel active and nothing else, the stored stream
offsets equal to where the reader finds each section."""

import numpy as np
import pytest

from oracle import vdb_oracle


def _roundtrip(lbm, tmp_path, shape, seed, **kw):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    xyz = rng.standard_normal((nx * ny * nz, 3)).astype(np.float32)
    xyz[rng.random(nx * ny * nz) < 0.1] = 0.0  # zeros stay active voxels
    path = tmp_path / "g.vdb"
    lbm.vdb_write_vec3(str(path), xyz, shape, **kw)
    f = vdb_oracle.read(str(path))
    return xyz, f


def _check_structure(f, shape, name="velocity"):
    assert f["file_version"] == 224 and f["has_grid_offsets"] == 1
    assert len(f["uuid"]) == 36 and f["uuid"][14] == "4"
    assert f["file_meta"] == {} and len(f["grids"]) == 1 and f["trailing_bytes"] == 0
    g = f["grids"][0]
    assert g["name"] == name and g["type"] == "Tree_vec3s_5_4_3" and g["parent"] == ""
    assert g["meta"]["class"] == "staggered" and g["meta"]["name"] == name
    nx, ny, nz = shape
    assert g["meta"]["file_bbox_min"] == (0, 0, 0)
    assert g["meta"]["file_bbox_max"] == (nx - 1, ny - 1, nz - 1)
    assert g["meta"]["file_voxel_count"] == nx * ny * nz
    assert g["stored_pos"] == (g["grid_pos_found"], g["block_pos_found"], g["end_pos_found"])
    assert g["tiles"] == []
    assert g["active_voxels"] == nx * ny * nz
    assert g["bbox"] == ((0, 0, 0), (nx - 1, ny - 1, nz - 1))
    assert len(g["leaves"]) == -(-nx // 8) * -(-ny // 8) * -(-nz // 8)
    return g


@pytest.mark.parametrize("shape", [(13, 9, 21), (8, 8, 8), (130, 7, 9), (1, 1, 1)])
def test_vec3_grid_roundtrip(lbm_lib, tmp_path, shape):
    xyz, f = _roundtrip(lbm_lib, tmp_path, shape, seed=sum(shape))
    g = _check_structure(f, shape)
    vals, act = vdb_oracle.dense(g, shape)
    assert act.all()
    assert np.array_equal(vals.view(np.uint32), xyz.view(np.uint32))
    t = g["transform"]
    assert t["map"] == "UniformScaleMap" and t["scale"] == (1.0, 1.0, 1.0)
    assert t["voxel_size"] == (1.0, 1.0, 1.0) and t["inv_twice_scale"] == (0.5, 0.5, 0.5)
    # inactive voxels of partial leaves hold the background
    for org, m, v in g["leaves"]:
        assert np.all(v[~m] == 0.0)


def test_two_root_children_in_order(lbm_lib, tmp_path):
    """A box wider than one 4096-voxel root child: two root children, in
    ascending x, each with its own internal nodes."""
    shape = (4100, 2, 3)
    xyz, f = _roundtrip(lbm_lib, tmp_path, shape, seed=5)
    g = _check_structure(f, shape)
    vals, act = vdb_oracle.dense(g, shape)
    assert act.all() and np.array_equal(vals, xyz)
    origins = [o for o, _, _ in g["leaves"]]
    assert origins == sorted(origins)  # x slowest at every level for this box
    assert origins[-1] == (4096, 0, 0)


def test_scale_and_translation(lbm_lib, tmp_path):
    shape = (9, 10, 11)
    xyz, f = _roundtrip(lbm_lib, tmp_path, shape, seed=9, voxel_size=0.5, origin=(1.0, -2.0, 0.25),
                        grid_name="u")
    g = _check_structure(f, shape, name="u")
    t = g["transform"]
    assert t["map"] == "UniformScaleTranslateMap"
    assert t["translation"] == (1.0, -2.0, 0.25)
    assert t["scale"] == (0.5, 0.5, 0.5) and t["scale_inverse"] == (2.0, 2.0, 2.0)
    assert t["inv_scale_sqr"] == (4.0, 4.0, 4.0) and t["inv_twice_scale"] == (1.0, 1.0, 1.0)
    vals, act = vdb_oracle.dense(g, shape)
    assert np.array_equal(vals, xyz)


def test_writer_errors(lbm_lib, tmp_path):
    lib = lbm_lib.load()
    xyz = np.zeros((8, 3), np.float32)
    assert lib.lbm_vdb_write_vec3(None, xyz.ctypes.data, 2, 2, 2, 1.0, None, None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_vdb_write_vec3(str(tmp_path / "a.vdb").encode(), xyz.ctypes.data, 0, 2, 2, 1.0, None,
                                  None) == lbm_lib.ERR_INVALID_ARG
    assert lib.lbm_vdb_write_vec3(str(tmp_path / "a.vdb").encode(), xyz.ctypes.data, 2, 2, 2, 0.0, None,
                                  None) == lbm_lib.ERR_INVALID_ARG
    rc = lib.lbm_vdb_write_vec3(str(tmp_path / "no" / "such" / "dir.vdb").encode(), xyz.ctypes.data,
                                2, 2, 2, 1.0, None, None)
    assert rc == lbm_lib.ERR_IO and b"cannot open" in lib.lbm_vdb_last_error()
    assert lib.lbm_vdb_export(None, b"x", 0, 0) == lbm_lib.ERR_INVALID_ARG


def test_reader_rejects_a_corrupt_file(lbm_lib, tmp_path):
    """The checker is not vacuous: a flipped leaf mask bit and a truncated
    file are both caught."""
    shape = (8, 8, 8)
    xyz, f = _roundtrip(lbm_lib, tmp_path, shape, seed=1)
    g = f["grids"][0]
    data = bytearray((tmp_path / "g.vdb").read_bytes())
    bad = bytearray(data)
    bad[g["block_pos_found"]] ^= 1  # first bit of the first leaf's buffer mask
    (tmp_path / "bad.vdb").write_bytes(bytes(bad))
    with pytest.raises(ValueError, match="mask differs"):
        vdb_oracle.read(str(tmp_path / "bad.vdb"))
    (tmp_path / "short.vdb").write_bytes(bytes(data[:-5]))
    with pytest.raises(ValueError, match="truncated"):
        vdb_oracle.read(str(tmp_path / "short.vdb"))


@pytest.mark.gpu
@pytest.mark.parametrize("f32", [False, True])
def test_lattice_export(gpu, tmp_path, f32):
    """lbm_vdb_export after a few steps of the reference preset: the file holds
    half_to_float of the rgba16f velocity (the reference's VDB payload), or
    with LBM_VDB_F32 the fp32 velocity, named velocity_<frame:06d>.vdb."""
    shape = (40, 24, 10)
    lat = gpu.Lattice(gpu.preset_desc(0, *shape))
    gpu.apply_preset(lat, 0)
    lat.step(30)
    path = lat.vdb_export(str(tmp_path), 42, f32=f32)
    assert path.endswith("velocity_000042.vdb")
    f = vdb_oracle.read(path)
    g = _check_structure(f, shape)
    vals, act = vdb_oracle.dense(g, shape)
    if f32:
        want = lat.read_moments(gpu.U_F32X3)[1]
    else:
        h = lat.read_moments(gpu.U_F16X4)[1]
        want = gpu.half_to_float(np.ascontiguousarray(h[:, :3]).reshape(-1)).reshape(-1, 3)
    assert act.all()
    assert np.array_equal(vals.view(np.uint32), want.view(np.uint32))
    lat.close()
