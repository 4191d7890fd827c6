"""Binary mesh export (rq_mesh_save_binary / Mesh.save_binary): the product writes the
reference's MSH2 file (Mesh::saveBinary, core/src/Mesh.cpp:751-811) byte for byte, so
the reference's loadBinary and tools read the meshes the GPU path solved on. Pinned by
the SHA-256 of the reference's own files (tests/golden/mesh_binary_sha256.json, written
by tests/golden/make_golden.py), and directly against oracle/_ref where it is built.
Host code only: no GPU needed."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle import checker as ck

DIGESTS = json.loads((Path(__file__).parent / "golden" / "mesh_binary_sha256.json").read_text())


@pytest.mark.parametrize("name", sorted(cases.MESH_BINARY_CASES))
def test_binary_mesh_matches_reference_file(rq, tmp_path, name):
    case = cases.MESH_BINARY_CASES[name]
    path = tmp_path / "mesh.bin"
    cases.product_mesh(rq, case).save_binary(path)
    data = path.read_bytes()
    assert len(data) == DIGESTS[name]["bytes"]
    assert hashlib.sha256(data).hexdigest() == DIGESTS[name]["sha256"]
    if ck.have("ref") and name in ("channel_3x24", "bump_24x16"):
        ref = tmp_path / "ref.bin"
        ck.mesh_save_binary(case, ref)
        assert ref.read_bytes() == data


def test_binary_mesh_unwritable_path_fails(rq, tmp_path):
    mesh = cases.product_mesh(rq, cases.MESH_BINARY_CASES["channel_3x24"])
    with pytest.raises(Exception, match="Cannot open binary mesh"):
        mesh.save_binary(tmp_path / "missing-dir" / "mesh.bin")


@pytest.mark.parametrize("name", ["channel_3x24", "bump_24x16"])
def test_mesh_introspection_matches_reference_mesh(rq, checker, name):
    """Mesh.n_faces / cell_centers / cell_volumes / face_centers / wall_patch_data as the
    reference binding returns them (bindings.cpp:128-246), against the checker's mesh
    (bitwise equal to the reference's, tests/test_oracle_pins.py)."""
    case = cases.MESH_BINARY_CASES[name]
    mesh = cases.product_mesh(rq, case)
    cells, faces, ni = ck.mesh(case, "oracle")
    assert mesh.n_cells() == len(cells) and mesh.n_faces() == len(faces)
    assert mesh.n_internal_faces() == ni and mesh.n_patches() == 2
    assert mesh.patch_types() == ["wall", "wall"]
    cc = mesh.cell_centers()
    np.testing.assert_array_equal(cc[:, :2], cells[:, :2])
    np.testing.assert_array_equal(cc[:, 2], 0.5)
    np.testing.assert_array_equal(mesh.cell_volumes(), cells[:, 2])
    np.testing.assert_array_equal(mesh.face_centers()[:, :2], faces[:, 2:4])
    assert mesh.node_coords().shape == (2 * (case.nx + 1) * (case.ny + 1), 3)
    top = mesh.wall_patch_data(mesh.patch_names()[1])
    wall = faces[ni + case.nx:]
    np.testing.assert_array_equal(top["owner"], wall[:, 0].astype(int))
    np.testing.assert_array_equal(top["delta"], wall[:, 7])
    np.testing.assert_array_equal(top["area"], wall[:, 6])
    np.testing.assert_array_equal(top["normal"][:, :2], wall[:, 4:6])
    with pytest.raises(RuntimeError, match="unknown patch"):
        mesh.wall_patch_data("inlet")
