"""Binary mesh export (rq_mesh_save_binary / Mesh.save_binary): the product writes the
reference's MSH2 file (Mesh::saveBinary, core/src/Mesh.cpp:751-811) byte for byte, so
the reference's loadBinary and tools read the meshes the GPU path solved on. Pinned by
the SHA-256 of the reference's own files (tests/golden/mesh_binary_sha256.json, written
by tests/golden/make_golden.py), and directly against oracle/_ref where it is built.
Host code only: no GPU needed."""
import hashlib
import json
from pathlib import Path

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
