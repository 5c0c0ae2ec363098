"""PLY output (mojo_poissonrecon_b200/ply.py): round trips through write_ply
and read_ply in both encodings, the header upstream tools read, and argument
checks.  Host code only."""

import numpy as np
import pytest

from mojo_poissonrecon_b200 import Mesh, read_ply, write_ply


def _mesh(nv=40, nf=60, seed=0):
    rng = np.random.default_rng(seed)
    return Mesh(rng.normal(size=(nv, 3)), rng.integers(0, nv, size=(nf, 3)).astype(np.int64),
                rng.random(nv) * 5.0, 0.123456789)


@pytest.mark.parametrize("binary", [True, False])
@pytest.mark.parametrize("coordinates", ["float", "double"])
def test_round_trip(tmp_path, binary, coordinates):
    mesh = _mesh()
    path = tmp_path / "m.ply"
    write_ply(path, mesh, binary=binary, coordinates=coordinates)
    back = read_ply(path)
    cast = np.float32 if coordinates == "float" else np.float64
    assert np.array_equal(back["vertices"], mesh.vertices.astype(cast).astype(np.float64))
    assert np.array_equal(back["properties"]["value"], mesh.density.astype(cast).astype(np.float64))
    assert np.array_equal(back["faces"], mesh.faces)
    assert any(c.startswith("iso_value 0.123456789") for c in back["comments"])


@pytest.mark.parametrize("binary", [True, False])
def test_vertex_properties(tmp_path, binary):
    """Per-vertex colours (uint8) and a float32 scalar round-trip in their own
    types, after the density."""
    mesh = _mesh(30, 20, seed=3)
    rng = np.random.default_rng(4)
    colours = {c: rng.integers(0, 256, 30).astype(np.uint8) for c in ("red", "green", "blue")}
    quality = rng.random(30).astype(np.float32)
    path = tmp_path / "c.ply"
    write_ply(path, mesh, binary=binary, properties={**colours, "quality": quality})
    head = path.read_bytes().split(b"end_header")[0].decode()
    assert "property uchar red" in head and "property float quality" in head
    assert head.index("property float value") < head.index("property uchar red")
    back = read_ply(path)
    for c, v in colours.items():
        assert back["properties"][c].dtype == np.uint8 and np.array_equal(back["properties"][c], v)
    assert np.array_equal(back["properties"]["quality"], quality)
    assert np.array_equal(back["faces"], mesh.faces)


def test_vertex_properties_rejected(tmp_path):
    mesh = _mesh(5, 3)
    for bad in ({"red": np.zeros(4, np.uint8)}, {"x": np.zeros(5)}, {"bad name": np.zeros(5)},
                {"flag": np.zeros(5, bool)}):
        with pytest.raises(ValueError):
            write_ply(tmp_path / "m.ply", mesh, properties=bad)


def test_header_and_sizes(tmp_path):
    mesh = _mesh(5, 4)
    path = tmp_path / "m.ply"
    write_ply(path, mesh)
    data = path.read_bytes()
    head = data[:data.index(b"end_header\n") + len(b"end_header\n")].decode()
    assert head.splitlines()[:2] == ["ply", "format binary_little_endian 1.0"]
    for line in ("element vertex 5", "property float x", "property float value", "element face 4",
                 "property list uchar int vertex_indices"):
        assert line in head.splitlines()
    assert len(data) == len(head) + 5 * 4 * 4 + 4 * (1 + 3 * 4)


def test_without_density_and_empty(tmp_path):
    path = tmp_path / "m.ply"
    write_ply(path, _mesh(), density=False)
    assert read_ply(path)["properties"] == {}
    empty = Mesh(np.empty((0, 3)), np.empty((0, 3), np.int64), np.empty(0), 0.0)
    for binary in (True, False):
        write_ply(path, empty, binary=binary)
        back = read_ply(path)
        assert back["vertices"].shape == (0, 3) and back["faces"].shape == (0, 3)


def test_rejects_bad_meshes(tmp_path):
    mesh = _mesh(4, 2)
    bad = Mesh(mesh.vertices, np.array([[0, 1, 4]]), mesh.density, 0.0)
    with pytest.raises(ValueError):
        write_ply(tmp_path / "m.ply", bad)
    with pytest.raises(ValueError):
        write_ply(tmp_path / "m.ply", Mesh(mesh.vertices, mesh.faces, mesh.density[:2], 0.0))
    with pytest.raises(ValueError):
        write_ply(tmp_path / "m.ply", mesh, coordinates="half")


def test_reconstructed_mesh_round_trip(tmp_path):
    """A mesh from the oracle's restatement of the reference pipeline (CPU)."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    import pipeline

    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere(2000, seed=0)
    mesh = pipeline.reconstruct(pts, nrm, depth=4)
    path = tmp_path / "sphere.ply"
    write_ply(path, mesh, coordinates="double")
    back = read_ply(path)
    assert np.array_equal(back["vertices"], mesh.vertices)
    assert np.array_equal(back["faces"], mesh.faces)


@pytest.mark.gpu
def test_device_mesh(tmp_path):
    """A mesh left on the device (device_out=True) writes the same file as its
    host copy."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    pts, nrm = workloads.sphere(5000, seed=1)
    dev = mpr.reconstruct(pts, nrm, depth=5, precision="fp32_refined", tol=1e-8, device_out=True)
    host = mpr.reconstruct(pts, nrm, depth=5, precision="fp32_refined", tol=1e-8)
    assert dev.vertices.is_cuda
    write_ply(tmp_path / "d.ply", dev)
    write_ply(tmp_path / "h.ply", host)
    assert (tmp_path / "d.ply").read_bytes() == (tmp_path / "h.ply").read_bytes()
    back = read_ply(tmp_path / "d.ply")
    assert np.array_equal(back["faces"], host.faces)
