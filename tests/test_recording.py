"""Recordings in the reference's ViewerFile layout: structure of the file, and a model + state
history that round-trips through save / load (CPU)."""

import json

import numpy as np
import pytest
import torch

from newton_b200 import Model, scenes
from newton_b200.recording import RecorderFile


def _scene():
    return scenes.single_cloth(n=8, side=0.5, seed=2, sphere=((0.0, 0.0, -0.5), 0.3), device="cpu")


def test_file_layout_matches_the_viewerfile_container(tmp_path):
    model, q0 = _scene()
    rec = RecorderFile(str(tmp_path / "cloth.json"), auto_save=False)
    rec.set_model(model)
    s = model.state()
    rec.log_state(s)
    rec.save_recording()
    data = json.load(open(tmp_path / "cloth.json"))
    assert data["__type__"] == "dict" and set(data["items"]) == {"model", "states"}
    m = data["items"]["model"]
    assert m["__type__"] == "Model" and "attributes" in m
    pq = m["attributes"]["particle_q"]
    assert pq["__type__"] == "warp.array" and pq["__dtype__"] == "<class 'warp.types.vec3f'>"
    assert pq["__scalar_type__"] == "float32" and pq["__type_length__"] == 3
    payload = pq["data"]
    assert payload["__type__"] == "numpy.ndarray" and payload["shape"] == [model.particle_count, 3]
    assert np.allclose(np.array(json.loads(payload["data"]), np.float32), model.particle_q)
    assert m["attributes"]["tri_poses"]["__dtype__"] == "<class 'warp.types.mat22f'>"
    assert m["attributes"]["tri_poses"]["__type_shape__"] == [2, 2]
    assert m["attributes"]["shape_transform"]["__dtype__"] == "<class 'warp.types.transformf'>"
    assert m["attributes"]["particle_count"] == {"__type__": "int", "value": model.particle_count}
    st = data["items"]["states"]
    assert st["__type__"] == "list" and len(st["items"]) == 1
    assert set(st["items"][0]["items"]) == {"particle_q", "particle_qd", "particle_f"}
    idx = [pq["cache_index"]] + [v["cache_index"] for v in st["items"][0]["items"].values()]
    assert len(set(idx)) == len(idx)


@pytest.mark.parametrize("ext", [".json", ".bin"])
def test_round_trip_model_and_states(tmp_path, ext):
    if ext == ".bin":
        pytest.importorskip("cbor2")
    model, q0 = _scene()
    rec = RecorderFile(str(tmp_path / ("run" + ext)), auto_save=False)
    rec.set_model(model)
    s = model.state()
    frames = []
    rng = np.random.default_rng(0)
    for k in range(4):
        s.particle_q.copy_(torch.from_numpy(q0 + rng.normal(scale=1e-3, size=q0.shape).astype(np.float32)))
        s.particle_qd.fill_(0.1 * k)
        rec.log_state(s)
        frames.append(s.particle_q.clone())
    rec.save_recording()

    back = RecorderFile(str(tmp_path / ("run" + ext)))
    back.load_recording()
    assert back.get_frame_count() == 4 and back.has_model()
    m2 = Model("cpu")
    back.load_model(m2)
    for name in ("particle_q", "particle_mass", "particle_flags", "tri_indices", "tri_poses", "tri_materials",
                 "edge_indices", "edge_rest_angle", "shape_transform", "shape_type", "gravity"):
        np.testing.assert_array_equal(np.asarray(getattr(m2, name)), np.asarray(getattr(model, name)), err_msg=name)
    assert m2.particle_count == model.particle_count and m2.shape_count == model.shape_count
    assert [g.tolist() for g in m2.particle_color_groups] == [np.asarray(g).tolist() for g in model.particle_color_groups]
    np.testing.assert_array_equal(m2.soft_mesh_adjacency.v_adj_tris, model.soft_mesh_adjacency.v_adj_tris)
    s2 = m2.state()
    for k in range(4):
        back.load_state(s2, k)
        assert torch.equal(s2.particle_q, frames[k])
        assert torch.allclose(s2.particle_qd, torch.full_like(s2.particle_qd, 0.1 * k))
    with pytest.raises(IndexError):
        back.load_state(s2, 4)


def test_binary_file_holds_the_arrays_as_cbor_byte_strings(tmp_path):
    """.bin: the same containers, each array's payload its C-order bytes with the numpy dtype
    string (serialize_ndarray's cbor2 branch, viewer_file.py:299-312)."""
    cbor2 = pytest.importorskip("cbor2")
    model, q0 = _scene()
    rec = RecorderFile(str(tmp_path / "cloth.bin"), auto_save=False)
    rec.set_model(model)
    rec.log_state(model.state())
    rec.save_recording()
    data = cbor2.loads((tmp_path / "cloth.bin").read_bytes())
    pq = data["items"]["model"]["attributes"]["particle_q"]
    assert pq["__type__"] == "warp.array" and pq["__dtype__"] == "<class 'warp.types.vec3f'>"
    payload = pq["data"]
    assert payload["__type__"] == "numpy.ndarray" and payload["dtype"] == "<f4" and payload["order"] == "C"
    assert list(payload["shape"]) == [model.particle_count, 3]
    got = np.frombuffer(payload["binary_data"], dtype=np.float32).reshape(model.particle_count, 3)
    np.testing.assert_array_equal(got, model.particle_q)


def test_binary_format_needs_cbor2(tmp_path):
    rec = RecorderFile(str(tmp_path / "x.bin"), auto_save=False)
    try:
        import cbor2  # noqa: F401
    except ImportError:
        with pytest.raises(ImportError):
            rec.save_recording()
    with pytest.raises(ValueError):
        RecorderFile(str(tmp_path / "x.txt"), auto_save=False).save_recording()
