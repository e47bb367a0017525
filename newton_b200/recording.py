"""Recording of cloth simulations in the reference's ``ViewerFile`` format (headless).

``RecorderFile`` keeps the API of ``newton.viewer.ViewerFile`` (``newton/_src/viewer/viewer_file.py
:1100-1511``) that a recording needs -- ``set_model``, ``log_state`` / ``record``, ``end_frame``,
``save_recording``, ``load_recording``, ``get_frame_count``, ``has_model``, ``load_model``,
``load_state``, ``close`` -- and writes the same file layout, so recordings move between this
package and Newton pipelines:

* the file is the serialisation of ``{"model": Model, "states": [ {name: array, ...}, ... ]}``
  (``_save_to_file``, :1263-1285): every container is ``{"__type__": <name>, "items": ...}``,
  every object ``{"__type__": <class>, "__module__": ..., "attributes": {...}}``, every scalar
  ``{"__type__": "int" | "float" | ..., "value": ...}`` (``serialize``, :402-490);
* every device array is a ``"warp.array"`` entry: ``__dtype__`` is the Warp class string of the
  element type (``"<class 'warp.types.vec3f'>"`` ...) with the vector/matrix metadata the
  reference's resolver reads (``_serialize_warp_dtype`` :497-536, ``_resolve_warp_dtype``
  :881-972), a ``cache_index``, and the payload as a ``"numpy.ndarray"`` entry whose ``data``
  is the JSON text of the nested list (``serialize_ndarray`` :281-346).

``.json`` and ``.bin`` are written and read; ``.bin`` is the same tree in CBOR with every
array's payload as its C-order bytes (the ``cbor2`` branch of ``serialize_ndarray``, :299-312)
and needs the ``cbor2`` package, as in the reference.  The model part holds the cloth fields (particles, triangles, hinges, static shapes,
colors, contact material, gravity); a Newton ``ViewerFile`` loads it field by field into a
``Model`` (its transfer is source-driven), and ``load_model`` here restores a ``Model`` of this
package (adjacency and colors rebuilt).
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np
import torch

from .mesh import MeshAdjacency
from .model import Model, State

# (attribute, warp element type, scalar type, vector length or None, matrix shape or None)
_MODEL_ARRAYS = [
    ("particle_q", "vec3f", "float32", 3, None),
    ("particle_qd", "vec3f", "float32", 3, None),
    ("particle_mass", "float32", "float32", None, None),
    ("particle_inv_mass", "float32", "float32", None, None),
    ("particle_radius", "float32", "float32", None, None),
    ("particle_flags", "int32", "int32", None, None),
    ("particle_world", "int32", "int32", None, None),
    ("tri_indices", "int32", "int32", None, None),
    ("tri_poses", "mat22f", "float32", 4, (2, 2)),
    ("tri_materials", "float32", "float32", None, None),
    ("tri_areas", "float32", "float32", None, None),
    ("edge_indices", "int32", "int32", None, None),
    ("edge_rest_angle", "float32", "float32", None, None),
    ("edge_rest_length", "float32", "float32", None, None),
    ("edge_bending_properties", "float32", "float32", None, None),
    ("shape_type", "int32", "int32", None, None),
    ("shape_transform", "transformf", "float32", 7, None),
    ("shape_scale", "vec3f", "float32", 3, None),
    ("shape_margin", "float32", "float32", None, None),
    ("shape_material_ke", "float32", "float32", None, None),
    ("shape_material_kd", "float32", "float32", None, None),
    ("shape_material_mu", "float32", "float32", None, None),
    ("shape_flags", "int32", "int32", None, None),
    ("shape_world", "int32", "int32", None, None),
    ("shape_body", "int32", "int32", None, None),
    ("gravity", "vec3f", "float32", 3, None),
]
_MODEL_SCALARS = ["world_count", "particle_count", "tri_count", "edge_count", "shape_count", "body_count",
                  "soft_contact_ke", "soft_contact_kd", "soft_contact_mu"]
_STATE_ARRAYS = ["particle_q", "particle_qd", "particle_f"]
_NP_DTYPES = {"float32": np.float32, "int32": np.int32}


def _format(path: str) -> str:
    ext = os.path.splitext(path.lower())[1]
    if ext == ".json":
        return "json"
    if ext == ".bin":
        try:
            import cbor2  # noqa: F401
        except ImportError:
            raise ImportError("cbor2 library is required for .bin files. Install with: pip install 'cbor2>=5.7.0'")
        return "cbor2"
    raise ValueError(f"Unsupported file extension '{ext}'. Supported extensions: .json, .bin")


def _ndarray(arr: np.ndarray, fmt: str) -> dict:
    arr = np.ascontiguousarray(arr)
    if fmt == "json":
        return {"__type__": "numpy.ndarray", "dtype": str(arr.dtype), "shape": list(arr.shape),
                "data": json.dumps(arr.tolist())}
    return {"__type__": "numpy.ndarray", "dtype": arr.dtype.str, "shape": list(arr.shape), "order": "C",
            "binary_data": arr.tobytes(order="C")}


class _Writer:
    def __init__(self, fmt: str):
        self.fmt = fmt
        self.next_index = 1

    def array(self, arr, warp_type: str, scalar: str, length, shape) -> dict:
        a = arr.detach().cpu().numpy() if isinstance(arr, torch.Tensor) else np.asarray(arr)
        a = a.astype(_NP_DTYPES[scalar], copy=False)
        entry = {"__type__": "warp.array", "__dtype__": f"<class 'warp.types.{warp_type}'>"}
        if length is not None:
            entry["__scalar_type__"] = scalar
            entry["__type_length__"] = int(length)
        if shape is not None:
            entry["__type_shape__"] = list(shape)
        entry["cache_index"] = self.next_index
        self.next_index += 1
        entry["data"] = _ndarray(a, self.fmt)
        return entry

    @staticmethod
    def scalar(v) -> dict:
        if isinstance(v, (bool, np.bool_)):
            return {"__type__": "bool", "value": bool(v)}
        if isinstance(v, (int, np.integer)):
            return {"__type__": "int", "value": int(v)}
        return {"__type__": "float", "value": float(v)}


def _decode_ndarray(d: dict) -> np.ndarray:
    dtype = np.dtype(d["dtype"])
    shape = tuple(d["shape"])
    if "binary_data" in d:
        return np.frombuffer(d["binary_data"], dtype=dtype).reshape(shape, order=d.get("order", "C")).copy()
    data = d["data"]
    if isinstance(data, str):
        data = json.loads(data)
    return np.array(data, dtype=dtype).reshape(shape)


def _decode(x, cache: dict):
    """Serialized entry -> Python value (numpy for arrays, dict of attributes for objects)."""
    if not isinstance(x, dict) or "__type__" not in x:
        return x
    t = x["__type__"]
    if t in ("str", "int", "float", "bool", "NoneType"):
        return x["value"]
    if t == "warp.array":
        arr = _decode_ndarray(x["data"])
        if "cache_index" in x:
            cache[int(x["cache_index"])] = arr
        return arr
    if t == "warp.array_ref":
        return cache.get(int(x["cache_index"]))
    if t == "numpy.ndarray":
        arr = _decode_ndarray(x)
        if "cache_index" in x:
            cache[int(x["cache_index"])] = arr
        return arr
    if t == "numpy.ndarray_ref":
        return cache.get(int(x["cache_index"]))
    if t.startswith("numpy."):
        return getattr(np, t.split(".")[-1])(x["value"])
    if t == "dict":
        return {k: _decode(v, cache) for k, v in x["items"].items()}
    if t in ("list", "tuple", "set"):
        items = [_decode(v, cache) for v in x["items"]]
        return tuple(items) if t == "tuple" else (set(items) if t == "set" else items)
    if "attributes" in x:
        return {k: _decode(v, cache) for k, v in x["attributes"].items()}
    if t in ("warp.HashGrid", "warp.Bvh", "warp.Mesh", "wp.Device", "callable"):
        return None
    return x.get("value", x)


class RecorderFile:
    """Records a model and a history of states to a ViewerFile-format file, and plays them back."""

    def __init__(self, output_path: str, auto_save: bool = True, save_interval: int = 100,
                 max_history_size: int | None = None):
        if not output_path:
            raise ValueError("output_path must be a non-empty path")
        self.output_path = Path(output_path)
        self.auto_save = auto_save
        self.save_interval = save_interval
        self.max_history_size = max_history_size
        self.history: list[dict] = []
        self.model: Model | None = None
        self.deserialized_model: dict | None = None
        self._frame_count = 0
        self._running = True

    # -- recording --------------------------------------------------------------------------
    def set_model(self, model: Model | None) -> None:
        if model is not None and self.model is None:
            self.model = model

    def record(self, state: State) -> None:
        snap = {}
        for name in _STATE_ARRAYS:
            v = getattr(state, name, None)
            if v is not None:
                snap[name] = v.detach().clone() if isinstance(v, torch.Tensor) else np.array(v, copy=True)
        self.history.append(snap)
        if self.max_history_size is not None and len(self.history) > self.max_history_size:
            del self.history[0]

    def log_state(self, state: State) -> None:
        self.record(state)
        self._frame_count += 1
        if self.auto_save and self._frame_count % self.save_interval == 0:
            self.save_recording()

    def end_frame(self) -> None:
        pass

    def is_running(self) -> bool:
        return self._running

    def close(self) -> None:
        if self._running and self.auto_save and self.history:
            self.save_recording()
        self._running = False

    def save_recording(self, file_path: str | None = None, verbose: bool = False) -> None:
        path = str(file_path if file_path is not None else self.output_path)
        fmt = _format(path)
        w = _Writer(fmt)
        model_entry = {"__type__": "NoneType", "value": None}
        if self.model is not None:
            attrs = {}
            for name in _MODEL_SCALARS:
                if hasattr(self.model, name):
                    attrs[name] = w.scalar(getattr(self.model, name))
            for name, wt, sc, ln, shp in _MODEL_ARRAYS:
                v = getattr(self.model, name, None)
                if v is not None and len(np.asarray(v).shape) > 0:
                    attrs[name] = w.array(v, wt, sc, ln, shp)
            attrs["particle_color_groups"] = {
                "__type__": "list",
                "items": [w.array(np.asarray(g, np.int32), "int32", "int32", None, None)
                          for g in self.model.particle_color_groups]}
            model_entry = {"__type__": "Model", "__module__": Model.__module__, "attributes": attrs}
        states = []
        for snap in self.history:
            items = {name: w.array(v, "vec3f", "float32", 3, None) for name, v in snap.items()}
            states.append({"__type__": "dict", "items": items})
        data = {"__type__": "dict", "items": {"model": model_entry, "states": {"__type__": "list", "items": states}}}
        if fmt == "json":
            with open(path, "w") as f:
                json.dump(data, f)
        else:
            import cbor2

            with open(path, "wb") as f:
                f.write(cbor2.dumps(data))
        if verbose:
            print(f"Recording saved to {path} ({len(self.history)} frames)")

    # -- playback ---------------------------------------------------------------------------
    def load_recording(self, file_path: str | None = None, verbose: bool = False) -> None:
        path = str(file_path if file_path is not None else self.output_path)
        fmt = _format(path)
        if fmt == "json":
            with open(path) as f:
                raw = json.load(f)
        else:
            import cbor2

            with open(path, "rb") as f:
                raw = cbor2.loads(f.read())
        cache: dict = {}
        data = _decode(raw, cache)
        self.deserialized_model = data.get("model")
        self.history = [dict(s) for s in (data.get("states") or [])]
        self._frame_count = len(self.history)
        if verbose:
            print(f"Loaded recording with {self._frame_count} frames from {path}")

    def get_frame_count(self) -> int:
        return self._frame_count

    def has_model(self) -> bool:
        return self.deserialized_model is not None

    def load_model(self, model: Model) -> None:
        """Fill ``model`` (this package's Model) with the recorded cloth fields."""
        d = self.deserialized_model
        if not d:
            raise ValueError("the loaded recording has no model")
        for name in _MODEL_SCALARS:
            if name in d and d[name] is not None:
                setattr(model, name, d[name])
        for name, _, sc, _, _ in _MODEL_ARRAYS:
            if name in d and d[name] is not None:
                setattr(model, name, np.asarray(d[name], dtype=_NP_DTYPES[sc]))
        V = int(model.particle_count)
        model.particle_q = model.particle_q.reshape(V, 3)
        model.particle_qd = model.particle_qd.reshape(V, 3)
        model.tri_indices = model.tri_indices.reshape(-1, 3)
        model.tri_poses = model.tri_poses.reshape(-1, 2, 2)
        model.tri_materials = model.tri_materials.reshape(-1, 5)
        model.edge_indices = model.edge_indices.reshape(-1, 4)
        model.edge_bending_properties = model.edge_bending_properties.reshape(-1, 2)
        model.shape_transform = np.asarray(getattr(model, "shape_transform", np.zeros((0, 7))), np.float32).reshape(-1, 7)
        model.shape_scale = np.asarray(getattr(model, "shape_scale", np.zeros((0, 3))), np.float32).reshape(-1, 3)
        model.gravity = np.asarray(model.gravity, np.float32).reshape(-1, 3)
        model.particle_color_groups = [np.asarray(g, np.int32) for g in d.get("particle_color_groups") or []]
        colors = np.full(V, -1, dtype=np.int32)
        for c, g in enumerate(model.particle_color_groups):
            colors[g] = c
        model.particle_colors = colors
        adj = MeshAdjacency(model.tri_indices, model.edge_indices)
        adj.init_vertex_adjacency(V)
        model.soft_mesh_adjacency = adj
        model.notify_model_changed()

    def load_state(self, state: State, frame_id: int) -> None:
        if not (0 <= frame_id < len(self.history)):
            raise IndexError(f"frame_id {frame_id} is out of range [0, {len(self.history)})")
        for name, v in self.history[frame_id].items():
            cur = getattr(state, name, None)
            t = torch.as_tensor(np.asarray(v.cpu() if isinstance(v, torch.Tensor) else v, dtype=np.float32))
            if isinstance(cur, torch.Tensor):
                cur.copy_(t.reshape(cur.shape).to(cur.device))
            else:
                setattr(state, name, t.reshape(-1, 3))
