"""Generate ``reference_cloth_meshes.json``: the cloth meshes embedded in the reference's cloth tests.

The reference's ``newton/tests/test_cloth.py`` builds its cloth experiments from literal vertex and
face lists (module constants ``CLOTH_POINTS`` / ``CLOTH_FACES`` and lists inside the ``ClothSim``
set-up methods).  The GPU tests that restate those experiments run where the reference is not
available, so this script reads the literals from the reference source with ``ast`` (no import of
the reference, which needs Warp) and stores them as a fixture.  Run it from the repository root:

    python tests/golden/make_cloth_fixtures.py [path/to/newton/tests/test_cloth.py]
"""

from __future__ import annotations

import ast
import json
import sys
from pathlib import Path

DEFAULT_SOURCE = Path("/root/reference/newton/tests/test_cloth.py")
OUT = Path(__file__).resolve().parent / "reference_cloth_meshes.json"

# (method of ClothSim, local variable) -> fixture key
METHOD_LISTS = {
    ("set_up_bending_experiment", "vs"): "bending_vertices",
    ("set_up_bending_experiment", "fs"): "bending_faces",
    ("set_collision_experiment", "vs1"): "collision_sheet_vertices",
    ("set_collision_experiment", "fs1"): "collision_sheet_faces",
    ("set_collision_experiment", "vs2"): "collision_triangle_vertices",
    ("set_collision_experiment", "fs2"): "collision_triangle_faces",
    ("set_up_non_zero_rest_angle_bending_experiment", "vs"): "cylinder_vertices",
    ("set_up_non_zero_rest_angle_bending_experiment", "fs"): "cylinder_faces",
    ("set_up_complex_rest_angle_bending_experiment", "vs"): "complex_rest_angle_vertices",
    ("set_up_complex_rest_angle_bending_experiment", "fs"): "complex_rest_angle_faces",
    ("set_up_body_cloth_contact_experiment", "vs"): "body_contact_vertices",
    ("set_up_body_cloth_contact_experiment", "fs"): "body_contact_faces",
}


def _literal(node):
    """A list literal, with ``wp.vec3(...)``-wrapped rows unwrapped."""
    if isinstance(node, ast.Call) and node.args:
        return _literal(node.args[0])
    if isinstance(node, ast.ListComp):
        return _literal(node.generators[0].iter)
    return ast.literal_eval(node)


def extract(source: Path) -> dict:
    tree = ast.parse(source.read_text())
    out = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            if name == "CLOTH_POINTS":
                out["cloth_points"] = [list(p) for p in ast.literal_eval(node.value)]
            elif name == "CLOTH_FACES":
                out["cloth_faces_one_based"] = list(ast.literal_eval(node.value))
        if isinstance(node, ast.ClassDef) and node.name == "ClothSim":
            for fn in node.body:
                if not isinstance(fn, ast.FunctionDef):
                    continue
                for stmt in ast.walk(fn):
                    if not (isinstance(stmt, ast.Assign) and len(stmt.targets) == 1
                            and isinstance(stmt.targets[0], ast.Name)):
                        continue
                    key = METHOD_LISTS.get((fn.name, stmt.targets[0].id))
                    if key is None or key in out:
                        continue
                    try:
                        val = _literal(stmt.value)
                    except (ValueError, SyntaxError):
                        continue  # e.g. vs = [wp.vec3(v) for v in vs] after the literal
                    out[key] = [list(v) if isinstance(v, (list, tuple)) else v for v in val]
    missing = sorted((set(METHOD_LISTS.values()) | {"cloth_points", "cloth_faces_one_based"}) - set(out))
    if missing:
        raise RuntimeError(f"not found in {source}: {missing}")
    return out


def main() -> None:
    src = Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_SOURCE
    data = extract(src)
    data["_source"] = "newton/tests/test_cloth.py (literal meshes of ClothSim's experiments)"
    OUT.write_text(json.dumps(data, separators=(",", ":")) + "\n")
    print(f"{OUT}: " + ", ".join(f"{k} {len(v)}" for k, v in data.items() if isinstance(v, list)))


if __name__ == "__main__":
    main()
