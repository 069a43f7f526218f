"""Regenerates the committed reference fixtures under tests/golden/.

Run once with the root of a reference checkout (the directory holding mujoco_warp/):
  python tests/golden/make_golden.py <reference_root>

It copies the reference's MJCF test models verbatim (they carry their own licence headers; the
humanoid is the benchmark model) into tests/golden/models/, and reads the reference's test files
*as text* (Python ``ast``) to extract their known-answer vectors and inline MJCF strings into
tests/golden/reference_fixtures.json:
  - math_test.py:22-88          closest segment-segment points (inputs, expected, decimals)
  - broad_phase_test.py:45-98   SAP model and its expected pair list
  - broad_phase_test.py:127-185 nxn model with keyframes
  - collision_driver_test.py:38-102 primitive collision models
Nothing at test or bench time reads the reference tree.
"""

import ast
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _lit(node):
  return ast.literal_eval(node)


def _vec3(call):
  # wp.vec3([x, y, z])
  return [float(x) for x in _lit(call.args[0])]


def math_cases(path):
  tree = ast.parse(open(path).read())
  cases = []
  for fn in ast.walk(tree):
    if not isinstance(fn, ast.FunctionDef) or not fn.name.startswith("test_"):
      continue
    vecs = {}
    expected = []
    for node in ast.walk(fn):
      if isinstance(node, ast.Assign):
        targets = node.targets[0]
        names = [t.id for t in targets.elts] if isinstance(targets, ast.Tuple) else [targets.id]
        values = node.value.elts if isinstance(node.value, ast.Tuple) else [node.value]
        for n, v in zip(names, values):
          if isinstance(v, ast.Call) and getattr(v.func, "attr", "") == "vec3":
            vecs[n] = _vec3(v)
      if (isinstance(node, ast.Call) and getattr(node.func, "attr", "") == "assertSequenceAlmostEqual"):
        expected.append({"var": node.args[0].id, "value": [float(x) for x in _lit(node.args[1])],
                         "places": int(_lit(node.args[2]))})
    cases.append({"name": fn.name, "inputs": vecs, "expected": expected})
  return cases


def module_constants(path):
  tree = ast.parse(open(path).read())
  out = {}
  for node in ast.walk(tree):
    if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
      try:
        out[node.targets[0].id] = _lit(node.value)
      except ValueError:
        pass
  return out


def main(ref_root):
  src = os.path.join(ref_root, "mujoco_warp")
  models = os.path.join(HERE, "models")
  os.makedirs(models, exist_ok=True)
  for rel in ("test_data/humanoid/humanoid.xml", "test_data/pendula.xml",
              "test_data/collision.xml", "test_data/constraints.xml"):
    shutil.copyfile(os.path.join(src, rel), os.path.join(models, os.path.basename(rel)))
  bp = module_constants(os.path.join(src, "_src", "broad_phase_test.py"))
  cd = module_constants(os.path.join(src, "_src", "collision_driver_test.py"))
  fixtures = {
    "source": "reference test files read as text by tests/golden/make_golden.py",
    "math_closest_segments": math_cases(os.path.join(src, "_src", "math_test.py")),
    "sap_model": bp["_SAP_MODEL"],
    "sap_expected_pairs": [list(p) for p in bp["collision_pair"]],
    "nxn_model": bp["_NXN_MODEL"],
    "primitive_models": cd["_MJCFS"],
  }
  with open(os.path.join(HERE, "reference_fixtures.json"), "w") as f:
    json.dump(fixtures, f, indent=1)
  print("wrote", os.path.join(HERE, "reference_fixtures.json"))


if __name__ == "__main__":
  if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py <reference_root>")
  main(sys.argv[1])
