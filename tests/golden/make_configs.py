"""Writes the project-written models of the uneven-contact configurations (not from the reference):

  python tests/golden/make_configs.py

- models/bin.xml: a bin (ground plane + 4 wall planes at x, y = +-0.5 m) holding 48 free spheres
  (radius ~ U(0.03, 0.08) m, density 1000) and 16 free capsules (radius 0.04 m, half-length
  0.1 m): nq = 448, nv = 384, 69 geoms.  Radii come from numpy's default_rng(seed=3); body
  positions are a grid (the tests draw seeded states).
- models/humanoid_spheres.xml: the humanoid of humanoid.xml plus 16 free spheres of radius 0.05 m
  (nq = 140, nv = 123); its keyframes are dropped (their qpos no longer fits), the tests append
  the spheres' qpos to the humanoid's own keyframes.

The output is deterministic; the committed files are what this script writes.
"""

import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = os.path.join(HERE, "models")


def bin_xml(seed=3, nsphere=48, ncapsule=16):
  rng = np.random.default_rng(seed)
  radii = rng.uniform(0.03, 0.08, nsphere)
  lines = [
    "<!-- Project-written model (not from the reference), written by make_configs.py: a bin",
    "     (ground plane + 4 wall planes at x, y = +-0.5 m) with 48 free spheres (radius",
    "     U(0.03, 0.08), density 1000) and 16 free capsules (radius 0.04, half-length 0.1);",
    "     nq=448, nv=384, 69 geoms. -->",
    '<mujoco model="bin">',
    '  <option timestep="0.002" integrator="Euler" cone="pyramidal" solver="Newton"',
    '          iterations="10" ls_iterations="10"/>',
    "  <default>",
    '    <geom condim="3"/>',
    "  </default>",
    "  <worldbody>",
    '    <geom name="floor" type="plane" size="0 0 0.05"/>',
    '    <geom name="wall_px" type="plane" pos="0.5 0 0" zaxis="-1 0 0" size="0 0 0.05"/>',
    '    <geom name="wall_nx" type="plane" pos="-0.5 0 0" zaxis="1 0 0" size="0 0 0.05"/>',
    '    <geom name="wall_py" type="plane" pos="0 0.5 0" zaxis="0 -1 0" size="0 0 0.05"/>',
    '    <geom name="wall_ny" type="plane" pos="0 -0.5 0" zaxis="0 1 0" size="0 0 0.05"/>',
  ]
  n = nsphere + ncapsule
  for i in range(n):  # a 4 x 4 grid per layer, 0.2 m apart, layers 0.2 m apart from z = 0.2
    x = -0.3 + 0.2 * (i % 4)
    y = -0.3 + 0.2 * ((i // 4) % 4)
    z = 0.2 + 0.2 * (i // 16)
    if i < nsphere:
      lines.append(f'    <body name="sphere{i}" pos="{x:.3f} {y:.3f} {z:.3f}">')
      lines.append("      <freejoint/>")
      lines.append(f'      <geom type="sphere" size="{radii[i]:.6f}"/>')
    else:
      lines.append(f'    <body name="capsule{i - nsphere}" pos="{x:.3f} {y:.3f} {z:.3f}">')
      lines.append("      <freejoint/>")
      lines.append('      <geom type="capsule" size="0.04 0.1"/>')
    lines.append("    </body>")
  lines += ["  </worldbody>", "</mujoco>", ""]
  return "\n".join(lines)


def humanoid_spheres_xml(nsphere=16):
  with open(os.path.join(MODELS, "humanoid.xml")) as f:
    src = f.read()
  src = re.sub(r"\s*<keyframe>.*?</keyframe>", "", src, flags=re.S)
  bodies = []
  for i in range(nsphere):
    x = 1.0 + 0.3 * (i % 4)
    y = -0.45 + 0.3 * (i // 4)
    bodies += [f'    <body name="ball{i}" pos="{x:.3f} {y:.3f} 0.5">', "      <freejoint/>",
               '      <geom type="sphere" size="0.05"/>', "    </body>"]
  head = ("<!-- Written by make_configs.py from humanoid.xml: the humanoid plus 16 free spheres of\n"
          "     radius 0.05 m (nq=140, nv=123); keyframes dropped. -->\n")
  return head + src.replace("  </worldbody>", "\n".join(bodies) + "\n  </worldbody>", 1)


def main():
  with open(os.path.join(MODELS, "bin.xml"), "w") as f:
    f.write(bin_xml())
  with open(os.path.join(MODELS, "humanoid_spheres.xml"), "w") as f:
    f.write(humanoid_spheres_xml())


if __name__ == "__main__":
  main()
