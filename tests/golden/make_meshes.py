"""Writes the OBJ fixtures of tests/golden/meshes/ (seeded, generated -- no external models).

    python tests/golden/make_meshes.py

* blob.obj       noisy level-3 icosphere (1,280 triangles), positions only: smooth normals
                 are generated; shared 'v' entries and separate 'v' entries at equal
                 positions both occur (the upper cap repeats its vertices).
* shapes.obj     quads (a box), a concave quad, a pentagon, a line (dropped), negative
                 indices, 'v/vt' corners, comments, o / g / usemtl / s statements (ignored).
* grid_vn.obj    a 6 x 4 grid with 'vn' normals, corners 'v//vn' and 'v/vt/vn', CRLF lines.
* near.obj       two triangles whose corners lie within and just outside the smoothing
                 distance (1e-4 x the bounding-box diagonal) of each other.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "meshes")
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from eos_b200 import scenes  # noqa: E402


def blob() -> str:
    rng = np.random.default_rng(4242)
    v, f = scenes.icosphere(3)
    v = v * (1.0 + 0.08 * rng.standard_normal((v.shape[0], 1)))
    lines = ["# noisy icosphere, no normals"]
    lines += [f"v {x:.6f} {y:.6f} {z:.6f}" for x, y, z in v]
    # faces touching the upper cap use a second copy of their vertices (same coordinates)
    cap = v[:, 1] > 0.7
    remap = {}
    for i in np.nonzero(cap)[0]:
        x, y, z = v[i]
        lines.append(f"v {x:.6f} {y:.6f} {z:.6f}")
        remap[i] = v.shape[0] + len(remap)
    for a, b, c in f:
        if cap[a] and cap[b] and cap[c]:
            a, b, c = remap[a], remap[b], remap[c]
        lines.append(f"f {a + 1} {b + 1} {c + 1}")
    return "\n".join(lines) + "\n"


def shapes() -> str:
    return """# quads, polygons, relative indices
mtllib shapes.mtl
o Box
g box
usemtl red
s 1
v -1 -1 -1
v 1 -1 -1
v 1 1 -1
v -1 1 -1
v -1 -1 1
v 1 -1 1
v 1 1 1
v -1 1 1
vt 0 0
vt 1 0
vt 1 1
f 1/1 4/2 3/3 2/1
f 5 6 7 8
f 1 2 6 5
f 2 3 7 6
f 3 4 8 7
f 4 1 5 8
o Arrow
s off
v 3 0 0
v 5 0 0
v 4 0.5 0
v 4 2 0
f -4 -3 -2 -1   # concave quad: corner 3 (4, 0.5) is the reflex corner
v 6 0 0
v 7 0 0.25
v 7.5 1 0.5
v 6.75 2 0.25
v 6 1.5 0
f -5 -4 -3 -2 -1
f 1 2
"""


def grid_vn() -> str:
    rng = np.random.default_rng(77)
    nx, nz = 6, 4
    lines = ["o Grid", "vt 0.5 0.5"]
    for j in range(nz + 1):
        for i in range(nx + 1):
            lines.append(f"v {i * 0.5 - 1.5:.4f} {0.1 * rng.standard_normal():.5f} {j * 0.5 - 1.0:.4f}")
    for k in range(3):
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        lines.append(f"vn {n[0]:.6f} {abs(n[1]) + 0.5:.6f} {n[2]:.6f}")
    for j in range(nz):
        for i in range(nx):
            a = j * (nx + 1) + i + 1
            b, c, d = a + 1, a + nx + 2, a + nx + 1
            k = (i + j) % 3 + 1
            if (i + j) % 2:
                lines.append(f"f {a}//{k} {b}//{k} {c}//{k} {d}//{k}")
            else:
                lines.append(f"f {a}/1/{k} {b}/1/{k} {c}/1/{(k % 3) + 1}")
                lines.append(f"f {a}/1/{k} {c}/1/{(k % 3) + 1} {d}/1/{k}")
    return "\r\n".join(lines) + "\r\n"


def near() -> str:
    # bounding-box diagonal 10*sqrt(3) -> smoothing distance about 1.7e-3
    return """v 0 0 0
v 10 0 0
v 0 10 0
v 0.001 0.0 0.0
v 0 0 10
v 10 10 10
v 0.0 0.003 0.0
v 5 5 10
f 1 2 3
f 4 5 6
f 7 8 5
"""


def main():
    os.makedirs(OUT, exist_ok=True)
    for name, fn in (("blob", blob), ("shapes", shapes), ("grid_vn", grid_vn), ("near", near)):
        text = fn()
        with open(os.path.join(OUT, f"{name}.obj"), "w", newline="") as f:
            f.write(text)
        print(name, len(text), "bytes")


if __name__ == "__main__":
    main()
