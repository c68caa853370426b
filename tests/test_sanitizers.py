"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer (CPU only: no GPU
sanitizer runs here).  The library's OBJ parser (eos_b200/csrc/mesh.cpp, plain host C++
behind eos_mesh_*) and the oracle (oracle/eos_oracle.c) are rebuilt with
-fsanitize=address,undefined and run on the mesh fixtures, the reference's models and
fuzzed inputs, and on the oracle's chain, ray-tree, anti-aliasing-grid, two-level and
FP64-adjoint code paths; any sanitizer report fails the test."""
import glob
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-g", "-O1"]
SAN_ENV = {"ASAN_OPTIONS": "detect_leaks=0:halt_on_error=1:verify_asan_link_order=0",
           "UBSAN_OPTIONS": "halt_on_error=1:print_stacktrace=1"}
REPORTS = ("ERROR: AddressSanitizer", "runtime error:", "UndefinedBehaviorSanitizer")


def _runtime(name):
    path = subprocess.run(["gcc", f"-print-file-name={name}"], capture_output=True, text=True).stdout.strip()
    return path if os.path.isabs(path) and os.path.exists(path) else None


def _clean(r):
    out = r.stdout + r.stderr
    return r.returncode == 0 and not any(k in out for k in REPORTS)


def _fuzzed(text: bytes, rng, n: int):
    """n damaged copies of an OBJ text: truncations, flipped bytes, hostile statements."""
    hostile = [b"f 1 2 99999999\n", b"f -5 -6 -7\n", b"f 0 0 0\n", b"v nan inf -inf\n", b"f 1/2/3 4//5 7/8\n",
               b"f\n", b"v 1e40 1 1\n", b"vn 0 0 0\n", b"f 1 1 1 1 1 1 1 1 1 1 1 1\n", b"v 1 2\n",
               b"f 2147483648 1 2\n", b"f -2147483649 1 2\n", b"vt 0.5\n", b"# " + b"x" * 100_000 + b"\n",
               b"f " + b" ".join(b"%d" % (k + 1) for k in range(300)) + b"\n"]
    alphabet = np.frombuffer(b" \n\t/0123456789-+.eEfvnt#", np.uint8)
    out = []
    for k in range(n):
        b = bytearray(text)
        kind = k % 3
        if kind == 0 and len(b) > 1:
            b = b[:int(rng.integers(0, len(b)))]
        elif kind == 1 and len(b):
            for pos in rng.integers(0, len(b), size=12):
                b[int(pos)] = int(rng.choice(alphabet))
        else:
            pos = int(rng.integers(0, len(b) + 1))
            b[pos:pos] = hostile[k % len(hostile)]
        out.append(bytes(b))
    return out


def test_obj_parser_under_sanitizers(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ absent")
    exe = str(tmp_path / "mesh_check")
    subprocess.run(["g++", "-std=c++17", *SAN, "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "eos_b200", "csrc", "mesh.cpp"), os.path.join(HERE, "cpp", "mesh_check.cpp"),
                    "-o", exe], check=True)
    files = sorted(glob.glob(os.path.join(HERE, "golden", "meshes", "*.obj")))
    import oracle
    models = os.path.join(oracle.REF_ROOT, "objmodels")
    if os.path.isdir(models):
        files += sorted(glob.glob(os.path.join(models, "*.obj")))
    rng = np.random.default_rng(11)
    fuzz_dir = tmp_path / "fuzz"
    fuzz_dir.mkdir()
    for src in sorted(glob.glob(os.path.join(HERE, "golden", "meshes", "*.obj"))):
        for k, data in enumerate(_fuzzed(open(src, "rb").read(), rng, 45)):
            p = fuzz_dir / f"{os.path.basename(src)}.{k}.obj"
            p.write_bytes(data)
            files.append(str(p))
    (fuzz_dir / "empty.obj").write_bytes(b"")
    files.append(str(fuzz_dir / "empty.obj"))
    env = {**os.environ, **SAN_ENV}
    r = subprocess.run([exe, *files], capture_output=True, text=True, env=env, timeout=600)
    assert _clean(r), (r.returncode, r.stderr[-3000:])
    lines = r.stdout.split("\n")[:-1]
    assert len(lines) == len(files)
    assert all(ln.startswith("0 ") for ln in lines[:4])  # the fixtures themselves parse


ORACLE_WORK = r"""
import numpy as np
import oracle
from eos_b200 import scenes
sc = scenes.small_random_scene(61, n_spheres=5, level=2, lights=3, refl=0.5, transparent=2, ambient_index=1.0002)
cam = scenes.look_at((1.0, 2.5, 8.0), (0, -0.5, 0), 55.0, 24, 18)
o = oracle.Oracle(sc)
r = o.render(cam, 4, pixel_offset=0.5, spp=2, jitter_seed=3)
o.render(cam, 2, pixel_offset=0.0, spp=4, aa_grid=True)
rng = np.random.default_rng(1)
rays = np.concatenate([rng.uniform(-4, 4, (256, 3)), rng.normal(size=(256, 3))], 1).astype(np.float32)
o.closest(rays); o.any(rays); o.closest_brute(rays[:64])
mp = sc.materials.astype(np.float64).copy(); mp[:, 6] = np.log(mp[:, 6])
o.frozen_f64([cam], 24, 18, 0.5, 4, r["hits"], r["shadows"], mp, sc.lights.astype(np.float64),
             g=np.ones((24 * 18, 3)), spp=2, jitter_seed=3)
both = scenes.small_random_scene(91, n_spheres=5, level=2, lights=3, refl=0.5, transparent=1, both=2,
                                 ambient_index=1.0002)
ob = oracle.Oracle(both)
t = ob.render_tree(cam, 3, pixel_offset=0.5)
ob.frozen_f64([cam], 24, 18, 0.5, 3, t["hits"], t["shadows"], both.materials.astype(np.float64),
              both.lights.astype(np.float64), g=np.ones((24 * 18, 3)), tree=True)
d = scenes.instanced_test_scene(4, n_instances=6, lights=2, transparent=1)
oracle.OracleInstanced(d).render(cam, 3, pixel_offset=0.5)
oracle.morton(sc.verts, sc.tris)
print("ok")
"""


def test_oracle_under_sanitizers(tmp_path):
    asan, ubsan = _runtime("libasan.so"), _runtime("libubsan.so")
    if shutil.which("gcc") is None or not asan or not ubsan:
        pytest.skip("gcc sanitizer runtimes absent")
    so = str(tmp_path / "liboracle_san.so")
    subprocess.run(["gcc", "-std=c11", "-shared", "-fPIC", "-fopenmp", "-ffp-contract=off", *SAN,
                    os.path.join(ROOT, "oracle", "eos_oracle.c"), "-o", so, "-lm"], check=True)
    env = {**os.environ, **SAN_ENV, "LD_PRELOAD": f"{asan}:{ubsan}", "EOS_ORACLE_LIB": so, "OMP_NUM_THREADS": "2"}
    r = subprocess.run([sys.executable, "-c", ORACLE_WORK], capture_output=True, text=True, env=env, cwd=ROOT,
                       timeout=900)
    assert _clean(r) and r.stdout.strip().endswith("ok"), (r.returncode, r.stderr[-3000:])
