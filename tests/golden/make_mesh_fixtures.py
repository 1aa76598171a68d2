"""Writes tests/golden/mfem_order1_meshes.npz: the order-1 MFEM meshes of
the reference's test data (src/tests/dray/data/{beam-hex, fichera, beam-tet,
beam-quad, beam-tri}.mesh) converted by devil_ray_b200.mesh_io into the
path's control-point arrays, so that GPU tests can run on them where the
reference checkout is absent.  Each mesh contributes <name>/ctrl_idx,
<name>/xyz, <name>/shape and <name>/sha256 (of the source file).

    python tests/golden/make_mesh_fixtures.py <reference checkout>/src/tests/dray/data
"""
import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

NAMES = ("beam-hex", "fichera", "beam-tet", "beam-quad", "beam-tri")
OUT = Path(__file__).resolve().parent / "mfem_order1_meshes.npz"


def main(data_dir: str):
    from devil_ray_b200 import mesh_io
    arrays = {}
    for name in NAMES:
        path = Path(data_dir) / f"{name}.mesh"
        m = mesh_io.read_mfem_mesh(path)
        arrays[f"{name}/ctrl_idx"] = m.ctrl_idx
        arrays[f"{name}/xyz"] = m.xyz
        arrays[f"{name}/shape"] = np.array(m.shape)
        arrays[f"{name}/sha256"] = np.array(hashlib.sha256(path.read_bytes()).hexdigest())
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
