"""Export the reference's built-in scenes 0-3 (src/scene.cu:14-218, read from its scenes/
directory by the asset loaders) to tests/golden/_reference_scenes.npz for the GPU parity test
against the reference's CUDA integrator (tests/test_gpu_reference_cuda.py).

The file holds the reference's scene data (meshes, materials, environment maps), so it is
kept out of version control; it is written on a machine that has the reference tree:

    python tests/golden/make_reference_scenes.py path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "gpu-pathed_b200"))

import pathed  # noqa: E402

OUT = os.path.join(HERE, "_reference_scenes.npz")
FIELDS = ("tri_vertices", "tri_normals", "tri_materials", "spheres", "sphere_materials", "material_types",
          "material_albedo", "material_emit", "material_ior", "material_alpha", "env_rgba", "camera")


def main(ref=None):
    ref = ref or (sys.argv[1] if len(sys.argv) > 1 else None)
    if not ref or not os.path.isdir(os.path.join(ref, "scenes")):
        sys.exit("usage: make_reference_scenes.py path/to/reference (the tree holding scenes/)")
    out = {}
    for idx in range(4):
        s = pathed.Session(64, 48)
        s.load_reference_scene(idx, os.path.join(ref, "scenes"))
        e = s.export_scene()
        c = s.counts()
        s.close()
        for k in FIELDS:
            v = e[k]
            out[f"s{idx}_{k}"] = np.zeros((0, 0, 4), np.float32) if v is None else v
        out[f"s{idx}_depth"] = np.int32(c.default_depth)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
