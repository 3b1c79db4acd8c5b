"""Writes ray-tracing_b200/data/scene_data.json: the caller-side inputs the workload scenes need.

* rough-transmittance eta slices (the set_eta step over ggx.dat) for every eta the seven materials
  use, made by liblrt's own host routine (lrt_rough_transmittance_eta_slice); the 1-D table for any
  alpha follows from a slice by lrt_rough_transmittance_at_alpha, and the CPU tests check that pair
  bit for bit against the reference's rough_transmittance.

(The Hosek sky state is not stored: the library cooks it, lrt_hosek_state.)

Run from the repository root after `make -C oracle ref` and `make -C ray-tracing_b200/csrc`:
    python tests/golden/make_scene_data.py
"""
import base64
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "ray-tracing_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import lrt  # noqa: E402
import oracle  # noqa: E402
import scenes  # noqa: E402


def main():
    data = {"note": "caller-side inputs of the workload scenes; made by tests/golden/make_scene_data.py"}
    pairs = []
    for name in scenes.MATERIAL_NAMES:
        mats, _ = scenes.material_library(name)
        pairs += scenes.required_tables(mats)
    data["eta_slices"] = {}
    for eta, alpha in pairs:
        key = scenes._f32_key(eta)
        if key in data["eta_slices"]:
            continue
        table, diffuse, rng = lrt.rough_transmittance_eta_slice(oracle.GGX_PATH, float(eta))
        data["eta_slices"][key] = {"eta": float(eta), "n_alpha": int(len(diffuse)),
                                   "alpha_range": [float(x) for x in rng],
                                   "table_f32_b64": base64.b64encode(table.astype("<f4").tobytes()).decode(),
                                   "diffuse_f32_b64": base64.b64encode(diffuse.astype("<f4").tobytes()).decode()}
    os.makedirs(scenes.DATA_DIR, exist_ok=True)
    with open(scenes.SCENE_DATA, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", scenes.SCENE_DATA, len(data["eta_slices"]), "eta slices")


if __name__ == "__main__":
    main()
