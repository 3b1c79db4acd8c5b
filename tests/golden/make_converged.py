"""Generates tests/golden/converged_kat.npz: 4096-spp renders by the reference's own path integrator
(the unmodified LinRT sources compiled by oracle/Makefile into oracle/_ref/liblrt_ref.so) of the two
benchmarked path-tracing configurations, with per-pixel second moments:

* the closed box (81,920-triangle displaced sphere, diffuse 0.8, ceiling light (17, 12, 4)) at its full
  256 x 256 frame, depth 6, Russian roulette from depth 3;
* each of the seven materials on the sphere in the box open to the Hosek sky, 512 x 512, depth 8,
  Russian roulette from depth 3, over a 64 x 64 crop of the frame (rows 224-287, columns 96-159: the
  sphere's left silhouette, the sphere and the red wall behind it).

Both use samples 65536.. of every pixel, disjoint from the samples 0.. a render draws by default, so a
render and the fixture are independent estimates of the same converged image. The reference draws the
same Sobol samples as main.cpp:121-136 (sampler.start(pixel, sample)).

    make -C oracle ref && python tests/golden/make_converged.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ray-tracing_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
import scenes  # noqa: E402

SPP = 4096
SAMPLE_OFFSET = 1 << 16
CROP = (224, 288, 96, 160)  # rows [224, 288), columns [96, 160) of the 512 x 512 frame


def main():
    out = {"spp": np.int32(SPP), "sample_offset": np.int32(SAMPLE_OFFSET), "crop": np.array(CROP, np.int32)}
    c0 = scenes.CONFIG0
    world = oracle.RefWorld(scenes.cornell_box())
    p = scenes.render_params(c0["width"], c0["height"], SPP, c0["max_depth"], c0["rr_depth"], SAMPLE_OFFSET)
    t = time.time()
    img, sq, _ = world.render(p, 0, True)
    world.close()
    out["closed_box_mean"], out["closed_box_sq"] = img, sq
    print("closed box 256x256 x %d spp: %.0f s" % (SPP, time.time() - t), flush=True)
    c1 = scenes.CONFIG1
    r0, r1, x0, x1 = CROP
    for name in scenes.MATERIAL_NAMES:
        world = oracle.RefWorld(scenes.open_box(name))
        p = scenes.render_params(c1["width"], c1["height"], SPP, c1["max_depth"], c1["rr_depth"], SAMPLE_OFFSET,
                                 row_begin=r0, row_end=r1)
        t = time.time()
        img, sq, _ = world.render_window(p, x0, x1)
        world.close()
        out["open_%s_mean" % name] = np.ascontiguousarray(img[r0:r1, x0:x1])
        out["open_%s_sq" % name] = np.ascontiguousarray(sq[r0:r1, x0:x1])
        print("open box %s crop x %d spp: %.0f s" % (name, SPP, time.time() - t), flush=True)
    path = os.path.join(HERE, "converged_kat.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
