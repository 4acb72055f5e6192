"""Regenerates the golden fixtures in this directory from the CPU oracle.

    python tests/golden/make_golden.py

cornell_64x64.npz  sample buffer of the 64x64 Cornell box (spp 2, depth 4,
                   frame 3, random pixel jitter), the image-parity golden
soup_trace.npz     closest- and any-hit records of 20k rays (regenerated
                   from their seeds) against a 10k-triangle soup, the
                   prim-id golden

The reference's own shaders cannot run on this machine (no Vulkan device,
Slang is a closed Windows/macOS binary), so these fixtures come from the
oracle's restatement; tests/test_golden.py re-derives them on every CPU run
and the GPU tests compare the kernels against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from strelka_b200 import scenes  # noqa: E402

CORNELL = dict(spp=2, max_depth=4, frame=3, sst=1)


def cornell_samples():
    s = scenes.cornell(64, 64, sphere_levels=4)
    p = s.param(spp=CORNELL["spp"], maxDepth=CORNELL["max_depth"], frameNumber=CORNELL["frame"],
                stratifiedSamplingType=CORNELL["sst"])
    return oracle.pathtrace(oracle.SceneView(s), p, threads=1)


def soup_records():
    s = scenes.soup(10_000, 21)
    v = oracle.SceneView(s)
    rays = np.concatenate([scenes.rays_soup(10_000, 22), scenes.rays_soup(10_000, 23, shadow=True)])
    closest, _, _ = oracle.trace(v, rays, threads=1)
    anyh, _, _ = oracle.trace(v, rays, any_hit=True, threads=1)
    return rays, closest, anyh


def main():
    samples = cornell_samples()
    np.savez_compressed(os.path.join(HERE, "cornell_64x64.npz"), samples=samples, **CORNELL)
    rays, closest, anyh = soup_records()
    np.savez_compressed(os.path.join(HERE, "soup_trace.npz"), closest=closest, any=anyh)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
