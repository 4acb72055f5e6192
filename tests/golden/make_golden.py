"""Regenerates the golden fixtures in this directory from the reference's own
shader code, compiled on the host (oracle/_ref, built by oracle/build_ref.sh
from the reference tree).

    python tests/golden/make_golden.py

cornell_64x64.npz  sample buffer of the 64x64 Cornell box (spp 2, depth 4,
                   frame 3, random pixel jitter) as the reference's
                   computeMain (pathtracerMdl.hlsl:406-423) produces it, and
                   the mask of samples whose path reads a buffer out of range
                   there (a diffuse bounce onto a light's emitter reads
                   mdlMaterials[(uint)-1]): their value is undefined in the
                   reference, so comparisons leave them out; the image-parity
                   golden
soup_trace.npz     closest- and any-hit records of 20k rays (regenerated
                   from their seeds) against a 10k-triangle soup, from the
                   reference's closestHit / anyHit (raytracing.h:198-286);
                   the prim-id golden

The materials are the project's native ones (the reference generates its
own with the MDL SDK, absent here); the Cornell box uses the Lambert
material, which follows the reference's shaders/pathtracer.hlsl:176-234.
tests/test_golden.py checks the oracle against these fixtures on every CPU
run, and the GPU tests check the kernels against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from strelka_b200 import scenes  # noqa: E402

CORNELL = dict(spp=2, max_depth=4, frame=3, sst=1)


def cornell_scene():
    s = scenes.cornell(64, 64, sphere_levels=4)
    p = s.param(spp=CORNELL["spp"], maxDepth=CORNELL["max_depth"], frameNumber=CORNELL["frame"],
                stratifiedSamplingType=CORNELL["sst"])
    return s, p


def soup_inputs():
    s = scenes.soup(10_000, 21)
    rays = np.concatenate([scenes.rays_soup(10_000, 22), scenes.rays_soup(10_000, 23, shadow=True)])
    return s, rays


def cornell_oracle():
    s, p = cornell_scene()
    return oracle.pathtrace(oracle.SceneView(s), p, threads=1)


def soup_oracle():
    s, rays = soup_inputs()
    v = oracle.SceneView(s)
    closest, _, _ = oracle.trace(v, rays, threads=1)
    anyh, _, _ = oracle.trace(v, rays, any_hit=True, threads=1)
    return closest, anyh


def main():
    from oracle import ref

    s, p = cornell_scene()
    samples, undefined = ref.pathtrace(oracle.SceneView(s), p, threads=1)
    np.savez_compressed(os.path.join(HERE, "cornell_64x64.npz"), samples=samples, undefined=undefined, **CORNELL)
    s, rays = soup_inputs()
    v = oracle.SceneView(s)
    closest, _ = ref.trace(v, rays)
    anyh, _ = ref.trace(v, rays, any_hit=True)
    np.savez_compressed(os.path.join(HERE, "soup_trace.npz"), closest=closest, any=anyh)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
