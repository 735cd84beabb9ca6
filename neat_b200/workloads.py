"""Synthetic workloads of the training step: phantom, scan geometry, octree
and model sizes of each configuration the step is measured and checked on.

Seeded synthetic data stands in for the reference's measured scans (KAUST
Pepper); the phantom is continuous, its density at any point and its line
integrals are exact in f64 (neat_synth.cu).  The octree comes from a greedy
density-variance refinement, which stands in for the reference's MIP
structure optimizer (or-tools).

  small  8 ellipsoids, 32 x 128^2 projections, depth-2 octree (64 leaves),
         C=4, G=11, decoder 4-64-64-1, M=16, 4096 rays per batch.
  full   64 ellipsoids + 200 void spheres, 360 x 512^2 projections with
         Poisson noise (I0 = 1e4), depth-4 octree refined to ~1500 active
         nodes, C=8, G=17, decoder 8-64-64-1, M=32, 2^18 rays per batch.
  large  porous volume: 2000 spheres (radius U[.002,.02], density U[.2,1])
         inside a density-0.3 cylinder, 64 x 1024^2 projections with Poisson
         noise (I0 = 5e3), depth-5 octree refined to ~3000 active nodes
         (levels 2 to 5, so rays per node are highly uneven), C=16, G=17,
         decoder 16-64-64-1, M=32, 2^19 rays per batch; trained with BF16
         grids and decoder operands and the learned sample proposal (12
         samples per segment).
"""
from . import scene as SC

WORKLOADS = {
    "full": dict(desc="plain FP32 full size: 64 ellipsoids + 200 voids, 360 x 512^2 projections, Poisson I0=1e4, "
                      "adaptive octree depth 4 (~1500 active), C=8, G=17, decoder 8-64-64-1, M=32, 2^18 rays/batch",
                 phantom="ellipsoids", n_ell=64, n_void=200, n_angles=360, w=512, h=512, photons=1e4, depth=4,
                 active=1500, C=8, G=17, M=32, R=1 << 18, seed=2, cpu_rays=1 << 14),
    "small": dict(desc="plain FP32 small: 8 ellipsoids, 32 x 128^2 projections, octree depth 2 (64 leaves), C=4, "
                       "G=11, decoder 4-64-64-1, M=16, 4096 rays/batch",
                  phantom="ellipsoids", n_ell=8, n_void=0, n_angles=32, w=128, h=128, photons=None, depth=2,
                  active=None, C=4, G=11, M=16, R=4096, seed=1, cpu_rays=4096),
    "large": dict(desc="large sparse-view, BF16 + learned proposal: porous 2000 spheres (r U[.002,.02], rho U[.2,1]) "
                       "in a rho=0.3 cylinder, 64 x 1024^2 projections, Poisson I0=5e3, adaptive octree depth 5 "
                       "(~3000 active, levels 2-5), C=16, G=17, decoder 16-64-64-1, 2^19 rays/batch, 12 proposal "
                       "samples per segment (32 on the uniform training steps)",
                  phantom="porous", n_spheres=2000, n_angles=64, w=1024, h=1024, photons=5e3, depth=5, active=3000,
                  C=16, G=17, M=32, R=1 << 19, seed=5, cpu_rays=1 << 12, proposal_budget=12),
}


def phantom(cfg):
    """The configuration's phantom objects (rows of 17 doubles, scene.py)."""
    if cfg.get("phantom", "ellipsoids") == "porous":
        return SC.porous_phantom(cfg["n_spheres"], seed=cfg["seed"])
    return SC.ellipsoid_phantom(cfg["n_ell"], cfg["n_void"], seed=cfg["seed"])


def build_workload(cfg, device):
    """(scene, tree, camera) of a configuration on a CUDA device: the phantom
    projected by the device projector (plus Poisson noise where the
    configuration has a photon count) and the octree refined by the phantom's
    density variance on a 4^3 lattice per node."""
    from .api import CameraModel
    from .tree import HyperTreeBase
    objs = phantom(cfg)
    scene = SC.SyntheticScene(objs, cfg["n_angles"], cfg["w"], cfg["h"], device=device, photons=cfg["photons"],
                              noise_seed=cfg["seed"])
    tree = HyperTreeBase(3, cfg["depth"])
    if cfg["active"]:
        tree.RefineByVariance(scene.density, cfg["active"], samples_per_axis=4)
    else:
        tree.SetActive(cfg["depth"])
    return scene, tree, CameraModel.from_scene(scene)
