"""Synthetic cone-beam scans standing in for the reference's measured data.

The reference trains on real X-ray scans (KAUST Pepper, converted by
samples/nikon2neat.cpp).  Here a seeded phantom of ellipsoids (and void
spheres) is projected analytically in f64 with the same camera model the
training step uses:

* kinds of objects: additive ellipsoids (0), override ellipsoids whose inside
  takes the object's density (1; a void has density 0) and additive cylinders
  along the local z axis (2);
* geometry after nikon2neat.cpp:268-301: volume [-1,1]^3, source at distance
  3 from the centre, detector at 1.5 behind it (SrcToDetector 4.5), source
  direction (sin(-a), -cos(-a), 0), up (0,0,-1), R = [right, up, forward],
  camera->world pose (q, t = source).  Angles a = 2 pi i / N (no duplicated
  last frame);
* intrinsics after nikon2neat.cpp:139-147: fx = fy = W / (2 tan(asin(1/sqrt 3)))
  so the cube's bounding sphere fills the detector, cx = W/2 - 0.5,
  cy = H/2 - 0.5;
* batches after RandomMultiSceneDataset::get_batch (src/data/Dataloader.cpp:8-49):
  uniform image, uniform integer pixel, uv = (x/(w-1), y/(h-1)), target = the
  pixel value (SampleProjection's bilinear lookup at a pixel centre).
"""
import math

import numpy as np
import torch

from . import _lib

OBJ_STRIDE = 17


# --------------------------------------------------------------------------
# phantom
# --------------------------------------------------------------------------
def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _obj(center, axes, R, density, kind):
    o = np.zeros(OBJ_STRIDE, np.float64)
    o[0:3] = center
    o[3:6] = axes
    o[6:15] = np.asarray(R, np.float64).reshape(9)
    o[15] = density
    o[16] = kind
    return o


def porous_phantom(n_spheres=2000, seed=0, radius=(0.002, 0.02), density=(0.2, 1.0), cylinder_radius=0.7,
                   cylinder_half_height=0.8, cylinder_density=0.3, max_tries=200000):
    """Porous volume: an additive cylinder of density cylinder_density along z
    (radius cylinder_radius, half-height cylinder_half_height, centred) holding
    n_spheres override spheres (radius U[radius], density U[density]; inside a
    sphere the density is the sphere's own).  Sphere centres are uniform in the
    cylinder, rejected until the sphere lies wholly inside it and touches no
    earlier sphere, so every point has one well-defined density."""
    rng = np.random.default_rng(seed)
    objs = [_obj([0.0, 0.0, 0.0], [cylinder_radius, cylinder_radius, cylinder_half_height], np.eye(3),
                 cylinder_density, 2)]
    centres = np.zeros((n_spheres, 3))
    radii = np.zeros(n_spheres)
    k = tries = 0
    while k < n_spheres:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("porous_phantom: could not place the spheres apart")
        r = rng.uniform(*radius)
        c = np.array([rng.uniform(-1, 1) * cylinder_radius, rng.uniform(-1, 1) * cylinder_radius,
                      rng.uniform(-1, 1) * cylinder_half_height])
        if math.hypot(c[0], c[1]) > cylinder_radius - r or abs(c[2]) > cylinder_half_height - r:
            continue
        if k and np.any(np.linalg.norm(centres[:k] - c, axis=1) < radii[:k] + r):
            continue
        centres[k], radii[k] = c, r
        objs.append(_obj(c, [r, r, r], np.eye(3), rng.uniform(*density), 1))
        k += 1
    return np.stack(objs)


def ellipsoid_phantom(n_ellipsoids=8, n_voids=0, seed=0):
    """Additive ellipsoids (centre U[-.6,.6]^3, semi-axes U[.05,.3], random
    rotation, density U[.1,1]) and void spheres (radius U[.005,.03]) whose
    inside is forced to density 0."""
    rng = np.random.default_rng(seed)
    objs = []
    for _ in range(n_ellipsoids):
        objs.append(_obj(rng.uniform(-0.6, 0.6, 3), rng.uniform(0.05, 0.3, 3), _random_rotation(rng),
                         rng.uniform(0.1, 1.0), 0))
    for _ in range(n_voids):
        r = rng.uniform(0.005, 0.03)
        objs.append(_obj(rng.uniform(-0.6, 0.6, 3), [r, r, r], np.eye(3), 0.0, 1))
    return np.stack(objs) if objs else np.zeros((0, OBJ_STRIDE))


# --------------------------------------------------------------------------
# geometry
# --------------------------------------------------------------------------
def _quat_from_matrix(R):
    """Unit quaternion (x, y, z, w) of a rotation matrix (Shepperd's method,
    as Eigen::Quaterniond(R))."""
    t = np.trace(R)
    if t > 0:
        s = math.sqrt(t + 1.0) * 2
        w = 0.25 * s
        x = (R[2, 1] - R[1, 2]) / s
        y = (R[0, 2] - R[2, 0]) / s
        z = (R[1, 0] - R[0, 1]) / s
    elif R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]:
        s = math.sqrt(1.0 + R[0, 0] - R[1, 1] - R[2, 2]) * 2
        w = (R[2, 1] - R[1, 2]) / s
        x = 0.25 * s
        y = (R[0, 1] + R[1, 0]) / s
        z = (R[0, 2] + R[2, 0]) / s
    elif R[1, 1] > R[2, 2]:
        s = math.sqrt(1.0 + R[1, 1] - R[0, 0] - R[2, 2]) * 2
        w = (R[0, 2] - R[2, 0]) / s
        x = (R[0, 1] + R[1, 0]) / s
        y = 0.25 * s
        z = (R[1, 2] + R[2, 1]) / s
    else:
        s = math.sqrt(1.0 + R[2, 2] - R[0, 0] - R[1, 1]) * 2
        w = (R[1, 0] - R[0, 1]) / s
        x = (R[0, 2] + R[2, 0]) / s
        y = (R[1, 2] + R[2, 1]) / s
        z = 0.25 * s
    q = np.array([x, y, z, w])
    return q / np.linalg.norm(q)


def cone_beam_geometry(n_angles, w, h, src_dist=3.0, det_dist=1.5):
    """Returns intrinsics [1,5], rotation [n,4] (x,y,z,w), translation [n,3], f64."""
    src_to_det = src_dist + det_dist
    half = math.asin(math.sqrt(3.0) / src_dist)  # the cube's bounding sphere (radius sqrt 3) fills the view
    det_w = 2 * src_to_det * math.tan(half)
    fx = w / det_w * src_to_det
    fy = h / det_w * src_to_det
    intr = np.array([[fx, fy, w / 2.0 - 0.5, h / 2.0 - 0.5, 0.0]], np.float64)
    rot = np.zeros((n_angles, 4))
    trans = np.zeros((n_angles, 3))
    up = np.array([0.0, 0.0, -1.0])
    for i in range(n_angles):
        a = 2 * math.pi * i / n_angles
        d = np.array([math.sin(-a), -math.cos(-a), 0.0])
        source = src_dist * d
        det_c = -d * det_dist
        fwd = det_c - source
        fwd /= np.linalg.norm(fwd)
        right = np.cross(up, fwd)
        right /= np.linalg.norm(right)
        R = np.stack([right, up, fwd], 1)
        rot[i] = _quat_from_matrix(R)
        trans[i] = source
    return intr, rot, trans


# --------------------------------------------------------------------------
# scene
# --------------------------------------------------------------------------
def pixel_to_uv(px, size):
    """PixelToUV with align_corners (src/modules/CameraPose.h:38-54): px / (size - 1)
    in float32, correctly rounded as the reference's CPU tensors divide.  The
    divisor is a tensor: torch divides a CUDA tensor by a Python scalar through
    its reciprocal, which is off by one ulp for some pixels."""
    xf = px.to(torch.float32)
    return xf / torch.full_like(xf, float(size - 1))


class SyntheticScene:
    """Projections [n_img, h, w] f32 on the device plus the camera model."""

    def __init__(self, objects, n_angles, w, h, device="cuda", photons=None, noise_seed=0, projections=None):
        self.objects = np.ascontiguousarray(objects, np.float64)
        self.n_img, self.w, self.h = n_angles, w, h
        self.intrinsics, self.rotation, self.translation = cone_beam_geometry(n_angles, w, h)
        self.device = torch.device(device)
        dev = self.device
        self.intr_t = torch.from_numpy(self.intrinsics).to(dev)
        self.rot_t = torch.from_numpy(self.rotation).to(dev)
        self.trans_t = torch.from_numpy(self.translation).to(dev)
        if projections is None:
            projections = self._project_device()
        self.projection = projections.to(dev).contiguous()
        if photons:
            gen = torch.Generator(device=dev)
            gen.manual_seed(noise_seed)
            lam = photons * torch.exp(-self.projection.double())
            counts = torch.poisson(lam, generator=gen).clamp_min(1.0)
            self.projection = (-torch.log(counts / photons)).float().contiguous()

    def _project_device(self):
        if self.device.type != "cuda":
            raise RuntimeError("device projection needs CUDA; pass projections= computed elsewhere")
        lib = _lib.load()
        obj = torch.from_numpy(self.objects).to(self.device)
        out = torch.empty((self.n_img, self.h, self.w), dtype=torch.float32, device=self.device)
        _lib.check(lib.neat_synth_project(obj.data_ptr(), obj.shape[0], self.n_img, self.w, self.h,
                                          self.intr_t.data_ptr(), self.rot_t.data_ptr(), self.trans_t.data_ptr(),
                                          out.data_ptr(), torch.cuda.current_stream(self.device).cuda_stream),
                   "neat_synth_project")
        return out

    def density(self, points):
        """Phantom density at f64 points [N,3] (device kernel)."""
        lib = _lib.load()
        obj = torch.from_numpy(self.objects).to(self.device)
        pts = torch.as_tensor(np.ascontiguousarray(points, np.float64)).to(self.device)
        out = torch.empty(pts.shape[0], dtype=torch.float64, device=self.device)
        _lib.check(lib.neat_synth_density(obj.data_ptr(), obj.shape[0], pts.data_ptr(), pts.shape[0], out.data_ptr(),
                                          torch.cuda.current_stream(self.device).cuda_stream), "neat_synth_density")
        return out.cpu().numpy()

    def density_volume(self, n):
        """Phantom density on the n^3 voxel-corner lattice of [-1,1]^3 (the
        positions of UniformSampledVolume: (c / (n-1)) * 2 - 1), f64 on the
        device, [n (z), n (y), n (x)]."""
        lib = _lib.load()
        dev = self.device
        obj = torch.from_numpy(self.objects).to(dev)
        lin = torch.arange(n, dtype=torch.float64, device=dev) / (n - 1) * 2 - 1
        z, y, x = torch.meshgrid(lin, lin, lin, indexing="ij")
        pts = torch.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], 1).contiguous()
        out = torch.empty(pts.shape[0], dtype=torch.float64, device=dev)
        _lib.check(lib.neat_synth_density(obj.data_ptr(), obj.shape[0], pts.data_ptr(), pts.shape[0], out.data_ptr(),
                                          torch.cuda.current_stream(dev).cuda_stream), "neat_synth_density")
        return out.reshape(n, n, n)

    def sample_batch(self, num_rays, generator, device=None, images=None):
        """uv [R,2] f32, image_id [R] i32, target [R] f32 (a1 of the hot path):
        uniform image (from `images`, the training split, when given), uniform
        integer pixel, uv = pixel / (size - 1), target = that pixel
        (RandomMultiSceneDataset::get_batch, src/data/Dataloader.cpp:8-49)."""
        dev = self.projection.device if device is None else torch.device(device)
        g = generator
        if images is None:
            img = torch.randint(0, self.n_img, (num_rays,), generator=g, device=g.device)
        else:
            ids = torch.as_tensor(images, dtype=torch.int64, device=g.device)
            img = ids[torch.randint(0, ids.numel(), (num_rays,), generator=g, device=g.device)]
        x = torch.randint(0, self.w, (num_rays,), generator=g, device=g.device)
        y = torch.randint(0, self.h, (num_rays,), generator=g, device=g.device)
        uv = torch.stack([pixel_to_uv(x, self.w), pixel_to_uv(y, self.h)], 1)
        proj = self.projection if self.projection.device == img.device else self.projection.to(img.device)
        target = proj[img, y, x]
        return uv.to(dev).contiguous(), img.to(torch.int32).to(dev).contiguous(), target.to(dev).contiguous()
