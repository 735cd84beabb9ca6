// neat_synth.cu -- synthetic cone-beam scans: analytic line integrals through
// a phantom of additive ellipsoids and cylinders and of override ellipsoids
// (inside them the density is the object's own: 0 for a void, a sphere's
// density for the inclusions of a porous volume), in f64.  This stands in for
// the reference's measured projections (KAUST Pepper, loaded by
// SceneBase::LoadImagesCT); it is data generation, not part of the training
// step.  Compiled with --fmad=false so every f64 operation is rounded as
// written.
//
// Object record (17 doubles): centre(3), semi-axes(3), rotation R(9, row-major,
// local = R^T (p - c)), density, kind.  kind 0: additive ellipsoid; kind 1:
// override ellipsoid; kind 2: additive cylinder along the local z axis (radii
// semi-axes x, y; half-height semi-axis z).  Override objects with a non-zero
// density must not overlap one another (a point inside two would take the
// first one's density, a line through both would count both).
#include "neat_common.cuh"

namespace neat
{

constexpr int OBJ = 17;
constexpr int MAX_VOID_HITS = 64;
constexpr double kFar = 1e300;  // unbounded extent of a chord along a cylinder's axis

// Ray o + t d in the object's scaled local frame: q = (R^T (o - c)) / axes, e = (R^T d) / axes.
__device__ void object_local(const double* ob, const double o[3], const double d[3], double q[3], double e[3])
{
    const double p[3] = {o[0] - ob[0], o[1] - ob[1], o[2] - ob[2]};
    const double* R   = ob + 6;
    for (int i = 0; i < 3; ++i)
    {
        const double lq = R[0 * 3 + i] * p[0] + R[1 * 3 + i] * p[1] + R[2 * 3 + i] * p[2];
        const double le = R[0 * 3 + i] * d[0] + R[1 * 3 + i] * d[1] + R[2 * 3 + i] * d[2];
        q[i]            = lq / ob[3 + i];
        e[i]            = le / ob[3 + i];
    }
}

__device__ bool ellipsoid_chord(const double* ob, const double o[3], const double d[3], double& t0, double& t1)
{
    double q[3], e[3];
    object_local(ob, o, d, q, e);
    const double A    = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    const double B    = q[0] * e[0] + q[1] * e[1] + q[2] * e[2];
    const double Cc   = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] - 1.0;
    const double disc = B * B - A * Cc;
    if (disc <= 0 || A <= 0) return false;
    const double sq = sqrt(disc);
    t0              = (-B - sq) / A;
    t1              = (-B + sq) / A;
    return true;
}

// Chord of the cylinder x^2 + y^2 <= 1, |z| <= 1 (scaled local frame): the
// ray's interval inside the infinite cylinder intersected with the slab.
__device__ bool cylinder_chord(const double* ob, const double o[3], const double d[3], double& t0, double& t1)
{
    double q[3], e[3];
    object_local(ob, o, d, q, e);
    double a0 = -kFar, a1 = kFar;
    const double A  = e[0] * e[0] + e[1] * e[1];
    const double B  = q[0] * e[0] + q[1] * e[1];
    const double Cc = q[0] * q[0] + q[1] * q[1] - 1.0;
    if (A > 0)
    {
        const double disc = B * B - A * Cc;
        if (disc <= 0) return false;
        const double sq = sqrt(disc);
        a0              = (-B - sq) / A;
        a1              = (-B + sq) / A;
    }
    else if (Cc > 0)
        return false;  // parallel to the axis, outside
    double z0 = -kFar, z1 = kFar;
    if (e[2] != 0)
    {
        z0 = (-1.0 - q[2]) / e[2];
        z1 = (1.0 - q[2]) / e[2];
        if (z0 > z1)
        {
            const double t = z0;
            z0             = z1;
            z1             = t;
        }
    }
    else if (q[2] < -1.0 || q[2] > 1.0)
        return false;  // in a plane of constant z outside the slab
    t0 = a0 > z0 ? a0 : z0;
    t1 = a1 < z1 ? a1 : z1;
    return t1 > t0;
}

__device__ bool object_chord(const double* ob, const double o[3], const double d[3], double& t0, double& t1)
{
    return ob[16] == 2.0 ? cylinder_chord(ob, o, d, t0, t1) : ellipsoid_chord(ob, o, d, t0, t1);
}

__device__ double phantom_line(const double* __restrict__ obj, int n_obj, const double o[3], const double d[3],
                               int* status)
{
    // override intervals (kind 1), merged; each adds its own density x chord
    double vs[MAX_VOID_HITS], ve[MAX_VOID_HITS];
    int nv       = 0;
    double total = 0;
    for (int k = 0; k < n_obj; ++k)
    {
        const double* ob = obj + OBJ * k;
        if (ob[16] != 1.0) continue;
        double t0, t1;
        if (!ellipsoid_chord(ob, o, d, t0, t1)) continue;
        if (nv == MAX_VOID_HITS)
        {
            raise_status(status, NEAT_ERR_CAPACITY);
            continue;
        }
        if (ob[15] != 0.0) total += ob[15] * (t1 - t0);
        // insertion by start
        int p = nv++;
        while (p > 0 && vs[p - 1] > t0)
        {
            vs[p] = vs[p - 1];
            ve[p] = ve[p - 1];
            --p;
        }
        vs[p] = t0;
        ve[p] = t1;
    }
    int m = 0;
    for (int k = 0; k < nv; ++k)
    {
        if (m > 0 && vs[k] <= ve[m - 1])
        {
            if (ve[k] > ve[m - 1]) ve[m - 1] = ve[k];
        }
        else
        {
            vs[m] = vs[k];
            ve[m] = ve[k];
            ++m;
        }
    }
    // additive objects (kinds 0 and 2), outside the override intervals
    for (int k = 0; k < n_obj; ++k)
    {
        const double* ob = obj + OBJ * k;
        if (ob[16] != 0.0 && ob[16] != 2.0) continue;
        double t0, t1;
        if (!object_chord(ob, o, d, t0, t1)) continue;
        double len = t1 - t0;
        for (int v = 0; v < m; ++v)
        {
            const double a = vs[v] > t0 ? vs[v] : t0;
            const double b = ve[v] < t1 ? ve[v] : t1;
            if (b > a) len -= (b - a);
        }
        total += ob[15] * len;
    }
    return total;
}

__global__ void k_synth_project(const double* __restrict__ obj, int n_obj, int n_img, int w, int h,
                                const double* __restrict__ intr, const double* __restrict__ rot,
                                const double* __restrict__ trans, float* __restrict__ out, int* status)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (int64_t)n_img * w * h) return;
    const int x   = (int)(p % w);
    const int y   = (int)((p / w) % h);
    const int img = (int)(p / ((int64_t)w * h));
    double cx = ((double)x - intr[2]) / intr[0];
    double cy = ((double)y - intr[3]) / intr[1];
    double cz = 1.0;
    const double n = sqrt((cx * cx + cy * cy) + cz * cz);
    cx /= n;
    cy /= n;
    cz /= n;
    const double* q = rot + 4 * img;
    const double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
    double ux = qy * cz - qz * cy, uy = qz * cx - qx * cz, uz = qx * cy - qy * cx;
    ux += ux;
    uy += uy;
    uz += uz;
    const double d[3] = {(cx + qw * ux) + (qy * uz - qz * uy), (cy + qw * uy) + (qz * ux - qx * uz),
                         (cz + qw * uz) + (qx * uy - qy * ux)};
    const double o[3] = {trans[3 * img], trans[3 * img + 1], trans[3 * img + 2]};
    out[p]            = (float)phantom_line(obj, n_obj, o, d, status);
}

__global__ void k_synth_density(const double* __restrict__ obj, int n_obj, const double* __restrict__ pts, int64_t n,
                                double* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    double rho        = 0;
    for (int k = 0; k < n_obj; ++k)
    {
        const double* ob = obj + OBJ * k;
        const double* R  = ob + 6;
        double l[3];
        for (int a = 0; a < 3; ++a)
        {
            l[a] = R[0 * 3 + a] * (p[0] - ob[0]) + R[1 * 3 + a] * (p[1] - ob[1]) + R[2 * 3 + a] * (p[2] - ob[2]);
            l[a] = l[a] / ob[3 + a];
        }
        const bool inside = ob[16] == 2.0 ? (l[0] * l[0] + l[1] * l[1] <= 1.0 && l[2] * l[2] <= 1.0)
                                          : ((l[0] * l[0] + l[1] * l[1]) + l[2] * l[2] <= 1.0);
        if (inside)
        {
            if (ob[16] == 1.0)
            {
                rho = ob[15];  // override: the first override object containing p
                break;
            }
            rho += ob[15];
        }
    }
    out[i] = rho;
}

}  // namespace neat

using namespace neat;

extern "C" int neat_synth_project(const double* objects, int num_objects, int num_images, int w, int h,
                                  const double* intrinsics, const double* rotation, const double* translation,
                                  float* out, neat_stream_t stream)
{
    if (num_objects < 0 || num_images < 0 || w < 1 || h < 1) return NEAT_ERR_BAD_INPUT;
    const int64_t total = (int64_t)num_images * w * h;
    if (total == 0) return NEAT_OK;
    if (!intrinsics || !rotation || !translation || !out || (num_objects > 0 && !objects)) return NEAT_ERR_BAD_INPUT;
    k_synth_project<<<(unsigned)((total + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        objects, num_objects, num_images, w, h, intrinsics, rotation, translation, out, nullptr);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}

extern "C" int neat_synth_density(const double* objects, int num_objects, const double* points, int64_t num_points,
                                  double* out, neat_stream_t stream)
{
    if (num_objects < 0 || num_points < 0) return NEAT_ERR_BAD_INPUT;
    if (num_points == 0) return NEAT_OK;
    if (!points || !out || (num_objects > 0 && !objects)) return NEAT_ERR_BAD_INPUT;
    k_synth_density<<<(unsigned)((num_points + 255) / 256), 256, 0, (cudaStream_t)stream>>>(objects, num_objects,
                                                                                           points, num_points, out);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
