// neat_pose.cu -- camera pose and intrinsics gradients of the step's loss and
// the reference's structure optimizer step on them.
//
// The chain is the reference's autograd:
//   sample position p = o[ray] + d[ray] t, t held constant
//     (CreateSamplesForRays, src/structure/HyperTree.cu:426-432)
//   -> local coordinates (p - min) / (max - min) * 2 - 1 (HyperTree.cu:177-192)
//   -> IGS with its uv gradient (src/modules/IndirectGridSample3D.cu:839-873)
//   -> decoder.
// The backward tile kernel leaves, per node-major segment, the sums over its
// samples of dL/d(ix, iy, iz) and of t times them; dix/dp = (G - 1) / (max - min)
// on each axis turns them into dL/do and dL/dd of the segment's ray.
// Rays (SceneBase::GetRays, src/data/SceneBase.cpp:171-193):
//   o = translation[img] (f64, cast to f32), px = u (w - 1), py = v (h - 1),
//   q = ((px - cx) / fx, (py - cy) / fy, 1), n = q / |q|  (Unproject, CameraPose.cu:262-274),
//   d = R(rotation[img]) n                                 (RotatePoint, CameraPose.cu:37-127).
// RotatePoint's rotation gradient is taken on a left tangent at zero, the
// form the optimizer applies (rotation <- exp(tangent) rotation,
// CameraPoseModuleImpl::ApplyTangent, CameraPose.cu:163-183):
//   d(exp(w) d)/dw = -[d]x at w = 0, so dL/dtangent = d x dL/dd,
// and dL/dn = R^T dL/dd.  The ray part runs in f64, as the reference's.
#include <algorithm>
#include <cmath>

#include "neat_common.cuh"
#include "neat_internal.h"

namespace neat
{

// v rotated by the unit quaternion (x, y, z, w): v + w t + u x t, t = 2 u x v.
__device__ __forceinline__ void quat_rotate(double qx, double qy, double qz, double qw, const double v[3],
                                            double out[3])
{
    const double tx = 2.0 * (qy * v[2] - qz * v[1]);
    const double ty = 2.0 * (qz * v[0] - qx * v[2]);
    const double tz = 2.0 * (qx * v[1] - qy * v[0]);
    out[0]          = v[0] + qw * tx + (qy * tz - qz * ty);
    out[1]          = v[1] + qw * ty + (qz * tx - qx * tz);
    out[2]          = v[2] + qw * tz + (qx * ty - qy * tx);
}

// Per node-major segment: sums of dL/d(ix,iy,iz) (and t times them) scaled by
// dix/dp into dL/do and dL/dd of its ray (f32 adds, as the reference's
// index_add over samples).
__global__ void k_seg_pose(const SegRec* __restrict__ segs, const int64_t* counters, const float* __restrict__ seg_pgrad,
                           int G, float* __restrict__ ray_pgrad)
{
    const int64_t nseg = counters[0];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nseg; i += (int64_t)gridDim.x * blockDim.x)
    {
        const float* g = seg_pgrad + 6 * i;
        float v[6];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 6; ++k)
        {
            v[k] = g[k];
            any  = any || v[k] != 0.0f;
        }
        if (!any) continue;
        const SegRec& r = segs[i];
        float* out      = ray_pgrad + 6 * (int64_t)r.ray;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
        {
            const float sc = __fdiv_rn((float)(G - 1), __fsub_rn(r.mx[ax], r.mn[ax]));
            atomicAdd(out + ax, v[ax] * sc);
            atomicAdd(out + 3 + ax, v[3 + ax] * sc);
        }
    }
}

// Per ray: dL/do -> translation, dL/dd -> rotation tangent and (through the
// normalisation and the unprojection) fx, fy, cx, cy.  Per-image sums by f64
// atomics; the single camera's intrinsics by a block reduction first.
__global__ void __launch_bounds__(256) k_ray_pose(int64_t R, const float* __restrict__ uv,
                                                  const int32_t* __restrict__ image_id, int w, int h,
                                                  const double* __restrict__ intr, const double* __restrict__ rot,
                                                  const float* __restrict__ ray_pgrad, double* __restrict__ g_tan,
                                                  double* __restrict__ g_tr, double* __restrict__ g_intr)
{
    __shared__ double red[4][256];
    double gi[4]    = {0.0, 0.0, 0.0, 0.0};
    const double fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x)
    {
        const float* g = ray_pgrad + 6 * r;
        double go[3], gd[3];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            go[k] = (double)g[k];
            gd[k] = (double)g[3 + k];
            any   = any || go[k] != 0.0 || gd[k] != 0.0;
        }
        if (!any) continue;
        const int img = image_id[r];
#pragma unroll
        for (int k = 0; k < 3; ++k) atomicAdd(g_tr + 3 * img + k, go[k]);
        // the ray's camera-space direction as the step formed it (make_ray)
        const float px    = __fmul_rn(uv[2 * r], (float)(w - 1));
        const float py    = __fmul_rn(uv[2 * r + 1], (float)(h - 1));
        const double x    = ((double)px - cx) / fx, y = ((double)py - cy) / fy;
        const double nr   = sqrt(x * x + y * y + 1.0);
        const double n[3] = {x / nr, y / nr, 1.0 / nr};
        const double qx = rot[4 * img], qy = rot[4 * img + 1], qz = rot[4 * img + 2], qw = rot[4 * img + 3];
        double d[3];
        quat_rotate(qx, qy, qz, qw, n, d);
        atomicAdd(g_tan + 3 * img + 0, d[1] * gd[2] - d[2] * gd[1]);
        atomicAdd(g_tan + 3 * img + 1, d[2] * gd[0] - d[0] * gd[2]);
        atomicAdd(g_tan + 3 * img + 2, d[0] * gd[1] - d[1] * gd[0]);
        // dL/dn = R^T dL/dd; dL/dq = (dL/dn - n (n . dL/dn)) / |q|
        double gn[3];
        quat_rotate(-qx, -qy, -qz, qw, gd, gn);
        const double dn  = n[0] * gn[0] + n[1] * gn[1] + n[2] * gn[2];
        const double gux = (gn[0] - n[0] * dn) / nr, guy = (gn[1] - n[1] * dn) / nr;
        gi[0] += -gux * ((double)px - cx) / (fx * fx);
        gi[1] += -guy * ((double)py - cy) / (fy * fy);
        gi[2] += -gux / fx;
        gi[3] += -guy / fy;
    }
    const int t = threadIdx.x;
#pragma unroll
    for (int k = 0; k < 4; ++k) red[k][t] = gi[k];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1)
    {
        if (t < o)
#pragma unroll
            for (int k = 0; k < 4; ++k) red[k][t] += red[k][t + o];
        __syncthreads();
    }
    if (t < 4 && red[t][0] != 0.0) atomicAdd(g_intr + t, red[t][0]);
}

// The structure optimizer step of one image (thread i) and of the camera
// (thread 0): SGD, then the rotation tangent applied on the left.
__global__ void k_pose_sgd(double* __restrict__ rot, double* __restrict__ trans, double* __restrict__ intr,
                           double* __restrict__ g_tan, double* __restrict__ g_tr, double* __restrict__ g_intr, int n,
                           double lr_p, double lr_i, int opt_pose, int opt_intr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        if (opt_pose)
        {
            // tangent after SGD from zero: w = -lr g; q <- exp(w) q (unit
            // quaternion exponential of the rotation vector, then the product)
            const double wx = -lr_p * g_tan[3 * i], wy = -lr_p * g_tan[3 * i + 1], wz = -lr_p * g_tan[3 * i + 2];
            const double th2 = wx * wx + wy * wy + wz * wz;
            double im, re;
            if (th2 < 1e-20)
            {
                im = 0.5 - th2 / 48.0;
                re = 1.0 - th2 / 8.0;
            }
            else
            {
                const double th = sqrt(th2);
                im              = sin(0.5 * th) / th;
                re              = cos(0.5 * th);
            }
            const double ax = im * wx, ay = im * wy, az = im * wz, aw = re;
            const double bx = rot[4 * i], by = rot[4 * i + 1], bz = rot[4 * i + 2], bw = rot[4 * i + 3];
            const double x  = aw * bx + ax * bw + ay * bz - az * by;
            const double y  = aw * by - ax * bz + ay * bw + az * bx;
            const double z  = aw * bz + ax * by - ay * bx + az * bw;
            const double q  = aw * bw - ax * bx - ay * by - az * bz;
            const double s  = 1.0 / sqrt(x * x + y * y + z * z + q * q);
            rot[4 * i]      = x * s;
            rot[4 * i + 1]  = y * s;
            rot[4 * i + 2]  = z * s;
            rot[4 * i + 3]  = q * s;
#pragma unroll
            for (int k = 0; k < 3; ++k) trans[3 * i + k] -= lr_p * g_tr[3 * i + k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            g_tan[3 * i + k] = 0.0;
            g_tr[3 * i + k]  = 0.0;
        }
    }
    if (i == 0)
    {
#pragma unroll
        for (int k = 0; k < 5; ++k)
        {
            if (opt_intr) intr[k] -= lr_i * g_intr[k];
            g_intr[k] = 0.0;
        }
    }
}

cudaError_t launch_pose_grad(const SegRec* segs, const int64_t* counters, const float* seg_pgrad, int G,
                             float* ray_pgrad, const float* uv, const int32_t* image_id, int64_t R, int w, int h,
                             const double* intrinsics, const double* rotation, const neat_pose_grad* pose,
                             cudaStream_t st)
{
    k_seg_pose<<<sm_count() * 8, 256, 0, st>>>(segs, counters, seg_pgrad, G, ray_pgrad);
    const int nb = (int)std::min<int64_t>((R + 255) / 256, (int64_t)sm_count() * 4);
    k_ray_pose<<<nb, 256, 0, st>>>(R, uv, image_id, w, h, intrinsics, rotation, ray_pgrad, pose->grad_tangent,
                                   pose->grad_translation, pose->grad_intrinsics);
    return cudaGetLastError();
}

}  // namespace neat

using namespace neat;

extern "C" int neat_pose_sgd(double* rotation, double* translation, double* intrinsics, const neat_pose_grad* grad,
                             double lr_pose, double lr_intrinsics, int optimize_pose, int optimize_intrinsics,
                             neat_stream_t stream)
{
    if (!rotation || !translation || !intrinsics || !grad || !grad->grad_tangent || !grad->grad_translation ||
        !grad->grad_intrinsics || grad->num_images < 1)
        return NEAT_ERR_BAD_INPUT;
    const int n = grad->num_images;
    k_pose_sgd<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(rotation, translation, intrinsics,
                                                                   grad->grad_tangent, grad->grad_translation,
                                                                   grad->grad_intrinsics, n, lr_pose, lr_intrinsics,
                                                                   optimize_pose, optimize_intrinsics);
    return cudaGetLastError() == cudaSuccess ? NEAT_OK : NEAT_ERR_CUDA;
}
