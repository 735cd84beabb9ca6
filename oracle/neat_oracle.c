/*
 * neat_oracle.c -- CPU restatement of the NeAT forward-projection hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py may call it.
 * The product (neat_b200/) never links, loads or calls it.
 *
 * Every function restates one piece of darglein/NeAT and cites the file:line
 * it follows.  Arithmetic is written so that gcc with -ffp-contract=off
 * evaluates exactly the operations listed (no FMA contraction, IEEE binary32
 * / binary64 round-to-nearest), which is the evaluation order the CUDA
 * kernels reproduce with __fmul_rn/__fadd_rn/__fdiv_rn.
 *
 * Parity pins: IGS forward is checked against torch.grid_sample (border,
 * align_corners) -- the equivalence the reference itself documents at
 * src/modules/IndirectGridSample3D.cu:30-40 -- and against the reference's own
 * CPU IGS (src/modules/IndirectGridSample3D.cu:27-429) compiled under
 * oracle/_ref when libtorch headers are present.  The slab test is checked on
 * known-answer cases and against the reference header compiled the same way.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as   */
/* easy as 1, 2, 3", SC'11).  Counter-based, so a sample's jitter depends   */
/* only on (seed, ray, index in ray, step) and not on thread scheduling.     */
/* ------------------------------------------------------------------------ */
static void philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1, uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    for (int r = 0; r < 10; ++r)
    {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void oracle_philox(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t* out4)
{
    uint32_t ctr[4] = {c0, c1, c2, c3};
    philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), out4);
}

/* uniform in [0,1): top 24 bits of the first Philox word. */
float oracle_uniform(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3)
{
    uint32_t o[4];
    oracle_philox(seed, c0, c1, c2, c3, o);
    return (float)(o[0] >> 8) * (1.0f / 16777216.0f);
}

/* Jitter stream id (4th counter word) for the stratified sample offsets. */
#define NEAT_STREAM_JITTER 0x4a495454u

/* ------------------------------------------------------------------------ */
/* Octree tables: HyperTreeBaseImpl constructor, src/structure/HyperTree.cpp:11-132.   */
/* Breadth-first ids, root 0 = [-1,1]^3; child i takes the upper half on    */
/* axis k when bit k of i is set.                                           */
/* ------------------------------------------------------------------------ */
int oracle_tree_num_nodes(int max_depth)
{
    int n = 0;
    long p = 1;
    for (int i = 0; i <= max_depth; ++i)
    {
        n += (int)p;
        p *= 8;
    }
    return n;
}

void oracle_tree_build(int max_depth, float* pmin, float* pmax, int* depth, int* parent, int* children)
{
    int N = oracle_tree_num_nodes(max_depth);
    for (int i = 0; i < N * 8; ++i) children[i] = -1;
    int cur = 0;
    for (int k = 0; k < 3; ++k)
    {
        pmin[k] = -1.0f;
        pmax[k] = 1.0f;
    }
    depth[0]  = 0;
    parent[0] = -1;
    cur       = 1;
    int layer_start = 0, layer_count = 1;
    for (int d = 1; d <= max_depth; ++d)
    {
        int next_start = cur;
        for (int j = 0; j < layer_count; ++j)
        {
            int nid = layer_start + j;
            float c[3];
            for (int k = 0; k < 3; ++k) c[k] = (pmin[nid * 3 + k] + pmax[nid * 3 + k]) * 0.5f;
            for (int i = 0; i < 8; ++i)
            {
                for (int k = 0; k < 3; ++k)
                {
                    if (((i >> k) & 1) == 0)
                    {
                        pmin[cur * 3 + k] = pmin[nid * 3 + k];
                        pmax[cur * 3 + k] = c[k];
                    }
                    else
                    {
                        pmin[cur * 3 + k] = c[k];
                        pmax[cur * 3 + k] = pmax[nid * 3 + k];
                    }
                }
                children[nid * 8 + i] = cur;
                depth[cur]            = d;
                parent[cur]           = nid;
                cur++;
            }
        }
        layer_start = next_start;
        layer_count = layer_count * 8;
    }
}

/* ------------------------------------------------------------------------ */
/* Ray generation: SceneBase::GetRays (src/data/SceneBase.cpp:171-193),      */
/* UVToPixel (src/modules/CameraPose.h:20-36, align_corners = true,          */
/* src/data/SceneBase.h:22), CameraModelModuleImpl::Unproject                 */
/* (src/modules/CameraPose.cu:262-274, f64), RotatePointGPUk                  */
/* (src/modules/CameraPose.cu:20-33, f64 quaternion rotation, Eigen's         */
/* q*v = v + w*(2 qv x v) + qv x (2 qv x v)).                                */
/* intr: [fx, fy, cx, cy, skew]; rot: [n,4] (x,y,z,w); trans: [n,3].        */
/* ------------------------------------------------------------------------ */
void oracle_make_ray(float u, float v, int img, int w, int h, const double* intr, const double* rot,
                     const double* trans, float* o, float* d)
{
    float px = u * (float)(w - 1);
    float py = v * (float)(h - 1);
    double x = ((double)px - intr[2]) / intr[0];
    double y = ((double)py - intr[3]) / intr[1];
    double z = 1.0;
    double n = sqrt((x * x + y * y) + z * z);
    x = x / n;
    y = y / n;
    z = z / n;
    const double* q = rot + 4 * (long)img;
    double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
    double ux = qy * z - qz * y;
    double uy = qz * x - qx * z;
    double uz = qx * y - qy * x;
    ux = ux + ux;
    uy = uy + uy;
    uz = uz + uz;
    double cx = qy * uz - qz * uy;
    double cy = qz * ux - qx * uz;
    double cz = qx * uy - qy * ux;
    double rx = (x + qw * ux) + cx;
    double ry = (y + qw * uy) + cy;
    double rz = (z + qw * uz) + cz;
    d[0] = (float)rx;
    d[1] = (float)ry;
    d[2] = (float)rz;
    const double* t = trans + 3 * (long)img;
    o[0] = (float)t[0];
    o[1] = (float)t[1];
    o[2] = (float)t[2];
}

void oracle_make_rays(int R, const float* uv, const int* image_id, int w, int h, const double* intr,
                      const double* rot, const double* trans, float* o, float* d)
{
    for (int r = 0; r < R; ++r)
        oracle_make_ray(uv[2 * r], uv[2 * r + 1], image_id[r], w, h, intr, rot, trans, o + 3 * r, d + 3 * r);
}

/* ------------------------------------------------------------------------ */
/* IntersectBoxRayPrecise, src/structure/HyperTree.h:41-83: slab parameters  */
/* in float, running near/far in double, early reject per axis; axis-        */
/* parallel rays reject when o < min or o >= max.                            */
/* ------------------------------------------------------------------------ */
int oracle_intersect_box(const float* pmin, const float* pmax, const float* o, const float* dir, float* tmin,
                         float* tmax)
{
    double t_near = -236436436;
    double t_far  = 43637575;
    for (int i = 0; i < 3; ++i)
    {
        if (dir[i] == 0)
        {
            if ((o[i] < pmin[i]) || (o[i] >= pmax[i])) return 0;
        }
        else
        {
            float T1 = (pmin[i] - o[i]) / dir[i];
            float T2 = (pmax[i] - o[i]) / dir[i];
            if (T1 > T2)
            {
                float tmp = T1;
                T1        = T2;
                T2        = tmp;
            }
            if (T1 > t_near) t_near = T1;
            if (T2 < t_far) t_far = T2;
            if ((t_near > t_far) || (t_far < 0)) return 0;
        }
    }
    *tmin = (float)t_near;
    *tmax = (float)t_far;
    return 1;
}

/* Batch form: pair i tests box (pmin[i], pmax[i]) against ray (o[i], d[i]). */
void oracle_intersect_boxes(long n, const float* pmin, const float* pmax, const float* o, const float* d, int* hit,
                            float* tmin, float* tmax)
{
    for (long i = 0; i < n; ++i)
    {
        float t0 = 0, t1 = 0;
        hit[i]  = oracle_intersect_box(pmin + 3 * i, pmax + 3 * i, o + 3 * i, d + 3 * i, &t0, &t1);
        tmin[i] = t0;
        tmax[i] = t1;
    }
}

/* Node diagonal as (box_max - box_min).norm() in float (HyperTree.cu:286);  */
/* Eigen's fixed-size reduction evaluates a0 + (a1 + a2).                    */
float oracle_node_diag(const float* pmin, const float* pmax)
{
    float dx = pmax[0] - pmin[0], dy = pmax[1] - pmin[1], dz = pmax[2] - pmin[2];
    float s  = dx * dx + (dy * dy + dz * dz);
    return sqrtf(s);
}

/* iCeil for positive arguments. */
static int icei(float x)
{
    int i = (int)x;
    return i + ((float)i < x);
}

typedef struct
{
    float tmin, tmax;
    int node;  /* global node id */
    int local; /* local active id */
    int n;
} hit_t;

static int hit_cmp(const void* a, const void* b)
{
    const hit_t* x = (const hit_t*)a;
    const hit_t* y = (const hit_t*)b;
    if (x->tmin < y->tmin) return -1;
    if (x->tmin > y->tmin) return 1;
    return (x->node < y->node) ? -1 : (x->node > y->node);
}

/* Per-ray hit list in canonical (tmin, node_id) order.  Segment rules from   */
/* ComputeRaySamples (src/structure/HyperTree.cu:258-292): skip when          */
/* tmax - tmin < 1e-5, n = iCeil(((tmax - tmin) / diag) * M).                 */
/* Returns the hit count, or -1 when more than max_hits intersections exist. */
static int ray_hits(const float* o, const float* d, int A, const long* active_ids, const float* pmin,
                    const float* pmax, int M, hit_t* hits, int max_hits)
{
    int k = 0;
    for (int a = 0; a < A; ++a)
    {
        long nid = active_ids[a];
        float t0 = 0, t1 = 0; /* a miss leaves (0, 0), as the reference's {false, 0, 0} */
        int hit = oracle_intersect_box(pmin + 3 * nid, pmax + 3 * nid, o, d, &t0, &t1);
        if ((double)(t1 - t0) < 1e-5) continue;  /* HyperTree.cu:274-277, before the hit check */
        if (!hit) continue;
        if (k >= max_hits) return -1;
        float diag    = oracle_node_diag(pmin + 3 * nid, pmax + 3 * nid);
        float dis     = t1 - t0;
        float rel     = dis / diag;
        hits[k].tmin  = t0;
        hits[k].tmax  = t1;
        hits[k].node  = (int)nid;
        hits[k].local = a;
        hits[k].n     = icei(rel * (float)M);
        k++;
    }
    qsort(hits, k, sizeof(hit_t), hit_cmp);
    return k;
}

/* Stratified sample j of a segment: HyperTree.cu:341-358, with the fused    */
/* multiply-adds the reference's nvcc build forms (contraction is on there):  */
/* t1 = fma(j, step, tmin), t2 = fma(j + 1, step, tmin),                      */
/* t = fma(t1, 1 - a, t2 * a).  This file is compiled with contraction off,   */
/* so every other operation rounds as written.                                */
static float seg_sample_t(float tmin, float step, int j, float a)
{
    float t1 = fmaf((float)j, step, tmin);
    float t2 = fmaf((float)(j + 1), step, tmin);
    return fmaf(t1, 1.0f - a, t2 * a);
}

static float jitter_a(int jitter, uint64_t seed, uint32_t step_id, int ray, int local_index)
{
    if (!jitter) return 0.5f;
    return oracle_uniform(seed, (uint32_t)ray, (uint32_t)local_index, step_id, NEAT_STREAM_JITTER);
}

/* Midpoint-interval weight of sample j: HyperTree.cu:372-389. */
static float seg_sample_w(float tmin, float tmax, float step, int n, int j, float tj, float tjm1, float tjp1)
{
    float lo = (j == 0) ? tmin : (tjm1 + tj) * 0.5f;
    float hi = (j == n - 1) ? tmax : (tjp1 + tj) * 0.5f;
    (void)step;
    return hi - lo;
}

/* ------------------------------------------------------------------------ */
/* CreateSamplesForRays (src/structure/HyperTree.cu:393-438) with canonical  */
/* ordering.  Outputs a SampleList (src/structure/HelperStructs.h:168-234):   */
/* coords [S,3], ray_t, weight, ray_index, local_index_in_ray, node_id.      */
/* Positions are recomputed as o + d*t (HyperTree.cu:426-432).               */
/* Returns S, or -1 on capacity overflow / -2 on >max_hits per ray.          */
/* ------------------------------------------------------------------------ */
long oracle_create_samples(int R, const float* o, const float* d, int A, const long* active_ids, const float* pmin,
                           const float* pmax, int M, int jitter, uint64_t seed, uint32_t step_id, long cap,
                           float* coords, float* ray_t, float* weight, long* ray_index, long* local_index,
                           long* node_id, int* max_per_ray, long* needed)
{
    /* pass 1: samples per ray (parallel over rays) */
    long* off = (long*)malloc(sizeof(long) * ((size_t)R + 1));
    int bad   = 0;
#pragma omp parallel
    {
        hit_t* hits = (hit_t*)malloc(sizeof(hit_t) * 256);
#pragma omp for schedule(dynamic, 64)
        for (int r = 0; r < R; ++r)
        {
            int k = ray_hits(o + 3 * r, d + 3 * r, A, active_ids, pmin, pmax, M, hits, 256);
            long n = 0;
            if (k < 0)
            {
#pragma omp atomic write
                bad = 1;
                k = 0;
            }
            for (int h = 0; h < k; ++h) n += hits[h].n;
            off[r + 1] = n;
        }
        free(hits);
    }
    if (bad)
    {
        free(off);
        return -2;
    }
    off[0] = 0;
    int mx = 0;
    for (int r = 0; r < R; ++r)
    {
        if (off[r + 1] > mx) mx = (int)off[r + 1];
        off[r + 1] += off[r];
    }
    long S = off[R];
    if (needed) *needed = S;
    if (S > cap)
    {
        free(off);
        return -1;
    }
    /* pass 2: write (parallel over rays) */
#pragma omp parallel
    {
        hit_t* hits = (hit_t*)malloc(sizeof(hit_t) * 256);
#pragma omp for schedule(dynamic, 64)
        for (int r = 0; r < R; ++r)
        {
            const float* orr = o + 3 * r;
            const float* dr  = d + 3 * r;
            int k            = ray_hits(orr, dr, A, active_ids, pmin, pmax, M, hits, 256);
            long base        = off[r];
            int local        = 0;
            for (int h = 0; h < k; ++h)
            {
                int n      = hits[h].n;
                float dis  = hits[h].tmax - hits[h].tmin;
                float step = dis / (float)n;
                for (int j = 0; j < n; ++j)
                {
                    float tj   = seg_sample_t(hits[h].tmin, step, j, jitter_a(jitter, seed, step_id, r, local + j));
                    float tjm1 = (j > 0) ? seg_sample_t(hits[h].tmin, step, j - 1,
                                                        jitter_a(jitter, seed, step_id, r, local + j - 1)) : 0;
                    float tjp1 = (j < n - 1) ? seg_sample_t(hits[h].tmin, step, j + 1,
                                                            jitter_a(jitter, seed, step_id, r, local + j + 1)) : 0;
                    long s     = base + local + j;
                    ray_t[s]   = tj;
                    weight[s]  = seg_sample_w(hits[h].tmin, hits[h].tmax, step, n, j, tj, tjm1, tjp1);
                    for (int c = 0; c < 3; ++c) coords[3 * s + c] = orr[c] + dr[c] * tj;
                    ray_index[s]   = r;
                    local_index[s] = local + j;
                    node_id[s]     = hits[h].node;
                }
                local += n;
            }
        }
        free(hits);
    }
    if (max_per_ray) *max_per_ray = mx;
    free(off);
    return S;
}

/* Line integrals for a list of pixels (x, y) of images img: the same rays as
 * oracle_project, for batches sampled on the host. */
void oracle_project_pixels(const double* obj, int n_obj, long n, const int* img, const int* px, const int* py,
                           const double* intr, const double* rot, const double* trans, float* out);

/* Segment lists only (the unit the fused training step works on):            */
/* per ray, hits in canonical order.  seg_* arrays have capacity cap.         */
/* Returns the segment count, -1 on overflow, -2 on >256 hits in one ray.    */
long oracle_ray_segments(int R, const float* o, const float* d, int A, const long* active_ids, const float* pmin,
                         const float* pmax, int M, long cap, int* seg_ray, int* seg_node, int* seg_local,
                         float* seg_tmin, float* seg_tmax, int* seg_n, int* ray_nseg)
{
    hit_t* hits = (hit_t*)malloc(sizeof(hit_t) * 256);
    long ns     = 0;
    for (int r = 0; r < R; ++r)
    {
        int k = ray_hits(o + 3 * r, d + 3 * r, A, active_ids, pmin, pmax, M, hits, 256);
        if (k < 0)
        {
            free(hits);
            return -2;
        }
        if (ns + k > cap)
        {
            free(hits);
            return -1;
        }
        for (int h = 0; h < k; ++h)
        {
            seg_ray[ns]   = r;
            seg_node[ns]  = hits[h].node;
            seg_local[ns] = hits[h].local;
            seg_tmin[ns]  = hits[h].tmin;
            seg_tmax[ns]  = hits[h].tmax;
            seg_n[ns]     = hits[h].n;
            ns++;
        }
        ray_nseg[r] = k;
    }
    free(hits);
    return ns;
}

/* ------------------------------------------------------------------------ */
/* ComputeLocalSamples (torch path, src/structure/HyperTree.cu:177-192):     */
/* local = (g - min) / (max - min) * 2 - 1, each op rounded separately.      */
/* ------------------------------------------------------------------------ */
void oracle_local_samples(long S, const float* g, const long* node_id, const float* pmin, const float* pmax,
                          float* out)
{
    for (long s = 0; s < S; ++s)
    {
        long n = node_id[s];
        for (int c = 0; c < 3; ++c)
        {
            float size = pmax[3 * n + c] - pmin[3 * n + c];
            float v    = g[3 * s + c] - pmin[3 * n + c];
            v          = v / size;
            v          = v * 2.0f;
            out[3 * s + c] = v - 1.0f;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* IndirectGridSample3D forward, reference CPU path                          */
/* src/modules/IndirectGridSample3D.cu:27-191.  grid [N,C,Z,Y,X] contiguous. */
/* Corner weights from unclamped corners, corner indices clamped to the      */
/* grid; accumulation order tnw,tne,tsw,tse,bnw,bne,bsw,bse, each term as an  */
/* fma (the contraction nvcc applies to the reference kernel, :556-569).       */
/* ------------------------------------------------------------------------ */
typedef struct
{
    int ix, iy, iz;             /* tnw corner (unclamped) */
    float fx, fy, fz;           /* scaled coordinates */
    float w[8];                 /* tnw tne tsw tse bnw bne bsw bse */
    int cx[2], cy[2], cz[2];    /* clamped corner indices (lo, hi) */
} igs_corner_t;

static int clampi(int v, int n) { return v < 0 ? 0 : (v > n - 1 ? n - 1 : v); }

static void igs_setup(const float* uv, int Z, int Y, int X, igs_corner_t* k)
{
    float ix = uv[0], iy = uv[1], iz = uv[2];
    ix = ((ix + 1) / 2) * (float)(X - 1);
    iy = ((iy + 1) / 2) * (float)(Y - 1);
    iz = ((iz + 1) / 2) * (float)(Z - 1);
    int x0 = (int)floorf(ix), y0 = (int)floorf(iy), z0 = (int)floorf(iz);
    int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    k->ix = x0; k->iy = y0; k->iz = z0;
    k->fx = ix; k->fy = iy; k->fz = iz;
    k->w[0] = ((float)x1 - ix) * ((float)y1 - iy) * ((float)z1 - iz); /* tnw */
    k->w[1] = (ix - (float)x0) * ((float)y1 - iy) * ((float)z1 - iz); /* tne */
    k->w[2] = ((float)x1 - ix) * (iy - (float)y0) * ((float)z1 - iz); /* tsw */
    k->w[3] = (ix - (float)x0) * (iy - (float)y0) * ((float)z1 - iz); /* tse */
    k->w[4] = ((float)x1 - ix) * ((float)y1 - iy) * (iz - (float)z0); /* bnw */
    k->w[5] = (ix - (float)x0) * ((float)y1 - iy) * (iz - (float)z0); /* bne */
    k->w[6] = ((float)x1 - ix) * (iy - (float)y0) * (iz - (float)z0); /* bsw */
    k->w[7] = (ix - (float)x0) * (iy - (float)y0) * (iz - (float)z0); /* bse */
    k->cx[0] = clampi(x0, X); k->cx[1] = clampi(x1, X);
    k->cy[0] = clampi(y0, Y); k->cy[1] = clampi(y1, Y);
    k->cz[0] = clampi(z0, Z); k->cz[1] = clampi(z1, Z);
}

/* corner c (0..7): x-bit = c&1, y-bit = (c>>1)&1, z-bit = (c>>2)&1 */
static long igs_off(const igs_corner_t* k, int c, int Y, int X)
{
    return ((long)k->cz[(c >> 2) & 1] * Y + k->cy[(c >> 1) & 1]) * X + k->cx[c & 1];
}

void oracle_igs_forward(const float* grid, long N, int C, int Z, int Y, int X, const long* index, const float* uv,
                        long S, float* out)
{
    (void)N;
    long G3 = (long)Z * Y * X;
    for (long i = 0; i < S; ++i)
    {
        igs_corner_t k;
        igs_setup(uv + 3 * i, Z, Y, X, &k);
        const float* g = grid + index[i] * (long)C * G3;
        for (int c = 0; c < C; ++c)
        {
            float acc = 0;
            for (int q = 0; q < 8; ++q) acc = fmaf(g[c * G3 + igs_off(&k, q, Y, X)], k.w[q], acc);
            out[i * C + c] = acc;
        }
    }
}

/* IGS backward, reference CPU path src/modules/IndirectGridSample3D.cu:194-429.
 * The per-term accumulations are written as the fused multiply-add that nvcc
 * emits for the reference CUDA kernel (IndirectGridSample3D.cu:740-770). */
void oracle_igs_backward(const float* grid, long N, int C, int Z, int Y, int X, const long* index, const float* uv,
                         long S, const float* grad_out, float* grad_grid, float* grad_uv)
{
    (void)N;
    long G3 = (long)Z * Y * X;
    for (long i = 0; i < S; ++i)
    {
        igs_corner_t k;
        igs_setup(uv + 3 * i, Z, Y, X, &k);
        const float* g = grid + index[i] * (long)C * G3;
        float* gg      = grad_grid + index[i] * (long)C * G3;
        float ix = k.fx, iy = k.fy, iz = k.fz;
        float x0 = (float)k.ix, y0 = (float)k.iy, z0 = (float)k.iz;
        float x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
        float gix = 0, giy = 0, giz = 0;
        for (int c = 0; c < C; ++c)
        {
            float go = grad_out[i * C + c];
            for (int q = 0; q < 8; ++q) gg[c * G3 + igs_off(&k, q, Y, X)] += k.w[q] * go;
            float v[8];
            for (int q = 0; q < 8; ++q) v[q] = g[c * G3 + igs_off(&k, q, Y, X)];
            float m1 = -1;
            gix = fmaf(m1 * v[0] * (y1 - iy) * (z1 - iz), go, gix);
            gix = fmaf(v[1] * (y1 - iy) * (z1 - iz), go, gix);
            gix = fmaf(m1 * v[2] * (iy - y0) * (z1 - iz), go, gix);
            gix = fmaf(v[3] * (iy - y0) * (z1 - iz), go, gix);
            gix = fmaf(m1 * v[4] * (y1 - iy) * (iz - z0), go, gix);
            gix = fmaf(v[5] * (y1 - iy) * (iz - z0), go, gix);
            gix = fmaf(m1 * v[6] * (iy - y0) * (iz - z0), go, gix);
            gix = fmaf(v[7] * (iy - y0) * (iz - z0), go, gix);

            giy = fmaf(m1 * v[0] * (x1 - ix) * (z1 - iz), go, giy);
            giy = fmaf(m1 * v[1] * (ix - x0) * (z1 - iz), go, giy);
            giy = fmaf(v[2] * (x1 - ix) * (z1 - iz), go, giy);
            giy = fmaf(v[3] * (ix - x0) * (z1 - iz), go, giy);
            giy = fmaf(m1 * v[4] * (x1 - ix) * (iz - z0), go, giy);
            giy = fmaf(m1 * v[5] * (ix - x0) * (iz - z0), go, giy);
            giy = fmaf(v[6] * (x1 - ix) * (iz - z0), go, giy);
            giy = fmaf(v[7] * (ix - x0) * (iz - z0), go, giy);

            giz = fmaf(m1 * v[0] * (x1 - ix) * (y1 - iy), go, giz);
            giz = fmaf(m1 * v[1] * (ix - x0) * (y1 - iy), go, giz);
            giz = fmaf(m1 * v[2] * (x1 - ix) * (iy - y0), go, giz);
            giz = fmaf(m1 * v[3] * (ix - x0) * (iy - y0), go, giz);
            giz = fmaf(v[4] * (x1 - ix) * (y1 - iy), go, giz);
            giz = fmaf(v[5] * (ix - x0) * (y1 - iy), go, giz);
            giz = fmaf(v[6] * (x1 - ix) * (iy - y0), go, giz);
            giz = fmaf(v[7] * (ix - x0) * (iy - y0), go, giz);
        }
        gix = gix * (float)(X - 1) / 2;
        giy = giy * (float)(Y - 1) / 2;
        giz = giz * (float)(Z - 1) / 2;
        grad_uv[3 * i + 0] += gix;
        grad_uv[3 * i + 1] += giy;
        grad_uv[3 * i + 2] += giz;
    }
}

/* ------------------------------------------------------------------------ */
/* Synthetic phantom (stands in for the reference's measured scans).         */
/* obj: [n_obj, 17] doubles = centre(3), semi-axes(3), rotation R(9,        */
/* row-major, local = R^T (p - c)), density, kind: 0 additive ellipsoid,     */
/* 1 override ellipsoid (inside, the density is the object's own: 0 for a    */
/* void), 2 additive cylinder along the local z axis (radii = semi-axes x,   */
/* y; half-height = semi-axis z).  Override objects with a non-zero density  */
/* must not overlap one another.                                             */
/* ------------------------------------------------------------------------ */
#define OBJ_STRIDE 17
#define FAR_T 1e300

static void object_local(const double* ob, const double* o, const double* d, double* q, double* e)
{
    double p[3] = {o[0] - ob[0], o[1] - ob[1], o[2] - ob[2]};
    const double* Rm = ob + 6;
    for (int i = 0; i < 3; ++i)
    {
        /* local_i = sum_j R[j][i] * p_j  (R^T p) */
        double lq = Rm[0 * 3 + i] * p[0] + Rm[1 * 3 + i] * p[1] + Rm[2 * 3 + i] * p[2];
        double le = Rm[0 * 3 + i] * d[0] + Rm[1 * 3 + i] * d[1] + Rm[2 * 3 + i] * d[2];
        q[i]      = lq / ob[3 + i];
        e[i]      = le / ob[3 + i];
    }
}

static int ellipsoid_chord(const double* ob, const double* o, const double* d, double* t0, double* t1)
{
    double q[3], e[3];
    object_local(ob, o, d, q, e);
    double A = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    double B = q[0] * e[0] + q[1] * e[1] + q[2] * e[2];
    double C = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] - 1.0;
    double disc = B * B - A * C;
    if (disc <= 0 || A <= 0) return 0;
    double sq = sqrt(disc);
    *t0 = (-B - sq) / A;
    *t1 = (-B + sq) / A;
    return 1;
}

/* The ray's interval inside x^2 + y^2 <= 1 (scaled local frame), intersected */
/* with the slab |z| <= 1.                                                    */
static int cylinder_chord(const double* ob, const double* o, const double* d, double* t0, double* t1)
{
    double q[3], e[3];
    object_local(ob, o, d, q, e);
    double a0 = -FAR_T, a1 = FAR_T;
    double A = e[0] * e[0] + e[1] * e[1];
    double B = q[0] * e[0] + q[1] * e[1];
    double C = q[0] * q[0] + q[1] * q[1] - 1.0;
    if (A > 0)
    {
        double disc = B * B - A * C;
        if (disc <= 0) return 0;
        double sq = sqrt(disc);
        a0 = (-B - sq) / A;
        a1 = (-B + sq) / A;
    }
    else if (C > 0)
        return 0;
    double z0 = -FAR_T, z1 = FAR_T;
    if (e[2] != 0)
    {
        z0 = (-1.0 - q[2]) / e[2];
        z1 = (1.0 - q[2]) / e[2];
        if (z0 > z1)
        {
            double t = z0;
            z0 = z1;
            z1 = t;
        }
    }
    else if (q[2] < -1.0 || q[2] > 1.0)
        return 0;
    *t0 = a0 > z0 ? a0 : z0;
    *t1 = a1 < z1 ? a1 : z1;
    return *t1 > *t0;
}

static int object_chord(const double* ob, const double* o, const double* d, double* t0, double* t1)
{
    return ob[16] == 2.0 ? cylinder_chord(ob, o, d, t0, t1) : ellipsoid_chord(ob, o, d, t0, t1);
}

static int dcmp(const void* a, const void* b)
{
    double x = *(const double*)a, y = *(const double*)b;
    return (x < y) ? -1 : (x > y);
}

/* Line integral of the phantom density along o + t d (|d| = 1), t in R:     */
/* each override object adds density x chord; additive objects add density  */
/* x (chord minus the union of the override intervals).                      */
double oracle_phantom_line(const double* obj, int n_obj, const double* o, const double* d)
{
    double vi[2 * 512];
    int nv = 0;
    double total = 0;
    for (int k = 0; k < n_obj; ++k)
    {
        const double* ob = obj + OBJ_STRIDE * k;
        if (ob[16] != 1.0) continue;
        double t0, t1;
        if (ellipsoid_chord(ob, o, d, &t0, &t1) && nv < 512)
        {
            if (ob[15] != 0.0) total += ob[15] * (t1 - t0);
            vi[2 * nv]     = t0;
            vi[2 * nv + 1] = t1;
            nv++;
        }
    }
    /* merge override intervals (sorted by start) */
    qsort(vi, nv, 2 * sizeof(double), dcmp);
    int m = 0;
    for (int k = 0; k < nv; ++k)
    {
        if (m > 0 && vi[2 * k] <= vi[2 * (m - 1) + 1])
        {
            if (vi[2 * k + 1] > vi[2 * (m - 1) + 1]) vi[2 * (m - 1) + 1] = vi[2 * k + 1];
        }
        else
        {
            vi[2 * m]     = vi[2 * k];
            vi[2 * m + 1] = vi[2 * k + 1];
            m++;
        }
    }
    for (int k = 0; k < n_obj; ++k)
    {
        const double* ob = obj + OBJ_STRIDE * k;
        if (ob[16] != 0.0 && ob[16] != 2.0) continue;
        double t0, t1;
        if (!object_chord(ob, o, d, &t0, &t1)) continue;
        double len = t1 - t0;
        for (int v = 0; v < m; ++v)
        {
            double a = vi[2 * v] > t0 ? vi[2 * v] : t0;
            double b = vi[2 * v + 1] < t1 ? vi[2 * v + 1] : t1;
            if (b > a) len -= (b - a);
        }
        total += ob[15] * len;
    }
    return total;
}

/* Density of the phantom at a point: the sum of the additive objects that   */
/* contain it, or the density of the first override object that does.        */
double oracle_phantom_density(const double* obj, int n_obj, const double* p)
{
    double rho = 0;
    for (int k = 0; k < n_obj; ++k)
    {
        const double* ob = obj + OBJ_STRIDE * k;
        const double* Rm = ob + 6;
        double l[3];
        for (int i = 0; i < 3; ++i)
        {
            l[i] = Rm[0 * 3 + i] * (p[0] - ob[0]) + Rm[1 * 3 + i] * (p[1] - ob[1]) + Rm[2 * 3 + i] * (p[2] - ob[2]);
            l[i] = l[i] / ob[3 + i];
        }
        int inside = ob[16] == 2.0 ? (l[0] * l[0] + l[1] * l[1] <= 1.0 && l[2] * l[2] <= 1.0)
                                   : ((l[0] * l[0] + l[1] * l[1]) + l[2] * l[2] <= 1.0);
        if (inside)
        {
            if (ob[16] == 1.0) return ob[15];
            rho += ob[15];
        }
    }
    return rho;
}

/* Projection image [n_img, h, w]: the line integral for the ray through     */
/* each pixel centre, generated with the same f64 camera model as            */
/* oracle_make_ray but without the float cast of the direction.              */
void oracle_project(const double* obj, int n_obj, int n_img, int w, int h, const double* intr, const double* rot,
                    const double* trans, float* out)
{
#pragma omp parallel for schedule(dynamic, 4)
    for (long p = 0; p < (long)n_img * h; ++p)
    {
        int img = (int)(p / h), y = (int)(p % h);
        for (int x = 0; x < w; ++x)
        {
            double cx = ((double)x - intr[2]) / intr[0];
            double cy = ((double)y - intr[3]) / intr[1];
            double cz = 1.0;
            double n  = sqrt((cx * cx + cy * cy) + cz * cz);
            cx /= n; cy /= n; cz /= n;
            const double* q = rot + 4 * img;
            double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
            double ux = qy * cz - qz * cy, uy = qz * cx - qx * cz, uz = qx * cy - qy * cx;
            ux += ux; uy += uy; uz += uz;
            double d[3] = {(cx + qw * ux) + (qy * uz - qz * uy), (cy + qw * uy) + (qz * ux - qx * uz),
                           (cz + qw * uz) + (qx * uy - qy * ux)};
            out[p * w + x] = (float)oracle_phantom_line(obj, n_obj, trans + 3 * img, d);
        }
    }
}

void oracle_project_pixels(const double* obj, int n_obj, long n, const int* img, const int* px, const int* py,
                           const double* intr, const double* rot, const double* trans, float* out)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < n; ++i)
    {
        double cx = ((double)px[i] - intr[2]) / intr[0];
        double cy = ((double)py[i] - intr[3]) / intr[1];
        double cz = 1.0;
        double nn = sqrt((cx * cx + cy * cy) + cz * cz);
        cx /= nn; cy /= nn; cz /= nn;
        const double* q = rot + 4 * img[i];
        double qx = q[0], qy = q[1], qz = q[2], qw = q[3];
        double ux = qy * cz - qz * cy, uy = qz * cx - qx * cz, uz = qx * cy - qy * cx;
        ux += ux; uy += uy; uz += uz;
        double d[3] = {(cx + qw * ux) + (qy * uz - qz * uy), (cy + qw * uy) + (qz * ux - qx * uz),
                       (cz + qw * uz) + (qx * uy - qy * ux)};
        out[i] = (float)oracle_phantom_line(obj, n_obj, trans + 3 * img[i], d);
    }
}

/* Density at many points (parallel). */
void oracle_phantom_density_batch(const double* obj, int n_obj, long n, const double* pts, double* out)
{
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) out[i] = oracle_phantom_density(obj, n_obj, pts + 3 * i);
}
