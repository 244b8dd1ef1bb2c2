// Grid scatter model (sysmat_scatter_grid): primary Compton scatter at points on a grid of
// cells inside every crystal and inside the tungsten of every collimator layer.  No reference
// counterpart: the reference scatters at one point per crystal (its centre) and one per
// layer-0 hole (ScatterGen_RayTracing_CircularHole/scatter.cu:1218-1223, :1707-1716).  The
// model's definition, restated in double, is oracle/oracle_grid.h:
//
//   S[d, v] = sum_{crystal cells p} w_p T(p, d, v) + sum_{septal cells p} w_p T(p, d, v)
//
// w_p: a crystal cell's photoelectric contribution from v (the local-coordinate FP32 element
// with the crystal divided into cells) times mu_C / mu_pe; a septal cell's Compton
// interaction probability V / (4 pi r^2) exp(-A(v -> p)) mu_C (in double).  T: the
// reference's scatter item with scatter point p, all crystals on the way as attenuators and the
// exact Klein-Nishina fraction.
//
// Execution (per call, voxels taken 48 at a time):
//   1. crystal-cell weights: the local sampled photoelectric kernel writes every sub-element's
//      contribution (pe_local.cuh) into Wc[voxel][crystal][cell];
//   2. septal-cell weights: one thread per (voxel, septal cell), in double, into Ws;
//   3. grid_sum_kernel: a block takes a tile of 64 detectors and a range of points; per chunk
//      of 256 points it stages the weights of all the chunk's voxels in shared memory, and per
//      detector it forms each point's detector-only terms in double once (position in the
//      detector's frame, absorption chord, attenuation sums of the crystals, tungsten and hole
//      media on the way, Lpe and Lc, so that the attenuation at any scattered energy E' is
//      Lpe (E0/E')^3 + Lc E0/E'), then evaluates the voxel-dependent part of every item in
//      float and sums per (detector, voxel) in FP64: warp sums, a shared tile of block sums,
//      one double atomic per (detector, voxel) and block.
// Calls are synchronous: the weights live in scratch allocated and freed by the call.
#include <cmath>
#include <cstdio>
#include <vector>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "../../include/sysmat.h"
#include "chord64.cuh"
#include "ctx.cuh"
#include "geom.cuh"
#include "pe.cuh"
#include "scatter.cuh"

#define CUDA_TRY(expr)                                                                     \
    do {                                                                                   \
        cudaError_t _e = (expr);                                                           \
        if (_e != cudaSuccess) {                                                           \
            std::fprintf(stderr, "sysmat: %s failed: %s (%s:%d)\n", #expr,                 \
                         cudaGetErrorString(_e), __FILE__, __LINE__);                      \
            return SYSMAT_ERR_CUDA;                                                        \
        }                                                                                  \
    } while (0)

namespace sysmat {

namespace {

constexpr int kGridThreads = 256;
constexpr int kGridChunk = 256;          // points per chunk (one per thread)
constexpr int kGridMaxVox = 48;          // voxels per pass
constexpr int kGridDetTile = 64;         // detectors per block
constexpr int kGridChunksPerBlock = 8;


// Septal cells are numbered brick by brick (bricks of 8 x 4 x 8 cells, x fastest inside a brick
// and among bricks), so that a chunk of consecutive septal cells is a compact region: the
// chunk's candidate holes and crystals (those near the segments from its points to a detector
// or a voxel) are then found once per chunk.
constexpr int kBrickX = 8, kBrickY = 4, kBrickZ = 8, kBrickCells = kBrickX * kBrickY * kBrickZ;

struct GridLayer {
    double x0, y0, z0;                   // plate box corner
    double cx, cy, cz;                   // cell size
    int nx, ny, nz;
    int nbx, nby, nbz;                   // bricks per axis
    int hole_begin, hole_count;
    float mu_t, mu_pe, mu_c;
};

struct GridGeom {
    int n_layers;
    GridLayer layer[kMaxLayers];
    long long sep_begin[kMaxLayers + 1];   // septal cells of layer m: [sep_begin[m], sep_begin[m+1])
    const int* sep_cell;                   // brick-ordered cell index within its layer (cell_of)
    const float* raw_col;                  // collimator parameters (hole media)
};

__device__ __forceinline__ void atomicMin_float(float* a, float v)
{
    v += 0.0f;                           // -0 -> +0: the integer orders below need one zero
    if (v >= 0.0f) atomicMin((int*)a, __float_as_int(v));
    else atomicMax((unsigned int*)a, __float_as_uint(v));
}

__device__ __forceinline__ void atomicMax_float(float* a, float v)
{
    v += 0.0f;
    if (v >= 0.0f) atomicMax((int*)a, __float_as_int(v));
    else atomicMin((unsigned int*)a, __float_as_uint(v));
}

__device__ __forceinline__ void voxel_centre64(const DevGeom& g, long long v, float rotation, double& x, double& y,
                                               double& z)
{
    const long long nxy = (long long)g.nx * g.ny;
    const int iz = (int)(v / nxy);
    const long long r = v - (long long)iz * nxy;
    const int iy = (int)(r / g.nx);
    const int ix = (int)(r - (long long)iy * g.nx);
    const double ang = (double)rotation * (double)g.angle_step;
    double sa, ca;
    sincos(ang, &sa, &ca);
    double xv = ((double)ix - (double)g.nx / 2.0 + 0.5) * (double)g.wx + (double)g.shx;
    double yv = ((double)iy - (double)g.ny / 2.0 + 0.5) * (double)g.wy + (double)g.shy;
    x = xv * ca - yv * sa;
    y = xv * sa + yv * ca;
    z = ((double)iz - (double)g.nz / 2.0 + 0.5) * (double)g.wz + (double)g.shz;
}

// Cell (ix, iy, iz) of brick-ordered index c of layer L (cells of a partial brick past the
// plate's edge have ix >= nx, iy >= ny or iz >= nz).
__device__ __forceinline__ void cell_of(const GridLayer& L, int c, int& ix, int& iy, int& iz)
{
    const int b = c / kBrickCells, w = c - b * kBrickCells;
    const int bx = b % L.nbx, by = (b / L.nbx) % L.nby, bz = b / (L.nbx * L.nby);
    ix = bx * kBrickX + (w % kBrickX);
    iy = by * kBrickY + (w / kBrickX) % kBrickY;
    iz = bz * kBrickZ + w / (kBrickX * kBrickY);
}

__device__ __forceinline__ void septal_point(const GridGeom& G, long long j, int& m, double p[3])
{
    m = 0;
    while (m + 1 < G.n_layers && j >= G.sep_begin[m + 1]) ++m;
    const GridLayer& L = G.layer[m];
    int ix, iy, iz;
    cell_of(L, __ldg(&G.sep_cell[j]), ix, iy, iz);
    p[0] = L.x0 + ((double)ix + 0.5) * L.cx;
    p[1] = L.y0 + ((double)iy + 0.5) * L.cy;
    p[2] = L.z0 + ((double)iz + 0.5) * L.cz;
}

// Candidate lists of a chunk of points (block shared memory): the crystals and, per layer, the
// holes that may lie on a segment from one of the chunk's points to a common far end.  A list
// longer than its capacity is not used (n = -1: scan everything).
constexpr int kCandCry = 1024, kCandHole = 2048;

struct Cands {
    int n_cry;
    int hole_off[kMaxLayers + 1];        // holes of layer m: hole[hole_off[m] .. hole_off[m+1]); -1 = all
    int cry[kCandCry];
    int hole[kCandHole];
    int warp_cnt[kGridThreads / 32];
    float lo[3], hi[3];                  // the chunk's bounding box
};

// Ordered compaction over the block of the items i in [0, n) with keep(i) into list[off ..]
// (capacity cap); returns the number kept, or -1 past the capacity.
template <class F>
__device__ int block_select(int n, F keep, int* list, int off, int cap, int* warp_cnt)
{
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int total = 0;
    for (int base = 0; base < n; base += kGridThreads) {
        const int i = base + t;
        const bool k = i < n && keep(i);
        const unsigned m = __ballot_sync(0xffffffffu, k);
        if (lane == 0) warp_cnt[warp] = __popc(m);
        __syncthreads();
        int before = 0, all = 0;
        for (int w = 0; w < kGridThreads / 32; ++w) {
            const int c = warp_cnt[w];
            if (w < warp) before += c;
            all += c;
        }
        const int pos = total + before + __popc(m & ((1u << lane) - 1u));
        if (k && pos < cap) list[off + pos] = i;
        total += all;
        __syncthreads();
    }
    return total <= cap ? total : -1;
}

// Bounding box of the block's points (threads without a point pass has = false).
__device__ void block_bounds(Cands& C, bool has, const double p[3])
{
    const int t = threadIdx.x;
    if (t < 3) { C.lo[t] = INFINITY; C.hi[t] = -INFINITY; }
    __syncthreads();
    if (has) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            atomicMin_float(&C.lo[a], (float)p[a]);
            atomicMax_float(&C.hi[a], (float)p[a]);
        }
    }
    __syncthreads();
}

// Candidates for segments from the chunk's points to E (far end): crystals (bounding spheres)
// when cry, and the holes of every layer when holes.  A point within r_c of the box centre c
// has its segment within r_c of the segment c -> E, so the tests widen by r_c.
__device__ void chunk_candidates(const DevGeom& g, const GridGeom& G, Cands& C, const double E[3], bool cry,
                                 bool holes)
{
    const float cx = 0.5f * (C.lo[0] + C.hi[0]), cy = 0.5f * (C.lo[1] + C.hi[1]), cz = 0.5f * (C.lo[2] + C.hi[2]);
    const float rc = 0.5f * sqrtf((C.hi[0] - C.lo[0]) * (C.hi[0] - C.lo[0]) + (C.hi[1] - C.lo[1]) * (C.hi[1] - C.lo[1]) +
                                  (C.hi[2] - C.lo[2]) * (C.hi[2] - C.lo[2])) + 2e-3f;
    const float ex = (float)E[0], ey = (float)E[1], ez = (float)E[2];
    const float gx = ex - cx, gy = ey - cy, gz = ez - cz;
    const float gl2 = gx * gx + gy * gy + gz * gz;
    if (cry) {
        const int n = block_select(g.n_det, [&](int a) {
            const float4 pa = __ldg(&g.cry.pos[a]);
            const float ra = 0.5f * __ldg(&g.cry.size[a].w) + 1e-3f + rc;
            const float hx = pa.x - cx, hy = pa.y - cy, hz = pa.z - cz;
            float u = gl2 > 0.0f ? (hx * gx + hy * gy + hz * gz) / gl2 : 0.0f;
            u = fminf(fmaxf(u, 0.0f), 1.0f);
            const float qx = hx - u * gx, qy = hy - u * gy, qz = hz - u * gz;
            return qx * qx + qy * qy + qz * qz <= ra * ra;
        }, C.cry, 0, kCandCry, C.warp_cnt);
        if (threadIdx.x == 0) C.n_cry = n;
    }
    if (holes) {
        int off = 0;
        for (int m = 0; m < G.n_layers; ++m) {
            const GridLayer& L = G.layer[m];
            int n = -1;
            if (off >= 0)
                n = block_select(L.hole_count, [&](int j) {
                    const float4 ha = __ldg(&g.hole.a[L.hole_begin + j]);
                    const float r = __ldg(&g.hole.b[L.hole_begin + j].x) + rc + 1e-3f;
                    const float hx = ha.x - cx, hz = ha.w - cz;
                    const float l2 = gx * gx + gz * gz;
                    float u = l2 > 0.0f ? (hx * gx + hz * gz) / l2 : 0.0f;
                    u = fminf(fmaxf(u, 0.0f), 1.0f);
                    const float qx = hx - u * gx, qz = hz - u * gz;
                    return qx * qx + qz * qz <= r * r;
                }, C.hole, off, kCandHole - off, C.warp_cnt);
            if (threadIdx.x == 0) C.hole_off[m] = off < 0 || n < 0 ? -1 : off;
            off = off < 0 || n < 0 ? -1 : off + n;
        }
        if (threadIdx.x == 0) C.hole_off[G.n_layers] = off;
    }
    __syncthreads();
}

// Hole h's axis (x, z) is farther than r from the xz projection of segment a -> b (with a
// small margin): the segment cannot meet the hole.
__device__ __forceinline__ bool hole_far(double ax, double az, double bx, double bz, double hx, double hz, double r)
{
    const double ex = bx - ax, ez = bz - az;
    const double l2 = ex * ex + ez * ez;
    double t = l2 > 0.0 ? ((hx - ax) * ex + (hz - az) * ez) / l2 : 0.0;
    t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
    const double dx = ax + t * ex - hx, dz = az + t * ez - hz;
    return dx * dx + dz * dz > (r + 1e-6) * (r + 1e-6);
}

// Length of segment A -> B inside the box [lo, hi]: the exact overlap of the segment's
// parameter range with the three slabs.  The grid model's paths start or end inside the plate
// or a crystal, where the reference's chords (full crossings between the two ends) do not apply.
__device__ double seg_box64(const double A[3], const double B[3], const double lo[3], const double hi[3])
{
    double t0 = 0.0, t1 = 1.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double d = B[a] - A[a];
        if (d == 0.0) {
            if (A[a] < lo[a] || A[a] > hi[a]) return 0.0;
            continue;
        }
        double u = (lo[a] - A[a]) / d, v = (hi[a] - A[a]) / d;
        if (u > v) { const double w = u; u = v; v = w; }
        t0 = fmax(t0, u);
        t1 = fmin(t1, v);
    }
    if (t1 <= t0) return 0.0;
    return (t1 - t0) * sqrt((B[0] - A[0]) * (B[0] - A[0]) + (B[1] - A[1]) * (B[1] - A[1]) + (B[2] - A[2]) * (B[2] - A[2]));
}

// Length of segment A -> B inside the y-parallel cylinder (x - xc)^2 + (z - zc)^2 <= r^2,
// y in [y1, y2] (exact overlap).  S: an elliptical hole's (rho_x, rho_z, cos, sin) (S.x > 0), in
// whose frame (u = dx cos + dz sin, w = -dx sin + dz cos, as the reference turns points),
// divided by the semi-axes, the segment meets the unit circle over the same parameter range.
__device__ double seg_cyl64(const double A[3], const double B[3], double xc, double zc, double y1, double y2, double r,
                            const D4& S)
{
    double t0 = 0.0, t1 = 1.0;
    const double dy = B[1] - A[1];
    if (dy == 0.0) {
        if (A[1] < y1 || A[1] > y2) return 0.0;
    } else {
        double u = (y1 - A[1]) / dy, v = (y2 - A[1]) / dy;
        if (u > v) { const double w = u; u = v; v = w; }
        t0 = fmax(t0, u);
        t1 = fmin(t1, v);
    }
    const double dx0 = B[0] - A[0], dz0 = B[2] - A[2];
    double dx = dx0, dz = dz0, ox = A[0] - xc, oz = A[2] - zc;
    if (S.x > 0.0) {
        const double pdx = (dx * S.z + dz * S.w) / S.x, pdz = (-dx * S.w + dz * S.z) / S.y;
        const double pox = (ox * S.z + oz * S.w) / S.x, poz = (-ox * S.w + oz * S.z) / S.y;
        dx = pdx; dz = pdz; ox = pox; oz = poz;
        r = 1.0;
    }
    const double a = dx * dx + dz * dz, b = ox * dx + oz * dz, c = ox * ox + oz * oz - r * r;
    if (a == 0.0) {
        if (c > 0.0) return 0.0;
    } else {
        const double disc = b * b - a * c;
        if (disc <= 0.0) return 0.0;
        const double sq = sqrt(disc);
        t0 = fmax(t0, (-b - sq) / a);
        t1 = fmin(t1, (-b + sq) / a);
    }
    if (t1 <= t0) return 0.0;
    return (t1 - t0) * sqrt(dx0 * dx0 + dz0 * dz0 + dy * dy);
}

// Attenuation sums (mu_total, mu_pe, mu_C times length) of layer m along segment A -> B: its
// length in the plate box minus its lengths in the layer's holes, with the layer's
// coefficients, plus its lengths in the holes with the holes' own coefficients.
__device__ void layer_path64(const DevGeom& g, const GridGeom& G, int m, const double A[3], const double B[3],
                             double& wt, double& wpe, double& wc, const Cands* C = nullptr)
{
    const double* Ly = g.t64.layer + kLayer64 * m;
    const double lo[3] = {Ly[0], Ly[2], Ly[4]}, hi[3] = {Ly[1], Ly[3], Ly[5]};
    const double box = seg_box64(A, B, lo, hi);
    if (box == 0.0) return;
    const GridLayer& L = G.layer[m];
    // candidate holes of the chunk (in hole order), or every hole of the layer
    const bool listed = C && C->hole_off[m] >= 0 && C->hole_off[m + 1] >= 0;
    const int n = listed ? C->hole_off[m + 1] - C->hole_off[m] : L.hole_count;
    double hsum = 0.0;
    for (int q = 0; q < n; ++q) {
        const int j = L.hole_begin + (listed ? C->hole[C->hole_off[m] + q] : q);
        const D4 a = g.t64.hole_a[j];
        const double r = g.t64.hole_b[j].x;
        if (hole_far(A[0], A[2], B[0], B[2], a.x, a.w, r)) continue;
        const D4 S = g.t64.hole_shape ? g.t64.hole_shape[j] : D4{0.0, 0.0, 1.0, 0.0};
        const double l = seg_cyl64(A, B, a.x, a.w, a.y, a.z, r, S);
        if (l == 0.0) continue;
        const float* hp = G.raw_col + 100 + 9 * j;
        hsum += l;
        wt += (double)__ldg(&hp[5]) * l;
        wpe += (double)__ldg(&hp[6]) * l;
        wc += (double)__ldg(&hp[7]) * l;
    }
    const double lw = box - hsum;
    if (lw > 0.0) {
        wt += (double)L.mu_t * lw;
        wpe += (double)L.mu_pe * lw;
        wc += (double)L.mu_c * lw;
    }
}

// Septal weight V / (4 pi r^2) exp(-A(v -> p)) mu_C for every (voxel, septal cell).
// Block (chunk of kGridThreads septal cells, voxel): the chunk's candidate holes for segments to
// the voxel are found once, then each thread forms its cell's weight.
__global__ void __launch_bounds__(kGridThreads) septal_weight_kernel(DevGeom g, GridGeom G, long long vox_begin,
                                                                     float rotation, long long n_sep,
                                                                     float* __restrict__ ws)
{
    __shared__ Cands C;
    const int vi = blockIdx.y;
    const long long j = (long long)blockIdx.x * kGridThreads + threadIdx.x;
    const bool has = j < n_sep;
    int m = 0;
    double p[3] = {0.0, 0.0, 0.0}, I3[3];
    if (has) septal_point(G, j, m, p);
    voxel_centre64(g, vox_begin + vi, rotation, I3[0], I3[1], I3[2]);
    block_bounds(C, has, p);
    chunk_candidates(g, G, C, I3, false, true);
    if (!has) return;
    double at = 0.0, ape = 0.0, ac = 0.0;
    for (int mm = 0; mm < G.n_layers; ++mm) layer_path64(g, G, mm, I3, p, at, ape, ac, &C);
    const GridLayer& L = G.layer[m];
    const double r2 = (p[0] - I3[0]) * (p[0] - I3[0]) + (p[1] - I3[1]) * (p[1] - I3[1]) + (p[2] - I3[2]) * (p[2] - I3[2]);
    const double vcell = L.cx * L.cy * L.cz;
    ws[(long long)vi * n_sep + j] = (float)(vcell / (4.0 * 3.14159265358979323846 * r2) * exp(-at) * (double)L.mu_c);
}

// Septal cells of layer m: cell centre outside every hole of the layer.
__global__ void septal_mark_kernel(DevGeom g, GridLayer L, int n_cells, unsigned char* __restrict__ flag)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    int ix, iy, iz;
    cell_of(L, c, ix, iy, iz);
    if (ix >= L.nx || iy >= L.ny || iz >= L.nz) {           // past the plate's edge
        flag[c] = 0;
        return;
    }
    const double x = L.x0 + ((double)ix + 0.5) * L.cx, y = L.y0 + ((double)iy + 0.5) * L.cy;
    const double z = L.z0 + ((double)iz + 0.5) * L.cz;
    unsigned char sep = 1;
    for (int j = L.hole_begin; j < L.hole_begin + L.hole_count && sep; ++j) {
        const D4 a = g.t64.hole_a[j];
        const double r = g.t64.hole_b[j].x;
        const double dx = x - a.x, dz = z - a.w;
        if (!(y >= a.y && y <= a.z)) continue;
        const D4 S = g.t64.hole_shape ? g.t64.hole_shape[j] : D4{0.0, 0.0, 1.0, 0.0};
        if (S.x > 0.0) {                                    // elliptical hole
            const double u = (dx * S.z + dz * S.w) / S.x, w = (-dx * S.w + dz * S.z) / S.y;
            if (u * u + w * w <= 1.0) sep = 0;
        } else if (dx * dx + dz * dz <= r * r) {
            sep = 0;
        }
    }
    flag[c] = sep;
}

struct GridSum {
    int det_begin, det_count;            // rows of this launch
    long long vox_begin;
    int nv;
    float rotation;
    int snx, sny, snz, n_sub;            // crystal cells
    long long n_cry_pts, n_pts;          // D * n_sub; + septal cells
    const float* wc;                     // [nv][D][n_sub]
    const float* ws;                     // [nv][n_sep]
    long long n_sep;
    double* acc;                         // [det_count][nv]
    float e0, lo, hi;
    int same_window;
    const double* kn_tab;
    double kn_total;
};

// Scatter point pidx: its position; k = its crystal (crystal cells) or -1, m = its layer (septal
// cells) or -1; conv = mu_C / mu_pe of its crystal (a crystal cell's weight is photoelectric).
__device__ void grid_point(const DevGeom& g, const GridGeom& G, const GridSum& S, long long pidx, double p[3], int& k,
                           int& m, double& conv)
{
    k = -1;
    m = -1;
    conv = 1.0;
    if (pidx < S.n_cry_pts) {
        k = (int)(pidx / S.n_sub);
        const int sidx = (int)(pidx - (long long)k * S.n_sub);
        const int nxy = S.snx * S.sny;
        const int iz = sidx / nxy, rem = sidx - iz * nxy, iy = rem / S.snx, ix = rem - iy * S.snx;
        const D4 P = g.t64.cry_pos[k], Z = g.t64.cry_size[k], T = g.t64.cry_trig[k];
        const double xDs = -Z.x / 2.0 + ((double)ix + 0.5) / (double)S.snx * Z.x;
        const double zDs = -Z.z / 2.0 + ((double)iz + 0.5) / (double)S.snz * Z.z;
        const double yDs = -Z.y / 2.0 + ((double)iy + 0.5) / (double)S.sny * Z.y;
        p[0] = P.x + (xDs * T.x - zDs * T.y);
        p[1] = P.y + yDs;
        p[2] = P.z + (xDs * T.y + zDs * T.x);
        const float4 mu = __ldg(&g.cry.mu[k]);
        conv = (double)mu.z / (double)mu.y;                   // photoelectric -> Compton weight
    } else {
        septal_point(G, pidx - S.n_cry_pts, m, p);
    }
}

// Detector-only terms of point p for detector d (double, rounded once): p in d's frame, the
// absorption chord of the extended ray p -> d's centre in d, and the attenuation sums Lpe, Lc
// of everything on the way (crystals other than d and the scattering crystal, and for septal
// points the tungsten and hole media), over the chunk's candidate crystals and holes C.
// Returns false when the point does not scatter into d.
__device__ bool point_terms(const DevGeom& g, const GridGeom& G, int d, const double p[3], int k, int m, double conv,
                            const Cands& C, float* out)
{
    if (k == d) return false;
    const D4 Pd = g.t64.cry_pos[d], Zd = g.t64.cry_size[d], Td = g.t64.cry_trig[d];
    const double D3[3] = {Pd.x, Pd.y, Pd.z};                  // centre of the 1 x 1 x 1 division
    const double ex = p[0] - Pd.x, ez = p[2] - Pd.z;
    const double ps[3] = {ex * Td.z - ez * Td.w, p[1] - Pd.y, ex * Td.w + ez * Td.z};
    const double lsd = sqrt(ps[0] * ps[0] + ps[1] * ps[1] + ps[2] * ps[2]);
    // absorption: the ray p -> centre extended 1000 mm through d (scatter.cu:1420-1424)
    const double labs = box_chord64(ps[0], ps[1], ps[2], -1000.0 * ps[0] / lsd, -1000.0 * ps[1] / lsd,
                                    -1000.0 * ps[2] / lsd, -0.5 * Zd.x, -0.5 * Zd.y, -0.5 * Zd.z, 0.5 * Zd.x,
                                    0.5 * Zd.y, 0.5 * Zd.z);
    double lpe = 0.0, lc = 0.0;
    // crystals on the way: bounding-sphere reject, then the reference box chord in double
    const float fx = (float)p[0], fy = (float)p[1], fz = (float)p[2];
    const float gx = (float)D3[0] - fx, gy = (float)D3[1] - fy, gz = (float)D3[2] - fz;
    const float gl2 = gx * gx + gy * gy + gz * gz;
    const int n_cry = C.n_cry >= 0 ? C.n_cry : g.n_det;
    for (int q = 0; q < n_cry; ++q) {
        const int a = C.n_cry >= 0 ? C.cry[q] : q;
        if (a == d || a == k) continue;
        const float4 pa = __ldg(&g.cry.pos[a]);
        const float ra = 0.5f * __ldg(&g.cry.size[a].w) + 1e-3f;
        const float hx = pa.x - fx, hy = pa.y - fy, hz = pa.z - fz;
        float t = (hx * gx + hy * gy + hz * gz) / gl2;
        t = fminf(fmaxf(t, 0.0f), 1.0f);
        const float qx = hx - t * gx, qy = hy - t * gy, qz = hz - t * gz;
        if (qx * qx + qy * qy + qz * qz > ra * ra) continue;
        const D4 Pa = g.t64.cry_pos[a], Za = g.t64.cry_size[a], Ta = g.t64.cry_trig[a];
        const double ax = p[0] - Pa.x, az = p[2] - Pa.z, bx = D3[0] - Pa.x, bz = D3[2] - Pa.z;
        const double la = box_chord64(ax * Ta.z - az * Ta.w, p[1] - Pa.y, ax * Ta.w + az * Ta.z,
                                      bx * Ta.z - bz * Ta.w, D3[1] - Pa.y, bx * Ta.w + bz * Ta.z, -0.5 * Za.x,
                                      -0.5 * Za.y, -0.5 * Za.z, 0.5 * Za.x, 0.5 * Za.y, 0.5 * Za.z);
        if (la != 0.0) {
            const float4 mu = __ldg(&g.cry.mu[a]);
            lpe += (double)mu.y * la;
            lc += (double)mu.z * la;
        }
    }
    if (k >= 0) {                                             // the rest of crystal k, from p to its exit
        const D4 Pk = g.t64.cry_pos[k], Zk = g.t64.cry_size[k], Tk = g.t64.cry_trig[k];
        const double ax = p[0] - Pk.x, az = p[2] - Pk.z, bx = D3[0] - Pk.x, bz = D3[2] - Pk.z;
        const double pa[3] = {ax * Tk.z - az * Tk.w, p[1] - Pk.y, ax * Tk.w + az * Tk.z};
        const double pb[3] = {bx * Tk.z - bz * Tk.w, D3[1] - Pk.y, bx * Tk.w + bz * Tk.z};
        const double lo[3] = {-0.5 * Zk.x, -0.5 * Zk.y, -0.5 * Zk.z}, hi[3] = {0.5 * Zk.x, 0.5 * Zk.y, 0.5 * Zk.z};
        const double lk = seg_box64(pa, pb, lo, hi);
        const float4 mu = __ldg(&g.cry.mu[k]);
        lpe += (double)mu.y * lk;
        lc += (double)mu.z * lk;
    }
    if (m >= 0) {                                             // tungsten and hole media on the way
        double wt = 0.0;
        for (int mm = 0; mm < G.n_layers; ++mm) layer_path64(g, G, mm, p, D3, wt, lpe, lc, &C);
    }
    out[0] = (float)ps[0];
    out[1] = (float)ps[1];
    out[2] = (float)ps[2];
    out[3] = (float)lsd;
    out[4] = (float)labs;
    out[5] = (float)lpe;
    out[6] = (float)lc;
    out[7] = (float)conv;
    return true;
}

__device__ __forceinline__ double kn_integral(const double* __restrict__ tab, double th)
{
    double G, F, P;
    kn_tab_eval(tab, th, G, F, P);
    return G;
}

constexpr int kTerms = 8;

struct GridSmem {
    Cands cand;                                 // the chunk's candidates for the current detector
    double acc[kGridDetTile][kGridMaxVox];      // block sums per (detector, voxel)
    float wt[kGridMaxVox][kGridChunk];          // the chunk's weights
    float terms[kTerms][kGridChunk];            // the chunk's detector-only terms
    float rlb[9][kGridChunk];                   // 1 / |corner c of d - p| (c < 8), 1 / |p - d|
    float4 vox_s[kGridMaxVox];                  // voxels in the current detector's frame
};

__global__ void __launch_bounds__(kGridThreads) grid_sum_kernel(DevGeom g, GridGeom G, GridSum S)
{
    extern __shared__ __align__(16) unsigned char grid_smem_raw[];
    GridSmem& sm = *reinterpret_cast<GridSmem*>(grid_smem_raw);
    auto& wt = sm.wt;
    auto& terms = sm.terms;
    auto& acc = sm.acc;
    auto& vox_s = sm.vox_s;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int d0 = S.det_begin + blockIdx.y * kGridDetTile;
    const int nd = min(kGridDetTile, S.det_begin + S.det_count - d0);
    for (int i = t; i < kGridDetTile * kGridMaxVox; i += kGridThreads) (&acc[0][0])[i] = 0.0;
    const float e0 = S.e0;
    const double inv_kn_total = 1.0 / S.kn_total;
    const float ang = S.rotation * g.angle_step;
    const float crot = cosf(ang), srot = sinf(ang);
    for (int ch = 0; ch < kGridChunksPerBlock; ++ch) {
        const long long p0 = ((long long)blockIdx.x * kGridChunksPerBlock + ch) * kGridChunk;
        if (p0 >= S.n_pts) break;
        const long long pidx = p0 + t;
        __syncthreads();
        double pt[3] = {0.0, 0.0, 0.0}, conv = 1.0;
        int kc = -1, mc = -1;
        const bool has = pidx < S.n_pts;
        if (has) grid_point(g, G, S, pidx, pt, kc, mc, conv);
        block_bounds(sm.cand, has, pt);
        const bool any_sep = __syncthreads_or(has && mc >= 0);
        for (int vi = 0; vi < S.nv; ++vi) {                     // stage the chunk's weights
            float w = 0.0f;
            if (pidx < S.n_cry_pts) w = S.wc[(long long)vi * S.n_cry_pts + pidx];
            else if (pidx < S.n_pts) w = S.ws[(long long)vi * S.n_sep + (pidx - S.n_cry_pts)];
            wt[vi][t] = w;
        }
        for (int dl = 0; dl < nd; ++dl) {
            const int d = d0 + dl;
            const float4 P = __ldg(&g.cry.pos[d]), T = __ldg(&g.cry.trig[d]), M = __ldg(&g.cry.mu[d]);
            const float4 Z = __ldg(&g.cry.size[d]);
            __syncthreads();                                    // previous detector's terms are consumed
            const D4 Pd = g.t64.cry_pos[d];
            const double E3[3] = {Pd.x, Pd.y, Pd.z};
            chunk_candidates(g, G, sm.cand, E3, true, any_sep);
            float tv[kTerms];
            const bool ok = has && point_terms(g, G, d, pt, kc, mc, conv, sm.cand, tv);
            if (!ok) tv[7] = 0.0f;                              // zero weight factor: no contribution
#pragma unroll
            for (int q = 0; q < kTerms; ++q) terms[q][t] = ok ? tv[q] : (q == 3 ? 1.0f : 0.0f);
            {                                                   // point -> corner distances of d
                const float hw = 0.5f * Z.x, ht = 0.5f * Z.y, hh = 0.5f * Z.z;
                const float px = ok ? tv[0] : 0.0f, py = ok ? tv[1] : 0.0f, pz = ok ? tv[2] : 0.0f;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const float bx = ((c & 1) ? hw : -hw) - px, by = ((c & 2) ? ht : -ht) - py;
                    const float bz = ((c & 4) ? hh : -hh) - pz;
                    sm.rlb[c][t] = 1.0f / sqrtf(bx * bx + by * by + bz * bz);
                }
                sm.rlb[8][t] = ok ? 1.0f / tv[3] : 0.0f;
            }
            if (t < S.nv) {
                float x, y, z, xs, ys, zs;
                voxel_centre(g, S.vox_begin + t, crot, srot, x, y, z);
                to_crystal_frame(P.x, P.y, P.z, T.z, T.w, x, y, z, xs, ys, zs);
                vox_s[t] = make_float4(xs, ys, zs, 0.0f);
            }
            __syncthreads();
            // window of crystal d (scatter.cu:1154-1163)
            const float lo = S.same_window ? S.lo : (1 - M.w / 2.0f) * e0;
            const float hi = S.same_window ? S.hi : (1 + M.w / 2.0f) * e0;
            const float rdet = 0.5f * Z.w;                      // sqrt(w^2 + h^2 + t^2) / 2
            const float hw = 0.5f * Z.x, ht = 0.5f * Z.y, hh = 0.5f * Z.z;
            for (int vi = warp; vi < S.nv; vi += kGridThreads / 32) {
                const float4 I = vox_s[vi];
                double sum = 0.0;
                for (int j = lane; j < kGridChunk; j += 32) {
                    const float w = wt[vi][j] * terms[7][j];
                    if (w == 0.0f) continue;
                    const float px = terms[0][j], py = terms[1][j], pz = terms[2][j], lsd = terms[3][j];
                    const float ax = px - I.x, ay = py - I.y, az = pz - I.z;      // v -> p
                    const float la = sqrtf(ax * ax + ay * ay + az * az);
                    const float rla = 1.0f / la;
                    // angle v -> p -> d (cosines as dot products times reciprocal lengths)
                    const float cc = fminf(fmaxf(-(ax * px + ay * py + az * pz) * rla * sm.rlb[8][j], -1.0f), 1.0f);
                    // the model restated in float with reciprocals where the reference's program
                    // divides (no bit-parity target here: the definition is the FP64 oracle)
                    const float r1 = 1.0f + (e0 / 511.0f) * (1.0f - cc);          // E0 / E'
                    const float es = __fdividef(e0, r1);
                    const float res = M.w * sqrtf(__fdividef(es, e0));
                    if ((es * (1 + 2 * res / 2.35482f)) <= lo || (es * (1 - 2 * res / 2.35482f)) >= hi) continue;
                    const float rs2 = __frcp_rn(res / 2.35482f * es * 1.41421356f);
                    const float pwin = 0.5f * (erff((hi - es) * rs2) - erff((lo - es) * rs2));
                    const float sc = sqrtf(fmaxf(1.0f - cc * cc, 0.0f));
                    float phi;
                    if (lsd * sc * 2.0f <= rdet) phi = (float)(2.0 * 3.14159265358979323846);
                    else phi = 4.0f * asinf(fminf(0.5f * rdet * sm.rlb[8][j] * __frcp_rn(sc), 1.0f));
                    // polar range over the corners of d, seen from p along v -> p (:1305-1335)
                    float cmin = INFINITY, cmax = -INFINITY;
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const float ck = (ax * (((c & 1) ? hw : -hw) - px) + ay * (((c & 2) ? ht : -ht) - py) +
                                          az * (((c & 4) ? hh : -hh) - pz)) * sm.rlb[c][j];
                        cmin = fminf(cmin, ck);
                        cmax = fmaxf(cmax, ck);
                    }
                    float tmin = acosf(fminf(fmaxf(cmax * rla, -1.0f), 1.0f));
                    const float tmax = acosf(fminf(fmaxf(cmin * rla, -1.0f), 1.0f));
                    const float lthr = box_chord(I.x, I.y, I.z, px + 1000.0f * ax * rla, py + 1000.0f * ay * rla,
                                                 pz + 1000.0f * az * rla, -hw, -ht, -hh, hw, ht, hh);
                    if (lthr > 0.001f) tmin = 0.0f;
                    const double ratio = (kn_integral(S.kn_tab, (double)tmax) - kn_integral(S.kn_tab, (double)tmin)) *
                                         inv_kn_total;
                    const float r3 = r1 * r1 * r1;
                    const float att = terms[5][j] * r3 + terms[6][j] * r1;
                    const float mpe_s = M.y * r3, mt_s = mpe_s + M.z * r1;
                    const float absf = -expm1f(-terms[4][j] * mt_s) * __fdividef(mpe_s, mt_s);
                    sum += (double)(w * phi * (float)(0.5 / 3.14159265358979323846) * pwin * expf(-att) * absf) *
                           ratio;
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
                if (lane == 0) acc[dl][vi] += sum;
            }
        }
    }
    __syncthreads();
    for (int i = t; i < nd * S.nv; i += kGridThreads) {
        const int dl = i / S.nv, vi = i - dl * S.nv;
        const double a = acc[dl][vi];
        if (a != 0.0) atomicAdd(&S.acc[(long long)(d0 - S.det_begin + dl) * S.nv + vi], a);
    }
}

__global__ void grid_store_kernel(const double* __restrict__ acc, int rows, int nv, float* __restrict__ out,
                                  long long ld, long long col0)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)rows * nv) return;
    const int r = (int)(i / nv), c = (int)(i - (long long)r * nv);
    out[(long long)r * ld + col0 + c] = (float)acc[i];
}

struct DevMem {
    void* p = nullptr;
    ~DevMem() { if (p) cudaFree(p); }
};

int grid_division(float size, float cell)
{
    const int n = (int)std::ceil((double)size / (double)cell - 1e-9);
    return n < 1 ? 1 : n;
}

}  // namespace

}  // namespace sysmat

using namespace sysmat;

extern "C" SYSMAT_API int sysmat_scatter_grid(sysmat_ctx* ctx, int parts, float cell, float rotation, int det_begin,
                                              int det_count, long long vox_begin, long long vox_count, float* d_out,
                                              long long ld, void* stream)
{
    int rc = check_block(ctx, det_begin, det_count, vox_begin, vox_count, d_out, ld);
    if (rc) return rc;
    if (parts < 1 || parts > 3 || !(cell > 0.0f)) return SYSMAT_ERR_ARG;
    if (ctx->h_phys.size() != (size_t)kNPhysics || ctx->h_det.size() != (size_t)kNDetector) return SYSMAT_ERR_ARG;
    if ((parts & 2) && ctx->g.n_layers < 1) return SYSMAT_ERR_ARG;
    if (det_count == 0 || vox_count == 0) return SYSMAT_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const DevGeom& g = ctx->g;
    const int D = g.n_det;
    const float* pD = ctx->h_det.data();
    const float* P = ctx->h_phys.data();
    if ((int)std::floor(P[0] + 0.5f) != 1) {                   // no Compton scatter (scatter.cu:1144)
        for (int r = 0; r < det_count; ++r)
            CUDA_TRY(cudaMemsetAsync(d_out + (long long)r * ld, 0, sizeof(float) * vox_count, s));
        return cudaStreamSynchronize(s) == cudaSuccess ? SYSMAT_OK : SYSMAT_ERR_CUDA;
    }
    // crystal cells: one division for every crystal
    const int snx = grid_division(pD[4], cell), sny = grid_division(pD[5], cell), snz = grid_division(pD[6], cell);
    for (int k = 1; k < D; ++k)
        if (grid_division(pD[12 * k + 4], cell) != snx || grid_division(pD[12 * k + 5], cell) != sny ||
            grid_division(pD[12 * k + 6], cell) != snz)
            return SYSMAT_ERR_ARG;
    const long long n_sub = (long long)snx * sny * snz;
    if (n_sub > (1 << 20)) return SYSMAT_ERR_CAPACITY;

    // septal cells of every layer (cell centres outside the layer's holes)
    GridGeom G{};
    G.n_layers = (parts & 2) ? g.n_layers : 0;
    G.raw_col = ctx->d_col;
    DevMem sep_mem;
    long long n_sep = 0;
    if (parts & 2) {
        std::vector<double> lay(kLayer64 * (size_t)g.n_layers);
        CUDA_TRY(cudaMemcpy(lay.data(), g.t64.layer, sizeof(double) * lay.size(), cudaMemcpyDeviceToHost));
        long long cells_max = 0;
        for (int m = 0; m < g.n_layers; ++m) {
            const double* Ly = lay.data() + kLayer64 * m;
            GridLayer& L = G.layer[m];
            L.x0 = Ly[0]; L.y0 = Ly[2]; L.z0 = Ly[4];
            L.nx = grid_division((float)(Ly[1] - Ly[0]), cell);
            L.ny = grid_division((float)(Ly[3] - Ly[2]), cell);
            L.nz = grid_division((float)(Ly[5] - Ly[4]), cell);
            L.cx = (Ly[1] - Ly[0]) / L.nx; L.cy = (Ly[3] - Ly[2]) / L.ny; L.cz = (Ly[5] - Ly[4]) / L.nz;
            L.nbx = (L.nx + kBrickX - 1) / kBrickX;
            L.nby = (L.ny + kBrickY - 1) / kBrickY;
            L.nbz = (L.nz + kBrickZ - 1) / kBrickZ;
            L.hole_begin = g.layer[m].hole_begin;
            L.hole_count = g.layer[m].hole_count;
            L.mu_t = g.layer[m].mu_total; L.mu_pe = g.layer[m].mu_pe; L.mu_c = g.layer[m].mu_c;
            const long long nc = (long long)L.nbx * L.nby * L.nbz * kBrickCells;   // brick-padded
            if (nc > (1ll << 30)) return SYSMAT_ERR_CAPACITY;
            cells_max = nc > cells_max ? nc : cells_max;
        }
        long long total_cells = 0;
        for (int m = 0; m < g.n_layers; ++m)
            total_cells += (long long)G.layer[m].nbx * G.layer[m].nby * G.layer[m].nbz * kBrickCells;
        size_t temp = 0;
        cub::DeviceSelect::Flagged(nullptr, temp, thrust::counting_iterator<int>(0), (unsigned char*)nullptr,
                                   (int*)nullptr, (int*)nullptr, (int)cells_max, s);
        DevMem flags, tmp, cnt;
        if (cudaMalloc(&sep_mem.p, sizeof(int) * (size_t)total_cells) != cudaSuccess ||
            cudaMalloc(&flags.p, (size_t)cells_max) != cudaSuccess || cudaMalloc(&tmp.p, temp + 16) != cudaSuccess ||
            cudaMalloc(&cnt.p, sizeof(int)) != cudaSuccess)
            return SYSMAT_ERR_NOMEM;
        int* sep = (int*)sep_mem.p;
        for (int m = 0; m < g.n_layers; ++m) {
            const GridLayer& L = G.layer[m];
            const int nc = L.nbx * L.nby * L.nbz * kBrickCells;
            septal_mark_kernel<<<(nc + 255) / 256, 256, 0, s>>>(g, L, nc, (unsigned char*)flags.p);
            size_t t2 = temp;
            cub::DeviceSelect::Flagged(tmp.p, t2, thrust::counting_iterator<int>(0), (unsigned char*)flags.p,
                                       sep + n_sep, (int*)cnt.p, nc, s);
            int nsel = 0;
            CUDA_TRY(cudaMemcpyAsync(&nsel, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaStreamSynchronize(s));
            G.sep_begin[m] = n_sep;
            n_sep += nsel;
        }
        for (int m = g.n_layers; m <= kMaxLayers; ++m) G.sep_begin[m] = n_sep;
        G.sep_cell = sep;
    }

    // Klein-Nishina table at the photopeak (shared with sysmat_scatter)
    if (!ctx->d_kn_tab || ctx->kn_e0 != P[7]) {
        std::vector<double> tab(3 * (size_t)(kKnTable + 1));
        kn_table_build((double)P[7], tab.data());
        if (!ctx->d_kn_tab && cudaMalloc(&ctx->d_kn_tab, sizeof(double) * tab.size()) != cudaSuccess) {
            ctx->d_kn_tab = nullptr;
            return SYSMAT_ERR_NOMEM;
        }
        CUDA_TRY(cudaMemcpyAsync(ctx->d_kn_tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        ctx->kn_e0 = P[7];
    }
    double kn_total = 0.0;
    CUDA_TRY(cudaMemcpy(&kn_total, ctx->d_kn_tab + kKnTable, sizeof(double), cudaMemcpyDeviceToHost));

    // scratch: weights of one pass of voxels, the photoelectric block, the FP64 sums
    const int nv_max = (int)(vox_count < kGridMaxVox ? vox_count : kGridMaxVox);
    const long long n_cry_pts = (parts & 1) ? (long long)D * n_sub : 0;
    DevMem wc, ws, pe, acc;
    if ((n_cry_pts && cudaMalloc(&wc.p, sizeof(float) * (size_t)nv_max * (size_t)n_cry_pts) != cudaSuccess) ||
        (n_sep && cudaMalloc(&ws.p, sizeof(float) * (size_t)nv_max * (size_t)n_sep) != cudaSuccess) ||
        ((parts & 1) && cudaMalloc(&pe.p, sizeof(float) * (size_t)nv_max * D) != cudaSuccess) ||
        cudaMalloc(&acc.p, sizeof(double) * (size_t)nv_max * det_count) != cudaSuccess)
        return SYSMAT_ERR_NOMEM;

    GridSum S{};
    S.det_begin = det_begin;
    S.det_count = det_count;
    S.rotation = rotation;
    S.snx = snx; S.sny = sny; S.snz = snz; S.n_sub = (int)n_sub;
    S.n_cry_pts = n_cry_pts;
    S.n_sep = n_sep;
    S.n_pts = n_cry_pts + n_sep;
    S.wc = (const float*)wc.p;
    S.ws = (const float*)ws.p;
    S.acc = (double*)acc.p;
    S.e0 = P[7];
    S.lo = P[5];
    S.hi = P[6];
    S.same_window = (int)std::floor(P[4] + 0.5f) > 0;
    S.kn_tab = ctx->d_kn_tab;
    S.kn_total = kn_total;
    CUDA_TRY(cudaFuncSetAttribute(grid_sum_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GridSmem)));
    for (long long vb = vox_begin; vb < vox_begin + vox_count; vb += kGridMaxVox) {
        const int nv = (int)((vox_begin + vox_count - vb) < kGridMaxVox ? (vox_begin + vox_count - vb) : kGridMaxVox);
        if (parts & 1) {                                          // crystal-cell weights
            PeLaunch L{};
            L.det_begin = 0;
            L.det_count = D;
            L.vox_begin = vb;
            L.vox_count = nv;
            L.ld = nv;
            L.rotation = rotation;
            L.out = (float*)pe.p;
            L.work_counter = ctx->d_counter;
            L.status = ctx->d_status;
            L.counters = nullptr;
            L.smp.nx = snx; L.smp.ny = sny; L.smp.nz = snz;
            L.smp.sx = L.smp.sy = L.smp.sz = 1;
            L.sub_out = (float*)wc.p;
            CUDA_TRY(cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), s));
            CUDA_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s));
            if (launch_pe_local_sampled(g, L, ctx->num_sms, s)) return SYSMAT_ERR_CUDA;
            int st = 0;
            CUDA_TRY(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
            CUDA_TRY(cudaStreamSynchronize(s));
            if (st & kStatusCapacity) return SYSMAT_ERR_CAPACITY;
        }
        if (n_sep) {                                              // septal-cell weights
            const dim3 sgrid((unsigned)((n_sep + kGridThreads - 1) / kGridThreads), (unsigned)nv);
            septal_weight_kernel<<<sgrid, kGridThreads, 0, s>>>(g, G, vb, rotation, n_sep, (float*)ws.p);
            if (cudaGetLastError() != cudaSuccess) return SYSMAT_ERR_CUDA;
        }
        S.vox_begin = vb;
        S.nv = nv;
        CUDA_TRY(cudaMemsetAsync(acc.p, 0, sizeof(double) * (size_t)nv * det_count, s));
        const long long pblocks = (S.n_pts + (long long)kGridChunk * kGridChunksPerBlock - 1) /
                                  ((long long)kGridChunk * kGridChunksPerBlock);
        dim3 grid((unsigned)pblocks, (unsigned)((det_count + kGridDetTile - 1) / kGridDetTile));
        grid_sum_kernel<<<grid, kGridThreads, sizeof(GridSmem), s>>>(g, G, S);
        if (cudaGetLastError() != cudaSuccess) return SYSMAT_ERR_CUDA;
        const long long n = (long long)nv * det_count;
        grid_store_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>((const double*)acc.p, det_count, nv, d_out, ld,
                                                                       vb - vox_begin);
        if (cudaGetLastError() != cudaSuccess) return SYSMAT_ERR_CUDA;
    }
    return cudaStreamSynchronize(s) == cudaSuccess ? SYSMAT_OK : SYSMAT_ERR_CUDA;
}
