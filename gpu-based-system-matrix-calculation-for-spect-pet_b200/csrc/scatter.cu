// Primary-Compton scatter kernels and geometry-relationship bitmaps for sm_100a.
//
// Physics follows the reference kernels crystalScatterSysMatCuda
// (ScatterGen_RayTracing_CircularHole/scatter.cu:1077-1437) and collimatorScatterSysMatCuda
// (:1544-1936; hole solid angle of the collimator-only program at
// ScatterGen_Collimator/scatter.cu:1212-1215).  Execution plan:
//
//  * everything that depends only on the (scatterer s, detector d) pair is computed once
//    per pair instead of once per (d, v, s) item: the scatter point in d's frame, the
//    scatter-to-detector distance, the absorption chord in d, and the list of attenuating
//    crystals flagged by the relationship bitmap with a non-zero chord (the reference scans
//    all D crystals of the bitmap for every item, :1343-1401);
//  * the self-attenuation term (:1404-1417) is exactly 0 with the reference's 1x1x1
//    detector sub-division (the crystal box and the sub-element box are the same floats), so
//    it is not evaluated;
//  * the Klein-Nishina angular ratio is the reference's left Riemann sum with
//    n = (int)((theta_max - theta_min) / 0.01f) + 1 terms (:980-993, :1338).  It is
//    evaluated through the Euler-Maclaurin identity
//      sum_{i=0..n} F(a + i h) h = int_a^b F + h/2 (F(a) + F(b)) + h^2/12 (F'(b) - F'(a)) + O(h^4)
//    with an 8-point Gauss-Legendre integral, instead of n+1 cos/sin evaluations; theta_min,
//    theta_max and n are computed with the reference's float formulas, so the step count
//    matches.  The normalisation over [0, pi] is a host FP64 sum;
//  * one thread per matrix element (d, v); a block shares d, so pair records are staged in
//    shared memory and attenuator lists are broadcast loads; each element sums its items in
//    FP64 (the reference adds float items with atomicAdd in an unspecified order).
#include <algorithm>
#include <cmath>

#include <cub/cub.cuh>

#include "scatter.cuh"

namespace sysmat {

namespace {

constexpr int kItemThreads = kScatterBlockVoxels;
constexpr int kPairChunk = 512;

// ---- reference helper formulas (scatter.cu:961-1038) ----

// Clamped cosine of the scattering angle at a between the directions s -> a and a -> d.
__device__ __forceinline__ float cone_cosine(float xs, float ys, float zs, float xa, float ya, float za,
                                             float xd, float yd, float zd)
{
    const float a0 = xa - xs, a1 = ya - ys, a2 = za - zs;
    const float b0 = xd - xa, b1 = yd - ya, b2 = zd - za;
    const float dot = b0 * a0 + b1 * a1 + b2 * a2;
    const float ma = sqrtf(a0 * a0 + a1 * a1 + a2 * a2);
    const float mb = sqrtf(b0 * b0 + b1 * b1 + b2 * b2);
    float c = dot / (ma * mb);
    if (c > 1.0f) c = 1.0f;
    if (c < -1.0f) c = -1.0f;
    return c;
}

__device__ __forceinline__ float cone_angle(float xs, float ys, float zs, float xa, float ya, float za,
                                            float xd, float yd, float zd)
{
    return acosf(cone_cosine(xs, ys, zs, xa, ya, za, xd, yd, zd));
}

__device__ __forceinline__ float dist3(float x1, float y1, float z1, float x2, float y2, float z2)
{
    return sqrtf((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2) + (z1 - z2) * (z1 - z2));
}

// Reference Riemann sum with n + 1 terms from a, step 0.01f, in FP64 from the table:
//   sum = G(b) - G(a) + h/2 (F(a) + F(b)) + h^2/12 (F'(b) - F'(a)),  b = a + n h
// (G, F and F' from kn_tab_eval, scatter.cuh).
__device__ __forceinline__ double kn_sum_tab(float a, int n, const double* __restrict__ tab)
{
    const double h = (double)0.01f;
    const double ad = (double)a, bd = ad + (double)n * h;
    double Ga, Fa, Pa, Gb, Fb, Pb;
    kn_tab_eval(tab, ad, Ga, Fa, Pa);
    kn_tab_eval(tab, bd, Gb, Fb, Pb);
    return (Gb - Ga) + 0.5 * h * (Fa + Fb) + (h * h / 12.0) * (Pb - Pa);
}

// Crystal d's single sub-element centre (1x1x1 division, :1242-1252) in its own frame and
// in world coordinates.
struct DetPoint {
    float xDs, yDs, zDs, xD, yD, zD;
};

__device__ __forceinline__ DetPoint det_point(float4 P, float4 S, float4 T)
{
    DetPoint q;
    const float w = S.x, t = S.y, h = S.z;
    q.xDs = -w / 2.0f + ((float)0 + 0.5f) / 1.0f * w;
    q.zDs = -h / 2.0f + ((float)0 + 0.5f) / 1.0f * h;
    q.yDs = -t / 2.0f + ((float)0 + 0.5f) / 1.0f * t;
    q.xD = P.x + (q.xDs * T.x - q.zDs * T.y);
    q.zD = P.z + (q.xDs * T.y + q.zDs * T.x);
    q.yD = P.y + q.yDs;
    return q;
}

// ---- relationship bitmaps, one thread per 32-bit word (no atomics) ----

__global__ void bitmap_crystal_kernel(const float* __restrict__ det, int n, long long words,
                                      uint32_t* __restrict__ out)
{
    const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    const long long total_pairs = (long long)n * (n + 1) / 2;
    long long bit = w * 32;
    long long pair = bit / n;
    int a = (int)(bit - pair * n);
    // row i of pair index p = i*n - i(i+1)/2 + j (i <= j)
    double disc = (2.0 * n + 1.0) * (2.0 * n + 1.0) - 8.0 * (double)pair;
    long long i = (long long)floor(((2.0 * n + 1.0) - sqrt(disc > 0 ? disc : 0)) / 2.0);
    if (i < 0) i = 0;
    while (i > 0 && i * n - i * (i - 1) / 2 > pair) --i;
    while ((i + 1) * n - (i + 1) * i / 2 <= pair) ++i;
    long long j = pair - (i * n - i * (i + 1) / 2);
    uint32_t word = 0;
    for (int b = 0; b < 32; ++b) {
        if (pair >= total_pairs) break;
        const int ii = (int)i, jj = (int)j, k = a;
        if (ii < jj && k != ii && k != jj) {
            // scatter.cu:1465-1534
            const float* pi = det + 12 * ii;
            const float* pj = det + 12 * jj;
            const float* pk = det + 12 * k;
            const float ri = sqrtf(pi[4] * pi[4] + pi[6] * pi[6] + pi[5] * pi[5]) / 2.0f;
            const float rj = sqrtf(pj[4] * pj[4] + pj[6] * pj[6] + pj[5] * pj[5]) / 2.0f;
            const float lij = dist3(pi[1], pi[2], pi[3], pj[1], pj[2], pj[3]);
            const float cij = ri / lij, cji = rj / lij;
            const float rk = sqrtf(pk[4] * pk[4] + pk[6] * pk[6] + pk[5] * pk[5]) / 2.0f;
            const float lik = dist3(pk[1], pk[2], pk[3], pi[1], pi[2], pi[3]);
            const float cki = rk / lik;
            const float ljk = dist3(pk[1], pk[2], pk[3], pj[1], pj[2], pj[3]);
            const float ckj = rk / ljk;
            const float d_i = dist3((pk[1] - pi[1]) / lik, (pk[2] - pi[2]) / lik, (pk[3] - pi[3]) / lik,
                                    (pj[1] - pi[1]) / lij, (pj[2] - pi[2]) / lij, (pj[3] - pi[3]) / lij);
            bool hit = d_i <= cki + cji;
            if (!hit) {
                const float d_j = dist3((pk[1] - pj[1]) / ljk, (pk[2] - pj[2]) / ljk, (pk[3] - pj[3]) / ljk,
                                        (pi[1] - pj[1]) / lij, (pi[2] - pj[2]) / lij, (pi[3] - pj[3]) / lij);
                hit = d_j <= ckj + cij;
            }
            if (hit) word |= 1u << b;
        }
        if (++a == n) {
            a = 0;
            ++pair;
            if (++j == n) { ++i; j = i; }
        }
    }
    out[w] = word;
}

// Whether crystal k may attenuate the path from hole i (raw parameters hr) to crystal j:
// k's bounding sphere within the angular cone of the hole-to-j segment, seen from the hole
// (scatter.cu:1963-2006; raw y, no FOV offset).
__device__ __forceinline__ bool collimator_related(const float* __restrict__ det, float4 hr, int j, int k)
{
    const float xi = hr.x, yi = (hr.y + hr.z) / 2.0f, zi = hr.w;
    const float* pj = det + 12 * j;
    const float* pk = det + 12 * k;
    const float rj = sqrtf(pj[4] * pj[4] + pj[6] * pj[6] + pj[5] * pj[5]) / 2.0f;
    const float lij = dist3(xi, yi, zi, pj[1], pj[2], pj[3]);
    const float cji = rj / lij;
    const float rk = sqrtf(pk[4] * pk[4] + pk[6] * pk[6] + pk[5] * pk[5]) / 2.0f;
    const float lik = dist3(pk[1], pk[2], pk[3], xi, yi, zi);
    const float cki = rk / lik;
    const float dd = dist3((pk[1] - xi) / lik, (pk[2] - yi) / lik, (pk[3] - zi) / lik,
                           (pj[1] - xi) / lij, (pj[2] - yi) / lij, (pj[3] - zi) / lij);
    return dd <= cki + cji;
}

__global__ void bitmap_collimator_kernel(const float* __restrict__ det, const float4* __restrict__ hraw,
                                         int n, int nh, long long words, uint32_t* __restrict__ out)
{
    const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= words) return;
    const long long total = (long long)nh * n * n;
    long long bit = w * 32;
    uint32_t word = 0;
    for (int b = 0; b < 32 && bit < total; ++b, ++bit) {
        const int k = (int)(bit % n);
        const long long ij = bit / n;
        const int j = (int)(ij % n);
        const int i = (int)(ij / n);
        if (collimator_related(det, __ldg(&hraw[i]), j, k)) word |= 1u << b;
    }
    out[w] = word;
}

// ---- pair tables ----

// Scatter point of scatterer s: crystal centre (y + FOV) or hole centre
// ((y1 + y2) / 2 + FOV), scatter.cu:1221-1223, :1707-1709.
__device__ __forceinline__ void scatter_point(const DevGeom& g, int s, float& xs, float& ys, float& zs)
{
    if (s < g.n_det) {
        const float4 p = __ldg(&g.cry.pos[s]);
        xs = p.x; ys = p.y; zs = p.z;
    } else {
        const float4 r = __ldg(&g.hole.raw[s - g.n_det]);
        xs = r.x;
        ys = (r.y + r.z) / 2.0f + g.fov;
        zs = r.w;
    }
}

// Pair-table kernels: one warp per (detector d, scatterer s) pair.  The pair's candidate
// attenuators (its bitmap row, or the relationship predicate) are compacted into a per-warp
// list in ascending crystal order, then the lanes take 32 list entries at a time, so every
// lane evaluates a chord instead of waiting on the lane with the most set bits.
constexpr int kPairWarps = 8;          // warps per block
constexpr int kPairSpan = 1024;        // candidates compacted per pass (32 per lane)

// Bit start of the n-bit row of pair (s, d): crystal pairs in the upper triangle (i < j),
// hole pairs by (hole, detector).
__device__ __forceinline__ long long pair_row_bit(int n, int s, int d)
{
    if (s < n) {
        const long long i = s < d ? s : d, j = s < d ? d : s;
        return (i * n - (i * (i + 1)) / 2 + j) * n;
    }
    return ((long long)(s - n) * n + d) * n;
}

// Candidates a0 .. a0+31 of pair (s, d) as a bit mask (bit k: crystal a0 + k), without
// crystal d and scatter crystal s.  NATIVE hole scatterers evaluate the predicate instead of
// reading a bitmap.
template <bool NATIVE>
__device__ __forceinline__ uint32_t candidate_mask(const DevGeom& g, const uint32_t* bm, long long base,
                                                   float4 hr, int s, int d, int a0)
{
    const int n = g.n_det;
    if (a0 >= n) return 0u;
    const int span = n - a0 < 32 ? n - a0 : 32;
    uint32_t m = 0u;
    if (NATIVE && s >= n) {
        for (int k = 0; k < span; ++k)
            if (collimator_related(g.raw_det, hr, d, a0 + k)) m |= 1u << k;
    } else {
        const long long b = base + a0, w = b >> 5;
        const int sh = (int)(b & 31);
        const uint32_t lo = __ldg(&bm[w]);
        // the next word only when the row continues into it
        const uint32_t hi = (sh != 0 && w + 1 <= ((base + n - 1) >> 5)) ? __ldg(&bm[w + 1]) : 0u;
        m = __funnelshift_r(lo, hi, sh);
        if (span < 32) m &= (1u << span) - 1u;
    }
    if (d >= a0 && d - a0 < 32) m &= ~(1u << (d - a0));
    if (s < n && s >= a0 && s - a0 < 32) m &= ~(1u << (s - a0));
    return m;
}

// Chord of the scatter point -> detector point segment inside attenuating crystal a
// (scatter.cu:1377-1394).
__device__ __forceinline__ float attenuator_chord(const DevGeom& g, int a, float xs, float ys, float zs,
                                                  const DetPoint& q)
{
    const float4 pa = __ldg(&g.cry.pos[a]);
    const float4 sa = __ldg(&g.cry.size[a]);
    const float4 ta = __ldg(&g.cry.trig[a]);
    float xa, ya, za, xb, yb, zb;
    to_crystal_frame(pa.x, pa.y, pa.z, ta.z, ta.w, xs, ys, zs, xa, ya, za);
    to_crystal_frame(pa.x, pa.y, pa.z, ta.z, ta.w, q.xD, q.yD, q.zD, xb, yb, zb);
    return box_chord(xa, ya, za, xb, yb, zb, -0.5f * sa.x, -0.5f * sa.y, -0.5f * sa.z, 0.5f * sa.x,
                     0.5f * sa.y, 0.5f * sa.z);
}

// Warp-collective walk over the attenuators of pair (s, d) in ascending crystal order: f(a,
// len, ok) is called by every lane for each group of 32 candidates (ok false on lanes past
// the group's end).  list: the warp's kPairSpan-entry shared buffer.
template <bool NATIVE, typename F>
__device__ __forceinline__ void warp_attenuators(const DevGeom& g, const uint32_t* bm_cry, const uint32_t* bm_col,
                                                 int s, int d, float xs, float ys, float zs, const DetPoint& q,
                                                 int lane, int* list, F&& f)
{
    const int n = g.n_det;
    const long long base = (NATIVE && s >= n) ? 0 : pair_row_bit(n, s, d);
    const uint32_t* bm = s < n ? bm_cry : bm_col;
    const float4 hr = (NATIVE && s >= n) ? __ldg(&g.hole.raw[s - n]) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int c0 = 0; c0 < n; c0 += kPairSpan) {
        const int a0 = c0 + 32 * lane;
        uint32_t m = candidate_mask<NATIVE>(g, bm, base, hr, s, d, a0);
        const int cnt = __popc(m);
        int incl = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int pos = incl - cnt;
        while (m) {
            list[pos++] = a0 + __ffs(m) - 1;
            m &= m - 1u;
        }
        __syncwarp();
        for (int b = 0; b < total; b += 32) {
            const bool ok = b + lane < total;
            const int a = ok ? list[b + lane] : 0;
            const float len = ok ? attenuator_chord(g, a, xs, ys, zs, q) : 0.0f;
            f(a, len, ok);
        }
        __syncwarp();
    }
}

__device__ __forceinline__ bool pair_enabled(const DevGeom& g, int parts, int s, int d)
{
    if (s < g.n_det) return (parts & 1) && s != d;
    return (parts & 2) != 0;
}

// Layer of hole h (global numbering, layer by layer).
__device__ __forceinline__ int hole_layer(const DevGeom& g, int h)
{
    int m = 0;
    while (m + 1 < g.n_layers && h >= g.layer[m + 1].hole_begin) ++m;
    return m;
}

// Distance from the centre (x, ym, z) of hole h along the unit direction k to where the
// path leaves the hole (side wall or cap), capped at len.
__device__ __forceinline__ float hole_exit(float4 a, float r, float ym, float kx, float ky, float kz, float len)
{
    const float kk = kx * kx + kz * kz;
    float t = len;
    if (kk > 0.0f) t = fminf(t, r / sqrtf(kk));
    if (ky > 0.0f) t = fminf(t, (a.z - ym) / ky);
    else if (ky < 0.0f) t = fminf(t, (a.y - ym) / ky);
    return t;
}

// Native model: tungsten crossed by the scattered photon from the centre S of hole h to the
// detector point D, as sum_m mu_pe,m L_m and sum_m mu_C,m L_m, L_m = plate chord of layer m
// minus the hole chords of layer m (the reference chords; the scatter hole's own part is its
// exit distance from S, and in its own layer the plate chord runs from the plate entry seen
// from D to S).
__device__ void tungsten_path(const DevGeom& g, int h, float sx, float sy, float sz, float dx, float dy, float dz,
                              float& w_pe, float& w_c)
{
    w_pe = 0.0f;
    w_c = 0.0f;
    const int mh = hole_layer(g, h);
    const float ex = dx - sx, ey = dy - sy, ez = dz - sz;
    const float len = sqrtf(ex * ex + ey * ey + ez * ez);
    const float kx = ex / len, ky = ey / len, kz = ez / len;
    const float n2 = ex * ex + ez * ez;
    for (int m = 0; m < g.n_layers; ++m) {
        const LayerInfo& Ly = g.layer[m];
        const float box = (m == mh) ? box_chord_inside(dx, dy, dz, sx, sy, sz, Ly.x1, Ly.y1, Ly.z1, Ly.x2, Ly.y2, Ly.z2)
                                    : box_chord(sx, sy, sz, dx, dy, dz, Ly.x1, Ly.y1, Ly.z1, Ly.x2, Ly.y2, Ly.z2);
        if (box == 0.0f) continue;
        float holes = 0.0f;
        for (int j = Ly.hole_begin; j < Ly.hole_begin + Ly.hole_count; ++j) {
            const float4 a = __ldg(&g.hole.a[j]);
            const float r = __ldg(&g.hole.b[j].x);
            if (j == h) {
                holes = holes + hole_exit(a, r, sy, kx, ky, kz, len);
                continue;
            }
            // the line keeps further than r from the axis: the chord is 0 (exact-safe reject)
            const float cr = ex * (a.w - sz) - ez * (a.x - sx);
            if (cr * cr > r * r * n2 * 1.001f + 1e-12f) continue;
            holes = holes + cyl_chord(sx, sy, sz, dx, dy, dz, a.x, a.y, a.z, a.w, r);
        }
        const float L = box - holes;
        if (L > 0.0f) {
            w_pe = w_pe + Ly.mu_pe * L;
            w_c = w_c + Ly.mu_c * L;
        }
    }
}

template <bool NATIVE>
__global__ void __launch_bounds__(32 * kPairWarps) pair_count_kernel(DevGeom g, int parts, const uint32_t* bm_cry,
                                                                     const uint32_t* bm_col, long long* counts)
{
    __shared__ int list[kPairWarps][kPairSpan];
    const int ns = g.n_det + (NATIVE ? g.n_holes : g.n_holes0);
    const long long np = (long long)g.n_det * ns;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (long long p = (long long)blockIdx.x * kPairWarps + wid; p < np; p += (long long)gridDim.x * kPairWarps) {
        const int d = (int)(p / ns), s = (int)(p - (long long)d * ns);
        int c = 0;
        if (pair_enabled(g, parts, s, d)) {
            float xs, ys, zs;
            scatter_point(g, s, xs, ys, zs);
            const DetPoint q = det_point(__ldg(&g.cry.pos[d]), __ldg(&g.cry.size[d]), __ldg(&g.cry.trig[d]));
            warp_attenuators<NATIVE>(g, bm_cry, bm_col, s, d, xs, ys, zs, q, lane, list[wid],
                                     [&](int, float len, bool ok) {
                                         c += __popc(__ballot_sync(0xffffffffu, ok && len != 0.0f));
                                     });
        }
        if (lane == 0) counts[p] = c;
    }
}

template <bool NATIVE>
__global__ void __launch_bounds__(32 * kPairWarps) pair_fill_kernel(DevGeom g, int parts, const uint32_t* bm_cry,
                                                                    const uint32_t* bm_col, const long long* offsets,
                                                                    PairRec* pairs, AttEntry* att)
{
    __shared__ int list[kPairWarps][kPairSpan];
    const int ns = g.n_det + (NATIVE ? g.n_holes : g.n_holes0);
    const long long np = (long long)g.n_det * ns;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (long long p = (long long)blockIdx.x * kPairWarps + wid; p < np; p += (long long)gridDim.x * kPairWarps) {
        const int d = (int)(p / ns), s = (int)(p - (long long)d * ns);
        PairRec r{};
        r.valid = pair_enabled(g, parts, s, d);
        if (r.valid) {
            float xs, ys, zs;
            scatter_point(g, s, xs, ys, zs);
            const float4 P = __ldg(&g.cry.pos[d]), S = __ldg(&g.cry.size[d]), T = __ldg(&g.cry.trig[d]);
            const DetPoint q = det_point(P, S, T);
            to_crystal_frame(P.x, P.y, P.z, T.z, T.w, xs, ys, zs, r.xss, r.yss, r.zss);   // :1290-1292
            r.lsd = dist3(xs, ys, zs, q.xD, q.yD, q.zD);                                   // :1275
            // absorption chord along the extended scatter->detector ray (:1420-1424)
            const float ux1 = ((float)0 / (float)1 - 0.5f) * S.x, ux2 = (((float)0 + 1.0f) / (float)1 - 0.5f) * S.x;
            const float uy1 = ((float)0 / (float)1 - 0.5f) * S.y, uy2 = (((float)0 + 1.0f) / (float)1 - 0.5f) * S.y;
            const float uz1 = ((float)0 / (float)1 - 0.5f) * S.z, uz2 = (((float)0 + 1.0f) / (float)1 - 0.5f) * S.z;
            const float xt = q.xDs + 1000.0f * (q.xDs - r.xss) / r.lsd;
            const float yt = q.yDs + 1000.0f * (q.yDs - r.yss) / r.lsd;
            const float zt = q.zDs + 1000.0f * (q.zDs - r.zss) / r.lsd;
            r.labs = box_chord(r.xss, r.yss, r.zss, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
            // row-relative start: a row holds at most ns * D entries, which fits an int
            r.att_begin = (int)(offsets[p] - offsets[(long long)d * ns]);
            AttEntry* dst = att + offsets[p];
            int k = 0;
            warp_attenuators<NATIVE>(g, bm_cry, bm_col, s, d, xs, ys, zs, q, lane, list[wid],
                                     [&](int a, float len, bool ok) {
                                         const bool nz = ok && len != 0.0f;
                                         const unsigned m = __ballot_sync(0xffffffffu, nz);
                                         if (nz) {
                                             const float4 mu = __ldg(&g.cry.mu[a]);
                                             dst[k + __popc(m & ((1u << lane) - 1u))] = AttEntry{len, mu.y, mu.z};
                                         }
                                         k += __popc(m);
                                     });
            r.att_count = k;
        }
        if (lane == 0) pairs[p] = r;
    }
}

// Native model: the tungsten terms of each pair, one thread per pair.
__global__ void pair_native_kernel(DevGeom g, int parts, PairNative* nat)
{
    const int ns = g.n_det + g.n_holes;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)g.n_det * ns) return;
    const int d = (int)(p / ns), s = (int)(p - (long long)d * ns);
    PairNative n{};
    if (s >= g.n_det && pair_enabled(g, parts, s, d)) {
        float xs, ys, zs;
        scatter_point(g, s, xs, ys, zs);
        const DetPoint q = det_point(__ldg(&g.cry.pos[d]), __ldg(&g.cry.size[d]), __ldg(&g.cry.trig[d]));
        const int h = s - g.n_det;
        tungsten_path(g, h, xs, ys, zs, q.xD, q.yD, q.zD, n.w_pe, n.w_c);
        const LayerInfo& Ly = g.layer[hole_layer(g, h)];
        n.mu_tot_h = Ly.mu_total;
        n.mu_c_h = Ly.mu_c;
    }
    nat[p] = n;
}

// ---- scatter items ----

struct ElemConst {
    float xI, yI, zI, xIs, yIs, zIs;
    DetPoint q;
    float w, t, h;
    float mu_pe, mu_c, eres;
    float lo, hi;
    float rdet;
    float ux1, ux2, uy1, uy2, uz1, uz2;
};

// One (d, v, s) item; w_s is the interaction weight (PE * muC/muPE or hole solid angle *
// muC/mu of layer 0).  Returns the float the reference would atomically add.
template <bool NATIVE>
__device__ float scatter_item(const ElemConst& e, const PairRec& pr, const PairNative& pn,
                              const AttEntry* __restrict__ att,
                              float xs, float ys, float zs, float w_s, float e0, float integ,
                              const double* __restrict__ kn_tab)
{
    const float cone = cone_angle(e.xI, e.yI, e.zI, xs, ys, zs, e.q.xD, e.q.yD, e.q.zD);
    const float es = e0 / (1.0f + (e0 / 511.0f) * (1.0f - cosf(cone)));     // :1016-1023
    const float res = e.eres * sqrtf(es / e0);
    if ((es * (1 + 2 * res / 2.35482f)) <= e.lo || (es * (1 - 2 * res / 2.35482f)) >= e.hi)
        return 0.0f;                                                         // :1263-1269
    const float pwin = window_prob(es, res, e.lo, e.hi);
    const float sc = sinf(cone);
    float phi;
    if (pr.lsd * sc * 2.0f <= e.rdet) phi = (float)(2.0f * 3.14159265358979323846);
    else {
        const float arg = e.rdet / 2.0f / pr.lsd / sc;
        phi = 4.0f * asinf((arg <= 1.0f) ? arg : 1.0f);
    }
    // theta range over the 8 corners of the (single) detector unit (:1305-1335)
    const float dis = dist3(pr.xss, pr.yss, pr.zss, e.xIs, e.yIs, e.zIs);
    const float xt = pr.xss + 1000.0f * (pr.xss - e.xIs) / dis;
    const float yt = pr.yss + 1000.0f * (pr.yss - e.yIs) / dis;
    const float zt = pr.zss + 1000.0f * (pr.zss - e.zIs) / dis;
    const float lthr = box_chord(e.xIs, e.yIs, e.zIs, xt, yt, zt, e.ux1, e.uy1, e.uz1, e.ux2, e.uy2, e.uz2);
    // The reference takes the extremes of the 8 corner angles acos(c_k); acos decreases, so
    // they are acos(max c_k) and acos(min c_k): two arc cosines instead of eight (the same
    // floats wherever acosf is monotone, which holds to within an ulp at ties).
    float cmin = 2.0f, cmax = -2.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int cx = c & 1, cy = (c >> 1) & 1, cz = c >> 2;
        const float ck = cone_cosine(e.xIs, e.yIs, e.zIs, pr.xss, pr.yss, pr.zss, cx ? e.ux2 : e.ux1,
                                     cy ? e.uy2 : e.uy1, cz ? e.uz2 : e.uz1);
        cmin = fminf(cmin, ck);
        cmax = fmaxf(cmax, ck);
    }
    float tmin = acosf(cmax), tmax = acosf(cmin);
    if (lthr > 0.001f) tmin = 0.0f;
    const int n = (int)((tmax - tmin) / 0.01f);
    const float ratio = (float)kn_sum_tab(tmin, n, kn_tab) / integ;
    // attenuation by the flagged crystals at the scattered energy (:1369-1396)
    // the scaled coefficient depends only on the attenuator's (mu_pe, mu_c) and E': it is
    // recomputed only when those change along the list (same operands, same float)
    float a_sum = 0.0f;
    float c_pe = NAN, c_c = NAN, mt = 0.0f;
    for (int k = 0; k < pr.att_count; ++k) {
        const AttEntry ae = att[pr.att_begin + k];
        if (!(ae.mu_pe == c_pe && ae.mu_c == c_c)) {
            c_pe = ae.mu_pe;
            c_c = ae.mu_c;
            const float mpe = ae.mu_pe * e0 * e0 * e0 / es / es / es;
            const float mc = ae.mu_c * e0 / es;
            mt = mpe + mc;
        }
        a_sum = a_sum + ae.len * mt;
    }
    if (NATIVE && (pn.w_pe != 0.0f || pn.w_c != 0.0f)) {  // native model: tungsten at E'
        const float mpe_w = pn.w_pe * e0 * e0 * e0 / es / es / es;
        const float mc_w = pn.w_c * e0 / es;
        a_sum = a_sum + (mpe_w + mc_w);
    }
    const float mpe_s = e.mu_pe * e0 * e0 * e0 / es / es / es;              // :1411-1417
    const float mc_s = e.mu_c * e0 / es;
    const float mt_s = mpe_s + mc_s;
    const double c = (double)(w_s * phi / 2.0f) * (1.0 / 3.14159265358979323846) * (double)ratio *
                     (double)pwin * (double)expf(-a_sum) *
                     (double)(1.0f - expf(-pr.labs * mt_s)) * (double)mpe_s / (double)mt_s;
    return (float)c;
}

// One block's share of a scatter launch: detector row di, voxels vblock * kItemThreads + t
// (t = threadIdx.x).  sp, spn: the block's pair staging buffers in shared memory.
template <bool NATIVE>
__device__ __forceinline__ void scatter_rows(const DevGeom& g, const ScatterPhysics& ph, const ScatterLaunch& L,
                                             int di, long long vblock, PairRec* sp, PairNative* spn)
{
    const int d = L.det_begin + di;
    const long long vi = vblock * kItemThreads + threadIdx.x;
    const bool active = vi < L.vox_count;
    const long long v = L.vox_begin + (active ? vi : 0);
    const int ns = g.n_det + (NATIVE ? g.n_holes : g.n_holes0);

    const float4 P = __ldg(&g.cry.pos[d]), S = __ldg(&g.cry.size[d]);
    const float4 M = __ldg(&g.cry.mu[d]), T = __ldg(&g.cry.trig[d]);
    const bool run = ph.use_compton && (M.x > 0.01f);                       // :1226-1228

    ElemConst e;
    const float ang = L.rotation * g.angle_step;
    voxel_centre(g, v, cosf(ang), sinf(ang), e.xI, e.yI, e.zI);
    to_crystal_frame(P.x, P.y, P.z, T.z, T.w, e.xI, e.yI, e.zI, e.xIs, e.yIs, e.zIs);
    e.q = det_point(P, S, T);
    e.w = S.x; e.t = S.y; e.h = S.z;
    e.mu_pe = M.y; e.mu_c = M.z; e.eres = M.w;
    if (ph.same_window) { e.lo = ph.lo; e.hi = ph.hi; }
    else {
        e.lo = (1 - e.eres / 2.0f) * ph.e0;                                  // :1161-1162
        e.hi = (1 + e.eres / 2.0f) * ph.e0;
    }
    e.rdet = sqrtf(e.w * e.w / (float)1 / (float)1 + e.h * e.h / (float)1 / (float)1 +
                   e.t * e.t / (float)1 / (float)1) / 2.0f;
    e.ux1 = ((float)0 / (float)1 - 0.5f) * e.w; e.ux2 = (((float)0 + 1.0f) / (float)1 - 0.5f) * e.w;
    e.uy1 = ((float)0 / (float)1 - 0.5f) * e.t; e.uy2 = (((float)0 + 1.0f) / (float)1 - 0.5f) * e.t;
    e.uz1 = ((float)0 / (float)1 - 0.5f) * e.h; e.uz2 = (((float)0 + 1.0f) / (float)1 - 0.5f) * e.h;

    double acc_c = 0.0, acc_h = 0.0;
    const int s_begin = (L.parts & 1) ? 0 : g.n_det;
    const int s_end = (L.parts & 2) ? ns : g.n_det;
    const PairRec* prow = L.pairs + (long long)d * ns;
    const AttEntry* att_row = L.att + L.att_offsets[(long long)d * ns];
    for (int s0 = s_begin; s0 < s_end; s0 += kPairChunk) {
        const int cnt = min(kPairChunk, s_end - s0);
        __syncthreads();
        for (int k = threadIdx.x; k < cnt; k += kItemThreads) {
            sp[k] = prow[s0 + k];
            if constexpr (NATIVE) spn[k] = L.native[(long long)d * ns + s0 + k];
        }
        __syncthreads();
        if (!run || !active) continue;
        for (int k = 0; k < cnt; ++k) {
            const int s = s0 + k;
            const PairRec& pr = sp[k];
            if (!pr.valid) continue;
            float xs, ys, zs, w_s;
            const bool crystal = s < g.n_det;
            if (crystal) {
                w_s = __ldg(&L.pe[(long long)s * g.nvox + v]) * e.mu_c / e.mu_pe;   // :1218-1219
                if (w_s == 0.0f) continue;          // the item is exactly 0
                const float4 ps = __ldg(&g.cry.pos[s]);
                xs = ps.x; ys = ps.y; zs = ps.z;
            } else {
                const float4 hr = __ldg(&g.hole.raw[s - g.n_det]);
                xs = hr.x;
                ys = (hr.y + hr.z) / 2.0f + g.fov;
                zs = hr.w;
                const float lih = dist3(e.xI, e.yI, e.zI, xs, ys, zs);
                float sa;
                if (L.hole_model != 1) {                                  // :1711-1715
                    const float vr = 0.1f;
                    // (pi vr^2 + h vr) / (4 pi lih^2) * |dy| / lih, with one double reciprocal
                    const double rl = 1.0 / (double)lih;
                    sa = (float)(((double)(vr * vr) * 3.14159265358979323846 + (double)((hr.z - hr.y) * vr)) *
                                 (1.0 / (4.0 * 3.14159265358979323846)) * rl * rl * (double)fabsf(ys - e.yI) * rl);
                } else {                                                  // ScatterGen_Collimator :1212-1215
                    const float vr = 0.2f;
                    sa = (vr * vr + (hr.z - hr.y) * vr) / (4.0f * lih * lih);
                }
                if (NATIVE) w_s = sa / spn[k].mu_tot_h * spn[k].mu_c_h;        // the hole's own layer
                else w_s = sa / ph.col_mu_tot0 * ph.col_mu_c0;            // :1716
            }
            // one call site keeps a single copy of the item code
            const double c = (double)scatter_item<NATIVE>(e, pr, spn[NATIVE ? k : 0], att_row, xs, ys, zs, w_s,
                                                          ph.e0, ph.integ, L.kn_tab);
            if (crystal) acc_c += c;
            else acc_h += c;
        }
    }
    if (!active) return;
    float outv;
    if ((L.parts & 3) == 3) outv = (float)acc_h + (float)acc_c;              // :2354-2357
    else if (L.parts & 1) outv = (float)acc_c;
    else outv = (float)acc_h;
    L.out[(long long)di * L.ld + vi] = outv;
}

template <bool NATIVE>
__global__ void __launch_bounds__(kItemThreads)
scatter_kernel(DevGeom g, ScatterPhysics ph, ScatterLaunch L)
{
    __shared__ PairRec sp[kPairChunk];
    __shared__ PairNative spn[NATIVE ? kPairChunk : 1];
    scatter_rows<NATIVE>(g, ph, L, blockIdx.y, blockIdx.x, sp, spn);
}

// Batched scatter: one persistent grid over the (row, voxel block) items of many tasks, taken
// from one counter; a block finds its item's task by binary search over the tasks' first item
// numbers and copies the task (and its geometry, when it changes) into shared memory.  Each
// item runs scatter_rows, so every element equals the single launch's bit for bit.
__global__ void __launch_bounds__(kItemThreads) scatter_batch_kernel(ScatterBatchLaunch B)
{
    __shared__ PairRec sp[kPairChunk];
    __shared__ PairNative spn[kPairChunk];
    __shared__ DevGeom sg;
    __shared__ ScatterTask st;
    __shared__ long long s_item;
    __shared__ int s_task;
    int cur_task = -1, cur_geom = -1;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long item = (long long)atomicAdd(B.work_counter, 1ull);
            int lo = 0, hi = B.n_tasks - 1;
            while (lo < hi) {                       // last task with item_begin <= item
                const int mid = (lo + hi + 1) >> 1;
                if (B.tasks[mid].item_begin <= item) lo = mid; else hi = mid - 1;
            }
            s_item = item;
            s_task = lo;
        }
        __syncthreads();
        const long long item = s_item;
        const int task = s_task;
        __syncthreads();
        if (item >= B.total_items) break;
        if (task != cur_task) {                     // block-uniform
            const int* src = reinterpret_cast<const int*>(B.tasks + task);
            int* dst = reinterpret_cast<int*>(&st);
            for (int i = threadIdx.x; i < (int)(sizeof(ScatterTask) / sizeof(int)); i += kItemThreads) dst[i] = src[i];
            __syncthreads();
            if (st.geom != cur_geom) {
                const int* gs = reinterpret_cast<const int*>(B.geoms + st.geom);
                int* gd = reinterpret_cast<int*>(&sg);
                for (int i = threadIdx.x; i < (int)(sizeof(DevGeom) / sizeof(int)); i += kItemThreads) gd[i] = gs[i];
                cur_geom = st.geom;
            }
            cur_task = task;
            __syncthreads();
        }
        const long long local = item - st.item_begin;
        const int di = (int)(local / st.n_vblocks);
        const long long vb = local - (long long)di * st.n_vblocks;
        if (st.L.hole_model == 2) scatter_rows<true>(sg, st.ph, st.L, di, vb, sp, spn);
        else scatter_rows<false>(sg, st.ph, st.L, di, vb, sp, spn);
    }
}

}  // namespace

long long bitmap_crystal_words(int n)
{
    const long long pairs = (long long)n * (n + 1) / 2;
    return (pairs * n + 31) / 32;
}

long long bitmap_collimator_words(int n, int nh0)
{
    return ((long long)n * n * nh0 + 31) / 32;
}

int launch_bitmap_crystal(const DevGeom& g, uint32_t* words, cudaStream_t s)
{
    const long long nw = bitmap_crystal_words(g.n_det);
    if (nw == 0) return 0;
    const long long blocks = (nw + 255) / 256;
    bitmap_crystal_kernel<<<(unsigned)blocks, 256, 0, s>>>(g.raw_det, g.n_det, nw, words);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_bitmap_collimator(const DevGeom& g, uint32_t* words, cudaStream_t s)
{
    const long long nw = bitmap_collimator_words(g.n_det, g.n_holes0);
    if (nw == 0) return 0;
    const long long blocks = (nw + 255) / 256;
    bitmap_collimator_kernel<<<(unsigned)blocks, 256, 0, s>>>(g.raw_det, g.hole.raw, g.n_det,
                                                              g.n_holes0, nw, words);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <bool NATIVE>
static int build_pairs(const DevGeom& g, int parts, const uint32_t* bm_cry, const uint32_t* bm_col,
                       ScatterScratch& scratch, PairRec** pairs, PairNative** native, AttEntry** att,
                       long long** att_offsets, cudaStream_t s)
{
    const int ns = g.n_det + (NATIVE ? g.n_holes : g.n_holes0);
    const long long np = (long long)g.n_det * ns;
    // layout: [counts (np+1)][64-bit offsets (np+1)][cub temp][pairs][native][att]
    size_t temp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, (long long*)nullptr, (long long*)nullptr, np + 1, s);
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t off_counts = 0;
    const size_t off_offsets = align(off_counts + sizeof(long long) * (np + 1));
    const size_t off_temp = align(off_offsets + sizeof(long long) * (np + 1));
    const size_t off_pairs = align(off_temp + temp_bytes);
    const size_t off_native = align(off_pairs + sizeof(PairRec) * np);
    const size_t fixed = align(off_native + (NATIVE ? sizeof(PairNative) * np : 0));
    if (scratch.bytes < fixed) {
        scatter_scratch_free(scratch);
        if (cudaMalloc(&scratch.base, fixed) != cudaSuccess) { scratch.base = nullptr; return -2; }
        scratch.bytes = fixed;
    }
    char* base = (char*)scratch.base;
    long long* counts = (long long*)(base + off_counts);
    long long* offsets = (long long*)(base + off_offsets);
    const unsigned blocks = (unsigned)((np + 255) / 256);
    // one warp per pair, grid-stride beyond 148 x 64 blocks (64 per SM of a B200)
    const unsigned warp_blocks = (unsigned)std::min<long long>((np + kPairWarps - 1) / kPairWarps, 148LL * 64);
    pair_count_kernel<NATIVE><<<warp_blocks, 32 * kPairWarps, 0, s>>>(g, parts, bm_cry, bm_col, counts);
    if (cudaMemsetAsync(counts + np, 0, sizeof(long long), s) != cudaSuccess) return -1;
    cub::DeviceScan::ExclusiveSum(base + off_temp, temp_bytes, counts, offsets, np + 1, s);
    long long total = 0;
    if (cudaMemcpyAsync(&total, offsets + np, sizeof(long long), cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    if (total < 0) return -1;
    const size_t need = fixed + sizeof(AttEntry) * (size_t)(total > 0 ? total : 1);
    if (scratch.bytes < need) {
        // grow, keeping nothing but the offsets (re-run the cheap count+scan afterwards)
        scatter_scratch_free(scratch);
        if (cudaMalloc(&scratch.base, need) != cudaSuccess) { scratch.base = nullptr; return -2; }
        scratch.bytes = need;
        base = (char*)scratch.base;
        counts = (long long*)(base + off_counts);
        offsets = (long long*)(base + off_offsets);
        pair_count_kernel<NATIVE><<<warp_blocks, 32 * kPairWarps, 0, s>>>(g, parts, bm_cry, bm_col, counts);
        if (cudaMemsetAsync(counts + np, 0, sizeof(long long), s) != cudaSuccess) return -1;
        cub::DeviceScan::ExclusiveSum(base + off_temp, temp_bytes, counts, offsets, np + 1, s);
    }
    *pairs = (PairRec*)(base + off_pairs);
    PairNative* nat = NATIVE ? (PairNative*)(base + off_native) : nullptr;
    if (native) *native = nat;
    *att = (AttEntry*)(base + fixed);
    *att_offsets = offsets;
    pair_fill_kernel<NATIVE><<<warp_blocks, 32 * kPairWarps, 0, s>>>(g, parts, bm_cry, bm_col, offsets, *pairs, *att);
    if (NATIVE) pair_native_kernel<<<blocks, 256, 0, s>>>(g, parts, nat);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int build_scatter_pairs(const DevGeom& g, int parts, const uint32_t* bm_cry, const uint32_t* bm_col,
                        ScatterScratch& scratch, PairRec** pairs, AttEntry** att, long long** att_offsets,
                        cudaStream_t s)
{
    return build_pairs<false>(g, parts, bm_cry, bm_col, scratch, pairs, nullptr, att, att_offsets, s);
}

int build_scatter_pairs_native(const DevGeom& g, int parts, const uint32_t* bm_cry, ScatterScratch& scratch,
                               PairRec** pairs, PairNative** native, AttEntry** att, long long** att_offsets,
                               cudaStream_t s)
{
    return build_pairs<true>(g, parts, bm_cry, nullptr, scratch, pairs, native, att, att_offsets, s);
}

int scatter_batch_blocks_per_sm()
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scatter_batch_kernel, kItemThreads, 0) != cudaSuccess)
        return 1;
    return per_sm < 1 ? 1 : per_sm;
}

int launch_scatter_batch(const ScatterBatchLaunch& B, int grid, cudaStream_t s)
{
    if (B.n_tasks < 1 || B.total_items < 1) return 0;
    scatter_batch_kernel<<<grid, kItemThreads, 0, s>>>(B);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_scatter(const DevGeom& g, const ScatterPhysics& ph, const ScatterLaunch& L, cudaStream_t s)
{
    if (L.det_count == 0 || L.vox_count == 0) return 0;
    dim3 grid((unsigned)((L.vox_count + kItemThreads - 1) / kItemThreads), (unsigned)L.det_count);
    if (L.hole_model == 2) scatter_kernel<true><<<grid, kItemThreads, 0, s>>>(g, ph, L);
    else scatter_kernel<false><<<grid, kItemThreads, 0, s>>>(g, ph, L);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static double kn_shape_sin(double th, double alpha)
{
    const double c = std::cos(th), sn = std::sin(th);
    const double f1 = alpha * (1.0 - c), f2 = 1.0 + c * c, p = 1.0 + f1;
    return f2 / p / p * (1.0 + f1 * f1 / f2 / p) * sn;
}

static double kn_shape_sin_prime(double th, double alpha)
{
    const double c = std::cos(th), s = std::sin(th), om = 1.0 - c, p = 1.0 + alpha * om;
    const double g = (1.0 + c * c) / (p * p) + alpha * alpha * om * om / (p * p * p);
    const double gp = 2.0 * c / (p * p) + 2.0 * alpha * (1.0 + c * c) / (p * p * p) -
                      2.0 * alpha * alpha * om / (p * p * p) + 3.0 * alpha * alpha * alpha * om * om / (p * p * p * p);
    return c * g - s * s * gp;
}

void kn_table_build(double e0, double* tab)
{
    const int N = kKnTable;
    const double alpha = e0 / 511.0, hc = 3.14159265358979323846 / N;
    static const double xg[4] = {0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363};
    static const double wg[4] = {0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
    double G = 0.0;
    for (int i = 0; i <= N; ++i) {
        const double th = i * hc;
        if (i > 0) {                       // exact-to-rounding 8-point Gauss-Legendre per cell
            const double mid = th - 0.5 * hc, half = 0.5 * hc;
            double acc = 0.0;
            for (int k = 0; k < 4; ++k)
                acc += wg[k] * (kn_shape_sin(mid - half * xg[k], alpha) + kn_shape_sin(mid + half * xg[k], alpha));
            G += half * acc;
        }
        tab[i] = G;
        tab[(N + 1) + i] = kn_shape_sin(th, alpha);
        tab[2 * (N + 1) + i] = kn_shape_sin_prime(th, alpha);
    }
}

double kn_normalisation(double e0)
{
    const float step = 0.01f;
    const int n = (int)((float)3.14159265358979323846 / step);
    const double alpha = e0 / 511.0;
    double sum = 0.0;
    for (int i = 0; i <= n; ++i) {
        const double th = (double)((float)i * step);
        const double c = std::cos(th), sn = std::sin(th);
        const double f1 = alpha * (1.0 - c), f2 = 1.0 + c * c, p = 1.0 + f1;
        sum += f2 / p / p * (1.0 + f1 * f1 / f2 / p) * sn * (double)step;
    }
    return sum;
}

}  // namespace sysmat
