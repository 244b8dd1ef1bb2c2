// Photoelectric system-matrix kernel for sm_100a.
//
// Computes A[d][v] = sum over the 8x16x8 sub-elements s of crystal d of
//   Omega_s * exp(-sum mu L) * (1 - exp(-mu_d L_abs,s)) * mu_pe,d / mu_d
// as the reference kernel photodetectorCudaMe defines it
// (PEGen_RayTracing_CircularHole/PESysMatGen.cu:951-1364), with a different execution plan:
//
//  * a block owns one crystal d and a 4x4x2 brick of voxels (work items handed out by an
//    atomic counter over a persistent grid); one warp per matrix element; the 32 lanes
//    take 32 consecutive sub-elements per round, 32 rounds;
//  * candidate culling runs in three stages.  (1) Block: a conservative superset of the
//    reference's cone test (:1105-1186) for every voxel of the brick, from the brick's
//    centre and radius, is compacted into shared memory in the reference's object order.
//    (2) Warp: the reference cone test itself, with the reference's float formula, on the
//    superset; a passing object is kept only if its direction-slope rectangle (dx/dy,
//    dz/dy seen from the voxel) overlaps the one of crystal d.  (3) Lane: an object whose
//    rectangle does not contain the sub-element ray's slope is skipped.  A skipped object
//    has an exactly-zero chord in the reference, and adding 0 or fma(mu, 0, x) leaves a
//    float unchanged, so no stage changes any float result;
//  * when an element has more kept objects than one shared-memory chunk holds, the warp
//    walks them chunk by chunk for every round, in the same order, so the attenuation
//    sums keep the reference's order;
//  * the plate-bypass penalty (:1240-1254) is skipped for rays whose slope lies inside the
//    plate's "through both faces" rectangle, where the chord is >= T >= 0.2 mm;
//  * sub-elements whose plate penalty fired contribute exp(-(>=1e5)) = 0 and stop early
//    (only when every attenuation coefficient is non-negative);
//  * the element sum is one float chain in the reference's sub-element order
//    (SYSMAT_MODE_REFERENCE, the reference's atomicAdd sequence at :1359) or an FP64
//    accumulation (SYSMAT_MODE_PRECISE); lane 0 writes dst[d][v].
//
// Two more instances share the execution plan: the FP64 mode (SYSMAT_MODE_FP64,
// pe_fp64.cuh: the element program in double, culling in float) and the sampled form
// (pe_element_sampled: crystal divisions and voxel source points as parameters).
#include "chord64.cuh"
#include "geom.cuh"
#include "pe.cuh"

namespace sysmat {

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kSuperCap = 1024;         // block superset capacity (objects)
constexpr int kChunk = 256;             // per-warp kept-object chunk
constexpr int kRound = 64;              // per-warp round buffer
constexpr float kSlopeMargin = 2e-4f;   // slope units; >> FP32 position error / depth
constexpr float kMinDepth = 1.0f;       // mm; slope rectangles need objects this far behind

struct WarpSmem {
    // kept objects of the element (reference cone test + bundle filter), reference order
    float4 rect[kChunk];
    int id[kChunk];                      // holes: hole index; crystals: n_holes + crystal
    // the current round's objects (kept objects whose rectangle meets the round's rays),
    // with their geometry, so the walk reads contiguous shared memory:
    //   hole:    A = (x, z, R, mu),   B = (y1, y2, -, -)
    //   crystal: A = (x, y, z, mu),   B = (cos(-rot), sin(-rot), w, t),
    //            C = (h, voxel x, y, z in the crystal's frame)
    float4 rr[kRound], ra[kRound], rb[kRound], rc[kRound];
    int rl[kRound];                      // layer of a hole entry; n_layers for crystals
    float4 inner[kMaxLayers];            // plate "through both faces" slope rectangle
    union {
        float chain[256];                // contributions of sub-elements 256p .. 256p+255
        double e64[32];                  // FP64 mode: the element's constants (Elem64)
    };
};

struct BlockSmem {
    float4 sdata[kSuperCap];             // holes: x, (y1+y2)/2, z, crit; crystals: x, y, z, diag
    int sid[kSuperCap];
    int warp_cnt[kWarps];
    int s_count;                         // superset size; -1 = superset overflowed, use all
    long long item;
    WarpSmem w[kWarps];
};

__device__ __forceinline__ bool in_rect(const float4& r, float a, float b)
{
    return a >= r.x && a <= r.y && b >= r.z && b <= r.w;
}

__device__ __forceinline__ bool rects_overlap(const float4& p, const float4& q)
{
    return p.x <= q.y && q.x <= p.y && p.z <= q.w && q.z <= p.w;
}

__device__ __forceinline__ float4 open_rect()
{
    return make_float4(-INFINITY, INFINITY, -INFINITY, INFINITY);
}

// Slope rectangle of a crystal box seen from (px, py, pz), widened by the margin; the open
// rectangle if any corner is closer than kMinDepth in y.
__device__ float4 crystal_rect(float4 pos, float4 size, float4 trig, float px, float py, float pz)
{
    const float hw = 0.5f * size.x, ht = 0.5f * size.y, hh = 0.5f * size.z;
    const float y0 = pos.y - ht - py, y1 = pos.y + ht - py;
    if (!(y0 >= kMinDepth)) return open_rect();
    const float r0 = 1.0f / y0, r1 = 1.0f / y1;
    float amin = INFINITY, amax = -INFINITY, bmin = INFINITY, bmax = -INFINITY;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float xs = (c & 1) ? hw : -hw;
        const float zs = (c & 2) ? hh : -hh;
        const float x = pos.x + (xs * trig.x - zs * trig.y) - px;
        const float z = pos.z + (xs * trig.y + zs * trig.x) - pz;
        amin = fminf(amin, fminf(x * r0, x * r1));
        amax = fmaxf(amax, fmaxf(x * r0, x * r1));
        bmin = fminf(bmin, fminf(z * r0, z * r1));
        bmax = fmaxf(bmax, fmaxf(z * r0, z * r1));
    }
    return make_float4(amin - kSlopeMargin, amax + kSlopeMargin, bmin - kSlopeMargin,
                       bmax + kSlopeMargin);
}

__device__ float4 hole_rect(float4 ha, float r, float px, float py, float pz)
{
    const float y0 = ha.y - py, y1 = ha.z - py;
    if (!(y0 >= kMinDepth) || !(y1 >= kMinDepth)) return open_rect();
    const float r0 = 1.0f / y0, r1 = 1.0f / y1;
    const float xa = ha.x - r - px, xb = ha.x + r - px;
    const float za = ha.w - r - pz, zb = ha.w + r - pz;
    const float amin = fminf(fminf(xa * r0, xa * r1), fminf(xb * r0, xb * r1));
    const float amax = fmaxf(fmaxf(xa * r0, xa * r1), fmaxf(xb * r0, xb * r1));
    const float bmin = fminf(fminf(za * r0, za * r1), fminf(zb * r0, zb * r1));
    const float bmax = fmaxf(fmaxf(za * r0, za * r1), fmaxf(zb * r0, zb * r1));
    return make_float4(amin - kSlopeMargin, amax + kSlopeMargin, bmin - kSlopeMargin,
                       bmax + kSlopeMargin);
}

// Object i in the reference's order: holes 0..H-1 (layer by layer), then crystals.
__device__ __forceinline__ float4 object_data(const DevGeom& g, int i)
{
    if (i < g.n_holes) {
        const float4 a = __ldg(&g.hole.a[i]);
        const float4 b = __ldg(&g.hole.b[i]);
        return make_float4(a.x, b.z, a.w, b.w);
    }
    const float4 p = __ldg(&g.cry.pos[i - g.n_holes]);
    return make_float4(p.x, p.y, p.z, __ldg(&g.cry.size[i - g.n_holes].w));
}

__device__ __forceinline__ int layer_of_hole(const DevGeom& g, int h)
{
    int m = 0;
    while (m + 1 < g.n_layers && h >= g.layer[m + 1].hole_begin) ++m;
    return m;
}

// Per-element constants shared by the lanes of a warp.
struct Elem {
    float xI, yI, zI;            // voxel centre (rotated)
    float xIs, yIs, zIs;         // voxel in crystal d's frame
    float xd, yd, zd, w, t, h;   // crystal d
    float cosr, sinr;
    float mu_t, mu_pe;
    float ux, uy, uz, crit_self; // reference cone test (:1110-1116)
    float4 rd;                   // slope rectangle of crystal d
    bool filt;
};

// Reference cone test of object i against element e (:1120-1184), then the bundle filter.
// Returns true if the object is kept; rect receives its slope rectangle.
__device__ __forceinline__ bool keep_object(const DevGeom& g, const Elem& e, int i, float4 od,
                                            int d, float4& rect)
{
    rect = open_rect();
    bool keep;
    if (i < g.n_holes) {
        const float L = sqrtf((e.xI - od.x) * (e.xI - od.x) + (e.yI - od.y) * (e.yI - od.y) +
                              (e.zI - od.z) * (e.zI - od.z));
        const float crit = od.w / L;
        const float vx = (od.x - e.xI) / L, vy = (od.y - e.yI) / L, vz = (od.z - e.zI) / L;
        keep = sqrtf((vz - e.uz) * (vz - e.uz) + (vy - e.uy) * (vy - e.uy) + (vx - e.ux) * (vx - e.ux)) <=
               crit + e.crit_self;
        if (keep && e.filt) {
            rect = hole_rect(__ldg(&g.hole.a[i]), __ldg(&g.hole.b[i].x), e.xI, e.yI, e.zI);
            keep = rects_overlap(rect, e.rd);
        }
    } else {
        const int o = i - g.n_holes;
        if (o == d) return false;
        const float L = sqrtf((e.xI - od.x) * (e.xI - od.x) + (e.yI - od.y) * (e.yI - od.y) +
                              (e.zI - od.z) * (e.zI - od.z));
        const float crit = od.w / L / 2.0f;
        const float vx = (od.x - e.xI) / L, vy = (od.y - e.yI) / L, vz = (od.z - e.zI) / L;
        keep = sqrtf((vz - e.uz) * (vz - e.uz) + (vy - e.uy) * (vy - e.uy) + (vx - e.ux) * (vx - e.ux)) <=
               crit + e.crit_self;
        if (keep && e.filt) {
            rect = crystal_rect(__ldg(&g.cry.pos[o]), __ldg(&g.cry.size[o]), __ldg(&g.cry.trig[o]),
                                e.xI, e.yI, e.zI);
            keep = rects_overlap(rect, e.rd);
        }
    }
    return keep;
}

// Fill the warp's chunk with kept objects, scanning source positions [cursor, n_src).
// Source = block superset (n_src = s_count) or all objects.  Returns the new cursor; the
// chunk count goes to *count.  Stops early when the chunk could overflow.
__device__ int build_chunk(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws, const Elem& e,
                           int d, int cursor, int n_src, bool from_super, int lane, int* count)
{
    int n = 0;
    while (cursor < n_src && n <= kChunk - 32) {
        const int j = cursor + lane;
        bool keep = false;
        float4 rect;
        int id = 0;
        if (j < n_src) {
            id = from_super ? bs.sid[j] : j;
            const float4 od = from_super ? bs.sdata[j] : object_data(g, j);
            keep = keep_object(g, e, id, od, d, rect);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int pos = n + __popc(m & ((1u << lane) - 1u));
            ws.rect[pos] = rect;
            ws.id[pos] = id;
        }
        n += __popc(m);
        cursor += 32;
    }
    __syncwarp();
    *count = n;
    return cursor < n_src ? cursor : n_src;
}

// Attenuation walk state of one lane (one sub-element).
struct Walk {
    float att;      // accumulated mu * L
    float len;      // hole chord sum of the current layer
    int lay;        // current layer
    int hole_hits;  // non-zero hole chords (work counters only)
    int cry_hits;   // non-zero crystal chords (work counters only)
    int hole_evals; // hole chords evaluated (work counters only)
    int cry_evals;  // crystal chords evaluated (work counters only)
};

__device__ __forceinline__ void close_layers(const DevGeom& g, Walk& s, int upto, float cosang)
{
    while (s.lay < upto) {                                    // :1281-1284
        const float lcol = g.layer[s.lay].thickness / cosang;
        if ((lcol - s.len) >= 0.00001f) s.att = s.att + g.layer[s.lay].mu_total * (lcol - s.len);
        s.len = 0.0f;
        ++s.lay;
    }
}

// Terms of the reference cylinder chord (PESysMatGen.cu:688-799) that depend only on the
// ray (voxel -> sub-element) and on the cap planes y1, y2.  Hoisting them out of the
// per-hole evaluation keeps every float identical: each is the same operation on the same
// operands as in the per-hole formula.
struct RayCyl {
    float xi, yi, zi, tio, kx, ky, kz, rx, rz, kk;
    float y1, y2;                // cap planes the cached terms below belong to
    bool degenerate;             // |y1 - y2| < 0.001
    float ta, tb, xl, xr, zl, zr;
};

__device__ __forceinline__ void ray_cyl_init(RayCyl& c, float xi, float yi, float zi, float xo, float yo,
                                             float zo)
{
    const float dx = xo - xi, dy = yo - yi, dz = zo - zi;
    c.xi = xi; c.yi = yi; c.zi = zi;
    c.tio = sqrtf(dx * dx + dy * dy + dz * dz);
    c.kx = dx / c.tio;
    c.ky = dy / c.tio;
    c.kz = dz / c.tio;
    c.rx = c.kx / c.ky;
    c.rz = c.kz / c.ky;
    c.kk = c.kx * c.kx + c.kz * c.kz;
    c.y1 = NAN;                  // no cap planes cached yet (NaN never compares equal)
    c.y2 = NAN;
}

__device__ __forceinline__ void ray_cyl_caps(RayCyl& c, float y1, float y2)
{
    if (y1 == c.y1 && y2 == c.y2) return;
    c.y1 = y1;
    c.y2 = y2;
    c.degenerate = fabsf(y1 - y2) < 0.001f;
    c.xl = c.xi + c.rx * (y1 - c.yi);
    c.xr = c.xi + c.rx * (y2 - c.yi);
    c.zl = c.zi + c.rz * (y1 - c.yi);
    c.zr = c.zi + c.rz * (y2 - c.yi);
    c.ta = (y1 - c.yi) / c.ky;
    c.tb = (y2 - c.yi) / c.ky;
}

// Cylinder chord of hole (xc, zc, r) with cap planes already cached in c.
__device__ __forceinline__ float ray_cyl_chord(const RayCyl& c, float xc, float zc, float r)
{
    if (c.degenerate) return 0.0f;
    const bool fl = (c.xl - xc) * (c.xl - xc) + (c.zl - zc) * (c.zl - zc) <= r * r;
    const bool fr = (c.xr - xc) * (c.xr - xc) + (c.zr - zc) * (c.zr - zc) <= r * r;
    if (fl && fr) {
        if (c.ta <= 0.0001f || c.tb <= 0.0001f) return 0.0f;
        if (c.ta >= c.tio || c.tb >= c.tio) return 0.0f;
        return fabsf(c.tb - c.ta);
    }
    const float ox = c.xi - xc, oz = c.zi - zc;
    const float disc = c.kk * r * r - (c.kx * oz - c.kz * ox) * (c.kx * oz - c.kz * ox);
    if (disc <= 0.00001f) return 0.0f;
    const float t1 = (-(c.kx * ox + c.kz * oz) - sqrtf(disc)) / c.kk;
    const float t2 = (-(c.kx * ox + c.kz * oz) + sqrtf(disc)) / c.kk;
    float ea, eb;
    if (!fl && !fr) {
        if (!(t1 >= c.ta && t2 <= c.tb)) return 0.0f;
        ea = t1; eb = t2;
    } else if (fl) { ea = c.ta; eb = t2; }
    else           { ea = t1; eb = c.tb; }
    if (eb <= 0.0001f || ea <= 0.0001f) return 0.0f;
    if (eb >= c.tio || ea >= c.tio) return 0.0f;
    return eb - ea;
}

// Slope-space shadow of a y-aligned object (hole cylinder, or crystal in the disk around its
// xz footprint) seen from the voxel: every line from the voxel that meets the object at a
// depth y in [y0, y1] has slopes within rho(y) = R/(y - yI) of the point c(y) on the
// segment c(y0) -> c(y1), so within rho(y0) of that segment (the capsule; its radius is
// inflated by the slope margin).
struct Capsule {
    float ax, az, dx, dz, rho;    // c(y0), c(y1) - c(y0), radius
};

__device__ __forceinline__ Capsule capsule_of(float xo, float zo, float y0, float y1, float R, const Elem& e)
{
    const float r0 = __frcp_rn(y0 - e.yI), r1 = __frcp_rn(y1 - e.yI);
    Capsule c;
    c.ax = (xo - e.xI) * r0;
    c.az = (zo - e.zI) * r0;
    c.dx = (xo - e.xI) * r1 - c.ax;
    c.dz = (zo - e.zI) * r1 - c.az;
    c.rho = R * r0 * 1.0001f + kSlopeMargin;
    return c;
}

// False only when the capsule is separated from the box along x, along z, or along the
// segment's normal; decided without divisions.
__device__ __forceinline__ bool capsule_meets_box(const Capsule& c, float4 box)
{
    const float bx = c.ax + c.dx, bz = c.az + c.dz, rho = c.rho;
    if (fminf(c.ax, bx) - rho > box.y || fmaxf(c.ax, bx) + rho < box.x) return false;
    if (fminf(c.az, bz) - rho > box.w || fmaxf(c.az, bz) + rho < box.z) return false;
    const float mx = 0.5f * (box.x + box.y) - c.ax, mz = 0.5f * (box.z + box.w) - c.az;
    const float sep = fabsf(c.dx * mz - c.dz * mx) - (fabsf(c.dz) * 0.5f * (box.y - box.x) +
                                                      fabsf(c.dx) * 0.5f * (box.w - box.z));
    return !(sep > 0.0f && sep * sep > rho * rho * (c.dx * c.dx + c.dz * c.dz));
}

__device__ __forceinline__ bool capsule_meets_box(float xo, float zo, float y0, float y1, float R,
                                                  const Elem& e, float4 box)
{
    return capsule_meets_box(capsule_of(xo, zo, y0, y1, R, e), box);
}

// Lane test of a hole entry of the round buffer: is the ray's slope (sa, sb) within the
// hole's capsule?  c = (c(y0), c(y1) - c(y0)), rho2 = radius^2 (infinite for an entry without
// a capsule: the hole is closer than kMinDepth to the voxel), inv_len2 = 1/|c(y1) - c(y0)|^2
// (0 for a degenerate segment).
__device__ __forceinline__ bool in_capsule(const float4& c, float rho2, float inv_len2, float sa, float sb)
{
    const float px = sa - c.x, pz = sb - c.y;
    const float t = fminf(fmaxf((px * c.z + pz * c.w) * inv_len2, 0.0f), 1.0f);
    const float ex = px - t * c.z, ez = pz - t * c.w;
    return ex * ex + ez * ez <= rho2;
}

// Copy kept entries [k0, k1) whose rectangle and capsule meet the round's slope box into
// the round buffer from position n, with their geometry (one entry per lane); returns the
// new count.  Stops before the buffer could overflow; *next receives the first entry not
// examined.  IDS: store each entry's object id (as the bits of ra.x) instead of its float
// geometry, for walks that read their own geometry tables (FP64 mode), and a hole entry's
// capsule in place of its rectangle for the lanes' test (hole_in_reach).  The float walks
// test the rectangle: the warp runs an entry's chord whenever any lane needs it, and the
// tighter lane test measured slower there (its cost without fewer warp-level evaluations).
template <bool ELL, bool IDS = false>
__device__ __forceinline__ int fill_round(const DevGeom& g, WarpSmem& ws, const Elem& e, int k0, int k1,
                                          float4 box, int n, int lane, int* next, int* nh)
{
    int k = k0;
    while (k < k1 && n <= kRound - 32) {
        const int kk = k + lane;
        bool keep = false;
        int id = 0;
        float4 rect;
        // hole entries carry their capsule for the lanes' test (none: every slope passes)
        float4 cap = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float rho2 = INFINITY, inv_len2 = 0.0f;
        if (kk < k1) {
            rect = ws.rect[kk];
            keep = rects_overlap(rect, box);
            if (keep && !isinf(rect.x)) {                  // finite: object wholly behind the voxel
                id = ws.id[kk];
                if (id < g.n_holes) {
                    const float4 ha = __ldg(&g.hole.a[id]);
                    const Capsule c = capsule_of(ha.x, ha.w, ha.y, ha.z, __ldg(&g.hole.b[id].x), e);
                    keep = capsule_meets_box(c, box);
                    cap = make_float4(c.ax, c.az, c.dx, c.dz);
                    rho2 = c.rho * c.rho;
                    const float l2 = c.dx * c.dx + c.dz * c.dz;
                    inv_len2 = l2 > 1e-30f ? __frcp_rn(l2) : 0.0f;
                } else {
                    const int o = id - g.n_holes;
                    const float4 po = __ldg(&g.cry.pos[o]);
                    const float4 so = __ldg(&g.cry.size[o]);
                    keep = capsule_meets_box(po.x, po.z, po.y - 0.5f * so.y, po.y + 0.5f * so.y,
                                             0.5f * sqrtf(so.x * so.x + so.z * so.z), e, box);
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) id = ws.id[kk];
        *nh += __popc(__ballot_sync(0xffffffffu, keep && id < g.n_holes));
        if (keep) {
            const int pos = n + __popc(m & ((1u << lane) - 1u));
            if constexpr (IDS) {
                ws.rr[pos] = id < g.n_holes ? cap : rect;
                ws.rb[pos] = make_float4(0.0f, 0.0f, rho2, inv_len2);
                ws.ra[pos].x = __int_as_float(id);
                ws.rl[pos] = id < g.n_holes ? layer_of_hole(g, id) : g.n_layers;
            } else if (id < g.n_holes) {
                const float4 ha = __ldg(&g.hole.a[id]);
                const float4 hb = __ldg(&g.hole.b[id]);
                ws.rr[pos] = rect;
                ws.ra[pos] = make_float4(ha.x, ha.w, hb.x, hb.y);
                ws.rb[pos] = make_float4(ha.y, ha.z, 0.0f, 0.0f);
                if constexpr (ELL) {        // rho_x, rho_z, cos, sin; a batch may mix in circular systems
                    ws.rc[pos] = g.hole_shape ? __ldg(&g.hole_shape[id]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                }
                ws.rl[pos] = layer_of_hole(g, id);
            } else {
                const int o = id - g.n_holes;
                const float4 po = __ldg(&g.cry.pos[o]);
                const float4 so = __ldg(&g.cry.size[o]);
                const float4 to = __ldg(&g.cry.trig[o]);
                float xa, ya, za;                                   // :1305-1307
                to_crystal_frame(po.x, po.y, po.z, to.z, to.w, e.xI, e.yI, e.zI, xa, ya, za);
                ws.rr[pos] = rect;
                ws.ra[pos] = make_float4(po.x, po.y, po.z, __ldg(&g.cry.mu[o].x));
                ws.rb[pos] = make_float4(to.z, to.w, so.x, so.y);
                ws.rc[pos] = make_float4(so.z, xa, ya, za);
                ws.rl[pos] = g.n_layers;
            }
        }
        n += __popc(m);
        k += 32;
    }
    __syncwarp();
    *next = k < k1 ? k : k1;
    return n;
}

// Lane test of round-buffer hole entry j of a fill_round<…, IDS> buffer (see in_capsule).
__device__ __forceinline__ bool hole_in_reach(const WarpSmem& ws, int j, float sa, float sb)
{
    const float4 b = ws.rb[j];
    return in_capsule(ws.rr[j], b.z, b.w, sa, sb);
}

// Walk round-buffer entries [0, nr) for one sub-element ray (voxel -> (xD, yD, zD)); holes
// occupy [0, nh) and crystals [nh, nr), both in the reference's object order; the layer
// terms are added when the walk leaves a layer.
template <bool ELL>
__device__ __forceinline__ void walk_round(const DevGeom& g, const WarpSmem& ws, int nh, int nr,
                                           float xD, float yD, float zD, float sa_a, float sa_b,
                                           float cosang, RayCyl& rc, Walk& s)
{
    // the next entry's layer and rectangle are loaded one iteration ahead (shared-memory
    // latency off the dependency chain: 4-5 % on the reference mode, same results)
    int m_next = nh > 0 ? ws.rl[0] : 0;
    float4 r_next = nh > 0 ? ws.rr[0] : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = 0; j < nh; ++j) {
        const int m = m_next;
        const float4 R = r_next;
        if (j + 1 < nh) {
            m_next = ws.rl[j + 1];
            r_next = ws.rr[j + 1];
        }
        if (m != s.lay) close_layers(g, s, m, cosang);
        if (!in_rect(R, sa_a, sa_b)) continue;
        const float4 A = ws.ra[j];
        const float4 B = ws.rb[j];
        float tmp;
        if constexpr (ELL) {
            const float4 S = ws.rc[j];
            if (S.x > 0.0f) {                                    // elliptical hole
                tmp = ell_chord(rc.xi, rc.yi, rc.zi, xD, yD, zD, A.x, B.x, B.y, A.y, S.x, S.y, S.z, S.w);
            } else {
                ray_cyl_caps(rc, B.x, B.y);
                tmp = ray_cyl_chord(rc, A.x, A.y, A.z);
            }
        } else {
            ray_cyl_caps(rc, B.x, B.y);
            tmp = ray_cyl_chord(rc, A.x, A.y, A.z);
        }
        s.len = s.len + tmp;                                     // :1276-1278
        s.att = s.att + A.w * tmp;
        s.hole_hits += (tmp != 0.0f);
        ++s.hole_evals;
    }
    if (nr <= nh) return;
    if (s.lay < g.n_layers) close_layers(g, s, g.n_layers, cosang);
    float4 c_next = ws.rr[nh];
    for (int j = nh; j < nr; ++j) {
        const float4 R = c_next;
        if (j + 1 < nr) c_next = ws.rr[j + 1];
        if (!in_rect(R, sa_a, sa_b)) continue;
        const float4 A = ws.ra[j];
        const float4 B = ws.rb[j];
        const float4 C = ws.rc[j];
        float xb, yb, zb;                                        // :1318-1320
        to_crystal_frame(A.x, A.y, A.z, B.x, B.y, xD, yD, zD, xb, yb, zb);
        const float la = box_chord(C.y, C.z, C.w, xb, yb, zb, -0.5f * B.z, -0.5f * B.w, -0.5f * C.x,
                                   0.5f * B.z, 0.5f * B.w, 0.5f * C.x);
        s.att = s.att + la * A.w;
        s.cry_hits += (la != 0.0f);
        ++s.cry_evals;
    }
}

struct SubElem {
    int ix, iy, iz;
    float xDs, yDs, zDs, xD, yD, zD, dsq, sq, cosang, sa_a, sa_b;
};

// Sub-element (ix, iy, iz) of a crystal divided into fx x fy x fz (x, depth, z) parts.
__device__ __forceinline__ SubElem sub_element_at(const Elem& e, int ix, int iy, int iz, float fx, float fy,
                                                  float fz)
{
    SubElem q;
    q.iz = iz;
    q.ix = ix;
    q.iy = iy;
    q.xDs = -e.w / 2.0f + ((float)q.ix + 0.5f) / fx * e.w;   // :1207-1217
    q.zDs = -e.h / 2.0f + ((float)q.iz + 0.5f) / fz * e.h;
    q.yDs = -e.t / 2.0f + ((float)q.iy + 0.5f) / fy * e.t;
    q.xD = e.xd + (q.xDs * e.cosr - q.zDs * e.sinr);
    q.zD = e.zd + (q.xDs * e.sinr + q.zDs * e.cosr);
    q.yD = e.yd + q.yDs;
    q.dsq = (q.yD - e.yI) * (q.yD - e.yI) + (q.xD - e.xI) * (q.xD - e.xI) + (q.zD - e.zI) * (q.zD - e.zI);
    q.sq = sqrtf(q.dsq);
    q.cosang = (q.yD - e.yI) / q.sq;
    if (e.filt) {             // every sub-element lies >= kMinDepth behind the voxel
        const float rdy = __frcp_rn(q.yD - e.yI);
        q.sa_a = (q.xD - e.xI) * rdy;
        q.sa_b = (q.zD - e.zI) * rdy;
    } else {                  // all rectangles are open: any finite slope passes
        q.sa_a = 0.0f;
        q.sa_b = 0.0f;
    }
    return q;
}

// Reference sub-element s = 128 iz + 16 ix + iy of the 8 x 16 x 8 division.
__device__ __forceinline__ SubElem sub_element(const Elem& e, int s)
{
    return sub_element_at(e, (s >> 4) & 7, s & 15, s >> 7, 8.0f, 16.0f, 8.0f);
}

// Plate penalty (:1240-1254); true if any layer fired.
__device__ __forceinline__ bool plate_penalty(const DevGeom& g, const WarpSmem& ws, const Elem& e,
                                              const SubElem& q, float& att)
{
    bool blocked = false;
    for (int m = 0; m < g.n_layers; ++m) {
        if (in_rect(ws.inner[m], q.sa_a, q.sa_b)) continue;
        const LayerInfo& Ly = g.layer[m];
        const float tl = box_chord(e.xI, e.yI, e.zI, q.xD, q.yD, q.zD, Ly.x1, Ly.y1, Ly.z1, Ly.x2,
                                   Ly.y2, Ly.z2);
        if (tl < 0.1f) { att = att + 100000.0f; blocked = true; }
    }
    return blocked;
}

// Self attenuation, absorption and solid angle for a sub-element of an fx x fy x fz
// division, given the attenuation accumulated outside crystal d (:1223-1231, :1329-1357).
__device__ __forceinline__ float finish_sub_element_at(const Elem& e, const SubElem& q, float att, float fx,
                                                       float fy, float fz)
{
    const float w = e.w, t = e.t, h = e.h;
    const float ux1 = ((float)q.ix / fx - 0.5f) * w;
    const float ux2 = (((float)q.ix + 1.0f) / fx - 0.5f) * w;
    const float uy1 = ((float)q.iy / fy - 0.5f) * t;
    const float uy2 = (((float)q.iy + 1.0f) / fy - 0.5f) * t;
    const float uz1 = ((float)q.iz / fz - 0.5f) * h;
    const float uz2 = (((float)q.iz + 1.0f) / fz - 0.5f) * h;
    const float cbox[6] = {-w / 2.0f, -t / 2.0f, -h / 2.0f, w / 2.0f, t / 2.0f, h / 2.0f};
    const float ubox[6] = {ux1, uy1, uz1, ux2, uy2, uz2};
    float l1, l2;
    box_chord_inside2(e.xIs, e.yIs, e.zIs, q.xDs, q.yDs, q.zDs, cbox, ubox, l1, l2);
    att = att + (l1 - l2) * e.mu_t;
    const float eff = 1.0f * expf(-att);
    const float xt = q.xDs + 1000.0f * (q.xDs - e.xIs) / q.sq;
    const float yt = q.yDs + 1000.0f * (q.yDs - e.yIs) / q.sq;
    const float zt = q.zDs + 1000.0f * (q.zDs - e.zIs) / q.sq;
    const float labs = box_chord(e.xIs, e.yIs, e.zIs, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
    const float absf = (1.0f - expf(-labs * e.mu_t)) * e.mu_pe / e.mu_t;
    // solid angle in double, as the reference's 4*M_PI promotion makes it; one shared
    // reciprocal (the float results round identically except in double-rounding ties)
    const double rq = 1.0 / ((4.0 * 3.14159265358979323846) * (double)q.dsq * (double)q.sq);
    const float ax = t * h / fz / fy, az = w * t / fx / fy, ay = w * h / fx / fz;
    const float sax = (float)((double)ax * (double)fabsf((q.xD - e.xI) * e.cosr - (q.zD - e.zI) * e.sinr) * rq);
    const float saz = (float)((double)az * (double)fabsf((q.xD - e.xI) * e.sinr + (q.zD - e.zI) * e.cosr) * rq);
    const float say = (float)((double)ay * (double)fabsf(q.yD - e.yI) * rq);
    const float sxy = (sax >= say) ? sax : say;
    const float sa = (sxy >= saz) ? sxy : saz;
    return eff * sa * absf;
}

__device__ __forceinline__ float finish_sub_element(const Elem& e, const SubElem& q, float att)
{
    return finish_sub_element_at(e, q, att, 8.0f, 16.0f, 8.0f);
}

// Per-element set-up shared by the lanes of a warp: voxel centre, crystal d, reference cone
// constants, slope rectangle and the plate "through both faces" rectangles.  False when the
// crystal's attenuation is too low for the reference to compute the element (it is 0).
__device__ __forceinline__ bool init_element(const DevGeom& g, WarpSmem& ws, int d, long long v, float cr,
                                             float sr, int lane, Elem& e, float fx = 0.5f, float fy = 0.5f,
                                             float fz = 0.5f)
{
    voxel_centre(g, v, cr, sr, e.xI, e.yI, e.zI, fx, fy, fz);   // the source point in the voxel
    const float4 P = __ldg(&g.cry.pos[d]);
    const float4 S = __ldg(&g.cry.size[d]);
    const float4 M = __ldg(&g.cry.mu[d]);
    const float4 T = __ldg(&g.cry.trig[d]);
    e.xd = P.x; e.yd = P.y; e.zd = P.z;
    e.w = S.x; e.t = S.y; e.h = S.z;
    e.mu_t = M.x; e.mu_pe = M.y;
    e.cosr = T.x; e.sinr = T.y;
    if (!(e.mu_t > 0.01f)) return false;                   // :1107, :1194
    to_crystal_frame(e.xd, e.yd, e.zd, T.z, T.w, e.xI, e.yI, e.zI, e.xIs, e.yIs, e.zIs);
    const float dist = sqrtf((e.yd - e.yI) * (e.yd - e.yI) + (e.xd - e.xI) * (e.xd - e.xI) +
                             (e.zd - e.zI) * (e.zd - e.zI));
    e.crit_self = S.w / dist / 2.0f;
    e.ux = (e.xd - e.xI) / dist;
    e.uy = (e.yd - e.yI) / dist;
    e.uz = (e.zd - e.zI) / dist;
    e.rd = crystal_rect(P, S, T, e.xI, e.yI, e.zI);
    e.filt = isfinite(e.rd.x);

    if (lane < g.n_layers) {          // plate "through both faces" rectangles
        const LayerInfo& Ly = g.layer[lane];
        float4 inner = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);   // empty
        const float f0 = Ly.y1 - e.yI, f1 = Ly.y2 - e.yI;
        const float behind = e.yd - 0.5f * e.t - Ly.y2;
        if (e.filt && f0 >= kMinDepth && behind >= kMinDepth && (Ly.y2 - Ly.y1) >= 0.2f) {
            const float r0 = 1.0f / f0, r1 = 1.0f / f1;
            inner.x = fmaxf((Ly.x1 - e.xI) * r0, (Ly.x1 - e.xI) * r1) + kSlopeMargin;
            inner.y = fminf((Ly.x2 - e.xI) * r0, (Ly.x2 - e.xI) * r1) - kSlopeMargin;
            inner.z = fmaxf((Ly.z1 - e.zI) * r0, (Ly.z1 - e.zI) * r1) + kSlopeMargin;
            inner.w = fminf((Ly.z2 - e.zI) * r0, (Ly.z2 - e.zI) * r1) - kSlopeMargin;
        }
        ws.inner[lane] = inner;
    }

    return true;
}

// Kept-list state of one element (source point) of a warp: the first chunk's end, whether the
// whole list fits one chunk, and the current chunk's entry count.
struct KeptList {
    int n_src, cursor, count;
    bool from_super, single;
};

__device__ __forceinline__ KeptList start_kept_list(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws,
                                                    const Elem& e, int d, int lane)
{
    KeptList k;
    k.from_super = bs.s_count >= 0;
    k.n_src = k.from_super ? bs.s_count : g.n_holes + g.n_det;
    k.count = 0;
    k.cursor = build_chunk(g, bs, ws, e, d, 0, k.n_src, k.from_super, lane, &k.count);
    k.single = k.cursor >= k.n_src;
    return k;
}

// Attenuation outside crystal d along the ray of sub-element q, into s: plate penalty, then
// the kept objects that meet the round's slope box, walked in round buffers (an overfull
// round in pieces: each lane's walk state carries over, so the attenuation order is kept).
// Returns whether the lane skips the sub-element: `dead`, or blocked with every mu >= 0 (the
// contribution is then exactly 0).  Used by the sampled form; pe_element keeps the same walk
// inline (through this helper the reference-order kernel measured 1.5 % slower).
template <bool COUNT, bool ELL>
__device__ __forceinline__ bool walk_sub_element(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws,
                                                 const Elem& e, int d, const SubElem& q, bool dead,
                                                 bool first_round, KeptList& kl, int lane, Walk& s,
                                                 long long& n_sub_entries)
{
    RayCyl rc;
    ray_cyl_init(rc, e.xI, e.yI, e.zI, q.xD, q.yD, q.zD);
    const bool blocked = plate_penalty(g, ws, e, q, s.att);
    const bool skip = dead || (blocked && g.nonneg_mu);
    // slope box of the rays that still need the walk in this round
    float4 box = make_float4(skip ? INFINITY : q.sa_a, skip ? -INFINITY : q.sa_a,
                             skip ? INFINITY : q.sa_b, skip ? -INFINITY : q.sa_b);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        box.x = fminf(box.x, __shfl_xor_sync(0xffffffffu, box.x, off));
        box.y = fmaxf(box.y, __shfl_xor_sync(0xffffffffu, box.y, off));
        box.z = fminf(box.z, __shfl_xor_sync(0xffffffffu, box.z, off));
        box.w = fmaxf(box.w, __shfl_xor_sync(0xffffffffu, box.w, off));
    }
    int cur = 0;
    bool first_chunk = true;
    while (true) {
        if (!kl.single && !first_chunk) {
            cur = build_chunk(g, bs, ws, e, d, cur, kl.n_src, kl.from_super, lane, &kl.count);
        } else if (!kl.single) {
            if (!first_round) cur = build_chunk(g, bs, ws, e, d, 0, kl.n_src, kl.from_super, lane, &kl.count);
            else cur = kl.cursor;
        }
        first_chunk = false;
        int k = 0;
        while (k < kl.count) {
            int next = kl.count, nh = 0;
            const int nr = fill_round<ELL>(g, ws, e, k, kl.count, box, 0, lane, &next, &nh);
            if constexpr (COUNT) n_sub_entries += nr;
            if (!skip) walk_round<ELL>(g, ws, nh, nr, q.xD, q.yD, q.zD, q.sa_a, q.sa_b, q.cosang, rc, s);
            __syncwarp();
            k = next;
        }
        if (kl.single || cur >= kl.n_src) break;
    }
    if (!skip && s.lay < g.n_layers) close_layers(g, s, g.n_layers, q.cosang);
    return skip;
}

template <int MODE, bool COUNT, bool ELL = false>
__device__ double pe_element(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws, int d,
                             long long v, float cr, float sr, int lane,
                             unsigned long long* counters)
{
    Elem e;
    if (!init_element(g, ws, d, v, cr, sr, lane, e)) return 0.0;
    const bool from_super = bs.s_count >= 0;
    const int n_src = from_super ? bs.s_count : g.n_holes + g.n_det;
    int count = 0;
    int cursor = build_chunk(g, bs, ws, e, d, 0, n_src, from_super, lane, &count);
    const bool single = cursor >= n_src;

    float chain = 0.0f;
    double dacc = 0.0;
    int n_hole_hits = 0, n_cry_hits = 0, n_blocked = 0, n_hole_evals = 0, n_cry_evals = 0;
    long long n_sub_entries = 0;
    // Round r covers sub-elements iz in {2p, 2p+1}, all 8 ix, iy in {2u, 2u+1} (p = r/8,
    // u = r%8): a compact patch of the crystal, so a small slope box.  The 8 rounds of one p
    // cover the reference indices s = 256p .. 256p+255, summed in index order after them.
    for (int r = 0; r < 32; ++r) {
        const int sidx = ((r >> 3) * 2 + (lane >> 4)) * 128 + ((lane >> 1) & 7) * 16 + (r & 7) * 2 +
                         (lane & 1);
        const SubElem q = sub_element(e, sidx);
        Walk s{0.0f, 0.0f, 0, 0, 0, 0, 0};
        RayCyl rc;
        ray_cyl_init(rc, e.xI, e.yI, e.zI, q.xD, q.yD, q.zD);
        const bool blocked = plate_penalty(g, ws, e, q, s.att);
        const bool skip = blocked && g.nonneg_mu;
        // slope box of the rays that still need the walk in this round
        float4 box = make_float4(skip ? INFINITY : q.sa_a, skip ? -INFINITY : q.sa_a,
                                 skip ? INFINITY : q.sa_b, skip ? -INFINITY : q.sa_b);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            box.x = fminf(box.x, __shfl_xor_sync(0xffffffffu, box.x, off));
            box.y = fmaxf(box.y, __shfl_xor_sync(0xffffffffu, box.y, off));
            box.z = fminf(box.z, __shfl_xor_sync(0xffffffffu, box.z, off));
            box.w = fmaxf(box.w, __shfl_xor_sync(0xffffffffu, box.w, off));
        }
        // walk this round's objects: kept entries meeting the round box, copied with their
        // geometry into the round buffer; an overfull round is walked in pieces (the walk
        // state of each lane carries over, so the attenuation order is unchanged)
        int cur = 0;
        bool first_chunk = true;
        while (true) {
            if (!single && !first_chunk) {
                cur = build_chunk(g, bs, ws, e, d, cur, n_src, from_super, lane, &count);
            } else if (!single) {
                if (r > 0) cur = build_chunk(g, bs, ws, e, d, 0, n_src, from_super, lane, &count);
                else cur = cursor;
            }
            first_chunk = false;
            int k = 0;
            while (k < count) {
                int next = count, nh = 0;
                const int nr = fill_round<ELL>(g, ws, e, k, count, box, 0, lane, &next, &nh);
                if constexpr (COUNT) n_sub_entries += nr;
                if (!skip) walk_round<ELL>(g, ws, nh, nr, q.xD, q.yD, q.zD, q.sa_a, q.sa_b, q.cosang, rc, s);
                __syncwarp();
                k = next;
            }
            if (single || cur >= n_src) break;
        }
        float contrib = 0.0f;
        if (!skip) {
            if (s.lay < g.n_layers) close_layers(g, s, g.n_layers, q.cosang);
            contrib = finish_sub_element(e, q, s.att);
        }
        if constexpr (COUNT) {
            n_hole_hits += s.hole_hits;
            n_cry_hits += s.cry_hits;
            n_hole_evals += s.hole_evals;
            n_cry_evals += s.cry_evals;
            n_blocked += skip;
        }
        if constexpr (MODE == 0) {
            ws.chain[sidx & 255] = contrib;
            if ((r & 7) == 7) {
                __syncwarp();
#pragma unroll 16
                for (int k = 0; k < 256; ++k) chain = chain + ws.chain[k];
                __syncwarp();
            }
        } else {
            dacc += (double)contrib;
        }
    }
    if constexpr (COUNT) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            n_hole_hits += __shfl_xor_sync(0xffffffffu, n_hole_hits, off);
            n_cry_hits += __shfl_xor_sync(0xffffffffu, n_cry_hits, off);
            n_blocked += __shfl_xor_sync(0xffffffffu, n_blocked, off);
            n_hole_evals += __shfl_xor_sync(0xffffffffu, n_hole_evals, off);
            n_cry_evals += __shfl_xor_sync(0xffffffffu, n_cry_evals, off);
        }
        if (lane == 0) {
            atomicAdd(&counters[0], 1024ull);
            atomicAdd(&counters[1], (unsigned long long)n_hole_hits);
            atomicAdd(&counters[2], (unsigned long long)n_cry_hits);
            atomicAdd(&counters[3], 1ull);
            atomicAdd(&counters[4], (unsigned long long)n_blocked);
            atomicAdd(&counters[5], single ? 0ull : 1ull);                 // chunked elements
            atomicAdd(&counters[6], (unsigned long long)count);            // kept objects (last chunk)
            atomicAdd(&counters[7], (unsigned long long)n_sub_entries);    // round sub-list entries
            atomicAdd(&counters[8], bs.s_count < 0 ? 1ull : 0ull);         // superset overflow
            atomicAdd(&counters[9], (unsigned long long)(bs.s_count < 0 ? 0 : bs.s_count));
            atomicAdd(&counters[10], (unsigned long long)n_hole_evals);
            atomicAdd(&counters[11], (unsigned long long)n_cry_evals);
        }
    }
    if constexpr (MODE == 0) {
        return chain;
    } else {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) dacc += __shfl_xor_sync(0xffffffffu, dacc, off);
        return dacc;
    }
}

// Element of the sampled form: the mean over the voxel's sx x sy x sz source points (centres of
// a grid over the voxel) of the reference's element with crystal d divided into nx x ny x nz
// sub-elements (x, depth, z), every contribution summed in FP64.  Each source point has its
// own cone test and kept list; its sub-elements are taken 32 at a time in (z, depth, x) order,
// x fastest, so a round is a compact patch of the crystal.  With 8 x 16 x 8 and 1 x 1 x 1 it
// runs pe_element<1>'s float program, summed in another order (a separately compiled
// instance: the compiler may contract the position expressions differently, in the last bit).
template <bool ELL>
__device__ double pe_element_sampled(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws, int d, long long v,
                                     float cr, float sr, int lane, const Sampling& sm)
{
    const int n_sub = sm.nx * sm.ny * sm.nz, nxy = sm.nx * sm.ny;
    const int n_pts = sm.sx * sm.sy * sm.sz;
    const float fx = (float)sm.nx, fy = (float)sm.ny, fz = (float)sm.nz;
    double dacc = 0.0;
    long long unused = 0;
    for (int p = 0; p < n_pts; ++p) {
        const int jx = p % sm.sx, jy = (p / sm.sx) % sm.sy, jz = p / (sm.sx * sm.sy);
        __syncwarp();                     // the previous point's lists are no longer read
        Elem e;
        if (!init_element(g, ws, d, v, cr, sr, lane, e, ((float)jx + 0.5f) / (float)sm.sx,
                          ((float)jy + 0.5f) / (float)sm.sy, ((float)jz + 0.5f) / (float)sm.sz))
            return 0.0;                   // the crystal's mu does not depend on the point
        KeptList kl = start_kept_list(g, bs, ws, e, d, lane);
        for (int base = 0; base < n_sub; base += 32) {
            const int sidx = min(base + lane, n_sub - 1);
            const int iz = sidx / nxy, rem = sidx - iz * nxy;
            const int iy = rem / sm.nx, ix = rem - iy * sm.nx;
            const SubElem q = sub_element_at(e, ix, iy, iz, fx, fy, fz);
            Walk s{0.0f, 0.0f, 0, 0, 0, 0, 0};
            const bool skip = walk_sub_element<false, ELL>(g, bs, ws, e, d, q, base + lane >= n_sub, base == 0,
                                                           kl, lane, s, unused);
            if (!skip) dacc += (double)finish_sub_element_at(e, q, s.att, fx, fy, fz);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dacc += __shfl_xor_sync(0xffffffffu, dacc, off);
    return dacc / (double)n_pts;
}

#include "pe_fp64.cuh"
#include "pe_local.cuh"

// Block superset of the reference cone test over all voxels within radius rho of
// (cx, cy, cz): keep object o when |u_o - u_d| <= (rho + r_o)/(L_o - rho)
// + (rho + r_d)/(L_d - rho) + 1e-4 at the centre (each direction moves by at most
// rho/(L - rho) in chord length, each angular radius r/L grows to at most r/(L - rho)).
__device__ void build_superset(const DevGeom& g, BlockSmem& bs, int d, float cx, float cy, float cz,
                               float rho)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const float4 P = __ldg(&g.cry.pos[d]);
    const float rdd = 0.5f * __ldg(&g.cry.size[d].w);
    const float Ld = sqrtf((P.x - cx) * (P.x - cx) + (P.y - cy) * (P.y - cy) + (P.z - cz) * (P.z - cz));
    const float uxd = (P.x - cx) / Ld, uyd = (P.y - cy) / Ld, uzd = (P.z - cz) / Ld;
    const bool near_d = !(Ld - rho > 0.5f);
    const float td = near_d ? 0.0f : (rho + rdd) / (Ld - rho);
    const int N = g.n_holes + g.n_det;
    int running = 0;
    for (int base = 0; base < N; base += kThreads) {
        const int i = base + threadIdx.x;
        bool keep = false;
        float4 od = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < N && !(i >= g.n_holes && i - g.n_holes == d)) {
            od = object_data(g, i);
            const float ro = (i < g.n_holes) ? od.w : 0.5f * od.w;
            const float Lo = sqrtf((od.x - cx) * (od.x - cx) + (od.y - cy) * (od.y - cy) +
                                   (od.z - cz) * (od.z - cz));
            if (near_d || !(Lo - rho > 0.5f)) {
                keep = true;
            } else {
                const float dx = (od.x - cx) / Lo - uxd, dy = (od.y - cy) / Lo - uyd,
                            dz = (od.z - cz) / Lo - uzd;
                const float thr = (rho + ro) / (Lo - rho) + td + 1e-4f;
                keep = sqrtf(dx * dx + dy * dy + dz * dz) <= thr;
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) bs.warp_cnt[wid] = __popc(m);
        __syncthreads();
        int off = running, tot = 0;
        for (int k = 0; k < kWarps; ++k) {
            const int c = bs.warp_cnt[k];
            if (k < wid) off += c;
            tot += c;
        }
        const int pos = off + __popc(m & ((1u << lane) - 1u));
        if (keep && pos < kSuperCap) {
            bs.sdata[pos] = od;
            bs.sid[pos] = i;
        }
        running += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) bs.s_count = (running <= kSuperCap) ? running : -1;
    __syncthreads();
}

// Output block of one brick: rows (crystals) from det_begin, voxels vox_begin .. vlast.
struct BrickOut {
    float* out;
    long long ld, vox_begin, vlast;
    int det_begin;
    float* sub_out;           // per-sub-element contributions (local sampled form), or nullptr
    int det_count;
};

// One work item: crystal det_begin + di against one voxel brick of bx x by x bz voxels (brick
// (gx, gy, gz) of the block's grid starting at z-plane iz0).  The block builds the cone
// superset of the brick, then its warps take the brick's voxels in turn.
// SAMPLED: elements of the sampled form `smp` (source points anywhere in the voxels: the
// superset radius grows by half a voxel diagonal).
template <int MODE, bool COUNT, bool ELL = false, bool SAMPLED = false>
__device__ __forceinline__ void pe_brick(const DevGeom& g, BlockSmem& bs, WarpSmem& ws, int lane, int wid,
                                         const BrickOut& O, int di, int gx, int gy, int gz, int iz0, int iz1,
                                         int bx, int by, int bz, float cr, float sr,
                                         unsigned long long* counters, const Sampling* smp = nullptr,
                                         float rotation = 0.0f)
{
    const int x0 = gx * bx, y0 = gy * by, z0 = iz0 + gz * bz;
    const int x1 = min(x0 + bx, g.nx) - 1, y1 = min(y0 + by, g.ny) - 1, z1 = min(z0 + bz, iz1 + 1) - 1;
    const int d = O.det_begin + di;
    // brick centre and radius from its extreme voxel centres (rotation about z keeps lengths)
    float ax, ay, az, bxx, byy, bzz;
    voxel_centre(g, x0 + g.nx * ((long long)y0 + g.ny * z0), 1.0f, 0.0f, ax, ay, az);
    voxel_centre(g, x1 + g.nx * ((long long)y1 + g.ny * z1), 1.0f, 0.0f, bxx, byy, bzz);
    const float mx = 0.5f * (ax + bxx), my = 0.5f * (ay + byy), mz = 0.5f * (az + bzz);
    float rho = 0.5f * sqrtf((bxx - ax) * (bxx - ax) + (byy - ay) * (byy - ay) +
                             (bzz - az) * (bzz - az)) + 1e-3f;
    if constexpr (SAMPLED) rho += 0.5f * sqrtf(g.wx * g.wx + g.wy * g.wy + g.wz * g.wz);
    build_superset(g, bs, d, mx * cr - my * sr, mx * sr + my * cr, mz, rho);
    const int n_slots = bx * by * bz;
    for (int slot = wid; slot < n_slots; slot += kWarps) {
        const int ox = slot % bx, oy = (slot / bx) % by, oz = slot / (bx * by);
        const int ix = x0 + ox, iy = y0 + oy, iz = z0 + oz;
        if (ix >= g.nx || iy >= g.ny || iz > z1) continue;
        const long long v = ix + g.nx * ((long long)iy + (long long)g.ny * iz);
        if (v < O.vox_begin || v > O.vlast) continue;
        float val;
        if constexpr (MODE == 3) {
            float* so = nullptr;
            if (SAMPLED && O.sub_out)
                so = O.sub_out + ((v - O.vox_begin) * O.det_count + di) * (long long)(smp->nx * smp->ny * smp->nz);
            val = (float)pe_element_local<ELL, SAMPLED>(g, bs, ws, d, v, cr, sr, rotation, lane, smp, so);
        } else if constexpr (SAMPLED) val = (float)pe_element_sampled<ELL>(g, bs, ws, d, v, cr, sr, lane, *smp);
        else if constexpr (MODE == 2) val = (float)pe_element64(g, bs, ws, d, v, cr, sr, rotation, lane);
        else val = (float)pe_element<MODE, COUNT, ELL>(g, bs, ws, d, v, cr, sr, lane, counters);
        if (lane == 0) O.out[(long long)di * O.ld + (v - O.vox_begin)] = val;
        __syncwarp();
    }
    __syncthreads();
}

template <int MODE, bool COUNT, bool ELL, bool SAMPLED = false>
__global__ void __launch_bounds__(kThreads, 2) pe_kernel(DevGeom g, PeLaunch L)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BlockSmem& bs = *reinterpret_cast<BlockSmem*>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem& ws = bs.w[wid];
    const float ang = L.rotation * g.angle_step;           // :1006
    const float cr = cosf(ang), sr = sinf(ang);
    const long long nxy = (long long)g.nx * g.ny;
    const long long vlast = L.vox_begin + L.vox_count - 1;
    const int iz0 = (int)(L.vox_begin / nxy), iz1 = (int)(vlast / nxy);
    constexpr int bx = 4, by = 4, bz = 2;                 // voxel brick of one work item
    const int nbx = (g.nx + bx - 1) / bx, nby = (g.ny + by - 1) / by;
    const int nbz = (iz1 - iz0 + 1 + bz - 1) / bz;
    const long long n_bricks = (long long)nbx * nby * nbz;
    const long long total = n_bricks * L.det_count;
    const BrickOut O{L.out, L.ld, L.vox_begin, vlast, L.det_begin, L.sub_out, L.det_count};
    for (;;) {
        if (threadIdx.x == 0) bs.item = (long long)atomicAdd(L.work_counter, 1ull);
        __syncthreads();
        const long long item = bs.item;
        __syncthreads();
        if (item >= total) break;
        const int di = (int)(item / n_bricks);
        const long long b = item - (long long)di * n_bricks;
        const int gz = (int)(b / ((long long)nbx * nby));
        const int rem = (int)(b - (long long)gz * nbx * nby);
        const int gy = rem / nbx, gx = rem - gy * nbx;
        pe_brick<MODE, COUNT, ELL, SAMPLED>(g, bs, ws, lane, wid, O, di, gx, gy, gz, iz0, iz1, bx, by, bz, cr, sr,
                                            L.counters, &L.smp, L.rotation);
    }
}

// Shared memory of the batched kernel: the block's working set plus the geometry of the
// task in hand (copied in when the block moves to a task of another geometry).
struct BatchSmem {
    BlockSmem bs;
    DevGeom g;
    int task;
};

// Batched launch: one persistent grid over the items of many (geometry, rotation, block)
// tasks, taken from one work counter; a block finds its item's task by binary search over
// the tasks' first item numbers.
template <int MODE, bool ELL>
__global__ void __launch_bounds__(kThreads, 2) pe_batch_kernel(BatchLaunch B)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BatchSmem& sm = *reinterpret_cast<BatchSmem*>(smem_raw);
    BlockSmem& bs = sm.bs;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem& ws = bs.w[wid];
    int cur_geom = -1;
    for (;;) {
        if (threadIdx.x == 0) {
            const long long item = (long long)atomicAdd(B.work_counter, 1ull);
            int lo = 0, hi = B.n_tasks - 1;
            while (lo < hi) {                       // last task with item_begin <= item
                const int mid = (lo + hi + 1) >> 1;
                if (B.tasks[mid].item_begin <= item) lo = mid; else hi = mid - 1;
            }
            bs.item = item;
            sm.task = lo;
        }
        __syncthreads();
        const long long item = bs.item;
        const BatchTask T = B.tasks[sm.task];
        __syncthreads();
        if (item >= B.total_items) break;
        if (T.geom != cur_geom) {                   // block-uniform
            const int* src = reinterpret_cast<const int*>(B.geoms + T.geom);
            int* dst = reinterpret_cast<int*>(&sm.g);
            for (int i = threadIdx.x; i < (int)(sizeof(DevGeom) / sizeof(int)); i += kThreads) dst[i] = src[i];
            cur_geom = T.geom;
            __syncthreads();
        }
        const DevGeom& g = sm.g;
        const float ang = T.rotation * g.angle_step;       // :1006
        const float cr = cosf(ang), sr = sinf(ang);
        const long long n_bricks = (long long)T.nbx * T.nby * T.nbz;
        const long long local = item - T.item_begin;
        const int di = (int)(local / n_bricks);
        const long long b = local - (long long)di * n_bricks;
        const int gz = (int)(b / ((long long)T.nbx * T.nby));
        const int rem = (int)(b - (long long)gz * T.nbx * T.nby);
        const int gy = rem / T.nbx, gx = rem - gy * T.nbx;
        const BrickOut O{T.out, T.ld, T.vox_begin, T.vox_begin + T.vox_count - 1, T.det_begin, nullptr, T.det_count};
        pe_brick<MODE, false, ELL>(g, bs, ws, lane, wid, O, di, gx, gy, gz, T.iz0, T.iz1, B.bx, B.by, B.bz, cr,
                                   sr, nullptr, nullptr, T.rotation);
    }
}

#include "pe_adjoint.cuh"

}  // namespace

template <int MODE, bool COUNT, bool ELL, bool SAMPLED = false>
static int launch_mode(const DevGeom& g, const PeLaunch& L, int num_sms, cudaStream_t stream)
{
    const int smem = (int)sizeof(BlockSmem);
    static unsigned long long configured = 0;   // one bit per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(__atomic_load_n(&configured, __ATOMIC_ACQUIRE) & bit)) {
        if (cudaFuncSetAttribute(pe_kernel<MODE, COUNT, ELL, SAMPLED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem) !=
            cudaSuccess)
            return -1;
        __atomic_fetch_or(&configured, bit, __ATOMIC_RELEASE);
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pe_kernel<MODE, COUNT, ELL, SAMPLED>, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    pe_kernel<MODE, COUNT, ELL, SAMPLED><<<num_sms * per_sm, kThreads, smem, stream>>>(g, L);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <int KIND, bool ELL>
static int launch_adjoint_kind(const DevGeom& g, const AdjLaunch& L, int num_sms, cudaStream_t stream)
{
    const int smem = (int)sizeof(AdjSmem);
    static unsigned long long configured = 0;   // one bit per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(__atomic_load_n(&configured, __ATOMIC_ACQUIRE) & bit)) {
        if (cudaFuncSetAttribute(pe_adjoint_kernel<KIND, ELL>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
            cudaSuccess)
            return -1;
        __atomic_fetch_or(&configured, bit, __ATOMIC_RELEASE);
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pe_adjoint_kernel<KIND, ELL>, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    pe_adjoint_kernel<KIND, ELL><<<num_sms * per_sm, kThreads, smem, stream>>>(g, L);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Systems with elliptical holes (sysmat_set_hole_shapes) run the elliptical instances.
int launch_pe_adjoint(const DevGeom& g, const AdjLaunch& L, int kind, int num_sms, cudaStream_t stream)
{
    if (g.hole_shape) {
        if (kind == 0) return launch_adjoint_kind<0, true>(g, L, num_sms, stream);
        if (kind == 1) return launch_adjoint_kind<1, true>(g, L, num_sms, stream);
        return launch_adjoint_kind<2, true>(g, L, num_sms, stream);
    }
    if (kind == 0) return launch_adjoint_kind<0, false>(g, L, num_sms, stream);
    if (kind == 1) return launch_adjoint_kind<1, false>(g, L, num_sms, stream);
    return launch_adjoint_kind<2, false>(g, L, num_sms, stream);
}

template <int MODE, bool ELL>
static int configure_batch_mode(int* per_sm)
{
    const int smem = (int)sizeof(BatchSmem);
    static unsigned long long configured = 0;   // one bit per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(__atomic_load_n(&configured, __ATOMIC_ACQUIRE) & bit)) {
        if (cudaFuncSetAttribute(pe_batch_kernel<MODE, ELL>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
            cudaSuccess)
            return -1;
        __atomic_fetch_or(&configured, bit, __ATOMIC_RELEASE);
    }
    *per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, pe_batch_kernel<MODE, ELL>, kThreads, smem) !=
        cudaSuccess)
        return -1;
    if (*per_sm < 1) *per_sm = 1;
    return 0;
}

int configure_pe_batch(int mode, bool ell, int* blocks_per_sm)
{
    if (mode == 2) return configure_batch_mode<2, false>(blocks_per_sm);   // shapes read at run time
    if (mode == 3) return ell ? configure_batch_mode<3, true>(blocks_per_sm) : configure_batch_mode<3, false>(blocks_per_sm);
    if (ell) {
        return mode == 0 ? configure_batch_mode<0, true>(blocks_per_sm)
                         : configure_batch_mode<1, true>(blocks_per_sm);
    }
    return mode == 0 ? configure_batch_mode<0, false>(blocks_per_sm) : configure_batch_mode<1, false>(blocks_per_sm);
}

int launch_pe_batch(const BatchLaunch& B, int mode, bool ell, int grid, cudaStream_t stream)
{
    if (B.n_tasks < 1 || B.total_items < 1) return 0;
    const int smem = (int)sizeof(BatchSmem);
    if (mode == 2) {                              // FP64: shapes read at run time
        pe_batch_kernel<2, false><<<grid, kThreads, smem, stream>>>(B);
    } else if (mode == 3) {
        if (ell) pe_batch_kernel<3, true><<<grid, kThreads, smem, stream>>>(B);
        else pe_batch_kernel<3, false><<<grid, kThreads, smem, stream>>>(B);
    } else if (ell) {
        if (mode == 0) pe_batch_kernel<0, true><<<grid, kThreads, smem, stream>>>(B);
        else pe_batch_kernel<1, true><<<grid, kThreads, smem, stream>>>(B);
    } else {
        if (mode == 0) pe_batch_kernel<0, false><<<grid, kThreads, smem, stream>>>(B);
        else pe_batch_kernel<1, false><<<grid, kThreads, smem, stream>>>(B);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_pe(const DevGeom& g, const PeLaunch& L, int mode, int num_sms, cudaStream_t stream)
{
    if (mode == 2) return g.t64.cry_pos ? launch_mode<2, false, false>(g, L, num_sms, stream) : -1;
    if (mode == 3) {
        if (!g.t64.cry_pos) return -1;
        return g.hole_shape ? launch_mode<3, false, true>(g, L, num_sms, stream)
                            : launch_mode<3, false, false>(g, L, num_sms, stream);
    }
    if (g.hole_shape) {                   // systems with elliptical holes
        if (L.counters) return launch_mode<0, true, true>(g, L, num_sms, stream);
        return mode == 0 ? launch_mode<0, false, true>(g, L, num_sms, stream)
                         : launch_mode<1, false, true>(g, L, num_sms, stream);
    }
    if (L.counters) return launch_mode<0, true, false>(g, L, num_sms, stream);
    return mode == 0 ? launch_mode<0, false, false>(g, L, num_sms, stream)
                     : launch_mode<1, false, false>(g, L, num_sms, stream);
}

int launch_pe_local_sampled(const DevGeom& g, const PeLaunch& L, int num_sms, cudaStream_t stream)
{
    if (!g.t64.cry_pos) return -1;
    return g.hole_shape ? launch_mode<3, false, true, true>(g, L, num_sms, stream)
                        : launch_mode<3, false, false, true>(g, L, num_sms, stream);
}

int launch_pe_sampled(const DevGeom& g, const PeLaunch& L, int num_sms, cudaStream_t stream)
{
    if (g.hole_shape) return launch_mode<1, false, true, true>(g, L, num_sms, stream);
    return launch_mode<1, false, false, true>(g, L, num_sms, stream);
}

}  // namespace sysmat
