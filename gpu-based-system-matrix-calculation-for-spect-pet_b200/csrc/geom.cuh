// Device-side geometry tables and ray-chord primitives for the system-matrix kernels.
//
// The chord functions restate the reference's float arithmetic
// (PEGen_RayTracing_CircularHole/PESysMatGen.cu:20-799) with identical operation order,
// thresholds and branch outcomes, so that every chord equals the reference's chord for
// the same inputs.  The code shape is ours: the general (no axis-parallel) case is the
// inlined fast path and the rare axis-parallel cases live in a separate function.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sysmat {

constexpr int kMaxLayers = 9;        // a 10th header would overlap the hole table (index 100)
constexpr int kNCollimator = 80000;
constexpr int kNDetector = 80000;
constexpr int kNImage = 100;
constexpr int kNPhysics = 100;

// Per-crystal derived table (structure of float4 arrays, one entry per crystal).
//   pos  : x, y + FOV-to-collimator, z, rotation about y
//   size : width (x), thickness (y), height (z), sqrt(w*w + h*h + t*t)
//   mu   : mu_total, mu_pe, mu_compton, energy resolution
//   trig : cos(rot), sin(rot), cos(-rot), sin(-rot)
struct CrystalTables {
    const float4* pos;
    const float4* size;
    const float4* mu;
    const float4* trig;
};

// Per-hole derived table.
//   a : x, y1 + FOV, y2 + FOV, z
//   b : radius, mu_total, (y1 + y2) / 2, sqrt(R*R*4 + (y1 - y2)^2) / 2
//   raw : x, raw y1, raw y2, z  (no FOV offset; used by the scatter path and bitmaps)
struct HoleTables {
    const float4* a;
    const float4* b;
    const float4* raw;
};

// FP64 mode: the derived geometry in double, formed from the raw float parameters with the
// double operations of the FP64 restatement (y + FOV and the like in double, not rounded to
// float as in the tables above).
struct alignas(32) D4 {
    double x, y, z, w;
};

struct Tables64 {
    const D4* hole_a;      // x, y1 + fov, y2 + fov, z
    const D4* hole_b;      // r, mu, y centre, cone radius sqrt(4 r^2 + (y1 - y2)^2) / 2
    const D4* cry_pos;     // x, y + fov, z, mu_total
    const D4* cry_size;    // w, t, h, mu_pe
    const D4* cry_trig;    // cos rot, sin rot, cos -rot, sin -rot
    const double* layer;   // kLayer64 values per layer: x1, x2, y1, y2, z1, z2, thickness, mu_total
    const D4* hole_shape;  // elliptical holes: rho_x, rho_z, cos theta, sin theta (rho_x = 0: circle), or nullptr
};
constexpr int kLayer64 = 8;

struct LayerInfo {
    float x1, x2, y1, y2, z1, z2;   // plate box (PESysMatGen.cu:1242-1249)
    float thickness;
    float mu_total;
    float mu_pe, mu_c;               // photoelectric and Compton parts (native scatter model)
    int hole_begin, hole_count;
};

struct DevGeom {
    int n_det;
    int n_holes;         // all layers
    int n_layers;
    int n_holes0;        // layer-0 holes (scatter scatterers; scatter.cu:1555)
    int nx, ny, nz;
    long long nvox;
    float wx, wy, wz;
    float shx, shy, shz;
    float fov;           // FOV-to-collimator distance, Params_Image[11]
    float angle_step;    // Params_Image[7]
    int nonneg_mu;       // all attenuation coefficients >= 0 (enables the blocked-ray early exit)
    const float* raw_det;   // Params_Detector as uploaded (bitmaps use raw, un-offset values)
    CrystalTables cry;
    HoleTables hole;
    // optional elliptical holes (sysmat_set_hole_shapes): per hole (rho_x, rho_z, cos theta,
    // sin theta), rho_x = 0 for a circular hole; nullptr when every hole is circular
    const float4* hole_shape;
    Tables64 t64;        // FP64 mode tables (nullptr pointers where a caller built no such tables)
    LayerInfo layer[kMaxLayers];
};

// ------------------------------------------------------------------------------------
// Chord primitives.  eps constants and their float/double comparison semantics follow
// the reference: comparisons against the double literals 0.001 / 0.0001 / 0.00001 are
// equivalent to comparisons against the float literals used here (no float lies between
// the two values; checked by tests/test_oracle.py).

constexpr float kEps = 0.001f;

__device__ __forceinline__ void slab_interval(float p0, float lo, float hi, float inv, float& t0,
                                              float& t1)
{
    if (inv < 0.0f) { t0 = (hi - p0) * inv; t1 = (lo - p0) * inv; }
    else            { t0 = (lo - p0) * inv; t1 = (hi - p0) * inv; }
}

// Slow path of both box chords: at least one axis with |delta| < eps.  inside = 0:
// PESysMatGen.cu:28-232 (full crossing), inside = 1: :328-589 (end point inside).
static __device__ __noinline__ float box_chord_parallel(float xi, float yi, float zi, float xo, float yo,
                                                 float zo, float x1, float y1, float z1, float x2,
                                                 float y2, float z2, int inside)
{
    const float p0[3] = {xi, yi, zi}, p1[3] = {xo, yo, zo};
    const float lo[3] = {x1, y1, z1}, hi[3] = {x2, y2, z2};
    bool par[3];
    int npar = 0;
    for (int a = 0; a < 3; ++a) {
        par[a] = fabsf(p1[a] - p0[a]) < kEps;
        npar += par[a];
    }
    if (npar == 3) return 0.0f;
    if (npar == 2) {
        const int m = !par[0] ? 0 : (!par[1] ? 1 : 2);
        for (int a = 0; a < 3; ++a)
            if (a != m && !(p0[a] >= lo[a] && p0[a] <= hi[a])) return 0.0f;
        if (!inside) {
            if ((p0[m] <= lo[m] && p1[m] >= hi[m]) || (p1[m] <= lo[m] && p0[m] >= hi[m]))
                return fabsf(hi[m] - lo[m]);
            return 0.0f;
        }
        if (p0[m] < p1[m]) return p1[m] - lo[m];
        return hi[m] - p1[m];       // p0[m] > p1[m]: axis m is not parallel
    }
    // exactly one parallel axis q: 2-D slab over the other two, length measured in them
    const int q = par[0] ? 0 : (par[1] ? 1 : 2);
    if (p0[q] >= hi[q] || p0[q] <= lo[q]) return 0.0f;
    const int a0 = (q == 0) ? 1 : 0;
    const int a1 = (q == 2) ? 1 : 2;
    const float d0 = p1[a0] - p0[a0], d1 = p1[a1] - p0[a1];
    const float tio = sqrtf(d0 * d0 + d1 * d1);
    float tmin, tmax, b0, b1;
    slab_interval(p0[a0], lo[a0], hi[a0], tio / d0, tmin, tmax);
    slab_interval(p0[a1], lo[a1], hi[a1], tio / d1, b0, b1);
    if (tmin > b1 || b0 > tmax) return 0.0f;
    tmin = (b0 > tmin) ? b0 : tmin;
    tmax = (b1 < tmax) ? b1 : tmax;
    if ((tmax - tmin) < kEps) return 0.0f;
    if (!inside) {
        if (tmin >= tio || tmax >= tio) return 0.0f;
        if (tmin <= kEps || tmax <= kEps) return 0.0f;
        return tmax - tmin;
    }
    if (tmin >= tio) return 0.0f;
    if (tmax <= kEps) return 0.0f;
    if ((tmax >= tio) && (tmin > kEps)) return tio - tmin;
    if ((tmin <= kEps) && (tmax <= tio)) return tmax;
    if ((tmin <= kEps) && (tmax >= tio)) return tio;
    return tmax - tmin;
}


// Chord of the segment (xi,yi,zi)->(xo,yo,zo) through the box; only full crossings count.
__device__ __forceinline__ float box_chord(float xi, float yi, float zi, float xo, float yo,
                                           float zo, float x1, float y1, float z1, float x2,
                                           float y2, float z2)
{
    const float dx = xo - xi, dy = yo - yi, dz = zo - zi;
    if (fabsf(dx) < kEps || fabsf(dy) < kEps || fabsf(dz) < kEps)
        return box_chord_parallel(xi, yi, zi, xo, yo, zo, x1, y1, z1, x2, y2, z2, 0);
    const float tio = sqrtf(dx * dx + dy * dy + dz * dz);
    float tmin, tmax, a0, a1;
    slab_interval(xi, x1, x2, tio / dx, tmin, tmax);
    slab_interval(yi, y1, y2, tio / dy, a0, a1);
    if (tmin > a1 || a0 > tmax) return 0.0f;
    tmin = (a0 > tmin) ? a0 : tmin;
    tmax = (a1 < tmax) ? a1 : tmax;
    slab_interval(zi, z1, z2, tio / dz, a0, a1);
    if (tmin > a1 || a0 > tmax) return 0.0f;
    tmin = (a0 > tmin) ? a0 : tmin;
    tmax = (a1 < tmax) ? a1 : tmax;
    if ((tmax - tmin) < kEps) return 0.0f;
    if (tmin >= tio || tmax >= tio) return 0.0f;
    if (tmin <= kEps || tmax <= kEps) return 0.0f;
    return tmax - tmin;
}

// Chord from the box entry to the end point, which lies inside the box.
__device__ __forceinline__ float box_chord_inside(float xi, float yi, float zi, float xo, float yo,
                                                  float zo, float x1, float y1, float z1, float x2,
                                                  float y2, float z2)
{
    const float dx = xo - xi, dy = yo - yi, dz = zo - zi;
    if (fabsf(dy) < 0.001f) return 0.0f;          // PESysMatGen.cu:321-324
    if (fabsf(dx) < kEps || fabsf(dz) < kEps)
        return box_chord_parallel(xi, yi, zi, xo, yo, zo, x1, y1, z1, x2, y2, z2, 1);
    const float tio = sqrtf(dx * dx + dy * dy + dz * dz);
    float tmin, tmax, a0, a1;
    slab_interval(xi, x1, x2, tio / dx, tmin, tmax);
    slab_interval(yi, y1, y2, tio / dy, a0, a1);
    if (tmin > a1 || a0 > tmax) return 0.0f;
    tmin = (a0 > tmin) ? a0 : tmin;
    tmax = (a1 < tmax) ? a1 : tmax;
    slab_interval(zi, z1, z2, tio / dz, a0, a1);
    if (tmin > a1 || a0 > tmax) return 0.0f;
    tmin = (a0 > tmin) ? a0 : tmin;
    tmax = (a1 < tmax) ? a1 : tmax;
    if ((tmax - tmin) < kEps) return 0.0f;
    if (tmin >= tio) return 0.0f;
    if (tmax <= kEps) return 0.0f;
    if ((tmax >= tio) && (tmin > kEps)) return tio - tmin;
    if ((tmin <= kEps) && (tmax <= tio)) return tmax;
    if ((tmin <= kEps) && (tmax >= tio)) return tio;
    return tmax - tmin;
}

// Interval part of box_chord_inside for one box, given the segment's shared terms.
__device__ __forceinline__ float inside_from_slabs(float xi, float yi, float zi, float ix, float iy,
                                                   float iz, float tio, float x1, float y1, float z1,
                                                   float x2, float y2, float z2)
{
    float tmin, tmax, a0, a1;
    slab_interval(xi, x1, x2, ix, tmin, tmax);
    slab_interval(yi, y1, y2, iy, a0, a1);
    if (tmin > a1 || a0 > tmax) return 0.0f;
    tmin = (a0 > tmin) ? a0 : tmin;
    tmax = (a1 < tmax) ? a1 : tmax;
    slab_interval(zi, z1, z2, iz, a0, a1);
    if (tmin > a1 || a0 > tmax) return 0.0f;
    tmin = (a0 > tmin) ? a0 : tmin;
    tmax = (a1 < tmax) ? a1 : tmax;
    if ((tmax - tmin) < kEps) return 0.0f;
    if (tmin >= tio) return 0.0f;
    if (tmax <= kEps) return 0.0f;
    if ((tmax >= tio) && (tmin > kEps)) return tio - tmin;
    if ((tmin <= kEps) && (tmax <= tio)) return tmax;
    if ((tmin <= kEps) && (tmax >= tio)) return tio;
    return tmax - tmin;
}

// box_chord_inside of one segment against two boxes A and B.  The segment terms (parallel
// tests, length, the three reciprocal steps) are computed once; every result is the float
// box_chord_inside returns for that box.
__device__ __forceinline__ void box_chord_inside2(float xi, float yi, float zi, float xo, float yo,
                                                  float zo, const float* a, const float* b,
                                                  float& la, float& lb)
{
    const float dx = xo - xi, dy = yo - yi, dz = zo - zi;
    if (fabsf(dy) < 0.001f) { la = 0.0f; lb = 0.0f; return; }
    if (fabsf(dx) < kEps || fabsf(dz) < kEps) {
        la = box_chord_parallel(xi, yi, zi, xo, yo, zo, a[0], a[1], a[2], a[3], a[4], a[5], 1);
        lb = box_chord_parallel(xi, yi, zi, xo, yo, zo, b[0], b[1], b[2], b[3], b[4], b[5], 1);
        return;
    }
    const float tio = sqrtf(dx * dx + dy * dy + dz * dz);
    const float ix = tio / dx, iy = tio / dy, iz = tio / dz;
    la = inside_from_slabs(xi, yi, zi, ix, iy, iz, tio, a[0], a[1], a[2], a[3], a[4], a[5]);
    lb = inside_from_slabs(xi, yi, zi, ix, iy, iz, tio, b[0], b[1], b[2], b[3], b[4], b[5]);
}

// Chord through the y-parallel cylinder (x-xc)^2 + (z-zc)^2 <= r^2, y in [y1, y2]
// (PESysMatGen.cu:688-799).
__device__ __forceinline__ float cyl_chord(float xi, float yi, float zi, float xo, float yo,
                                           float zo, float xc, float y1, float y2, float zc, float r)
{
    if (fabsf(y1 - y2) < 0.001f) return 0.0f;
    const float dx = xo - xi, dy = yo - yi, dz = zo - zi;
    const float tio = sqrtf(dx * dx + dy * dy + dz * dz);
    const float kx = dx / tio, ky = dy / tio, kz = dz / tio;
    const float xl = xi + kx / ky * (y1 - yi);
    const float xr = xi + kx / ky * (y2 - yi);
    const float zl = zi + kz / ky * (y1 - yi);
    const float zr = zi + kz / ky * (y2 - yi);
    const float ta = (y1 - yi) / ky;
    const float tb = (y2 - yi) / ky;
    const bool fl = (xl - xc) * (xl - xc) + (zl - zc) * (zl - zc) <= r * r;
    const bool fr = (xr - xc) * (xr - xc) + (zr - zc) * (zr - zc) <= r * r;
    if (fl && fr) {
        if (ta <= 0.0001f || tb <= 0.0001f) return 0.0f;
        if (ta >= tio || tb >= tio) return 0.0f;
        return fabsf(tb - ta);
    }
    const float ox = xi - xc, oz = zi - zc;
    const float disc = (kx * kx + kz * kz) * r * r - (kx * oz - kz * ox) * (kx * oz - kz * ox);
    if (disc <= 0.00001f) return 0.0f;
    const float t1 = (-(kx * ox + kz * oz) - sqrtf(disc)) / (kx * kx + kz * kz);
    const float t2 = (-(kx * ox + kz * oz) + sqrtf(disc)) / (kx * kx + kz * kz);
    float ea, eb;
    if (!fl && !fr) {
        if (!(t1 >= ta && t2 <= tb)) return 0.0f;
        ea = t1; eb = t2;
    } else if (fl) { ea = ta; eb = t2; }
    else           { ea = t1; eb = tb; }
    if (eb <= 0.0001f || ea <= 0.0001f) return 0.0f;
    if (eb >= tio || ea >= tio) return 0.0f;
    return eb - ea;
}

// Chord through the y-parallel elliptical cylinder ((x'-xc)/rx)^2 + ((z'-zc)/rz)^2 <= 1,
// y in [y1, y2], with the segment's points rotated by theta about the axis first
// (PESysMatGen.cu:801-947, defined but not called by the reference kernels).  ct, st are
// cos(theta), sin(theta) as the reference evaluates them; each expression is written as the
// reference writes it, so nvcc contracts it the same way.
__device__ __forceinline__ float ell_chord(float x_in, float y_in, float z_in, float x_out, float y_out,
                                           float z_out, float xc, float y1, float y2, float zc, float rx,
                                           float rz, float ct, float st)
{
    const float x_in_ = x_in - xc;
    const float z_in_ = z_in - zc;
    const float x_out_ = x_out - xc;
    const float z_out_ = z_out - zc;
    x_in = xc + x_in_ * ct + z_in_ * st;
    z_in = zc - x_in_ * st + z_in_ * ct;
    x_out = xc + x_out_ * ct + z_out_ * st;
    z_out = zc - x_out_ * st + z_out_ * ct;
    if (fabsf(y1 - y2) < 0.001f) return 0.0f;
    const float tio = sqrtf((x_out - x_in) * (x_out - x_in) + (y_out - y_in) * (y_out - y_in) +
                            (z_out - z_in) * (z_out - z_in));
    const float kx = (x_out - x_in) / tio;
    const float ky = (y_out - y_in) / tio;
    const float kz = (z_out - z_in) / tio;
    const float xl = x_in + kx / ky * (y1 - y_in);
    const float xr = x_in + kx / ky * (y2 - y_in);
    const float zl = z_in + kz / ky * (y1 - y_in);
    const float zr = z_in + kz / ky * (y2 - y_in);
    const float ta = (y1 - y_in) / ky;
    const float tb = (y2 - y_in) / ky;
    const bool fl = ((xl - xc) * (xl - xc) / rx / rx + (zl - zc) * (zl - zc) / rz / rz) <= 1.0f;
    const bool fr = ((xr - xc) * (xr - xc) / rx / rx + (zr - zc) * (zr - zc) / rz / rz) <= 1.0f;
    if (fr && fl) {
        if (ta <= 0.0001f || tb <= 0.0001f) return 0.0f;
        if (ta >= tio || tb >= tio) return 0.0f;
        return fabsf(tb - ta);
    }
    const float x_ = x_in - xc;
    const float z_ = z_in - zc;
    const float a = (kx * kx * rz * rz + kz * kz * rx * rx);
    const float b = kx * x_ * rz * rz + kz * z_ * rx * rx;
    const float c = rz * rz * x_ * x_ + rx * rx * z_ * z_ - rx * rx * rz * rz;
    const float delta = (b * b - a * c);
    if (delta <= 0.00001f) return 0.0f;
    const float t1 = (-b - sqrtf(delta)) / a;
    const float t2 = (-b + sqrtf(delta)) / a;
    if (!fr && !fl) {
        if (!((t1 >= ta) && (t2 <= tb))) return 0.0f;
        if (t2 <= 0.0001f || t1 <= 0.0001f) return 0.0f;
        if (t2 >= tio || t1 >= tio) return 0.0f;
        return t2 - t1;
    }
    if (fl && !fr) {
        if (t2 <= 0.0001f || ta <= 0.0001f) return 0.0f;
        if (t2 >= tio || ta >= tio) return 0.0f;
        return t2 - ta;
    }
    if (tb <= 0.0001f || t1 <= 0.0001f) return 0.0f;
    if (tb >= tio || t1 >= tio) return 0.0f;
    return tb - t1;
}

// World point -> frame of a crystal rotated about y, given cos(-rot), sin(-rot)
// (PESysMatGen.cu:1066-1068, :1305-1320).
__device__ __forceinline__ void to_crystal_frame(float cx, float cy, float cz, float cn, float sn,
                                                 float x, float y, float z, float& xs, float& ys,
                                                 float& zs)
{
    xs = (x - cx) * cn - (z - cz) * sn;
    ys = y - cy;
    zs = (x - cx) * sn + (z - cz) * cn;
}

// Voxel centre of flat index v, rotated about z (PESysMatGen.cu:1031-1052).
// Point of voxel v at fractions (fx, fy, fz) of its extent (1/2: the centre the reference
// uses), rotated about z (PESysMatGen.cu:1031-1052).
__device__ __forceinline__ void voxel_centre(const DevGeom& g, long long v, float cr, float sr,
                                             float& x, float& y, float& z, float fx = 0.5f,
                                             float fy = 0.5f, float fz = 0.5f)
{
    const long long nxy = (long long)g.nx * g.ny;
    const int iz = (int)(v / nxy);
    const long long r = v - (long long)iz * nxy;
    const int iy = (int)(r / g.nx);
    const int ix = (int)(r - (long long)iy * g.nx);
    float xv = ((float)ix - (float)g.nx / 2.0f + fx) * g.wx;
    float yv = ((float)iy - (float)g.ny / 2.0f + fy) * g.wy;
    float zv = ((float)iz - (float)g.nz / 2.0f + fz) * g.wz;
    xv = xv + g.shx;
    yv = yv + g.shy;
    zv = zv + g.shz;
    x = xv * cr - yv * sr;
    y = xv * sr + yv * cr;
    z = zv;
}

}  // namespace sysmat
