// Chord primitives of the FP64 mode (SYSMAT_MODE_FP64): the reference's box and cylinder
// chords (PESysMatGen.cu:20-799) evaluated in double, with the branch structure and the
// thresholds of their restatement: the box chords' eps is the float literal 0.001f widened
// to double, the cylinder chord and the inside chord's depth test compare against the
// double literals the reference writes (0.001, 0.0001, 0.00001).
//
// These are not bit-matched to any float program: they are the FP64 computation the
// float kernels approximate, so divisions by a shared denominator become one reciprocal.
#pragma once

#include <cuda_runtime.h>

namespace sysmat {

constexpr double kEps64 = (double)0.001f;

__device__ __forceinline__ void slab64(double p0, double lo, double hi, double inv, double& t0, double& t1)
{
    if (inv < 0.0) { t0 = (hi - p0) * inv; t1 = (lo - p0) * inv; }
    else           { t0 = (lo - p0) * inv; t1 = (hi - p0) * inv; }
}

// Parallel-axis cases of both box chords (at least one |delta| < eps).  inside = false:
// full crossings only (PESysMatGen.cu:28-232); inside = true: the segment ends inside the
// box (:328-589).  Returns true and sets tmin, tmax, tio when the caller must finish with
// the interval tests; returns false with the result in *out otherwise.
static __device__ __noinline__ bool box64_parallel(const double p0[3], const double p1[3], const double lo[3],
                                            const double hi[3], bool inside, double* out, double* tmin,
                                            double* tmax, double* tio)
{
    bool par[3];
    int npar = 0;
    for (int a = 0; a < 3; ++a) {
        par[a] = fabs(p1[a] - p0[a]) < kEps64;
        npar += par[a];
    }
    *out = 0.0;
    if (npar == 3) return false;
    if (npar == 2) {
        const int m = !par[0] ? 0 : (!par[1] ? 1 : 2);
        for (int a = 0; a < 3; ++a)
            if (a != m && !(p0[a] >= lo[a] && p0[a] <= hi[a])) return false;
        if (!inside) {
            if ((p0[m] <= lo[m] && p1[m] >= hi[m]) || (p1[m] <= lo[m] && p0[m] >= hi[m])) *out = fabs(hi[m] - lo[m]);
            return false;
        }
        *out = p0[m] < p1[m] ? p1[m] - lo[m] : hi[m] - p1[m];
        return false;
    }
    const int q = par[0] ? 0 : (par[1] ? 1 : 2);          // exactly one parallel axis
    if (p0[q] >= hi[q] || p0[q] <= lo[q]) return false;
    const int a0 = (q == 0) ? 1 : 0, a1 = (q == 2) ? 1 : 2;
    const double d0 = p1[a0] - p0[a0], d1 = p1[a1] - p0[a1];
    *tio = sqrt(d0 * d0 + d1 * d1);
    double b0, b1;
    slab64(p0[a0], lo[a0], hi[a0], *tio / d0, *tmin, *tmax);
    slab64(p0[a1], lo[a1], hi[a1], *tio / d1, b0, b1);
    if (*tmin > b1 || b0 > *tmax) return false;
    if (b0 > *tmin) *tmin = b0;
    if (b1 < *tmax) *tmax = b1;
    return true;
}

// Chord of the segment (xi,yi,zi)->(xo,yo,zo) through the box; only full crossings count.
__device__ __forceinline__ double box_chord64(double xi, double yi, double zi, double xo, double yo, double zo,
                                              double x1, double y1, double z1, double x2, double y2, double z2)
{
    const double dx = xo - xi, dy = yo - yi, dz = zo - zi;
    double tmin, tmax, tio;
    if (fabs(dx) < kEps64 || fabs(dy) < kEps64 || fabs(dz) < kEps64) {
        const double p0[3] = {xi, yi, zi}, p1[3] = {xo, yo, zo}, lo[3] = {x1, y1, z1}, hi[3] = {x2, y2, z2};
        double out;
        if (!box64_parallel(p0, p1, lo, hi, false, &out, &tmin, &tmax, &tio)) return out;
    } else {
        tio = sqrt(dx * dx + dy * dy + dz * dz);
        double a0, a1;
        slab64(xi, x1, x2, tio / dx, tmin, tmax);
        slab64(yi, y1, y2, tio / dy, a0, a1);
        if (tmin > a1 || a0 > tmax) return 0.0;
        tmin = a0 > tmin ? a0 : tmin;
        tmax = a1 < tmax ? a1 : tmax;
        slab64(zi, z1, z2, tio / dz, a0, a1);
        if (tmin > a1 || a0 > tmax) return 0.0;
        tmin = a0 > tmin ? a0 : tmin;
        tmax = a1 < tmax ? a1 : tmax;
    }
    if ((tmax - tmin) < kEps64) return 0.0;
    if (tmin >= tio || tmax >= tio) return 0.0;
    if (tmin <= kEps64 || tmax <= kEps64) return 0.0;
    return tmax - tmin;
}

// Chord from the box entry to the end point, which lies inside the box (:314-686).
__device__ __forceinline__ double box_chord_inside64(double xi, double yi, double zi, double xo, double yo,
                                                     double zo, double x1, double y1, double z1, double x2,
                                                     double y2, double z2)
{
    const double dx = xo - xi, dy = yo - yi, dz = zo - zi;
    if (fabs(dy) < 0.001) return 0.0;                       // :321-324
    double tmin, tmax, tio;
    // dy too: in double, 0.001 <= |dy| < (double)0.001f is possible
    if (fabs(dx) < kEps64 || fabs(dy) < kEps64 || fabs(dz) < kEps64) {
        const double p0[3] = {xi, yi, zi}, p1[3] = {xo, yo, zo}, lo[3] = {x1, y1, z1}, hi[3] = {x2, y2, z2};
        double out;
        if (!box64_parallel(p0, p1, lo, hi, true, &out, &tmin, &tmax, &tio)) return out;
    } else {
        tio = sqrt(dx * dx + dy * dy + dz * dz);
        double a0, a1;
        slab64(xi, x1, x2, tio / dx, tmin, tmax);
        slab64(yi, y1, y2, tio / dy, a0, a1);
        if (tmin > a1 || a0 > tmax) return 0.0;
        tmin = a0 > tmin ? a0 : tmin;
        tmax = a1 < tmax ? a1 : tmax;
        slab64(zi, z1, z2, tio / dz, a0, a1);
        if (tmin > a1 || a0 > tmax) return 0.0;
        tmin = a0 > tmin ? a0 : tmin;
        tmax = a1 < tmax ? a1 : tmax;
    }
    if ((tmax - tmin) < kEps64) return 0.0;
    if (tmin >= tio) return 0.0;
    if (tmax <= kEps64) return 0.0;
    if ((tmax >= tio) && (tmin > kEps64)) return tio - tmin;
    if ((tmin <= kEps64) && (tmax <= tio)) return tmax;
    if ((tmin <= kEps64) && (tmax >= tio)) return tio;
    return tmax - tmin;
}

// Terms of the cylinder chord (:688-799) that depend only on the ray (the ray's start point
// is passed to each call: it is shared by a warp's rays and kept outside this per-lane state).
struct RayCyl64 {
    double tio, kx, kz, rx, rz, kk, ikk, iky;
};

__device__ __forceinline__ void ray_cyl64_init(RayCyl64& c, double xi, double yi, double zi, double xo, double yo,
                                               double zo)
{
    const double dx = xo - xi, dy = yo - yi, dz = zo - zi;
    c.tio = sqrt(dx * dx + dy * dy + dz * dz);
    const double it = 1.0 / c.tio;
    c.kx = dx * it;
    const double ky = dy * it;
    c.kz = dz * it;
    c.iky = 1.0 / ky;
    c.rx = c.kx * c.iky;
    c.rz = c.kz * c.iky;
    c.kk = c.kx * c.kx + c.kz * c.kz;
    c.ikk = 1.0 / c.kk;
}

// Chord through the y-parallel cylinder (x - xc)^2 + (z - zc)^2 <= r^2, y in [y1, y2].
// The reference picks one of four entry/exit pairs from the cap tests fl, fr and then checks
// the pair against the cap planes (:730-791).  Where fl, fr and the side crossings t1, t2
// agree, every pair is the overlap [max(t1, ta), min(t2, tb)] of the side and cap intervals;
// at a tie (the ray crossing a cap plane exactly on the rim) the cap test and the side
// crossing are decided by independent roundings and the reference's pair can drop the
// whole chord.  This form takes the overlap, which is continuous there, and keeps the
// reference's thresholds.
__device__ __forceinline__ double ray_cyl64_chord(const RayCyl64& c, double xi, double yi, double zi, double xc,
                                                  double y1, double y2, double zc, double r)
{
    if (fabs(y1 - y2) < 0.001) return 0.0;
    const double xl = xi + c.rx * (y1 - yi), xr = xi + c.rx * (y2 - yi);
    const double zl = zi + c.rz * (y1 - yi), zr = zi + c.rz * (y2 - yi);
    const double ta = (y1 - yi) * c.iky, tb = (y2 - yi) * c.iky;
    const bool fl = (xl - xc) * (xl - xc) + (zl - zc) * (zl - zc) <= r * r;
    const bool fr = (xr - xc) * (xr - xc) + (zr - zc) * (zr - zc) <= r * r;
    if (fl && fr) {
        if (ta <= 0.0001 || tb <= 0.0001) return 0.0;
        if (ta >= c.tio || tb >= c.tio) return 0.0;
        return fabs(tb - ta);
    }
    const double ox = xi - xc, oz = zi - zc;
    const double cr = c.kx * oz - c.kz * ox;
    const double disc = c.kk * r * r - cr * cr;
    if (disc <= 0.00001) return 0.0;
    const double b = -(c.kx * ox + c.kz * oz), sd = sqrt(disc);
    const double t1 = (b - sd) * c.ikk, t2 = (b + sd) * c.ikk;
    const double ea = t1 > ta ? t1 : ta, eb = t2 < tb ? t2 : tb;
    if (!(eb > ea)) return 0.0;                             // side crossings outside the caps
    if (eb <= 0.0001 || ea <= 0.0001) return 0.0;
    if (eb >= c.tio || ea >= c.tio) return 0.0;
    return eb - ea;
}

// Elliptical cylinder ((x' - xc)/rx)^2 + ((z' - zc)/rz)^2 <= 1, y in [y1, y2], with the
// segment's points rotated by theta about the axis first (PESysMatGen.cu:801-947, defined but
// not called by the reference kernels); ct, st = cos(theta), sin(theta).  The expressions are
// the reference's in double; the ending takes the overlap of the side and cap intervals, as
// ray_cyl64_chord does.
__device__ __forceinline__ double ell_chord64(double xi, double yi, double zi, double xo, double yo, double zo,
                                              double xc, double y1, double y2, double zc, double rx, double rz,
                                              double ct, double st)
{
    const double xi_ = xi - xc, zi_ = zi - zc, xo_ = xo - xc, zo_ = zo - zc;
    xi = xc + xi_ * ct + zi_ * st;
    zi = zc - xi_ * st + zi_ * ct;
    xo = xc + xo_ * ct + zo_ * st;
    zo = zc - xo_ * st + zo_ * ct;
    if (fabs(y1 - y2) < 0.001) return 0.0;
    const double tio = sqrt((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
    const double kx = (xo - xi) / tio, ky = (yo - yi) / tio, kz = (zo - zi) / tio;
    const double xl = xi + kx / ky * (y1 - yi), xr = xi + kx / ky * (y2 - yi);
    const double zl = zi + kz / ky * (y1 - yi), zr = zi + kz / ky * (y2 - yi);
    const double ta = (y1 - yi) / ky, tb = (y2 - yi) / ky;
    const bool fl = ((xl - xc) * (xl - xc) / rx / rx + (zl - zc) * (zl - zc) / rz / rz) <= 1.0;
    const bool fr = ((xr - xc) * (xr - xc) / rx / rx + (zr - zc) * (zr - zc) / rz / rz) <= 1.0;
    if (fr && fl) {
        if (ta <= 0.0001 || tb <= 0.0001) return 0.0;
        if (ta >= tio || tb >= tio) return 0.0;
        return fabs(tb - ta);
    }
    const double x_ = xi - xc, z_ = zi - zc;
    const double a = kx * kx * rz * rz + kz * kz * rx * rx;
    const double b = kx * x_ * rz * rz + kz * z_ * rx * rx;
    const double c = rz * rz * x_ * x_ + rx * rx * z_ * z_ - rx * rx * rz * rz;
    const double delta = b * b - a * c;
    if (delta <= 0.00001) return 0.0;
    const double t1 = (-b - sqrt(delta)) / a, t2 = (-b + sqrt(delta)) / a;
    const double ea = t1 > ta ? t1 : ta, eb = t2 < tb ? t2 : tb;
    if (!(eb > ea)) return 0.0;
    if (eb <= 0.0001 || ea <= 0.0001) return 0.0;
    if (eb >= tio || ea >= tio) return 0.0;
    return eb - ea;
}

}  // namespace sysmat
