/* Oracle body, instantiated twice by sysmat_oracle.c: REAL = float (FP32 twin of the
 * reference's arithmetic) and REAL = double (every float variable widened; constants
 * keep the values the reference stores them with).  TEST INFRASTRUCTURE ONLY.
 *
 * Each function states the reference lines it restates.  Expression shapes follow the
 * reference where rounding depends on them (summation order, division order, the places
 * where a double constant promotes a float expression).  Branch thresholds compared
 * against double literals in the reference are compared in double here as well.
 */

#define FN(name) CAT(name, SUFFIX)
#define CAT(a, b) CAT2(a, b)
#define CAT2(a, b) a##b

static inline REAL FN(rmax)(REAL a, REAL b) { return (a >= b) ? a : b; }  /* PESysMatGen.cu:15 */
static inline REAL FN(rmin)(REAL a, REAL b) { return (a <= b) ? a : b; }  /* PESysMatGen.cu:16 */

/* Entry/exit parameters of a segment p0 + t*(p1-p0)/|.| against the slab [lo, hi] of one
 * axis, with the axis' reciprocal step inv = |seg| / (p1 - p0) (PESysMatGen.cu:82-103). */
static inline void FN(slab)(REAL p0, REAL lo, REAL hi, REAL inv, REAL* t0, REAL* t1)
{
    if (inv < 0) { *t0 = (hi - p0) * inv; *t1 = (lo - p0) * inv; }
    else         { *t0 = (lo - p0) * inv; *t1 = (hi - p0) * inv; }
}

/* Common slab intersection for the "one axis parallel" (2 active axes) and general
 * (3 active axes) cases of both box chords.  Returns 0 if the active-axis intervals do
 * not overlap, else 1 with the merged interval; *tio is the segment length measured in
 * the active axes only (PESysMatGen.cu:75-121, :131-177, :186-231, :236-304). */
static int FN(slab_merge)(const REAL p0[3], const REAL p1[3], const REAL lo[3],
                          const REAL hi[3], const int active[3], REAL* tmin, REAL* tmax, REAL* tio)
{
    REAL s = 0;
    int a;
    for (a = 0; a < 3; ++a)
        if (active[a]) s = s + (p1[a] - p0[a]) * (p1[a] - p0[a]);
    *tio = SQRT(s);
    int first = 1;
    REAL lo_t = 0, hi_t = 0;
    for (a = 0; a < 3; ++a) {
        if (!active[a]) continue;
        REAL inv = *tio / (p1[a] - p0[a]);
        REAL t0, t1;
        FN(slab)(p0[a], lo[a], hi[a], inv, &t0, &t1);
        if (first) { lo_t = t0; hi_t = t1; first = 0; continue; }
        if (lo_t > t1 || t0 > hi_t) return 0;
        if (t0 > lo_t) lo_t = t0;
        if (t1 < hi_t) hi_t = t1;
    }
    *tmin = lo_t;
    *tmax = hi_t;
    return 1;
}

/* Chord of segment p0->p1 through the axis-aligned box [lo, hi]; only full crossings
 * count (PESysMatGen.cu:20-312, duplicated at scatter.cu:31-323). */
static REAL FN(box_chord)(REAL xi, REAL yi, REAL zi, REAL xo, REAL yo, REAL zo,
                          REAL x1, REAL y1, REAL z1, REAL x2, REAL y2, REAL z2)
{
    const REAL eps = (REAL)0.001f;
    const REAL p0[3] = {xi, yi, zi}, p1[3] = {xo, yo, zo};
    const REAL lo[3] = {x1, y1, z1}, hi[3] = {x2, y2, z2};
    int par[3], npar = 0, a;
    for (a = 0; a < 3; ++a) { par[a] = FABS(p1[a] - p0[a]) < eps; npar += par[a]; }
    if (npar == 3) return 0;
    if (npar == 2) {
        /* axis-parallel ray: full extent if it starts inside the other two ranges and
         * crosses the whole box along its own axis (:33-66) */
        int m = !par[0] ? 0 : (!par[1] ? 1 : 2);
        for (a = 0; a < 3; ++a)
            if (a != m && !(p0[a] >= lo[a] && p0[a] <= hi[a])) return 0;
        if ((p0[m] <= lo[m] && p1[m] >= hi[m]) || (p1[m] <= lo[m] && p0[m] >= hi[m]))
            return FABS(hi[m] - lo[m]);
        return 0;
    }
    int active[3] = {1, 1, 1};
    if (npar == 1) {
        int q = par[0] ? 0 : (par[1] ? 1 : 2);
        if (p0[q] >= hi[q] || p0[q] <= lo[q]) return 0;       /* :69-72, :125-128, :180-183 */
        active[q] = 0;
    }
    REAL tmin, tmax, tio;
    if (!FN(slab_merge)(p0, p1, lo, hi, active, &tmin, &tmax, &tio)) return 0;
    if ((tmax - tmin) < eps) return 0;                        /* :297-304 */
    if (tmin >= tio || tmax >= tio) return 0;
    if (tmin <= eps || tmax <= eps) return 0;
    return tmax - tmin;
}

/* Chord from the box entry to p1 when p1 lies inside the box (PESysMatGen.cu:314-686). */
static REAL FN(box_chord_inside)(REAL xi, REAL yi, REAL zi, REAL xo, REAL yo, REAL zo,
                                 REAL x1, REAL y1, REAL z1, REAL x2, REAL y2, REAL z2)
{
    if ((double)FABS(yo - yi) < 0.001) return 0;              /* :321-324 */
    const REAL eps = (REAL)0.001f;
    const REAL p0[3] = {xi, yi, zi}, p1[3] = {xo, yo, zo};
    const REAL lo[3] = {x1, y1, z1}, hi[3] = {x2, y2, z2};
    int par[3], npar = 0, a;
    for (a = 0; a < 3; ++a) { par[a] = FABS(p1[a] - p0[a]) < eps; npar += par[a]; }
    if (npar == 3) return 0;
    if (npar == 2) {                                          /* :333-382 */
        int m = !par[0] ? 0 : (!par[1] ? 1 : 2);
        for (a = 0; a < 3; ++a)
            if (a != m && !(p0[a] >= lo[a] && p0[a] <= hi[a])) return 0;
        if (p0[m] < p1[m]) return p1[m] - lo[m];
        if (p0[m] > p1[m]) return hi[m] - p1[m];
        /* equal coordinates cannot occur here: axis m is not parallel */
    }
    int active[3] = {1, 1, 1};
    if (npar == 1) {
        int q = par[0] ? 0 : (par[1] ? 1 : 2);
        if (p0[q] >= hi[q] || p0[q] <= lo[q]) return 0;
        active[q] = 0;
    }
    REAL tmin, tmax, tio;
    if (!FN(slab_merge)(p0, p1, lo, hi, active, &tmin, &tmax, &tio)) return 0;
    if ((tmax - tmin) < eps) return 0;                        /* :657-676 */
    if (tmin >= tio) return 0;
    if (tmax <= eps) return 0;
    if ((tmax >= tio) && (tmin > eps)) return tio - tmin;
    if ((tmin <= eps) && (tmax <= tio)) return tmax;
    if ((tmin <= eps) && (tmax >= tio)) return tio;
    return tmax - tmin;
}

/* Chord through the y-parallel cylinder (x-xc)^2+(z-zc)^2 <= R^2, y in [y1, y2]
 * (PESysMatGen.cu:688-799). */
static REAL FN(cyl_chord)(REAL xi, REAL yi, REAL zi, REAL xo, REAL yo, REAL zo,
                          REAL xc, REAL y1, REAL y2, REAL zc, REAL r)
{
    if ((double)FABS(y1 - y2) < 0.001) return 0;
    REAL dx = xo - xi, dy = yo - yi, dz = zo - zi;
    REAL tio = SQRT(dx * dx + dy * dy + dz * dz);
    REAL kx = dx / tio, ky = dy / tio, kz = dz / tio;
    REAL xl = xi + kx / ky * (y1 - yi);
    REAL xr = xi + kx / ky * (y2 - yi);
    REAL zl = zi + kz / ky * (y1 - yi);
    REAL zr = zi + kz / ky * (y2 - yi);
    REAL ta = (y1 - yi) / ky;
    REAL tb = (y2 - yi) / ky;
    int fl = (xl - xc) * (xl - xc) + (zl - zc) * (zl - zc) <= r * r;
    int fr = (xr - xc) * (xr - xc) + (zr - zc) * (zr - zc) <= r * r;
    if (fl && fr) {                                           /* both caps inside: :730-738 */
        if ((double)ta <= 0.0001 || (double)tb <= 0.0001) return 0;
        if (ta >= tio || tb >= tio) return 0;
        return FABS(tb - ta);
    }
    REAL ox = xi - xc, oz = zi - zc;
    REAL disc = (kx * kx + kz * kz) * r * r - (kx * oz - kz * ox) * (kx * oz - kz * ox);
    if ((double)disc <= 0.00001) return 0;                    /* :745-748 */
    REAL t1 = (-(kx * ox + kz * oz) - SQRT(disc)) / (kx * kx + kz * kz);
    REAL t2 = (-(kx * ox + kz * oz) + SQRT(disc)) / (kx * kx + kz * kz);
    REAL ea, eb;
    if (!fl && !fr) {                                         /* side in, side out: :755-771 */
        if (!(t1 >= ta && t2 <= tb)) return 0;
        ea = t1; eb = t2;
    } else if (fl) { ea = ta; eb = t2; }                      /* left cap in:  :773-781 */
    else           { ea = t1; eb = tb; }                      /* right cap out: :783-791 */
    if ((double)eb <= 0.0001 || (double)ea <= 0.0001) return 0;
    if (eb >= tio || ea >= tio) return 0;
    return eb - ea;
}

/* Chord through the y-parallel elliptical cylinder ((x'-xc)/rx)^2 + ((z'-zc)/rz)^2 <= 1,
 * y in [y1, y2], where (x', z') are the ray's points rotated by theta about the axis
 * (PESysMatGen.cu:801-947; defined there but not called by the reference kernels).
 * ct, st: cos(theta), sin(theta). */
static REAL FN(ell_chord)(REAL xi, REAL yi, REAL zi, REAL xo, REAL yo, REAL zo, REAL xc, REAL y1,
                          REAL y2, REAL zc, REAL rx, REAL rz, REAL ct, REAL st)
{
    REAL xi_ = xi - xc, zi_ = zi - zc, xo_ = xo - xc, zo_ = zo - zc;
    xi = xc + xi_ * ct + zi_ * st;
    zi = zc - xi_ * st + zi_ * ct;
    xo = xc + xo_ * ct + zo_ * st;
    zo = zc - xo_ * st + zo_ * ct;
    if ((double)FABS(y1 - y2) < 0.001) return 0;
    REAL tio = SQRT((xo - xi) * (xo - xi) + (yo - yi) * (yo - yi) + (zo - zi) * (zo - zi));
    REAL kx = (xo - xi) / tio, ky = (yo - yi) / tio, kz = (zo - zi) / tio;
    REAL xl = xi + kx / ky * (y1 - yi);
    REAL xr = xi + kx / ky * (y2 - yi);
    REAL zl = zi + kz / ky * (y1 - yi);
    REAL zr = zi + kz / ky * (y2 - yi);
    REAL ta = (y1 - yi) / ky, tb = (y2 - yi) / ky;
    int fl = ((xl - xc) * (xl - xc) / rx / rx + (zl - zc) * (zl - zc) / rz / rz) <= 1;
    int fr = ((xr - xc) * (xr - xc) / rx / rx + (zr - zc) * (zr - zc) / rz / rz) <= 1;
    if (fr && fl) {
        if ((double)ta <= 0.0001 || (double)tb <= 0.0001) return 0;
        if (ta >= tio || tb >= tio) return 0;
        return FABS(tb - ta);
    }
    REAL x_ = xi - xc, z_ = zi - zc;
    REAL a = kx * kx * rz * rz + kz * kz * rx * rx;
    REAL b = kx * x_ * rz * rz + kz * z_ * rx * rx;
    REAL c = rz * rz * x_ * x_ + rx * rx * z_ * z_ - rx * rx * rz * rz;
    REAL delta = b * b - a * c;
    if ((double)delta <= 0.00001) return 0;
    REAL t1 = (-b - SQRT(delta)) / a;
    REAL t2 = (-b + SQRT(delta)) / a;
    if (!fr && !fl) {
        if (!(t1 >= ta && t2 <= tb)) return 0;
        if ((double)t2 <= 0.0001 || (double)t1 <= 0.0001) return 0;
        if (t2 >= tio || t1 >= tio) return 0;
        return t2 - t1;
    }
    if (fl && !fr) {
        if ((double)t2 <= 0.0001 || (double)ta <= 0.0001) return 0;
        if (t2 >= tio || ta >= tio) return 0;
        return t2 - ta;
    }
    if ((double)tb <= 0.0001 || (double)t1 <= 0.0001) return 0;
    if (tb >= tio || t1 >= tio) return 0;
    return tb - t1;
}

/* ---------------------------------------------------------------------------------- */
/* Geometry decoding shared by the element functions.                                  */

typedef struct {
    REAL x, y, z;
} FN(vec3);

/* Point of voxel v at fractions (fx, fy, fz) of its extent, rotated about z by I[20]*I[7]
 * (PESysMatGen.cu:1031-1052, where the fractions are 1/2: the voxel centre). */
static void FN(voxel_point)(const ogeo* g, long long v, REAL fx, REAL fy, REAL fz, REAL* xo, REAL* yo,
                            REAL* zo)
{
    const float* I = g->I;
    long long nxy = (long long)g->nx * g->ny;
    int iz = (int)(v / nxy);
    long long r = v % nxy;
    int iy = (int)(r / g->nx);
    int ix = (int)(r % g->nx);
    REAL ang = (REAL)I[20] * (REAL)I[7];
    REAL x = ((REAL)ix - (REAL)g->nx / (REAL)2.0f + fx) * (REAL)I[3];
    REAL y = ((REAL)iy - (REAL)g->ny / (REAL)2.0f + fy) * (REAL)I[4];
    REAL z = ((REAL)iz - (REAL)g->nz / (REAL)2.0f + fz) * (REAL)I[5];
    x = x + (REAL)I[8];
    y = y + (REAL)I[9];
    z = z + (REAL)I[10];
    *xo = x * COS(ang) - y * SIN(ang);
    *yo = x * SIN(ang) + y * COS(ang);
    *zo = z;
}

static void FN(voxel_centre)(const ogeo* g, long long v, REAL* xo, REAL* yo, REAL* zo)
{
    FN(voxel_point)(g, v, (REAL)0.5f, (REAL)0.5f, (REAL)0.5f, xo, yo, zo);
}

typedef struct {
    REAL x, y, z;          /* centre, y including the FOV-to-collimator distance */
    REAL w, t, h;          /* x width, y thickness, z height */
    REAL rot;
    REAL mu_t, mu_pe, mu_c, eres;
} FN(crystal);

static void FN(load_crystal)(const ogeo* g, int d, FN(crystal)* c)
{
    const float* D = g->D;
    c->x = (REAL)D[12 * d + 1];
    c->y = (REAL)D[12 * d + 2] + (REAL)g->I[11];
    c->z = (REAL)D[12 * d + 3];
    c->w = (REAL)D[12 * d + 4];
    c->t = (REAL)D[12 * d + 5];
    c->h = (REAL)D[12 * d + 6];
    c->mu_t = (REAL)D[12 * d + 7];
    c->mu_pe = (REAL)D[12 * d + 8];
    c->mu_c = (REAL)D[12 * d + 9];
    c->eres = (REAL)D[12 * d + 10];
    c->rot = (REAL)D[12 * d + 11];
}

/* World point -> frame of a crystal rotated by rot about y (PESysMatGen.cu:1066-1068). */
static inline void FN(to_frame)(const FN(crystal)* c, REAL x, REAL y, REAL z,
                                REAL* xs, REAL* ys, REAL* zs)
{
    *xs = (x - c->x) * COS(-c->rot) - (z - c->z) * SIN(-c->rot);
    *ys = y - c->y;
    *zs = (x - c->x) * SIN(-c->rot) + (z - c->z) * COS(-c->rot);
}

/* ---------------------------------------------------------------------------------- */
/* Photoelectric matrix element A[d][v] (PESysMatGen.cu:951-1364) for a source at
 * (xI, yI, zI), with g->div[0..2] sub-elements of crystal d along x, depth and z (the
 * reference's 8 x 16 x 8).                                                              */

static REAL FN(pe_element_at)(const ogeo* g, int d, REAL xI, REAL yI, REAL zI, int* cand_c, int* cand_h,
                              int* ncand_h, pe_counts* cnt, REAL* per_sub)
{
    const float* C = g->C;
    const REAL fov = (REAL)g->I[11];
    FN(crystal) cd;
    FN(load_crystal)(g, d, &cd);
    REAL xIs, yIs, zIs;
    FN(to_frame)(&cd, xI, yI, zI, &xIs, &yIs, &zIs);
    const REAL bx1 = -cd.w / (REAL)2.0f, bx2 = cd.w / (REAL)2.0f;
    const REAL by1 = -cd.t / (REAL)2.0f, by2 = cd.t / (REAL)2.0f;
    const REAL bz1 = -cd.h / (REAL)2.0f, bz2 = cd.h / (REAL)2.0f;
    if (!(cd.mu_t > (REAL)0.01f)) return 0;                    /* :1107, :1194 */

    /* ---- cone culling of other crystals and of holes (:1105-1186) ---- */
    REAL dist = SQRT((cd.y - yI) * (cd.y - yI) + (cd.x - xI) * (cd.x - xI) + (cd.z - zI) * (cd.z - zI));
    REAL crit_self = SQRT(cd.w * cd.w + cd.h * cd.h + cd.t * cd.t) / dist / (REAL)2.0f;
    REAL ux = (cd.x - xI) / dist, uy = (cd.y - yI) / dist, uz = (cd.z - zI) / dist;
    int nc = 0;
    for (int o = 0; o < g->ncry; ++o) {
        if (o == d) continue;
        FN(crystal) co;
        FN(load_crystal)(g, o, &co);
        REAL crit = SQRT(co.w * co.w + co.h * co.h + co.t * co.t);
        REAL L = SQRT((xI - co.x) * (xI - co.x) + (yI - co.y) * (yI - co.y) + (zI - co.z) * (zI - co.z));
        crit = crit / L / (REAL)2.0f;
        REAL vx = (co.x - xI) / L, vy = (co.y - yI) / L, vz = (co.z - zI) / L;
        if (SQRT((vz - uz) * (vz - uz) + (vy - uy) * (vy - uy) + (vx - ux) * (vx - ux)) <= crit + crit_self)
            cand_c[nc++] = o;
    }
    int hid = 0, hoff = 0;
    for (int m = 0; m < g->L; ++m) {
        int n = 0;
        for (int j = 0; j < g->nh[m]; ++j, ++hid) {
            REAL hx = (REAL)C[hid * 9 + 100];
            REAL hy1 = (REAL)C[hid * 9 + 101] + fov;
            REAL hy2 = (REAL)C[hid * 9 + 102] + fov;
            REAL hz = (REAL)C[hid * 9 + 103];
            REAL hr = (REAL)C[hid * 9 + 104];
            REAL hy = (hy1 + hy2) / (REAL)2.0f;
            REAL crit = SQRT(hr * hr * (REAL)4 + (hy1 - hy2) * (hy1 - hy2)) / (REAL)2.0f;
            REAL L = SQRT((xI - hx) * (xI - hx) + (yI - hy) * (yI - hy) + (zI - hz) * (zI - hz));
            crit = crit / L;
            REAL vx = (hx - xI) / L, vy = (hy - yI) / L, vz = (hz - zI) / L;
            if (SQRT((vz - uz) * (vz - uz) + (vy - uy) * (vy - uy) + (vx - ux) * (vx - ux)) <= crit + crit_self)
                cand_h[hoff + n++] = hid;
        }
        ncand_h[m] = n;
        hoff += n;
    }
    if (cnt) { cnt->cand_crystals = nc; cnt->cand_holes = hoff; }

    /* ---- sub-element loop, order z, x, y (:1196-1362) ---- */
    const unsigned NXS = (unsigned)g->div[0], NYS = (unsigned)g->div[1], NZS = (unsigned)g->div[2];
    const REAL cr = COS(cd.rot), sr = SIN(cd.rot);
    REAL sum = 0;
    for (unsigned iz = 0; iz < NZS; ++iz)
    for (unsigned ix = 0; ix < NXS; ++ix)
    for (unsigned iy = 0; iy < NYS; ++iy) {
        REAL xDs = -cd.w / (REAL)2.0f + (REAL)((REAL)ix + (REAL)0.5f) / (REAL)NXS * cd.w;
        REAL zDs = -cd.h / (REAL)2.0f + (REAL)((REAL)iz + (REAL)0.5f) / (REAL)NZS * cd.h;
        REAL yDs = -cd.t / (REAL)2.0f + (REAL)((REAL)iy + (REAL)0.5f) / (REAL)NYS * cd.t;
        REAL xD = cd.x + (xDs * cr - zDs * sr);
        REAL zD = cd.z + (xDs * sr + zDs * cr);
        REAL yD = cd.y + yDs;
        REAL dsq = (yD - yI) * (yD - yI) + (xD - xI) * (xD - xI) + (zD - zI) * (zD - zI);
        REAL cosang = (yD - yI) / SQRT(dsq);

        /* solid angle: largest of the three face projections, evaluated in double
         * because 4*M_PI promotes the expression (:1223-1231) */
        double fourpi_d2 = 4 * M_PI * (double)dsq;
        REAL sax = (REAL)((double)(cd.t * cd.h / (REAL)NZS / (REAL)NYS) / fourpi_d2 *
                          (double)FABS((xD - xI) * cr - (zD - zI) * sr) / (double)SQRT(dsq));
        REAL saz = (REAL)((double)(cd.w * cd.t / (REAL)NXS / (REAL)NYS) / fourpi_d2 *
                          (double)FABS((xD - xI) * sr + (zD - zI) * cr) / (double)SQRT(dsq));
        REAL say = (REAL)((double)(cd.w * cd.h / (REAL)NXS / (REAL)NZS) / fourpi_d2 *
                          (double)FABS(yD - yI) / (double)SQRT(dsq));
        REAL sa = FN(rmax)(FN(rmax)(sax, say), saz);

        REAL att = 0;
        for (int m = 0; m < g->L; ++m) {                        /* plate bypass penalty :1240-1254 */
            const float* Lh = C + (m + 1) * 10;
            REAL x1 = -(REAL)Lh[1] / (REAL)2.0f, x2 = (REAL)Lh[1] / (REAL)2.0f;
            REAL y1 = -(REAL)Lh[2] / (REAL)2.0f + fov + (REAL)Lh[4];
            REAL y2 = (REAL)Lh[2] / (REAL)2.0f + fov + (REAL)Lh[4];
            REAL z1 = -(REAL)Lh[3] / (REAL)2.0f, z2 = (REAL)Lh[3] / (REAL)2.0f;
            REAL tl = FN(box_chord)(xI, yI, zI, xD, yD, zD, x1, y1, z1, x2, y2, z2);
            if (tl < (REAL)0.1f) att = att + (REAL)100000.0f;
        }
        hoff = 0;
        for (int m = 0; m < g->L; ++m) {                        /* holes and septa :1257-1286 */
            REAL len = 0;
            REAL lcol = (REAL)C[(m + 1) * 10 + 2] / cosang;
            REAL mu_layer = (REAL)C[(m + 1) * 10 + 5];
            for (int j = 0; j < ncand_h[m]; ++j) {
                int h = cand_h[hoff + j];
                REAL tmp;
                if (g->S && g->S[3 * h] > 0.0f) {               /* elliptical hole (extension) */
                    const REAL th = (REAL)g->S[3 * h + 2];
                    tmp = FN(ell_chord)(xI, yI, zI, xD, yD, zD, (REAL)C[h * 9 + 100],
                                        (REAL)C[h * 9 + 101] + fov, (REAL)C[h * 9 + 102] + fov,
                                        (REAL)C[h * 9 + 103], (REAL)g->S[3 * h], (REAL)g->S[3 * h + 1],
                                        COS(th), SIN(th));
                } else {
                    tmp = FN(cyl_chord)(xI, yI, zI, xD, yD, zD, (REAL)C[h * 9 + 100],
                                        (REAL)C[h * 9 + 101] + fov, (REAL)C[h * 9 + 102] + fov,
                                        (REAL)C[h * 9 + 103], (REAL)C[h * 9 + 104]);
                }
                if (cnt && tmp != 0) cnt->hole_hits++;
                len = len + tmp;
                att = att + (REAL)C[h * 9 + 105] * tmp;
            }
            hoff += ncand_h[m];
            if ((lcol - len) >= (REAL)0.00001f) att = att + mu_layer * (lcol - len);
        }
        for (int j = 0; j < nc; ++j) {                          /* other crystals :1290-1325 */
            FN(crystal) co;
            FN(load_crystal)(g, cand_c[j], &co);
            REAL xa, ya, za, xb, yb, zb;
            FN(to_frame)(&co, xI, yI, zI, &xa, &ya, &za);
            FN(to_frame)(&co, xD, yD, zD, &xb, &yb, &zb);
            REAL la = FN(box_chord)(xa, ya, za, xb, yb, zb, (REAL)-0.5f * co.w, (REAL)-0.5f * co.t,
                                    (REAL)-0.5f * co.h, (REAL)0.5f * co.w, (REAL)0.5f * co.t,
                                    (REAL)0.5f * co.h);
            if (cnt && la != 0) cnt->crystal_hits++;
            att = att + la * co.mu_t;
        }
        /* self attenuation from crystal entry to the sub-element entry (:1329-1346) */
        REAL ux1 = ((REAL)ix / (REAL)NXS - (REAL)0.5f) * cd.w;
        REAL ux2 = (((REAL)ix + (REAL)1.0f) / (REAL)NXS - (REAL)0.5f) * cd.w;
        REAL uy1 = ((REAL)iy / (REAL)NYS - (REAL)0.5f) * cd.t;
        REAL uy2 = (((REAL)iy + (REAL)1.0f) / (REAL)NYS - (REAL)0.5f) * cd.t;
        REAL uz1 = ((REAL)iz / (REAL)NZS - (REAL)0.5f) * cd.h;
        REAL uz2 = (((REAL)iz + (REAL)1.0f) / (REAL)NZS - (REAL)0.5f) * cd.h;
        REAL l1 = FN(box_chord_inside)(xIs, yIs, zIs, xDs, yDs, zDs, bx1, by1, bz1, bx2, by2, bz2);
        REAL l2 = FN(box_chord_inside)(xIs, yIs, zIs, xDs, yDs, zDs, ux1, uy1, uz1, ux2, uy2, uz2);
        att = att + (l1 - l2) * cd.mu_t;
        REAL eff = (REAL)1.0f * EXP(-att);
        /* absorption along the extended ray inside the sub-element (:1352-1357) */
        REAL dl = SQRT(dsq);
        REAL xt = xDs + (REAL)1000.0f * (xDs - xIs) / dl;
        REAL yt = yDs + (REAL)1000.0f * (yDs - yIs) / dl;
        REAL zt = zDs + (REAL)1000.0f * (zDs - zIs) / dl;
        REAL labs = FN(box_chord)(xIs, yIs, zIs, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
        REAL absf = ((REAL)1.0f - EXP(-labs * cd.mu_t)) * cd.mu_pe / cd.mu_t;
        if (cnt) cnt->subelements++;
        if (per_sub) per_sub[((long long)iz * NXS + ix) * NYS + iy] = eff * sa * absf;
        sum = sum + eff * sa * absf;
    }
    return sum;
}

/* Element of voxel v: the reference's voxel-centre source when g->vsub is 1 x 1 x 1, else
 * the mean over the centres of a vsub[0] x vsub[1] x vsub[2] grid of source points over the
 * voxel (an extension: the reference has one source point per voxel), summed in double. */
static REAL FN(pe_element)(const ogeo* g, int d, long long v, int* cand_c, int* cand_h,
                           int* ncand_h, pe_counts* cnt)
{
    const int sx = g->vsub[0], sy = g->vsub[1], sz = g->vsub[2];
    REAL xI, yI, zI;
    if (sx == 1 && sy == 1 && sz == 1) {
        FN(voxel_centre)(g, v, &xI, &yI, &zI);
        return FN(pe_element_at)(g, d, xI, yI, zI, cand_c, cand_h, ncand_h, cnt, NULL);
    }
    double acc = 0.0;
    for (int jz = 0; jz < sz; ++jz)
    for (int jy = 0; jy < sy; ++jy)
    for (int jx = 0; jx < sx; ++jx) {
        FN(voxel_point)(g, v, ((REAL)jx + (REAL)0.5f) / (REAL)sx, ((REAL)jy + (REAL)0.5f) / (REAL)sy,
                        ((REAL)jz + (REAL)0.5f) / (REAL)sz, &xI, &yI, &zI);
        acc += (double)FN(pe_element_at)(g, d, xI, yI, zI, cand_c, cand_h, ncand_h, cnt, NULL);
    }
    return (REAL)(acc / (double)(sx * sy * sz));
}

/* ---------------------------------------------------------------------------------- */
/* Compton helpers (scatter.cu:961-1038).                                               */

static REAL FN(kn_shape)(REAL theta, REAL e0)
{
    REAL c = COS(theta);
    REAL alpha = e0 / (REAL)511.0f;
    REAL f1 = alpha * ((REAL)1.0f - c);
    REAL f2 = (REAL)1.0f + c * c;
    return f2 / ((REAL)1.0f + f1) / ((REAL)1.0f + f1) * ((REAL)1.0f + f1 * f1 / f2 / ((REAL)1.0f + f1));
}

/* Left Riemann sum with floor((hi-lo)/step)+1 terms (scatter.cu:980-993). */
static REAL FN(kn_sum)(REAL e0, REAL lo, REAL hi, REAL step)
{
    REAL s = 0;
    int n = (int)((hi - lo) / step);
    for (int i = 0; i <= n; ++i) {
        REAL th = lo + (REAL)i * step;
        s = s + FN(kn_shape)(th, e0) * SIN(th) * step;
    }
    return s;
}

static REAL FN(cone_angle)(REAL xs, REAL ys, REAL zs, REAL xa, REAL ya, REAL za,
                           REAL xd, REAL yd, REAL zd)
{
    REAL a0 = xa - xs, a1 = ya - ys, a2 = za - zs;
    REAL b0 = xd - xa, b1 = yd - ya, b2 = zd - za;
    REAL dot = b0 * a0 + b1 * a1 + b2 * a2;
    REAL ma = SQRT(a0 * a0 + a1 * a1 + a2 * a2);
    REAL mb = SQRT(b0 * b0 + b1 * b1 + b2 * b2);
    REAL c = dot / (ma * mb);
    if (c > (REAL)1.0f) c = (REAL)1.0f;
    if (c < (REAL)-1.0f) c = (REAL)-1.0f;
    return ACOS(c);
}

static REAL FN(window_prob)(REAL e, REAL res, REAL lo, REAL hi)
{
    REAL sigma = res / (REAL)2.35482f * e;
    REAL s2 = (REAL)((double)sigma * sqrt(2.0));
    REAL z1 = (lo - e) / s2;
    REAL z2 = (hi - e) / s2;
    return (REAL)0.5f * (ERF(z2) - ERF(z1));
}

static inline REAL FN(dist3)(REAL x1, REAL y1, REAL z1, REAL x2, REAL y2, REAL z2)
{
    return SQRT((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2) + (z1 - z2) * (z1 - z2));
}

/* One primary-Compton work item: scatter point S with weight w_s (already including the
 * interaction probability), detector crystal d, voxel v.  Shared tail of
 * crystalScatterSysMatCuda (scatter.cu:1232-1427) and collimatorScatterSysMatCuda
 * (scatter.cu:1728-1924).  `kind` 1 = crystal k is the scatterer (attenuators skip d and
 * k, crystal bitmap), 2 = hole k (attenuators skip d, collimator bitmap).  Returns the
 * contribution rounded as the reference's float atomicAdd does. */
/* ---- native collimator-scatter model (an extension, no reference counterpart) ---- */

static int FN(hole_layer)(const ogeo* g, int h, int* begin)
{
    int b = 0;
    for (int m = 0; m < g->L; ++m) {
        if (h < b + g->nh[m]) { if (begin) *begin = b; return m; }
        b += g->nh[m];
    }
    if (begin) *begin = b;
    return g->L - 1;
}

/* The reference's crystal-relationship predicate for hole i and crystals j, k
 * (scatter.cu:1963-2006, raw coordinates), for any hole. */
static int FN(collimator_related)(const ogeo* g, int i, int j, int k)
{
    const float* C = g->C;
    const float* D = g->D;
    float xi = C[100 + 9 * i], yi = (C[101 + 9 * i] + C[102 + 9 * i]) / 2.0f, zi = C[103 + 9 * i];
    const float *pj = D + 12 * j, *pk = D + 12 * k;
    float rj = sqrtf(pj[4] * pj[4] + pj[6] * pj[6] + pj[5] * pj[5]) / 2.0f;
    float lij = sqrtf((xi - pj[1]) * (xi - pj[1]) + (yi - pj[2]) * (yi - pj[2]) + (zi - pj[3]) * (zi - pj[3]));
    float cji = rj / lij;
    float rk = sqrtf(pk[4] * pk[4] + pk[6] * pk[6] + pk[5] * pk[5]) / 2.0f;
    float lik = sqrtf((pk[1] - xi) * (pk[1] - xi) + (pk[2] - yi) * (pk[2] - yi) + (pk[3] - zi) * (pk[3] - zi));
    float cki = rk / lik;
    float ax = (pk[1] - xi) / lik, ay = (pk[2] - yi) / lik, az = (pk[3] - zi) / lik;
    float bx = (pj[1] - xi) / lij, by = (pj[2] - yi) / lij, bz = (pj[3] - zi) / lij;
    float dd = sqrtf((ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz));
    return dd <= cki + cji;
}

/* Tungsten from the centre S of hole h to the detector point: sum_m mu_pe,m L_m and
 * sum_m mu_C,m L_m with L_m = plate chord of layer m minus its hole chords (the scatter hole's
 * own part is its exit distance from S; in its own layer the plate chord runs from the plate
 * entry seen from the detector point to S). */
static void FN(tungsten_path)(const ogeo* g, int h, REAL sx, REAL sy, REAL sz, REAL dx, REAL dy, REAL dz,
                              REAL* w_pe, REAL* w_c)
{
    const float* C = g->C;
    const REAL fov = (REAL)g->I[11];
    *w_pe = 0;
    *w_c = 0;
    int hb;
    const int mh = FN(hole_layer)(g, h, &hb);
    REAL ex = dx - sx, ey = dy - sy, ez = dz - sz;
    REAL len = SQRT(ex * ex + ey * ey + ez * ez);
    REAL kx = ex / len, ky = ey / len, kz = ez / len;
    int begin = 0;
    for (int m = 0; m < g->L; ++m) {
        const float* Lh = C + (m + 1) * 10;
        REAL x1 = -(REAL)Lh[1] / (REAL)2.0f, x2 = (REAL)Lh[1] / (REAL)2.0f;
        REAL y1 = -(REAL)Lh[2] / (REAL)2.0f + fov + (REAL)Lh[4];
        REAL y2 = (REAL)Lh[2] / (REAL)2.0f + fov + (REAL)Lh[4];
        REAL z1 = -(REAL)Lh[3] / (REAL)2.0f, z2 = (REAL)Lh[3] / (REAL)2.0f;
        REAL box = (m == mh) ? FN(box_chord_inside)(dx, dy, dz, sx, sy, sz, x1, y1, z1, x2, y2, z2)
                             : FN(box_chord)(sx, sy, sz, dx, dy, dz, x1, y1, z1, x2, y2, z2);
        if (box != 0) {
            REAL holes = 0;
            for (int j = begin; j < begin + g->nh[m]; ++j) {
                REAL hx = (REAL)C[100 + 9 * j], hy1 = (REAL)C[101 + 9 * j] + fov, hy2 = (REAL)C[102 + 9 * j] + fov;
                REAL hz = (REAL)C[103 + 9 * j], r = (REAL)C[104 + 9 * j];
                if (j == h) {
                    REAL kk = kx * kx + kz * kz, t = len;
                    if (kk > 0) t = FN(rmin)(t, r / SQRT(kk));
                    if (ky > 0) t = FN(rmin)(t, (hy2 - sy) / ky);
                    else if (ky < 0) t = FN(rmin)(t, (hy1 - sy) / ky);
                    holes = holes + t;
                } else {
                    holes = holes + FN(cyl_chord)(sx, sy, sz, dx, dy, dz, hx, hy1, hy2, hz, r);
                }
            }
            REAL L = box - holes;
            if (L > 0) {
                *w_pe = *w_pe + (REAL)Lh[6] * L;
                *w_c = *w_c + (REAL)Lh[7] * L;
            }
        }
        begin += g->nh[m];
    }
}

static REAL FN(scatter_item)(const ogeo* g, int kind, int d, int k, REAL xs, REAL ys, REAL zs,
                             REAL w_s, const FN(crystal)* cd, REAL xI, REAL yI, REAL zI,
                             REAL xIs, REAL yIs, REAL zIs, REAL e0, REAL lo_w, REAL hi_w,
                             REAL integ, const uint32_t* bitmap, double* trace)
{
    REAL xDs = -cd->w / (REAL)2.0f + (REAL)((REAL)0 + (REAL)0.5f) / (REAL)1 * cd->w;
    REAL zDs = -cd->h / (REAL)2.0f + (REAL)((REAL)0 + (REAL)0.5f) / (REAL)1 * cd->h;
    REAL yDs = -cd->t / (REAL)2.0f + (REAL)((REAL)0 + (REAL)0.5f) / (REAL)1 * cd->t;
    REAL xD = cd->x + (xDs * COS(cd->rot) - zDs * SIN(cd->rot));
    REAL zD = cd->z + (xDs * SIN(cd->rot) + zDs * COS(cd->rot));
    REAL yD = cd->y + yDs;

    REAL cone = FN(cone_angle)(xI, yI, zI, xs, ys, zs, xD, yD, zD);
    REAL es = e0 / ((REAL)1.0f + (e0 / (REAL)511.0f) * ((REAL)1.0f - COS(cone)));
    REAL res_s = cd->eres * SQRT(es / e0);
    if (trace) {
        trace[1] = (double)(es * ((REAL)1 + (REAL)2 * res_s / (REAL)2.35482f)) - (double)lo_w;
        trace[2] = (double)hi_w - (double)(es * ((REAL)1 - (REAL)2 * res_s / (REAL)2.35482f));
    }
    if ((es * ((REAL)1 + (REAL)2 * res_s / (REAL)2.35482f)) <= lo_w ||
        (es * ((REAL)1 - (REAL)2 * res_s / (REAL)2.35482f)) >= hi_w)
        return 0;                                              /* 2-sigma window reject :1263 */
    REAL pwin = FN(window_prob)(es, res_s, lo_w, hi_w);
    REAL lsd = FN(dist3)(xs, ys, zs, xD, yD, zD);
    REAL rdet = SQRT(cd->w * cd->w / (REAL)1 / (REAL)1 + cd->h * cd->h / (REAL)1 / (REAL)1 +
                     cd->t * cd->t / (REAL)1 / (REAL)1) / (REAL)2.0f;
    REAL phi;
    if (lsd * SIN(cone) * (REAL)2.0f <= rdet) phi = (REAL)(2.0f * M_PI);
    else phi = (REAL)4.0f * ASIN(FN(rmin)(rdet / (REAL)2.0f / lsd / SIN(cone), (REAL)1.0f));

    REAL xss, yss, zss;
    FN(to_frame)(cd, xs, ys, zs, &xss, &yss, &zss);
    REAL ux1 = ((REAL)0 / (REAL)1 - (REAL)0.5f) * cd->w, ux2 = (((REAL)0 + (REAL)1.0f) / (REAL)1 - (REAL)0.5f) * cd->w;
    REAL uy1 = ((REAL)0 / (REAL)1 - (REAL)0.5f) * cd->t, uy2 = (((REAL)0 + (REAL)1.0f) / (REAL)1 - (REAL)0.5f) * cd->t;
    REAL uz1 = ((REAL)0 / (REAL)1 - (REAL)0.5f) * cd->h, uz2 = (((REAL)0 + (REAL)1.0f) / (REAL)1 - (REAL)0.5f) * cd->h;
    REAL dis = FN(dist3)(xss, yss, zss, xIs, yIs, zIs);
    REAL xt = xss + (REAL)1000.0f * (xss - xIs) / dis;
    REAL yt = yss + (REAL)1000.0f * (yss - yIs) / dis;
    REAL zt = zss + (REAL)1000.0f * (zss - zIs) / dis;
    REAL lthr = FN(box_chord)(xIs, yIs, zIs, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
    const REAL cx[8] = {ux1, ux2, ux1, ux1, ux2, ux2, ux1, ux2};   /* corner order :1313-1320 */
    const REAL cy[8] = {uy1, uy1, uy2, uy1, uy2, uy1, uy2, uy2};
    const REAL cz[8] = {uz1, uz1, uz1, uz2, uz1, uz2, uz2, uz2};
    REAL th[8];
    for (int i = 0; i < 8; ++i)
        th[i] = FN(cone_angle)(xIs, yIs, zIs, xss, yss, zss, cx[i], cy[i], cz[i]);
    REAL tmin = th[0], tmax = th[0];
    for (int i = 1; i < 8; ++i) {
        if (th[i] > tmax) tmax = th[i];
        if (th[i] < tmin) tmin = th[i];
    }
    if (lthr > (REAL)0.001f) tmin = 0;
    if (trace) {
        trace[3] = (double)lthr;
        trace[4] = (double)((tmax - tmin) / (REAL)0.01f);
        trace[5] = (double)tmin;
        trace[6] = (double)tmax;
    }
    REAL ratio = FN(kn_sum)(e0, tmin, tmax, (REAL)0.01f) / integ;

    /* attenuation by other crystals flagged in the relationship bitmap (:1343-1401) */
    REAL att = 0;
    for (int a = 0; a < g->ncry; ++a) {
        if (a == d) continue;
        if (kind == 1 && a == k) continue;
        if (kind == 3) {                                       /* native: predicate, any layer */
            if (!FN(collimator_related)(g, k, d, a)) continue;
        } else {
            long long bit;
            if (kind == 1) {
                long long i = k < d ? k : d, j = k < d ? d : k;
                long long pair = i * g->ncry - (i * (i + 1)) / 2 + j;
                bit = pair * g->ncry + a;
            } else {
                bit = ((long long)k * g->ncry + d) * g->ncry + a;
            }
            if (!((bitmap[bit >> 5] >> (bit & 31)) & 1u)) continue;
        }
        FN(crystal) ca;
        FN(load_crystal)(g, a, &ca);
        REAL mpe = ca.mu_pe * e0 * e0 * e0 / es / es / es;
        REAL mc = ca.mu_c * e0 / es;
        REAL mt = mpe + mc;
        REAL xa, ya, za, xb, yb, zb;
        FN(to_frame)(&ca, xs, ys, zs, &xa, &ya, &za);
        FN(to_frame)(&ca, xD, yD, zD, &xb, &yb, &zb);
        REAL la = FN(box_chord)(xa, ya, za, xb, yb, zb, (REAL)-0.5f * ca.w, (REAL)-0.5f * ca.t,
                                (REAL)-0.5f * ca.h, (REAL)0.5f * ca.w, (REAL)0.5f * ca.t,
                                (REAL)0.5f * ca.h);
        att = att + la * mt;
    }
    if (kind == 3) {                                           /* native: tungsten at E' */
        REAL w_pe, w_c;
        FN(tungsten_path)(g, k, xs, ys, zs, xD, yD, zD, &w_pe, &w_c);
        if (w_pe != 0 || w_c != 0) {
            REAL mpe_w = w_pe * e0 * e0 * e0 / es / es / es;
            REAL mc_w = w_c * e0 / es;
            att = att + (mpe_w + mc_w);
        }
    }
    const REAL bx1 = -cd->w / (REAL)2.0f, bx2 = cd->w / (REAL)2.0f;
    const REAL by1 = -cd->t / (REAL)2.0f, by2 = cd->t / (REAL)2.0f;
    const REAL bz1 = -cd->h / (REAL)2.0f, bz2 = cd->h / (REAL)2.0f;
    REAL l1 = FN(box_chord_inside)(xss, yss, zss, xDs, yDs, zDs, bx1, by1, bz1, bx2, by2, bz2);
    REAL l2 = FN(box_chord_inside)(xss, yss, zss, xDs, yDs, zDs, ux1, uy1, uz1, ux2, uy2, uz2);
    REAL mpe_s = cd->mu_pe * e0 * e0 * e0 / es / es / es;
    REAL mc_s = cd->mu_c * e0 / es;
    REAL mt_s = mpe_s + mc_s;
    att = att + (l1 - l2) * mt_s;
    xt = xDs + (REAL)1000.0f * (xDs - xss) / lsd;
    yt = yDs + (REAL)1000.0f * (yDs - yss) / lsd;
    zt = zDs + (REAL)1000.0f * (zDs - zss) / lsd;
    REAL labs = FN(box_chord)(xss, yss, zss, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
    double c = (double)(w_s * phi / (REAL)2.0f) / M_PI * (double)ratio * (double)pwin *
               (double)EXP(-att) * (double)((REAL)1.0f - EXP(-labs * mt_s)) * (double)mpe_s / (double)mt_s;
    if (trace) {
        trace[0] = (double)(REAL)c;
        trace[7] = (double)att;
        trace[8] = (double)phi;
    }
    return (REAL)c;
}

/* Scatter matrix element for (d, v): part 1 = crystal scatter (scatter.cu:1077-1437),
 * part 2 = collimator scatter with the combined program's hole solid angle
 * (scatter.cu:1711-1716), part 3 = collimator scatter with the collimator-only program's
 * solid angle (ScatterGen_Collimator/scatter.cu:1212-1215). */
static REAL FN(scatter_element)(const ogeo* g, int part, int d, long long v, const float* pe,
                                const uint32_t* bitmap, double* trace)
{
    const float* P = g->P;
    const float* C = g->C;
    if ((int)floor((double)(P[0] + 0.5f)) != 1) return 0;
    FN(crystal) cd;
    FN(load_crystal)(g, d, &cd);
    if (!(cd.mu_t > (REAL)0.01f)) return 0;
    REAL e0 = (REAL)P[7];
    REAL lo_w, hi_w;
    if ((int)floor((double)(P[4] + 0.5f)) > 0) { lo_w = (REAL)P[5]; hi_w = (REAL)P[6]; }
    else {
        lo_w = ((REAL)1 - cd.eres / (REAL)2.0f) * e0;
        hi_w = ((REAL)1 + cd.eres / (REAL)2.0f) * e0;
    }
    REAL integ = FN(kn_sum)(e0, (REAL)0.0f, (REAL)(float)M_PI, (REAL)0.01f);
    REAL xI, yI, zI;
    FN(voxel_centre)(g, v, &xI, &yI, &zI);
    REAL xIs, yIs, zIs;
    FN(to_frame)(&cd, xI, yI, zI, &xIs, &yIs, &zIs);
    const REAL fov = (REAL)g->I[11];
    REAL sum = 0;
    if (part == 1) {
        for (int k = 0; k < g->ncry; ++k) {
            if (k == d) continue;
            REAL prob = (REAL)pe[(long long)k * g->nvox + v] * cd.mu_c / cd.mu_pe;
            FN(crystal) ck;
            FN(load_crystal)(g, k, &ck);
            sum = sum + FN(scatter_item)(g, 1, d, k, ck.x, ck.y, ck.z, prob, &cd, xI, yI, zI,
                                         xIs, yIs, zIs, e0, lo_w, hi_w, integ, bitmap,
                                         trace ? trace + 9 * k : NULL);
        }
    } else if (part == 4) {                                    /* native collimator model */
        for (int h = 0; h < g->nholes; ++h) {
            const int m = FN(hole_layer)(g, h, NULL);
            REAL hx = (REAL)C[h * 9 + 100];
            REAL hy = ((REAL)C[h * 9 + 101] + (REAL)C[h * 9 + 102]) / (REAL)2.0f + fov;
            REAL hz = (REAL)C[h * 9 + 103];
            REAL lih = FN(dist3)(xI, yI, zI, hx, hy, hz);
            REAL T = (REAL)C[h * 9 + 102] - (REAL)C[h * 9 + 101];
            REAL vr = (REAL)0.1f;
            REAL sa = (REAL)(((double)(vr * vr) * M_PI + (double)(T * vr)) /
                             (4.0f * M_PI * (double)lih * (double)lih) * (double)FABS(hy - yI) / (double)lih);
            REAL prob = sa / (REAL)C[(m + 1) * 10 + 5] * (REAL)C[(m + 1) * 10 + 7];
            sum = sum + FN(scatter_item)(g, 3, d, h, hx, hy, hz, prob, &cd, xI, yI, zI,
                                         xIs, yIs, zIs, e0, lo_w, hi_w, integ, bitmap,
                                         trace ? trace + 9 * h : NULL);
        }
    } else {
        for (int h = 0; h < g->nh0; ++h) {
            REAL hx = (REAL)C[h * 9 + 100];
            REAL hy = ((REAL)C[h * 9 + 101] + (REAL)C[h * 9 + 102]) / (REAL)2.0f + fov;
            REAL hz = (REAL)C[h * 9 + 103];
            REAL lih = FN(dist3)(xI, yI, zI, hx, hy, hz);
            REAL T = (REAL)C[h * 9 + 102] - (REAL)C[h * 9 + 101];
            REAL sa;
            if (part == 2) {
                REAL vr = (REAL)0.1f;
                sa = (REAL)(((double)(vr * vr) * M_PI + (double)(T * vr)) /
                            (4.0f * M_PI * (double)lih * (double)lih) * (double)FABS(hy - yI) /
                            (double)lih);
            } else {
                REAL vr = (REAL)0.2f;
                sa = (vr * vr + T * vr) / ((REAL)4.0f * lih * lih);
            }
            REAL prob = sa / (REAL)C[15] * (REAL)C[17];
            sum = sum + FN(scatter_item)(g, 2, d, h, hx, hy, hz, prob, &cd, xI, yI, zI,
                                         xIs, yIs, zIs, e0, lo_w, hi_w, integ, bitmap,
                                         trace ? trace + 9 * h : NULL);
        }
    }
    return sum;
}

#undef FN
#undef CAT
#undef CAT2
