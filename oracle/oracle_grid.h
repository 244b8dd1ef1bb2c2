/* Grid scatter model (an extension with no reference counterpart), FP64, included by
 * sysmat_oracle.c after the FP64 instance of oracle_body.h.  TEST INFRASTRUCTURE ONLY: the
 * definition the library's sysmat_scatter_grid is checked against.
 *
 * The reference scatters at one point per crystal (its centre, weighted by the crystal's
 * photoelectric element, ScatterGen_RayTracing_CircularHole/scatter.cu:1218-1223) and one
 * point per layer-0 hole (its centre, weighted by a virtual-hole solid angle, :1707-1716).
 * This model puts scatter points on a grid of cells of side `cell` (0.25 mm) inside every
 * crystal and inside the tungsten of every collimator layer:
 *
 *   S[d, v] = sum over crystals k != d, cells p of k:   w_p T(p, d, v)
 *           + sum over layers m, septal cells p of m:  w_p T(p, d, v)
 *
 *   crystal cell p (crystal k divided into ceil(w/cell) x ceil(t/cell) x ceil(h/cell) parts):
 *     w_p = the reference's photoelectric contribution of that sub-element from voxel v
 *           (PESysMatGen.cu:1196-1357 with this division) * mu_C,k / mu_pe,k;
 *   septal cell p (the layer's plate box divided into cells, centre outside every hole):
 *     w_p = V_cell / (4 pi r^2) * exp(-A(v -> p)) * mu_C,m, r = |p - v|, A the attenuation at
 *           the photopeak along v -> p through the layers' tungsten (plate chord minus the
 *           reference's hole chords) and the holes' own media;
 *   T(p, d, v) = the reference's item (scatter.cu:1232-1427) with scatter point p: cone angle,
 *     Compton energy, 2-sigma window reject and window probability, azimuth range, polar range
 *     over crystal d's corners, absorption in d, attenuation at the scattered energy by every
 *     crystal other than d that the segment p -> d's centre crosses (all crystals, no
 *     relationship bitmap; for a crystal cell, its own crystal from p to the exit) and, for
 *     septal points, by the tungsten and hole media on the way (exact segment lengths: the
 *     paths start or end inside the plate, where the reference's full-crossing chords do not
 *     apply);
 *     the Klein-Nishina fraction is the exact integral of the reference's Klein-Nishina shape
 *     over [theta_min, theta_max] divided by its integral over [0, pi] (closed form), in place
 *     of the reference's 0.01 rad Riemann sum.
 * Every element sums about 10^6 cells, in double.
 */

/* Antiderivative in x = cos(theta) of the reference's Klein-Nishina shape (scatter.cu:961-978)
 * f(x) = (1+x^2)/(1+a(1-x))^2 + a^2(1-x)^2/(1+a(1-x))^3, a = E/511: with u = 1 + a(1-x),
 * F = -(u - 2b ln u - (a^2+b^2)/u)/a^3 - (ln u + 2/u - 1/(2u^2))/a, b = 1 + a. */
static double kn_prim(double x, double a)
{
    const double b = 1.0 + a, u = 1.0 + a * (1.0 - x);
    return -(u - 2.0 * b * log(u) - (a * a + b * b) / u) / (a * a * a) - (log(u) + 2.0 / u - 0.5 / (u * u)) / a;
}

/* Fraction of the Klein-Nishina shape between polar angles tmin and tmax. */
static double kn_frac(double tmin, double tmax, double a)
{
    return (kn_prim(cos(tmin), a) - kn_prim(cos(tmax), a)) / (kn_prim(1.0, a) - kn_prim(-1.0, a));
}

/* Length of segment A -> B inside the box [lo, hi] (exact overlap of the segment's parameter
 * range with the three slabs).  The grid model's paths start or end inside the plate, where
 * the reference's box and cylinder chords (full crossings between the two ends) do not
 * apply. */
static double seg_box(const double A[3], const double B[3], const double lo[3], const double hi[3])
{
    double t0 = 0, t1 = 1;
    for (int a = 0; a < 3; ++a) {
        const double d = B[a] - A[a];
        if (d == 0) {
            if (A[a] < lo[a] || A[a] > hi[a]) return 0;
            continue;
        }
        double u = (lo[a] - A[a]) / d, v = (hi[a] - A[a]) / d;
        if (u > v) { const double w = u; u = v; v = w; }
        if (u > t0) t0 = u;
        if (v < t1) t1 = v;
    }
    if (t1 <= t0) return 0;
    const double len = sqrt((B[0] - A[0]) * (B[0] - A[0]) + (B[1] - A[1]) * (B[1] - A[1]) + (B[2] - A[2]) * (B[2] - A[2]));
    return (t1 - t0) * len;
}

/* Elliptical hole j (g->S, an extension): semi-axes and cos, sin of its angle in double. */
static int grid_ellipse(const ogeo* g, int j, double* ex, double* ez, double* c, double* s)
{
    if (!g->S || !(g->S[3 * j] > 0.0f)) return 0;
    *ex = (double)g->S[3 * j];
    *ez = (double)g->S[3 * j + 1];
    *c = cos((double)g->S[3 * j + 2]);
    *s = sin((double)g->S[3 * j + 2]);
    return 1;
}

/* Length of segment A -> B inside the y-parallel cylinder (x - xc)^2 + (z - zc)^2 <= r^2,
 * y in [y1, y2] (exact overlap); with ell, inside the elliptical cylinder of semi-axes ex, ez
 * in the hole's frame turned by (c, s) (u = dx c + dz s, w = -dx s + dz c, as the reference
 * turns points): the segment's offsets mapped to that frame and divided by the semi-axes meet
 * the unit circle over the same parameter range. */
static double seg_cyl_shape(const double A[3], const double B[3], double xc, double zc, double y1, double y2,
                            double r, int ell, double ex, double ez, double c, double s)
{
    double t0 = 0, t1 = 1;
    const double dy = B[1] - A[1];
    if (dy == 0) {
        if (A[1] < y1 || A[1] > y2) return 0;
    } else {
        double u = (y1 - A[1]) / dy, v = (y2 - A[1]) / dy;
        if (u > v) { const double w = u; u = v; v = w; }
        if (u > t0) t0 = u;
        if (v < t1) t1 = v;
    }
    const double dx0 = B[0] - A[0], dz0 = B[2] - A[2];
    double dx = dx0, dz = dz0, ox = A[0] - xc, oz = A[2] - zc;
    if (ell) {
        const double pdx = (dx * c + dz * s) / ex, pdz = (-dx * s + dz * c) / ez;
        const double pox = (ox * c + oz * s) / ex, poz = (-ox * s + oz * c) / ez;
        dx = pdx; dz = pdz; ox = pox; oz = poz; r = 1.0;
    }
    const double a = dx * dx + dz * dz, b = ox * dx + oz * dz, cc = ox * ox + oz * oz - r * r;
    if (a == 0) {
        if (cc > 0) return 0;
    } else {
        const double disc = b * b - a * cc;
        if (disc <= 0) return 0;
        const double sq = sqrt(disc);
        const double u = (-b - sq) / a, v = (-b + sq) / a;
        if (u > t0) t0 = u;
        if (v < t1) t1 = v;
    }
    if (t1 <= t0) return 0;
    return (t1 - t0) * sqrt(dx0 * dx0 + dz0 * dz0 + dy * dy);
}

static double seg_cyl(const double A[3], const double B[3], double xc, double zc, double y1, double y2, double r)
{
    return seg_cyl_shape(A, B, xc, zc, y1, y2, r, 0, 1, 1, 1, 0);
}

static void grid_plate_box(const ogeo* g, int m, double b[6])
{
    const float* Lh = g->C + (m + 1) * 10;
    const double fov = (double)g->I[11];
    b[0] = -(double)Lh[1] / 2.0; b[3] = (double)Lh[1] / 2.0;
    b[1] = -(double)Lh[2] / 2.0 + fov + (double)Lh[4]; b[4] = (double)Lh[2] / 2.0 + fov + (double)Lh[4];
    b[2] = -(double)Lh[3] / 2.0; b[5] = (double)Lh[3] / 2.0;
}

/* Attenuation sums (mu_total, mu_pe, mu_C times length) of layer m along the segment A -> B:
 * the segment's length in the plate box minus its lengths in the layer's holes, times the
 * layer's coefficients, plus its lengths in the holes times the holes' coefficients (exact
 * overlaps: A or B may lie inside the plate). */
static void grid_layer_path(const ogeo* g, int m, int hole_begin, const double A[3], const double B[3],
                            double* wt, double* wpe, double* wc)
{
    const float* C = g->C;
    const double fov = (double)g->I[11];
    double b[6];
    grid_plate_box(g, m, b);
    const double lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
    const double box = seg_box(A, B, lo, hi);
    if (box == 0) return;
    double hsum = 0;
    const double ex = B[0] - A[0], ez = B[2] - A[2], l2 = ex * ex + ez * ez;
    for (int j = hole_begin; j < hole_begin + g->nh[m]; ++j) {
        const float* h = C + 100 + 9 * j;
        /* a hole whose axis stays farther than its radius from the segment's xz projection has
         * a zero length: skipped without evaluating it */
        double t = l2 > 0 ? (((double)h[0] - A[0]) * ex + ((double)h[3] - A[2]) * ez) / l2 : 0;
        t = t < 0 ? 0 : (t > 1 ? 1 : t);
        const double dx = A[0] + t * ex - (double)h[0], dz = A[2] + t * ez - (double)h[3];
        if (dx * dx + dz * dz > ((double)h[4] + 1e-6) * ((double)h[4] + 1e-6)) continue;
        double ex = 1, ez = 1, c = 1, s = 0;
        const int ell = grid_ellipse(g, j, &ex, &ez, &c, &s);
        const double l = seg_cyl_shape(A, B, (double)h[0], (double)h[3], (double)h[1] + fov, (double)h[2] + fov,
                                       (double)h[4], ell, ex, ez, c, s);
        if (l == 0) continue;
        hsum += l;
        *wt += (double)h[5] * l;
        *wpe += (double)h[6] * l;
        *wc += (double)h[7] * l;
    }
    const double lw = box - hsum;
    if (lw > 0) {
        const float* Lh = C + (m + 1) * 10;
        *wt += (double)Lh[5] * lw;
        *wpe += (double)Lh[6] * lw;
        *wc += (double)Lh[7] * lw;
    }
}

/* T(p, d, v) times the weight w (see the file comment).  skip_k: the scatterer crystal (crystal
 * cells; the scattered photon's path through the rest of it is attenuated too) or -1; layer_p:
 * the layer holding a septal point, or -1. */
static double grid_item(const ogeo* g, int d, const crystal_f64* cd, const double I3[3], const double Is[3],
                        const double p[3], double w, int skip_k, int layer_p, double e0, double lo_w, double hi_w)
{
    const double xDs = 0.0 * cd->w, yDs = 0.0 * cd->t, zDs = 0.0 * cd->h;   /* 1 x 1 x 1 division: centre */
    const double D3[3] = {cd->x + (xDs * cos(cd->rot) - zDs * sin(cd->rot)), cd->y + yDs,
                          cd->z + (xDs * sin(cd->rot) + zDs * cos(cd->rot))};
    const double cone = cone_angle_f64(I3[0], I3[1], I3[2], p[0], p[1], p[2], D3[0], D3[1], D3[2]);
    const double es = e0 / (1.0 + (e0 / 511.0) * (1.0 - cos(cone)));
    const double res = cd->eres * sqrt(es / e0);
    if ((es * (1 + 2 * res / (double)2.35482f)) <= lo_w || (es * (1 - 2 * res / (double)2.35482f)) >= hi_w)
        return 0;                                                   /* :1263 */
    const double pwin = window_prob_f64(es, res, lo_w, hi_w);
    const double lsd = dist3_f64(p[0], p[1], p[2], D3[0], D3[1], D3[2]);
    const double rdet = sqrt(cd->w * cd->w + cd->h * cd->h + cd->t * cd->t) / 2.0;
    const double phi = (lsd * sin(cone) * 2.0 <= rdet) ? 2.0 * M_PI
                                                        : 4.0 * asin(rmin_f64(rdet / 2.0 / lsd / sin(cone), 1.0));
    double ps[3];
    to_frame_f64(cd, p[0], p[1], p[2], &ps[0], &ps[1], &ps[2]);
    const double ux1 = -0.5 * cd->w, ux2 = 0.5 * cd->w, uy1 = -0.5 * cd->t, uy2 = 0.5 * cd->t;
    const double uz1 = -0.5 * cd->h, uz2 = 0.5 * cd->h;
    const double dis = dist3_f64(ps[0], ps[1], ps[2], Is[0], Is[1], Is[2]);
    double xt = ps[0] + 1000.0 * (ps[0] - Is[0]) / dis, yt = ps[1] + 1000.0 * (ps[1] - Is[1]) / dis;
    double zt = ps[2] + 1000.0 * (ps[2] - Is[2]) / dis;
    const double lthr = box_chord_f64(Is[0], Is[1], Is[2], xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
    double tmin = 10, tmax = -10;
    for (int c = 0; c < 8; ++c) {
        const double th = cone_angle_f64(Is[0], Is[1], Is[2], ps[0], ps[1], ps[2], (c & 1) ? ux2 : ux1,
                                         (c & 2) ? uy2 : uy1, (c & 4) ? uz2 : uz1);
        if (th < tmin) tmin = th;
        if (th > tmax) tmax = th;
    }
    if (lthr > (double)0.001f) tmin = 0;
    const double ratio = kn_frac(tmin, tmax, e0 / 511.0);
    const double sc_pe = e0 * e0 * e0 / es / es / es, sc_c = e0 / es;
    double att = 0;
    const double gx = D3[0] - p[0], gy = D3[1] - p[1], gz = D3[2] - p[2], gl2 = gx * gx + gy * gy + gz * gz;
    for (int a = 0; a < g->ncry; ++a) {                             /* crystals on the way */
        if (a == d || a == skip_k) continue;
        crystal_f64 ca;
        load_crystal_f64(g, a, &ca);
        /* a crystal whose bounding sphere misses the segment has a zero chord: skipped */
        const double hx = ca.x - p[0], hy = ca.y - p[1], hz = ca.z - p[2];
        double t = (hx * gx + hy * gy + hz * gz) / gl2;
        t = t < 0 ? 0 : (t > 1 ? 1 : t);
        const double qx = hx - t * gx, qy = hy - t * gy, qz = hz - t * gz;
        const double ra = sqrt(ca.w * ca.w + ca.t * ca.t + ca.h * ca.h) / 2.0 + 1e-6;
        if (qx * qx + qy * qy + qz * qz > ra * ra) continue;
        double xa, ya, za, xb, yb, zb;
        to_frame_f64(&ca, p[0], p[1], p[2], &xa, &ya, &za);
        to_frame_f64(&ca, D3[0], D3[1], D3[2], &xb, &yb, &zb);
        const double la = box_chord_f64(xa, ya, za, xb, yb, zb, -0.5 * ca.w, -0.5 * ca.t, -0.5 * ca.h, 0.5 * ca.w,
                                        0.5 * ca.t, 0.5 * ca.h);
        if (la != 0) att += la * (ca.mu_pe * sc_pe + ca.mu_c * sc_c);
    }
    if (skip_k >= 0) {                    /* the rest of the scattering crystal, from p to its exit */
        crystal_f64 ck;
        load_crystal_f64(g, skip_k, &ck);
        double pa[3], pb[3];
        to_frame_f64(&ck, p[0], p[1], p[2], &pa[0], &pa[1], &pa[2]);
        to_frame_f64(&ck, D3[0], D3[1], D3[2], &pb[0], &pb[1], &pb[2]);
        const double lo[3] = {-0.5 * ck.w, -0.5 * ck.t, -0.5 * ck.h}, hi[3] = {0.5 * ck.w, 0.5 * ck.t, 0.5 * ck.h};
        att += seg_box(pa, pb, lo, hi) * (ck.mu_pe * sc_pe + ck.mu_c * sc_c);
    }
    if (layer_p >= 0) {                                             /* tungsten and holes on the way */
        int hb = 0;
        for (int m = 0; m < g->L; ++m) {
            double wt = 0, wpe = 0, wc = 0;
            grid_layer_path(g, m, hb, p, D3, &wt, &wpe, &wc);
            att += wpe * sc_pe + wc * sc_c;
            hb += g->nh[m];
        }
    }
    const double mpe_s = cd->mu_pe * sc_pe, mt_s = mpe_s + cd->mu_c * sc_c;
    xt = xDs + 1000.0 * (xDs - ps[0]) / lsd;
    yt = yDs + 1000.0 * (yDs - ps[1]) / lsd;
    zt = zDs + 1000.0 * (zDs - ps[2]) / lsd;
    const double labs = box_chord_f64(ps[0], ps[1], ps[2], xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
    return (w * phi / 2.0) / M_PI * ratio * pwin * exp(-att) * (-expm1(-labs * mt_s)) * mpe_s / mt_s;
}

/* Septal weight of cell centre p of layer m (hole_begin: its first hole) from voxel I3. */
static double grid_septal_weight(const ogeo* g, int m, int hole_begin, const double I3[3], const double p[3],
                                 double vcell)
{
    double at = 0, ape = 0, ac = 0;
    int hb = 0;
    for (int mm = 0; mm < g->L; ++mm) {
        grid_layer_path(g, mm, hb, I3, p, &at, &ape, &ac);
        hb += g->nh[mm];
    }
    const double r2 = (p[0] - I3[0]) * (p[0] - I3[0]) + (p[1] - I3[1]) * (p[1] - I3[1]) + (p[2] - I3[2]) * (p[2] - I3[2]);
    (void)hole_begin;
    return vcell / (4.0 * M_PI * r2) * exp(-at) * (double)g->C[(m + 1) * 10 + 7];
}

static int grid_div(double size, double cell)
{
    int n = (int)ceil(size / cell - 1e-9);
    return n < 1 ? 1 : n;
}

/* Cells of layer m: count along x, y, z and the cell centre of (ix, iy, iz). */
static void grid_layer_cells(const ogeo* g, int m, double cell, int n[3], double b[6])
{
    grid_plate_box(g, m, b);
    n[0] = grid_div(b[3] - b[0], cell);
    n[1] = grid_div(b[4] - b[1], cell);
    n[2] = grid_div(b[5] - b[2], cell);
}

static int grid_in_hole(const ogeo* g, int hole_begin, int m, const double p[3])
{
    const float* C = g->C;
    const double fov = (double)g->I[11];
    for (int j = hole_begin; j < hole_begin + g->nh[m]; ++j) {
        const float* h = C + 100 + 9 * j;
        const double dx = p[0] - (double)h[0], dz = p[2] - (double)h[3], r = (double)h[4];
        if (!(p[1] >= (double)h[1] + fov && p[1] <= (double)h[2] + fov)) continue;
        double ex, ez, c, s;
        if (grid_ellipse(g, j, &ex, &ez, &c, &s)) {
            const double u = (dx * c + dz * s) / ex, w = (-dx * s + dz * c) / ez;
            if (u * u + w * w <= 1.0) return 1;
        } else if (dx * dx + dz * dz <= r * r) {
            return 1;
        }
    }
    return 0;
}

/* One element of the grid model (the parts selected by `parts`: 1 crystal cells, 2 septal
 * cells), summed in double with the work spread over threads. */
static double grid_element(const ogeo* g0, int parts, int d, long long v, double cell, int nthreads)
{
    const float* P = g0->P;
    if ((int)floor((double)(P[0] + 0.5f)) != 1) return 0;
    crystal_f64 cd;
    load_crystal_f64(g0, d, &cd);
    if (!(cd.mu_t > (double)0.01f)) return 0;
    const double e0 = (double)P[7];
    double lo_w, hi_w;
    if ((int)floor((double)(P[4] + 0.5f)) > 0) { lo_w = (double)P[5]; hi_w = (double)P[6]; }
    else { lo_w = (1 - cd.eres / 2.0) * e0; hi_w = (1 + cd.eres / 2.0) * e0; }
    double I3[3], Is[3];
    voxel_centre_f64(g0, v, &I3[0], &I3[1], &I3[2]);
    to_frame_f64(&cd, I3[0], I3[1], I3[2], &Is[0], &Is[1], &Is[2]);
    double total = 0;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    if (parts & 1) {
#pragma omp parallel reduction(+ : total)
        {
            ogeo g = *g0;
            g.vsub[0] = g.vsub[1] = g.vsub[2] = 1;
            int* cc = (int*)malloc(sizeof(int) * (size_t)(g.ncry + 1));
            int* ch = (int*)malloc(sizeof(int) * (size_t)(g.nholes + 1));
            int nch[MAX_LAYERS];
            double* sub = NULL;
            size_t sub_cap = 0;
#pragma omp for schedule(dynamic, 1)
            for (int k = 0; k < g.ncry; ++k) {
                if (k == d) continue;
                crystal_f64 ck;
                load_crystal_f64(&g, k, &ck);
                if (!(ck.mu_t > (double)0.01f)) continue;
                g.div[0] = grid_div(ck.w, cell);
                g.div[1] = grid_div(ck.t, cell);
                g.div[2] = grid_div(ck.h, cell);
                const size_t ns = (size_t)g.div[0] * g.div[1] * g.div[2];
                if (ns > sub_cap) { free(sub); sub = (double*)malloc(sizeof(double) * ns); sub_cap = ns; }
                pe_element_at_f64(&g, k, I3[0], I3[1], I3[2], cc, ch, nch, NULL, sub);
                const double conv = ck.mu_c / ck.mu_pe;
                const double cr = cos(ck.rot), sr = sin(ck.rot);
                for (int iz = 0; iz < g.div[2]; ++iz)
                for (int ix = 0; ix < g.div[0]; ++ix)
                for (int iy = 0; iy < g.div[1]; ++iy) {
                    const double ws = sub[((size_t)iz * g.div[0] + ix) * g.div[1] + iy];
                    if (ws == 0) continue;
                    const double xDs = -ck.w / 2.0 + ((double)ix + 0.5) / (double)g.div[0] * ck.w;
                    const double zDs = -ck.h / 2.0 + ((double)iz + 0.5) / (double)g.div[2] * ck.h;
                    const double yDs = -ck.t / 2.0 + ((double)iy + 0.5) / (double)g.div[1] * ck.t;
                    const double p[3] = {ck.x + (xDs * cr - zDs * sr), ck.y + yDs, ck.z + (xDs * sr + zDs * cr)};
                    total += grid_item(&g, d, &cd, I3, Is, p, ws * conv, k, -1, e0, lo_w, hi_w);
                }
            }
            free(sub);
            free(cc);
            free(ch);
        }
    }
    if (parts & 2) {
        int hb = 0;
        for (int m = 0; m < g0->L; ++m) {
            int n[3];
            double b[6];
            grid_layer_cells(g0, m, cell, n, b);
            const double cx = (b[3] - b[0]) / n[0], cy = (b[4] - b[1]) / n[1], cz = (b[5] - b[2]) / n[2];
            const double vcell = cx * cy * cz;
            double lt = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : lt)
            for (int iz = 0; iz < n[2]; ++iz)
            for (int iy = 0; iy < n[1]; ++iy)
            for (int ix = 0; ix < n[0]; ++ix) {
                const double p[3] = {b[0] + (ix + 0.5) * cx, b[1] + (iy + 0.5) * cy, b[2] + (iz + 0.5) * cz};
                if (grid_in_hole(g0, hb, m, p)) continue;
                const double w = grid_septal_weight(g0, m, hb, I3, p, vcell);
                if (w == 0) continue;
                lt += grid_item(g0, d, &cd, I3, Is, p, w, -1, m, e0, lo_w, hi_w);
            }
            total += lt;
            hb += g0->nh[m];
        }
    }
    return total;
}
