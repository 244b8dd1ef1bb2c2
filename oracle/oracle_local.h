/* Local-coordinate FP32 form of the photoelectric element (an extension with no reference
 * counterpart), included by sysmat_oracle.c after the FP32 and FP64 instances of
 * oracle_body.h.  TEST INFRASTRUCTURE ONLY: the CPU twin of the library's
 * SYSMAT_MODE_LOCAL kernel, checked against the FP64 restatement.
 *
 * The element is the reference's (PESysMatGen.cu:951-1364): the same cone test, the same
 * chords with the same thresholds, the same solid angle.  What changes is where rounding
 * happens.  The reference's float program works in absolute coordinates: cap planes and
 * plate faces are y + FOV rounded to float (an ulp of ~60 mm), every chord is a difference
 * of ray parameters measured from the voxel (~80 mm), and the septal length T/cos - sum L
 * cancels.  Those errors are common to all rays of an element and do not average out.
 * Here:
 *   - per element, in double: the voxel centre, the vector from the voxel to crystal d's
 *     centre and its slopes, each candidate hole's offset from that central ray at the
 *     hole's entry plane, the plate boxes relative to the voxel, and each candidate crystal's
 *     centre relative to crystal d;
 *   - per ray, in float, on small numbers only: the sub-element's offset from crystal d's
 *     centre, the slope difference to the central ray (formed without cancellation), hole
 *     chords as y-extents inside the hole's circle in the hole's own frame, the septal
 *     length as (T - sum of y-extents) / cos, and crystal chords measured from the
 *     sub-element (near end of the ray) instead of from the voxel;
 *   - contributions summed with Neumaier's compensated summation.
 */

typedef struct {
    double hx, hz;    /* ray through crystal d's centre minus hole centre, at the hole's y1 */
    float dy;         /* y1 - yI */
    float th;         /* y2 - y1 */
    float r, mu;
    float ex, ez;     /* semi-axes of an elliptical hole (ex = 0: circle) */
    float ct, st;     /* cos, sin of its angle (double of the float angle, rounded once) */
} lhole;

typedef struct {
    float px, py, pz;            /* crystal d's centre minus crystal k's centre, in k's frame */
    float c, s;                  /* cos, sin of -rot_k */
    float w, t, h, mu;
} lcry;

typedef struct {
    float x1, y1, z1, x2, y2, z2;   /* plate box minus the voxel centre */
    float T, mu;
} lplate;

/* Distance from P along direction u (|u| = 1) to where the line leaves the slab
 * [lo, hi] of one axis, for both directions: *fwd along u, *bwd along -u. */
static inline void slab_exit_f(float p, float u, float lo, float hi, float* fwd, float* bwd)
{
    if (u > 0) { *fwd = (hi - p) / u; *bwd = (p - lo) / u; }
    else       { *fwd = (lo - p) / u; *bwd = (p - hi) / u; }
}

/* Reference box chord (PESysMatGen.cu:20-312) of the segment voxel -> P through the box
 * [lo, hi], evaluated from the near end: P is the segment's end point, q = P - voxel (the
 * segment vector), all in the box's frame with P close to the box.  Only full crossings
 * count, as in the reference: the box must lie strictly between the two ends. */
static float box_chord_near_f(const float P[3], const float q[3], const float lo[3], const float hi[3])
{
    const float eps = 0.001f;
    int par[3], npar = 0;
    for (int a = 0; a < 3; ++a) { par[a] = fabsf(q[a]) < eps; npar += par[a]; }
    if (npar == 3) return 0;
    if (npar == 2) {                                   /* axis-parallel ray (:33-66) */
        int m = !par[0] ? 0 : (!par[1] ? 1 : 2);
        for (int a = 0; a < 3; ++a) {
            if (a == m) continue;
            const float p0 = P[a] - q[a];
            if (!(p0 >= lo[a] && p0 <= hi[a])) return 0;
        }
        const float p0 = P[m] - q[m], p1 = P[m];
        if ((p0 <= lo[m] && p1 >= hi[m]) || (p1 <= lo[m] && p0 >= hi[m])) return fabsf(hi[m] - lo[m]);
        return 0;
    }
    float s2 = 0;
    for (int a = 0; a < 3; ++a) {
        if (par[a]) {
            const float p0 = P[a] - q[a];
            if (p0 >= hi[a] || p0 <= lo[a]) return 0;   /* :69-72 */
            continue;
        }
        s2 += q[a] * q[a];
    }
    const float tio = sqrtf(s2);
    /* the line P + s v, v = -q / tio (towards the voxel): the box occupies s in [smin, smax] */
    float smin = -INFINITY, smax = INFINITY;
    for (int a = 0; a < 3; ++a) {
        if (par[a]) continue;
        const float v = -q[a] / tio;
        float f, b;
        slab_exit_f(P[a], v, lo[a], hi[a], &f, &b);
        /* along +v the slab spans [-b, f] */
        if (-b > smin) smin = -b;
        if (f < smax) smax = f;
    }
    if (smin > smax) return 0;
    if ((smax - smin) < eps) return 0;
    /* reference parameters t = tio - s: tmax >= tio <=> smin <= 0, tmin <= eps <=> smax >= tio - eps */
    if (smin <= 0 || smax <= 0) return 0;
    if (smax >= tio - eps || smin >= tio - eps) return 0;
    return smax - smin;
}

/* Hole chord as a y-extent: the ray's offset from the hole axis at the hole's entry plane is
 * (u0, w0), its slopes are (rx, rz) per unit y (a = rx^2 + rz^2, ia = 1/a), the hole spans
 * y in [0, th] relative to that plane.  Follows the reference's cap/side cases and thresholds
 * (PESysMatGen.cu:688-799); t-parameters (length from the voxel) enter only the threshold
 * tests: ta = dy * sec, tb = (dy + th) * sec, tio = ray length.  Offsets, slopes and roots are
 * in double: near a tangent, and for a hole met far from where the ray enters the plate, the
 * chord is ill-conditioned in them. */
static float hole_extent_f(double u0d, double w0d, double rxd, double rzd, double ad, double iad, float r, float th,
                           float dy, float sec, float tio, float ky, double tq)
{
    if (fabsf(th) < 0.001f) return 0;
    const double u1d = u0d + rxd * (double)th, w1d = w0d + rzd * (double)th;
    const double r2 = (double)r * (double)r;
    const int fl = u0d * u0d + w0d * w0d <= r2;
    const int fr = u1d * u1d + w1d * w1d <= r2;
    if (fl && fr) {
        const float ta = dy * sec, tb = (dy + th) * sec;
        if ((double)ta <= 0.0001 || (double)tb <= 0.0001) return 0;
        if (ta >= tio || tb >= tio) return 0;
        return th;
    }
    const double cross = u0d * rzd - w0d * rxd;
    const double qd = ad * r2 - cross * cross;          /* b^2 - a c (Lagrange identity) */
    if ((double)(ky * ky) * tq * qd <= (double)0.00001f) return 0;   /* the reference's discriminant */
    const double bd = u0d * rxd + w0d * rzd;
    const double sq = (double)sqrtf((float)qd);
    const double s1 = (-bd - sq) * iad, s2 = (-bd + sq) * iad;
    double ea, eb;
    if (!fl && !fr) {
        if (!(s1 >= 0 && s2 <= (double)th)) return 0;
        ea = s1; eb = s2;
    } else if (fl) { ea = 0; eb = s2; }
    else           { ea = s1; eb = (double)th; }
    const float t1 = (dy + (float)ea) * sec, t2 = (dy + (float)eb) * sec;
    if ((double)t2 <= 0.0001 || (double)t1 <= 0.0001) return 0;
    if (t2 >= tio || t1 >= tio) return 0;
    if (!fl && !fr) return (float)(2.0 * sq * iad);
    return (float)(eb - ea);
}

static float pe_element_local(const ogeo* g, int d, double xI, double yI, double zI, int* cand_c, int* cand_h,
                              int* ncand_h, lhole* lh, lcry* lc, float* per_sub)
{
    const float* C = g->C;
    const double fov = (double)g->I[11];
    crystal_f64 cd;
    load_crystal_f64(g, d, &cd);
    if (!(cd.mu_t > (double)0.01f)) return 0;                 /* :1107, :1194 */

    /* ---- cone culling in double: the candidate sets of the FP64 restatement ---- */
    double dist = sqrt((cd.y - yI) * (cd.y - yI) + (cd.x - xI) * (cd.x - xI) + (cd.z - zI) * (cd.z - zI));
    double crit_self = sqrt(cd.w * cd.w + cd.h * cd.h + cd.t * cd.t) / dist / 2.0;
    double ux = (cd.x - xI) / dist, uy = (cd.y - yI) / dist, uz = (cd.z - zI) / dist;
    const double dcx = cd.x - xI, dcy = cd.y - yI, dcz = cd.z - zI;
    const double rxc = dcx / dcy, rzc = dcz / dcy;
    int nc = 0;
    for (int o = 0; o < g->ncry; ++o) {
        if (o == d) continue;
        crystal_f64 co;
        load_crystal_f64(g, o, &co);
        double crit = sqrt(co.w * co.w + co.h * co.h + co.t * co.t);
        double L = sqrt((xI - co.x) * (xI - co.x) + (yI - co.y) * (yI - co.y) + (zI - co.z) * (zI - co.z));
        crit = crit / L / 2.0;
        double vx = (co.x - xI) / L, vy = (co.y - yI) / L, vz = (co.z - zI) / L;
        if (sqrt((vz - uz) * (vz - uz) + (vy - uy) * (vy - uy) + (vx - ux) * (vx - ux)) <= crit + crit_self) {
            const double c = cos(-co.rot), s = sin(-co.rot);
            const double ex = cd.x - co.x, ey = cd.y - co.y, ez = cd.z - co.z;
            lcry* k = &lc[nc];
            k->px = (float)(ex * c - ez * s);
            k->py = (float)ey;
            k->pz = (float)(ex * s + ez * c);
            k->c = (float)c;
            k->s = (float)s;
            k->w = (float)co.w; k->t = (float)co.t; k->h = (float)co.h; k->mu = (float)co.mu_t;
            cand_c[nc++] = o;
        }
    }
    int hid = 0, hoff = 0;
    for (int m = 0; m < g->L; ++m) {
        int n = 0;
        for (int j = 0; j < g->nh[m]; ++j, ++hid) {
            double hx = (double)C[hid * 9 + 100];
            double hy1 = (double)C[hid * 9 + 101] + fov;
            double hy2 = (double)C[hid * 9 + 102] + fov;
            double hz = (double)C[hid * 9 + 103];
            double hr = (double)C[hid * 9 + 104];
            double hy = (hy1 + hy2) / 2.0;
            double crit = sqrt(hr * hr * 4 + (hy1 - hy2) * (hy1 - hy2)) / 2.0;
            double L = sqrt((xI - hx) * (xI - hx) + (yI - hy) * (yI - hy) + (zI - hz) * (zI - hz));
            crit = crit / L;
            double vx = (hx - xI) / L, vy = (hy - yI) / L, vz = (hz - zI) / L;
            if (sqrt((vz - uz) * (vz - uz) + (vy - uy) * (vy - uy) + (vx - ux) * (vx - ux)) <= crit + crit_self) {
                lhole* e = &lh[hoff + n];
                const double dy = hy1 - yI;
                e->hx = (xI - hx) + rxc * dy;
                e->hz = (zI - hz) + rzc * dy;
                e->dy = (float)dy;
                e->th = (float)(hy2 - hy1);
                e->r = (float)hr;
                e->mu = (float)C[hid * 9 + 105];
                e->ex = 0;
                e->ez = 0;
                e->ct = 1;
                e->st = 0;
                if (g->S && g->S[3 * hid] > 0.0f) {            /* elliptical hole (extension) */
                    e->ex = g->S[3 * hid];
                    e->ez = g->S[3 * hid + 1];
                    e->ct = (float)cos((double)g->S[3 * hid + 2]);
                    e->st = (float)sin((double)g->S[3 * hid + 2]);
                }
                cand_h[hoff + n++] = hid;
            }
        }
        ncand_h[m] = n;
        hoff += n;
    }
    lplate pl[MAX_LAYERS];
    for (int m = 0; m < g->L; ++m) {
        const float* Lh = C + (m + 1) * 10;
        pl[m].x1 = (float)(-(double)Lh[1] / 2.0 - xI);
        pl[m].x2 = (float)((double)Lh[1] / 2.0 - xI);
        pl[m].y1 = (float)(-(double)Lh[2] / 2.0 + fov + (double)Lh[4] - yI);
        pl[m].y2 = (float)((double)Lh[2] / 2.0 + fov + (double)Lh[4] - yI);
        pl[m].z1 = (float)(-(double)Lh[3] / 2.0 - zI);
        pl[m].z2 = (float)((double)Lh[3] / 2.0 - zI);
        pl[m].T = Lh[2];
        pl[m].mu = Lh[5];
    }

    /* ---- sub-element loop, order z, x, y (:1196-1362) ---- */
    const unsigned NXS = (unsigned)g->div[0], NYS = (unsigned)g->div[1], NZS = (unsigned)g->div[2];
    const float w = (float)cd.w, t = (float)cd.t, h = (float)cd.h;
    const float cr = (float)cos(cd.rot), sr = (float)sin(cd.rot);       /* d's frame -> world */
    const float cmr = (float)cos(-cd.rot), smr = (float)sin(-cd.rot);   /* world -> d's frame */
    const float fdx = (float)dcx, fdy = (float)dcy, fdz = (float)dcz;
    const float mu_t = (float)cd.mu_t, mu_pe = (float)cd.mu_pe;
    float sum = 0, comp = 0;
    for (unsigned iz = 0; iz < NZS; ++iz)
    for (unsigned ix = 0; ix < NXS; ++ix)
    for (unsigned iy = 0; iy < NYS; ++iy) {
        const float xDs = -w / 2.0f + ((float)ix + 0.5f) / (float)NXS * w;
        const float zDs = -h / 2.0f + ((float)iz + 0.5f) / (float)NZS * h;
        const float yDs = -t / 2.0f + ((float)iy + 0.5f) / (float)NYS * t;
        const float ox = xDs * cr - zDs * sr, oy = yDs, oz = xDs * sr + zDs * cr;   /* world offset */
        const float qx = fdx + ox, qy = fdy + oy, qz = fdz + oz;                 /* sub-element - voxel */
        const float dsq = qy * qy + qx * qx + qz * qz;
        const float sq = sqrtf(dsq);
        const float ky = qy / sq, sec = sq / qy;
        /* 1 / cos in double (septal lengths of heavily attenuated rays) */
        const double ddx = dcx + (double)ox, ddy = dcy + (double)oy, ddz = dcz + (double)oz;
        const double dsec = sqrt(ddx * ddx + ddy * ddy + ddz * ddz) / ddy;
        const double ddrx = ((double)ox * dcy - dcx * (double)oy) / (ddy * dcy);
        const double ddrz = ((double)oz * dcy - dcz * (double)oy) / (ddy * dcy);
        const double rxd = rxc + ddrx, rzd = rzc + ddrz, ad = rxd * rxd + rzd * rzd, iad = 1.0 / ad;

        /* solid angle in double, as the reference (:1223-1231) */
        const double fourpi_d2 = 4 * M_PI * (double)dsq;
        const float sax = (float)((double)(t * h / (float)NZS / (float)NYS) / fourpi_d2 *
                                  (double)fabsf(qx * cr - qz * sr) / (double)sq);
        const float saz = (float)((double)(w * t / (float)NXS / (float)NYS) / fourpi_d2 *
                                  (double)fabsf(qx * sr + qz * cr) / (double)sq);
        const float say = (float)((double)(w * h / (float)NXS / (float)NZS) / fourpi_d2 * (double)fabsf(qy) /
                                  (double)sq);
        const float sa = rmax_f32(rmax_f32(sax, say), saz);

        double att = 0;   /* in double: its float rounding alone would move exp(-att) by ~1e-5 */
        for (int m = 0; m < g->L; ++m) {                       /* plate bypass penalty :1240-1254 */
            const float tl = box_chord_f32(0, 0, 0, qx, qy, qz, pl[m].x1, pl[m].y1, pl[m].z1, pl[m].x2, pl[m].y2,
                                           pl[m].z2);
            if (tl < 0.1f) att = att + 100000.0;
        }
        hoff = 0;
        for (int m = 0; m < g->L; ++m) {                       /* holes and septa :1257-1286 */
            float ext = 0, hatt = 0;
            for (int j = 0; j < ncand_h[m]; ++j) {
                const lhole* e = &lh[hoff + j];
                double u0 = e->hx + ddrx * (double)e->dy, w0 = e->hz + ddrz * (double)e->dy;
                double rx = rxd, rz = rzd, a = ad, ia = iad, tq = 1.0;
                float rad = e->r;
                if (e->ex > 0.0f) {
                    /* elliptical: the ray's offset and slopes turned into the hole's frame and
                     * divided by the semi-axes (the unit circle); the reference's discriminant
                     * b^2 - a c is rho_x^4 rho_z^4 ky^2 times the unit circle's */
                    const double c = (double)e->ct, sn = (double)e->st;
                    const double iex = 1.0 / (double)e->ex, iez = 1.0 / (double)e->ez;
                    const double p = (u0 * c + w0 * sn) * iex, q = (-u0 * sn + w0 * c) * iez;
                    const double al = (rxd * c + rzd * sn) * iex, be = (-rxd * sn + rzd * c) * iez;
                    u0 = p; w0 = q; rx = al; rz = be;
                    a = al * al + be * be;
                    ia = 1.0 / a;
                    rad = 1.0f;
                    const double e2 = (double)e->ex * (double)e->ex * (double)e->ez * (double)e->ez;
                    tq = e2 * e2;
                }
                const float s = hole_extent_f(u0, w0, rx, rz, a, ia, rad, e->th, e->dy, sec, sq, ky, tq);
                ext = ext + s;
                hatt = hatt + e->mu * s;
            }
            hoff += ncand_h[m];
            att = att + (double)hatt * dsec;
            const double sept = (double)(pl[m].T - ext) * dsec;
            if (sept >= (double)0.00001f) att = att + (double)pl[m].mu * sept;
        }
        for (int j = 0; j < nc; ++j) {                         /* other crystals :1290-1325 */
            const lcry* k = &lc[j];
            const float P[3] = {k->px + (ox * k->c - oz * k->s), k->py + oy, k->pz + (ox * k->s + oz * k->c)};
            const float q[3] = {qx * k->c - qz * k->s, qy, qx * k->s + qz * k->c};
            const float lo[3] = {-0.5f * k->w, -0.5f * k->t, -0.5f * k->h};
            const float hi[3] = {0.5f * k->w, 0.5f * k->t, 0.5f * k->h};
            att = att + (double)(box_chord_near_f(P, q, lo, hi) * k->mu);
        }
        /* self attenuation and absorption in crystal d's frame, from the sub-element centre */
        const float vq[3] = {qx * cmr - qz * smr, qy, qx * smr + qz * cmr};    /* ray vector in d's frame */
        const float D3[3] = {xDs, yDs, zDs};
        const float ub_lo[3] = {((float)ix / (float)NXS - 0.5f) * w, ((float)iy / (float)NYS - 0.5f) * t,
                                ((float)iz / (float)NZS - 0.5f) * h};
        const float ub_hi[3] = {(((float)ix + 1.0f) / (float)NXS - 0.5f) * w,
                                (((float)iy + 1.0f) / (float)NYS - 0.5f) * t,
                                (((float)iz + 1.0f) / (float)NZS - 0.5f) * h};
        const float cb_lo[3] = {-w / 2.0f, -t / 2.0f, -h / 2.0f}, cb_hi[3] = {w / 2.0f, t / 2.0f, h / 2.0f};
        float l1 = 0, l2 = 0, labs = 0;
        if (!((double)fabsf(vq[1]) < 0.001)) {                 /* box_chord_inside :321-324 */
            /* backward exits from the sub-element centre: crystal entry and sub-element entry */
            float b1 = INFINITY, b2 = INFINITY;
            int ok1 = 1, ok2 = 1;
            for (int a = 0; a < 3; ++a) {
                if (fabsf(vq[a]) < 0.001f) {
                    /* axis parallel to the ray: the voxel's coordinate must lie in the slab */
                    const float p0 = D3[a] - vq[a];
                    if (p0 >= cb_hi[a] || p0 <= cb_lo[a]) ok1 = 0;
                    if (p0 >= ub_hi[a] || p0 <= ub_lo[a]) ok2 = 0;
                    continue;
                }
                const float v = vq[a] / sq;
                float f, b;
                slab_exit_f(D3[a], v, cb_lo[a], cb_hi[a], &f, &b);
                if (b < b1) b1 = b;
                slab_exit_f(D3[a], v, ub_lo[a], ub_hi[a], &f, &b);
                if (b < b2) b2 = b;
            }
            if (ok1) l1 = b1;
            if (ok2) l2 = b2;
        }
        {
            /* absorption: chord of the extended ray (voxel -> 1000 mm past the sub-element)
             * through the sub-element box, a full crossing (:1352-1357) */
            const float ext = 1.0f + 1000.0f / sq;
            float fwd = INFINITY, bwd = INFINITY;
            int ok = 1, npar = 0, m = 0;
            for (int a = 0; a < 3; ++a) npar += fabsf(vq[a] * ext) < 0.001f;
            for (int a = 0; a < 3; ++a) {
                if (fabsf(vq[a] * ext) < 0.001f) {
                    const float p0 = D3[a] - vq[a];
                    if (npar == 1 ? (p0 >= ub_hi[a] || p0 <= ub_lo[a]) : !(p0 >= ub_lo[a] && p0 <= ub_hi[a])) ok = 0;
                    continue;
                }
                m = a;
                const float v = vq[a] / sq;
                float f, b;
                slab_exit_f(D3[a], v, ub_lo[a], ub_hi[a], &f, &b);
                if (f < fwd) fwd = f;
                if (b < bwd) bwd = b;
            }
            if (npar == 3) ok = 0;
            if (ok && npar == 2) labs = fabsf(ub_hi[m] - ub_lo[m]);
            else if (ok) labs = fwd + bwd;
            if (labs < 0.001f) labs = 0;
        }
        att = att + (double)((l1 - l2) * mu_t);
        const float a_hi = (float)att, a_lo = (float)(att - (double)a_hi);
        const float eff = expf(-a_hi) * (1.0f - a_lo);
        const float absf = -expm1f(-labs * mu_t) * mu_pe / mu_t;
        const float term = eff * sa * absf;
        if (per_sub) per_sub[(iz * NXS + ix) * NYS + iy] = term;
        /* Neumaier compensated sum */
        const float tsum = sum + term;
        if (fabsf(sum) >= fabsf(term)) comp += (sum - tsum) + term;
        else comp += (term - tsum) + sum;
        sum = tsum;
    }
    return sum + comp;
}
