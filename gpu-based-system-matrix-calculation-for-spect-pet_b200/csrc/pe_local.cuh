// Local-coordinate FP32 mode of the photoelectric element (SYSMAT_MODE_LOCAL), included by
// pe.cu inside its anonymous namespace.  No reference counterpart: it evaluates the
// reference's element (PESysMatGen.cu:951-1364; same cone test, chords, thresholds and solid
// angle) in float arithmetic that stays within 1e-5 of the FP64 restatement.
//
// The reference's float program loses up to ~2e-5 of an element because it works in absolute
// coordinates: cap planes and plate faces are y + FOV rounded to float (an ulp of ~60 mm),
// chords are differences of ray parameters measured from the voxel (~80 mm), and the septal
// length T/cos - sum L cancels.  These errors are shared by all rays of an element, so they do
// not average out.  Here every quantity that is large or shared is formed once per element in
// double and only small differences are rounded to float:
//   - per element (lane 0, in the warp's shared slot): the voxel centre, crystal d's centre
//     and the slopes of the central ray voxel -> centre, the plate boxes relative to the
//     voxel; per kept object and round (fill_round_local): a hole's offset from the central
//     ray at its entry plane, its depth below the voxel and its length; a crystal's centre
//     relative to crystal d's, in its own frame;
//   - per ray, in float: the sub-element's offset from crystal d's centre, the slope
//     difference to the central ray (formed without cancellation), hole chords as y-extents
//     inside the hole's circle (or ellipse) in the hole's frame, the septal length (T - sum of extents) /
//     cos, crystal chords measured from the sub-element, self-attenuation and absorption
//     chords from the sub-element centre in crystal d's frame;
//   - the 1024 contributions are summed with Neumaier's compensated summation, per lane and
//     across the warp.
// The culling (superset, slope rectangles, capsules) is the float kernel's; its margins are far
// above float rounding, and the kept list's cone test is the double one of the FP64 mode.

struct ElemL {
    Elem64 e64;                  // double constants of the cone test (init_elem64)
    double rxc, rzc;             // slopes dx/dy, dz/dy of the ray voxel -> crystal d's centre
    double idyc;                 // 1 / dy of that ray
    float fdx, fdy, fdz;         // crystal d's centre minus the voxel
    float frxc, frzc;
    float cr, sr, cmr, smr;      // cos, sin of rot_d and of -rot_d
    float w, t, h, mu_t, mu_pe;
    float plate[kMaxLayers][6];  // plate boxes minus the voxel: x1, y1, z1, x2, y2, z2
    int nx, ny, nz;              // sub-elements along x, depth (y), z (the reference: 8, 16, 8)
    float rfx, rfy, rfz;         // 1/nx, 1/ny, 1/nz
};

__device__ __forceinline__ void init_elem_local(const DevGeom& g, int d, long long v, float rotation, int nx, int ny,
                                                int nz, ElemL& L, double fx = 0.5, double fy = 0.5, double fz = 0.5)
{
    init_elem64(g, d, v, rotation, L.e64, fx, fy, fz);
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.rfx = 1.0f / (float)nx;
    L.rfy = 1.0f / (float)ny;
    L.rfz = 1.0f / (float)nz;
    const Elem64& E = L.e64;
    const double dx = E.xd - E.xI, dy = E.yd - E.yI, dz = E.zd - E.zI;
    L.idyc = 1.0 / dy;
    L.rxc = dx * L.idyc;
    L.rzc = dz * L.idyc;
    L.fdx = (float)dx;
    L.fdy = (float)dy;
    L.fdz = (float)dz;
    L.frxc = (float)L.rxc;
    L.frzc = (float)L.rzc;
    const D4 T = g.t64.cry_trig[d];
    L.cr = (float)T.x;
    L.sr = (float)T.y;
    L.cmr = (float)T.z;
    L.smr = (float)T.w;
    const float4 S = __ldg(&g.cry.size[d]);
    const float4 M = __ldg(&g.cry.mu[d]);
    L.w = S.x; L.t = S.y; L.h = S.z;
    L.mu_t = M.x; L.mu_pe = M.y;
    for (int m = 0; m < g.n_layers; ++m) {
        const double* Ly = g.t64.layer + kLayer64 * m;
        L.plate[m][0] = (float)(Ly[0] - E.xI);
        L.plate[m][1] = (float)(Ly[2] - E.yI);
        L.plate[m][2] = (float)(Ly[4] - E.zI);
        L.plate[m][3] = (float)(Ly[1] - E.xI);
        L.plate[m][4] = (float)(Ly[3] - E.yI);
        L.plate[m][5] = (float)(Ly[5] - E.zI);
    }
}

// Distances from p along u (|u| = 1) to where the line leaves the slab [lo, hi]: fwd along
// u, bwd along -u; iu = 1 / u.  This form's error budget (1e-5 of FP64 per element) allows a
// reciprocal multiply where the reference's exact program divides.
__device__ __forceinline__ void slab_exit(float p, float iu, float lo, float hi, float& fwd, float& bwd)
{
    if (iu > 0.0f) { fwd = (hi - p) * iu; bwd = (p - lo) * iu; }
    else           { fwd = (lo - p) * iu; bwd = (p - hi) * iu; }
}

// The reference box chord (PESysMatGen.cu:20-312) of the segment voxel -> P through the box
// [lo, hi], evaluated from the near end P (q = P - voxel, in the box's frame): only full
// crossings strictly between the two ends count.
__device__ __forceinline__ float box_chord_near(const float P[3], const float q[3], const float lo[3],
                                                const float hi[3])
{
    bool par[3];
    int npar = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        par[a] = fabsf(q[a]) < kEps;
        npar += par[a];
    }
    if (npar == 3) return 0.0f;
    if (npar == 2) {                                             // axis-parallel ray (:33-66)
        const int m = !par[0] ? 0 : (!par[1] ? 1 : 2);
        for (int a = 0; a < 3; ++a) {
            if (a == m) continue;
            const float p0 = P[a] - q[a];
            if (!(p0 >= lo[a] && p0 <= hi[a])) return 0.0f;
        }
        const float p0 = P[m] - q[m], p1 = P[m];
        if ((p0 <= lo[m] && p1 >= hi[m]) || (p1 <= lo[m] && p0 >= hi[m])) return fabsf(hi[m] - lo[m]);
        return 0.0f;
    }
    float s2 = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (par[a]) {
            const float p0 = P[a] - q[a];
            if (p0 >= hi[a] || p0 <= lo[a]) return 0.0f;          // :69-72
        } else {
            s2 += q[a] * q[a];
        }
    }
    const float tio = sqrtf(s2);
    float smin = -INFINITY, smax = INFINITY;                      // along P + s * (-q / tio)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (par[a]) continue;
        float f, b;
        slab_exit(P[a], __fdividef(-tio, q[a]), lo[a], hi[a], f, b);
        smin = fmaxf(smin, -b);
        smax = fminf(smax, f);
    }
    if (!(smin <= smax)) return 0.0f;
    if ((smax - smin) < kEps) return 0.0f;
    // the reference's parameters from the voxel are t = tio - s
    if (smin <= 0.0f || smax >= tio - kEps) return 0.0f;
    return smax - smin;
}

// Hole chord as a y-extent (see the file comment): the ray's offset from the hole axis at the
// hole's entry plane is (u0, w0), its slopes are (rx, rz) per unit y (a = rx^2 + rz^2, ia =
// 1/a), the hole spans [0, th] in y from that plane, dy below the voxel.  Cap/side cases and
// thresholds follow the reference (PESysMatGen.cu:688-799); the t parameters (length from the
// voxel: ta = dy * sec, ...) enter only its threshold tests.  Offsets, slopes and the roots are
// in double: near a tangent, and for a hole met far from where the ray enters the plate, the
// chord is ill-conditioned in them, and float offsets or slopes would move it by ~1e-5 mm.
// tq scales the reference's discriminant threshold (1 for a circle; an ellipse passes its
// offsets and slopes divided by its semi-axes with r = 1, and tq = rho_x^4 rho_z^4).
__device__ __forceinline__ float hole_extent(double u0d, double w0d, double rxd, double rzd, double ad, double iad,
                                             float r, float th, float dy, float sec, float tio, float ky,
                                             double tq = 1.0)
{
    if (fabsf(th) < kEps) return 0.0f;
    const double u1d = u0d + rxd * (double)th, w1d = w0d + rzd * (double)th;
    const double r2 = (double)r * (double)r;
    const bool fl = u0d * u0d + w0d * w0d <= r2;
    const bool fr = u1d * u1d + w1d * w1d <= r2;
    if (fl && fr) {
        const float ta = dy * sec, tb = (dy + th) * sec;
        if (ta <= 0.0001f || tb <= 0.0001f) return 0.0f;
        if (ta >= tio || tb >= tio) return 0.0f;
        return th;
    }
    const double cross = u0d * rzd - w0d * rxd;
    const double qd = ad * r2 - cross * cross;                 // b^2 - a c (Lagrange identity)
    if ((double)(ky * ky) * tq * qd <= (double)0.00001f) return 0.0f;   // the reference's discriminant
    const double bd = u0d * rxd + w0d * rzd;
    const double sq = (double)sqrtf((float)qd);
    const double s1 = (-bd - sq) * iad, s2 = (-bd + sq) * iad;
    double ea, eb;
    if (!fl && !fr) {
        if (!(s1 >= 0.0 && s2 <= (double)th)) return 0.0f;
        ea = s1; eb = s2;
    } else if (fl) { ea = 0.0; eb = s2; }
    else           { ea = s1; eb = (double)th; }
    const float t1 = (dy + (float)ea) * sec, t2 = (dy + (float)eb) * sec;
    if (t2 <= 0.0001f || t1 <= 0.0001f) return 0.0f;
    if (t2 >= tio || t1 >= tio) return 0.0f;
    if (!fl && !fr) return (float)(2.0 * sq * iad);
    return (float)(eb - ea);
}

// Elliptical hole (length_ellipticalcylinder_ray, PESysMatGen.cu:801-947, the y-parallel
// cylinder ((u'/rho_x)^2 + (w'/rho_z)^2 <= 1 in the hole's frame turned by theta): the ray's
// offset (u, w) and slopes (rx, rz) turned into that frame (u' = u cos + w sin,
// w' = -u sin + w cos, as the reference turns the segment's points) and divided by the
// semi-axes reduce it to the unit circle, whose y-extent hole_extent gives with the
// discriminant threshold rescaled: the reference's b^2 - a c equals rho_x^4 rho_z^4 ky^2 times
// the unit circle's.  Rewrites the arguments of hole_extent in place.
__device__ __forceinline__ void to_unit_circle(double& u, double& w, double& rx, double& rz, double& a, double& ia,
                                               float& r, double& tq, float ex, float ez, float ct, float st)
{
    const double c = (double)ct, s = (double)st, iex = 1.0 / (double)ex, iez = 1.0 / (double)ez;
    const double p = (u * c + w * s) * iex, q = (-u * s + w * c) * iez;
    const double al = (rx * c + rz * s) * iex, be = (-rx * s + rz * c) * iez;
    u = p;
    w = q;
    rx = al;
    rz = be;
    a = al * al + be * be;
    ia = 1.0 / a;
    r = 1.0f;
    const double e2 = (double)ex * (double)ex * (double)ez * (double)ez;
    tq = e2 * e2;
}

// Copy kept entries [k0, k1) whose rectangle and capsule meet the round's slope box into the
// round buffer with their local geometry (one entry per lane):
//   hole:    ra = (semi-axes rho_x, rho_z of an elliptical hole, 0 for a circle; radius; mu),
//            rb = (y1 - yI, y2 - y1, offset of the central ray from the axis at y1: x as the two
//            halves of a double), rc = (z the same way; cos, sin of the ellipse's angle)
//   crystal: ra = (crystal d's centre minus this crystal's centre in its frame: x, y, z; mu),
//            rb = (cos(-rot), sin(-rot), w, t), rc = (h, -, -, -)
// Returns the new count; *next receives the first entry not examined.
template <bool ELL>
__device__ __forceinline__ int fill_round_local(const DevGeom& g, WarpSmem& ws, const Elem& e, const ElemL& L,
                                                int k0, int k1, float4 box, int n, int lane, int* next, int* nh)
{
    int k = k0;
    while (k < k1 && n <= kRound - 32) {
        const int kk = k + lane;
        bool keep = false;
        int id = 0;
        float4 rect;
        if (kk < k1) {
            rect = ws.rect[kk];
            keep = rects_overlap(rect, box);
            if (keep && !isinf(rect.x)) {
                id = ws.id[kk];
                if (id < g.n_holes) {
                    const float4 ha = __ldg(&g.hole.a[id]);
                    keep = capsule_meets_box(ha.x, ha.w, ha.y, ha.z, __ldg(&g.hole.b[id].x), e, box);
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
            ws.rr[pos] = rect;
            const Elem64& E = L.e64;
            if (id < g.n_holes) {
                const D4 a = g.t64.hole_a[id];
                const float4 hb = __ldg(&g.hole.b[id]);
                const double dy = a.y - E.yI;
                const double hx = (E.xI - a.x) + L.rxc * dy, hz = (E.zI - a.w) + L.rzc * dy;
                // elliptical: semi-axes and the cos, sin of the float angle in double, rounded once
                const D4 S = (ELL && g.t64.hole_shape) ? g.t64.hole_shape[id] : D4{0.0, 0.0, 1.0, 0.0};
                ws.ra[pos] = make_float4((float)S.x, (float)S.y, hb.x, hb.y);
                // the offsets in double, as the bit patterns of two floats each
                ws.rb[pos] = make_float4((float)dy, (float)(a.z - a.y), __int_as_float(__double2hiint(hx)),
                                         __int_as_float(__double2loint(hx)));
                ws.rc[pos] = make_float4(__int_as_float(__double2hiint(hz)), __int_as_float(__double2loint(hz)),
                                         (float)S.z, (float)S.w);
                ws.rl[pos] = layer_of_hole(g, id);
            } else {
                const int o = id - g.n_holes;
                const D4 P = g.t64.cry_pos[o], T = g.t64.cry_trig[o];
                const double ex = E.xd - P.x, ey = E.yd - P.y, ez = E.zd - P.z;
                const float4 so = __ldg(&g.cry.size[o]);
                ws.ra[pos] = make_float4((float)(ex * T.z - ez * T.w), (float)ey, (float)(ex * T.w + ez * T.z),
                                         __ldg(&g.cry.mu[o].x));
                ws.rb[pos] = make_float4((float)T.z, (float)T.w, so.x, so.y);
                ws.rc[pos] = make_float4(so.z, 0.0f, 0.0f, 0.0f);
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

// One ray of the local form: the sub-element's offset from crystal d's centre and the ray
// terms derived from it.
struct RayL {
    float ox, oy, oz;            // sub-element centre minus crystal d's centre (world axes)
    float qx, qy, qz;            // sub-element centre minus the voxel
    float sq, sec, ky;           // ray length, 1 / cos, cos
    float drx, drz, rx, rz;      // slope difference to the central ray, slopes
    double dsec;                 // 1 / cos in double (septal lengths: heavily attenuated rays)
    double ddrx, ddrz;           // slope difference to the central ray, in double
    double drx_, drz_, da, dia;  // slopes in double, a = rx^2 + rz^2 and 1/a
};

__device__ __forceinline__ RayL ray_local(const ElemL& L, float xDs, float yDs, float zDs)
{
    RayL r;
    r.ox = xDs * L.cr - zDs * L.sr;
    r.oy = yDs;
    r.oz = xDs * L.sr + zDs * L.cr;
    r.qx = L.fdx + r.ox;
    r.qy = L.fdy + r.oy;
    r.qz = L.fdz + r.oz;
    r.sq = sqrtf(r.qy * r.qy + r.qx * r.qx + r.qz * r.qz);
    r.ky = __fdividef(r.qy, r.sq);
    r.sec = __fdividef(r.sq, r.qy);
    const float den = __fdividef(1.0f, r.qy * L.fdy);
    r.drx = (r.ox * L.fdy - L.fdx * r.oy) * den;
    r.drz = (r.oz * L.fdy - L.fdz * r.oy) * den;
    r.rx = L.frxc + r.drx;
    r.rz = L.frzc + r.drz;
    const Elem64& E = L.e64;
    const double cx = E.xd - E.xI, cy = E.yd - E.yI, cz = E.zd - E.zI;   // voxel -> crystal d's centre
    const double dx = cx + (double)r.ox, dy = cy + (double)r.oy, dz = cz + (double)r.oz;
    const double idy = 1.0 / dy;
    r.dsec = sqrt(dx * dx + dy * dy + dz * dz) * idy;
    const double f = idy * L.idyc;
    r.ddrx = ((double)r.ox * cy - cx * (double)r.oy) * f;
    r.ddrz = ((double)r.oz * cy - cz * (double)r.oy) * f;
    r.drx_ = L.rxc + r.ddrx;
    r.drz_ = L.rzc + r.ddrz;
    r.da = r.drx_ * r.drx_ + r.drz_ * r.drz_;
    r.dia = 1.0 / r.da;
    return r;
}

// The attenuation sum is kept in double: its float rounding (an ulp of ~50 for the rays that
// cross the most tungsten) would alone move exp(-att) by ~1e-5.
struct WalkL {
    double att;     // accumulated mu * L
    float ext;      // hole y-extents of the current layer
    float hatt;     // mu-weighted hole y-extents of the current layer
    int lay;
};

__device__ __forceinline__ void close_layers_local(const DevGeom& g, WalkL& s, int upto, double sec)
{
    while (s.lay < upto) {                                           // :1276-1284
        const LayerInfo& Ly = g.layer[s.lay];
        s.att = s.att + (double)s.hatt * sec;
        const double sept = (double)(Ly.thickness - s.ext) * sec;
        if (sept >= (double)0.00001f) s.att = s.att + (double)Ly.mu_total * sept;
        s.ext = 0.0f;
        s.hatt = 0.0f;
        ++s.lay;
    }
}

template <bool ELL>
__device__ __forceinline__ void walk_round_local(const DevGeom& g, const WarpSmem& ws, int nh, int nr, const RayL& r,
                                                 float sa_a, float sa_b, WalkL& s)
{
    for (int j = 0; j < nh; ++j) {
        const int m = ws.rl[j];
        if (m != s.lay) close_layers_local(g, s, m, r.dsec);
        if (!in_rect(ws.rr[j], sa_a, sa_b)) continue;
        const float4 A = ws.ra[j];
        const float4 B = ws.rb[j];
        const float4 Cc = ws.rc[j];
        const double hx = __hiloint2double(__float_as_int(B.z), __float_as_int(B.w));
        const double hz = __hiloint2double(__float_as_int(Cc.x), __float_as_int(Cc.y));
        double u0 = hx + r.ddrx * (double)B.x, w0 = hz + r.ddrz * (double)B.x;
        double rx = r.drx_, rz = r.drz_, a = r.da, ia = r.dia, tq = 1.0;
        float rad = A.z;
        if (ELL && A.x > 0.0f) to_unit_circle(u0, w0, rx, rz, a, ia, rad, tq, A.x, A.y, Cc.z, Cc.w);   // elliptical
        const float ext = hole_extent(u0, w0, rx, rz, a, ia, rad, B.y, B.x, r.sec, r.sq, r.ky, tq);
        s.ext = s.ext + ext;
        s.hatt = s.hatt + A.w * ext;
    }
    if (nr <= nh) return;
    if (s.lay < g.n_layers) close_layers_local(g, s, g.n_layers, r.dsec);
    for (int j = nh; j < nr; ++j) {                                  // :1290-1325
        if (!in_rect(ws.rr[j], sa_a, sa_b)) continue;
        const float4 A = ws.ra[j];
        const float4 B = ws.rb[j];
        const float hh = ws.rc[j].x;
        const float P[3] = {A.x + (r.ox * B.x - r.oz * B.y), A.y + r.oy, A.z + (r.ox * B.y + r.oz * B.x)};
        const float q[3] = {r.qx * B.x - r.qz * B.y, r.qy, r.qx * B.y + r.qz * B.x};
        const float lo[3] = {-0.5f * B.z, -0.5f * B.w, -0.5f * hh};
        const float hi[3] = {0.5f * B.z, 0.5f * B.w, 0.5f * hh};
        s.att = s.att + (double)(box_chord_near(P, q, lo, hi) * A.w);
    }
}

// Self attenuation, absorption and solid angle of sub-element (ix, iy, iz) of the L.nx x L.ny
// x L.nz division, from its centre (xDs, yDs, zDs) in crystal d's frame (:1223-1231,
// :1329-1357).
__device__ __forceinline__ float finish_local(const ElemL& L, const RayL& r, int ix, int iy, int iz, float xDs,
                                              float yDs, float zDs, double att)
{
    const float w = L.w, t = L.t, h = L.h;
    const float gx = L.rfx, gy = L.rfy, gz = L.rfz;
    const float vq[3] = {r.qx * L.cmr - r.qz * L.smr, r.qy, r.qx * L.smr + r.qz * L.cmr};   // ray in d's frame
    const float D3[3] = {xDs, yDs, zDs};
    const float ulo[3] = {((float)ix * gx - 0.5f) * w, ((float)iy * gy - 0.5f) * t, ((float)iz * gz - 0.5f) * h};
    const float uhi[3] = {(((float)ix + 1.0f) * gx - 0.5f) * w, (((float)iy + 1.0f) * gy - 0.5f) * t,
                          (((float)iz + 1.0f) * gz - 0.5f) * h};
    const float clo[3] = {-w / 2.0f, -t / 2.0f, -h / 2.0f}, chi[3] = {w / 2.0f, t / 2.0f, h / 2.0f};

    // crystal entry and sub-element entry, as distances back from the sub-element centre
    // (box_chord_inside, :321-324 and its parallel-axis cases); absorption: the full chord of
    // the extended ray through the sub-element (box_chord to 1000 mm past it, :1352-1357)
    float l1 = 0.0f, l2 = 0.0f;
    float b1 = INFINITY, b2 = INFINITY, f2 = INFINITY, fa = INFINITY, ba = INFINITY;
    const bool y_ok = fabsf(vq[1]) >= 0.001f;
    bool ok1 = y_ok, ok2 = y_ok, ok_abs = true;
    const float ext = 1.0f + __fdividef(1000.0f, r.sq);
    int npar_abs = 0, m_abs = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) npar_abs += fabsf(vq[a] * ext) < kEps;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float p0 = D3[a] - vq[a];                 // the voxel's coordinate
        const bool par_in = fabsf(vq[a]) < kEps;
        const bool par_abs = fabsf(vq[a] * ext) < kEps;
        const float iv = __fdividef(r.sq, vq[a]);      // 1 / (direction cosine along a)
        float f, b;
        if (par_in) {
            if (p0 >= chi[a] || p0 <= clo[a]) ok1 = false;
            if (p0 >= uhi[a] || p0 <= ulo[a]) ok2 = false;
        } else {
            slab_exit(D3[a], iv, clo[a], chi[a], f, b);
            b1 = fminf(b1, b);
            slab_exit(D3[a], iv, ulo[a], uhi[a], f, b);
            b2 = fminf(b2, b);
            f2 = fminf(f2, f);
        }
        if (par_abs) {
            if (npar_abs == 1 ? (p0 >= uhi[a] || p0 <= ulo[a]) : !(p0 >= ulo[a] && p0 <= uhi[a])) ok_abs = false;
        } else {
            m_abs = a;
            if (par_in) slab_exit(D3[a], iv, ulo[a], uhi[a], f, b);
            else { f = f2; b = b2; }
            fa = fminf(fa, f);
            ba = fminf(ba, b);
        }
    }
    if (ok1) l1 = b1;
    if (ok2) l2 = b2;
    float labs = 0.0f;
    if (ok_abs && npar_abs < 3) labs = (npar_abs == 2) ? fabsf(uhi[m_abs] - ulo[m_abs]) : fa + ba;
    if (labs < kEps) labs = 0.0f;
    att = att + (double)((l1 - l2) * L.mu_t);
    // exp(-att) = exp(-hi) exp(-lo), hi = att rounded to float: keeps expf's relative accuracy
    const float a_hi = (float)att, a_lo = (float)(att - (double)a_hi);
    const float eff = expf(-a_hi) * (1.0f - a_lo);
    const float absf = -expm1f(-labs * L.mu_t) * L.mu_pe / L.mu_t;
    // solid angle in double, as the reference's 4*M_PI promotion makes it
    const double dsq = (double)(r.qy * r.qy + r.qx * r.qx + r.qz * r.qz);
    const double rq = 1.0 / ((4.0 * 3.14159265358979323846) * dsq * (double)r.sq);
    const float ax = t * h * gz * gy, az = w * t * gx * gy, ay = w * h * gx * gz;
    const float sax = (float)((double)ax * (double)fabsf(r.qx * L.cr - r.qz * L.sr) * rq);
    const float saz = (float)((double)az * (double)fabsf(r.qx * L.sr + r.qz * L.cr) * rq);
    const float say = (float)((double)ay * (double)fabsf(r.qy) * rq);
    const float sxy = (sax >= say) ? sax : say;
    const float sa = (sxy >= saz) ? sxy : saz;
    return eff * sa * absf;
}

// Neumaier compensated accumulation of x into (s, c).
__device__ __forceinline__ void neumaier_add(float& s, float& c, float x)
{
    const float t = s + x;
    if (fabsf(s) >= fabsf(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

// The element of the local form.  smp: the crystal division and the voxel's source points (the
// element is the mean over the centres of an sx x sy x sz grid over the voxel, as in the
// sampled form); nullptr = the reference's 8 x 16 x 8 division and the voxel centre.  The
// reference division's rounds are the compact 2 z x 8 x x 2 depth patches of the
// reference-order kernel; other divisions go 32 to a round in (z, depth, x) order, x fastest.
// sub_out (one source point only): each sub-element's contribution is also written there, at
// index (iz * ny + iy) * nx + ix (the scatter grid's crystal-cell weights).
template <bool ELL, bool SMP>
__device__ double pe_element_local(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws, int d, long long v, float cr,
                                   float sr, float rotation, int lane, const Sampling* smp = nullptr,
                                   float* sub_out = nullptr)
{
    static_assert(sizeof(ElemL) <= sizeof(ws.chain), "ElemL exceeds its shared-memory slot");
    ElemL& L = *reinterpret_cast<ElemL*>(ws.chain);
    if constexpr (!SMP) smp = nullptr;               // the reference's sampling: constants below
    const int nx = SMP ? smp->nx : 8, ny = SMP ? smp->ny : 16, nz = SMP ? smp->nz : 8;
    const int n_sub = nx * ny * nz, nxy = nx * ny;
    const int sxn = SMP ? smp->sx : 1, syn = SMP ? smp->sy : 1, szn = SMP ? smp->sz : 1;
    const int n_pts = sxn * syn * szn;
    float sum = 0.0f, comp = 0.0f;
    for (int src = 0; src < n_pts; ++src) {
        // source point at fractions ((j + 0.5) / n) of the voxel along x, y, z
        const int jx = src % sxn, jy = (src / sxn) % syn, jz = src / (sxn * syn);
        const double fxd = ((double)jx + 0.5) / (double)sxn, fyd = ((double)jy + 0.5) / (double)syn;
        const double fzd = ((double)jz + 0.5) / (double)szn;
        __syncwarp();                                    // the previous point's ElemL and plate rectangles are done
        Elem e;
        if (!init_element(g, ws, d, v, cr, sr, lane, e, (float)fxd, (float)fyd, (float)fzd)) {   // mu_t <= 0.01
            if (sub_out) {                                                                     // (:1107, :1194)
                for (int i = lane; i < n_sub; i += 32) sub_out[i] = 0.0f;
            }
            return 0.0;
        }
        if (lane == 0) init_elem_local(g, d, v, rotation, nx, ny, nz, L, fxd, fyd, fzd);
        __syncwarp();
        const bool from_super = bs.s_count >= 0;
        const int n_src = from_super ? bs.s_count : g.n_holes + g.n_det;
        int count = 0;
        const int cursor = build_chunk64(g, bs, ws, e, L.e64, d, 0, n_src, from_super, lane, &count);
        const bool single = cursor >= n_src;
        const float gx = L.rfx, gy = L.rfy, gz = L.rfz;
        for (int base = 0; base < n_sub; base += 32) {
            const bool dead = base + lane >= n_sub;
            int sidx, ix, iy, iz;
            if constexpr (!SMP) {             // s = 128 iz + 16 ix + iy, as in pe_element's rounds
                const int rr = base >> 5;
                const int s = ((rr >> 3) * 2 + (lane >> 4)) * 128 + ((lane >> 1) & 7) * 16 + (rr & 7) * 2 + (lane & 1);
                iz = s >> 7;
                ix = (s >> 4) & 7;
                iy = s & 15;
                sidx = (iz * ny + iy) * nx + ix;
            } else {
                sidx = dead ? n_sub - 1 : base + lane;
                iz = sidx / nxy;
                const int rem = sidx - iz * nxy;
                iy = rem / nx;
                ix = rem - iy * nx;
            }
            const float xDs = -L.w / 2.0f + ((float)ix + 0.5f) * gx * L.w;       // :1207-1217
            const float zDs = -L.h / 2.0f + ((float)iz + 0.5f) * gz * L.h;
            const float yDs = -L.t / 2.0f + ((float)iy + 0.5f) * gy * L.t;
            const RayL r = ray_local(L, xDs, yDs, zDs);
            const float sa_a = e.filt ? r.rx : 0.0f, sa_b = e.filt ? r.rz : 0.0f;
            WalkL s{0.0, 0.0f, 0.0f, 0};
            bool blocked = false;
            for (int m = 0; m < g.n_layers; ++m) {                             // plate penalty :1240-1254
                if (in_rect(ws.inner[m], sa_a, sa_b)) continue;
                const float* pb = L.plate[m];
                const float tl = box_chord(0.0f, 0.0f, 0.0f, r.qx, r.qy, r.qz, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5]);
                if (tl < 0.1f) { s.att = s.att + 100000.0; blocked = true; }
            }
            const bool skip = dead || (blocked && g.nonneg_mu);
            float4 box = make_float4(skip ? INFINITY : sa_a, skip ? -INFINITY : sa_a, skip ? INFINITY : sa_b,
                                     skip ? -INFINITY : sa_b);
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
                if (!single && !first_chunk) {
                    cur = build_chunk64(g, bs, ws, e, L.e64, d, cur, n_src, from_super, lane, &count);
                } else if (!single) {
                    if (base > 0) cur = build_chunk64(g, bs, ws, e, L.e64, d, 0, n_src, from_super, lane, &count);
                    else cur = cursor;
                }
                first_chunk = false;
                int k = 0;
                while (k < count) {
                    int next = count, nh = 0;
                    const int nr = fill_round_local<ELL>(g, ws, e, L, k, count, box, 0, lane, &next, &nh);
                    if (!skip) walk_round_local<ELL>(g, ws, nh, nr, r, sa_a, sa_b, s);
                    __syncwarp();
                    k = next;
                }
                if (single || cur >= n_src) break;
            }
            float term = 0.0f;
            if (!skip) {
                if (s.lay < g.n_layers) close_layers_local(g, s, g.n_layers, r.dsec);
                term = finish_local(L, r, ix, iy, iz, xDs, yDs, zDs, s.att);
                neumaier_add(sum, comp, term);
            }
            if (sub_out && !dead) sub_out[sidx] = term;
        }
    }
    // warp sum of the (sum, compensation) pairs, compensated as well
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float os = __shfl_xor_sync(0xffffffffu, sum, off);
        const float oc = __shfl_xor_sync(0xffffffffu, comp, off);
        neumaier_add(sum, comp, os);
        comp += oc;
    }
    __syncwarp();                                    // L is rewritten by the warp's next element
    return ((double)sum + (double)comp) / (double)n_pts;
}
