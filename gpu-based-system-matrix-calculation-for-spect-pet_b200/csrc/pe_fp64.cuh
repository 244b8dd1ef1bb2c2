// FP64 mode of the photoelectric element (SYSMAT_MODE_FP64), included by pe.cu inside its
// anonymous namespace.
//
// The element is the reference's program (PESysMatGen.cu:951-1364) evaluated in double from
// the float parameter arrays: voxel source, crystal frames, cone test, sub-element positions,
// plate, hole, layer and crystal chords, attenuation sum, exponentials and solid angle.  The
// reference's float program loses up to ~2e-5 of an element to rounding: y + FOV rounded to
// float moves cap planes and plate faces by an ulp of ~60 mm, and T/cos(theta) - sum L cancels.
// In double those errors are ~1e-15.
//
// The culling machinery is the float kernel's: block superset, slope rectangles, round
// capsules and per-lane rectangles are geometric filters with margins far above float
// rounding, so every object they skip has a zero chord in double too.  The kept list's cone
// test, which is part of the reference's model rather than a filter, is evaluated in double.

// Per-element constants in double.
struct Elem64 {
    double xI, yI, zI;            // voxel centre
    double xIs, yIs, zIs;         // voxel in crystal d's frame
    double xd, yd, zd, w, t, h;   // crystal d
    double cr, sr;                // cos rot, sin rot
    double mu_t, mu_pe;
    double ux, uy, uz, crit_self; // cone test (:1110-1116)
};

// Element constants for the source point at fractions (fx, fy, fz) of voxel v's extent (1/2:
// the voxel centre, the reference's source).
__device__ __forceinline__ void init_elem64(const DevGeom& g, int d, long long v, float rotation, Elem64& E,
                                            double fx = 0.5, double fy = 0.5, double fz = 0.5)
{
    const long long nxy = (long long)g.nx * g.ny;
    const int iz = (int)(v / nxy);
    const long long r = v - (long long)iz * nxy;
    const int iy = (int)(r / g.nx);
    const int ix = (int)(r - (long long)iy * g.nx);
    const double ang = (double)rotation * (double)g.angle_step;   // :1006
    double sa, ca;
    sincos(ang, &sa, &ca);
    double x = ((double)ix - (double)g.nx / 2.0 + fx) * (double)g.wx;
    double y = ((double)iy - (double)g.ny / 2.0 + fy) * (double)g.wy;
    const double z = ((double)iz - (double)g.nz / 2.0 + fz) * (double)g.wz + (double)g.shz;
    x = x + (double)g.shx;
    y = y + (double)g.shy;
    E.xI = x * ca - y * sa;
    E.yI = x * sa + y * ca;
    E.zI = z;
    const D4 P = g.t64.cry_pos[d], S = g.t64.cry_size[d], T = g.t64.cry_trig[d];
    E.xd = P.x; E.yd = P.y; E.zd = P.z; E.mu_t = P.w;
    E.w = S.x; E.t = S.y; E.h = S.z; E.mu_pe = S.w;
    E.cr = T.x; E.sr = T.y;
    E.xIs = (E.xI - E.xd) * T.z - (E.zI - E.zd) * T.w;              // :1066-1068
    E.yIs = E.yI - E.yd;
    E.zIs = (E.xI - E.xd) * T.w + (E.zI - E.zd) * T.z;
    const double dist = sqrt((E.yd - E.yI) * (E.yd - E.yI) + (E.xd - E.xI) * (E.xd - E.xI) +
                             (E.zd - E.zI) * (E.zd - E.zI));
    E.crit_self = sqrt(E.w * E.w + E.h * E.h + E.t * E.t) / dist / 2.0;
    E.ux = (E.xd - E.xI) / dist;
    E.uy = (E.yd - E.yI) / dist;
    E.uz = (E.zd - E.zI) / dist;
}

// Cone test of object i (:1120-1184) in double, then the float bundle filter.
__device__ __forceinline__ bool keep_object64(const DevGeom& g, const Elem& e, const Elem64& E, int i, int d,
                                              float4& rect)
{
    rect = open_rect();
    double ox, oy, oz, crit;
    if (i < g.n_holes) {
        const D4 a = g.t64.hole_a[i], b = g.t64.hole_b[i];
        ox = a.x; oy = b.z; oz = a.w;
        crit = b.w;
    } else {
        const int o = i - g.n_holes;
        if (o == d) return false;
        const D4 P = g.t64.cry_pos[o], S = g.t64.cry_size[o];
        ox = P.x; oy = P.y; oz = P.z;
        crit = sqrt(S.x * S.x + S.z * S.z + S.y * S.y) / 2.0;
    }
    const double L = sqrt((E.xI - ox) * (E.xI - ox) + (E.yI - oy) * (E.yI - oy) + (E.zI - oz) * (E.zI - oz));
    const double vx = (ox - E.xI) / L, vy = (oy - E.yI) / L, vz = (oz - E.zI) / L;
    bool keep = sqrt((vz - E.uz) * (vz - E.uz) + (vy - E.uy) * (vy - E.uy) + (vx - E.ux) * (vx - E.ux)) <=
                crit / L + E.crit_self;
    if (keep && e.filt) {
        if (i < g.n_holes) {
            rect = hole_rect(__ldg(&g.hole.a[i]), __ldg(&g.hole.b[i].x), e.xI, e.yI, e.zI);
        } else {
            const int o = i - g.n_holes;
            rect = crystal_rect(__ldg(&g.cry.pos[o]), __ldg(&g.cry.size[o]), __ldg(&g.cry.trig[o]), e.xI, e.yI,
                                e.zI);
        }
        keep = rects_overlap(rect, e.rd);
    }
    return keep;
}

// build_chunk with the double cone test.
__device__ int build_chunk64(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws, const Elem& e, const Elem64& E,
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
            keep = keep_object64(g, e, E, id, d, rect);
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

// Sub-element (ix, iy, iz) of the 8 x 16 x 8 division in double (:1207-1221): its centre in
// crystal d's frame, in world coordinates, and the ray's length and direction cosine.
struct Sub64 {
    int ix, iy, iz;
    double xD, yD, zD, sq, cosang;
};

__device__ __forceinline__ void sub_local64(const Elem64& E, int ix, int iy, int iz, double& xDs, double& yDs,
                                            double& zDs)
{
    xDs = -E.w / 2.0 + ((double)ix + 0.5) / 8.0 * E.w;
    zDs = -E.h / 2.0 + ((double)iz + 0.5) / 8.0 * E.h;
    yDs = -E.t / 2.0 + ((double)iy + 0.5) / 16.0 * E.t;
}

__device__ __forceinline__ Sub64 sub_element64(const Elem64& E, int ix, int iy, int iz)
{
    Sub64 q;
    q.ix = ix; q.iy = iy; q.iz = iz;
    double xDs, yDs, zDs;
    sub_local64(E, ix, iy, iz, xDs, yDs, zDs);
    q.xD = E.xd + (xDs * E.cr - zDs * E.sr);
    q.zD = E.zd + (xDs * E.sr + zDs * E.cr);
    q.yD = E.yd + yDs;
    q.sq = sqrt((q.yD - E.yI) * (q.yD - E.yI) + (q.xD - E.xI) * (q.xD - E.xI) + (q.zD - E.zI) * (q.zD - E.zI));
    q.cosang = (q.yD - E.yI) / q.sq;
    return q;
}

struct Walk64 {
    double att, len;
    int lay;
};

__device__ __forceinline__ void close_layers64(const DevGeom& g, Walk64& s, int upto, double cosang)
{
    while (s.lay < upto) {                                    // :1281-1284
        const double* Ly = g.t64.layer + kLayer64 * s.lay;
        const double lcol = Ly[6] / cosang;
        if ((lcol - s.len) >= (double)0.00001f) s.att = s.att + Ly[7] * (lcol - s.len);
        s.len = 0.0;
        ++s.lay;
    }
}

// Plate penalty (:1240-1254) in double; the float "through both faces" rectangle skips rays
// whose chord is at least the plate thickness.
__device__ __forceinline__ bool plate_penalty64(const DevGeom& g, const WarpSmem& ws, const Elem64& E,
                                                const Sub64& Q, float sa_a, float sa_b, double& att)
{
    bool blocked = false;
    for (int m = 0; m < g.n_layers; ++m) {
        if (in_rect(ws.inner[m], sa_a, sa_b)) continue;
        const double* Ly = g.t64.layer + kLayer64 * m;
        const double tl = box_chord64(E.xI, E.yI, E.zI, Q.xD, Q.yD, Q.zD, Ly[0], Ly[2], Ly[4], Ly[1], Ly[3], Ly[5]);
        if (tl < (double)0.1f) { att = att + 100000.0; blocked = true; }
    }
    return blocked;
}

// Walk round-buffer entries [0, nr) (object ids: holes [0, nh), crystals [nh, nr)) for one
// ray in double.
__device__ __forceinline__ void walk_round64(const DevGeom& g, const WarpSmem& ws, int nh, int nr, const Elem64& E,
                                             const Sub64& Q, float sa_a, float sa_b, RayCyl64& rc, Walk64& s)
{
    for (int j = 0; j < nh; ++j) {
        const int m = ws.rl[j];
        if (m != s.lay) close_layers64(g, s, m, Q.cosang);
        if (!hole_in_reach(ws, j, sa_a, sa_b)) continue;
        const int id = __float_as_int(ws.ra[j].x);
        const D4 a = g.t64.hole_a[id], b = g.t64.hole_b[id];
        double tmp;
        const D4 S = g.t64.hole_shape ? g.t64.hole_shape[id] : D4{0.0, 0.0, 1.0, 0.0};
        if (S.x > 0.0)                                          // elliptical hole
            tmp = ell_chord64(E.xI, E.yI, E.zI, Q.xD, Q.yD, Q.zD, a.x, a.y, a.z, a.w, S.x, S.y, S.z, S.w);
        else
            tmp = ray_cyl64_chord(rc, E.xI, E.yI, E.zI, a.x, a.y, a.z, a.w, b.x);
        s.len = s.len + tmp;                                   // :1276-1278
        s.att = s.att + b.y * tmp;
    }
    if (nr <= nh) return;
    if (s.lay < g.n_layers) close_layers64(g, s, g.n_layers, Q.cosang);
    for (int j = nh; j < nr; ++j) {                            // :1290-1325
        if (!in_rect(ws.rr[j], sa_a, sa_b)) continue;
        const int o = __float_as_int(ws.ra[j].x) - g.n_holes;
        const D4 P = g.t64.cry_pos[o], S = g.t64.cry_size[o], T = g.t64.cry_trig[o];
        const double xa = (E.xI - P.x) * T.z - (E.zI - P.z) * T.w, ya = E.yI - P.y;
        const double za = (E.xI - P.x) * T.w + (E.zI - P.z) * T.z;
        const double xb = (Q.xD - P.x) * T.z - (Q.zD - P.z) * T.w, yb = Q.yD - P.y;
        const double zb = (Q.xD - P.x) * T.w + (Q.zD - P.z) * T.z;
        const double la = box_chord64(xa, ya, za, xb, yb, zb, -0.5 * S.x, -0.5 * S.y, -0.5 * S.z, 0.5 * S.x,
                                      0.5 * S.y, 0.5 * S.z);
        s.att = s.att + la * P.w;
    }
}

// Self attenuation, absorption and solid angle in double (:1223-1231, :1329-1357).
__device__ __forceinline__ double finish64(const Elem64& E, const Sub64& Q, double att)
{
    const double w = E.w, t = E.t, h = E.h;
    double xDs, yDs, zDs;
    sub_local64(E, Q.ix, Q.iy, Q.iz, xDs, yDs, zDs);
    const double ux1 = ((double)Q.ix / 8.0 - 0.5) * w, ux2 = (((double)Q.ix + 1.0) / 8.0 - 0.5) * w;
    const double uy1 = ((double)Q.iy / 16.0 - 0.5) * t, uy2 = (((double)Q.iy + 1.0) / 16.0 - 0.5) * t;
    const double uz1 = ((double)Q.iz / 8.0 - 0.5) * h, uz2 = (((double)Q.iz + 1.0) / 8.0 - 0.5) * h;
    const double l1 = box_chord_inside64(E.xIs, E.yIs, E.zIs, xDs, yDs, zDs, -w / 2.0, -t / 2.0, -h / 2.0,
                                         w / 2.0, t / 2.0, h / 2.0);
    const double l2 = box_chord_inside64(E.xIs, E.yIs, E.zIs, xDs, yDs, zDs, ux1, uy1, uz1, ux2, uy2, uz2);
    att = att + (l1 - l2) * E.mu_t;
    const double eff = exp(-att);
    const double xt = xDs + 1000.0 * (xDs - E.xIs) / Q.sq;
    const double yt = yDs + 1000.0 * (yDs - E.yIs) / Q.sq;
    const double zt = zDs + 1000.0 * (zDs - E.zIs) / Q.sq;
    const double labs = box_chord64(E.xIs, E.yIs, E.zIs, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
    const double absf = -expm1(-labs * E.mu_t) * E.mu_pe / E.mu_t;
    const double rq = 1.0 / ((4.0 * 3.14159265358979323846) * (Q.sq * Q.sq) * Q.sq);
    const double sax = t * h / 8.0 / 16.0 * fabs((Q.xD - E.xI) * E.cr - (Q.zD - E.zI) * E.sr) * rq;
    const double saz = w * t / 8.0 / 16.0 * fabs((Q.xD - E.xI) * E.sr + (Q.zD - E.zI) * E.cr) * rq;
    const double say = w * h / 8.0 / 8.0 * fabs(Q.yD - E.yI) * rq;
    const double sxy = (sax >= say) ? sax : say;
    const double sa = (sxy >= saz) ? sxy : saz;
    return eff * sa * absf;
}

// Element in double.  Rounds, round boxes and chunking as pe_element; the float Elem and
// SubElem drive the filters only.
__device__ double pe_element64(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws, int d, long long v, float cr,
                               float sr, float rotation, int lane)
{
    Elem e;
    if (!init_element(g, ws, d, v, cr, sr, lane, e)) return 0.0;   // mu_t <= 0.01 (:1107, :1194)
    // warp-uniform constants in the warp's shared slot (registers would spill)
    static_assert(sizeof(Elem64) <= sizeof(ws.e64), "Elem64 exceeds its shared-memory slot");
    Elem64& E = *reinterpret_cast<Elem64*>(ws.e64);
    if (lane == 0) init_elem64(g, d, v, rotation, E);
    __syncwarp();
    const bool from_super = bs.s_count >= 0;
    const int n_src = from_super ? bs.s_count : g.n_holes + g.n_det;
    int count = 0;
    const int cursor = build_chunk64(g, bs, ws, e, E, d, 0, n_src, from_super, lane, &count);
    const bool single = cursor >= n_src;
    double dacc = 0.0;
    for (int r = 0; r < 32; ++r) {
        const int sidx = ((r >> 3) * 2 + (lane >> 4)) * 128 + ((lane >> 1) & 7) * 16 + (r & 7) * 2 + (lane & 1);
        const SubElem q = sub_element(e, sidx);
        const Sub64 Q = sub_element64(E, q.ix, q.iy, q.iz);
        Walk64 s{0.0, 0.0, 0};
        RayCyl64 rc;
        ray_cyl64_init(rc, E.xI, E.yI, E.zI, Q.xD, Q.yD, Q.zD);
        const bool blocked = plate_penalty64(g, ws, E, Q, q.sa_a, q.sa_b, s.att);
        const bool skip = blocked && g.nonneg_mu;
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
            if (!single && !first_chunk) {
                cur = build_chunk64(g, bs, ws, e, E, d, cur, n_src, from_super, lane, &count);
            } else if (!single) {
                if (r > 0) cur = build_chunk64(g, bs, ws, e, E, d, 0, n_src, from_super, lane, &count);
                else cur = cursor;
            }
            first_chunk = false;
            int k = 0;
            while (k < count) {
                int next = count, nh = 0;
                const int nr = fill_round<false, true>(g, ws, e, k, count, box, 0, lane, &next, &nh);
                if (!skip) walk_round64(g, ws, nh, nr, E, Q, q.sa_a, q.sa_b, rc, s);
                __syncwarp();
                k = next;
            }
            if (single || cur >= n_src) break;
        }
        if (!skip) {
            if (s.lay < g.n_layers) close_layers64(g, s, g.n_layers, Q.cosang);
            dacc += finish64(E, Q, s.att);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dacc += __shfl_xor_sync(0xffffffffu, dacc, off);
    __syncwarp();                                    // E is rewritten by the warp's next element
    return dacc;
}
