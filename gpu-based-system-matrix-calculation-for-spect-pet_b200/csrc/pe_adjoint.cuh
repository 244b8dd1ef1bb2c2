// Forward projection p = A(theta) x and its vector-Jacobian product, computed brick by brick
// without storing A.  Included by pe.cu inside its anonymous namespace (it uses the element
// set-up, candidate lists and round buffers of the photoelectric kernel).
//
// theta = (mu_W, mu_crystal, hole radius, collimator offset dx, dy, dz, tilt):
//   mu_W        attenuation of every collimator layer (Params_Collimator[(m+1)*10+5]);
//   mu_crystal  total attenuation of every crystal (Params_Detector[12d+7]; mu_pe fixed);
//   radius      radius of every hole (Params_Collimator[100+9h+4]);
//   dx, dz      shift of every hole centre; dy shift of the hole caps and layer planes;
//   tilt        rotation of the hole pattern about the y axis (x' = x cos - z sin,
//               z' = x sin + z cos), the one collimator rotation that keeps holes
//               parallel to y as the reference's cylinder chord requires; it turns an
//               elliptical hole's frame with it (theta_h + tilt).
// Elliptical holes (PESysMatGen.cu:801-947, sysmat_set_hole_shapes) contribute the partials
// of their chord with respect to the centre, the caps and the frame angle; their chord does
// not read the radius field (it only bounds the ellipse for the cone test), so the radius
// partial has no elliptical term.
// The derivative of A[d,v] = sum_s Omega_s exp(-att_s) absf_s follows the reference's float
// program branch by branch (PESysMatGen.cu:1240-1357): each non-zero hole chord contributes
// its analytic partials, the layer term mu_L (T/cos - sum L) its own, crystal chords and the
// self-attenuation term their lengths.  Thresholds (plate penalty, eps cut-offs, the 1e-5
// layer-term gate) are piecewise constant and contribute nothing.

constexpr int kThetaN = 7;

// Partials of the chord of ray_cyl_chord (same case analysis) with respect to the hole radius
// r, the centre (xc, zc) and a common shift dy of both cap planes.  Zero for a zero chord.
struct CylGrad {
    float dr, dx, dz, dy;
};

__device__ __forceinline__ float ray_cyl_chord_grad(const RayCyl& c, float xc, float zc, float r, CylGrad& gr)
{
    gr = CylGrad{0.0f, 0.0f, 0.0f, 0.0f};
    const float L = ray_cyl_chord(c, xc, zc, r);
    if (L == 0.0f) return L;
    const bool fl = (c.xl - xc) * (c.xl - xc) + (c.zl - zc) * (c.zl - zc) <= r * r;
    const bool fr = (c.xr - xc) * (c.xr - xc) + (c.zr - zc) * (c.zr - zc) <= r * r;
    if (fl && fr) return L;                     // |tb - ta|: cap to cap, shift invariant
    const float ox = c.xi - xc, oz = c.zi - zc;
    const float C = c.kx * oz - c.kz * ox;     // cross term; disc = kk r^2 - C^2
    const float sq = sqrtf(c.kk * r * r - C * C);
    const float isq = 1.0f / sq, ikk = 1.0f / c.kk;
    // side crossings t1,2 = (-(kx ox + kz oz) -+ sq) / kk
    const float dsq_r = c.kk * r * isq, dsq_x = -C * c.kz * isq, dsq_z = C * c.kx * isq;
    const float dt2_r = dsq_r * ikk, dt2_x = (c.kx + dsq_x) * ikk, dt2_z = (c.kz + dsq_z) * ikk;
    const float dt1_r = -dsq_r * ikk, dt1_x = (c.kx - dsq_x) * ikk, dt1_z = (c.kz - dsq_z) * ikk;
    if (!fl && !fr) {                           // side to side
        gr = CylGrad{dt2_r - dt1_r, dt2_x - dt1_x, dt2_z - dt1_z, 0.0f};
    } else if (fl) {                            // cap y1 to side: t2 - ta
        gr = CylGrad{dt2_r, dt2_x, dt2_z, -1.0f / c.ky};
    } else {                                    // side to cap y2: tb - t1
        gr = CylGrad{-dt1_r, -dt1_x, -dt1_z, 1.0f / c.ky};
    }
    return L;
}

// Partials of the elliptical-cylinder chord (ell_chord, same case analysis) with respect to the
// centre (xc, zc), a common shift dy of both cap planes and the frame angle theta (carried in
// CylGrad.dr).  In the hole's frame the ray is p(t) = (u0 + kx t, y_in + ky t, w0 + kz t) and
// the side crossings solve a t^2 + 2 b t + c = 0 with a = kx^2 rz^2 + kz^2 rx^2,
// b = kx u0 rz^2 + kz w0 rx^2, c = rz^2 u0^2 + rx^2 w0^2 - rx^2 rz^2; the centre moves
// (u0, w0) and the angle turns (u0, w0) and (kx, kz) together.
__device__ __forceinline__ float ell_chord_grad(float xi, float yi, float zi, float xo, float yo, float zo,
                                                float xc, float y1, float y2, float zc, float rx, float rz,
                                                float ct, float st, CylGrad& gr)
{
    gr = CylGrad{0.0f, 0.0f, 0.0f, 0.0f};
    const float L = ell_chord(xi, yi, zi, xo, yo, zo, xc, y1, y2, zc, rx, rz, ct, st);
    if (L == 0.0f) return L;
    // the frame quantities of ell_chord, with its expressions (same case flags)
    const float xi_ = xi - xc, zi_ = zi - zc, xo_ = xo - xc, zo_ = zo - zc;
    const float xin = xc + xi_ * ct + zi_ * st, zin = zc - xi_ * st + zi_ * ct;
    const float xout = xc + xo_ * ct + zo_ * st, zout = zc - xo_ * st + zo_ * ct;
    const float tio = sqrtf((xout - xin) * (xout - xin) + (yo - yi) * (yo - yi) + (zout - zin) * (zout - zin));
    const float kx = (xout - xin) / tio, ky = (yo - yi) / tio, kz = (zout - zin) / tio;
    const float xl = xin + kx / ky * (y1 - yi), xr = xin + kx / ky * (y2 - yi);
    const float zl = zin + kz / ky * (y1 - yi), zr = zin + kz / ky * (y2 - yi);
    const bool fl = ((xl - xc) * (xl - xc) / rx / rx + (zl - zc) * (zl - zc) / rz / rz) <= 1.0f;
    const bool fr = ((xr - xc) * (xr - xc) / rx / rx + (zr - zc) * (zr - zc) / rz / rz) <= 1.0f;
    if (fl && fr) return L;                     // |tb - ta|: cap to cap, shift and turn invariant
    const float u0 = xin - xc, w0 = zin - zc;
    const float rx2 = rx * rx, rz2 = rz * rz;
    const float a = kx * kx * rz2 + kz * kz * rx2;
    const float b = kx * u0 * rz2 + kz * w0 * rx2;
    const float c = rz2 * u0 * u0 + rx2 * w0 * w0 - rx2 * rz2;
    const float sq = sqrtf(b * b - a * c);
    const float ia = 1.0f / a, isq = 0.5f / sq;
    const float t1 = (-b - sq) * ia, t2 = (-b + sq) * ia;
    // d(t1), d(t2) for a parameter moving (u0, w0, kx, kz) by (du, dw, dkx, dkz)
    auto dts = [&](float du, float dw, float dkx, float dkz, float& d1, float& d2) {
        const float da = 2.0f * (kx * dkx * rz2 + kz * dkz * rx2);
        const float db = (dkx * u0 + kx * du) * rz2 + (dkz * w0 + kz * dw) * rx2;
        const float dc = 2.0f * (rz2 * u0 * du + rx2 * w0 * dw);
        const float dsq = (2.0f * b * db - da * c - a * dc) * isq;
        d1 = (-db - dsq - t1 * da) * ia;
        d2 = (-db + dsq - t2 * da) * ia;
    };
    float x1, x2, z1, z2, p1, p2;
    dts(-ct, st, 0.0f, 0.0f, x1, x2);           // xc: u0 = (x - xc) ct + ..., w0 = -(x - xc) st + ...
    dts(-st, -ct, 0.0f, 0.0f, z1, z2);          // zc
    dts(w0, -u0, kz, -kx, p1, p2);              // frame angle
    if (!fl && !fr) {                           // side to side
        gr = CylGrad{p2 - p1, x2 - x1, z2 - z1, 0.0f};
    } else if (fl) {                            // cap y1 to side: t2 - ta
        gr = CylGrad{p2, x2, z2, -1.0f / ky};
    } else {                                    // side to cap y2: tb - t1
        gr = CylGrad{-p1, -x1, -z1, 1.0f / ky};
    }
    return L;
}

// Walk state with the partials of att (index: theta order) and the current layer's sums of
// hole-chord partials (radius, x, z, y, tilt).
struct WalkGrad {
    float att, len;
    int lay;
    float da[kThetaN];
    float lr, lx, lz, ly, lp;
};

__device__ __forceinline__ void close_layers_grad(const DevGeom& g, WalkGrad& s, int upto, float cosang)
{
    while (s.lay < upto) {                                    // :1281-1284
        const float mu = g.layer[s.lay].mu_total;
        const float lcol = g.layer[s.lay].thickness / cosang;
        if ((lcol - s.len) >= 0.00001f) {
            s.att = s.att + mu * (lcol - s.len);
            s.da[0] += lcol - s.len;
            s.da[2] -= mu * s.lr;
            s.da[3] -= mu * s.lx;
            s.da[4] -= mu * s.ly;
            s.da[5] -= mu * s.lz;
            s.da[6] -= mu * s.lp;
        }
        s.len = 0.0f;
        s.lr = s.lx = s.lz = s.ly = s.lp = 0.0f;
        ++s.lay;
    }
}

template <bool ELL>
__device__ __forceinline__ void walk_round_grad(const DevGeom& g, const WarpSmem& ws, int nh, int nr, float xD,
                                                float yD, float zD, float sa_a, float sa_b, float cosang,
                                                RayCyl& rc, WalkGrad& s)
{
    for (int j = 0; j < nh; ++j) {
        const int m = ws.rl[j];
        if (m != s.lay) close_layers_grad(g, s, m, cosang);
        if (!in_rect(ws.rr[j], sa_a, sa_b)) continue;
        const float4 A = ws.ra[j];               // x, z, R, mu of the hole
        const float4 B = ws.rb[j];
        CylGrad gr;
        float tmp, dr = 0.0f, dth = 0.0f;        // radius and frame-angle partials
        bool ell = false;
        if constexpr (ELL) {
            const float4 S = ws.rc[j];
            if (S.x > 0.0f) {                    // elliptical hole: gr.dr holds the angle partial
                tmp = ell_chord_grad(rc.xi, rc.yi, rc.zi, xD, yD, zD, A.x, B.x, B.y, A.y, S.x, S.y, S.z, S.w, gr);
                dth = gr.dr;
                ell = true;
            }
        }
        if (!ell) {
            ray_cyl_caps(rc, B.x, B.y);
            tmp = ray_cyl_chord_grad(rc, A.x, A.y, A.z, gr);
            dr = gr.dr;
        }
        s.len = s.len + tmp;                                     // :1276-1278
        s.att = s.att + A.w * tmp;
        if (tmp != 0.0f) {
            const float dp = -A.y * gr.dx + A.x * gr.dz + dth;   // tilt about the y axis
            s.lr += dr; s.lx += gr.dx; s.lz += gr.dz; s.ly += gr.dy; s.lp += dp;
            s.da[2] += A.w * dr; s.da[3] += A.w * gr.dx; s.da[4] += A.w * gr.dy;
            s.da[5] += A.w * gr.dz; s.da[6] += A.w * dp;
        }
    }
    if (nr <= nh) return;
    if (s.lay < g.n_layers) close_layers_grad(g, s, g.n_layers, cosang);
    for (int j = nh; j < nr; ++j) {
        if (!in_rect(ws.rr[j], sa_a, sa_b)) continue;
        const float4 A = ws.ra[j];
        const float4 B = ws.rb[j];
        const float4 C = ws.rc[j];
        float xb, yb, zb;                                        // :1318-1320
        to_crystal_frame(A.x, A.y, A.z, B.x, B.y, xD, yD, zD, xb, yb, zb);
        const float la = box_chord(C.y, C.z, C.w, xb, yb, zb, -0.5f * B.z, -0.5f * B.w, -0.5f * C.x,
                                   0.5f * B.z, 0.5f * B.w, 0.5f * C.x);
        s.att = s.att + la * A.w;
        s.da[1] += la;
    }
}

// finish_sub_element with the partials of its contribution: dc[i] = d contrib / d theta_i.
__device__ __forceinline__ float finish_sub_element_grad(const Elem& e, const SubElem& q, WalkGrad& s,
                                                         float* dc)
{
    const float w = e.w, t = e.t, h = e.h;
    const float ux1 = ((float)q.ix / 8.0f - 0.5f) * w;
    const float ux2 = (((float)q.ix + 1.0f) / 8.0f - 0.5f) * w;
    const float uy1 = ((float)q.iy / 16.0f - 0.5f) * t;
    const float uy2 = (((float)q.iy + 1.0f) / 16.0f - 0.5f) * t;
    const float uz1 = ((float)q.iz / 8.0f - 0.5f) * h;
    const float uz2 = (((float)q.iz + 1.0f) / 8.0f - 0.5f) * h;
    const float cbox[6] = {-w / 2.0f, -t / 2.0f, -h / 2.0f, w / 2.0f, t / 2.0f, h / 2.0f};
    const float ubox[6] = {ux1, uy1, uz1, ux2, uy2, uz2};
    float l1, l2;
    box_chord_inside2(e.xIs, e.yIs, e.zIs, q.xDs, q.yDs, q.zDs, cbox, ubox, l1, l2);
    const float att = s.att + (l1 - l2) * e.mu_t;
    s.da[1] += l1 - l2;
    const float eff = 1.0f * expf(-att);
    const float xt = q.xDs + 1000.0f * (q.xDs - e.xIs) / q.sq;
    const float yt = q.yDs + 1000.0f * (q.yDs - e.yIs) / q.sq;
    const float zt = q.zDs + 1000.0f * (q.zDs - e.zIs) / q.sq;
    const float labs = box_chord(e.xIs, e.yIs, e.zIs, xt, yt, zt, ux1, uy1, uz1, ux2, uy2, uz2);
    const float ea = expf(-labs * e.mu_t);
    const float absf = (1.0f - ea) * e.mu_pe / e.mu_t;
    const float dabsf = labs * ea * e.mu_pe / e.mu_t - (1.0f - ea) * e.mu_pe / (e.mu_t * e.mu_t);
    const double rq = 1.0 / ((4.0 * 3.14159265358979323846) * (double)q.dsq * (double)q.sq);
    const float ax = t * h / 8.0f / 16.0f, az = w * t / 8.0f / 16.0f, ay = w * h / 8.0f / 8.0f;
    const float sax = (float)((double)ax * (double)fabsf((q.xD - e.xI) * e.cosr - (q.zD - e.zI) * e.sinr) * rq);
    const float saz = (float)((double)az * (double)fabsf((q.xD - e.xI) * e.sinr + (q.zD - e.zI) * e.cosr) * rq);
    const float say = (float)((double)ay * (double)fabsf(q.yD - e.yI) * rq);
    const float sxy = (sax >= say) ? sax : say;
    const float sa = (sxy >= saz) ? sxy : saz;
    const float base = eff * sa;
#pragma unroll
    for (int i = 0; i < kThetaN; ++i) dc[i] = -base * absf * s.da[i];
    dc[1] += base * dabsf;
    return base * absf;
}

// Value and theta-partials of element (d, v), summed over its sub-elements in double; every
// lane returns the warp's totals in acc[0..7] (acc[kThetaN] = the value).
template <bool ELL>
__device__ __forceinline__ void pe_element_grad(const DevGeom& g, const BlockSmem& bs, WarpSmem& ws, int d, long long v,
                                float cr, float sr, int lane, double* acc)
{
#pragma unroll
    for (int i = 0; i <= kThetaN; ++i) acc[i] = 0.0;
    Elem e;
    if (!init_element(g, ws, d, v, cr, sr, lane, e)) return;
    const bool from_super = bs.s_count >= 0;
    const int n_src = from_super ? bs.s_count : g.n_holes + g.n_det;
    int count = 0;
    const int cursor = build_chunk(g, bs, ws, e, d, 0, n_src, from_super, lane, &count);
    const bool single = cursor >= n_src;
    for (int r = 0; r < 32; ++r) {
        const int sidx = ((r >> 3) * 2 + (lane >> 4)) * 128 + ((lane >> 1) & 7) * 16 + (r & 7) * 2 +
                         (lane & 1);
        const SubElem q = sub_element(e, sidx);
        WalkGrad s;
        s.att = 0.0f;
        s.len = 0.0f;
        s.lay = 0;
        s.lr = s.lx = s.lz = s.ly = s.lp = 0.0f;
#pragma unroll
        for (int i = 0; i < kThetaN; ++i) s.da[i] = 0.0f;
        RayCyl rc;
        ray_cyl_init(rc, e.xI, e.yI, e.zI, q.xD, q.yD, q.zD);
        const bool blocked = plate_penalty(g, ws, e, q, s.att);
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
                if (!skip) walk_round_grad<ELL>(g, ws, nh, nr, q.xD, q.yD, q.zD, q.sa_a, q.sa_b, q.cosang, rc, s);
                __syncwarp();
                k = next;
            }
            if (single || cur >= n_src) break;
        }
        if (!skip) {
            if (s.lay < g.n_layers) close_layers_grad(g, s, g.n_layers, q.cosang);
            float dc[kThetaN];
            acc[kThetaN] += (double)finish_sub_element_grad(e, q, s, dc);
#pragma unroll
            for (int i = 0; i < kThetaN; ++i) acc[i] += (double)dc[i];
        }
    }
#pragma unroll
    for (int i = 0; i <= kThetaN; ++i)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
}

struct AdjSmem {
    BlockSmem bs;
    double acc[kWarps][kThetaN + 1];
    int any;
};

// KIND 0: p[d - det_begin] += sum_v A[d,v] x[v] (precise-mode elements).
// KIND 1: grad[i] += sum_{d,v} u[d - det_begin] x[v] dA[d,v]/dtheta_i, grad[7] += u^T A x.
// KIND 2: q[v] += sum_d A[d,v] u[d - det_begin] (back projection; x is not read).
// Elements of zero weight are skipped, and so are bricks whose voxels all have x = 0.
template <int KIND, bool ELL>
__global__ void __launch_bounds__(kThreads, 2) pe_adjoint_kernel(DevGeom g, AdjLaunch L)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    AdjSmem& sm = *reinterpret_cast<AdjSmem*>(smem_raw);
    BlockSmem& bs = sm.bs;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem& ws = bs.w[wid];
    if (KIND == 1 && lane <= kThetaN) sm.acc[wid][lane] = 0.0;
    const float ang = L.rotation * g.angle_step;           // :1006
    const float cr = cosf(ang), sr = sinf(ang);
    const int nbx = (g.nx + L.bx - 1) / L.bx, nby = (g.ny + L.by - 1) / L.by, nbz = (g.nz + L.bz - 1) / L.bz;
    const long long n_bricks = (long long)nbx * nby * nbz;
    const long long total = n_bricks * L.det_count;
    const int n_slots = L.bx * L.by * L.bz;
    for (;;) {
        if (threadIdx.x == 0) {
            bs.item = (long long)atomicAdd(L.work_counter, 1ull);
            sm.any = 0;
        }
        __syncthreads();
        const long long item = bs.item;
        if (item >= total) break;
        const int di = (int)(item / n_bricks);
        const long long b = item - (long long)di * n_bricks;
        const int gz = (int)(b / ((long long)nbx * nby));
        const int rem = (int)(b - (long long)gz * nbx * nby);
        const int gy = rem / nbx, gx = rem - gy * nbx;
        const int x0 = gx * L.bx, y0 = gy * L.by, z0 = gz * L.bz;
        const float ud = KIND >= 1 ? L.u[di] : 1.0f;
        // any voxel of the brick with a non-zero weight?
        for (int slot = threadIdx.x; slot < n_slots; slot += kThreads) {
            const int ix = x0 + slot % L.bx, iy = y0 + (slot / L.bx) % L.by, iz = z0 + slot / (L.bx * L.by);
            if (ix < g.nx && iy < g.ny && iz < g.nz && ud != 0.0f &&
                (KIND == 2 || L.x[ix + g.nx * ((long long)iy + (long long)g.ny * iz)] != 0.0f))
                sm.any = 1;
        }
        __syncthreads();
        if (sm.any) {
            const int x1 = min(x0 + L.bx, g.nx) - 1, y1 = min(y0 + L.by, g.ny) - 1, z1 = min(z0 + L.bz, g.nz) - 1;
            const int d = L.det_begin + di;
            float ax, ay, az, bxx, byy, bzz;
            voxel_centre(g, x0 + g.nx * ((long long)y0 + g.ny * z0), 1.0f, 0.0f, ax, ay, az);
            voxel_centre(g, x1 + g.nx * ((long long)y1 + g.ny * z1), 1.0f, 0.0f, bxx, byy, bzz);
            const float mx = 0.5f * (ax + bxx), my = 0.5f * (ay + byy), mz = 0.5f * (az + bzz);
            const float rho = 0.5f * sqrtf((bxx - ax) * (bxx - ax) + (byy - ay) * (byy - ay) +
                                           (bzz - az) * (bzz - az)) + 1e-3f;
            build_superset(g, bs, d, mx * cr - my * sr, mx * sr + my * cr, mz, rho);
            for (int slot = wid; slot < n_slots; slot += kWarps) {
                const int ix = x0 + slot % L.bx, iy = y0 + (slot / L.bx) % L.by, iz = z0 + slot / (L.bx * L.by);
                if (ix >= g.nx || iy >= g.ny || iz >= g.nz) continue;
                const long long v = ix + g.nx * ((long long)iy + (long long)g.ny * iz);
                const float xv = KIND == 2 ? 1.0f : L.x[v];
                if (xv == 0.0f || ud == 0.0f) continue;
                if constexpr (KIND == 0) {
                    const double val = pe_element<1, false, ELL>(g, bs, ws, d, v, cr, sr, lane, nullptr);
                    if (lane == 0) atomicAdd(&L.p[di], val * (double)xv);
                } else if constexpr (KIND == 2) {
                    const double val = pe_element<1, false, ELL>(g, bs, ws, d, v, cr, sr, lane, nullptr);
                    if (lane == 0) atomicAdd(&L.q[v], val * (double)ud);
                } else {
                    double acc[kThetaN + 1];
                    pe_element_grad<ELL>(g, bs, ws, d, v, cr, sr, lane, acc);
                    const double wgt = (double)ud * (double)xv;
                    if (lane == 0)
#pragma unroll
                        for (int i = 0; i <= kThetaN; ++i) sm.acc[wid][i] += wgt * acc[i];
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
    if constexpr (KIND == 1) {
        __syncthreads();
        if (threadIdx.x <= kThetaN) {
            double t = 0.0;
            for (int w = 0; w < kWarps; ++w) t += sm.acc[w][threadIdx.x];
            atomicAdd(&L.grad[threadIdx.x], t);
        }
    }
}
