/* CPU oracle for the SPECT system-matrix path.  TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's photoelectric kernel
 * (PEGen_RayTracing_CircularHole/PESysMatGen.cu:20-799, :951-1364), its primary-Compton
 * kernels (ScatterGen_RayTracing_CircularHole/scatter.cu:961-1437, :1544-1936,
 * ScatterGen_Collimator/scatter.cu:1212-1215) and the geometry-relationship bitmaps
 * (scatter.cu:1440-1540, :1939-2009).  The element functions live in oracle_body.h and
 * are compiled twice: FP32 (the reference's arithmetic in float, double where the
 * reference promotes) and FP64 (every float variable widened).
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg call this library, as the
 * checker.  Nothing in the product links or loads it.
 *
 * Parity pin: the FP32 twin is checked against golden vectors produced by the
 * reference's own CUDA build (tests/golden/make_golden.py).
 */
#define _GNU_SOURCE
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define MAX_LAYERS 16

typedef struct {
    const float *C, *D, *I, *P;
    const float* S;    /* optional hole shapes: rho_x, rho_z, theta per hole (rho_x <= 0: circle) */
    int L, ncry, nx, ny, nz, nh0, nholes;
    int div[3];        /* PE crystal sub-elements along x, depth, z (reference: 8, 16, 8) */
    int vsub[3];       /* PE source points per voxel along x, y, z (reference: 1, 1, 1) */
    long long nvox;
    int nh[MAX_LAYERS];
} ogeo;

typedef struct {
    long long subelements, hole_hits, crystal_hits;
    long long cand_crystals, cand_holes;
} pe_counts;

/* ---- FP32 instantiation ---- */
#define REAL float
#define SUFFIX _f32
#define SQRT sqrtf
#define EXP expf
#define COS cosf
#define SIN sinf
#define ACOS acosf
#define ASIN asinf
#define ERF erff
#define FABS fabsf
#include "oracle_body.h"
#undef REAL
#undef SUFFIX
#undef SQRT
#undef EXP
#undef COS
#undef SIN
#undef ACOS
#undef ASIN
#undef ERF
#undef FABS

/* ---- FP64 instantiation ---- */
#define REAL double
#define SUFFIX _f64
#define SQRT sqrt
#define EXP exp
#define COS cos
#define SIN sin
#define ACOS acos
#define ASIN asin
#define ERF erf
#define FABS fabs
#include "oracle_body.h"

#undef REAL
#undef SUFFIX
#undef SQRT
#undef EXP
#undef COS
#undef SIN
#undef ACOS
#undef ASIN
#undef ERF
#undef FABS

#include "oracle_local.h"
#include "oracle_grid.h"

/* Decode counts the way the reference kernels do (PESysMatGen.cu:964-1013,
 * scatter.cu:1555, :1108-1110). */
static int parse(ogeo* g, const float* C, const float* D, const float* I, const float* P)
{
    memset(g, 0, sizeof(*g));
    g->C = C; g->D = D; g->I = I; g->P = P;
    g->L = C ? (int)floorf(C[0] + 0.000001f) : 0;
    g->ncry = (int)floorf(D[0] + 0.000001f);
    g->nx = (int)floorf(I[0]);
    g->ny = (int)floorf(I[1]);
    g->nz = (int)floorf(I[2]);
    g->nvox = (long long)g->nx * g->ny * g->nz;
    if (g->L < 0 || g->L > MAX_LAYERS) return -1;
    for (int m = 0; m < g->L; ++m) {
        g->nh[m] = (int)floorf(C[(m + 1) * 10]);
        g->nholes += g->nh[m];
    }
    g->nh0 = C ? (int)floorf(C[10] + 0.000001f) : 0;
    g->div[0] = 8; g->div[1] = 16; g->div[2] = 8;
    g->vsub[0] = g->vsub[1] = g->vsub[2] = 1;
    return 0;
}

/* PE elements for detectors dets[0..ndet) and voxels [v0, v0+nv), row-major into out
 * (ndet x nv).  prec: 32 or 64.  counts (optional, ndet*nv*5 int64) receives the
 * instrumented work counts per element. */
static int run_pe(const ogeo* gp, int prec, const int* dets, int ndet, long long v0, long long nv, double* out,
                  long long* counts, int nthreads)
{
    const ogeo g = *gp;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    long long total = (long long)ndet * nv;
    int err = 0;
#pragma omp parallel
    {
        int* cc = (int*)malloc(sizeof(int) * (size_t)(g.ncry + 1));
        int* ch = (int*)malloc(sizeof(int) * (size_t)(g.nholes + 1));
        int nch[MAX_LAYERS];
        if (!cc || !ch) err = 1;
#pragma omp for schedule(dynamic, 16)
        for (long long e = 0; e < total; ++e) {
            if (!cc || !ch) continue;
            int d = dets[e / nv];
            long long v = v0 + e % nv;
            pe_counts pc;
            memset(&pc, 0, sizeof(pc));
            pe_counts* pcp = counts ? &pc : NULL;
            if (prec == 32) out[e] = (double)pe_element_f32(&g, d, v, cc, ch, nch, pcp);
            else            out[e] = pe_element_f64(&g, d, v, cc, ch, nch, pcp);
            if (counts) {
                counts[e * 5 + 0] = pc.subelements;
                counts[e * 5 + 1] = pc.hole_hits;
                counts[e * 5 + 2] = pc.crystal_hits;
                counts[e * 5 + 3] = pc.cand_crystals;
                counts[e * 5 + 4] = pc.cand_holes;
            }
        }
        free(cc);
        free(ch);
    }
    return err ? -2 : 0;
}

int oracle_pe_shapes(const float* C, const float* D, const float* I, const float* S, int prec, const int* dets,
                     int ndet, long long v0, long long nv, double* out, long long* counts, int nthreads)
{
    ogeo g;
    if (parse(&g, C, D, I, NULL)) return -1;
    g.S = S;
    return run_pe(&g, prec, dets, ndet, v0, nv, out, counts, nthreads);
}

/* PE elements of the sampled form: div[3] crystal sub-elements along x, depth, z and vsub[3]
 * source points per voxel along x, y, z (the reference: 8 x 16 x 8 and 1 x 1 x 1).  S: optional
 * hole shapes as for oracle_pe_shapes. */
int oracle_pe_sampled(const float* C, const float* D, const float* I, const float* S, const int* div,
                      const int* vsub, int prec, const int* dets, int ndet, long long v0, long long nv, double* out,
                      int nthreads)
{
    ogeo g;
    if (parse(&g, C, D, I, NULL)) return -1;
    g.S = S;
    for (int k = 0; k < 3; ++k) {
        if (div[k] < 1 || vsub[k] < 1) return -1;
        g.div[k] = div[k];
        g.vsub[k] = vsub[k];
    }
    return run_pe(&g, prec, dets, ndet, v0, nv, out, NULL, nthreads);
}

/* PE elements of the local-coordinate FP32 form (oracle_local.h) with div[3] crystal
 * sub-elements along x, depth, z and vsub[3] source points per voxel along x, y, z (the element
 * is the mean over the source points, in double), as float values widened to double.  S:
 * optional hole shapes (rho_x, rho_z, theta per hole; NULL: every hole circular). */
int oracle_pe_local_sampled(const float* C, const float* D, const float* I, const float* S, const int* div,
                            const int* vsub, const int* dets, int ndet, long long v0, long long nv, double* out,
                            int nthreads)
{
    ogeo g;
    if (parse(&g, C, D, I, NULL)) return -1;
    g.S = S;
    for (int k = 0; k < 3; ++k) {
        if (div[k] < 1 || vsub[k] < 1) return -1;
        g.div[k] = div[k];
        g.vsub[k] = vsub[k];
    }
    const int sx = vsub[0], sy = vsub[1], sz = vsub[2];
    if (nthreads > 0) omp_set_num_threads(nthreads);
    long long total = (long long)ndet * nv;
    int err = 0;
#pragma omp parallel
    {
        int* cc = (int*)malloc(sizeof(int) * (size_t)(g.ncry + 1));
        int* ch = (int*)malloc(sizeof(int) * (size_t)(g.nholes + 1));
        lhole* lh = (lhole*)malloc(sizeof(lhole) * (size_t)(g.nholes + 1));
        lcry* lc = (lcry*)malloc(sizeof(lcry) * (size_t)(g.ncry + 1));
        int nch[MAX_LAYERS];
        if (!cc || !ch || !lh || !lc) err = 1;
#pragma omp for schedule(dynamic, 16)
        for (long long e = 0; e < total; ++e) {
            if (!cc || !ch || !lh || !lc) continue;
            int d = dets[e / nv];
            long long v = v0 + e % nv;
            double acc = 0.0;
            for (int jz = 0; jz < sz; ++jz)
            for (int jy = 0; jy < sy; ++jy)
            for (int jx = 0; jx < sx; ++jx) {
                double xI, yI, zI;
                voxel_point_f64(&g, v, ((double)jx + 0.5) / (double)sx, ((double)jy + 0.5) / (double)sy,
                                ((double)jz + 0.5) / (double)sz, &xI, &yI, &zI);
                acc += (double)pe_element_local(&g, d, xI, yI, zI, cc, ch, nch, lh, lc, NULL);
            }
            out[e] = acc / (double)(sx * sy * sz);
        }
        free(cc);
        free(ch);
        free(lh);
        free(lc);
    }
    return err ? -2 : 0;
}

/* The local form at the reference's sampling (8 x 16 x 8 sub-elements, voxel centres). */
int oracle_pe_local(const float* C, const float* D, const float* I, const int* dets, int ndet, long long v0,
                    long long nv, double* out, int nthreads)
{
    const int div[3] = {8, 16, 8}, vsub[3] = {1, 1, 1};
    return oracle_pe_local_sampled(C, D, I, NULL, div, vsub, dets, ndet, v0, nv, out, nthreads);
}

/* Elements of the grid scatter model (oracle_grid.h) for detectors dets[0..ndet) and voxels
 * [v0, v0+nv), in double; parts: 1 crystal cells, 2 septal cells; cell: grid step (mm); S:
 * optional hole shapes (NULL: circular holes).  Each element spreads its cells over the
 * threads. */
int oracle_scatter_grid(const float* C, const float* D, const float* I, const float* P, const float* S, int parts,
                        double cell, const int* dets, int ndet, long long v0, long long nv, double* out, int nthreads)
{
    ogeo g;
    if (parse(&g, C, D, I, P)) return -1;
    g.S = S;
    if (!(cell > 0)) return -1;
    for (long long e = 0; e < (long long)ndet * nv; ++e)
        out[e] = grid_element(&g, parts, dets[e / nv], v0 + e % nv, cell, nthreads);
    return 0;
}

/* Per-sub-element contributions of element (d, v) (8 x 16 x 8, index (iz * 8 + ix) * 16 + iy):
 * which = 32 the FP32 twin, 64 the FP64 restatement, 0 the local-coordinate FP32 form.  For
 * locating where two evaluations of one element part. */
int oracle_pe_subelements(const float* C, const float* D, const float* I, int which, int d, long long v, double* out)
{
    ogeo g;
    if (parse(&g, C, D, I, NULL)) return -1;
    int* cc = (int*)malloc(sizeof(int) * (size_t)(g.ncry + 1));
    int* ch = (int*)malloc(sizeof(int) * (size_t)(g.nholes + 1));
    lhole* lh = (lhole*)malloc(sizeof(lhole) * (size_t)(g.nholes + 1));
    lcry* lc = (lcry*)malloc(sizeof(lcry) * (size_t)(g.ncry + 1));
    int nch[MAX_LAYERS];
    int rc = 0;
    if (!cc || !ch || !lh || !lc) rc = -2;
    else if (which == 64) {
        double xI, yI, zI;
        voxel_centre_f64(&g, v, &xI, &yI, &zI);
        pe_element_at_f64(&g, d, xI, yI, zI, cc, ch, nch, NULL, out);
    } else if (which == 32) {
        float xI, yI, zI, tmp[1024];
        voxel_centre_f32(&g, v, &xI, &yI, &zI);
        pe_element_at_f32(&g, d, xI, yI, zI, cc, ch, nch, NULL, tmp);
        for (int i = 0; i < 1024; ++i) out[i] = tmp[i];
    } else {
        double xI, yI, zI;
        float tmp[1024];
        voxel_centre_f64(&g, v, &xI, &yI, &zI);
        pe_element_local(&g, d, xI, yI, zI, cc, ch, nch, lh, lc, tmp);
        for (int i = 0; i < 1024; ++i) out[i] = tmp[i];
    }
    free(cc); free(ch); free(lh); free(lc);
    return rc;
}

int oracle_pe(const float* C, const float* D, const float* I, int prec, const int* dets, int ndet,
              long long v0, long long nv, double* out, long long* counts, int nthreads)
{
    return oracle_pe_shapes(C, D, I, NULL, prec, dets, ndet, v0, nv, out, counts, nthreads);
}

/* Scatter elements.  part: 1 crystal scatter, 2 collimator scatter (combined program's
 * hole solid angle), 3 collimator scatter (collimator-only program's solid angle).
 * pe: the D x V photoelectric matrix the reference reads from offset 0.  bitmap: the
 * crystal (part 1) or collimator (parts 2, 3) relationship bitmap. */
int oracle_scatter(const float* C, const float* D, const float* I, const float* P, const float* pe,
                   const uint32_t* bitmap, int part, int prec, const int* dets, int ndet,
                   long long v0, long long nv, double* out, int nthreads)
{
    ogeo g;
    if (parse(&g, C, D, I, P)) return -1;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    long long total = (long long)ndet * nv;
#pragma omp parallel for schedule(dynamic, 4)
    for (long long e = 0; e < total; ++e) {
        int d = dets[e / nv];
        long long v = v0 + e % nv;
        if (prec == 32) out[e] = (double)scatter_element_f32(&g, part, d, v, pe, bitmap, NULL);
        else            out[e] = scatter_element_f64(&g, part, d, v, pe, bitmap, NULL);
    }
    return 0;
}

/* Crystal-pair relationship bitmap (scatter.cu:1440-1540).  Words: ceil(D(D+1)/2*D/32). */
long long oracle_bitmap_crystal_words(const float* D)
{
    long long n = (long long)floorf(D[0] + 0.0001f);
    long long bits = n * (n + 1) / 2 * n;
    return (bits + 31) / 32;
}

void oracle_bitmap_crystal(const float* D, uint32_t* out, int nthreads)
{
    int n = (int)D[0];
    long long words = oracle_bitmap_crystal_words(D);
    memset(out, 0, sizeof(uint32_t) * (size_t)words);
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            const float *pi = D + 12 * i, *pj = D + 12 * j;
            float ri = sqrtf(pi[4] * pi[4] + pi[6] * pi[6] + pi[5] * pi[5]) / 2.0f;
            float rj = sqrtf(pj[4] * pj[4] + pj[6] * pj[6] + pj[5] * pj[5]) / 2.0f;
            float lij = dist3_f32(pi[1], pi[2], pi[3], pj[1], pj[2], pj[3]);
            float cij = ri / lij, cji = rj / lij;
            float uijx = (pi[1] - pj[1]) / lij, uijy = (pi[2] - pj[2]) / lij, uijz = (pi[3] - pj[3]) / lij;
            float ujix = (pj[1] - pi[1]) / lij, ujiy = (pj[2] - pi[2]) / lij, ujiz = (pj[3] - pi[3]) / lij;
            long long pair = (long long)i * n - ((long long)i * (i + 1)) / 2 + j;
            for (int k = 0; k < n; ++k) {
                if (k == i || k == j) continue;
                const float* pk = D + 12 * k;
                float rk = sqrtf(pk[4] * pk[4] + pk[6] * pk[6] + pk[5] * pk[5]) / 2.0f;
                float lik = dist3_f32(pk[1], pk[2], pk[3], pi[1], pi[2], pi[3]);
                float cki = rk / lik;
                float ljk = dist3_f32(pk[1], pk[2], pk[3], pj[1], pj[2], pj[3]);
                float ckj = rk / ljk;
                float ukix = (pk[1] - pi[1]) / lik, ukiy = (pk[2] - pi[2]) / lik, ukiz = (pk[3] - pi[3]) / lik;
                float ukjx = (pk[1] - pj[1]) / ljk, ukjy = (pk[2] - pj[2]) / ljk, ukjz = (pk[3] - pj[3]) / ljk;
                int hit = dist3_f32(ukix, ukiy, ukiz, ujix, ujiy, ujiz) <= cki + cji;
                if (!hit) hit = dist3_f32(ukjx, ukjy, ukjz, uijx, uijy, uijz) <= ckj + cij;
                if (hit) {
                    long long bit = pair * n + k;
                    __atomic_fetch_or(&out[bit >> 5], 1u << (bit & 31), __ATOMIC_RELAXED);
                }
            }
        }
    }
}

long long oracle_bitmap_collimator_words(const float* C, const float* D)
{
    long long n = (long long)floorf(D[0] + 0.0001f);
    long long h = (long long)floorf(C[10] + 0.01f);
    return (n * n * h + 31) / 32;
}

/* Hole-to-crystal relationship bitmap (scatter.cu:1939-2009). */
void oracle_bitmap_collimator(const float* C, const float* D, uint32_t* out, int nthreads)
{
    int n = (int)D[0];
    int nh = (int)C[10];
    long long words = oracle_bitmap_collimator_words(C, D);
    memset(out, 0, sizeof(uint32_t) * (size_t)words);
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < nh; ++i) {
        float xi = C[9 * i + 100], yi = (C[9 * i + 101] + C[9 * i + 102]) / 2.0f, zi = C[9 * i + 103];
        for (int j = 0; j < n; ++j) {
            const float* pj = D + 12 * j;
            float rj = sqrtf(pj[4] * pj[4] + pj[6] * pj[6] + pj[5] * pj[5]) / 2.0f;
            float lij = dist3_f32(xi, yi, zi, pj[1], pj[2], pj[3]);
            float cji = rj / lij;
            float ux = (pj[1] - xi) / lij, uy = (pj[2] - yi) / lij, uz = (pj[3] - zi) / lij;
            for (int k = 0; k < n; ++k) {
                const float* pk = D + 12 * k;
                float rk = sqrtf(pk[4] * pk[4] + pk[6] * pk[6] + pk[5] * pk[5]) / 2.0f;
                float lik = dist3_f32(pk[1], pk[2], pk[3], xi, yi, zi);
                float cki = rk / lik;
                float vx = (pk[1] - xi) / lik, vy = (pk[2] - yi) / lik, vz = (pk[3] - zi) / lik;
                if (dist3_f32(vx, vy, vz, ux, uy, uz) <= cki + cji) {
                    long long bit = ((long long)i * n + j) * n + k;
                    __atomic_fetch_or(&out[bit >> 5], 1u << (bit & 31), __ATOMIC_RELAXED);
                }
            }
        }
    }
}

/* Primitive chords for unit tests.  a: 12 values (box) or 11 values (cylinder). */
double oracle_box_chord(int prec, const double* a)
{
    if (prec == 32)
        return box_chord_f32((float)a[0], (float)a[1], (float)a[2], (float)a[3], (float)a[4],
                             (float)a[5], (float)a[6], (float)a[7], (float)a[8], (float)a[9],
                             (float)a[10], (float)a[11]);
    return box_chord_f64(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
}

double oracle_box_chord_inside(int prec, const double* a)
{
    if (prec == 32)
        return box_chord_inside_f32((float)a[0], (float)a[1], (float)a[2], (float)a[3], (float)a[4],
                                    (float)a[5], (float)a[6], (float)a[7], (float)a[8], (float)a[9],
                                    (float)a[10], (float)a[11]);
    return box_chord_inside_f64(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10],
                                a[11]);
}

double oracle_cyl_chord(int prec, const double* a)
{
    if (prec == 32)
        return cyl_chord_f32((float)a[0], (float)a[1], (float)a[2], (float)a[3], (float)a[4],
                             (float)a[5], (float)a[6], (float)a[7], (float)a[8], (float)a[9],
                             (float)a[10]);
    return cyl_chord_f64(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10]);
}

/* a: 13 values (x_in, y_in, z_in, x_out, y_out, z_out, xc, y1, y2, zc, rho_x, rho_z, theta). */
double oracle_ell_chord(int prec, const double* a)
{
    if (prec == 32)
        return ell_chord_f32((float)a[0], (float)a[1], (float)a[2], (float)a[3], (float)a[4], (float)a[5],
                             (float)a[6], (float)a[7], (float)a[8], (float)a[9], (float)a[10], (float)a[11],
                             cosf((float)a[12]), sinf((float)a[12]));
    return ell_chord_f64(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11], cos(a[12]),
                         sin(a[12]));
}

double oracle_kn_sum(int prec, double e0, double lo, double hi)
{
    if (prec == 32) return kn_sum_f32((float)e0, (float)lo, (float)hi, 0.01f);
    return kn_sum_f64(e0, lo, hi, (double)0.01f);
}

/* Per-item trace of one scatter element (debugging and tests): for item s, 9 values at
 * trace[9*s]: contribution, window margins (lower, upper), extended-ray chord, KN step
 * ratio (theta_max-theta_min)/0.01, theta_min, theta_max, attenuation, phi range.  Items
 * rejected before a field is computed leave it unchanged. */
double oracle_scatter_trace(const float* C, const float* D, const float* I, const float* P,
                            const float* pe, const uint32_t* bitmap, int part, int prec, int d,
                            long long v, double* trace)
{
    ogeo g;
    if (parse(&g, C, D, I, P)) return NAN;
    if (prec == 32) return (double)scatter_element_f32(&g, part, d, v, pe, bitmap, trace);
    return scatter_element_f64(&g, part, d, v, pe, bitmap, trace);
}
