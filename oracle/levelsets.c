/*
 * levelsets.c -- oracle for level sets and volume fractions (FP64).
 * TEST INFRASTRUCTURE ONLY (see fi_oracle.h).
 *
 * Restates src/LevelSets/volume_fractions.jl, volume_fractions_kernels.jl,
 * signed_distances.jl and compute_levelsets.jl.  Small 3x3 determinants follow
 * the StaticArrays formula dot(c1, cross(c2, c3)) that GeometryBasics vectors use;
 * dot products sum left to right.
 */
#include "fi_oracle.h"
#include <math.h>
#include <stddef.h>

typedef struct { double x, y, z; } v3;
typedef struct { double x, y; } v2;

static v3 v3sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 v3scale(v3 a, double s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static double v3dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3 v3cross(v3 a, v3 b) {
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}

/* volume_fractions.jl:1 */
static double perturb(double p) { return fabs(p) > 1e-20 ? p : (p > 0.0 ? 1e-20 : -1e-20); }

/* volume_fractions.jl:5 */
static double tetvol(v3 a, v3 b, v3 c, v3 d) {
    v3 c1 = v3sub(b, a), c2 = v3sub(c, a), c3 = v3sub(d, a);
    return (1.0 / 6.0) * fabs(v3dot(c1, v3cross(c2, c3)));
}

/* vij: volume_fractions.jl:49 */
static v3 vij(const double *ps, const v3 *v, int i, int j) {
    double den = ps[i] - ps[j];
    return v3sub(v3scale(v[j], ps[i] / den), v3scale(v[i], ps[j] / den));
}

/* volume_fractions.jl:48-103 (0-based indices here) */
static double tet_cut(const double ps[4], const v3 v[4]) {
    int nneg = (ps[0] < 0) + (ps[1] < 0) + (ps[2] < 0) + (ps[3] < 0);
    if (nneg == 0) return 0.0;
    if (nneg == 1) {
        if (ps[0] < 0) return tetvol(v[0], vij(ps, v, 0, 1), vij(ps, v, 0, 2), vij(ps, v, 0, 3));
        if (ps[1] < 0) return tetvol(v[1], vij(ps, v, 1, 0), vij(ps, v, 1, 2), vij(ps, v, 1, 3));
        if (ps[2] < 0) return tetvol(v[2], vij(ps, v, 2, 0), vij(ps, v, 2, 1), vij(ps, v, 2, 3));
        return tetvol(v[3], vij(ps, v, 3, 0), vij(ps, v, 3, 1), vij(ps, v, 3, 2));
    }
    if (nneg == 2) {
        if (ps[0] < 0 && ps[1] < 0)
            return tetvol(v[0], v[1], vij(ps, v, 0, 2), vij(ps, v, 1, 3)) +
                   tetvol(vij(ps, v, 1, 2), v[1], vij(ps, v, 0, 2), vij(ps, v, 1, 3)) +
                   tetvol(v[0], vij(ps, v, 0, 3), vij(ps, v, 0, 2), vij(ps, v, 1, 3));
        if (ps[0] < 0 && ps[2] < 0)
            return tetvol(v[0], v[2], vij(ps, v, 0, 3), vij(ps, v, 2, 1)) +
                   tetvol(vij(ps, v, 2, 3), v[2], vij(ps, v, 0, 3), vij(ps, v, 2, 1)) +
                   tetvol(v[0], vij(ps, v, 0, 1), vij(ps, v, 0, 3), vij(ps, v, 2, 1));
        if (ps[0] < 0 && ps[3] < 0)
            return tetvol(v[0], v[3], vij(ps, v, 0, 1), vij(ps, v, 3, 2)) +
                   tetvol(vij(ps, v, 3, 1), v[3], vij(ps, v, 0, 1), vij(ps, v, 3, 2)) +
                   tetvol(v[0], vij(ps, v, 0, 2), vij(ps, v, 0, 1), vij(ps, v, 3, 2));
        if (ps[1] < 0 && ps[2] < 0)
            return tetvol(v[2], v[1], vij(ps, v, 2, 0), vij(ps, v, 1, 3)) +
                   tetvol(vij(ps, v, 1, 0), v[1], vij(ps, v, 2, 0), vij(ps, v, 1, 3)) +
                   tetvol(v[2], vij(ps, v, 2, 3), vij(ps, v, 2, 0), vij(ps, v, 1, 3));
        if (ps[1] < 0 && ps[3] < 0)
            return tetvol(v[3], v[1], vij(ps, v, 3, 0), vij(ps, v, 1, 2)) +
                   tetvol(vij(ps, v, 1, 0), v[1], vij(ps, v, 3, 0), vij(ps, v, 1, 2)) +
                   tetvol(v[3], vij(ps, v, 3, 2), vij(ps, v, 3, 0), vij(ps, v, 1, 2));
        return tetvol(v[2], v[3], vij(ps, v, 2, 0), vij(ps, v, 3, 1)) +
               tetvol(vij(ps, v, 3, 0), v[3], vij(ps, v, 2, 0), vij(ps, v, 3, 1)) +
               tetvol(v[2], vij(ps, v, 2, 1), vij(ps, v, 2, 0), vij(ps, v, 3, 1));
    }
    if (nneg == 3) {
        double tot = tetvol(v[0], v[1], v[2], v[3]);
        if (ps[0] >= 0) return tot - tetvol(v[0], vij(ps, v, 0, 1), vij(ps, v, 0, 2), vij(ps, v, 0, 3));
        if (ps[1] >= 0) return tot - tetvol(v[1], vij(ps, v, 1, 0), vij(ps, v, 1, 2), vij(ps, v, 1, 3));
        if (ps[2] >= 0) return tot - tetvol(v[2], vij(ps, v, 2, 0), vij(ps, v, 2, 1), vij(ps, v, 2, 3));
        return tot - tetvol(v[3], vij(ps, v, 3, 0), vij(ps, v, 3, 1), vij(ps, v, 3, 2));
    }
    return tetvol(v[0], v[1], v[2], v[3]);
}

/* box split into 5 tetrahedra: volume_fractions.jl:106-115.  psi[m] belongs to
 * the corner with offsets (m&1, m>>1&1, m>>2&1) in (x, y, z). */
double fo_vol_box3(const double psi_in[8], const double d[3]) {
    double ps[8];
    for (int m = 0; m < 8; m++) ps[m] = perturb(psi_in[m]);
    v3 v000 = {0, 0, 0}, v001 = {d[0], 0, 0}, v010 = {0, d[1], 0}, v011 = {d[0], d[1], 0};
    v3 v100 = {0, 0, d[2]}, v101 = {d[0], 0, d[2]}, v110 = {0, d[1], d[2]}, v111 = {d[0], d[1], d[2]};
    double t1p[4] = {ps[0], ps[4], ps[2], ps[1]};
    v3 t1v[4] = {v000, v100, v010, v001};
    double t2p[4] = {ps[6], ps[4], ps[2], ps[7]};
    v3 t2v[4] = {v110, v100, v010, v111};
    double t3p[4] = {ps[5], ps[4], ps[7], ps[1]};
    v3 t3v[4] = {v101, v100, v111, v001};
    double t4p[4] = {ps[3], ps[7], ps[2], ps[1]};
    v3 t4v[4] = {v011, v111, v010, v001};
    double t5p[4] = {ps[7], ps[4], ps[2], ps[1]};
    v3 t5v[4] = {v111, v100, v010, v001};
    return tet_cut(t1p, t1v) + tet_cut(t2p, t2v) + tet_cut(t3p, t3v) + tet_cut(t4p, t4v) + tet_cut(t5p, t5v);
}

/* 2D: volume_fractions.jl:4, 8-37, 40-45 */
static double trivol(v2 a, v2 b, v2 c) {
    double c1x = c.x - a.x, c1y = c.y - a.y; /* column 1 = v3 - v1 */
    double c2x = b.x - a.x, c2y = b.y - a.y; /* column 2 = v2 - v1 */
    return 0.5 * fabs(c1x * c2y - c2x * c1y);
}
static v2 vij2(const double *ps, const v2 *v, int i, int j) {
    double den = ps[i] - ps[j];
    double a = ps[i] / den, b = ps[j] / den;
    v2 r = {v[j].x * a - v[i].x * b, v[j].y * a - v[i].y * b};
    return r;
}
static double tri_cut(const double ps[3], const v2 v[3]) {
    if (ps[0] < 0 && ps[1] < 0 && ps[2] < 0) return trivol(v[0], v[1], v[2]);
    if (ps[0] > 0 && ps[1] > 0 && ps[2] > 0) return 0.0;
    v2 v12 = vij2(ps, v, 0, 1), v13 = vij2(ps, v, 0, 2), v23 = vij2(ps, v, 1, 2);
    if (ps[0] < 0) {
        if (ps[1] < 0) return trivol(v[0], v23, v13) + trivol(v[0], v[1], v23);
        if (ps[2] < 0) return trivol(v[2], v12, v23) + trivol(v[2], v[0], v12);
        return trivol(v[0], v12, v13);
    }
    if (ps[1] < 0) {
        if (ps[2] < 0) return trivol(v[1], v13, v12) + trivol(v[1], v[2], v13);
        return trivol(v12, v[1], v23);
    }
    return trivol(v13, v23, v[2]);
}
double fo_vol_box2(const double psi_in[4], const double d[2]) {
    double p00 = perturb(psi_in[0]), p01 = perturb(psi_in[1]), p10 = perturb(psi_in[2]), p11 = perturb(psi_in[3]);
    v2 v00 = {0, 0}, v01 = {d[0], 0}, v10 = {0, d[1]}, v11 = {d[0], d[1]};
    double a[3] = {p00, p01, p11};
    v2 av[3] = {v00, v01, v11};
    double b[3] = {p00, p11, p10};
    v2 bv[3] = {v00, v11, v10};
    return tri_cut(a, av) + tri_cut(b, bv);
}

/* _omega_from_psi! 3D: volume_fractions_kernels.jl:31-97.  Output components
 * w[0..7] = ccc vvv vcc cvc ccv vvc vcv cvv, written over the vertex index range. */
void fo_volfrac3d(const int n[3], const double dx[3], const double *psi, double *w[8]) {
    size_t sx = (size_t)n[0] + 3, sy = (size_t)n[1] + 3, sxy = sx * sy;
    double pd = dx[0] * dx[1] * dx[2];
#define PS(i, j, k) psi[(size_t)(i) + sx * (size_t)(j) + sxy * (size_t)(k)]
#define LX(i, j, k) (0.5 * (PS(i, j, k) + PS((i) + 1, j, k)))
#define LY(i, j, k) (0.5 * (PS(i, j, k) + PS(i, (j) + 1, k)))
#define LZ(i, j, k) (0.5 * (PS(i, j, k) + PS(i, j, (k) + 1)))
#define LXY(i, j, k) (0.5 * (LX(i, j, k) + LX(i, (j) + 1, k)))
#define LXZ(i, j, k) (0.5 * (LX(i, j, k) + LX(i, j, (k) + 1)))
#define LYZ(i, j, k) (0.5 * (LY(i, j, k) + LY(i, j, (k) + 1)))
#define LXYZ(i, j, k) (0.5 * (LXY(i, j, k) + LXY(i, j, (k) + 1)))
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= n[2] + 1; k++)
        for (int j = 1; j <= n[1] + 1; j++)
            for (int i = 1; i <= n[0] + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                double c[8];
                /* ccc: vertex corners (i..i+1, j..j+1, k..k+1) */
                for (int m = 0; m < 8; m++) c[m] = PS(i + (m & 1), j + ((m >> 1) & 1), k + ((m >> 2) & 1));
                w[0][I] = fo_vol_box3(c, dx) / pd;
                /* vvv: centre-interpolated corners at (i-1..i, j-1..j, k-1..k) */
                for (int m = 0; m < 8; m++) c[m] = LXYZ(i - 1 + (m & 1), j - 1 + ((m >> 1) & 1), k - 1 + ((m >> 2) & 1));
                w[1][I] = fo_vol_box3(c, dx) / pd;
                /* vcc: lerp to (C,V,V) at (i-1..i, j..j+1, k..k+1) */
                for (int m = 0; m < 8; m++) c[m] = LX(i - 1 + (m & 1), j + ((m >> 1) & 1), k + ((m >> 2) & 1));
                w[2][I] = fo_vol_box3(c, dx) / pd;
                /* cvc: lerp to (V,C,V) at (i..i+1, j-1..j, k..k+1) */
                for (int m = 0; m < 8; m++) c[m] = LY(i + (m & 1), j - 1 + ((m >> 1) & 1), k + ((m >> 2) & 1));
                w[3][I] = fo_vol_box3(c, dx) / pd;
                /* ccv: lerp to (V,V,C) at (i..i+1, j..j+1, k-1..k) */
                for (int m = 0; m < 8; m++) c[m] = LZ(i + (m & 1), j + ((m >> 1) & 1), k - 1 + ((m >> 2) & 1));
                w[4][I] = fo_vol_box3(c, dx) / pd;
                /* vvc: lerp to (C,C,V) at (i-1..i, j-1..j, k..k+1) */
                for (int m = 0; m < 8; m++) c[m] = LXY(i - 1 + (m & 1), j - 1 + ((m >> 1) & 1), k + ((m >> 2) & 1));
                w[5][I] = fo_vol_box3(c, dx) / pd;
                /* vcv: lerp to (C,V,C) at (i-1..i, j..j+1, k-1..k) */
                for (int m = 0; m < 8; m++) c[m] = LXZ(i - 1 + (m & 1), j + ((m >> 1) & 1), k - 1 + ((m >> 2) & 1));
                w[6][I] = fo_vol_box3(c, dx) / pd;
                /* cvv: lerp to (V,C,C) at (i..i+1, j-1..j, k-1..k) */
                for (int m = 0; m < 8; m++) c[m] = LYZ(i + (m & 1), j - 1 + ((m >> 1) & 1), k - 1 + ((m >> 2) & 1));
                w[7][I] = fo_vol_box3(c, dx) / pd;
            }
#undef PS
#undef LX
#undef LY
#undef LZ
#undef LXY
#undef LXZ
#undef LYZ
#undef LXYZ
}

/* _omega_from_psi! 2D: volume_fractions_kernels.jl:2-28; w = cc vv vc cv */
void fo_volfrac2d(const int n[2], const double dx[2], const double *psi, double *w[4]) {
    size_t sx = (size_t)n[0] + 3;
    double pd = dx[0] * dx[1];
#define PS(i, j) psi[(size_t)(i) + sx * (size_t)(j)]
#define LX(i, j) (0.5 * (PS(i, j) + PS((i) + 1, j)))
#define LY(i, j) (0.5 * (PS(i, j) + PS(i, (j) + 1)))
#define LXY(i, j) (0.5 * (LX(i, j) + LX(i, (j) + 1)))
    for (int j = 1; j <= n[1] + 1; j++)
        for (int i = 1; i <= n[0] + 1; i++) {
            size_t I = (size_t)i + sx * (size_t)j;
            double c[4];
            for (int m = 0; m < 4; m++) c[m] = PS(i + (m & 1), j + (m >> 1));
            w[0][I] = fo_vol_box2(c, dx) / pd;
            for (int m = 0; m < 4; m++) c[m] = LXY(i - 1 + (m & 1), j - 1 + (m >> 1));
            w[1][I] = fo_vol_box2(c, dx) / pd;
            for (int m = 0; m < 4; m++) c[m] = LX(i - 1 + (m & 1), j + (m >> 1));
            w[2][I] = fo_vol_box2(c, dx) / pd;
            for (int m = 0; m < 4; m++) c[m] = LY(i + (m & 1), j - 1 + (m >> 1));
            w[3][I] = fo_vol_box2(c, dx) / pd;
        }
#undef PS
#undef LX
#undef LY
#undef LXY
}

/* signed_distances.jl:22-43 */
static double jsign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
static double S1(double x) { return x == 0.0 ? 1.0 : jsign(x); }
static double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }
static double ud_triangle(v3 p, v3 a, v3 b, v3 c) {
    v3 ba = v3sub(b, a), pa = v3sub(p, a), cb = v3sub(c, b), pb = v3sub(p, b), ac = v3sub(a, c), pc = v3sub(p, c);
    v3 nor = v3cross(ba, ac);
    double sg = jsign(v3dot(v3cross(ba, nor), pa)) + jsign(v3dot(v3cross(cb, nor), pb)) + jsign(v3dot(v3cross(ac, nor), pc));
    double r;
    if (sg < 2) {
        v3 e1 = v3sub(v3scale(ba, clamp01(v3dot(ba, pa) / v3dot(ba, ba))), pa);
        v3 e2 = v3sub(v3scale(cb, clamp01(v3dot(cb, pb) / v3dot(cb, cb))), pb);
        v3 e3 = v3sub(v3scale(ac, clamp01(v3dot(ac, pc) / v3dot(ac, ac))), pc);
        double d1 = v3dot(e1, e1), d2 = v3dot(e2, e2), d3 = v3dot(e3, e3);
        r = d1 < d2 ? d1 : d2;
        r = r < d3 ? r : d3;
    } else {
        double d = v3dot(nor, pa);
        r = d * d / v3dot(nor, nor);
    }
    return sqrt(r);
}

/* Julia fld(a, b) for floats: round((a - mod(a, b)) / b) */
static double jfld(double a, double b) {
    double r = fmod(a, b);
    if (r == 0.0) r = copysign(0.0, b);
    else if ((r > 0) != (b > 0)) r += b;
    return nearbyint((a - r) / b);
}

/* signed_distances.jl:45-53 (clamped vertex index, 1-based) */
static int closest_vertex(double p, double o, double d, int nv) {
    double X = jfld(p - o, d);
    long I = (long)X + 1;
    if (I < 1) I = 1;
    if (I > nv) I = nv;
    return (int)I;
}

/* compute_levelsets.jl:1-8 with sd_dem (signed_distances.jl:78-92).  The DEM is
 * a 2D vertex array in halo storage ((n2+3) per dim) with values valid up to
 * index n2+2; psi is a 3D vertex array in halo storage.  R is row-major 3x3 or
 * NULL for the identity. */
void fo_levelset_from_dem(const int n3[3], const double o3[3], const double dx3[3], const int n2[2],
                          const double o2[2], const double dx2[2], const double *dem, const double *Rm,
                          double cutoff, double *psi) {
    size_t sx = (size_t)n3[0] + 3, sy = (size_t)n3[1] + 3, sxy = sx * sy;
    size_t dsx = (size_t)n2[0] + 3;
    double ext2[2] = {dx2[0] * n2[0], dx2[1] * n2[1]};
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 1; k <= n3[2] + 1; k++)
        for (int j = 1; j <= n3[1] + 1; j++)
            for (int i = 1; i <= n3[0] + 1; i++) {
                double x = o3[0] + (double)(i - 1) * dx3[0];
                double y = o3[1] + (double)(j - 1) * dx3[1];
                double z = o3[2] + (double)(k - 1) * dx3[2];
                v3 P;
                if (Rm) {
                    P.x = Rm[0] * x + Rm[1] * y + Rm[2] * z;
                    P.y = Rm[3] * x + Rm[4] * y + Rm[5] * z;
                    P.z = Rm[6] * x + Rm[7] * y + Rm[8] * z;
                } else {
                    P.x = x; P.y = y; P.z = z;
                }
                double px = P.x, py = P.y;
                double lo0 = o2[0], hi0 = o2[0] + ext2[0], lo1 = o2[1], hi1 = o2[1] + ext2[1];
                px = px < lo0 ? lo0 : (px > hi0 ? hi0 : px);
                py = py < lo1 ? lo1 : (py > hi1 ? hi1 : py);
                int blx = closest_vertex(px - cutoff, o2[0], dx2[0], n2[0] + 1);
                int bly = closest_vertex(py - cutoff, o2[1], dx2[1], n2[1] + 1);
                int trx = closest_vertex(px + cutoff, o2[0], dx2[0], n2[0] + 1);
                int try_ = closest_vertex(py + cutoff, o2[1], dx2[1], n2[1] + 1);
                int icx = closest_vertex(px, o2[0], dx2[0], n2[0] + 1);
                int icy = closest_vertex(py, o2[1], dx2[1], n2[1] + 1);
                double ud = INFINITY, sgn = 1.0;
                for (int pass = 0; pass < 2; pass++) {
                    int ylo = pass == 0 ? icy : bly, yhi = pass == 0 ? icy : try_;
                    int xlo = pass == 0 ? icx : blx, xhi = pass == 0 ? icx : trx;
                    for (int jv = ylo; jv <= yhi; jv++)
                        for (int iv = xlo; iv <= xhi; iv++) {
                            if (pass == 1 && iv == icx && jv == icy) continue;
                            /* triangle_pair: signed_distances.jl:58-66 */
                            v3 s00 = {o2[0] + (double)(iv - 1) * dx2[0], o2[1] + (double)(jv - 1) * dx2[1],
                                      dem[(size_t)iv + dsx * (size_t)jv]};
                            v3 s10 = {o2[0] + (double)(iv)*dx2[0], o2[1] + (double)(jv - 1) * dx2[1],
                                      dem[(size_t)iv + 1 + dsx * (size_t)jv]};
                            v3 s01 = {o2[0] + (double)(iv - 1) * dx2[0], o2[1] + (double)(jv)*dx2[1],
                                      dem[(size_t)iv + dsx * (size_t)(jv + 1)]};
                            v3 s11 = {o2[0] + (double)(iv)*dx2[0], o2[1] + (double)(jv)*dx2[1],
                                      dem[(size_t)iv + 1 + dsx * (size_t)(jv + 1)]};
                            double d1 = ud_triangle(P, s00, s10, s01);
                            double d2 = ud_triangle(P, s01, s10, s11);
                            double dp = d1 < d2 ? d1 : d2;
                            if (pass == 0) {
                                ud = dp;
                                sgn = S1(v3dot(v3sub(P, s00), v3cross(v3sub(s10, s00), v3sub(s01, s00))));
                            } else if (dp < ud) {
                                ud = dp;
                            }
                        }
                }
                psi[(size_t)i + sx * (size_t)j + sxy * (size_t)k] = ud * sgn;
            }
    fo_neumann_vertex3(n3, psi);
}

/* Neumann on a 3D vertex field (adopted contract: f[0]=f[2], f[n+2]=f[n]),
 * dims x, y, z in order */
void fo_neumann_vertex3(const int n3[3], double *psi) {
    size_t sx = (size_t)n3[0] + 3, sy = (size_t)n3[1] + 3, sxy = sx * sy;
    /* x faces: j,k interior */
    for (int k = 1; k <= n3[2] + 1; k++)
        for (int j = 1; j <= n3[1] + 1; j++) {
            size_t B = sx * (size_t)j + sxy * (size_t)k;
            psi[B + 0] = psi[B + 2];
            psi[B + (size_t)n3[0] + 2] = psi[B + (size_t)n3[0]];
        }
    /* y faces: i full, k interior */
    for (int k = 1; k <= n3[2] + 1; k++)
        for (int i = 0; i <= n3[0] + 2; i++) {
            size_t B = (size_t)i + sxy * (size_t)k;
            psi[B] = psi[B + 2 * sx];
            psi[B + sx * ((size_t)n3[1] + 2)] = psi[B + sx * (size_t)n3[1]];
        }
    /* z faces: i, j full */
    for (int j = 0; j <= n3[1] + 2; j++)
        for (int i = 0; i <= n3[0] + 2; i++) {
            size_t B = (size_t)i + sx * (size_t)j;
            psi[B] = psi[B + 2 * sxy];
            psi[B + sxy * ((size_t)n3[2] + 2)] = psi[B + sxy * (size_t)n3[2]];
        }
}

/* compute_levelsets.jl:10-14, 32-35 */
void fo_invert_levelset(const int n3[3], double *psi) {
    size_t sx = (size_t)n3[0] + 3, sy = (size_t)n3[1] + 3, sxy = sx * sy;
    for (int k = 1; k <= n3[2] + 1; k++)
        for (int j = 1; j <= n3[1] + 1; j++)
            for (int i = 1; i <= n3[0] + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                psi[I] = -psi[I];
            }
    fo_neumann_vertex3(n3, psi);
}
