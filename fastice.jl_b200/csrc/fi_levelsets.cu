// fi_levelsets.cu -- level set from a DEM and level set -> volume fractions.
//
// ω_from_ψ!: src/LevelSets/volume_fractions_kernels.jl:2-110 with the exact
// cut-cell volumes of src/LevelSets/volume_fractions.jl (box split into five
// tetrahedra in 3D, two triangles in 2D).  One thread per grid index computes
// all staggered components; ψ is read through the read-only cache (each value
// feeds up to 64 dual-cell corners of neighbouring threads).
//
// compute_levelset_from_dem!: src/LevelSets/compute_levelsets.jl:1-35 and
// signed_distances.jl:22-92: unsigned distance to the two triangles of every
// DEM cell inside a window of +-cutoff around the point, sign from the
// bottom-left triangle of the closest cell.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "fi_internal.h"

namespace fi {

namespace {

struct v3 {
    double x, y, z;
};
__device__ __forceinline__ v3 sub(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 scl(v3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

__device__ __forceinline__ double perturb(double p) { return fabs(p) > 1e-20 ? p : (p > 0.0 ? 1e-20 : -1e-20); }

__device__ __forceinline__ double tetvol(v3 a, v3 b, v3 c, v3 d) {
    return (1.0 / 6.0) * fabs(dot(sub(b, a), cross(sub(c, a), sub(d, a))));
}

__device__ __forceinline__ v3 vij(const double *ps, const v3 *v, int i, int j) {
    double den = ps[i] - ps[j];
    return sub(scl(v[j], ps[i] / den), scl(v[i], ps[j] / den));
}

// volume of {ψ < 0} in a tetrahedron (volume_fractions.jl:48-103)
__device__ double tet_cut(const double ps[4], const v3 v[4]) {
    int nneg = (ps[0] < 0) + (ps[1] < 0) + (ps[2] < 0) + (ps[3] < 0);
    if (nneg == 0) return 0.0;
    if (nneg == 4) return tetvol(v[0], v[1], v[2], v[3]);
    if (nneg == 1 || nneg == 3) {
        // the odd vertex out: the single negative (nneg==1) or the single non-negative (nneg==3)
        int q;
        if (nneg == 1) q = ps[0] < 0 ? 0 : ps[1] < 0 ? 1 : ps[2] < 0 ? 2 : 3;
        else q = ps[0] >= 0 ? 0 : ps[1] >= 0 ? 1 : ps[2] >= 0 ? 2 : 3;
        int o[3], n = 0;
        for (int k = 0; k < 4; k++)
            if (k != q) o[n++] = k;
        double corner = tetvol(v[q], vij(ps, v, q, o[0]), vij(ps, v, q, o[1]), vij(ps, v, q, o[2]));
        if (nneg == 1) return corner;
        return tetvol(v[0], v[1], v[2], v[3]) - corner;
    }
    // two negative vertices a < b, two non-negative c, d: the three-tetrahedron
    // decomposition of volume_fractions.jl:63-88 for the matching case
    int a, b, cc, d;
    if (ps[0] < 0 && ps[1] < 0) { a = 0; b = 1; cc = 2; d = 3; }
    else if (ps[0] < 0 && ps[2] < 0) { a = 0; b = 2; cc = 3; d = 1; }
    else if (ps[0] < 0 && ps[3] < 0) { a = 0; b = 3; cc = 1; d = 2; }
    else if (ps[1] < 0 && ps[2] < 0) { a = 2; b = 1; cc = 0; d = 3; }
    else if (ps[1] < 0 && ps[3] < 0) { a = 3; b = 1; cc = 0; d = 2; }
    else { a = 2; b = 3; cc = 0; d = 1; }
    v3 ac = vij(ps, v, a, cc), bd = vij(ps, v, b, d), bc = vij(ps, v, b, cc), ad = vij(ps, v, a, d);
    return tetvol(v[a], v[b], ac, bd) + tetvol(bc, v[b], ac, bd) + tetvol(v[a], ad, ac, bd);
}

__device__ double vol_box3(const double psi[8], double dx, double dy, double dz) {
    double ps[8];
    for (int m = 0; m < 8; m++) ps[m] = perturb(psi[m]);
    const v3 v000 = {0, 0, 0}, v001 = {dx, 0, 0}, v010 = {0, dy, 0}, v011 = {dx, dy, 0};
    const v3 v100 = {0, 0, dz}, v101 = {dx, 0, dz}, v110 = {0, dy, dz}, v111 = {dx, dy, dz};
    double p1[4] = {ps[0], ps[4], ps[2], ps[1]};
    v3 t1[4] = {v000, v100, v010, v001};
    double p2[4] = {ps[6], ps[4], ps[2], ps[7]};
    v3 t2[4] = {v110, v100, v010, v111};
    double p3[4] = {ps[5], ps[4], ps[7], ps[1]};
    v3 t3[4] = {v101, v100, v111, v001};
    double p4[4] = {ps[3], ps[7], ps[2], ps[1]};
    v3 t4[4] = {v011, v111, v010, v001};
    double p5[4] = {ps[7], ps[4], ps[2], ps[1]};
    v3 t5[4] = {v111, v100, v010, v001};
    return tet_cut(p1, t1) + tet_cut(p2, t2) + tet_cut(p3, t3) + tet_cut(p4, t4) + tet_cut(p5, t5);
}

struct v2 {
    double x, y;
};
__device__ __forceinline__ double trivol(v2 a, v2 b, v2 c) {
    double c1x = c.x - a.x, c1y = c.y - a.y, c2x = b.x - a.x, c2y = b.y - a.y;
    return 0.5 * fabs(c1x * c2y - c2x * c1y);
}
__device__ __forceinline__ v2 vij2(const double *ps, const v2 *v, int i, int j) {
    double den = ps[i] - ps[j];
    double a = ps[i] / den, b = ps[j] / den;
    return {v[j].x * a - v[i].x * b, v[j].y * a - v[i].y * b};
}
__device__ double tri_cut(const double ps[3], const v2 v[3]) {
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
__device__ double vol_box2(const double psi[4], double dx, double dy) {
    double p00 = perturb(psi[0]), p01 = perturb(psi[1]), p10 = perturb(psi[2]), p11 = perturb(psi[3]);
    v2 v00 = {0, 0}, v01 = {dx, 0}, v10 = {0, dy}, v11 = {dx, dy};
    double a[3] = {p00, p01, p11};
    v2 av[3] = {v00, v01, v11};
    double b[3] = {p00, p11, p10};
    v2 bv[3] = {v00, v11, v10};
    return tri_cut(a, av) + tri_cut(b, bv);
}

__global__ void volfrac3d_kernel(Geom g, double dx, double dy, double dz, const double *__restrict__ psi, double *w0,
                                 double *w1, double *w2, double *w3, double *w4, double *w5, double *w6, double *w7) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > g.n[0] + 1 || j > g.n[1] + 1) return;
    const long long sx = g.pitch, sxy = g.sxy;
    const long long I = i + sx * j + sxy * k;
    auto PS = [&](int a, int b, int c) { return __ldg(psi + I + a + sx * b + sxy * c); };
    auto LX = [&](int a, int b, int c) { return 0.5 * (PS(a, b, c) + PS(a + 1, b, c)); };
    auto LY = [&](int a, int b, int c) { return 0.5 * (PS(a, b, c) + PS(a, b + 1, c)); };
    auto LZ = [&](int a, int b, int c) { return 0.5 * (PS(a, b, c) + PS(a, b, c + 1)); };
    auto LXY = [&](int a, int b, int c) { return 0.5 * (LX(a, b, c) + LX(a, b + 1, c)); };
    auto LXZ = [&](int a, int b, int c) { return 0.5 * (LX(a, b, c) + LX(a, b, c + 1)); };
    auto LYZ = [&](int a, int b, int c) { return 0.5 * (LY(a, b, c) + LY(a, b, c + 1)); };
    auto LXYZ = [&](int a, int b, int c) { return 0.5 * (LXY(a, b, c) + LXY(a, b, c + 1)); };
    const double pd = dx * dy * dz;
    double c[8];
#define CORNERS(expr, ox, oy, oz)                                                      \
    for (int m = 0; m < 8; m++) {                                                      \
        int a_ = (ox) + (m & 1), b_ = (oy) + ((m >> 1) & 1), c_ = (oz) + ((m >> 2) & 1); \
        c[m] = expr(a_, b_, c_);                                                       \
    }
    CORNERS(PS, 0, 0, 0);
    w0[I] = vol_box3(c, dx, dy, dz) / pd;
    CORNERS(LXYZ, -1, -1, -1);
    w1[I] = vol_box3(c, dx, dy, dz) / pd;
    CORNERS(LX, -1, 0, 0);
    w2[I] = vol_box3(c, dx, dy, dz) / pd;
    CORNERS(LY, 0, -1, 0);
    w3[I] = vol_box3(c, dx, dy, dz) / pd;
    CORNERS(LZ, 0, 0, -1);
    w4[I] = vol_box3(c, dx, dy, dz) / pd;
    CORNERS(LXY, -1, -1, 0);
    w5[I] = vol_box3(c, dx, dy, dz) / pd;
    CORNERS(LXZ, -1, 0, -1);
    w6[I] = vol_box3(c, dx, dy, dz) / pd;
    CORNERS(LYZ, 0, -1, -1);
    w7[I] = vol_box3(c, dx, dy, dz) / pd;
#undef CORNERS
}

__global__ void volfrac2d_kernel(Geom g, double dx, double dy, const double *__restrict__ psi, double *w0, double *w1,
                                 double *w2, double *w3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i > g.n[0] + 1 || j > g.n[1] + 1) return;
    const long long sx = g.pitch;
    const long long I = i + sx * j;
    auto PS = [&](int a, int b) { return __ldg(psi + I + a + sx * b); };
    auto LX = [&](int a, int b) { return 0.5 * (PS(a, b) + PS(a + 1, b)); };
    auto LY = [&](int a, int b) { return 0.5 * (PS(a, b) + PS(a, b + 1)); };
    auto LXY = [&](int a, int b) { return 0.5 * (LX(a, b) + LX(a, b + 1)); };
    const double pd = dx * dy;
    double c[4];
    for (int m = 0; m < 4; m++) c[m] = PS(m & 1, m >> 1);
    w0[I] = vol_box2(c, dx, dy) / pd;
    for (int m = 0; m < 4; m++) c[m] = LXY(-1 + (m & 1), -1 + (m >> 1));
    w1[I] = vol_box2(c, dx, dy) / pd;
    for (int m = 0; m < 4; m++) c[m] = LX(-1 + (m & 1), m >> 1);
    w2[I] = vol_box2(c, dx, dy) / pd;
    for (int m = 0; m < 4; m++) c[m] = LY(m & 1, -1 + (m >> 1));
    w3[I] = vol_box2(c, dx, dy) / pd;
}

// ---- signed distance to a DEM -------------------------------------------------
__device__ __forceinline__ double jsign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
__device__ __forceinline__ double clamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

__device__ double ud_triangle(v3 p, v3 a, v3 b, v3 c) {
    v3 ba = sub(b, a), pa = sub(p, a), cb = sub(c, b), pb = sub(p, b), ac = sub(a, c), pc = sub(p, c);
    v3 nor = cross(ba, ac);
    double sg = jsign(dot(cross(ba, nor), pa)) + jsign(dot(cross(cb, nor), pb)) + jsign(dot(cross(ac, nor), pc));
    double r;
    if (sg < 2) {
        v3 e1 = sub(scl(ba, clamp01(dot(ba, pa) / dot(ba, ba))), pa);
        v3 e2 = sub(scl(cb, clamp01(dot(cb, pb) / dot(cb, cb))), pb);
        v3 e3 = sub(scl(ac, clamp01(dot(ac, pc) / dot(ac, ac))), pc);
        double d1 = dot(e1, e1), d2 = dot(e2, e2), d3 = dot(e3, e3);
        r = d1 < d2 ? d1 : d2;
        r = r < d3 ? r : d3;
    } else {
        double d = dot(nor, pa);
        r = d * d / dot(nor, nor);
    }
    return sqrt(r);
}

__device__ double jfld(double a, double b) {
    double r = fmod(a, b);
    if (r == 0.0) r = copysign(0.0, b);
    else if ((r > 0) != (b > 0)) r += b;
    return rint((a - r) / b);
}

__device__ int closest_vertex(double p, double o, double d, int nv) {
    double X = jfld(p - o, d);
    long long I = (long long)X + 1;
    if (I < 1) I = 1;
    if (I > nv) I = nv;
    return (int)I;
}

struct DemArgs {
    double o3[3], dx3[3], o2[2], dx2[2], R[9], cutoff;
    int n2[2];
    int has_R, invert;
    long long dem_pitch;
};

__global__ void levelset_kernel(Geom g, DemArgs a, const double *__restrict__ dem, double *psi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > g.n[0] + 1 || j > g.n[1] + 1) return;
    double x = a.o3[0] + (double)(i - 1) * a.dx3[0];
    double y = a.o3[1] + (double)(j - 1) * a.dx3[1];
    double z = a.o3[2] + (double)(k - 1) * a.dx3[2];
    v3 P;
    if (a.has_R) {
        P.x = a.R[0] * x + a.R[1] * y + a.R[2] * z;
        P.y = a.R[3] * x + a.R[4] * y + a.R[5] * z;
        P.z = a.R[6] * x + a.R[7] * y + a.R[8] * z;
    } else {
        P = {x, y, z};
    }
    const double lo0 = a.o2[0], hi0 = a.o2[0] + a.dx2[0] * a.n2[0], lo1 = a.o2[1], hi1 = a.o2[1] + a.dx2[1] * a.n2[1];
    double px = P.x < lo0 ? lo0 : (P.x > hi0 ? hi0 : P.x);
    double py = P.y < lo1 ? lo1 : (P.y > hi1 ? hi1 : P.y);
    int blx = closest_vertex(px - a.cutoff, a.o2[0], a.dx2[0], a.n2[0] + 1);
    int bly = closest_vertex(py - a.cutoff, a.o2[1], a.dx2[1], a.n2[1] + 1);
    int trx = closest_vertex(px + a.cutoff, a.o2[0], a.dx2[0], a.n2[0] + 1);
    int try_ = closest_vertex(py + a.cutoff, a.o2[1], a.dx2[1], a.n2[1] + 1);
    int icx = closest_vertex(px, a.o2[0], a.dx2[0], a.n2[0] + 1);
    int icy = closest_vertex(py, a.o2[1], a.dx2[1], a.n2[1] + 1);
    auto sample = [&](int iv, int jv) -> v3 {
        return {a.o2[0] + (double)(iv - 1) * a.dx2[0], a.o2[1] + (double)(jv - 1) * a.dx2[1],
                __ldg(dem + iv + a.dem_pitch * jv)};
    };
    double ud = 0.0, sgn = 1.0;
    {
        v3 s00 = sample(icx, icy), s10 = sample(icx + 1, icy), s01 = sample(icx, icy + 1), s11 = sample(icx + 1, icy + 1);
        double d1 = ud_triangle(P, s00, s10, s01), d2 = ud_triangle(P, s01, s10, s11);
        ud = d1 < d2 ? d1 : d2;
        double sd = dot(sub(P, s00), cross(sub(s10, s00), sub(s01, s00)));
        sgn = sd == 0.0 ? 1.0 : jsign(sd);
    }
    for (int jv = bly; jv <= try_; jv++)
        for (int iv = blx; iv <= trx; iv++) {
            if (iv == icx && jv == icy) continue;
            v3 s00 = sample(iv, jv), s10 = sample(iv + 1, jv), s01 = sample(iv, jv + 1), s11 = sample(iv + 1, jv + 1);
            double d1 = ud_triangle(P, s00, s10, s01), d2 = ud_triangle(P, s01, s10, s11);
            double dp = d1 < d2 ? d1 : d2;
            if (dp < ud) ud = dp;
        }
    double v = ud * sgn;
    if (a.invert) v = -v;
    psi[i + g.pitch * j + g.sxy * k] = v;
}

// Neumann on a vertex field, one dim at a time (x faces over interior y,z; y
// faces over all x and interior z; z faces over all x, y)
__global__ void neumann_vertex_kernel(Geom g, double *f, int d) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    const long long sx = g.pitch, sxy = g.sxy;
    int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
    if (d == 0) {
        int j = a + 1, k = b + 1;
        if (j > n1 + 1 || k > n2 + 1) return;
        long long B = sx * j + sxy * k;
        f[B] = f[B + 2];
        f[B + n0 + 2] = f[B + n0];
    } else if (d == 1) {
        int i = a, k = b + 1;
        if (i > n0 + 2 || k > n2 + 1) return;
        long long B = i + sxy * k;
        f[B] = f[B + 2 * sx];
        f[B + sx * (n1 + 2)] = f[B + sx * n1];
    } else {
        int i = a, j = b;
        if (i > n0 + 2 || j > n1 + 2) return;
        long long B = i + sx * j;
        f[B] = f[B + 2 * sxy];
        f[B + sxy * (n2 + 2)] = f[B + sxy * n2];
    }
}

template <typename T>
__global__ void convert_kernel(const double *src, T *dst, long long n) {
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[t] = T(src[t]);
}

}  // namespace

cudaError_t launch_convert_f64_f32(const double *src, float *dst, long long n, cudaStream_t s) {
    convert_kernel<float><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_volfrac3d(const Geom &g, const double dx[3], const double *psi, double *const w[8], cudaStream_t s) {
    dim3 blk(32, 4);
    dim3 grd((g.n[0] + 1 + 31) / 32, (g.n[1] + 1 + 3) / 4, g.n[2] + 1);
    volfrac3d_kernel<<<grd, blk, 0, s>>>(g, dx[0], dx[1], dx[2], psi, w[0], w[1], w[2], w[3], w[4], w[5], w[6], w[7]);
    return cudaGetLastError();
}

cudaError_t launch_volfrac2d(const Geom &g, const double dx[2], const double *psi, double *const w[4], cudaStream_t s) {
    dim3 blk(32, 4);
    dim3 grd((g.n[0] + 1 + 31) / 32, (g.n[1] + 1 + 3) / 4, 1);
    volfrac2d_kernel<<<grd, blk, 0, s>>>(g, dx[0], dx[1], psi, w[0], w[1], w[2], w[3]);
    return cudaGetLastError();
}

cudaError_t launch_levelset(const Geom &g3, const double o3[3], const double dx3[3], const int n2[2], const double o2[2],
                            const double dx2[2], long long dem_pitch, const double *dem, const double *R, int has_R,
                            double cutoff, int invert, double *psi, cudaStream_t s) {
    DemArgs a{};
    for (int q = 0; q < 3; q++) {
        a.o3[q] = o3[q];
        a.dx3[q] = dx3[q];
    }
    for (int q = 0; q < 2; q++) {
        a.o2[q] = o2[q];
        a.dx2[q] = dx2[q];
        a.n2[q] = n2[q];
    }
    a.has_R = has_R;
    if (has_R)
        for (int q = 0; q < 9; q++) a.R[q] = R[q];
    a.cutoff = cutoff;
    a.invert = invert;
    a.dem_pitch = dem_pitch;
    dim3 blk(32, 4);
    dim3 grd((g3.n[0] + 1 + 31) / 32, (g3.n[1] + 1 + 3) / 4, g3.n[2] + 1);
    levelset_kernel<<<grd, blk, 0, s>>>(g3, a, dem, psi);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int n0 = g3.n[0], n1 = g3.n[1], nz = g3.n[2];
    neumann_vertex_kernel<<<dim3((n1 + 1 + 31) / 32, (nz + 1 + 7) / 8), dim3(32, 8), 0, s>>>(g3, psi, 0);
    neumann_vertex_kernel<<<dim3((n0 + 3 + 31) / 32, (nz + 1 + 7) / 8), dim3(32, 8), 0, s>>>(g3, psi, 1);
    neumann_vertex_kernel<<<dim3((n0 + 3 + 31) / 32, (n1 + 3 + 7) / 8), dim3(32, 8), 0, s>>>(g3, psi, 2);
    return cudaGetLastError();
}

}  // namespace fi

using namespace fi;

namespace {

Geom geom_of(const fi_grid &gr, bool pad) {
    Geom g{};
    g.nd = gr.nd;
    for (int k = 0; k < 3; k++) g.n[k] = k < gr.nd ? gr.n[k] : 0;
    g.pitch = pad ? ((long long)gr.n[0] + 3 + 31) / 32 * 32 : (long long)gr.n[0] + 3;
    g.rows = gr.n[1] + 3;
    g.sxy = g.pitch * g.rows;
    g.planes = gr.nd == 3 ? gr.n[2] + 3 : 1;
    return g;
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" {

fi_status fi_volfrac(const fi_grid *grid, const double *psi_host, double **w_host, int32_t device) {
    if (!grid || !psi_host || !w_host) return set_error("bad argument"), FI_ERR_ARG;
    if (grid->nd != 2 && grid->nd != 3) return set_error("grid.nd must be 2 or 3"), FI_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaSetDevice");
    Geom g = geom_of(*grid, false);
    size_t elems = (size_t)g.sxy * g.planes, bytes = elems * sizeof(double);
    int ncomp = grid->nd == 3 ? 8 : 4;
    DevBuf dpsi, dw[8];
    if (cudaMalloc(&dpsi.p, bytes) != cudaSuccess) return set_error("allocation failed"), FI_ERR_OOM;
    for (int c = 0; c < ncomp; c++) {
        if (cudaMalloc(&dw[c].p, bytes) != cudaSuccess) return set_error("allocation failed"), FI_ERR_OOM;
        if (cudaMemset(dw[c].p, 0, bytes) != cudaSuccess) return cuda_fail(cudaGetLastError(), "memset");
    }
    if (cudaMemcpy(dpsi.p, psi_host, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "psi upload");
    double dx[3];
    for (int k = 0; k < grid->nd; k++) dx[k] = grid->extent[k] / grid->n[k];
    double *w[8];
    for (int c = 0; c < 8; c++) w[c] = (double *)dw[c].p;
    cudaError_t e = grid->nd == 3 ? launch_volfrac3d(g, dx, (const double *)dpsi.p, w, 0)
                                  : launch_volfrac2d(g, dx, (const double *)dpsi.p, w, 0);
    if (e != cudaSuccess) return cuda_fail(e, "volfrac kernel");
    for (int c = 0; c < ncomp; c++)
        if (cudaMemcpy(w_host[c], w[c], bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "volfrac download");
    return FI_OK;
}

fi_status fi_levelset_from_dem(const fi_grid *grid3, const fi_grid *dem_grid2, const double *dem_host, const double *R,
                               int32_t invert, double *psi_host, int32_t device) {
    if (!grid3 || !dem_grid2 || !dem_host || !psi_host) return set_error("bad argument"), FI_ERR_ARG;
    if (grid3->nd != 3 || dem_grid2->nd != 2) return set_error("need a 3D grid and a 2D DEM grid"), FI_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return cuda_fail(cudaGetLastError(), "cudaSetDevice");
    Geom g = geom_of(*grid3, false);
    size_t elems = (size_t)g.sxy * g.planes;
    size_t dem_elems = (size_t)(dem_grid2->n[0] + 3) * (dem_grid2->n[1] + 3);
    DevBuf dpsi, ddem;
    if (cudaMalloc(&dpsi.p, elems * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&ddem.p, dem_elems * sizeof(double)) != cudaSuccess)
        return set_error("allocation failed"), FI_ERR_OOM;
    cudaMemset(dpsi.p, 0, elems * sizeof(double));
    if (cudaMemcpy(ddem.p, dem_host, dem_elems * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "dem upload");
    double o3[3], dx3[3], o2[2], dx2[2];
    int n2[2];
    double mx = 0.0;
    for (int q = 0; q < 3; q++) {
        o3[q] = grid3->origin[q];
        dx3[q] = grid3->extent[q] / grid3->n[q];
        mx = dx3[q] > mx ? dx3[q] : mx;
    }
    for (int q = 0; q < 2; q++) {
        o2[q] = dem_grid2->origin[q];
        dx2[q] = dem_grid2->extent[q] / dem_grid2->n[q];
        n2[q] = dem_grid2->n[q];
    }
    double cutoff = 4.0 * mx;  // compute_levelsets.jl:22
    cudaError_t e = launch_levelset(g, o3, dx3, n2, o2, dx2, dem_grid2->n[0] + 3, (const double *)ddem.p, R, R != nullptr,
                                    cutoff, invert, (double *)dpsi.p, 0);
    if (e != cudaSuccess) return cuda_fail(e, "levelset kernel");
    if (cudaMemcpy(psi_host, dpsi.p, elems * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "psi download");
    return FI_OK;
}

}  // extern "C"
