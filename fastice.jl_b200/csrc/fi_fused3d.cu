// fi_fused3d.cu -- fused single-pass 3D PT iteration (update_σ! + stress BCs +
// update_V! + velocity/η_next BCs in one kernel).
//
// Reference semantics: src/Models/FullStokes/Isothermal/Isothermal.jl:91-112
// with kernels_3d.jl:3-40 and boundary_conditions.jl.  The two reference
// kernels touch the state twice per iteration (33 array passes); this sweep
// touches it once (22 passes: P, τ(6), V(3) read + written, η read, η_next
// written) by keeping the new stresses on chip.
//
// Work decomposition.  A CTA owns a TX x TY column of grid positions (x, y) and a
// block of z planes [kb, ke).  It marches up in z: at step t it computes the new
// stresses of plane t+1 on its column widened by one position on every side
// (the ring is recomputed redundantly by neighbouring CTAs so that no grid-wide
// synchronisation is needed), applies the stress boundary conditions to that
// plane in shared memory, then updates V and η_next of plane t from the stress
// planes t-1, t, t+1 held in shared-memory plane rings.
//
// Double buffering.  Stresses and velocities are read from `in` and written to
// `out` (distinct buffers), so a CTA never sees a value another CTA already
// updated; the pointwise in-place updates of the reference are equivalent.
//
// Boundary conditions.  Stress BCs are applied per plane in the order x-faces,
// y-faces, z-faces (a face of dim d spans all positions in the dims before d and
// the field's interior in the dims after d), exactly as the CPU oracle does.
// Velocity Dirichlet values are written at the boundary nodes; ghost values
// (Velocity BC ghosts 2c - v, η_next Neumann copies, periodic images) are
// written by the thread that computes the interior value they derive from.
// Periodic dims (x, y) need no stress fix-up: the ring is computed from the
// wrapped ghosts of the previous iteration.
#include "fi_device.cuh"

namespace fi {

namespace {

constexpr int TX = 32;

struct Variant {
    int ty;
    int zb;
};
constexpr Variant kVariants[] = {{8, 32}, {8, 64}, {8, 128}, {4, 64}, {16, 32}, {8, 16}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// shared-memory plane rings: field base plane and ring length
enum { SL_P = 0, SL_ZZ = 3, SL_XX = 6, SL_YY = 8, SL_XY = 10, SL_XZ = 12, SL_YZ = 14, SL_COUNT = 16 };

template <typename T>
struct BcSide {
    int kind;
    T c[3];
};

template <typename T, int TY>
struct Ctx {
    static constexpr int RX = TX + 2;
    static constexpr int RY = TY + 2;
    static constexpr int RXY = RX * RY;
    static constexpr int NT = TX * TY;

    T *sm;
    int i0, j0, kb, ke;
    int n0, n1, n2;
    long long sx, sxy;
    bool perx, pery;
    BcSide<T> bc[3][2];

    __device__ __forceinline__ int slot(int base, int len, int s) const { return (base + s % len) * RXY; }
    __device__ __forceinline__ int rpos(int i, int j) const { return (j - j0 + 1) * RX + (i - i0 + 1); }
    __device__ __forceinline__ T &P(int s, int i, int j) const { return sm[slot(SL_P, 3, s) + rpos(i, j)]; }
    __device__ __forceinline__ T &Tzz(int s, int i, int j) const { return sm[slot(SL_ZZ, 3, s) + rpos(i, j)]; }
    __device__ __forceinline__ T &Txx(int s, int i, int j) const { return sm[slot(SL_XX, 2, s) + rpos(i, j)]; }
    __device__ __forceinline__ T &Tyy(int s, int i, int j) const { return sm[slot(SL_YY, 2, s) + rpos(i, j)]; }
    __device__ __forceinline__ T &Txy(int s, int i, int j) const { return sm[slot(SL_XY, 2, s) + rpos(i, j)]; }
    __device__ __forceinline__ T &Txz(int s, int i, int j) const { return sm[slot(SL_XZ, 2, s) + rpos(i, j)]; }
    __device__ __forceinline__ T &Tyz(int s, int i, int j) const { return sm[slot(SL_YZ, 2, s) + rpos(i, j)]; }
    __device__ __forceinline__ long long gidx(int i, int j, int k) const {
        return (long long)i + sx * (long long)j + sxy * (long long)k;
    }
    // owner of an x (y) position: tile range, plus the ghosts beyond the domain
    __device__ __forceinline__ bool own_x(int i) const {
        if (i >= 1 && i <= n0 + 1) return i >= i0 && i < i0 + TX;
        if (i == 0) return i0 == 1;
        return i == n0 + 2 && n0 + 1 < i0 + TX && n0 + 1 >= i0;
    }
    __device__ __forceinline__ bool own_y(int j) const {
        if (j >= 1 && j <= n1 + 1) return j >= j0 && j < j0 + TY;
        if (j == 0) return j0 == 1;
        return j == n1 + 2 && n1 + 1 < j0 + TY && n1 + 1 >= j0;
    }
};

template <typename T>
__device__ __forceinline__ T h(T x) { return T(0.5) * x; }

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// new stresses of plane s on the widened column, BC fix-ups, owned writes
// ---------------------------------------------------------------------------
template <typename T, int TY>
__device__ void sigma_plane(const Ctx<T, TY> &c, const KParams &p, const Ptrs<T> &in, const Ptrs<T> &out, int s) {
    using C = Ctx<T, TY>;
    const int tid = threadIdx.x;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]), idz = T(p.inv_dx[2]);
    const long long sx = c.sx, sxy = c.sxy;
    const bool cz = s >= 1 && s <= c.n2, vz = s >= 1 && s <= c.n2 + 1;
    for (int r = tid; r < C::RXY; r += C::NT) {
        const int i = c.i0 - 1 + r % C::RX, j = c.j0 - 1 + r / C::RX;
        T vP = T(0), vxx = T(0), vyy = T(0), vzz = T(0), vxy = T(0), vxz = T(0), vyz = T(0);
        if (i <= c.n0 + 2 && j <= c.n1 + 2) {
            const bool cx = (i >= 1 && i <= c.n0) || (c.perx && (i == 0 || i == c.n0 + 1));
            const bool vx = i >= 1 && i <= c.n0 + 1;
            const bool cy = (j >= 1 && j <= c.n1) || (c.pery && (j == 0 || j == c.n1 + 1));
            const bool vy = j >= 1 && j <= c.n1 + 1;
            const long long I = c.gidx(i, j, s);
            const T *Vx = in.Vx, *Vy = in.Vy, *Vz = in.Vz, *eta = in.eta;
            if (cx && cy && cz) {
                T exx = (ld(Vx + I + 1) - ld(Vx + I)) * idx;
                T eyy = (ld(Vy + I + sx) - ld(Vy + I)) * idy;
                T ezz = (ld(Vz + I + sxy) - ld(Vz + I)) * idz;
                T divV = exx + eyy + ezz;
                T etac = ld(eta + I);
                T P0 = ld(in.P + I), xx0 = ld(in.txx + I), yy0 = ld(in.tyy + I), zz0 = ld(in.tzz + I);
                vP = P0 - divV * etac * T(p.dt_P);
                vxx = xx0 - (xx0 - T(2.0) * etac * (exx - divV / T(3.0))) * T(p.dt_tau[0]);
                vyy = yy0 - (yy0 - T(2.0) * etac * (eyy - divV / T(3.0))) * T(p.dt_tau[1]);
                vzz = zz0 - (zz0 - T(2.0) * etac * (ezz - divV / T(3.0))) * T(p.dt_tau[2]);
            }
            if (vx && vy && cz) {
                T exy = T(0.5) * ((ld(Vy + I) - ld(Vy + I - 1)) * idx + (ld(Vx + I) - ld(Vx + I - sx)) * idy);
                T e_xy = h(h(ld(eta + I - 1 - sx) + ld(eta + I - sx)) + h(ld(eta + I - 1) + ld(eta + I)));
                T xy0 = ld(in.txy + I);
                vxy = xy0 - (xy0 - T(2.0) * e_xy * exy) * T(p.dt_tau[3]);
            }
            if (vx && cy && vz) {
                T exz = T(0.5) * ((ld(Vz + I) - ld(Vz + I - 1)) * idx + (ld(Vx + I) - ld(Vx + I - sxy)) * idz);
                T e_xz = h(h(ld(eta + I - 1 - sxy) + ld(eta + I - sxy)) + h(ld(eta + I - 1) + ld(eta + I)));
                T xz0 = ld(in.txz + I);
                vxz = xz0 - (xz0 - T(2.0) * e_xz * exz) * T(p.dt_tau[4]);
            }
            if (cx && vy && vz) {
                T eyz = T(0.5) * ((ld(Vz + I) - ld(Vz + I - sx)) * idy + (ld(Vy + I) - ld(Vy + I - sxy)) * idz);
                T e_yz = h(h(ld(eta + I - sx - sxy) + ld(eta + I - sxy)) + h(ld(eta + I - sx) + ld(eta + I)));
                T yz0 = ld(in.tyz + I);
                vyz = yz0 - (yz0 - T(2.0) * e_yz * eyz) * T(p.dt_tau[5]);
            }
        }
        const int rp = r;
        c.sm[c.slot(SL_P, 3, s) + rp] = vP;
        c.sm[c.slot(SL_ZZ, 3, s) + rp] = vzz;
        c.sm[c.slot(SL_XX, 2, s) + rp] = vxx;
        c.sm[c.slot(SL_YY, 2, s) + rp] = vyy;
        c.sm[c.slot(SL_XY, 2, s) + rp] = vxy;
        c.sm[c.slot(SL_XZ, 2, s) + rp] = vxz;
        c.sm[c.slot(SL_YZ, 2, s) + rp] = vyz;
    }
    __syncthreads();

    // ---- x faces (boundary_conditions.jl:51-58, 78-84): j, s in the field's interior
    const bool touch_x = (c.i0 == 1 || c.i0 + TX >= c.n0 + 1) && !c.perx;
    if (touch_x) {
        for (int r = tid; r < C::RXY; r += C::NT) {
            const int i = c.i0 - 1 + r % C::RX, j = c.j0 - 1 + r / C::RX;
            for (int side = 0; side < 2; side++) {
                const BcSide<T> &b = c.bc[0][side];
                if (b.kind != FI_BC_TRACTION && b.kind != FI_BC_SLIP) continue;
                const int ghost = side == 0 ? 0 : c.n0 + 1, adj = side == 0 ? 1 : c.n0, node = side == 0 ? 1 : c.n0 + 1;
                if (b.kind == FI_BC_TRACTION && i == ghost && j >= 1 && j <= c.n1 && cz && adj >= c.i0 - 1 &&
                    adj <= c.i0 + TX) {
                    T tv = T(2.0) * b.c[0];
                    c.P(s, i, j) = tv - c.P(s, adj, j);
                    c.Txx(s, i, j) = tv - c.Txx(s, adj, j);
                }
                if (i == node) {
                    if (j >= 1 && j <= c.n1 + 1 && cz) c.Txy(s, i, j) = b.c[1];
                    if (j >= 1 && j <= c.n1 && vz) c.Txz(s, i, j) = b.c[2];
                }
            }
        }
        __syncthreads();
    }
    // ---- y faces (boundary_conditions.jl:60-67, 86-92): all x, s in the field's interior
    const bool touch_y = (c.j0 == 1 || c.j0 + TY >= c.n1 + 1) && !c.pery;
    if (touch_y) {
        for (int r = tid; r < C::RXY; r += C::NT) {
            const int i = c.i0 - 1 + r % C::RX, j = c.j0 - 1 + r / C::RX;
            for (int side = 0; side < 2; side++) {
                const BcSide<T> &b = c.bc[1][side];
                if (b.kind != FI_BC_TRACTION && b.kind != FI_BC_SLIP) continue;
                const int ghost = side == 0 ? 0 : c.n1 + 1, adj = side == 0 ? 1 : c.n1, node = side == 0 ? 1 : c.n1 + 1;
                if (b.kind == FI_BC_TRACTION && j == ghost && cz && adj >= c.j0 - 1 && adj <= c.j0 + TY) {
                    T tv = T(2.0) * b.c[1];
                    c.P(s, i, j) = tv - c.P(s, i, adj);
                    c.Tyy(s, i, j) = tv - c.Tyy(s, i, adj);
                }
                if (j == node) {
                    if (cz) c.Txy(s, i, j) = b.c[0];
                    if (vz) c.Tyz(s, i, j) = b.c[2];
                }
            }
        }
        __syncthreads();
    }
    // ---- z faces (boundary_conditions.jl:69-76, 94-100): all x and y
    if (s == 1 || s == c.n2 + 1) {
        const int side = s == 1 ? 0 : 1;
        const BcSide<T> &b = c.bc[2][side];
        if (b.kind == FI_BC_TRACTION || b.kind == FI_BC_SLIP) {
            for (int r = tid; r < C::RXY; r += C::NT) {
                const int i = c.i0 - 1 + r % C::RX, j = c.j0 - 1 + r / C::RX;
                if (b.kind == FI_BC_TRACTION) {
                    T tv = T(2.0) * b.c[2];
                    if (side == 0) {  // ghost plane 0 from plane 1
                        c.P(0, i, j) = tv - c.P(1, i, j);
                        c.Tzz(0, i, j) = tv - c.Tzz(1, i, j);
                    } else {  // ghost plane n2+1 from plane n2
                        c.P(s, i, j) = tv - c.P(s - 1, i, j);
                        c.Tzz(s, i, j) = tv - c.Tzz(s - 1, i, j);
                    }
                }
                c.Txz(s, i, j) = b.c[0];
                c.Tyz(s, i, j) = b.c[1];
            }
            __syncthreads();
        }
    }
    // ---- owned writes (the next iteration reads these, ghosts included)
    const bool own_s = s >= c.kb && s < c.ke;
    const bool own_0 = s == 1 && c.kb == 1;
    if (own_s || own_0) {
        for (int r = tid; r < C::RXY; r += C::NT) {
            const int i = c.i0 - 1 + r % C::RX, j = c.j0 - 1 + r / C::RX;
            if (i > c.n0 + 2 || j > c.n1 + 2 || !c.own_x(i) || !c.own_y(j)) continue;
            if (own_s) {
                const long long I = c.gidx(i, j, s);
                out.P[I] = c.P(s, i, j);
                out.txx[I] = c.Txx(s, i, j);
                out.tyy[I] = c.Tyy(s, i, j);
                out.tzz[I] = c.Tzz(s, i, j);
                out.txy[I] = c.Txy(s, i, j);
                out.txz[I] = c.Txz(s, i, j);
                out.tyz[I] = c.Tyz(s, i, j);
            }
            if (own_0) {
                const long long I0 = c.gidx(i, j, 0);
                out.P[I0] = c.P(0, i, j);
                out.tzz[I0] = c.Tzz(0, i, j);
            }
        }
    }
}

// images of a value written at an interior position: per dim up to three
// (position, mode) entries; mode 0 = copy, 1 = Dirichlet ghost 2c - v
template <typename T>
struct DimImg {
    int n;
    int pos[3];
    int mode[3];
    T c[3];
    __device__ __forceinline__ void add(int ps, int md, T cv) {
        pos[n] = ps;
        mode[n] = md;
        c[n] = cv;
        n++;
    }
};

// dim image list for a Center-located value at index q (1..N) along a dim.
// vel_comp >= 0: Velocity-BC Dirichlet ghosts of that component; -1: Neumann (η)
template <typename T>
__device__ __forceinline__ DimImg<T> img_center(int q, int N, bool periodic, const BcSide<T> *bc, int vel_comp) {
    DimImg<T> d;
    d.n = 0;
    d.add(q, 0, T(0));
    if (periodic) {
        if (q == 1) d.add(N + 1, 0, T(0));
        if (q == N) d.add(0, 0, T(0));
        return d;
    }
    if (bc) {
        if (vel_comp < 0) {
            if (q == 1) d.add(0, 0, T(0));
            if (q == N) d.add(N + 1, 0, T(0));
        } else {
            if (q == 1 && bc[0].kind == FI_BC_VELOCITY) d.add(0, 1, bc[0].c[vel_comp]);
            if (q == N && bc[1].kind == FI_BC_VELOCITY) d.add(N + 1, 1, bc[1].c[vel_comp]);
        }
    }
    return d;
}

// dim image list for a Vertex-located value at index q (1..N+1)
template <typename T>
__device__ __forceinline__ DimImg<T> img_vertex(int q, int N, bool periodic) {
    DimImg<T> d;
    d.n = 0;
    d.add(q, 0, T(0));
    if (periodic) {
        if (q == 1) d.add(N + 1, 0, T(0));
        if (q == 2) d.add(N + 2, 0, T(0));
        if (q == N) d.add(0, 0, T(0));
    }
    return d;
}

template <typename T, int TY>
__device__ __forceinline__ void write_with_images(const Ctx<T, TY> &c, T *f, T v, const DimImg<T> &ix,
                                                  const DimImg<T> &iy, const DimImg<T> &iz) {
    for (int a = 0; a < ix.n; a++) {
        T va = ix.mode[a] ? T(2.0) * ix.c[a] - v : v;
        for (int b = 0; b < iy.n; b++) {
            T vb = iy.mode[b] ? T(2.0) * iy.c[b] - va : va;
            for (int e = 0; e < iz.n; e++) {
                T ve = iz.mode[e] ? T(2.0) * iz.c[e] - vb : vb;
                f[c.gidx(ix.pos[a], iy.pos[b], iz.pos[e])] = ve;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// new V and η_next of plane t on the CTA's own column
// ---------------------------------------------------------------------------
template <typename T, int TY>
__device__ void v_plane(const Ctx<T, TY> &c, const KParams &p, const Ptrs<T> &in, const Ptrs<T> &out, int t) {
    const int i = c.i0 + (threadIdx.x % TX), j = c.j0 + (threadIdx.x / TX);
    if (i > c.n0 + 1 || j > c.n1 + 1) return;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]), idz = T(p.inv_dx[2]);
    const long long I = c.gidx(i, j, t);
    const long long sx = c.sx, sxy = c.sxy;
    const T *eta = in.eta;
    const int n0 = c.n0, n1 = c.n1, n2 = c.n2;
    const BcSide<T> *bx = c.bc[0], *by = c.bc[1], *bz = c.bc[2];
    auto node_fixed = [](const BcSide<T> &b) { return b.kind == FI_BC_SLIP || b.kind == FI_BC_VELOCITY; };

    // ---- V.x at (V, C, C)
    if (j <= n1 && t >= 1 && t <= n2 && !(c.perx && i == n0 + 1)) {
        T v;
        if (!c.perx && i == 1 && node_fixed(bx[0])) v = bx[0].c[0];
        else if (!c.perx && i == n0 + 1 && node_fixed(bx[1])) v = bx[1].c[0];
        else {
            T gx = gravity_dev(p, in.gx, 0, I);
            T ex = h(ld(eta + I - 1) + ld(eta + I));
            v = ld(in.Vx + I) + div_dev(-(c.P(t, i, j) - c.P(t, i - 1, j)) * idx + (c.Txx(t, i, j) - c.Txx(t, i - 1, j)) * idx +
                                            (c.Txy(t, i, j + 1) - c.Txy(t, i, j)) * idy +
                                            (c.Txz(t + 1, i, j) - c.Txz(t, i, j)) * idz - gx,
                                        ex) *
                                    T(p.dt_V[0]);
        }
        write_with_images(c, out.Vx, v, img_vertex<T>(i, n0, c.perx),
                          img_center<T>(j, n1, c.pery, c.pery ? nullptr : by, 0),
                          img_center<T>(t, n2, false, bz, 0));
    }
    // ---- V.y at (C, V, C)
    if (i <= n0 && t >= 1 && t <= n2 && !(c.pery && j == n1 + 1)) {
        T v;
        if (!c.pery && j == 1 && node_fixed(by[0])) v = by[0].c[1];
        else if (!c.pery && j == n1 + 1 && node_fixed(by[1])) v = by[1].c[1];
        else {
            T gy = gravity_dev(p, in.gy, 1, I);
            T ey = h(ld(eta + I - sx) + ld(eta + I));
            v = ld(in.Vy + I) + div_dev(-(c.P(t, i, j) - c.P(t, i, j - 1)) * idy + (c.Tyy(t, i, j) - c.Tyy(t, i, j - 1)) * idy +
                                            (c.Txy(t, i + 1, j) - c.Txy(t, i, j)) * idx +
                                            (c.Tyz(t + 1, i, j) - c.Tyz(t, i, j)) * idz - gy,
                                        ey) *
                                    T(p.dt_V[1]);
        }
        write_with_images(c, out.Vy, v, img_center<T>(i, n0, c.perx, c.perx ? nullptr : bx, 1),
                          img_vertex<T>(j, n1, c.pery), img_center<T>(t, n2, false, bz, 1));
    }
    // ---- V.z at (C, C, V)
    if (i <= n0 && j <= n1 && t >= 1 && t <= n2 + 1) {
        T v;
        if (t == 1 && node_fixed(bz[0])) v = bz[0].c[2];
        else if (t == n2 + 1 && node_fixed(bz[1])) v = bz[1].c[2];
        else {
            T gz = gravity_dev(p, in.gz, 2, I);
            T ez = h(ld(eta + I - sxy) + ld(eta + I));
            v = ld(in.Vz + I) + div_dev(-(c.P(t, i, j) - c.P(t - 1, i, j)) * idz + (c.Tzz(t, i, j) - c.Tzz(t - 1, i, j)) * idz +
                                            (c.Txz(t, i + 1, j) - c.Txz(t, i, j)) * idx +
                                            (c.Tyz(t, i, j + 1) - c.Tyz(t, i, j)) * idy - gz,
                                        ez) *
                                    T(p.dt_V[2]);
        }
        DimImg<T> iz;
        iz.n = 0;
        iz.add(t, 0, T(0));
        write_with_images(c, out.Vz, v, img_center<T>(i, n0, c.perx, c.perx ? nullptr : bx, 2),
                          img_center<T>(j, n1, c.pery, c.pery ? nullptr : by, 2), iz);
    }
    // ---- τII and η_next at (C, C, C)
    if (i <= n0 && j <= n1 && t >= 1 && t <= n2) {
        T xx = c.Txx(t, i, j), yy = c.Tyy(t, i, j), zz = c.Tzz(t, i, j);
        T lxy = h(h(c.Txy(t, i, j) + c.Txy(t, i + 1, j)) + h(c.Txy(t, i, j + 1) + c.Txy(t, i + 1, j + 1)));
        T lxz = h(h(c.Txz(t, i, j) + c.Txz(t, i + 1, j)) + h(c.Txz(t + 1, i, j) + c.Txz(t + 1, i + 1, j)));
        T lyz = h(h(c.Tyz(t, i, j) + c.Tyz(t, i, j + 1)) + h(c.Tyz(t + 1, i, j) + c.Tyz(t + 1, i, j + 1)));
        T s2 = T(0.5) * (xx * xx + yy * yy + zz * zz) + lxy * lxy + lxz * lxz + lyz * lyz;
        T tII = sqrt_dev(s2);
        T en = rheology_dev(p, in.eta_lin, in.A, ld(eta + I), I, tII);
        write_with_images(c, out.eta_next, en, img_center<T>(i, n0, c.perx, c.perx ? nullptr : bx, -1),
                          img_center<T>(j, n1, c.pery, c.pery ? nullptr : by, -1), img_center<T>(t, n2, false, bz, -1));
    }
}

template <typename T, int TY>
__global__ void __launch_bounds__(TX *TY, (TY <= 8 ? 2 : 1)) fused3d_kernel(Geom g, KParams p, Ptrs<T> in, Ptrs<T> out,
                                                                             int zb) {
    using C = Ctx<T, TY>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C c;
    c.sm = reinterpret_cast<T *>(smem_raw);
    c.i0 = 1 + blockIdx.x * TX;
    c.j0 = 1 + blockIdx.y * TY;
    c.kb = 1 + blockIdx.z * zb;
    c.n0 = g.n[0];
    c.n1 = g.n[1];
    c.n2 = g.n[2];
    c.ke = min(c.kb + zb, c.n2 + 2);
    c.sx = g.pitch;
    c.sxy = g.sxy;
    c.perx = p.bc_kind[0][0] == FI_BC_PERIODIC;
    c.pery = p.bc_kind[1][0] == FI_BC_PERIODIC;
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++) {
            c.bc[d][s].kind = p.bc_kind[d][s];
            for (int q = 0; q < 3; q++) c.bc[d][s].c[q] = T(p.bc_val[d][s][q]);
        }
    for (int r = threadIdx.x; r < SL_COUNT * C::RXY; r += C::NT) c.sm[r] = T(0);
    __syncthreads();

    if (c.kb - 1 >= 1) sigma_plane<T, TY>(c, p, in, out, c.kb - 1);
    sigma_plane<T, TY>(c, p, in, out, c.kb);
    for (int t = c.kb; t < c.ke; t++) {
        if (t + 1 <= c.n2 + 1) sigma_plane<T, TY>(c, p, in, out, t + 1);
        __syncthreads();
        v_plane<T, TY>(c, p, in, out, t);
        __syncthreads();
    }
}

template <typename T, int TY>
cudaError_t launch_variant(const Geom &g, const KParams &p, const Ptrs<T> &in, const Ptrs<T> &out, int zb,
                           cudaStream_t s) {
    using C = Ctx<T, TY>;
    size_t shmem = (size_t)SL_COUNT * C::RXY * sizeof(T);
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(fused3d_kernel<T, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    dim3 grd((g.n[0] + 1 + TX - 1) / TX, (g.n[1] + 1 + TY - 1) / TY, (g.n[2] + 1 + zb - 1) / zb);
    fused3d_kernel<T, TY><<<grd, C::NT, shmem, s>>>(g, p, in, out, zb);
    return cudaGetLastError();
}

}  // namespace

int fused3d_num_variants() { return kNumVariants; }
const char *fused3d_variant_name(int v) {
    static char buf[kNumVariants][32];
    if (v < 0 || v >= kNumVariants) return "?";
    snprintf(buf[v], sizeof(buf[v]), "tile32x%d_zb%d", kVariants[v].ty, kVariants[v].zb);
    return buf[v];
}

template <typename T>
bool fused3d_supported(const Geom &g, const KParams &p, bool ib) {
    if (g.nd != 3 || ib) return false;
    if (p.bc_kind[2][0] == FI_BC_PERIODIC) return false;
    return true;
}

template <typename T>
cudaError_t launch_fused3d(const Geom &g, const KParams &p, const Ptrs<T> &in, const Ptrs<T> &out, bool ib, int variant,
                           cudaStream_t s) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant v = kVariants[variant];
    switch (v.ty) {
        case 4: return launch_variant<T, 4>(g, p, in, out, v.zb, s);
        case 16: return launch_variant<T, 16>(g, p, in, out, v.zb, s);
        default: return launch_variant<T, 8>(g, p, in, out, v.zb, s);
    }
}

template bool fused3d_supported<double>(const Geom &, const KParams &, bool);
template bool fused3d_supported<float>(const Geom &, const KParams &, bool);
template cudaError_t launch_fused3d<double>(const Geom &, const KParams &, const Ptrs<double> &, const Ptrs<double> &,
                                            bool, int, cudaStream_t);
template cudaError_t launch_fused3d<float>(const Geom &, const KParams &, const Ptrs<float> &, const Ptrs<float> &,
                                           bool, int, cudaStream_t);

}  // namespace fi
