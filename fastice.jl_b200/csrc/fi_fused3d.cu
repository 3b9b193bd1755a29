// fi_fused3d.cu -- fused single-pass 3D PT iteration (update_σ! + stress BCs +
// update_V! + velocity/η_next BCs in one kernel), TMA-staged.
//
// Reference semantics: src/Models/FullStokes/Isothermal/Isothermal.jl:91-112
// with kernels_3d.jl:3-40 and boundary_conditions.jl.  The two reference
// kernels touch the state twice per iteration (33 array passes); this sweep
// reads P, τ(6), V(3), η once and writes P, τ(6), V(3), η_next once (22 passes).
//
// Work decomposition.  A CTA owns a TX x TY column of grid positions (x, y) and a
// block of z planes (TX = 32 or 64: one or two x positions per thread, 32·TY
// threads).  It marches up in z.  For every plane s the tensor-memory
// accelerator copies an (x, y) box of each of the eleven input fields (old P, τ,
// V, η; V.z one plane higher) into shared-memory plane rings, one plane ahead of
// the compute, signalled by an mbarrier.  The new stresses of plane s are
// computed in place over the column (all seven components) and over a
// one-position ring (only the components the velocity update reads there), the
// stress boundary conditions are applied to the plane in shared memory, and V /
// η_next of plane s-1 are updated from the stress planes s-2, s-1, s.
// Neighbouring CTAs recompute each other's ring: no grid-wide synchronisation.
//
// Boxes.  A CTA whose column touches an x or y boundary loads every field over the
// column plus the whole one-position ring (the boundary fix-ups and ghost writes
// reach all of it).  An interior CTA of a "trimmed" launch shape loads each
// stress component only where the sweep reads it: the ring stresses the velocity
// update needs are P and τxx left of the column, P and τyy below it, τxy and τxz
// right of it, τxy and τyz above it (and τxy at the upper right corner); τzz needs
// no ring at all.  V and η keep the full ring.  This cuts the DRAM sectors an
// interior column reads per plane by about a sixth (the ring is re-read by the
// neighbouring columns).
//
// Clusters.  A launch shape may group CTAs into thread-block clusters (2x2, ...)
// purely for co-scheduling: cluster members start together on one GPC and march
// through z at the same pace, so the ring rows one member reads are the rows its
// neighbour reads at about the same time and the second read hits L2.  There is no
// cross-CTA communication and no multicast; a CTA may leave the cluster at any time.
//
// Double buffering.  Stresses and velocities are read from `in` and written to
// `out` (distinct buffers), so the pointwise in-place updates of the reference
// are reproduced exactly.  With a no-FMA build the sweep matches the CPU oracle
// bit for bit.
//
// Boundary conditions.  Stress BCs are applied per plane in the order x-faces,
// y-faces, z-faces (a face of dim d spans all positions in the dims before d and
// the field's interior in the dims after d), as the CPU oracle does.  Velocity
// Dirichlet values are written at the boundary nodes; ghost values (Velocity BC
// ghosts 2c - v, η_next Neumann copies, periodic images) are written by the
// thread that computes the interior value they derive from.  Periodic x / y need
// no stress fix-up: ghost-ring stresses follow from the wrapped ghosts of the
// previous iteration.
//
// Waits.  Every mbarrier wait is bounded (about one second of SM clock); on
// expiry the CTA records FI_ERR_TIMEOUT in the model's error word, waits once
// more (bounded) for its own copies in flight, and returns.
#include <cuda.h>

// Layout and box constants of shapes a precision does not launch are still instantiated by
// the host-side box tables: their unreferenced members are expected.
#pragma nv_diag_suppress 177
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstdlib>

#include "fi_device.cuh"
#include "fi_tma.cuh"

namespace fi {

namespace {

// Launch shapes: tile width and height, z-block depth, cluster shape (x, y) and
// whether interior tiles load trimmed stress boxes.  (Issuing the copies of plane
// s+1 after the stress barrier of step s instead, which saves the barrier closing
// each step, measured 15-20 % slower at 511^3: the copies then lose half their
// lead.  Z-blocks of 16 and 24 planes on 32x8 tiles measured 3 % slower and equal
// to 32 planes at 511^3 in both precisions: shorter blocks refill their rings
// more often.)  Shapes whose shared memory does not fit a CTA for a precision
// are not offered for it.
struct Variant {
    int tx, ty, zb, cx, cy, trim;
};
// Measured at 511^3 (CUDA events, 30 iterations per shape, one box): the 32x8 tiles
// with z-blocks of 32 lead in both precisions; trimmed interior boxes (5.23 against
// 5.09 ms in FP64), clusters (5.39-5.90 ms) and 64-wide FP32 tiles (4.51-9.5 against
// 3.40 ms) are slower, and their DRAM reads per cell at 255^3 are within 5 % of the
// plain shape's (the ring sectors they save were L2 hits already).  They stay in the
// table so that the autotuner re-checks them on every device.
constexpr Variant kVariants[] = {
    {32, 8, 32, 1, 1, 0},  {32, 8, 64, 1, 1, 0},  {32, 8, 128, 1, 1, 0}, {32, 4, 64, 1, 1, 0},
    {32, 16, 32, 1, 1, 0}, {32, 16, 64, 1, 1, 0}, {32, 16, 128, 1, 1, 0},
    // trimmed interior boxes, clusters
    {32, 8, 32, 1, 1, 1},  {32, 8, 32, 1, 4, 1},  {32, 8, 32, 2, 2, 0},
    // 64-wide tiles (two x positions per thread; FP32 only)
    {64, 8, 32, 1, 1, 0},  {64, 8, 32, 1, 1, 1}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// input fields in map order
enum { M_P = 0, M_XX, M_YY, M_ZZ, M_XY, M_XZ, M_YZ, M_VX, M_VY, M_VZ, M_ET, M_COUNT };
constexpr int kTrimmed = 7;  // fields with a trimmed box (the stresses)

// shared-memory plane slots: ring base and length per field
enum {
    S_P = 0, R_P = 4,
    S_ZZ = 4, R_ZZ = 4,
    S_XX = 8, R_XX = 3,
    S_YY = 11, R_YY = 3,
    S_XY = 14, R_XY = 3,
    S_XZ = 17, R_XZ = 3,
    S_YZ = 20, R_YZ = 3,
    S_VX = 23, R_VX = 3,
    S_VY = 26, R_VY = 3,
    S_VZ = 29, R_VZ = 4,
    S_ET = 33, R_ET = 4,
    S_COUNT = 37
};
constexpr int kBars = 3;
constexpr int kSmemPerSM = 233472;  // bytes of shared memory per SM (228 KB)

template <typename T, int TX, int TY>
struct Layout {
    // the box starts XB positions left of the column so that its global x
    // coordinate times the element size is a multiple of 16 bytes
    static constexpr int XB = 16 / (int)sizeof(T);
    static constexpr int BX = ((TX + 1 + XB + XB - 1) / XB) * XB;  // full box width (column + ring, aligned)
    static constexpr int RY = TY + 2;
    static constexpr int PLANE = BX * RY;  // elements in one full box
    static constexpr int PLANE_BYTES = PLANE * (int)sizeof(T);
    static constexpr int SLOT = ((PLANE_BYTES + 127) / 128) * 128 / (int)sizeof(T);  // 128-byte aligned slots
    static constexpr int NT = 32 * TY;
    static constexpr int PX = TX / 32;  // x positions per thread
    static constexpr size_t SMEM = (size_t)S_COUNT * SLOT * sizeof(T) + 128;
    static constexpr int MINB_RAW = kSmemPerSM / (int)(SMEM + 1024);
    static constexpr int MINB = MINB_RAW < 1 ? 1 : (MINB_RAW > 4 ? 4 : MINB_RAW);
};

// Box of input field F relative to the column origin (i0, j0): x from i0 + ox,
// width bw; y from j0 + oy, height bh.  Full boxes cover the ring on all sides;
// trimmed boxes (stresses of interior CTAs) only the ring sides read there.
template <typename T, int TX, int TY, bool TRIM, int F>
struct FBox {
    using L = Layout<T, TX, TY>;
    static constexpr bool full = !TRIM || F >= kTrimmed;
    static constexpr int ox = full ? -L::XB : ((F == M_P || F == M_XX) ? -L::XB : 0);
    static constexpr int bw = full ? L::BX : ((F == M_ZZ || F == M_YY || F == M_YZ) ? TX : TX + L::XB);
    static constexpr int oy = full ? -1 : ((F == M_P || F == M_YY) ? -1 : 0);
    static constexpr int bh = full ? TY + 2 : ((F == M_XX || F == M_ZZ || F == M_XZ) ? TY : TY + 1);
    static constexpr int bytes = bw * bh * (int)sizeof(T);
    static_assert(bw * bh <= L::SLOT, "box fits its slot");
    static_assert((bw * (int)sizeof(T)) % 16 == 0, "TMA box rows are whole 16-byte units");
};

// the input maps of one sweep: eleven full-box maps in map order, then the trimmed
// maps of the seven stress fields (used by interior CTAs of trimmed shapes)
struct InMaps {
    CUtensorMap m[M_COUNT];
    CUtensorMap t[kTrimmed];
};

template <typename T, int TX, int TY, bool TRIM>
struct Ctx {
    using Lay = Layout<T, TX, TY>;
    T *sm;
    int i0, j0, kb, ke;
    int n0, n1, n2;
    long long sx, sxy;
    // the ghost layer on the low / high side of x / y comes from elsewhere: a periodic
    // image, or a neighbouring subdomain's halo (FI_BC_PERIODIC / FI_BC_HALO)
    bool hx0, hx1, hy0, hy1;
    bool bnd_x, bnd_y;  // column touches an x / y boundary (needs fix-ups or ghost writes)
    // Ring positions relative to the plane step sref: element offsets of the
    // planes around sref inside three- and four-slot rings, computed once per plane
    // step.  Every access names its plane as sref plus a constant, so after
    // inlining the choice folds to one register (no modulo per access).
    int sref;
    int o3m, o30, o3p;                 // three-slot rings: planes sref-1, sref, sref+1
    int o4m2, o4m, o40, o4p, o4p2;     // four-slot rings: planes sref-2 .. sref+2

    __device__ __forceinline__ void set_plane(int s) {
        sref = s;
        const int m3 = s % 3, m4 = s & 3;
        o30 = m3 * Lay::SLOT;
        o3p = (m3 == 2 ? 0 : m3 + 1) * Lay::SLOT;
        o3m = (m3 == 0 ? 2 : m3 - 1) * Lay::SLOT;
        o4m2 = ((m4 + 2) & 3) * Lay::SLOT;
        o4m = ((m4 + 3) & 3) * Lay::SLOT;
        o40 = m4 * Lay::SLOT;
        o4p = ((m4 + 1) & 3) * Lay::SLOT;
        o4p2 = o4m2;
    }
    // element index of (i, j) inside field F's box
    template <int F>
    __device__ __forceinline__ int ix(int i, int j) const {
        using B = FBox<T, TX, TY, TRIM, F>;
        return (j - j0 - B::oy) * B::bw + (i - i0 - B::ox);
    }
    template <int F>
    __device__ __forceinline__ bool in_box(int i, int j) const {
        using B = FBox<T, TX, TY, TRIM, F>;
        const int a = i - i0 - B::ox, b = j - j0 - B::oy;
        return a >= 0 && a < B::bw && b >= 0 && b < B::bh;
    }
    __device__ __forceinline__ T *slot(int base, int len, int p) const {
        const int d = p - sref;
        const int off = len == 3 ? (d < 0 ? o3m : d == 0 ? o30 : o3p)
                                 : (d < -1 ? o4m2 : d == -1 ? o4m : d == 0 ? o40 : d == 1 ? o4p : o4p2);
        return sm + base * Lay::SLOT + off;
    }
    __device__ __forceinline__ T &P(int p, int i, int j) const { return slot(S_P, R_P, p)[ix<M_P>(i, j)]; }
    __device__ __forceinline__ T &Tzz(int p, int i, int j) const { return slot(S_ZZ, R_ZZ, p)[ix<M_ZZ>(i, j)]; }
    __device__ __forceinline__ T &Txx(int p, int i, int j) const { return slot(S_XX, R_XX, p)[ix<M_XX>(i, j)]; }
    __device__ __forceinline__ T &Tyy(int p, int i, int j) const { return slot(S_YY, R_YY, p)[ix<M_YY>(i, j)]; }
    __device__ __forceinline__ T &Txy(int p, int i, int j) const { return slot(S_XY, R_XY, p)[ix<M_XY>(i, j)]; }
    __device__ __forceinline__ T &Txz(int p, int i, int j) const { return slot(S_XZ, R_XZ, p)[ix<M_XZ>(i, j)]; }
    __device__ __forceinline__ T &Tyz(int p, int i, int j) const { return slot(S_YZ, R_YZ, p)[ix<M_YZ>(i, j)]; }
    __device__ __forceinline__ T Vx(int p, int i, int j) const { return slot(S_VX, R_VX, p)[ix<M_VX>(i, j)]; }
    __device__ __forceinline__ T Vy(int p, int i, int j) const { return slot(S_VY, R_VY, p)[ix<M_VY>(i, j)]; }
    __device__ __forceinline__ T Vz(int p, int i, int j) const { return slot(S_VZ, R_VZ, p)[ix<M_VZ>(i, j)]; }
    __device__ __forceinline__ T Eta(int p, int i, int j) const { return slot(S_ET, R_ET, p)[ix<M_ET>(i, j)]; }
    __device__ __forceinline__ long long gidx(int i, int j, int k) const {
        return (long long)i + sx * (long long)j + sxy * (long long)k;
    }
    __device__ __forceinline__ bool own_x(int i) const {
        if (i >= 1 && i <= n0 + 1) return i >= i0 && i < i0 + TX;
        if (i == 0) return i0 == 1;
        return i == n0 + 2 && n0 + 1 < i0 + TX;
    }
    __device__ __forceinline__ bool own_y(int j) const {
        if (j >= 1 && j <= n1 + 1) return j >= j0 && j < j0 + TY;
        if (j == 0) return j0 == 1;
        return j == n1 + 2 && n1 + 1 < j0 + TY;
    }
};

template <typename T>
__device__ __forceinline__ T h(T x) { return T(0.5) * x; }

// one box copy of field F of plane p into its ring slot
template <int F, typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void load_box(const Ctx<T, TX, TY, TRIM> &c, const InMaps &mp, T *dst, int p, uint64_t *bar) {
    using B = FBox<T, TX, TY, TRIM, F>;
    const CUtensorMap *map = (TRIM && F < kTrimmed) ? &mp.t[F] : &mp.m[F];
    tma_load_3d(dst, map, (int)kXOff + c.i0 + B::ox, c.j0 + B::oy, p, bar);
}

// issue the TMA copies of input group p (planes: σ_old(p), Vx(p), Vy(p), Vz(p+1), η(p))
template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void issue_group(const Ctx<T, TX, TY, TRIM> &c, const InMaps &mp, int p, bool full,
                                            uint64_t *bar) {
    constexpr uint32_t vbytes = FBox<T, TX, TY, TRIM, M_VX>::bytes + FBox<T, TX, TY, TRIM, M_VY>::bytes +
                                FBox<T, TX, TY, TRIM, M_VZ>::bytes + FBox<T, TX, TY, TRIM, M_ET>::bytes;
    constexpr uint32_t sbytes = FBox<T, TX, TY, TRIM, M_P>::bytes + FBox<T, TX, TY, TRIM, M_XX>::bytes +
                                FBox<T, TX, TY, TRIM, M_YY>::bytes + FBox<T, TX, TY, TRIM, M_ZZ>::bytes +
                                FBox<T, TX, TY, TRIM, M_XY>::bytes + FBox<T, TX, TY, TRIM, M_XZ>::bytes +
                                FBox<T, TX, TY, TRIM, M_YZ>::bytes;
    mbar_expect_tx(bar, full ? vbytes + sbytes : vbytes);
    if (full) {
        load_box<M_P>(c, mp, c.slot(S_P, R_P, p), p, bar);
        load_box<M_XX>(c, mp, c.slot(S_XX, R_XX, p), p, bar);
        load_box<M_YY>(c, mp, c.slot(S_YY, R_YY, p), p, bar);
        load_box<M_ZZ>(c, mp, c.slot(S_ZZ, R_ZZ, p), p, bar);
        load_box<M_XY>(c, mp, c.slot(S_XY, R_XY, p), p, bar);
        load_box<M_XZ>(c, mp, c.slot(S_XZ, R_XZ, p), p, bar);
        load_box<M_YZ>(c, mp, c.slot(S_YZ, R_YZ, p), p, bar);
    }
    load_box<M_VX>(c, mp, c.slot(S_VX, R_VX, p), p, bar);
    load_box<M_VY>(c, mp, c.slot(S_VY, R_VY, p), p, bar);
    load_box<M_VZ>(c, mp, c.slot(S_VZ, R_VZ, p + 1), p + 1, bar);
    load_box<M_ET>(c, mp, c.slot(S_ET, R_ET, p), p, bar);
}

// raw stress update of plane s at (i, j): which components is a compile-time mask.
// Every shared-memory operand is loaded before the first store (the in-place stress
// stores and the global writes go through pointers the compiler cannot separate from
// the loads), so the seven updates form independent chains.  A component outside the
// mask is neither loaded nor stored (a trimmed box may not hold it at (i, j)).
enum { F_P = 1, F_XX = 2, F_YY = 4, F_ZZ = 8, F_XY = 16, F_XZ = 32, F_YZ = 64, F_ALL = 127 };

// XYI: the column and its ring lie inside every x / y range (no boundary column),
// so only the z ranges are tested
template <typename T, int TX, int TY, bool TRIM, bool XYI>
__device__ __forceinline__ void sigma_point(const Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q, int s,
                                            int i, int j, int mask, bool write_now, const Ptrs<T> &out) {
    if (!XYI && (i > c.n0 + 2 || j > c.n1 + 2)) return;
    using Cx = Ctx<T, TX, TY, TRIM>;
    constexpr int BV = FBox<T, TX, TY, TRIM, M_VX>::bw;  // row pitch of the V and η boxes
    const T idx = q.inv_dx[0], idy = q.inv_dx[1], idz = q.inv_dx[2];
    const bool cz = s >= 1 && s <= c.n2, vz = s >= 1 && s <= c.n2 + 1;
    const bool cx = XYI || (i >= 1 && i <= c.n0) || (c.hx0 && i == 0) || (c.hx1 && i == c.n0 + 1);
    const bool vx = XYI || (i >= 1 && i <= c.n0 + 1);
    const bool cy = XYI || (j >= 1 && j <= c.n1) || (c.hy0 && j == 0) || (c.hy1 && j == c.n1 + 1);
    const bool vy = XYI || (j >= 1 && j <= c.n1 + 1);
    const int a = c.template ix<M_VX>(i, j);
    const T *vxs = c.slot(S_VX, R_VX, s), *vys = c.slot(S_VY, R_VY, s), *vzs = c.slot(S_VZ, R_VZ, s);
    const T *vxm = c.slot(S_VX, R_VX, s - 1), *vym = c.slot(S_VY, R_VY, s - 1), *vzp = c.slot(S_VZ, R_VZ, s + 1);
    const T *et = c.slot(S_ET, R_ET, s), *etm = c.slot(S_ET, R_ET, s - 1);
    T *sP = c.slot(S_P, R_P, s) + c.template ix<M_P>(i, j);
    T *sXX = c.slot(S_XX, R_XX, s) + c.template ix<M_XX>(i, j);
    T *sYY = c.slot(S_YY, R_YY, s) + c.template ix<M_YY>(i, j);
    T *sZZ = c.slot(S_ZZ, R_ZZ, s) + c.template ix<M_ZZ>(i, j);
    T *sXY = c.slot(S_XY, R_XY, s) + c.template ix<M_XY>(i, j);
    T *sXZ = c.slot(S_XZ, R_XZ, s) + c.template ix<M_XZ>(i, j);
    T *sYZ = c.slot(S_YZ, R_YZ, s) + c.template ix<M_YZ>(i, j);
    (void)sizeof(Cx);
    const bool dc = (mask & (F_P | F_XX | F_YY | F_ZZ)) && cx && cy && cz;
    const bool dxy = (mask & F_XY) && vx && vy && cz;
    const bool dxz = (mask & F_XZ) && vx && cy && vz;
    const bool dyz = (mask & F_YZ) && cx && vy && vz;
    // old values (all seven when the point is written out)
    const int lmask = write_now ? F_ALL : mask;
    T oP = T(0), oXX = T(0), oYY = T(0), oZZ = T(0), oXY = T(0), oXZ = T(0), oYZ = T(0);
    if (lmask & F_P) oP = *sP;
    if (lmask & F_XX) oXX = *sXX;
    if (lmask & F_YY) oYY = *sYY;
    if (lmask & F_ZZ) oZZ = *sZZ;
    if (lmask & F_XY) oXY = *sXY;
    if (lmask & F_XZ) oXZ = *sXZ;
    if (lmask & F_YZ) oYZ = *sYZ;
    T nP = oP, nXX = oXX, nYY = oYY, nZZ = oZZ, nXY = oXY, nXZ = oXZ, nYZ = oYZ;
    if (dc) {
        T exx = (vxs[a + 1] - vxs[a]) * idx;
        T eyy = (vys[a + BV] - vys[a]) * idy;
        T ezz = (vzp[a] - vzs[a]) * idz;
        T divV = exx + eyy + ezz;
        T etac = et[a];
        if (mask & F_P) nP = oP - (p.p_forcing ? divV + __ldg(out.fP + c.gidx(i, j, s)) : divV) * etac * q.dt_P;
        if (mask & F_XX) nXX = oXX - (oXX - T(2.0) * etac * (exx - third(divV))) * q.dt_tau[0];
        if (mask & F_YY) nYY = oYY - (oYY - T(2.0) * etac * (eyy - third(divV))) * q.dt_tau[1];
        if (mask & F_ZZ) nZZ = oZZ - (oZZ - T(2.0) * etac * (ezz - third(divV))) * q.dt_tau[2];
    }
    if (dxy) {
        T exy = T(0.5) * ((vys[a] - vys[a - 1]) * idx + (vxs[a] - vxs[a - BV]) * idy);
        T e_xy = h(h(et[a - 1 - BV] + et[a - BV]) + h(et[a - 1] + et[a]));
        nXY = oXY - (oXY - T(2.0) * e_xy * exy) * q.dt_tau[3];
    }
    if (dxz) {
        T exz = T(0.5) * ((vzs[a] - vzs[a - 1]) * idx + (vxs[a] - vxm[a]) * idz);
        T e_xz = h(h(etm[a - 1] + etm[a]) + h(et[a - 1] + et[a]));
        nXZ = oXZ - (oXZ - T(2.0) * e_xz * exz) * q.dt_tau[4];
    }
    if (dyz) {
        T eyz = T(0.5) * ((vzs[a] - vzs[a - BV]) * idy + (vys[a] - vym[a]) * idz);
        T e_yz = h(h(etm[a - BV] + etm[a]) + h(et[a - BV] + et[a]));
        nYZ = oYZ - (oYZ - T(2.0) * e_yz * eyz) * q.dt_tau[5];
    }
    if (dc) {
        if (mask & F_P) *sP = nP;
        if (mask & F_XX) *sXX = nXX;
        if (mask & F_YY) *sYY = nYY;
        if (mask & F_ZZ) *sZZ = nZZ;
    }
    if (dxy) *sXY = nXY;
    if (dxz) *sXZ = nXZ;
    if (dyz) *sYZ = nYZ;
    if (write_now) {
        const long long I = c.gidx(i, j, s);
        out.P[I] = nP;
        out.txx[I] = nXX;
        out.tyy[I] = nYY;
        out.tzz[I] = nZZ;
        out.txy[I] = nXY;
        out.txz[I] = nXZ;
        out.tyz[I] = nYZ;
    }
}

// ring stresses of plane s (see sigma_plane); a warp spans a row of 32 positions
// (TX / 32 per lane), TY < 32
template <typename T, int TX, int TY, bool TRIM, bool XYI>
__device__ __forceinline__ void sigma_ring(const Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q, int s,
                                           const Ptrs<T> &out) {
    constexpr int NW = Layout<T, TX, TY>::NT / 32;
    constexpr int PX = TX / 32;
    static_assert(TY < 32 && NW >= 4, "one ring side per warp");
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (w == NW - 4) {
#pragma unroll
        for (int u = 0; u < PX; u++)
            sigma_point<T, TX, TY, TRIM, XYI>(c, p, q, s, c.i0 + lane + 32 * u, c.j0 - 1, F_P | F_YY, false, out);
    } else if (w == NW - 3) {
#pragma unroll
        for (int u = 0; u < PX; u++)
            sigma_point<T, TX, TY, TRIM, XYI>(c, p, q, s, c.i0 + lane + 32 * u, c.j0 + TY, F_XY | F_YZ, false, out);
    } else if (w == NW - 2) {
        if (lane < TY) sigma_point<T, TX, TY, TRIM, XYI>(c, p, q, s, c.i0 - 1, c.j0 + lane, F_P | F_XX, false, out);
    } else if (w == NW - 1) {
        if (lane < TY) sigma_point<T, TX, TY, TRIM, XYI>(c, p, q, s, c.i0 + TX, c.j0 + lane, F_XY | F_XZ, false, out);
        else if (lane == TY) sigma_point<T, TX, TY, TRIM, XYI>(c, p, q, s, c.i0 + TX, c.j0 + TY, F_XY, false, out);
    }
}

// stress boundary fix-ups of one face side on plane s at region point (i, j)
// (boundary columns only: full boxes)
template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void fix_x(const Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q, int s, int i,
                                      int j, int side) {
    const int kind = p.bc_kind[0][side];
    if (kind != FI_BC_TRACTION && kind != FI_BC_SLIP) return;
    const bool cz = s >= 1 && s <= c.n2, vz = s >= 1 && s <= c.n2 + 1;
    const int ghost = side == 0 ? 0 : c.n0 + 1, adj = side == 0 ? 1 : c.n0, node = side == 0 ? 1 : c.n0 + 1;
    if (kind == FI_BC_TRACTION && i == ghost && j >= 1 && j <= c.n1 && cz && adj >= c.i0 - 1 && adj <= c.i0 + TX) {
        T tv = T(2.0) * q.bc_val[0][side][0];
        c.P(s, i, j) = tv - c.P(s, adj, j);
        c.Txx(s, i, j) = tv - c.Txx(s, adj, j);
    }
    if (i == node) {
        if (j >= 1 && j <= c.n1 + 1 && cz) c.Txy(s, i, j) = q.bc_val[0][side][1];
        if (j >= 1 && j <= c.n1 && vz) c.Txz(s, i, j) = q.bc_val[0][side][2];
    }
}
template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void fix_y(const Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q, int s, int i,
                                      int j, int side) {
    const int kind = p.bc_kind[1][side];
    if (kind != FI_BC_TRACTION && kind != FI_BC_SLIP) return;
    const bool cz = s >= 1 && s <= c.n2, vz = s >= 1 && s <= c.n2 + 1;
    const int ghost = side == 0 ? 0 : c.n1 + 1, adj = side == 0 ? 1 : c.n1, node = side == 0 ? 1 : c.n1 + 1;
    if (kind == FI_BC_TRACTION && j == ghost && cz && adj >= c.j0 - 1 && adj <= c.j0 + TY) {
        T tv = T(2.0) * q.bc_val[1][side][1];
        c.P(s, i, j) = tv - c.P(s, i, adj);
        c.Tyy(s, i, j) = tv - c.Tyy(s, i, adj);
    }
    if (j == node) {
        if (cz) c.Txy(s, i, j) = q.bc_val[1][side][0];
        if (vz) c.Tyz(s, i, j) = q.bc_val[1][side][2];
    }
}

template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void sigma_plane(const Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q,
                                            const Ptrs<T> &out, int s) {
    using Lay = Layout<T, TX, TY>;
    using Cx = Ctx<T, TX, TY, TRIM>;
    constexpr int PX = Lay::PX;
    const int tid = threadIdx.x, lane = tid % 32, row = tid / 32;
    const bool zb_plane = s == 1 || s == c.n2 + 1;
    const bool late = c.bnd_x || c.bnd_y || zb_plane;
    const bool own_s = s >= c.kb && s < c.ke;
    // pass 1: the column, all components; pass 2: the ring, only the components read
    // there, one ring side per warp on the last four warps (one per scheduler), so
    // that every ring warp takes a single branch path: the row below (P, τyy), the
    // row above (τxy, τyz), the column left (P, τxx), the column right (τxy, τxz)
    // with the corner above it (τxy)
    if (TRIM || (!c.bnd_x && !c.bnd_y)) {
#pragma unroll
        for (int u = 0; u < PX; u++)
            sigma_point<T, TX, TY, TRIM, true>(c, p, q, s, c.i0 + lane + 32 * u, c.j0 + row, F_ALL, own_s && !late, out);
        sigma_ring<T, TX, TY, TRIM, true>(c, p, q, s, out);
    } else {
#pragma unroll
        for (int u = 0; u < PX; u++)
            sigma_point<T, TX, TY, TRIM, false>(c, p, q, s, c.i0 + lane + 32 * u, c.j0 + row, F_ALL, own_s && !late,
                                                out);
        sigma_ring<T, TX, TY, TRIM, false>(c, p, q, s, out);
    }
    __syncthreads();
    if (!late) return;
    constexpr int NREG = (TX + 2) * (TY + 2);
    if constexpr (!TRIM) {
        if (c.bnd_x && !(c.hx0 && c.hx1)) {  // fix_x leaves periodic and halo sides alone
            for (int r = tid; r < NREG; r += Lay::NT) {
                const int i = c.i0 - 1 + r % (TX + 2), j = c.j0 - 1 + r / (TX + 2);
                fix_x<T, TX, TY, TRIM>(c, p, q, s, i, j, 0);
                fix_x<T, TX, TY, TRIM>(c, p, q, s, i, j, 1);
            }
            __syncthreads();
        }
        if (c.bnd_y && !(c.hy0 && c.hy1)) {
            for (int r = tid; r < NREG; r += Lay::NT) {
                const int i = c.i0 - 1 + r % (TX + 2), j = c.j0 - 1 + r / (TX + 2);
                fix_y<T, TX, TY, TRIM>(c, p, q, s, i, j, 0);
                fix_y<T, TX, TY, TRIM>(c, p, q, s, i, j, 1);
            }
            __syncthreads();
        }
    }
    if (zb_plane) {
        const int side = s == 1 ? 0 : 1;
        const int kind = p.bc_kind[2][side];
        if (kind == FI_BC_TRACTION || kind == FI_BC_SLIP) {
            const T c0 = q.bc_val[2][side][0], c1 = q.bc_val[2][side][1], tv = T(2.0) * q.bc_val[2][side][2];
            for (int r = tid; r < NREG; r += Lay::NT) {
                const int i = c.i0 - 1 + r % (TX + 2), j = c.j0 - 1 + r / (TX + 2);
                // a trimmed box holds a component only where the sweep reads it
                if (kind == FI_BC_TRACTION) {
                    if (side == 0) {  // s == 1: ghost plane 0 from plane 1
                        if (c.template in_box<M_P>(i, j)) c.P(s - 1, i, j) = tv - c.P(s, i, j);
                        if (c.template in_box<M_ZZ>(i, j)) c.Tzz(s - 1, i, j) = tv - c.Tzz(s, i, j);
                    } else {
                        if (c.template in_box<M_P>(i, j)) c.P(s, i, j) = tv - c.P(s - 1, i, j);
                        if (c.template in_box<M_ZZ>(i, j)) c.Tzz(s, i, j) = tv - c.Tzz(s - 1, i, j);
                    }
                }
                if (c.template in_box<M_XZ>(i, j)) c.Txz(s, i, j) = c0;
                if (c.template in_box<M_YZ>(i, j)) c.Tyz(s, i, j) = c1;
            }
            __syncthreads();
        }
    }
    (void)sizeof(Cx);
    const bool own_0 = s == 1 && c.kb == 1 && p.bc_kind[2][0] == FI_BC_TRACTION;
    if (own_s || own_0) {
        for (int r = tid; r < NREG; r += Lay::NT) {
            const int i = c.i0 - 1 + r % (TX + 2), j = c.j0 - 1 + r / (TX + 2);
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
                out.P[I0] = c.P(s - 1, i, j);  // own_0: s == 1, ghost plane 0
                out.tzz[I0] = c.Tzz(s - 1, i, j);
            }
        }
    }
    // the V update of the same step reads the fixed-up plane
    __syncthreads();
}

// ---- ghost / image writes: per dim a fixed three-entry list (own, low, high) ----
template <typename T>
struct Img {
    int pos[3];
    bool ok[3];
    bool dir[3];  // Dirichlet ghost 2c - v (else copy)
    T c[3];
};

template <typename T>
__device__ __forceinline__ Img<T> img_own(int q) {
    Img<T> d;
    d.pos[0] = q; d.ok[0] = true; d.dir[0] = false; d.c[0] = T(0);
    d.pos[1] = 0; d.ok[1] = false; d.dir[1] = false; d.c[1] = T(0);
    d.pos[2] = 0; d.ok[2] = false; d.dir[2] = false; d.c[2] = T(0);
    return d;
}
// Center-located value at index q (1..N) along a dim with BC kinds kl/kr; lo / hi:
// the low / high ghost comes from elsewhere (a periodic image of this model's own
// value, which a subdomain's halo exchange replaces with its neighbour's).
// neumann: copies (η_next); else Velocity-BC ghosts 2c - v of a velocity component
template <typename T>
__device__ __forceinline__ Img<T> img_center(int q, int N, bool lo, bool hi, int kl, int kr, T cl, T cr, bool neumann) {
    Img<T> d = img_own<T>(q);
    if (lo) {
        if (q == N) { d.pos[1] = 0; d.ok[1] = true; }
    } else if (neumann) {
        if (q == 1) { d.pos[1] = 0; d.ok[1] = true; }
    } else if (q == 1 && kl == FI_BC_VELOCITY) {
        d.pos[1] = 0; d.ok[1] = true; d.dir[1] = true; d.c[1] = cl;
    }
    if (hi) {
        if (q == 1) { d.pos[2] = N + 1; d.ok[2] = true; }
    } else if (neumann) {
        if (q == N) { d.pos[2] = N + 1; d.ok[2] = true; }
    } else if (q == N && kr == FI_BC_VELOCITY) {
        d.pos[2] = N + 1; d.ok[2] = true; d.dir[2] = true; d.c[2] = cr;
    }
    return d;
}
template <typename T>
__device__ __forceinline__ Img<T> img_vertex(int q, int N, bool lo, bool hi) {
    Img<T> d = img_own<T>(q);
    if (lo && q == N) { d.pos[1] = 0; d.ok[1] = true; }
    if (hi && q == 1) { d.pos[2] = N + 1; d.ok[2] = true; }
    if (hi && q == 2) { d.pos[2] = N + 2; d.ok[2] = true; }
    return d;
}

template <typename T, typename C>
__device__ __forceinline__ void write_images(const C &c, T *f, T v, const Img<T> &ix, const Img<T> &iy,
                                             const Img<T> &iz) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (!ix.ok[a]) continue;
        T va = ix.dir[a] ? T(2.0) * ix.c[a] - v : v;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            if (!iy.ok[b]) continue;
            T vb = iy.dir[b] ? T(2.0) * iy.c[b] - va : va;
#pragma unroll
            for (int e = 0; e < 3; e++) {
                if (!iz.ok[e]) continue;
                T ve = iz.dir[e] ? T(2.0) * iz.c[e] - vb : vb;
                f[c.gidx(ix.pos[a], iy.pos[b], iz.pos[e])] = ve;
            }
        }
    }
}

// ---- velocity / η_next update of plane t on the column ----------------------------
template <typename T, typename C>
__device__ __forceinline__ T vx_raw(const C &c, const KParams &p, const TConst<T> &q, const Ptrs<T> &in, int t, int i,
                                    int j, long long I) {
    const T idx = q.inv_dx[0], idy = q.inv_dx[1], idz = q.inv_dx[2];
    T gx = (p.g_kind[0] == FI_G_FIELD ? in.gx[I] : q.g_val[0]);
    T ex = h(c.Eta(t, i - 1, j) + c.Eta(t, i, j));
    return c.Vx(t, i, j) + div_fast(-(c.P(t, i, j) - c.P(t, i - 1, j)) * idx + (c.Txx(t, i, j) - c.Txx(t, i - 1, j)) * idx +
                                       (c.Txy(t, i, j + 1) - c.Txy(t, i, j)) * idy +
                                       (c.Txz(t + 1, i, j) - c.Txz(t, i, j)) * idz - gx,
                                   ex) *
                               q.dt_V[0];
}
template <typename T, typename C>
__device__ __forceinline__ T vy_raw(const C &c, const KParams &p, const TConst<T> &q, const Ptrs<T> &in, int t, int i,
                                    int j, long long I) {
    const T idx = q.inv_dx[0], idy = q.inv_dx[1], idz = q.inv_dx[2];
    T gy = (p.g_kind[1] == FI_G_FIELD ? in.gy[I] : q.g_val[1]);
    T ey = h(c.Eta(t, i, j - 1) + c.Eta(t, i, j));
    return c.Vy(t, i, j) + div_fast(-(c.P(t, i, j) - c.P(t, i, j - 1)) * idy + (c.Tyy(t, i, j) - c.Tyy(t, i, j - 1)) * idy +
                                       (c.Txy(t, i + 1, j) - c.Txy(t, i, j)) * idx +
                                       (c.Tyz(t + 1, i, j) - c.Tyz(t, i, j)) * idz - gy,
                                   ey) *
                               q.dt_V[1];
}
template <typename T, typename C>
__device__ __forceinline__ T vz_raw(const C &c, const KParams &p, const TConst<T> &q, const Ptrs<T> &in, int t, int i,
                                    int j, long long I) {
    const T idx = q.inv_dx[0], idy = q.inv_dx[1], idz = q.inv_dx[2];
    T gz = (p.g_kind[2] == FI_G_FIELD ? in.gz[I] : q.g_val[2]);
    T ez = h(c.Eta(t - 1, i, j) + c.Eta(t, i, j));
    return c.Vz(t, i, j) + div_fast(-(c.P(t, i, j) - c.P(t - 1, i, j)) * idz + (c.Tzz(t, i, j) - c.Tzz(t - 1, i, j)) * idz +
                                       (c.Txz(t, i + 1, j) - c.Txz(t, i, j)) * idx +
                                       (c.Tyz(t, i, j + 1) - c.Tyz(t, i, j)) * idy - gz,
                                   ez) *
                               q.dt_V[2];
}
template <typename T, typename C>
__device__ __forceinline__ T eta_raw(const C &c, const KParams &p, const TConst<T> &q, const Ptrs<T> &in, int t, int i,
                                     int j, long long I) {
    T xx = c.Txx(t, i, j), yy = c.Tyy(t, i, j), zz = c.Tzz(t, i, j);
    T lxy = h(h(c.Txy(t, i, j) + c.Txy(t, i + 1, j)) + h(c.Txy(t, i, j + 1) + c.Txy(t, i + 1, j + 1)));
    T lxz = h(h(c.Txz(t, i, j) + c.Txz(t, i + 1, j)) + h(c.Txz(t + 1, i, j) + c.Txz(t + 1, i + 1, j)));
    T lyz = h(h(c.Tyz(t, i, j) + c.Tyz(t, i, j + 1)) + h(c.Tyz(t + 1, i, j) + c.Tyz(t + 1, i, j + 1)));
    T s2 = T(0.5) * (xx * xx + yy * yy + zz * zz) + lxy * lxy + lxz * lxz + lyz * lyz;
    return rheology_s2(p, q.rheo_A, q.rheo_inv_eta_reg, in.eta_lin, in.A, c.Eta(t, i, j), I, s2);
}

template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void v_point(const Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q,
                                        const Ptrs<T> &in, const Ptrs<T> &out, int t, int i, int j) {
    const int n0 = c.n0, n1 = c.n1, n2 = c.n2;
    if (i > n0 + 1 || j > n1 + 1) return;
    const long long I = c.gidx(i, j, t);
    const bool near = i <= 2 || i >= n0 || j <= 2 || j >= n1 || t <= 1 || t >= n2;
    if (!near) {
        // all four values before the first store (see sigma_point)
        const T vxn = vx_raw(c, p, q, in, t, i, j, I);
        const T vyn = vy_raw(c, p, q, in, t, i, j, I);
        const T vzn = vz_raw(c, p, q, in, t, i, j, I);
        const T etn = p.freeze_eta ? T(0) : eta_raw(c, p, q, in, t, i, j, I);
        out.Vx[I] = vxn;
        out.Vy[I] = vyn;
        out.Vz[I] = vzn;
        if (!p.freeze_eta) out.eta_next[I] = etn;
        return;
    }
    auto node_fixed = [](int kind) { return kind == FI_BC_SLIP || kind == FI_BC_VELOCITY; };
    const int xl = p.bc_kind[0][0], xr = p.bc_kind[0][1], yl = p.bc_kind[1][0], yr = p.bc_kind[1][1];
    const int zl = p.bc_kind[2][0], zr = p.bc_kind[2][1];
    // ---- V.x at (V, C, C)
    if (j <= n1 && t >= 1 && t <= n2 && !(c.hx1 && i == n0 + 1)) {
        T v;
        if (!c.hx0 && i == 1 && node_fixed(xl)) v = q.bc_val[0][0][0];
        else if (!c.hx1 && i == n0 + 1 && node_fixed(xr)) v = q.bc_val[0][1][0];
        else v = vx_raw(c, p, q, in, t, i, j, I);
        write_images(c, out.Vx, v, img_vertex<T>(i, n0, c.hx0, c.hx1),
                     img_center<T>(j, n1, c.hy0, c.hy1, yl, yr, q.bc_val[1][0][0], q.bc_val[1][1][0], false),
                     img_center<T>(t, n2, false, false, zl, zr, q.bc_val[2][0][0], q.bc_val[2][1][0], false));
    }
    // A value on a fixed node of its own dim d is written there last by the
    // reference's dim-d node assignment, which spans the ghosts of the dims before
    // d: its images along those dims are copies, not mirrors (as_copies).
    auto as_copies = [](Img<T> d) {
        d.dir[1] = false;
        d.dir[2] = false;
        return d;
    };
    // ---- V.y at (C, V, C)
    if (i <= n0 && t >= 1 && t <= n2 && !(c.hy1 && j == n1 + 1)) {
        T v;
        const bool y_node = (!c.hy0 && j == 1 && node_fixed(yl)) || (!c.hy1 && j == n1 + 1 && node_fixed(yr));
        if (!c.hy0 && j == 1 && node_fixed(yl)) v = q.bc_val[1][0][1];
        else if (!c.hy1 && j == n1 + 1 && node_fixed(yr)) v = q.bc_val[1][1][1];
        else v = vy_raw(c, p, q, in, t, i, j, I);
        Img<T> ix = img_center<T>(i, n0, c.hx0, c.hx1, xl, xr, q.bc_val[0][0][1], q.bc_val[0][1][1], false);
        write_images(c, out.Vy, v, y_node ? as_copies(ix) : ix, img_vertex<T>(j, n1, c.hy0, c.hy1),
                     img_center<T>(t, n2, false, false, zl, zr, q.bc_val[2][0][1], q.bc_val[2][1][1], false));
    }
    // ---- V.z at (C, C, V)
    if (i <= n0 && j <= n1 && t >= 1 && t <= n2 + 1) {
        T v;
        const bool z_node = (t == 1 && node_fixed(zl)) || (t == n2 + 1 && node_fixed(zr));
        if (t == 1 && node_fixed(zl)) v = q.bc_val[2][0][2];
        else if (t == n2 + 1 && node_fixed(zr)) v = q.bc_val[2][1][2];
        else v = vz_raw(c, p, q, in, t, i, j, I);
        Img<T> ix = img_center<T>(i, n0, c.hx0, c.hx1, xl, xr, q.bc_val[0][0][2], q.bc_val[0][1][2], false);
        Img<T> iy = img_center<T>(j, n1, c.hy0, c.hy1, yl, yr, q.bc_val[1][0][2], q.bc_val[1][1][2], false);
        write_images(c, out.Vz, v, z_node ? as_copies(ix) : ix, z_node ? as_copies(iy) : iy, img_own<T>(t));
    }
    // ---- η_next at (C, C, C), Neumann / periodic ghosts
    if (!p.freeze_eta && i <= n0 && j <= n1 && t >= 1 && t <= n2) {
        T en = eta_raw(c, p, q, in, t, i, j, I);
        write_images(c, out.eta_next, en, img_center<T>(i, n0, c.hx0, c.hx1, xl, xr, T(0), T(0), true),
                     img_center<T>(j, n1, c.hy0, c.hy1, yl, yr, T(0), T(0), true),
                     img_center<T>(t, n2, false, false, zl, zr, T(0), T(0), true));
    }
}

template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void v_plane(const Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q,
                                        const Ptrs<T> &in, const Ptrs<T> &out, int t) {
    const int lane = threadIdx.x % 32, j = c.j0 + (int)(threadIdx.x / 32);
#pragma unroll
    for (int u = 0; u < TX / 32; u++) v_point(c, p, q, in, out, t, c.i0 + lane + 32 * u, j);
}

// the plane march of one CTA (TRIM: an interior column of a trimmed launch shape)
template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void sweep(Ctx<T, TX, TY, TRIM> &c, const KParams &p, const TConst<T> &q, const Ptrs<T> &in,
                                      const Ptrs<T> &out, const InMaps &maps, uint64_t *bars, int *err) {
    const int tid = threadIdx.x;
    const int f = max(c.kb - 1, 1), last = min(c.ke, c.n2 + 1);
    uint32_t phase = 0;  // bit b: parity of the next completion of bars[b]
    c.set_plane(f);
    if (tid == 0) {
        issue_group(c, maps, f - 1, false, &bars[(f - 1) % kBars]);
        issue_group(c, maps, f, true, &bars[f % kBars]);
    }
    auto wait_group = [&](int pl) -> bool {
        const int b = pl % kBars;
        bool ok = mbar_wait(&bars[b], (phase >> b) & 1u);
        phase ^= 1u << b;
        return ok;
    };
    bool ok = wait_group(f - 1);
    for (int s = f; s <= last && ok; s++) {
        c.set_plane(s);
        if (tid == 0 && s + 1 <= last) {
            fence_proxy_async();
            issue_group(c, maps, s + 1, true, &bars[(s + 1) % kBars]);
        }
        ok = wait_group(s);
        if (!ok) break;
        sigma_plane(c, p, q, out, s);
        if (s - 1 >= c.kb && s - 1 < c.ke) v_plane(c, p, q, in, out, s - 1);
        __syncthreads();
    }
    if (ok) {
        if (c.ke - 1 == last && last == c.n2 + 1) {
            c.set_plane(last);
            v_plane(c, p, q, in, out, last);
        }
        return;
    }
    // bounded wait expired: record it and drain this CTA's own copies (bounded) before leaving
    atomicExch(err, (int)FI_ERR_TIMEOUT);
    for (int b = 0; b < kBars; b++) mbar_wait(&bars[b], (phase >> b) & 1u);
}

// Tiles of one launch along a split dimension: a launch runs either every tile, or
// part of them (the overlapped halo exchange runs the tiles next to the split faces
// first and the others while the halo moves).  Along `dim`, grid block b stands for
// tile b + base + (b >= nlow ? shift : 0).
struct TileMap {
    int dim;  // 0: x, 1: y, -1: every tile
    int base, nlow, shift;
};

__device__ __forceinline__ int tile_x(const TileMap &tm) {
    const int b = (int)blockIdx.x;
    return tm.dim == 0 ? b + tm.base + (b >= tm.nlow ? tm.shift : 0) : b;
}
__device__ __forceinline__ int tile_y(const TileMap &tm) {
    const int b = (int)blockIdx.y;
    return tm.dim == 1 ? b + tm.base + (b >= tm.nlow ? tm.shift : 0) : b;
}

template <typename T, int TX, int TY, bool TRIM>
__device__ __forceinline__ void init_ctx(Ctx<T, TX, TY, TRIM> &c, const Geom &g, const KParams &p, unsigned char *smem,
                                         int zb, const TileMap &tm) {
    c.sm = reinterpret_cast<T *>(smem);
    c.i0 = 1 + tile_x(tm) * TX;
    c.j0 = 1 + tile_y(tm) * TY;
    c.kb = 1 + blockIdx.z * zb;
    c.n0 = g.n[0];
    c.n1 = g.n[1];
    c.n2 = g.n[2];
    c.ke = min(c.kb + zb, c.n2 + 2);
    c.sx = g.pitch;
    c.sxy = g.sxy;
    auto away = [](int k) { return k == FI_BC_PERIODIC || k == FI_BC_HALO; };
    c.hx0 = away(p.bc_kind[0][0]);
    c.hx1 = away(p.bc_kind[0][1]);
    c.hy0 = away(p.bc_kind[1][0]);
    c.hy1 = away(p.bc_kind[1][1]);
    c.bnd_x = c.i0 == 1 || c.i0 + TX >= c.n0 + 1;
    c.bnd_y = c.j0 == 1 || c.j0 + TY >= c.n1 + 1;
}

// TRIMK: the kernel holds the trimmed path for interior columns (shapes without it keep
// one plane-march body, as small as before trimming existed)
template <typename T, int TX, int TY, bool TRIMK>
__global__ void __launch_bounds__(Layout<T, TX, TY>::NT, Layout<T, TX, TY>::MINB)
    fused3d_kernel(Geom g, KParams p, TConst<T> q, Ptrs<T> in, Ptrs<T> out, const __grid_constant__ InMaps maps, int zb,
                   TileMap tm, int *err) {
    using Lay = Layout<T, TX, TY>;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // the grid is padded to whole clusters: columns past the vertex range have no work
    if (1 + tile_x(tm) * TX > g.n[0] + 1 || 1 + tile_y(tm) * TY > g.n[1] + 1) return;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + (size_t)S_COUNT * Lay::SLOT * sizeof(T));
    if (threadIdx.x == 0) {
        for (int b = 0; b < kBars; b++) mbar_init(&bars[b], 1);
        mbar_fence_init();
    }
    __syncthreads();
    Ctx<T, TX, TY, false> c;
    init_ctx(c, g, p, smem_raw, zb, tm);
    if constexpr (TRIMK) {
        if (!c.bnd_x && !c.bnd_y) {
            Ctx<T, TX, TY, true> ct;
            init_ctx(ct, g, p, smem_raw, zb, tm);
            sweep(ct, p, q, in, out, maps, bars, err);
            return;
        }
    }
    sweep(c, p, q, in, out, maps, bars, err);
}

template <typename T, int TX, int TY>
cudaError_t launch_variant(const Geom &g, const KParams &p, const Ptrs<T> &in, const Ptrs<T> &out, const InMaps &maps,
                           Variant v, int *err, cudaStream_t s, int part_dim, int part) {
    using Lay = Layout<T, TX, TY>;
    int dev = 0;
    cudaGetDevice(&dev);
    static bool attr_set[2][64] = {};
    if (dev < 64 && !attr_set[v.trim][dev]) {
        cudaError_t e = cudaFuncSetAttribute(v.trim ? fused3d_kernel<T, TX, TY, true> : fused3d_kernel<T, TX, TY, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::SMEM);
        if (e != cudaSuccess) return e;
        attr_set[v.trim][dev] = true;
    }
    auto up = [](int a, int b) { return (a + b - 1) / b * b; };
    TileMap tm{-1, 0, 1 << 30, 0};
    const int nbx = (g.n[0] + 1 + TX - 1) / TX, nby = (g.n[1] + 1 + TY - 1) / TY;
    int gx = nbx, gy = nby;
    if (part_dim == 0 || part_dim == 1) {
        // part 0: the tiles of the split faces -- tile 0 (positions 1 and 2) and the
        // tile of position n: the layers a slab sends and the ghost images it
        // writes; part 1: every other tile.  No clusters in partial launches.
        const int T_d = part_dim == 0 ? TX : TY, nb = part_dim == 0 ? nbx : nby;
        const int last = (g.n[part_dim] - 1) / T_d;
        int cnt;
        if (part == 0) {
            tm = {part_dim, 0, 1, last - 1};
            cnt = last > 0 ? 2 : 1;
        } else {
            // tiles 1 .. last-1, then last+1 .. nb-1
            tm = last > 0 ? TileMap{part_dim, 1, last - 1, 1} : TileMap{part_dim, 1, 1 << 30, 0};
            cnt = nb - (last > 0 ? 2 : 1);
            if (cnt <= 0) return cudaSuccess;
        }
        (part_dim == 0 ? gx : gy) = cnt;
        v.cx = v.cy = 1;
    }
    dim3 grd(up(gx, v.cx), up(gy, v.cy), (g.n[2] + 1 + v.zb - 1) / v.zb);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grd;
    cfg.blockDim = dim3(Lay::NT);
    cfg.dynamicSmemBytes = Lay::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    if (v.cx * v.cy > 1) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = v.cx;
        attr[0].val.clusterDim.y = v.cy;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    const TConst<T> q = make_tconst<T>(p);
    if (v.trim) return cudaLaunchKernelEx(&cfg, fused3d_kernel<T, TX, TY, true>, g, p, q, in, out, maps, v.zb, tm, err);
    return cudaLaunchKernelEx(&cfg, fused3d_kernel<T, TX, TY, false>, g, p, q, in, out, maps, v.zb, tm, err);
}

template <typename T>
size_t variant_smem(const Variant &v) {
    if (v.tx == 64) return v.ty == 4 ? Layout<T, 64, 4>::SMEM : Layout<T, 64, 8>::SMEM;
    return v.ty == 4 ? Layout<T, 32, 4>::SMEM : v.ty == 16 ? Layout<T, 32, 16>::SMEM : Layout<T, 32, 8>::SMEM;
}

PFN_cuTensorMapEncodeTiled_v12000 get_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *ptr = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)ptr;
    }
    return fn;
}

// box (width, height) of input field f for tile tx x ty (trimmed: the interior box)
template <typename T, int TX, int TY>
void box_of(int f, bool trimmed, int *bw, int *bh) {
#define FI_BOX_CASE(F)                                      \
    case F:                                                 \
        if (trimmed) {                                      \
            *bw = FBox<T, TX, TY, true, F>::bw;             \
            *bh = FBox<T, TX, TY, true, F>::bh;             \
        } else {                                            \
            *bw = FBox<T, TX, TY, false, F>::bw;            \
            *bh = FBox<T, TX, TY, false, F>::bh;            \
        }                                                   \
        return;
    switch (f) {
        FI_BOX_CASE(M_P)
        FI_BOX_CASE(M_XX)
        FI_BOX_CASE(M_YY)
        FI_BOX_CASE(M_ZZ)
        FI_BOX_CASE(M_XY)
        FI_BOX_CASE(M_XZ)
        FI_BOX_CASE(M_YZ)
        default: FI_BOX_CASE(M_VX)
    }
#undef FI_BOX_CASE
}

template <typename T>
void variant_box(const Variant &v, int f, bool trimmed, int *bw, int *bh) {
    if (v.tx == 64) {
        if (v.ty == 4) box_of<T, 64, 4>(f, trimmed, bw, bh);
        else box_of<T, 64, 8>(f, trimmed, bw, bh);
    } else if (v.ty == 4) {
        box_of<T, 32, 4>(f, trimmed, bw, bh);
    } else if (v.ty == 16) {
        box_of<T, 32, 16>(f, trimmed, bw, bh);
    } else {
        box_of<T, 32, 8>(f, trimmed, bw, bh);
    }
}

}  // namespace

int fused3d_num_variants() { return kNumVariants; }
const char *fused3d_variant_name(int v) {
    static char buf[kNumVariants][48];
    if (v < 0 || v >= kNumVariants) return "?";
    const Variant &w = kVariants[v];
    int n = snprintf(buf[v], sizeof(buf[v]), "tile%dx%d_zb%d", w.tx, w.ty, w.zb);
    if (w.trim) n += snprintf(buf[v] + n, sizeof(buf[v]) - n, "_trim");
    if (w.cx * w.cy > 1) snprintf(buf[v] + n, sizeof(buf[v]) - n, "_cl%dx%d", w.cx, w.cy);
    return buf[v];
}
int fused3d_variant_key(int v) {
    const Variant &w = kVariants[(v < 0 || v >= kNumVariants) ? 0 : v];
    return w.tx * 1000 + w.ty;
}
bool fused3d_variant_fits(int v, int esz) {
    if (v < 0 || v >= kNumVariants) return false;
    const size_t smem = esz == 8 ? variant_smem<double>(kVariants[v]) : variant_smem<float>(kVariants[v]);
    // 64-wide FP64 tiles would hold one CTA per SM: not offered
    if (esz == 8 && kVariants[v].tx == 64) return false;
    return smem <= 227 * 1024;
}

template <typename T>
bool fused3d_supported(const Geom &g, const KParams &p, bool ib) {
    if (g.nd != 3 || ib) return false;
    if (p.bc_kind[2][0] == FI_BC_PERIODIC) return false;
    return g.pitch >= kXOff + g.n[0] + 3;
}

// a 2D or 3D tiled tensor map (no interleave, no swizzle, zero fill out of range)
// over `nd` dims of a field allocation; strides in bytes (dims 1..nd-1)
bool tma_encode(void *raw_base, int nd, const unsigned long long *dims, const unsigned long long *strides,
                const unsigned *box, int esz, void *map_out) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = get_encoder();
    if (!enc || nd < 1 || nd > 3) return false;
    cuuint64_t d[3], st[2];
    cuuint32_t bx[3], estr[3] = {1, 1, 1};
    for (int k = 0; k < nd; k++) {
        d[k] = dims[k];
        bx[k] = box[k];
        if (k > 0) st[k - 1] = strides[k - 1];
    }
    CUresult r = enc((CUtensorMap *)map_out, esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     nd, raw_base, d, st, bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// the 3D tensor map of input field f (map order) over a field allocation (raw
// base, aligned) for a launch shape: box = one plane of the field's full box, or
// of its trimmed box (stress fields of interior columns)
bool fused3d_encode_map(void *raw_base, const Geom &g, int esz, int variant, int field, bool trimmed, void *map_out) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = get_encoder();
    if (!enc || variant < 0 || variant >= kNumVariants || field < 0 || field >= M_COUNT) return false;
    int bw = 0, bh = 0;
    if (esz == 8) variant_box<double>(kVariants[variant], field, trimmed && field < kTrimmed, &bw, &bh);
    else variant_box<float>(kVariants[variant], field, trimmed && field < kTrimmed, &bw, &bh);
    cuuint64_t dims[3] = {(cuuint64_t)g.pitch, (cuuint64_t)g.rows, (cuuint64_t)g.planes};
    cuuint64_t strides[2] = {(cuuint64_t)(g.pitch * esz), (cuuint64_t)(g.sxy * esz)};
    cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    // L2 promotion of the box rows; FI_TMA_L2_PROMOTION=0/64/128/256 overrides
    CUtensorMapL2promotion promo = CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
    if (const char *e = getenv("FI_TMA_L2_PROMOTION")) {
        int v = atoi(e);
        promo = v == 0 ? CU_TENSOR_MAP_L2_PROMOTION_NONE
                       : v == 64 ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
                                 : v == 128 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B : CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
    }
    CUresult r = enc((CUtensorMap *)map_out, esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                     3, raw_base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <typename T>
cudaError_t launch_fused3d(const Geom &g, const KParams &p, const Ptrs<T> &in, const Ptrs<T> &out, const void *maps18,
                           int variant, int *err, cudaStream_t s, int part_dim, int part) {
    if (variant < 0 || variant >= kNumVariants) variant = 0;
    const Variant v = kVariants[variant];
    if (!fused3d_variant_fits(variant, (int)sizeof(T))) return cudaErrorInvalidConfiguration;
    const InMaps &mp = *reinterpret_cast<const InMaps *>(maps18);
    if (v.tx == 64) {
        if constexpr (sizeof(T) == 4) {
            if (v.ty == 4) return launch_variant<T, 64, 4>(g, p, in, out, mp, v, err, s, part_dim, part);
            return launch_variant<T, 64, 8>(g, p, in, out, mp, v, err, s, part_dim, part);
        }
        return cudaErrorInvalidConfiguration;
    }
    switch (v.ty) {
        case 4: return launch_variant<T, 32, 4>(g, p, in, out, mp, v, err, s, part_dim, part);
        case 16: return launch_variant<T, 32, 16>(g, p, in, out, mp, v, err, s, part_dim, part);
        default: return launch_variant<T, 32, 8>(g, p, in, out, mp, v, err, s, part_dim, part);
    }
}

template bool fused3d_supported<double>(const Geom &, const KParams &, bool);
template bool fused3d_supported<float>(const Geom &, const KParams &, bool);
template cudaError_t launch_fused3d<double>(const Geom &, const KParams &, const Ptrs<double> &, const Ptrs<double> &,
                                            const void *, int, int *, cudaStream_t, int, int);
template cudaError_t launch_fused3d<float>(const Geom &, const KParams &, const Ptrs<float> &, const Ptrs<float> &,
                                           const void *, int, int *, cudaStream_t, int, int);

}  // namespace fi
