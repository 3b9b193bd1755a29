// fi_batch.cu -- batched 2D PT solves: many independent 2D Stokes instances of
// different sizes advanced together, one persistent launch per PT iteration.
//
// Reference semantics per instance: advance_iteration! of the 2D
// IsothermalFullStokesModel (src/Models/FullStokes/Isothermal/Isothermal.jl:91-112,
// kernels_2d.jl:3-29, boundary_conditions.jl:26-47 and :104-115) with a linear
// viscosity that stays fixed (η = η_next = the rheology's viscosity, the state
// the reference reaches after its first η swap).
//
// Work decomposition.  Every instance is cut into 32 x TY tiles of its vertex
// range.  A device-side work list holds the tiles of the instances still
// iterating; a persistent grid (a multiple of the SM count) strides over it.  A
// CTA stages its tile plus a one-position ring of the seven input fields (P, τxx,
// τyy, τxy, Vx, Vy, η) in shared memory, computes the new stresses on the tile
// and the ring components the velocity update needs, applies the stress boundary
// conditions in shared memory (x faces, then y faces), updates the velocities
// with their boundary values and ghost images, and writes the new state to the
// instance's other buffer (double buffering: each sweep reads buffer s % 2 and
// writes the other one).
//
// Checks.  Every ncheck sweeps a residual kernel evaluates r_P and r_V of every
// active instance in FP64 arithmetic and folds per-instance maxima (bit patterns
// of non-negative doubles, atomicMax: exact, order independent); a bookkeeping
// kernel turns them into each instance's measure, retires converged, stalled or
// failed instances, and a compaction pass rebuilds the work list.  The whole
// check-to-check step is a fixed launch sequence, captured once as a CUDA graph
// and replayed; the host reads back one word (instances still active) per replay.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "fi_device.cuh"
#include "fi_model.h"
#include "fi_tma.cuh"

namespace fi {
namespace {

constexpr int BTX = 32;
constexpr int kBatchTY[] = {8, 4, 16};
constexpr int kBatchVariants = sizeof(kBatchTY) / sizeof(kBatchTY[0]);
constexpr int kSlots = 4;  // per-instance check maxima: |r_P|, |r_V|, |P, τ|, |V|

template <typename T>
struct alignas(16) BInst {  // copied whole into shared memory (bulk copy: 16-byte granules)
    int n0, n1;
    long long pitch;
    T idx, idy, dtP, dxx, dyy, dxy, dVx, dVy;
    T gval[2];
    int gkind[2];
    int bc_kind[2][2];
    T bc_val[2][2][2];
    T *P[2], *txx[2], *tyy[2], *txy[2], *Vx[2], *Vy[2];
    const T *eta;
    const T *gx, *gy;
    const T *fP;  // pressure forcing of a defect-correction problem (pforce), else unused
    int pforce;
    int pad_;
    double h;  // smallest grid spacing (scales the check's measure)
};

// per-instance solve state on the device
struct BState {
    int status;  // fi_batch_item_status
    int iters;
    int since;   // sweeps since the best measure last halved
    int pad;
    double best;
    double measure;
};

__device__ __forceinline__ bool node_fixed(int kind) { return kind == FI_BC_SLIP || kind == FI_BC_VELOCITY; }

// TMA box width (elements) and the column's offset inside it: the box starts XB
// positions left of the tile so that its x coordinate is 16-byte aligned
template <typename T>
struct BBox;
template <>
struct BBox<double> {
    static constexpr int BX = 36, XB = 2;
};
template <>
struct BBox<float> {
    static constexpr int BX = 40, XB = 4;
};

// per-member tensor maps: [buffer][P, txx, tyy, txy, Vx, Vy, eta] (eta is the same
// array for both buffers)
struct alignas(128) BMaps {
    unsigned char m[2][7][128];
};

template <typename T, int TY>
struct Tile {
    static constexpr int BX = BBox<T>::BX, XB = BBox<T>::XB, RW = BTX + 2, RY = TY + 2, NT = BTX * TY;
    static constexpr int BOXB = BX * RY * (int)sizeof(T);
    static constexpr int SLOTB = (BOXB + 127) / 128 * 128;
    static constexpr int PARB = ((int)sizeof(BInst<T>) + 127) / 128 * 128;
    static constexpr int STAGEB = 7 * SLOTB + PARB + 128;  // 7 boxes, the member's parameters, the tile descriptor
    static constexpr uint32_t TX_BYTES = 7u * BOXB + (uint32_t)sizeof(BInst<T>);
    T *sP, *sXX, *sYY, *sXY, *sVx, *sVy, *sEt;
    int i0, j0, n0, n1;
    __device__ __forceinline__ int at(int i, int j) const { return (j - j0 + 1) * BX + (i - i0 + XB); }
    __device__ __forceinline__ bool own_x(int i) const {
        if (i >= 1 && i <= n0 + 1) return i >= i0 && i < i0 + BTX;
        if (i == 0) return i0 == 1;
        return i == n0 + 2 && n0 + 1 < i0 + BTX;
    }
    __device__ __forceinline__ bool own_y(int j) const {
        if (j >= 1 && j <= n1 + 1) return j >= j0 && j < j0 + TY;
        if (j == 0) return j0 == 1;
        return j == n1 + 2 && n1 + 1 < j0 + TY;
    }
};

enum { M_P = 1, M_XX = 2, M_YY = 4, M_XY = 8, M_ALL = 15 };

// new stresses at (i, j) in shared memory (kernels_2d.jl:3-18), components in mask;
// all operands are loaded before the first store
template <typename T, int TY>
__device__ __forceinline__ void sigma2(const Tile<T, TY> &t, const BInst<T> &b, int i, int j, int mask) {
    constexpr int BX = Tile<T, TY>::BX;
    const int a = t.at(i, j);
    const bool dc = (mask & (M_P | M_XX | M_YY)) && i >= 1 && i <= t.n0 && j >= 1 && j <= t.n1;
    const bool dxy = (mask & M_XY) && i >= 1 && i <= t.n0 + 1 && j >= 1 && j <= t.n1 + 1;
    if (dc) {
        const T oP = t.sP[a], oXX = t.sXX[a], oYY = t.sYY[a];
        T exx = (t.sVx[a + 1] - t.sVx[a]) * b.idx;
        T eyy = (t.sVy[a + BX] - t.sVy[a]) * b.idy;
        T divV = exx + eyy;
        T etac = t.sEt[a];
        T nXY = T(0), oXY = T(0);
        if (dxy) {
            oXY = t.sXY[a];
            T exy = T(0.5) * ((t.sVy[a] - t.sVy[a - 1]) * b.idx + (t.sVx[a] - t.sVx[a - BX]) * b.idy);
            T e_xy = T(0.5) * (T(0.5) * (t.sEt[a - 1 - BX] + t.sEt[a - BX]) + T(0.5) * (t.sEt[a - 1] + t.sEt[a]));
            nXY = oXY - (oXY - T(2.0) * e_xy * exy) * b.dxy;
        }
        if (mask & M_P) {
            // the forced pressure update of a correction problem (as update_σ! with p_forcing)
            const T dv = b.pforce ? divV + b.fP[(long long)i + b.pitch * (long long)j] : divV;
            t.sP[a] = oP - dv * etac * b.dtP;
        }
        if (mask & M_XX) t.sXX[a] = oXX - (oXX - T(2.0) * etac * (exx - third(divV))) * b.dxx;
        if (mask & M_YY) t.sYY[a] = oYY - (oYY - T(2.0) * etac * (eyy - third(divV))) * b.dyy;
        if (dxy) t.sXY[a] = nXY;
    } else if (dxy) {
        const T oXY = t.sXY[a];
        T exy = T(0.5) * ((t.sVy[a] - t.sVy[a - 1]) * b.idx + (t.sVx[a] - t.sVx[a - BX]) * b.idy);
        T e_xy = T(0.5) * (T(0.5) * (t.sEt[a - 1 - BX] + t.sEt[a - BX]) + T(0.5) * (t.sEt[a - 1] + t.sEt[a]));
        t.sXY[a] = oXY - (oXY - T(2.0) * e_xy * exy) * b.dxy;
    }
}

// Dirichlet ghost images of a velocity value along one dim (boundary_conditions.jl:104-115):
// a Center-located component next to a Velocity side gets the ghost 2c - v.  When
// the value sits on a fixed node of a later dim, that dim's node assignment (which
// spans the earlier dims' ghosts) runs last and leaves the ghost equal to the node
// value: copy instead of mirror.
template <typename T>
__device__ __forceinline__ void center_ghosts(int q, int N, int kl, int kr, T cl, T cr, int *pos, T *val, bool *ok,
                                              T v, bool later_node) {
    ok[0] = ok[1] = false;
    if (q == 1 && kl == FI_BC_VELOCITY) { pos[0] = 0; val[0] = later_node ? v : T(2.0) * cl - v; ok[0] = true; }
    if (q == N && kr == FI_BC_VELOCITY) { pos[1] = N + 1; val[1] = later_node ? v : T(2.0) * cr - v; ok[1] = true; }
}

// copies of tile d (member d.x, tile origin (d.y, d.z)) into one stage: the seven
// input boxes (tensor maps of buffer src), the member's parameter block and the
// descriptor itself (read by the other threads once the stage's barrier completes)
template <typename T, int TY>
__device__ __forceinline__ void issue_tile(const BInst<T> *__restrict__ insts, const BMaps *__restrict__ maps, int4 d,
                                           int src, unsigned char *stage, uint64_t *bar) {
    using TL = Tile<T, TY>;
    *reinterpret_cast<int4 *>(stage + 7 * TL::SLOTB + TL::PARB) = d;
    mbar_expect_tx(bar, TL::TX_BYTES);
    const BMaps &mp = maps[d.x];
    const int x = (int)kXOff + d.y - TL::XB, y = d.z - 1;
#pragma unroll
    for (int f = 0; f < 7; f++) tma_load_2d(stage + f * TL::SLOTB, mp.m[src][f], x, y, bar);
    bulk_load(stage + 7 * TL::SLOTB, insts + d.x, (uint32_t)sizeof(BInst<T>), bar);
}

// One PT iteration of every tile in the work list.  A persistent CTA strides over
// the list through three stages: while tile k is computed, the copies of tiles
// k+1 and k+2 of its stride are in flight, and the descriptor of tile k+3 is
// fetched one step early, so the issuing thread never waits on it.  Tile k+2 is
// issued into the stage tile k-1 used, right after the block barrier that follows
// tile k's stress update: every thread passes that barrier only after finishing
// tile k-1 (its velocity update included), so one barrier per interior tile
// suffices.
constexpr int kStages = 3;
// 48 resident warps per SM in FP32 (at most 42 registers a thread), 32 in FP64
template <typename T, int TY>
__global__ void __launch_bounds__(BTX *TY, (sizeof(T) == 8 ? 1024 : 1536) / (BTX * TY)) batch2d_sweep(const BInst<T> *__restrict__ insts,
                                                         const BMaps *__restrict__ maps, const int4 *__restrict__ tiles,
                                                         const int *__restrict__ ntiles, int src, int *err) {
    using TL = Tile<T, TY>;
    extern __shared__ __align__(1024) unsigned char batch_smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(batch_smem + kStages * TL::STAGEB);
    TL t;
    const int tid = threadIdx.x, dst = src ^ 1;
    const int nt = *ntiles, G = gridDim.x;
    if (tid == 0) {
        for (int q = 0; q < kStages; q++) mbar_init(&bars[q], 1);
        mbar_fence_init();
    }
    __syncthreads();
    int4 dnext = make_int4(0, 1, 1, 0);
    if (tid == 0) {
        for (int q = 0; q < kStages - 1; q++)
            if ((int)blockIdx.x + q * G < nt)
                issue_tile<T, TY>(insts, maps, tiles[blockIdx.x + q * G], src, batch_smem + q * TL::STAGEB, &bars[q]);
        if ((int)blockIdx.x + (kStages - 1) * G < nt) dnext = tiles[blockIdx.x + (kStages - 1) * G];
    }
    uint32_t phase = 0;
    bool failed = false;
    int cur = 0;
    for (int w = blockIdx.x; w < nt; w += G, cur = cur == kStages - 1 ? 0 : cur + 1) {
        // a wait that expires is recorded and the remaining tiles are computed from
        // whatever the stage holds (the solve reports FI_ERR_TIMEOUT); later waits
        // of this thread are single polls, so the launch ends in bounded time
        const bool ok = failed ? mbar_try_wait(&bars[cur], (phase >> cur) & 1u) : mbar_wait(&bars[cur], (phase >> cur) & 1u);
        phase ^= 1u << cur;
        if (!ok && !failed) {
            failed = true;
            atomicExch(err, (int)FI_ERR_TIMEOUT);
        }
        unsigned char *stage = batch_smem + cur * TL::STAGEB;
        T *sm = reinterpret_cast<T *>(stage);
        constexpr int SE = TL::SLOTB / (int)sizeof(T);
        t.sP = sm;
        t.sXX = sm + SE;
        t.sYY = sm + 2 * SE;
        t.sXY = sm + 3 * SE;
        t.sVx = sm + 4 * SE;
        t.sVy = sm + 5 * SE;
        t.sEt = sm + 6 * SE;
        const BInst<T> &b = *reinterpret_cast<const BInst<T> *>(stage + 7 * TL::SLOTB);
        const int4 d = *reinterpret_cast<const int4 *>(stage + 7 * TL::SLOTB + TL::PARB);
        t.i0 = d.y;
        t.j0 = d.z;
        t.n0 = b.n0;
        t.n1 = b.n1;
        const long long sx = b.pitch;
        const bool bnd_x = t.i0 == 1 || t.i0 + BTX >= t.n0 + 1;
        const bool bnd_y = t.j0 == 1 || t.j0 + TY >= t.n1 + 1;
        const bool late = bnd_x || bnd_y;
        const int ci = t.i0 + tid % BTX, cj = t.j0 + tid / BTX;
        // pass 1: the tile, every component; pass 2: the ring components the V update
        // reads, one ring side per warp on the last four warps (one branch path per warp)
        sigma2<T, TY>(t, b, ci, cj, M_ALL);
        {
            constexpr int NW = TL::NT / 32;
            static_assert(NW >= 4 && TY <= 32, "one ring side per warp");
            const int wp = tid / 32, lane = tid % 32;
            int i = 0, j = 0, mask = 0;
            if (wp == NW - 4) { i = t.i0 - 1; j = t.j0 + lane; mask = lane < TY ? (M_P | M_XX) : 0; }
            else if (wp == NW - 3) { i = t.i0 + lane; j = t.j0 - 1; mask = M_P | M_YY; }
            else if (wp == NW - 2) { i = t.i0 + lane; j = t.j0 + TY; mask = M_XY; }
            else if (wp == NW - 1) { i = t.i0 + BTX; j = t.j0 + lane; mask = lane < TY ? M_XY : 0; }
            if (mask && i <= t.n0 + 2 && j <= t.n1 + 2) sigma2<T, TY>(t, b, i, j, mask);
        }
        __syncthreads();
        if (tid == 0 && !failed && w + (kStages - 1) * G < nt) {
            const int nx = cur == 0 ? kStages - 1 : cur - 1;  // the stage of tile k-1
            fence_proxy_async();
            issue_tile<T, TY>(insts, maps, dnext, src, batch_smem + nx * TL::STAGEB, &bars[nx]);
            if (w + kStages * G < nt) dnext = tiles[w + kStages * G];
        }
        const long long Ic = (long long)ci + sx * (long long)cj;
        if (!late) {
            const int a = t.at(ci, cj);
            b.P[dst][Ic] = t.sP[a];
            b.txx[dst][Ic] = t.sXX[a];
            b.tyy[dst][Ic] = t.sYY[a];
            b.txy[dst][Ic] = t.sXY[a];
        } else {
            constexpr int REG = TL::RW * TL::RY;
            // stress boundary conditions on the staged region: the x faces the tile
            // touches (both sides in one pass: their writes and reads are disjoint),
            // then the y faces
            const bool fx[2] = {t.i0 == 1, t.i0 + BTX >= t.n0 + 1}, fy[2] = {t.j0 == 1, t.j0 + TY >= t.n1 + 1};
            bool any_x = false, any_y = false;
            for (int side = 0; side < 2; side++) {
                const int kx = b.bc_kind[0][side], ky = b.bc_kind[1][side];
                any_x |= fx[side] && (kx == FI_BC_TRACTION || kx == FI_BC_SLIP);
                any_y |= fy[side] && (ky == FI_BC_TRACTION || ky == FI_BC_SLIP);
            }
            if (any_x) {
                for (int r = tid; r < REG; r += TL::NT) {
                    const int i = t.i0 - 1 + r % TL::RW, j = t.j0 - 1 + r / TL::RW;
                    const int a = t.at(i, j);
                    for (int side = 0; side < 2; side++) {
                        const int kind = b.bc_kind[0][side];
                        if (!fx[side] || (kind != FI_BC_TRACTION && kind != FI_BC_SLIP)) continue;
                        const int ghost = side == 0 ? 0 : t.n0 + 1, adj = side == 0 ? 1 : t.n0,
                                  node = side == 0 ? 1 : t.n0 + 1;
                        if (kind == FI_BC_TRACTION && i == ghost && j >= 1 && j <= t.n1 && adj >= t.i0 - 1 &&
                            adj <= t.i0 + BTX) {
                            const T tv = T(2.0) * b.bc_val[0][side][0];
                            t.sP[a] = tv - t.sP[t.at(adj, j)];
                            t.sXX[a] = tv - t.sXX[t.at(adj, j)];
                        }
                        if (i == node && j >= 1 && j <= t.n1 + 1) t.sXY[a] = b.bc_val[0][side][1];
                    }
                }
                __syncthreads();
            }
            if (any_y) {
                for (int r = tid; r < REG; r += TL::NT) {
                    const int i = t.i0 - 1 + r % TL::RW, j = t.j0 - 1 + r / TL::RW;
                    const int a = t.at(i, j);
                    for (int side = 0; side < 2; side++) {
                        const int kind = b.bc_kind[1][side];
                        if (!fy[side] || (kind != FI_BC_TRACTION && kind != FI_BC_SLIP)) continue;
                        const int ghost = side == 0 ? 0 : t.n1 + 1, adj = side == 0 ? 1 : t.n1,
                                  node = side == 0 ? 1 : t.n1 + 1;
                        if (kind == FI_BC_TRACTION && j == ghost && adj >= t.j0 - 1 && adj <= t.j0 + TY) {
                            const T tv = T(2.0) * b.bc_val[1][side][1];
                            t.sP[a] = tv - t.sP[t.at(i, adj)];
                            t.sYY[a] = tv - t.sYY[t.at(i, adj)];
                        }
                        if (j == node) t.sXY[a] = b.bc_val[1][side][0];
                    }
                }
                __syncthreads();
            }
            // write-back of the owned region (reads only: the velocity update below
            // reads the same final values, so no barrier in between)
            for (int r = tid; r < REG; r += TL::NT) {
                const int i = t.i0 - 1 + r % TL::RW, j = t.j0 - 1 + r / TL::RW;
                if (i > t.n0 + 2 || j > t.n1 + 2 || !t.own_x(i) || !t.own_y(j)) continue;
                const int a = t.at(i, j);
                const long long I = (long long)i + sx * (long long)j;
                b.P[dst][I] = t.sP[a];
                b.txx[dst][I] = t.sXX[a];
                b.tyy[dst][I] = t.sYY[a];
                b.txy[dst][I] = t.sXY[a];
            }
        }
        // velocity update of the tile (kernels_2d.jl:20-29) with boundary values and ghost images
        if (ci <= t.n0 + 1 && cj <= t.n1 + 1) {
            constexpr int BX = TL::BX;
            const int a = t.at(ci, cj);
            const int xl = b.bc_kind[0][0], xr = b.bc_kind[0][1], yl = b.bc_kind[1][0], yr = b.bc_kind[1][1];
            if (cj <= t.n1) {
                T v;
                if (ci == 1 && node_fixed(xl)) v = b.bc_val[0][0][0];
                else if (ci == t.n0 + 1 && node_fixed(xr)) v = b.bc_val[0][1][0];
                else {
                    const T gx = b.gkind[0] == FI_G_FIELD ? b.gx[Ic] : b.gval[0];
                    const T ex = T(0.5) * (t.sEt[a - 1] + t.sEt[a]);
                    v = t.sVx[a] + div_fast(-(t.sP[a] - t.sP[a - 1]) * b.idx + (t.sXX[a] - t.sXX[a - 1]) * b.idx +
                                               (t.sXY[a + BX] - t.sXY[a]) * b.idy - gx,
                                           ex) *
                                       b.dVx;
                }
                b.Vx[dst][Ic] = v;
                int pos[2];
                T val[2];
                bool okg[2];
                center_ghosts<T>(cj, t.n1, yl, yr, b.bc_val[1][0][0], b.bc_val[1][1][0], pos, val, okg, v, false);
                for (int q = 0; q < 2; q++)
                    if (okg[q]) b.Vx[dst][(long long)ci + sx * (long long)pos[q]] = val[q];
            }
            if (ci <= t.n0) {
                T v;
                const bool y_node = (cj == 1 && node_fixed(yl)) || (cj == t.n1 + 1 && node_fixed(yr));
                if (cj == 1 && node_fixed(yl)) v = b.bc_val[1][0][1];
                else if (cj == t.n1 + 1 && node_fixed(yr)) v = b.bc_val[1][1][1];
                else {
                    const T gy = b.gkind[1] == FI_G_FIELD ? b.gy[Ic] : b.gval[1];
                    const T ey = T(0.5) * (t.sEt[a - BX] + t.sEt[a]);
                    v = t.sVy[a] + div_fast(-(t.sP[a] - t.sP[a - BX]) * b.idy + (t.sYY[a] - t.sYY[a - BX]) * b.idy +
                                               (t.sXY[a + 1] - t.sXY[a]) * b.idx - gy,
                                           ey) *
                                       b.dVy;
                }
                b.Vy[dst][Ic] = v;
                int pos[2];
                T val[2];
                bool okg[2];
                center_ghosts<T>(ci, t.n0, xl, xr, b.bc_val[0][0][1], b.bc_val[0][1][1], pos, val, okg, v, y_node);
                for (int q = 0; q < 2; q++)
                    if (okg[q]) b.Vy[dst][(long long)pos[q] + sx * (long long)cj] = val[q];
            }
        }
        // no closing barrier: the stage of this tile is refilled only after every
        // thread has passed the stress barrier of the next tile
    }
    if (tid == 0 && failed) {
        // drain (bounded) the copies whose wait expired before the stages are
        // released: the last phase waited on per stage (an unused stage passes at once)
        for (int q = 0; q < kStages; q++) mbar_wait(&bars[q], ((phase >> q) & 1u) ^ 1u);
    }
}

__device__ __forceinline__ void fold_max(unsigned long long *slot, double v) {
    // non-negative doubles (and NaN, whose bits exceed +inf) order like their bit patterns
    atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

// FP64 residuals of the active instances' current state (buffer 0)
// (compute_residuals!, kernels_2d.jl:46-54, with the residual boundary batch of
// boundary_conditions.jl:120-128 excluded from the maxima)
template <typename T, int TY>
__global__ void __launch_bounds__(BTX *TY) batch2d_check(const BInst<T> *__restrict__ insts, const int4 *__restrict__ tiles,
                                                         const int *__restrict__ ntiles, unsigned long long *slots) {
    __shared__ double red[kSlots][TY];
    const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
    const int nt = *ntiles;
    for (int w = blockIdx.x; w < nt; w += gridDim.x) {
        const int4 d = tiles[w];
        const BInst<T> &b = insts[d.x];
        const int i = d.y + tid % BTX, j = d.z + tid / BTX;
        const long long sx = b.pitch, I = (long long)i + sx * (long long)j;
        const T *P = b.P[0], *XX = b.txx[0], *YY = b.tyy[0], *XY = b.txy[0], *VX = b.Vx[0], *VY = b.Vy[0];
        const double idx = (double)b.idx, idy = (double)b.idy;
        double m[kSlots] = {0.0, 0.0, 0.0, 0.0};
        if (i <= b.n0 + 1 && j <= b.n1 + 1) {
            const bool ci = i <= b.n0, cj = j <= b.n1;
            if (ci && cj) {
                double rP = ((double)VX[I + 1] - (double)VX[I]) * idx + ((double)VY[I + sx] - (double)VY[I]) * idy;
                if (b.pforce) rP = rP + (double)b.fP[I];
                m[0] = fabs(rP);
                m[2] = fmax(fmax(fabs((double)P[I]), fabs((double)XX[I])), fabs((double)YY[I]));
            }
            m[2] = fmax(m[2], fabs((double)XY[I]));
            const bool fx_l = b.bc_kind[0][0] != FI_BC_TRACTION, fx_r = b.bc_kind[0][1] != FI_BC_TRACTION;
            const bool fy_l = b.bc_kind[1][0] != FI_BC_TRACTION, fy_r = b.bc_kind[1][1] != FI_BC_TRACTION;
            if (cj) {
                m[3] = fabs((double)VX[I]);
                if (!((i == 1 && fx_l) || (i == b.n0 + 1 && fx_r))) {
                    const double gx = b.gkind[0] == FI_G_FIELD ? (double)b.gx[I] : (double)b.gval[0];
                    const double r = -((double)P[I] - (double)P[I - 1]) * idx + ((double)XX[I] - (double)XX[I - 1]) * idx +
                                     ((double)XY[I + sx] - (double)XY[I]) * idy - gx;
                    m[1] = fabs(r);
                }
            }
            if (ci) {
                m[3] = fmax(m[3], fabs((double)VY[I]));
                if (!((j == 1 && fy_l) || (j == b.n1 + 1 && fy_r))) {
                    const double gy = b.gkind[1] == FI_G_FIELD ? (double)b.gy[I] : (double)b.gval[1];
                    const double r = -((double)P[I] - (double)P[I - sx]) * idy + ((double)YY[I] - (double)YY[I - sx]) * idy +
                                     ((double)XY[I + 1] - (double)XY[I]) * idx - gy;
                    m[1] = fmax(m[1], fabs(r));
                }
            }
        }
        // NaN-propagating maxima: fmax drops NaN, so carry it explicitly
        for (int q = 0; q < kSlots; q++) {
            double v = m[q];
            for (int o = 16; o > 0; o >>= 1) {
                const double u = __shfl_xor_sync(0xffffffffu, v, o);
                v = (isnan(u) || u > v) ? u : v;
            }
            if (lane == 0) red[q][warp] = v;
        }
        __syncthreads();
        if (tid < kSlots) {
            double v = red[tid][0];
            for (int q = 1; q < TY; q++) v = (isnan(red[tid][q]) || red[tid][q] > v) ? red[tid][q] : v;
            fold_max(&slots[(long long)d.x * kSlots + tid], v);
        }
        __syncthreads();
    }
}

// per-instance bookkeeping after a check: measure, retirement, slot reset
__global__ void batch_update(int count, const double *__restrict__ h, unsigned long long *slots, BState *st, int k,
                             double tol, int window, int max_iter) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    BState s = st[q];
    if (s.status == FI_ITEM_ACTIVE) {
        double v[kSlots];
        for (int c = 0; c < kSlots; c++) v[c] = __longlong_as_double((long long)slots[(long long)q * kSlots + c]);
        s.iters += k;
        const double rV = v[1] * h[q], rP = v[0] * h[q];
        const double meas = fmax(v[2] > 0.0 ? rV / v[2] : rV, v[3] > 0.0 ? rP / v[3] : rP);
        s.measure = meas;
        if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2]) || !isfinite(v[3])) {
            s.status = FI_ITEM_DIVERGED;
        } else if (meas < tol) {
            s.status = FI_ITEM_CONVERGED;
        } else {
            if (meas < 0.5 * s.best) {
                s.best = meas;
                s.since = 0;
            } else {
                s.since += k;
            }
            if (window > 0 && s.since >= window) s.status = FI_ITEM_STALLED;
            else if (s.iters >= max_iter) s.status = FI_ITEM_MAXITER;
        }
        st[q] = s;
    }
    for (int c = 0; c < kSlots; c++) slots[(long long)q * kSlots + c] = 0ull;
}

// work-list compaction, step 1 (one block): tile offsets of the active instances
__global__ void batch_scan(int count, const int *__restrict__ tile_count, const BState *__restrict__ st, int *offset,
                           int *ntiles, int *nactive) {
    __shared__ int part[1024];
    const int tid = threadIdx.x, per = (count + blockDim.x - 1) / blockDim.x;
    const int lo = tid * per, hi = min(lo + per, count);
    int sum = 0, act = 0;
    for (int q = lo; q < hi; q++)
        if (st[q].status == FI_ITEM_ACTIVE) {
            sum += tile_count[q];
            act++;
        }
    part[tid] = sum;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {  // inclusive Hillis-Steele scan
        int v = tid >= o ? part[tid - o] : 0;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    int run = part[tid] - sum;
    for (int q = lo; q < hi; q++) {
        offset[q] = run;
        if (st[q].status == FI_ITEM_ACTIVE) run += tile_count[q];
    }
    if (tid == blockDim.x - 1) *ntiles = part[tid];
    // active count: a second reduction over the same layout
    __syncthreads();
    part[tid] = act;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (tid < o) part[tid] += part[tid + o];
        __syncthreads();
    }
    if (tid == 0) *nactive = part[0];
}

// step 2: copy the active instances' tiles from the full list
__global__ void batch_fill(int total, const int4 *__restrict__ all, const int *__restrict__ first,
                           const int *__restrict__ offset, const BState *__restrict__ st, int4 *out) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        const int4 d = all[g];
        if (st[d.x].status == FI_ITEM_ACTIVE) out[offset[d.x] + (g - first[d.x])] = d;
    }
}

template <typename T, int TY>
constexpr size_t sweep_smem() {
    return kStages * (size_t)Tile<T, TY>::STAGEB + kStages * sizeof(uint64_t);
}

// resident sweep CTAs per SM (queried once per instantiation, outside any capture;
// also lifts the dynamic shared-memory limit where the two staging buffers need it)
template <typename T, int TY>
int sweep_blocks_per_sm() {
    static const int nb = [] {
        cudaFuncSetAttribute(batch2d_sweep<T, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sweep_smem<T, TY>());
        int v = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, batch2d_sweep<T, TY>, BTX * TY, sweep_smem<T, TY>()) !=
            cudaSuccess)
            v = 1;
        return std::max(v, 1);
    }();
    return nb;
}

}  // namespace
}  // namespace fi

using namespace fi;

struct fi_batch {
    std::vector<fi_model *> models;
    std::vector<BState> h_state;  // host copy of the members' solve state (valid when !state_on_device)
    bool state_on_device = false;
    bool dirty = true;            // membership changed: per-member arrays, tile lists and graph are stale
    bool f64 = false;
    int device = 0;
    int sms = 148;
    int variant = 0;
    int capacity = 0;
    cudaStream_t stream = nullptr;
    void *d_inst = nullptr;               // BInst<T>[capacity]
    BMaps *d_maps = nullptr;              // per-member tensor maps [capacity]
    std::vector<BMaps> h_maps;
    int maps_ty = -1;
    int *d_err = nullptr;                 // device error word (bounded waits)
    std::vector<unsigned char> h_inst;    // host image of the table
    int4 *d_all = nullptr, *d_work = nullptr;
    int tile_capacity = 0;
    int *d_first = nullptr, *d_count = nullptr, *d_offset = nullptr;
    int *d_ntiles = nullptr, *d_nactive = nullptr, *h_nactive = nullptr;
    int *d_full_ntiles = nullptr;
    double *d_h = nullptr;
    unsigned long long *d_slots = nullptr;
    BState *d_state = nullptr;
    int total_tiles = 0;
    int list_ty = -1;
    cudaGraphExec_t graph = nullptr;
    int graph_k = -1, graph_ty = -1;
    double graph_tol = -1;
    int graph_window = -1, graph_max = -1;
    int count() const { return (int)models.size(); }
};

namespace {

#define FB_CHECK(expr, where)                                \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, where);  \
    } while (0)

BState fresh_state() {
    BState s;
    s.status = FI_ITEM_ACTIVE;
    s.iters = 0;
    s.since = 0;
    s.pad = 0;
    s.best = 1e300;
    s.measure = 0.0;
    return s;
}

template <typename T>
void fill_inst(const fi_model *m, BInst<T> &b) {
    std::memset(&b, 0, sizeof(b));
    b.n0 = m->d.grid.n[0];
    b.n1 = m->d.grid.n[1];
    b.pitch = m->g.pitch;
    const KParams &p = m->kp;
    b.idx = T(p.inv_dx[0]);
    b.idy = T(p.inv_dx[1]);
    b.dtP = T(p.dt_P);
    b.dxx = T(p.dt_tau[0]);
    b.dyy = T(p.dt_tau[1]);
    b.dxy = T(p.dt_tau[3]);
    b.dVx = T(p.dt_V[0]);
    b.dVy = T(p.dt_V[1]);
    for (int c = 0; c < 2; c++) {
        b.gkind[c] = p.g_kind[c];
        b.gval[c] = T(p.g_val[c]);
    }
    for (int d = 0; d < 2; d++)
        for (int s = 0; s < 2; s++) {
            b.bc_kind[d][s] = p.bc_kind[d][s];
            for (int c = 0; c < 2; c++) b.bc_val[d][s][c] = T(p.bc_val[d][s][c]);
        }
    const int F[6] = {FI_FIELD_P, FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TXY, FI_FIELD_VX, FI_FIELD_VY};
    T **dst[6] = {b.P, b.txx, b.tyy, b.txy, b.Vx, b.Vy};
    for (int q = 0; q < 6; q++) {
        dst[q][0] = (T *)m->cur(F[q]);
        dst[q][1] = (T *)m->nxt(F[q]);
    }
    b.eta = (const T *)m->cur(FI_FIELD_ETA);
    b.gx = (const T *)m->base[FI_FIELD_GX];
    b.gy = (const T *)m->base[FI_FIELD_GY];
    b.fP = (const T *)m->fP;
    b.pforce = p.p_forcing && m->fP ? 1 : 0;
    b.h = std::min(1.0 / p.inv_dx[0], 1.0 / p.inv_dx[1]);
}

fi_status validate_member(const fi_batch *b, const fi_model *m) {
    if (!m) return set_error("null model in the batch"), FI_ERR_ARG;
    const fi_model_desc &d = m->d;
    if (d.grid.nd != 2) return set_error("the batched solver takes 2D models"), FI_ERR_UNSUPPORTED;
    if (m->ib) return set_error("the batched solver does not cover the immersed-boundary model"), FI_ERR_UNSUPPORTED;
    if (d.rheology.inner != FI_RHEO_LINEAR || d.rheology.has_reg || d.rheology.relax != FI_RELAX_NONE)
        return set_error("the batched solver holds the viscosity fixed: linear rheology only"), FI_ERR_UNSUPPORTED;
    for (int k = 0; k < 2; k++)
        for (int s = 0; s < 2; s++)
            if (d.bc[k][s].kind == FI_BC_PERIODIC)
                return set_error("the batched solver does not cover periodic sides"), FI_ERR_UNSUPPORTED;
    if ((d.dtype == FI_F64) != b->f64) return set_error("all batch members need one dtype"), FI_ERR_ARG;
    if (d.device != b->device) return set_error("all batch members need one device"), FI_ERR_ARG;
    for (const fi_model *o : b->models)
        if (o == m) return set_error("a model appears twice in the batch"), FI_ERR_ARG;
    return FI_OK;
}

// the members' solve state back on the host (before membership changes)
fi_status pull_state(fi_batch *b) {
    if (!b->state_on_device) return FI_OK;
    b->h_state.resize(b->count());
    if (b->count() > 0)
        FB_CHECK(cudaMemcpy(b->h_state.data(), b->d_state, sizeof(BState) * b->count(), cudaMemcpyDeviceToHost),
                 "batch state");
    b->state_on_device = false;
    return FI_OK;
}

template <typename P>
cudaError_t grow(P **ptr, size_t n) {
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    return cudaMalloc(ptr, std::max<size_t>(n, 1) * sizeof(P));
}

// per-member device arrays sized for the current membership
fi_status ensure_capacity(fi_batch *b) {
    const int n = b->count();
    if (n <= b->capacity) return FI_OK;
    const int cap = std::max(n, 2 * b->capacity);
    const size_t esz = b->f64 ? sizeof(BInst<double>) : sizeof(BInst<float>);
    if (b->d_inst) cudaFree(b->d_inst);
    b->d_inst = nullptr;
    FB_CHECK(cudaMalloc(&b->d_inst, esz * cap), "batch table");
    FB_CHECK(grow(&b->d_maps, cap), "batch tensor maps");
    FB_CHECK(grow(&b->d_first, cap), "batch arrays");
    FB_CHECK(grow(&b->d_count, cap), "batch arrays");
    FB_CHECK(grow(&b->d_offset, cap), "batch arrays");
    FB_CHECK(grow(&b->d_h, cap), "batch arrays");
    FB_CHECK(grow(&b->d_slots, (size_t)kSlots * cap), "batch arrays");
    FB_CHECK(cudaMemset(b->d_slots, 0, sizeof(unsigned long long) * kSlots * cap), "batch arrays");
    FB_CHECK(grow(&b->d_state, cap), "batch arrays");
    b->capacity = cap;
    return FI_OK;
}

// instance table from the models' current buffers (index 0 = current state)
fi_status upload_table(fi_batch *b) {
    const int n = b->count();
    const size_t esz = b->f64 ? sizeof(BInst<double>) : sizeof(BInst<float>);
    b->h_inst.resize(esz * std::max(n, 1));
    std::vector<double> hs(std::max(n, 1));
    for (int q = 0; q < n; q++) {
        if (b->f64) {
            BInst<double> v;
            fill_inst<double>(b->models[q], v);
            std::memcpy(b->h_inst.data() + q * esz, &v, esz);
            hs[q] = v.h;
        } else {
            BInst<float> v;
            fill_inst<float>(b->models[q], v);
            std::memcpy(b->h_inst.data() + q * esz, &v, esz);
            hs[q] = v.h;
        }
    }
    if (n == 0) return FI_OK;
    // tensor maps of every member's buffers, box = one tile of the current variant
    const int ty = kBatchTY[b->variant];
    const int bx = b->f64 ? BBox<double>::BX : BBox<float>::BX;
    const int ez = b->f64 ? 8 : 4;
    b->h_maps.resize(n);
    const int F[6] = {FI_FIELD_P, FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TXY, FI_FIELD_VX, FI_FIELD_VY};
    for (int q = 0; q < n; q++) {
        const fi_model *m = b->models[q];
        const unsigned long long dims[2] = {(unsigned long long)m->g.pitch, (unsigned long long)m->g.rows};
        const unsigned long long strides[1] = {(unsigned long long)(m->g.pitch * ez)};
        const unsigned box[2] = {(unsigned)bx, (unsigned)(ty + 2)};
        for (int buf = 0; buf < 2; buf++) {
            for (int f = 0; f < 7; f++) {
                void *ptr = f < 6 ? (buf == 0 ? m->cur(F[f]) : m->nxt(F[f])) : m->cur(FI_FIELD_ETA);
                void *raw = (char *)ptr - kXOff * ez;
                if (!tma_encode(raw, 2, dims, strides, box, ez, b->h_maps[q].m[buf][f]))
                    return set_error("tensor map encoding failed (batch member)"), FI_ERR_CUDA;
            }
        }
    }
    b->maps_ty = ty;
    FB_CHECK(cudaMemcpy(b->d_maps, b->h_maps.data(), sizeof(BMaps) * n, cudaMemcpyHostToDevice), "batch tensor maps");
    FB_CHECK(cudaMemcpy(b->d_inst, b->h_inst.data(), esz * n, cudaMemcpyHostToDevice), "batch table");
    FB_CHECK(cudaMemcpy(b->d_h, hs.data(), sizeof(double) * n, cudaMemcpyHostToDevice), "batch spacings");
    return FI_OK;
}

// full tile list for tile height ty (all members); the work list starts as its copy
fi_status build_tiles(fi_batch *b, int ty) {
    if (b->list_ty == ty && !b->dirty) return FI_OK;
    const int n = b->count();
    std::vector<int4> all;
    std::vector<int> first(std::max(n, 1)), cnt(std::max(n, 1));
    for (int q = 0; q < n; q++) {
        const fi_model *m = b->models[q];
        const int n0 = m->d.grid.n[0], n1 = m->d.grid.n[1];
        first[q] = (int)all.size();
        for (int j0 = 1; j0 <= n1 + 1; j0 += ty)
            for (int i0 = 1; i0 <= n0 + 1; i0 += BTX) all.push_back(make_int4(q, i0, j0, 0));
        cnt[q] = (int)all.size() - first[q];
    }
    if ((int)all.size() > b->tile_capacity) {
        const int cap = std::max((int)all.size(), 2 * b->tile_capacity);
        FB_CHECK(grow(&b->d_all, cap), "tile list");
        FB_CHECK(grow(&b->d_work, cap), "work list");
        b->tile_capacity = cap;
    }
    b->total_tiles = (int)all.size();
    if (!all.empty()) {
        FB_CHECK(cudaMemcpy(b->d_all, all.data(), sizeof(int4) * all.size(), cudaMemcpyHostToDevice), "tile list");
        FB_CHECK(cudaMemcpy(b->d_work, all.data(), sizeof(int4) * all.size(), cudaMemcpyHostToDevice), "work list");
        FB_CHECK(cudaMemcpy(b->d_first, first.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "tile offsets");
        FB_CHECK(cudaMemcpy(b->d_count, cnt.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "tile counts");
    }
    int tot = b->total_tiles;
    FB_CHECK(cudaMemcpy(b->d_full_ntiles, &tot, sizeof(int), cudaMemcpyHostToDevice), "tile total");
    FB_CHECK(cudaMemcpy(b->d_ntiles, &tot, sizeof(int), cudaMemcpyHostToDevice), "tile total");
    b->list_ty = ty;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return FI_OK;
}

template <typename T, int TY>
cudaError_t launch_sweep_t(fi_batch *b, const int4 *list, const int *nt, int src) {
    const int grid = b->sms * sweep_blocks_per_sm<T, TY>();
    batch2d_sweep<T, TY><<<grid, BTX * TY, sweep_smem<T, TY>(), b->stream>>>((const BInst<T> *)b->d_inst, b->d_maps,
                                                                               list, nt, src, b->d_err);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_sweep_ty(fi_batch *b, const int4 *list, const int *nt, int src) {
    switch (kBatchTY[b->variant]) {
        case 4: return launch_sweep_t<T, 4>(b, list, nt, src);
        case 16: return launch_sweep_t<T, 16>(b, list, nt, src);
        default: return launch_sweep_t<T, 8>(b, list, nt, src);
    }
}
cudaError_t launch_sweep(fi_batch *b, const int4 *list, const int *nt, int src) {
    return b->f64 ? launch_sweep_ty<double>(b, list, nt, src) : launch_sweep_ty<float>(b, list, nt, src);
}

template <typename T, int TY>
cudaError_t launch_check_t(fi_batch *b, const int4 *list, const int *nt) {
    batch2d_check<T, TY><<<b->sms * 8, BTX * TY, 0, b->stream>>>((const BInst<T> *)b->d_inst, list, nt, b->d_slots);
    return cudaGetLastError();
}
cudaError_t launch_check(fi_batch *b, const int4 *list, const int *nt) {
    const int ty = kBatchTY[b->variant];
    if (b->f64)
        return ty == 4 ? launch_check_t<double, 4>(b, list, nt)
                       : ty == 16 ? launch_check_t<double, 16>(b, list, nt) : launch_check_t<double, 8>(b, list, nt);
    return ty == 4 ? launch_check_t<float, 4>(b, list, nt)
                   : ty == 16 ? launch_check_t<float, 16>(b, list, nt) : launch_check_t<float, 8>(b, list, nt);
}

// rebuild the work list from the members' state (scan + fill)
cudaError_t enqueue_compaction(fi_batch *b) {
    batch_scan<<<1, 1024, 0, b->stream>>>(b->count(), b->d_count, b->d_state, b->d_offset, b->d_ntiles, b->d_nactive);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    batch_fill<<<std::max(1, std::min((b->total_tiles + 255) / 256, b->sms * 8)), 256, 0, b->stream>>>(
        b->total_tiles, b->d_all, b->d_first, b->d_offset, b->d_state, b->d_work);
    return cudaGetLastError();
}

// one check-to-check step: k sweeps, the check, bookkeeping, compaction
cudaError_t enqueue_round(fi_batch *b, int k, double tol, int window, int max_iter) {
    cudaError_t e;
    for (int s = 0; s < k; s++)
        if ((e = launch_sweep(b, b->d_work, b->d_ntiles, s & 1)) != cudaSuccess) return e;
    if ((e = launch_check(b, b->d_work, b->d_ntiles)) != cudaSuccess) return e;
    batch_update<<<(b->count() + 255) / 256, 256, 0, b->stream>>>(b->count(), b->d_h, b->d_slots, b->d_state, k, tol,
                                                                   window, max_iter);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return enqueue_compaction(b);
}

// make the device arrays, tables and lists match the membership; state pushed to the device
fi_status prepare(fi_batch *b) {
    FB_CHECK(cudaSetDevice(b->device), "cudaSetDevice");
    fi_status st;
    for (fi_model *m : b->models) {
        FB_CHECK(cudaStreamSynchronize(m->stream), "model stream");
        if ((st = model_ensure_second_state(m)) != FI_OK) return st;
    }
    if (b->dirty) {
        if ((st = pull_state(b)) != FI_OK) return st;
        if ((st = ensure_capacity(b)) != FI_OK) return st;
    }
    if ((st = upload_table(b)) != FI_OK) return st;
    if ((st = build_tiles(b, kBatchTY[b->variant])) != FI_OK) return st;
    if (!b->state_on_device) {
        if (b->count() > 0)
            FB_CHECK(cudaMemcpy(b->d_state, b->h_state.data(), sizeof(BState) * b->count(), cudaMemcpyHostToDevice),
                     "batch state");
        b->state_on_device = true;
    }
    b->dirty = false;
    return FI_OK;
}

void free_batch(fi_batch *b) {
    if (!b) return;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    void *ptrs[] = {b->d_inst, b->d_all, b->d_work, b->d_first, b->d_count, b->d_offset, b->d_ntiles,
                    b->d_nactive, b->d_full_ntiles, b->d_h, b->d_slots, b->d_state, b->d_maps, b->d_err};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (b->h_nactive) cudaFreeHost(b->h_nactive);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

void finish_sweeps(fi_batch *b, const std::vector<int> &sweeps) {
    for (int q = 0; q < b->count(); q++) {
        if (sweeps[q] & 1) b->models[q]->parity ^= 1;
        b->models[q]->iterations += sweeps[q];
    }
}

// the sweep's error word (a bounded wait that expired), cleared after reading
fi_status check_batch_err(fi_batch *b) {
    int e = 0;
    FB_CHECK(cudaMemcpy(&e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost), "batch error word");
    if (e == 0) return FI_OK;
    cudaMemset(b->d_err, 0, sizeof(int));
    set_error("batched sweep: a tile's copies did not arrive within the wait bound");
    return (fi_status)e;
}

// check rounds until no member is active or max_rounds; items/nactive may be NULL
fi_status run_rounds(fi_batch *b, const fi_batch_opts *o, int max_rounds, fi_batch_item *items, int32_t *nactive) {
    const int n = b->count();
    std::vector<BState> before(n);
    if (n > 0)
        FB_CHECK(cudaMemcpy(before.data(), b->d_state, sizeof(BState) * n, cudaMemcpyDeviceToHost), "batch state");
    FB_CHECK(enqueue_compaction(b), "work list");
    FB_CHECK(cudaMemcpyAsync(b->h_nactive, b->d_nactive, sizeof(int), cudaMemcpyDeviceToHost, b->stream), "active");
    FB_CHECK(cudaStreamSynchronize(b->stream), "batch sync");
    const int window = o->window > 0 ? o->window : 0;
    const bool use_graph = o->use_graph != 0;
    if (use_graph && *b->h_nactive > 0 &&
        (!b->graph || b->graph_k != o->ncheck || b->graph_ty != kBatchTY[b->variant] || b->graph_tol != o->tol ||
         b->graph_window != window || b->graph_max != o->max_iter)) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaGraph_t g = nullptr;
        FB_CHECK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
        cudaError_t ce = enqueue_round(b, o->ncheck, o->tol, window, o->max_iter);
        cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
        if (ce != cudaSuccess) return cuda_fail(ce, "graph capture");
        if (ee != cudaSuccess) return cuda_fail(ee, "graph capture");
        cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return cuda_fail(ie, "graph instantiate");
        b->graph_k = o->ncheck;
        b->graph_ty = kBatchTY[b->variant];
        b->graph_tol = o->tol;
        b->graph_window = window;
        b->graph_max = o->max_iter;
    }
    for (int r = 0; r < max_rounds && *b->h_nactive > 0; r++) {
        if (use_graph) FB_CHECK(cudaGraphLaunch(b->graph, b->stream), "graph launch");
        else FB_CHECK(enqueue_round(b, o->ncheck, o->tol, window, o->max_iter), "batch round");
        FB_CHECK(cudaMemcpyAsync(b->h_nactive, b->d_nactive, sizeof(int), cudaMemcpyDeviceToHost, b->stream), "active");
        FB_CHECK(cudaStreamSynchronize(b->stream), "batch sync");
    }
    std::vector<BState> fin(n);
    if (n > 0) FB_CHECK(cudaMemcpy(fin.data(), b->d_state, sizeof(BState) * n, cudaMemcpyDeviceToHost), "batch state");
    const fi_status es = check_batch_err(b);
    std::vector<int> sw(n);
    for (int q = 0; q < n; q++) {
        if (items) {
            items[q].iterations = fin[q].iters;
            items[q].status = fin[q].status;
            items[q].measure = fin[q].measure;
        }
        sw[q] = fin[q].iters - before[q].iters;
    }
    finish_sweeps(b, sw);
    if (nactive) *nactive = *b->h_nactive;
    return es;
}

fi_status check_opts(const fi_batch_opts *o) {
    if (o->ncheck <= 0 || (o->ncheck & 1)) return set_error("ncheck must be a positive even number"), FI_ERR_ARG;
    if (o->max_iter <= 0) return set_error("max_iter must be positive"), FI_ERR_ARG;
    return FI_OK;
}

}  // namespace

extern "C" {

int fi_batch_variant_count(void) { return kBatchVariants; }

const char *fi_batch_variant_name(int32_t v) {
    static char buf[kBatchVariants][24];
    if (v < 0 || v >= kBatchVariants) return "?";
    snprintf(buf[v], sizeof(buf[v]), "tile32x%d", kBatchTY[v]);
    return buf[v];
}

fi_status fi_batch_create(fi_model *const *models, int32_t count, fi_batch **out) {
    if (!out || count < 0 || (count > 0 && !models)) return set_error("bad argument"), FI_ERR_ARG;
    *out = nullptr;
    if (count == 0) return set_error("fi_batch_create needs a first member (it fixes dtype and device)"), FI_ERR_ARG;
    fi_batch *b = new fi_batch();
    b->f64 = models[0] && models[0]->d.dtype == FI_F64;
    b->device = models[0] ? models[0]->d.device : 0;
    for (int q = 0; q < count; q++) {
        fi_status st = validate_member(b, models[q]);
        if (st != FI_OK) {
            delete b;
            return st;
        }
        b->models.push_back(models[q]);
        b->h_state.push_back(fresh_state());
    }
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_ntiles, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_full_ntiles, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_nactive, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_nactive, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        fi_status st = cuda_fail(e, "batch allocation");
        free_batch(b);
        return st;
    }
    fi_status st = prepare(b);
    if (st != FI_OK) {
        free_batch(b);
        return st;
    }
    *out = b;
    return FI_OK;
}

fi_status fi_batch_destroy(fi_batch *b) {
    if (!b) return FI_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    free_batch(b);
    return FI_OK;
}

fi_status fi_batch_add(fi_batch *b, fi_model *m) {
    if (!b) return set_error("bad argument"), FI_ERR_ARG;
    fi_status st = validate_member(b, m);
    if (st != FI_OK) return st;
    FB_CHECK(cudaSetDevice(b->device), "cudaSetDevice");
    if ((st = pull_state(b)) != FI_OK) return st;
    b->models.push_back(m);
    b->h_state.push_back(fresh_state());
    b->dirty = true;
    return FI_OK;
}

fi_status fi_batch_remove(fi_batch *b, fi_model *m) {
    if (!b || !m) return set_error("bad argument"), FI_ERR_ARG;
    auto it = std::find(b->models.begin(), b->models.end(), m);
    if (it == b->models.end()) return set_error("the model is not a member of the batch"), FI_ERR_ARG;
    FB_CHECK(cudaSetDevice(b->device), "cudaSetDevice");
    FB_CHECK(cudaStreamSynchronize(b->stream), "batch sync");
    fi_status st = pull_state(b);
    if (st != FI_OK) return st;
    const size_t q = (size_t)(it - b->models.begin());
    b->models.erase(it);
    b->h_state.erase(b->h_state.begin() + q);
    b->dirty = true;
    return FI_OK;
}

int32_t fi_batch_size(const fi_batch *b) { return b ? b->count() : 0; }

fi_status fi_batch_advance(fi_batch *b, int32_t niter) {
    if (!b || niter < 0) return set_error("bad argument"), FI_ERR_ARG;
    fi_status st = prepare(b);
    if (st != FI_OK) return st;
    for (int s = 0; s < niter; s++) FB_CHECK(launch_sweep(b, b->d_all, b->d_full_ntiles, s & 1), "batch sweep");
    FB_CHECK(cudaStreamSynchronize(b->stream), "batch sync");
    finish_sweeps(b, std::vector<int>(b->count(), niter));
    return check_batch_err(b);
}

fi_status fi_batch_set_variant(fi_batch *b, int32_t v) {
    if (!b || v < 0 || v >= kBatchVariants) return set_error("bad argument"), FI_ERR_ARG;
    b->variant = v;
    return FI_OK;
}

fi_status fi_batch_autotune(fi_batch *b, int32_t iters, int32_t *best, double *ms) {
    if (!b || iters <= 0 || !best) return set_error("bad argument"), FI_ERR_ARG;
    FB_CHECK(cudaSetDevice(b->device), "cudaSetDevice");
    cudaEvent_t e0, e1;
    FB_CHECK(cudaEventCreate(&e0), "event");
    FB_CHECK(cudaEventCreate(&e1), "event");
    double best_ms = 1e300;
    int best_v = 0;
    fi_status st = FI_OK;
    for (int v = 0; v < kBatchVariants && st == FI_OK; v++) {
        b->variant = v;
        if ((st = fi_batch_advance(b, 2)) != FI_OK) break;  // warm-up (and the variant's tile list)
        cudaEventRecord(e0, b->stream);
        for (int s = 0; s < iters; s++) launch_sweep(b, b->d_all, b->d_full_ntiles, s & 1);
        cudaEventRecord(e1, b->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "autotune");
            break;
        }
        finish_sweeps(b, std::vector<int>(b->count(), iters));
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        const double per = t / iters;
        if (ms) ms[v] = per;
        if (per < best_ms) {
            best_ms = per;
            best_v = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != FI_OK) return st;
    if ((st = check_batch_err(b)) != FI_OK) return st;
    b->variant = best_v;
    *best = best_v;
    return FI_OK;
}

fi_status fi_batch_solve(fi_batch *b, const fi_batch_opts *o, fi_batch_item *items, double *seconds) {
    if (!b || !o || !items) return set_error("bad argument"), FI_ERR_ARG;
    fi_status st = check_opts(o);
    if (st != FI_OK) return st;
    auto t0 = std::chrono::steady_clock::now();
    if ((st = pull_state(b)) != FI_OK) return st;
    for (auto &s : b->h_state) s = fresh_state();
    if ((st = prepare(b)) != FI_OK) return st;
    FB_CHECK(cudaMemsetAsync(b->d_slots, 0, sizeof(unsigned long long) * kSlots * b->count(), b->stream), "slots");
    const int max_rounds = (o->max_iter + o->ncheck - 1) / o->ncheck;
    if ((st = run_rounds(b, o, max_rounds, items, nullptr)) != FI_OK) return st;
    for (int q = 0; q < b->count(); q++)
        if (items[q].status == FI_ITEM_ACTIVE) items[q].status = FI_ITEM_MAXITER;
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return FI_OK;
}

fi_status fi_batch_step(fi_batch *b, const fi_batch_opts *o, int32_t max_rounds, fi_batch_item *items,
                        int32_t *nactive) {
    if (!b || !o || max_rounds < 0) return set_error("bad argument"), FI_ERR_ARG;
    fi_status st = check_opts(o);
    if (st != FI_OK) return st;
    if ((st = prepare(b)) != FI_OK) return st;
    return run_rounds(b, o, max_rounds, items, nactive);
}

constexpr double kPhaseATol = 2e-4;

fi_status fi_batch_solve_mixed(fi_batch *b, const fi_batch_opts *o, double inner_tol, fi_batch_item *items,
                               double *seconds) {
    if (!b || !o || !items) return set_error("bad argument"), FI_ERR_ARG;
    if (!b->f64) return set_error("the mixed-precision batch refines FP64 members"), FI_ERR_ARG;
    fi_status st = check_opts(o);
    if (st != FI_OK) return st;
    const double corr_tol = inner_tol > 0 ? inner_tol : 1e-3;
    auto t0 = std::chrono::steady_clock::now();
    const int n = b->count();
    if ((st = pull_state(b)) != FI_OK) return st;
    std::vector<fi_model *> shadows(n);
    for (int q = 0; q < n; q++) {
        if ((st = mixed_shadow(b->models[q])) != FI_OK) return st;
        shadows[q] = b->models[q]->shadow;
    }
    fi_batch *sb = nullptr;
    if ((st = fi_batch_create(shadows.data(), n, &sb)) != FI_OK) return st;
    struct Guard {
        fi_batch *p;
        ~Guard() { fi_batch_destroy(p); }
    } guard{sb};
    sb->variant = b->variant;
    std::vector<int> sweeps(n, 0), status(n, FI_ITEM_ACTIVE), stale(n, 0);
    std::vector<double> best(n, 1e300), meas(n, 0.0);
    std::vector<fi_batch_item> it(n);
    // phase A: every member's full problem in FP32 storage, batched, to the measure
    // kPhaseATol (above the FP32 rounding floor of these measures, 2e-5 at 255^2 and
    // growing with the grid; the stall window ends a member that meets its floor
    // first).  PT contracts the residual at a fixed rate per sweep, so stopping here
    // and reducing the rest by corrections costs no more sweeps than going on.
    for (int q = 0; q < n; q++)
        if ((st = mixed_phase_a_begin(b->models[q])) != FI_OK) return st;
    fi_batch_opts oa = *o;
    oa.tol = std::max(o->tol, kPhaseATol);
    if ((st = fi_batch_solve(sb, &oa, it.data(), nullptr)) != FI_OK) return st;
    for (int q = 0; q < n; q++) {
        sweeps[q] += it[q].iterations;
        if ((st = mixed_phase_a_end(b->models[q])) != FI_OK) return st;
        if (it[q].status == FI_ITEM_DIVERGED) {
            status[q] = FI_ITEM_DIVERGED;
            if ((st = fi_batch_remove(sb, shadows[q])) != FI_OK) return st;
        }
    }
    // FP64 defect correction: every outer step measures the FP64 members, retires the
    // converged ones and runs the corrections of the others as one FP32 batch
    while (true) {
        if ((st = fi_batch_measure(b, meas.data())) != FI_OK) return st;
        std::vector<fi_model *> act;
        for (int q = 0; q < n; q++) {
            if (status[q] != FI_ITEM_ACTIVE) continue;
            if (!std::isfinite(meas[q])) status[q] = FI_ITEM_DIVERGED;
            else if (meas[q] < o->tol) status[q] = FI_ITEM_CONVERGED;
            else if (sweeps[q] >= o->max_iter) status[q] = FI_ITEM_MAXITER;
            else {
                // three outer steps without halving the FP64 measure: the corrections no
                // longer reach the residual
                if (meas[q] < 0.5 * best[q]) stale[q] = 0;
                else if (++stale[q] >= 3) status[q] = FI_ITEM_STALLED;
                best[q] = std::min(best[q], meas[q]);
            }
            if (status[q] == FI_ITEM_ACTIVE) act.push_back(b->models[q]);
            else if ((st = fi_batch_remove(sb, shadows[q])) != FI_OK && st != FI_ERR_ARG) return st;
        }
        if (act.empty()) break;
        for (fi_model *m : act) {
            if ((st = mixed_picard(m)) != FI_OK) return st;
            if ((st = mixed_correction_begin(m)) != FI_OK) return st;
        }
        fi_batch_opts oc = *o;
        oc.tol = corr_tol;
        std::vector<fi_batch_item> ic(sb->count());
        if ((st = fi_batch_solve(sb, &oc, ic.data(), nullptr)) != FI_OK) return st;
        for (int k = 0; k < sb->count(); k++) {
            int q = 0;
            while (shadows[q] != sb->models[k]) q++;
            sweeps[q] += ic[k].iterations;
            if (ic[k].status == FI_ITEM_DIVERGED) status[q] = FI_ITEM_DIVERGED;
        }
        for (fi_model *m : act)
            if ((st = mixed_correction_end(m)) != FI_OK) return st;
        for (fi_model *m : act) FB_CHECK(cudaStreamSynchronize(m->stream), "accumulate");
    }
    for (int q = 0; q < n; q++) {
        items[q].iterations = sweeps[q];
        items[q].status = status[q];
        items[q].measure = meas[q];
    }
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return FI_OK;
}

fi_status fi_batch_measure(fi_batch *b, double *out) {
    if (!b || !out) return set_error("bad argument"), FI_ERR_ARG;
    fi_status st = prepare(b);
    if (st != FI_OK) return st;
    const int n = b->count();
    if (n == 0) return FI_OK;
    FB_CHECK(cudaMemsetAsync(b->d_slots, 0, sizeof(unsigned long long) * kSlots * n, b->stream), "slots");
    FB_CHECK(launch_check(b, b->d_all, b->d_full_ntiles), "batch check");
    std::vector<unsigned long long> sl((size_t)kSlots * n);
    FB_CHECK(cudaMemcpyAsync(sl.data(), b->d_slots, sizeof(unsigned long long) * sl.size(), cudaMemcpyDeviceToHost,
                             b->stream),
             "slots");
    FB_CHECK(cudaMemsetAsync(b->d_slots, 0, sizeof(unsigned long long) * kSlots * n, b->stream), "slots");
    FB_CHECK(cudaStreamSynchronize(b->stream), "batch sync");
    const BInst<float> *hf = reinterpret_cast<const BInst<float> *>(b->h_inst.data());
    const BInst<double> *hd = reinterpret_cast<const BInst<double> *>(b->h_inst.data());
    for (int q = 0; q < n; q++) {
        double v[kSlots];
        for (int c = 0; c < kSlots; c++) std::memcpy(&v[c], &sl[(size_t)q * kSlots + c], sizeof(double));
        const double h = b->f64 ? hd[q].h : hf[q].h;
        const double rV = v[1] * h, rP = v[0] * h;
        out[q] = std::max(v[2] > 0.0 ? rV / v[2] : rV, v[3] > 0.0 ? rP / v[3] : rP);
    }
    return FI_OK;
}

}  // extern "C"
