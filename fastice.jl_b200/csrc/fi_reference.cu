// fi_reference.cu -- reference-shaped kernels: one thread per grid index over the
// vertex-sized range 1..n+1 (the Chmy Launcher worksize), boundary-condition
// batches applied dimension by dimension, and the fused residual-norm reduction.
//
// These kernels follow src/Models/FullStokes/Isothermal/kernels_{2d,3d}.jl and
// src/Models/ImmersedBoundaryFullStokes/Isothermal/kernels_3d.jl operation by
// operation (same grouping of sums and products), so a build without FMA
// contraction reproduces the CPU oracle bit for bit.  They serve as the
// FI_PATH_REFERENCE path and for the shapes the fused sweep does not cover.
#include <algorithm>

#include "fi_device.cuh"

namespace fi {

namespace {

template <typename T>
__device__ __forceinline__ T h(T x) { return T(0.5) * x; }

struct Idx {
    long long I;
    int i, j, k;
    bool ok;
};

__device__ __forceinline__ Idx vertex_index_of(const Geom &g, unsigned bx, unsigned by, unsigned bz) {
    Idx r;
    r.i = bx * blockDim.x + threadIdx.x + 1;
    r.j = by * blockDim.y + threadIdx.y + 1;
    r.k = g.nd == 3 ? (int)bz + 1 : 0;
    r.ok = r.i <= g.n[0] + 1 && r.j <= g.n[1] + 1;
    r.I = (long long)r.i + g.pitch * ((long long)r.j + g.rows * (long long)r.k);
    return r;
}

__device__ __forceinline__ Idx vertex_index(const Geom &g) { return vertex_index_of(g, blockIdx.x, blockIdx.y, blockIdx.z); }

// the point of this thread in a launch over the whole grid or over a block list
__device__ __forceinline__ Idx vertex_index(const Geom &g, const BlockList &bl) {
    if (!bl.ids) return vertex_index(g);
    const uint2 b = bl.ids[blockIdx.x];
    return vertex_index_of(g, b.x & 0xffffu, b.x >> 16, b.y);
}

dim3 vertex_grid(const Geom &g, dim3 blk) {
    return dim3((g.n[0] + 1 + blk.x - 1) / blk.x, (g.n[1] + 1 + blk.y - 1) / blk.y, g.nd == 3 ? g.n[2] + 1 : 1);
}

// ---------------------------------------------------------------------------
// Immersed-boundary update_σ! and update_V! (IB kernels_3d.jl:3-74).  A thread
// owns C points of one row, 32 apart (x = i, i + 32, ...): one warp covers
// 32·C consecutive positions and each load instruction stays coalesced, while
// the loads of a masked group for all C points go out together.  The activity
// byte gates each group; a group's stores come after its loads for all points
// but before the next group's loads (the outputs may alias the inputs as far as
// the compiler knows), so a thread makes several dependent round trips to
// memory.  FP32 takes C = 2: its loads carry half the bytes of FP64 ones and one
// point per thread keeps too few bytes in flight.  FP64 takes C = 1 (C = 2
// measured 10 % slower at 383^3: 48 and 62 registers, fewer warps, and the FP64
// loads already carry enough bytes).
// Loads for a point past the vertex range (the second point of the last block
// of a row) stay inside the field's allocation (the row pitch, or the slack
// after the last row) and are discarded; nothing is stored there.  Forms that
// load every input of a point before any store (predicated loads, or one
// decision per warp with unconditional loads) were measured slower in both
// precisions: the extra registers cost more occupancy than the shorter chain
// gains.
// ---------------------------------------------------------------------------
template <typename T>
constexpr int ib_points() { return sizeof(T) == 4 ? 2 : 1; }

struct IbRow {
    long long I;  // index of the first point
    int i, j, k;  // its position
};

__device__ __forceinline__ IbRow ib_row_at(const Geom &g, unsigned bx, unsigned by, unsigned bz, int C) {
    IbRow r;
    r.i = bx * (32 * C) + threadIdx.x + 1;
    r.j = by * blockDim.y + threadIdx.y + 1;
    r.k = (int)bz + 1;
    r.I = (long long)r.i + g.pitch * ((long long)r.j + g.rows * (long long)r.k);
    return r;
}

__device__ __forceinline__ IbRow ib_row(const Geom &g, const BlockList &bl, int C) {
    unsigned bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    if (bl.ids) {
        const uint2 b = bl.ids[blockIdx.x];
        bx = b.x & 0xffffu, by = b.x >> 16, bz = b.y;
    }
    return ib_row_at(g, bx, by, bz, C);
}

dim3 ib_grid(const Geom &g, int C) {
    return dim3((g.n[0] + 1 + 32 * C - 1) / (32 * C), (g.n[1] + 1 + 7) / 8, g.n[2] + 1);
}

template <typename T, int C>
__device__ __forceinline__ void ib_sigma_body(const Geom &g, const KParams &p, const Ptrs<T> &f, const IbRow &r) {
    if (r.i > g.n[0] + 1 || r.j > g.n[1] + 1) return;
    const long long sx = g.pitch, sxy = g.sxy;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]), idz = T(p.inv_dx[2]);
    const T *Vx = f.Vx, *Vy = f.Vy, *Vz = f.Vz, *eta = f.eta;
    const T *nx = f.wns[W_VCC], *ny = f.wns[W_CVC], *nz = f.wns[W_CCV];
    const bool jk_inner = r.j >= 2 && r.j <= g.n[1] && r.k >= 2 && r.k <= g.n[2];
    bool ok[C], skip0[C];
    unsigned fl[C], any = 0;
#pragma unroll
    for (int c = 0; c < C; c++) {
        const int i = r.i + 32 * c;
        ok[c] = i <= g.n[0] + 1;
        skip0[c] = p.skip_zeros && jk_inner && i >= 2 && i <= g.n[0];
        fl[c] = ok[c] ? ib_flags_at(f, r.I + 32 * c, sx, sxy, T(p.small)) : 0u;
        any |= fl[c];
    }
    if (any & IBF_S_CCC) {
        T nP[C], nxx[C], nyy[C], nzz[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            T exx = (__ldg(nx + I + 1) * __ldg(Vx + I + 1) - __ldg(nx + I) * __ldg(Vx + I)) * idx;
            T eyy = (__ldg(ny + I + sx) * __ldg(Vy + I + sx) - __ldg(ny + I) * __ldg(Vy + I)) * idy;
            T ezz = (__ldg(nz + I + sxy) * __ldg(Vz + I + sxy) - __ldg(nz + I) * __ldg(Vz + I)) * idz;
            T divV = exx + eyy + ezz;
            T etac = __ldg(eta + I);
            nP[c] = f.P[I] - (p.p_forcing ? divV + f.fP[I] : divV) * etac * T(p.dt_P);
            nxx[c] = f.txx[I] - (f.txx[I] - T(2.0) * etac * (exx - third(divV))) * T(p.dt_tau[0]);
            nyy[c] = f.tyy[I] - (f.tyy[I] - T(2.0) * etac * (eyy - third(divV))) * T(p.dt_tau[1]);
            nzz[c] = f.tzz[I] - (f.tzz[I] - T(2.0) * etac * (ezz - third(divV))) * T(p.dt_tau[2]);
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            const bool on = fl[c] & IBF_S_CCC;
            if (on || (ok[c] && !skip0[c])) {
                f.P[I] = on ? nP[c] : T(0);
                f.txx[I] = on ? nxx[c] : T(0);
                f.tyy[I] = on ? nyy[c] : T(0);
                f.tzz[I] = on ? nzz[c] : T(0);
            }
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c] && !skip0[c]) {
                const long long I = r.I + 32 * c;
                f.P[I] = T(0);
                f.txx[I] = T(0);
                f.tyy[I] = T(0);
                f.tzz[I] = T(0);
            }
    }
    // the three shear components: edge viscosity from four centres, masked strain rate
    if (any & IBF_S_VVC) {
        T v[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            T exy = T(0.5) * ((__ldg(ny + I) * __ldg(Vy + I) - __ldg(ny + I - 1) * __ldg(Vy + I - 1)) * idx + (__ldg(nx + I) * __ldg(Vx + I) - __ldg(nx + I - sx) * __ldg(Vx + I - sx)) * idy);
            T e_xy = h(h(__ldg(eta + I - 1 - sx) + __ldg(eta + I - sx)) + h(__ldg(eta + I - 1) + __ldg(eta + I)));
            v[c] = f.txy[I] - (f.txy[I] - T(2.0) * e_xy * exy) * T(p.dt_tau[3]);
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const bool on = fl[c] & IBF_S_VVC;
            if (on || (ok[c] && !skip0[c])) f.txy[r.I + 32 * c] = on ? v[c] : T(0);
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c] && !skip0[c]) f.txy[r.I + 32 * c] = T(0);
    }
    if (any & IBF_S_VCV) {
        T v[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            T exz = T(0.5) * ((__ldg(nz + I) * __ldg(Vz + I) - __ldg(nz + I - 1) * __ldg(Vz + I - 1)) * idx + (__ldg(nx + I) * __ldg(Vx + I) - __ldg(nx + I - sxy) * __ldg(Vx + I - sxy)) * idz);
            T e_xz = h(h(__ldg(eta + I - 1 - sxy) + __ldg(eta + I - sxy)) + h(__ldg(eta + I - 1) + __ldg(eta + I)));
            v[c] = f.txz[I] - (f.txz[I] - T(2.0) * e_xz * exz) * T(p.dt_tau[4]);
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const bool on = fl[c] & IBF_S_VCV;
            if (on || (ok[c] && !skip0[c])) f.txz[r.I + 32 * c] = on ? v[c] : T(0);
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c] && !skip0[c]) f.txz[r.I + 32 * c] = T(0);
    }
    if (any & IBF_S_CVV) {
        T v[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            T eyz = T(0.5) * ((__ldg(nz + I) * __ldg(Vz + I) - __ldg(nz + I - sx) * __ldg(Vz + I - sx)) * idy + (__ldg(ny + I) * __ldg(Vy + I) - __ldg(ny + I - sxy) * __ldg(Vy + I - sxy)) * idz);
            T e_yz = h(h(__ldg(eta + I - sx - sxy) + __ldg(eta + I - sxy)) + h(__ldg(eta + I - sx) + __ldg(eta + I)));
            v[c] = f.tyz[I] - (f.tyz[I] - T(2.0) * e_yz * eyz) * T(p.dt_tau[5]);
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const bool on = fl[c] & IBF_S_CVV;
            if (on || (ok[c] && !skip0[c])) f.tyz[r.I + 32 * c] = on ? v[c] : T(0);
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c] && !skip0[c]) f.tyz[r.I + 32 * c] = T(0);
    }
}

template <typename T, int C>
__global__ void __launch_bounds__(256) ib_sigma_kernel(Geom g, KParams p, Ptrs<T> f, BlockList bl) {
    ib_sigma_body<T, C>(g, p, f, ib_row(g, bl, C));
}

template <typename T, int C>
__device__ __forceinline__ void ib_V_body(const Geom &g, const KParams &p, const Ptrs<T> &f, const IbRow &r) {
    if (r.i > g.n[0] + 1 || r.j > g.n[1] + 1) return;
    const long long sx = g.pitch, sxy = g.sxy;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]), idz = T(p.inv_dx[2]);
    const T *P = f.P, *txx = f.txx, *tyy = f.tyy, *tzz = f.tzz, *txy = f.txy, *txz = f.txz, *tyz = f.tyz, *eta = f.eta;
    const T *wc = f.wna[W_CCC], *wvvc = f.wna[W_VVC], *wvcv = f.wna[W_VCV], *wcvv = f.wna[W_CVV];
    const bool jk_inner = r.j >= 2 && r.j <= g.n[1] && r.k >= 2 && r.k <= g.n[2];
    bool ok[C], skip0[C];
    unsigned fl[C], any = 0;
#pragma unroll
    for (int c = 0; c < C; c++) {
        const int i = r.i + 32 * c;
        ok[c] = i <= g.n[0] + 1;
        skip0[c] = p.skip_zeros && jk_inner && i >= 2 && i <= g.n[0];
        fl[c] = ok[c] ? ib_flags_at(f, r.I + 32 * c, sx, sxy, T(p.small)) : 0u;
        any |= fl[c];
    }
    if (any & IBF_V_VCC) {
        T v[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            const T gx = gravity_dev(p, f.gx, 0, I);
            T ex = h(__ldg(eta + I - 1) + __ldg(eta + I));
            v[c] = f.Vx[I] + div_fast(div_fast(-(__ldg(wc + I) * __ldg(P + I) - __ldg(wc + I - 1) * __ldg(P + I - 1)) * idx +
                                                   (__ldg(wc + I) * __ldg(txx + I) - __ldg(wc + I - 1) * __ldg(txx + I - 1)) * idx +
                                                   (__ldg(wvvc + I + sx) * __ldg(txy + I + sx) - __ldg(wvvc + I) * __ldg(txy + I)) * idy +
                                                   (__ldg(wvcv + I + sxy) * __ldg(txz + I + sxy) - __ldg(wvcv + I) * __ldg(txz + I)) * idz - gx,
                                               ex),
                                      __ldg(f.wns[W_VCC] + I)) *
                                 T(p.dt_V[0]);
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const bool on = fl[c] & IBF_V_VCC;
            if (on || (ok[c] && !skip0[c])) f.Vx[r.I + 32 * c] = on ? v[c] : T(0);
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c] && !skip0[c]) f.Vx[r.I + 32 * c] = T(0);
    }
    if (any & IBF_V_CVC) {
        T v[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            const T gy = gravity_dev(p, f.gy, 1, I);
            T ey = h(__ldg(eta + I - sx) + __ldg(eta + I));
            v[c] = f.Vy[I] + div_fast(div_fast(-(__ldg(wc + I) * __ldg(P + I) - __ldg(wc + I - sx) * __ldg(P + I - sx)) * idy +
                                                   (__ldg(wc + I) * __ldg(tyy + I) - __ldg(wc + I - sx) * __ldg(tyy + I - sx)) * idy +
                                                   (__ldg(wvvc + I + 1) * __ldg(txy + I + 1) - __ldg(wvvc + I) * __ldg(txy + I)) * idx +
                                                   (__ldg(wcvv + I + sxy) * __ldg(tyz + I + sxy) - __ldg(wcvv + I) * __ldg(tyz + I)) * idz - gy,
                                               ey),
                                      __ldg(f.wns[W_CVC] + I)) *
                                 T(p.dt_V[1]);
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const bool on = fl[c] & IBF_V_CVC;
            if (on || (ok[c] && !skip0[c])) f.Vy[r.I + 32 * c] = on ? v[c] : T(0);
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c] && !skip0[c]) f.Vy[r.I + 32 * c] = T(0);
    }
    if (any & IBF_V_CCV) {
        T v[C];
#pragma unroll
        for (int c = 0; c < C; c++) {
            const long long I = r.I + 32 * c;
            const T gz = gravity_dev(p, f.gz, 2, I);
            T ez = h(__ldg(eta + I - sxy) + __ldg(eta + I));
            v[c] = f.Vz[I] + div_fast(div_fast(-(__ldg(wc + I) * __ldg(P + I) - __ldg(wc + I - sxy) * __ldg(P + I - sxy)) * idz +
                                                   (__ldg(wc + I) * __ldg(tzz + I) - __ldg(wc + I - sxy) * __ldg(tzz + I - sxy)) * idz +
                                                   (__ldg(wvcv + I + 1) * __ldg(txz + I + 1) - __ldg(wvcv + I) * __ldg(txz + I)) * idx +
                                                   (__ldg(wcvv + I + sx) * __ldg(tyz + I + sx) - __ldg(wcvv + I) * __ldg(tyz + I)) * idy - gz,
                                               ez),
                                      __ldg(f.wns[W_CCV] + I)) *
                                 T(p.dt_V[2]);
        }
#pragma unroll
        for (int c = 0; c < C; c++) {
            const bool on = fl[c] & IBF_V_CCV;
            if (on || (ok[c] && !skip0[c])) f.Vz[r.I + 32 * c] = on ? v[c] : T(0);
        }
    } else {
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c] && !skip0[c]) f.Vz[r.I + 32 * c] = T(0);
    }
    // η_next at every point of the range (kernels_3d.jl:36-40)
    if (p.freeze_eta) return;
    if (linear_unrelaxed(p)) {  // the stress invariant is not needed
#pragma unroll
        for (int c = 0; c < C; c++)
            if (ok[c]) f.eta_next[r.I + 32 * c] = p.rheo_eta_is_field ? f.eta_lin[r.I + 32 * c] : T(p.rheo_eta);
        return;
    }
    T en[C];
#pragma unroll
    for (int c = 0; c < C; c++) {
        const long long I = r.I + 32 * c;
        T lxy = h(h(__ldg(txy + I) + __ldg(txy + I + 1)) + h(__ldg(txy + I + sx) + __ldg(txy + I + sx + 1)));
        T lxz = h(h(__ldg(txz + I) + __ldg(txz + I + 1)) + h(__ldg(txz + I + sxy) + __ldg(txz + I + sxy + 1)));
        T lyz = h(h(__ldg(tyz + I) + __ldg(tyz + I + sx)) + h(__ldg(tyz + I + sxy) + __ldg(tyz + I + sxy + sx)));
        T s2 = T(0.5) * (__ldg(txx + I) * __ldg(txx + I) + __ldg(tyy + I) * __ldg(tyy + I) + __ldg(tzz + I) * __ldg(tzz + I)) + lxy * lxy + lxz * lxz + lyz * lyz;
        en[c] = ok[c] ? rheology_s2(p, T(p.rheo_A), T(p.rheo_inv_eta_reg), f.eta_lin, f.A, __ldg(eta + I), I, s2) : T(0);
    }
#pragma unroll
    for (int c = 0; c < C; c++)
        if (ok[c]) f.eta_next[r.I + 32 * c] = en[c];
}

// resident blocks per SM asked of the compiler: 6 (40 registers) for one point per
// thread, 4 (64) for two (5 at 48 registers with spills measured 2 % slower in FP32)
template <typename T, int C>
__global__ void __launch_bounds__(256, C == 1 ? 6 : 4) ib_V_kernel(Geom g, KParams p, Ptrs<T> f, BlockList bl) {
    ib_V_body<T, C>(g, p, f, ib_row(g, bl, C));
}

// ---------------------------------------------------------------------------
// Batched immersed-boundary updates: one launch runs the blocks of several
// models.  Work item = (member, block x | block y << 16, block z); the block
// copies its member's geometry, parameters and field pointers into shared
// memory and runs the same body as the single-model kernel, so each member's
// arithmetic is exactly its own model's.  epar picks the member's η roles for
// this iteration (f[0]: as when the table was built, f[1]: swapped).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ const IbMember<T> &ib_member_smem(const IbMember<T> *members, unsigned q,
                                                              IbMember<T> *sm) {
    constexpr int W = (int)(sizeof(IbMember<T>) / 4);
    const unsigned *src = reinterpret_cast<const unsigned *>(members + q);
    unsigned *dst = reinterpret_cast<unsigned *>(sm);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    for (int w = tid; w < W; w += blockDim.x * blockDim.y) dst[w] = __ldg(src + w);
    __syncthreads();
    return *sm;
}

template <typename T, int C>
__global__ void __launch_bounds__(256) ib_sigma_batched(const IbMember<T> *members, const uint4 *items, int epar) {
    __shared__ __align__(16) IbMember<T> sm;
    const uint4 it = items[blockIdx.x];
    const IbMember<T> &m = ib_member_smem(members, it.x, &sm);
    ib_sigma_body<T, C>(m.g, m.p, m.f[epar], ib_row_at(m.g, it.y & 0xffffu, it.y >> 16, it.z, C));
}

template <typename T, int C>
__global__ void __launch_bounds__(256, C == 1 ? 5 : 4) ib_V_batched(const IbMember<T> *members, const uint4 *items,
                                                                     int epar) {
    __shared__ __align__(16) IbMember<T> sm;
    const uint4 it = items[blockIdx.x];
    const IbMember<T> &m = ib_member_smem(members, it.x, &sm);
    ib_V_body<T, C>(m.g, m.p, m.f[epar], ib_row_at(m.g, it.y & 0xffffu, it.y >> 16, it.z, C));
}

// the work items of one member: its block list (uint2 x | y << 16, z) with the member index
__global__ void ib_items_from_list(const uint2 *list, int count, unsigned q, uint4 *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint2 b = list[i];
        out[i] = make_uint4(q, b.x, b.y, 0u);
    }
}
// or its whole grid of blocks (nbx x nby x nbz)
__global__ void ib_items_full(int nbx, int nby, int nbz, unsigned q, uint4 *out) {
    const long long total = (long long)nbx * nby * nbz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const unsigned bx = (unsigned)(i % nbx), by = (unsigned)((i / nbx) % nby), bz = (unsigned)(i / ((long long)nbx * nby));
        out[i] = make_uint4(q, bx | (by << 16), bz, 0u);
    }
}

template <typename T, int ND>
__global__ void __launch_bounds__(256) update_sigma_kernel(Geom g, KParams p, Ptrs<T> f, BlockList bl) {
    Idx x = vertex_index(g, bl);
    if (!x.ok) return;
    const long long I = x.I, sx = g.pitch, sxy = g.sxy;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]);
    const T *Vx = f.Vx, *Vy = f.Vy, *eta = f.eta;
    if (ND == 2) {
        T exx = (Vx[I + 1] - Vx[I]) * idx;
        T eyy = (Vy[I + sx] - Vy[I]) * idy;
        T exy = T(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
        T divV = exx + eyy;
        T etac = eta[I];
        f.P[I] = f.P[I] - (p.p_forcing ? divV + f.fP[I] : divV) * etac * T(p.dt_P);
        f.txx[I] = f.txx[I] - (f.txx[I] - T(2.0) * etac * (exx - third(divV))) * T(p.dt_tau[0]);
        f.tyy[I] = f.tyy[I] - (f.tyy[I] - T(2.0) * etac * (eyy - third(divV))) * T(p.dt_tau[1]);
        T exy_eta = h(h(eta[I - 1 - sx] + eta[I - sx]) + h(eta[I - 1] + eta[I]));
        f.txy[I] = f.txy[I] - (f.txy[I] - T(2.0) * exy_eta * exy) * T(p.dt_tau[3]);
        return;
    }
    const T idz = T(p.inv_dx[2]);
    const T *Vz = f.Vz;
    T exx = (Vx[I + 1] - Vx[I]) * idx;
    T eyy = (Vy[I + sx] - Vy[I]) * idy;
    T ezz = (Vz[I + sxy] - Vz[I]) * idz;
    T exy = T(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
    T exz = T(0.5) * ((Vz[I] - Vz[I - 1]) * idx + (Vx[I] - Vx[I - sxy]) * idz);
    T eyz = T(0.5) * ((Vz[I] - Vz[I - sx]) * idy + (Vy[I] - Vy[I - sxy]) * idz);
    T divV = exx + eyy + ezz;
    T etac = eta[I];
    f.P[I] = f.P[I] - (p.p_forcing ? divV + f.fP[I] : divV) * etac * T(p.dt_P);
    f.txx[I] = f.txx[I] - (f.txx[I] - T(2.0) * etac * (exx - third(divV))) * T(p.dt_tau[0]);
    f.tyy[I] = f.tyy[I] - (f.tyy[I] - T(2.0) * etac * (eyy - third(divV))) * T(p.dt_tau[1]);
    f.tzz[I] = f.tzz[I] - (f.tzz[I] - T(2.0) * etac * (ezz - third(divV))) * T(p.dt_tau[2]);
    T e_xy = h(h(eta[I - 1 - sx] + eta[I - sx]) + h(eta[I - 1] + eta[I]));
    T e_xz = h(h(eta[I - 1 - sxy] + eta[I - sxy]) + h(eta[I - 1] + eta[I]));
    T e_yz = h(h(eta[I - sx - sxy] + eta[I - sxy]) + h(eta[I - sx] + eta[I]));
    f.txy[I] = f.txy[I] - (f.txy[I] - T(2.0) * e_xy * exy) * T(p.dt_tau[3]);
    f.txz[I] = f.txz[I] - (f.txz[I] - T(2.0) * e_xz * exz) * T(p.dt_tau[4]);
    f.tyz[I] = f.tyz[I] - (f.tyz[I] - T(2.0) * e_yz * eyz) * T(p.dt_tau[5]);
}

// ---------------------------------------------------------------------------
// update_V!  (kernels_3d.jl:27-40, kernels_2d.jl:20-29; IB kernels_3d.jl:46-74)
// ---------------------------------------------------------------------------
// resident blocks per SM asked of the compiler: 6 (40 registers) for the 2D form,
// 4 (64) for the 3D form
template <int ND>
constexpr int update_V_min_blocks() { return ND == 2 ? 6 : 4; }

template <typename T, int ND>
__global__ void __launch_bounds__(256, update_V_min_blocks<ND>()) update_V_kernel(Geom g, KParams p, Ptrs<T> f, BlockList bl) {
    Idx x = vertex_index(g, bl);
    if (!x.ok) return;
    const long long I = x.I, sx = g.pitch, sxy = g.sxy;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]);
    const T *P = f.P, *txx = f.txx, *tyy = f.tyy, *txy = f.txy, *eta = f.eta;
    if (ND == 2) {
        T gx = gravity_dev(p, f.gx, 0, I), gy = gravity_dev(p, f.gy, 1, I);
        T ex = h(eta[I - 1] + eta[I]);
        T ey = h(eta[I - sx] + eta[I]);
        f.Vx[I] = f.Vx[I] +
                  div_fast(-(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy - gx, ex) *
                      T(p.dt_V[0]);
        f.Vy[I] = f.Vy[I] +
                  div_fast(-(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx - gy, ey) *
                      T(p.dt_V[1]);
        if (p.freeze_eta) return;
        if (linear_unrelaxed(p)) {
            f.eta_next[I] = p.rheo_eta_is_field ? f.eta_lin[I] : T(p.rheo_eta);
            return;
        }
        T lxy = h(h(txy[I] + txy[I + 1]) + h(txy[I + sx] + txy[I + sx + 1]));
        T s2 = T(0.5) * (txx[I] * txx[I] + tyy[I] * tyy[I]) + lxy * lxy;
        f.eta_next[I] = rheology_s2(p, T(p.rheo_A), T(p.rheo_inv_eta_reg), f.eta_lin, f.A, eta[I], I, s2);
        return;
    }
    const T idz = T(p.inv_dx[2]);
    const T *tzz = f.tzz, *txz = f.txz, *tyz = f.tyz;
    T gx = gravity_dev(p, f.gx, 0, I), gy = gravity_dev(p, f.gy, 1, I), gz = gravity_dev(p, f.gz, 2, I);
    T ex = h(eta[I - 1] + eta[I]);
    T ey = h(eta[I - sx] + eta[I]);
    T ez = h(eta[I - sxy] + eta[I]);
    f.Vx[I] = f.Vx[I] + div_fast(-(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy +
                                    (txz[I + sxy] - txz[I]) * idz - gx,
                                ex) *
                            T(p.dt_V[0]);
    f.Vy[I] = f.Vy[I] + div_fast(-(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx +
                                    (tyz[I + sxy] - tyz[I]) * idz - gy,
                                ey) *
                            T(p.dt_V[1]);
    f.Vz[I] = f.Vz[I] + div_fast(-(P[I] - P[I - sxy]) * idz + (tzz[I] - tzz[I - sxy]) * idz + (txz[I + 1] - txz[I]) * idx +
                                    (tyz[I + sx] - tyz[I]) * idy - gz,
                                ez) *
                            T(p.dt_V[2]);
    if (p.freeze_eta) return;
    if (linear_unrelaxed(p)) {  // the stress invariant is not needed
        f.eta_next[I] = p.rheo_eta_is_field ? f.eta_lin[I] : T(p.rheo_eta);
        return;
    }
    T lxy = h(h(txy[I] + txy[I + 1]) + h(txy[I + sx] + txy[I + sx + 1]));
    T lxz = h(h(txz[I] + txz[I + 1]) + h(txz[I + sxy] + txz[I + sxy + 1]));
    T lyz = h(h(tyz[I] + tyz[I + sx]) + h(tyz[I + sxy] + tyz[I + sxy + sx]));
    T s = T(0.5) * (txx[I] * txx[I] + tyy[I] * tyy[I] + tzz[I] * tzz[I]) + lxy * lxy + lxz * lxz + lyz * lyz;
    f.eta_next[I] = rheology_s2(p, T(p.rheo_A), T(p.rheo_inv_eta_reg), f.eta_lin, f.A, eta[I], I, s);
}

// ---------------------------------------------------------------------------
// compute_residuals!  (kernels_3d.jl:66-75, kernels_2d.jl:46-54; IB :118-143)
// ---------------------------------------------------------------------------
template <typename T, int ND, bool IB>
struct Resid {
    T rP, rVx, rVy, rVz;
};

template <typename T, int ND, bool IB>
__device__ __forceinline__ Resid<T, ND, IB> residual_at(const Geom &g, const KParams &p, const Ptrs<T> &f, long long I) {
    Resid<T, ND, IB> r;
    const long long sx = g.pitch, sxy = g.sxy;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]);
    const T *P = f.P, *txx = f.txx, *tyy = f.tyy, *txy = f.txy, *Vx = f.Vx, *Vy = f.Vy;
    if (ND == 2) {
        T gx = gravity_dev(p, f.gx, 0, I), gy = gravity_dev(p, f.gy, 1, I);
        r.rP = (Vx[I + 1] - Vx[I]) * idx + (Vy[I + sx] - Vy[I]) * idy;
        r.rVx = -(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy - gx;
        r.rVy = -(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx - gy;
        r.rVz = T(0);
        return r;
    }
    const T idz = T(p.inv_dx[2]);
    const T *tzz = f.tzz, *txz = f.txz, *tyz = f.tyz, *Vz = f.Vz;
    T gx = gravity_dev(p, f.gx, 0, I), gy = gravity_dev(p, f.gy, 1, I), gz = gravity_dev(p, f.gz, 2, I);
    if (!IB) {
        r.rP = (Vx[I + 1] - Vx[I]) * idx + (Vy[I + sx] - Vy[I]) * idy + (Vz[I + sxy] - Vz[I]) * idz;
        r.rVx = -(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy +
                (txz[I + sxy] - txz[I]) * idz - gx;
        r.rVy = -(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx +
                (tyz[I + sxy] - tyz[I]) * idz - gy;
        r.rVz = -(P[I] - P[I - sxy]) * idz + (tzz[I] - tzz[I - sxy]) * idz + (txz[I + 1] - txz[I]) * idx +
                (tyz[I + sx] - tyz[I]) * idy - gz;
        return r;
    }
    const T *const *na = f.wna;
    const T *const *ns = f.wns;
    const T thr = T(p.small);
    const T *wc = na[W_CCC], *wvvc = na[W_VVC], *wvcv = na[W_VCV], *wcvv = na[W_CVV];
    const unsigned fl = ib_flags_at(f, I, sx, sxy, thr);
    r.rP = (fl & IBF_S_CCC)
               ? (ns[W_VCC][I + 1] * Vx[I + 1] - ns[W_VCC][I] * Vx[I]) * idx +
                     (ns[W_CVC][I + sx] * Vy[I + sx] - ns[W_CVC][I] * Vy[I]) * idy +
                     (ns[W_CCV][I + sxy] * Vz[I + sxy] - ns[W_CCV][I] * Vz[I]) * idz
               : T(0);
    r.rVx = (fl & IBF_V_VCC)
                ? -(wc[I] * P[I] - wc[I - 1] * P[I - 1]) * idx + (wc[I] * txx[I] - wc[I - 1] * txx[I - 1]) * idx +
                      (wvvc[I + sx] * txy[I + sx] - wvvc[I] * txy[I]) * idy +
                      (wvcv[I + sxy] * txz[I + sxy] - wvcv[I] * txz[I]) * idz - gx
                : T(0);
    r.rVy = (fl & IBF_V_CVC)
                ? -(wc[I] * P[I] - wc[I - sx] * P[I - sx]) * idy + (wc[I] * tyy[I] - wc[I - sx] * tyy[I - sx]) * idy +
                      (wvvc[I + 1] * txy[I + 1] - wvvc[I] * txy[I]) * idx +
                      (wcvv[I + sxy] * tyz[I + sxy] - wcvv[I] * tyz[I]) * idz - gy
                : T(0);
    r.rVz = (fl & IBF_V_CCV)
                ? -(wc[I] * P[I] - wc[I - sxy] * P[I - sxy]) * idz + (wc[I] * tzz[I] - wc[I - sxy] * tzz[I - sxy]) * idz +
                      (wvcv[I + 1] * txz[I + 1] - wvcv[I] * txz[I]) * idx +
                      (wcvv[I + sx] * tyz[I + sx] - wcvv[I] * tyz[I]) * idy - gz
                : T(0);
    return r;
}

template <typename T, int ND, bool IB>
__global__ void __launch_bounds__(256) compute_residuals_kernel(Geom g, KParams p, Ptrs<T> f) {
    Idx x = vertex_index(g);
    if (!x.ok) return;
    Resid<T, ND, IB> r = residual_at<T, ND, IB>(g, p, f, x.I);
    if (p.p_forcing) r.rP = r.rP + f.fP[x.I];
    f.rP[x.I] = r.rP;
    f.rVx[x.I] = r.rVx;
    f.rVy[x.I] = r.rVy;
    if (ND == 3) f.rVz[x.I] = r.rVz;
}

// compute_τ!  (kernels_3d.jl:44-64, kernels_2d.jl:33-44)
template <typename T, int ND>
__global__ void __launch_bounds__(256) compute_tau_kernel(Geom g, KParams p, Ptrs<T> f) {
    Idx x = vertex_index(g);
    if (!x.ok) return;
    const long long I = x.I, sx = g.pitch, sxy = g.sxy;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]);
    const T *Vx = f.Vx, *Vy = f.Vy, *eta = f.eta;
    if (ND == 2) {
        T exx = (Vx[I + 1] - Vx[I]) * idx;
        T eyy = (Vy[I + sx] - Vy[I]) * idy;
        T exy = T(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
        T divV = exx + eyy;
        f.txx[I] = T(2.0) * eta[I] * (exx - divV / T(3.0));
        f.tyy[I] = T(2.0) * eta[I] * (eyy - divV / T(3.0));
        T e_xy = h(h(eta[I - 1 - sx] + eta[I - sx]) + h(eta[I - 1] + eta[I]));
        f.txy[I] = T(2.0) * e_xy * exy;
        return;
    }
    const T idz = T(p.inv_dx[2]);
    const T *Vz = f.Vz;
    T exx = (Vx[I + 1] - Vx[I]) * idx;
    T eyy = (Vy[I + sx] - Vy[I]) * idy;
    T ezz = (Vz[I + sxy] - Vz[I]) * idz;
    T exy = T(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
    T exz = T(0.5) * ((Vz[I] - Vz[I - 1]) * idx + (Vx[I] - Vx[I - sxy]) * idz);
    T eyz = T(0.5) * ((Vz[I] - Vz[I - sx]) * idy + (Vy[I] - Vy[I - sxy]) * idz);
    T divV = exx + eyy + ezz;
    f.txx[I] = T(2.0) * eta[I] * (exx - divV / T(3.0));
    f.tyy[I] = T(2.0) * eta[I] * (eyy - divV / T(3.0));
    f.tzz[I] = T(2.0) * eta[I] * (ezz - divV / T(3.0));
    T e_xy = h(h(eta[I - 1 - sx] + eta[I - sx]) + h(eta[I - 1] + eta[I]));
    T e_xz = h(h(eta[I - 1 - sxy] + eta[I - sxy]) + h(eta[I - 1] + eta[I]));
    T e_yz = h(h(eta[I - sx - sxy] + eta[I - sxy]) + h(eta[I - sx] + eta[I]));
    f.txy[I] = T(2.0) * e_xy * exy;
    f.txz[I] = T(2.0) * e_xz * exz;
    f.tyz[I] = T(2.0) * e_yz * eyz;
}

// Masked projection τ = 2η dev ε̇(V) of the immersed-boundary model: the strain
// rates, activity tests and zeroing of update_σ! (IB kernels_3d.jl:3-44) with the
// relaxation replaced by the assignment.  The reference's own IB compute_τ!
// (IB kernels_3d.jl:76-100) cannot run (it names the undefined `Pr`); this is its
// evident intent, used by the mixed-precision solve's projection step.
template <typename T>
__global__ void __launch_bounds__(256) compute_tau_ib_kernel(Geom g, KParams p, Ptrs<T> f) {
    Idx x = vertex_index(g);
    if (!x.ok) return;
    const long long I = x.I, sx = g.pitch, sxy = g.sxy;
    const T idx = T(p.inv_dx[0]), idy = T(p.inv_dx[1]), idz = T(p.inv_dx[2]);
    const T *Vx = f.Vx, *Vy = f.Vy, *Vz = f.Vz, *eta = f.eta;
    const T *const *ns = f.wns;
    const T thr = T(p.small);
    const unsigned fl = ib_flags_at(f, I, sx, sxy, thr);
    if (fl & IBF_S_CCC) {
        T exx = (ns[W_VCC][I + 1] * Vx[I + 1] - ns[W_VCC][I] * Vx[I]) * idx;
        T eyy = (ns[W_CVC][I + sx] * Vy[I + sx] - ns[W_CVC][I] * Vy[I]) * idy;
        T ezz = (ns[W_CCV][I + sxy] * Vz[I + sxy] - ns[W_CCV][I] * Vz[I]) * idz;
        T divV = exx + eyy + ezz;
        T etac = eta[I];
        f.txx[I] = T(2.0) * etac * (exx - divV / T(3.0));
        f.tyy[I] = T(2.0) * etac * (eyy - divV / T(3.0));
        f.tzz[I] = T(2.0) * etac * (ezz - divV / T(3.0));
    } else {
        f.txx[I] = T(0);
        f.tyy[I] = T(0);
        f.tzz[I] = T(0);
    }
    if (fl & IBF_S_VVC) {
        T exy = T(0.5) * ((ns[W_CVC][I] * Vy[I] - ns[W_CVC][I - 1] * Vy[I - 1]) * idx +
                          (ns[W_VCC][I] * Vx[I] - ns[W_VCC][I - sx] * Vx[I - sx]) * idy);
        T e_xy = h(h(eta[I - 1 - sx] + eta[I - sx]) + h(eta[I - 1] + eta[I]));
        f.txy[I] = T(2.0) * e_xy * exy;
    } else {
        f.txy[I] = T(0);
    }
    if (fl & IBF_S_VCV) {
        T exz = T(0.5) * ((ns[W_CCV][I] * Vz[I] - ns[W_CCV][I - 1] * Vz[I - 1]) * idx +
                          (ns[W_VCC][I] * Vx[I] - ns[W_VCC][I - sxy] * Vx[I - sxy]) * idz);
        T e_xz = h(h(eta[I - 1 - sxy] + eta[I - sxy]) + h(eta[I - 1] + eta[I]));
        f.txz[I] = T(2.0) * e_xz * exz;
    } else {
        f.txz[I] = T(0);
    }
    if (fl & IBF_S_CVV) {
        T eyz = T(0.5) * ((ns[W_CCV][I] * Vz[I] - ns[W_CCV][I - sx] * Vz[I - sx]) * idy +
                          (ns[W_CVC][I] * Vy[I] - ns[W_CVC][I - sxy] * Vy[I - sxy]) * idz);
        T e_yz = h(h(eta[I - sx - sxy] + eta[I - sxy]) + h(eta[I - sx] + eta[I]));
        f.tyz[I] = T(2.0) * e_yz * eyz;
    } else {
        f.tyz[I] = T(0);
    }
}

// ---------------------------------------------------------------------------
// Boundary-condition batch for one dimension: the face of dim d spans the full
// storage range of the dims before d and the interior range of the dims after
// d (per field location); left and right sides of every field in the batch.
// Each op of the batch has its own grid slice (blockIdx.z): the ops of a batch
// touch distinct (field, side) pairs, whose reads and writes do not overlap
// when the dimension has 3 or more cells, so they need no order among them;
// otherwise (b.serial) one thread applies them all in the batch's order.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void bc_dim_body(const Geom &g, const BcBatch &b, int opz) {
    const int d = b.dim;
    int e1 = -1, e2 = -1;
    for (int e = 0; e < g.nd; e++) {
        if (e == d) continue;
        if (e1 < 0) e1 = e;
        else e2 = e;
    }
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y * blockDim.y + threadIdx.y;
    if (a > g.n[e1] + 2) return;
    if (e2 >= 0 && c > g.n[e2] + 2) return;
    if (e2 < 0 && c > 0) return;
    const long long st[3] = {1, g.pitch, g.sxy};
    const int q0 = b.serial ? 0 : opz, q1 = b.serial ? b.count : q0 + 1;
    for (int q = q0; q < q1; q++) {
        const BcOpDesc &op = b.ops[q];
        // range check for the other dims
        int pos[3] = {0, 0, 0};
        pos[e1] = a;
        if (e2 >= 0) pos[e2] = c;
        bool ok = true;
        for (int e = 0; e < g.nd; e++) {
            if (e == d) continue;
            if (e > d && (pos[e] < 1 || pos[e] > g.n[e] + op.loc[e])) ok = false;
        }
        if (!ok) continue;
        T *f = (T *)op.f;
        long long B = (long long)pos[0] + g.pitch * ((long long)pos[1] + g.rows * (long long)pos[2]);
        const long long sd = st[d];
        const int N = g.n[d];
#define A(q_) f[B + (long long)(q_)*sd]
        if (op.op == BC_DIRICHLET) {
            T v = T(op.v);
            T two_v = T(2.0) * v;
            if (op.loc[d] == 0) {
                if (op.side == 0) A(0) = two_v - A(1);
                else A(N + 1) = two_v - A(N);
            } else {
                if (op.side == 0) A(1) = v;
                else A(N + 1) = v;
            }
        } else if (op.op == BC_NEUMANN) {
            if (op.loc[d] == 0) {
                if (op.side == 0) A(0) = A(1);
                else A(N + 1) = A(N);
            } else {
                if (op.side == 0) A(0) = A(2);
                else A(N + 2) = A(N);
            }
        } else {
            if (op.loc[d] == 0) {
                A(0) = A(N);
                A(N + 1) = A(1);
            } else {
                A(N + 1) = A(1);
                A(0) = A(N);
                A(N + 2) = A(2);
            }
        }
#undef A
    }
}

template <typename T>
__global__ void bc_dim_kernel(Geom g, BcBatch b) {
    bc_dim_body<T>(g, b, (int)blockIdx.z);
}

// the boundary batch of one dimension for several models: grid slice z = member *
// kMaxBcOps + op (a serial batch runs its ops in slice op 0)
template <typename T>
__global__ void bc_dim_batched(const BcMember *list) {
    const int q = (int)blockIdx.z / kMaxBcOps, op = (int)blockIdx.z % kMaxBcOps;
    const BcMember &m = list[q];
    if (op >= (m.b.serial ? 1 : m.b.count)) return;
    bc_dim_body<T>(m.g, m.b, op);
}

// ---------------------------------------------------------------------------
// Fused residual + norms: r is evaluated at every interior position of each
// component (normal velocity residual = 0 on non-traction, non-periodic walls,
// boundary_conditions.jl:120-128) and reduced to max|r|, sum r^2, max|V| per
// block (warp shuffles, then shared memory); a second single-block pass adds
// the per-block partials in a fixed order in FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) {
        double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = (w > v || w != w) ? w : v;  // NaN-propagating max
    }
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double nmax(double a, double b) { return (b > a || b != b) ? b : a; }

constexpr int kNormThreads = 256;

template <typename T, int ND, bool IB>
__global__ void __launch_bounds__(kNormThreads) residual_norms_kernel(Geom g, KParams p, Ptrs<T> f, double *partials) {
    double mx[4] = {0, 0, 0, 0}, ss[4] = {0, 0, 0, 0}, vm[3] = {0, 0, 0};
    const long long nx = g.n[0] + 1, ny = g.n[1] + 1, nz = ND == 3 ? g.n[2] + 1 : 1;
    const long long total = nx * ny * nz;
    bool wall0[3][2];
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++) {
            int k = d < ND ? p.bc_kind[d][s] : FI_BC_TRACTION;
            wall0[d][s] = !(k == FI_BC_TRACTION || k == FI_BC_PERIODIC || k == FI_BC_HALO);
        }
    // grid-stride loop over the vertex range; the position (ii, jj, kk) steps by the
    // stride's own decomposition with carries instead of two 64-bit divisions per point
    const long long S = (long long)gridDim.x * blockDim.x;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int ii = int(t % nx), jj = int((t / nx) % ny), kk = int(t / nx / ny);
    const int si = int(S % nx), sj = int((S / nx) % ny), sk = int(S / nx / ny);
    for (; t < total; t += S) {
        const int i = ii + 1, j = jj + 1, k = ND == 3 ? kk + 1 : 0;
        ii += si;
        const int c1 = ii >= nx;
        ii -= c1 ? int(nx) : 0;
        jj += sj + c1;
        const int c2 = jj >= ny;
        jj -= c2 ? int(ny) : 0;
        kk += sk + c2;
        long long I = (long long)i + g.pitch * ((long long)j + g.rows * (long long)k);
        Resid<T, ND, IB> r = residual_at<T, ND, IB>(g, p, f, I);
        if (p.p_forcing) r.rP = r.rP + f.fP[I];
        bool cx = i <= g.n[0], cy = j <= g.n[1], cz = ND == 3 ? k <= g.n[2] : true;
        // r_P at (C,C,C)
        if (cx && cy && cz) {
            double v = fabs(double(r.rP));
            mx[0] = nmax(mx[0], v);
            ss[0] += double(r.rP) * double(r.rP);
        }
        // r_Vx at (V,C,C)
        if (cy && cz) {
            double v = double(r.rVx);
            if ((i == 1 && wall0[0][0]) || (i == g.n[0] + 1 && wall0[0][1])) v = 0.0;
            mx[1] = nmax(mx[1], fabs(v));
            ss[1] += v * v;
            vm[0] = nmax(vm[0], fabs(double(f.Vx[I])));
        }
        if (cx && cz) {
            double v = double(r.rVy);
            if ((j == 1 && wall0[1][0]) || (j == g.n[1] + 1 && wall0[1][1])) v = 0.0;
            mx[2] = nmax(mx[2], fabs(v));
            ss[2] += v * v;
            vm[1] = nmax(vm[1], fabs(double(f.Vy[I])));
        }
        if (ND == 3 && cx && cy) {
            double v = double(r.rVz);
            if ((k == 1 && wall0[2][0]) || (k == g.n[2] + 1 && wall0[2][1])) v = 0.0;
            mx[3] = nmax(mx[3], fabs(v));
            ss[3] += v * v;
            vm[2] = nmax(vm[2], fabs(double(f.Vz[I])));
        }
    }
    __shared__ double sh[kNormThreads / 32][11];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double vals[11] = {mx[0], mx[1], mx[2], mx[3], ss[0], ss[1], ss[2], ss[3], vm[0], vm[1], vm[2]};
#pragma unroll
    for (int q = 0; q < 11; q++) {
        double v = (q >= 4 && q < 8) ? warp_sum(vals[q]) : warp_max(vals[q]);
        if (lane == 0) sh[wid][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < 11) {
        int q = threadIdx.x;
        double acc = sh[0][q];
        for (int w = 1; w < kNormThreads / 32; w++) acc = (q >= 4 && q < 8) ? acc + sh[w][q] : nmax(acc, sh[w][q]);
        partials[(long long)blockIdx.x * kNormSlots + q] = acc;
    }
}

__global__ void norms_finalize_kernel(const double *partials, int nblocks, double *out) {
    // one warp per slot; fixed-order per-lane strided sums then a fixed shuffle tree
    int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (q >= 11) return;
    double acc = (q >= 4 && q < 8) ? 0.0 : 0.0;
    for (int b = lane; b < nblocks; b += 32) {
        double v = partials[(long long)b * kNormSlots + q];
        acc = (q >= 4 && q < 8) ? acc + v : nmax(acc, v);
    }
    acc = (q >= 4 && q < 8) ? warp_sum(acc) : warp_max(acc);
    if (lane == 0) {
        if (q >= 4 && q < 8) acc = sqrt(acc);
        out[q] = acc;
    }
    if (threadIdx.x == 0) out[11] = 0.0;
}

__global__ void norms_flag_kernel(double *out) {
    bool bad = false;
    for (int q = 0; q < 11; q++) bad |= !isfinite(out[q]);
    out[11] = bad ? 1.0 : 0.0;
}

}  // namespace

int norm_blocks(const Geom &g) {
    long long total = (long long)(g.n[0] + 1) * (g.n[1] + 1) * (g.nd == 3 ? g.n[2] + 1 : 1);
    long long b = (total + kNormThreads * 8 - 1) / (kNormThreads * 8);
    if (b < 1) b = 1;
    if (b > 148 * 8) b = 148 * 8;
    return (int)b;
}

template <typename T>
cudaError_t launch_update_sigma(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s,
                                const BlockList *bl) {
    dim3 blk(32, 8);
    dim3 grd = vertex_grid(g, blk);
    const BlockList none{nullptr, 0};
    constexpr int C = ib_points<T>();
    if (g.nd == 2) update_sigma_kernel<T, 2><<<grd, blk, 0, s>>>(g, p, f, none);
    else if (ib) ib_sigma_kernel<T, C><<<bl ? dim3(bl->count) : ib_grid(g, C), blk, 0, s>>>(g, p, f, bl ? *bl : none);
    else update_sigma_kernel<T, 3><<<grd, blk, 0, s>>>(g, p, f, none);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_update_V(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s,
                            const BlockList *bl) {
    dim3 blk(32, 8);
    dim3 grd = vertex_grid(g, blk);
    const BlockList none{nullptr, 0};
    constexpr int C = ib_points<T>();
    if (g.nd == 2) update_V_kernel<T, 2><<<grd, blk, 0, s>>>(g, p, f, none);
    else if (ib) ib_V_kernel<T, C><<<bl ? dim3(bl->count) : ib_grid(g, C), blk, 0, s>>>(g, p, f, bl ? *bl : none);
    else update_V_kernel<T, 3><<<grd, blk, 0, s>>>(g, p, f, none);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_compute_residuals(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s) {
    dim3 blk(32, 8);
    dim3 grd = vertex_grid(g, blk);
    if (g.nd == 2) compute_residuals_kernel<T, 2, false><<<grd, blk, 0, s>>>(g, p, f);
    else if (ib) compute_residuals_kernel<T, 3, true><<<grd, blk, 0, s>>>(g, p, f);
    else compute_residuals_kernel<T, 3, false><<<grd, blk, 0, s>>>(g, p, f);
    return cudaGetLastError();
}

// activity bytes over the vertex range (null_spaces.jl:41-43 at the seven
// locations the masked kernels test)
template <typename T>
__global__ void __launch_bounds__(256) ib_flags_kernel(Geom g, KParams p, Ptrs<T> f, unsigned char *flags) {
    Idx x = vertex_index(g);
    if (!x.ok) return;
    Ptrs<T> q = f;
    q.ibf = nullptr;
    flags[x.I] = (unsigned char)ib_flags_at(q, x.I, g.pitch, g.sxy, T(p.small));
}

template <typename T>
cudaError_t launch_ib_flags(const Geom &g, const KParams &p, const Ptrs<T> &f, unsigned char *flags, cudaStream_t s) {
    dim3 blk(32, 8);
    dim3 grd = vertex_grid(g, blk);
    ib_flags_kernel<T><<<grd, blk, 0, s>>>(g, p, f, flags);
    return cudaGetLastError();
}

// Blocks of the immersed-boundary launch (32·C positions of a row by 8 rows, one
// plane; C = ib_points) that hold a point outside the strict interior (index 1
// or n+1 in some dimension: boundary batches write there) or a point p with an
// activity bit at p + {0,1}^3.  The viscosity update at p reads τ at those eight
// points, and τ is zero where no bit is set, so elsewhere η_next is the rheology
// of a zero invariant: the same value every iteration.  The eight reads stay
// inside the vertex range because p is strictly inside.
template <int C>
__global__ void __launch_bounds__(256) ib_blocks_kernel(Geom g, const unsigned char *flags, uint2 *list, int *count) {
    const BlockList none{nullptr, 0};
    const IbRow r = ib_row(g, none, C);
    bool need = false;
#pragma unroll
    for (int c = 0; c < C; c++) {
        const int i = r.i + 32 * c;
        if (i > g.n[0] + 1 || r.j > g.n[1] + 1) continue;
        const bool inner = i >= 2 && i <= g.n[0] && r.j >= 2 && r.j <= g.n[1] && r.k >= 2 && r.k <= g.n[2];
        if (!inner) {
            need = true;
        } else {
            const long long I = r.I + 32 * c, sx = g.pitch, sxy = g.sxy;
            need |= (flags[I] | flags[I + 1] | flags[I + sx] | flags[I + sx + 1] | flags[I + sxy] | flags[I + sxy + 1] |
                     flags[I + sxy + sx] | flags[I + sxy + sx + 1]) != 0;
        }
    }
    if (__syncthreads_or(need) && threadIdx.x == 0 && threadIdx.y == 0)
        list[atomicAdd(count, 1)] = make_uint2(blockIdx.x | (blockIdx.y << 16), blockIdx.z);
}

template <typename T>
cudaError_t launch_ib_blocks(const Geom &g, const unsigned char *flags, uint2 *list, int *count, cudaStream_t s) {
    constexpr int C = ib_points<T>();
    ib_blocks_kernel<C><<<ib_grid(g, C), dim3(32, 8), 0, s>>>(g, flags, list, count);
    return cudaGetLastError();
}

long long vertex_grid_blocks(const Geom &g) {
    dim3 grd = vertex_grid(g, dim3(32, 8));
    return (long long)grd.x * grd.y * grd.z;
}

template <typename T>
cudaError_t launch_compute_tau(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s) {
    dim3 blk(32, 8);
    dim3 grd = vertex_grid(g, blk);
    if (g.nd == 2) compute_tau_kernel<T, 2><<<grd, blk, 0, s>>>(g, p, f);
    else if (ib) compute_tau_ib_kernel<T><<<grd, blk, 0, s>>>(g, p, f);
    else compute_tau_kernel<T, 3><<<grd, blk, 0, s>>>(g, p, f);
    return cudaGetLastError();
}

// whether the ops of a batch must run in order by one thread (a dimension of fewer
// than 3 cells, or two ops on one field whose faces may meet)
void bc_set_serial(const Geom &g, BcBatch &b) {
    b.serial = g.n[b.dim] < 3;
    for (int q = 0; q < b.count && !b.serial; q++)
        for (int r = 0; r < q; r++)
            if (b.ops[r].f == b.ops[q].f &&
                (b.ops[r].side == b.ops[q].side || b.ops[r].op == BC_PERIODIC || b.ops[q].op == BC_PERIODIC))
                b.serial = 1;
}

template <typename T>
cudaError_t launch_bc_batch(const Geom &g, const BcBatch &b, cudaStream_t s) {
    if (b.count == 0) return cudaSuccess;
    int e1 = -1, e2 = -1;
    for (int e = 0; e < g.nd; e++) {
        if (e == b.dim) continue;
        if (e1 < 0) e1 = e;
        else e2 = e;
    }
    int na = g.n[e1] + 3, nc = e2 >= 0 ? g.n[e2] + 3 : 1;
    BcBatch bb = b;
    bc_set_serial(g, bb);
    dim3 blk(32, 8);
    dim3 grd((na + 31) / 32, (nc + 7) / 8, bb.serial ? 1 : b.count);
    bc_dim_kernel<T><<<grd, blk, 0, s>>>(g, bb);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual_norms(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, double *partials,
                                  int nblocks, double *out_dev, cudaStream_t s) {
    if (g.nd == 2) residual_norms_kernel<T, 2, false><<<nblocks, kNormThreads, 0, s>>>(g, p, f, partials);
    else if (ib) residual_norms_kernel<T, 3, true><<<nblocks, kNormThreads, 0, s>>>(g, p, f, partials);
    else residual_norms_kernel<T, 3, false><<<nblocks, kNormThreads, 0, s>>>(g, p, f, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    norms_finalize_kernel<<<1, 11 * 32, 0, s>>>(partials, nblocks, out_dev);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    norms_flag_kernel<<<1, 1, 0, s>>>(out_dev);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_ib_batched(const IbMember<T> *members, const uint4 *items, int nitems, int epar, bool velocity,
                              cudaStream_t s) {
    if (nitems <= 0) return cudaSuccess;
    constexpr int C = ib_points<T>();
    if (velocity) ib_V_batched<T, C><<<nitems, dim3(32, 8), 0, s>>>(members, items, epar);
    else ib_sigma_batched<T, C><<<nitems, dim3(32, 8), 0, s>>>(members, items, epar);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_bc_batched(const BcMember *list, int count, int max_a, int max_c, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    dim3 blk(32, 8);
    bc_dim_batched<T><<<dim3((max_a + 31) / 32, (max_c + 7) / 8, count * kMaxBcOps), blk, 0, s>>>(list);
    return cudaGetLastError();
}

cudaError_t launch_ib_items(const Geom &g, bool full, const uint2 *list, int count, unsigned q, uint4 *out, bool f32,
                            cudaStream_t s) {
    if (full) {
        const dim3 gr = ib_grid(g, f32 ? 2 : 1);
        const long long total = (long long)gr.x * gr.y * gr.z;
        ib_items_full<<<(int)std::min<long long>((total + 255) / 256, 4096), 256, 0, s>>>(gr.x, gr.y, gr.z, q, out);
    } else if (count > 0) {
        ib_items_from_list<<<std::min((count + 255) / 256, 4096), 256, 0, s>>>(list, count, q, out);
    }
    return cudaGetLastError();
}

long long ib_grid_blocks(const Geom &g, bool f32) {
    const dim3 gr = ib_grid(g, f32 ? 2 : 1);
    return (long long)gr.x * gr.y * gr.z;
}

#define FI_INST(T)                                                                                                \
    template cudaError_t launch_update_sigma<T>(const Geom &, const KParams &, const Ptrs<T> &, bool, cudaStream_t,   \
                                                const BlockList *);                                               \
    template cudaError_t launch_update_V<T>(const Geom &, const KParams &, const Ptrs<T> &, bool, cudaStream_t,       \
                                            const BlockList *);                                                   \
    template cudaError_t launch_compute_residuals<T>(const Geom &, const KParams &, const Ptrs<T> &, bool,          \
                                                     cudaStream_t);                                               \
    template cudaError_t launch_compute_tau<T>(const Geom &, const KParams &, const Ptrs<T> &, bool, cudaStream_t);   \
    template cudaError_t launch_ib_flags<T>(const Geom &, const KParams &, const Ptrs<T> &, unsigned char *, cudaStream_t);       \
    template cudaError_t launch_bc_batch<T>(const Geom &, const BcBatch &, cudaStream_t);                          \
    template cudaError_t launch_ib_blocks<T>(const Geom &, const unsigned char *, uint2 *, int *, cudaStream_t);   \
    template cudaError_t launch_residual_norms<T>(const Geom &, const KParams &, const Ptrs<T> &, bool, double *,  \
                                                  int, double *, cudaStream_t);                                    \
    template cudaError_t launch_ib_batched<T>(const IbMember<T> *, const uint4 *, int, int, bool, cudaStream_t);    \
    template cudaError_t launch_bc_batched<T>(const BcMember *, int, int, int, cudaStream_t);
FI_INST(double)
FI_INST(float)
#undef FI_INST

}  // namespace fi
