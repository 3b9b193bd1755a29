// fi_heat.cu -- pseudo-transient heat diffusion (src/Models/Diffusion/Heat/):
// HeatDiffusionModel and advance_iteration! restated, one fused sweep per PT
// iteration.
//
// The reference iteration (kernels.jl:3-29, Heat.jl:45-61) is update_q!, the Flux
// boundary nodes of q, update_T!, the Value ghosts of T.  The sweep here does all
// of it in one pass over the cells: a cell's thread computes the new flux on both
// faces of its cell along every dimension (the face it shares with a neighbour is
// computed by both, with the same operands and operations, so they agree to the
// bit), takes the Flux value on a boundary face, updates T, writes its low faces
// (and the high boundary face) of q and, next to a Value side, the ghost 2v - T.
// T and q are double-buffered (read one copy, write the other), which makes the
// single pass equal to the reference's two kernels.
//
// Arithmetic as the reference writes it: λ_ρCp * (T[I] - T[I-e_d]) / Δ_d (a true
// division), ∇q summed x, then y, then z, (T - T_o) / Δt.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "fi_internal.h"

#define FI_CHECK_CUDA(expr, where)                          \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, where); \
    } while (0)

struct fi_heat {
    fi_heat_desc d{};
    size_t esz = 8, elems = 0;
    long long pitch = 0, rows = 0;
    void *T[2] = {}, *q[3][2] = {}, *To = nullptr;
    int cur = 0;  // buffer holding the current T and q
    cudaStream_t stream = nullptr;
};

namespace fi {
namespace {

constexpr long long kHeatOff = 31;  // field pointer offset inside its allocation (interior rows 128/256-byte aligned)

template <typename T>
struct HeatArgs {
    const T *T0, *To, *qx0, *qy0, *qz0;
    T *T1, *qx1, *qy1, *qz1;
    int n[3];
    long long sx, sxy;
    T D[3], lam, dtq, dtT, dt;
    T iD[3], idt;  // 1/D and 1/dt, rounded once on the host
    int kind[3][2];
    T val[3][2];
};

// x / D[d] and x / dt: production builds multiply by the rounded reciprocals
// (within an ulp or so of the quotient, and no division sequence per cell);
// FI_EXACT_ORDER builds divide as the reference does
template <typename T>
__device__ __forceinline__ T over_D(const HeatArgs<T> &a, T x, int d) {
#ifdef FI_EXACT_ORDER
    return x / a.D[d];
#else
    return x * a.iD[d];
#endif
}
template <typename T>
__device__ __forceinline__ T over_dt(const HeatArgs<T> &a, T x) {
#ifdef FI_EXACT_ORDER
    return x / a.dt;
#else
    return x * a.idt;
#endif
}

template <typename T>
__global__ void __launch_bounds__(256) heat_sweep(HeatArgs<T> a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > a.n[0] || j > a.n[1]) return;
    const long long st[3] = {1, a.sx, a.sxy};
    const long long I = (long long)i + a.sx * j + a.sxy * k;
    const int ix[3] = {i, j, k};
    const T *q0[3] = {a.qx0, a.qy0, a.qz0};
    T *q1[3] = {a.qx1, a.qy1, a.qz1};
    const T Tc = a.T0[I];
    T ql[3], qr[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const T Tm = a.T0[I - st[d]], Tp = a.T0[I + st[d]];
        const T qlo = q0[d][I], qhi = q0[d][I + st[d]];
        const T dl = over_D(a, a.lam * (Tc - Tm), d), dr = over_D(a, a.lam * (Tp - Tc), d);
        ql[d] = (ix[d] == 1 && a.kind[d][0] == FI_HEAT_FLUX) ? a.val[d][0] : qlo - (qlo + dl) * a.dtq;
        qr[d] = (ix[d] == a.n[d] && a.kind[d][1] == FI_HEAT_FLUX) ? a.val[d][1] : qhi - (qhi + dr) * a.dtq;
    }
    const T gq = over_D(a, qr[0] - ql[0], 0) + over_D(a, qr[1] - ql[1], 1) + over_D(a, qr[2] - ql[2], 2);
    const T Tn = Tc - (over_dt(a, Tc - a.To[I]) + gq) * a.dtT;
    a.T1[I] = Tn;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        q1[d][I] = ql[d];
        if (ix[d] == a.n[d]) q1[d][I + st[d]] = qr[d];
        if (ix[d] == 1 && a.kind[d][0] == FI_HEAT_VALUE) a.T1[I - st[d]] = T(2.0) * a.val[d][0] - Tn;
        if (ix[d] == a.n[d] && a.kind[d][1] == FI_HEAT_VALUE) a.T1[I + st[d]] = T(2.0) * a.val[d][1] - Tn;
    }
}

// initial boundary fill (the drivers' _apply_bcs! after set!): Flux nodes of q,
// then Value ghosts of T, faces as in the oracle (dims before d over their whole
// storage range, dims after d over the interior)
template <typename T>
__global__ void heat_face(T *f, int n0, int n1, int n2, long long sx, long long sxy, int d, int side, int vertex, T v) {
    const int n[3] = {n0, n1, n2};
    int lo[3], cnt[3];
    for (int e = 0; e < 3; e++) {
        const int nv = n[e] + ((vertex && e == d) ? 1 : 0);
        if (e < d) { lo[e] = 0; cnt[e] = n[e] + 3; }
        else { lo[e] = 1; cnt[e] = nv; }
    }
    const int at = vertex ? (side == 0 ? 1 : n[d] + 1) : (side == 0 ? 0 : n[d] + 1);
    const int adj = side == 0 ? 1 : n[d];
    cnt[d] = 1;
    const long long total = (long long)cnt[0] * cnt[1] * cnt[2];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int c[3];
        c[0] = lo[0] + (int)(t % cnt[0]);
        c[1] = lo[1] + (int)((t / cnt[0]) % cnt[1]);
        c[2] = lo[2] + (int)(t / ((long long)cnt[0] * cnt[1]));
        c[d] = at;
        const long long I = c[0] + sx * c[1] + sxy * c[2];
        if (vertex) {
            f[I] = v;
        } else {
            int a2[3] = {c[0], c[1], c[2]};
            a2[d] = adj;
            f[I] = T(2.0) * v - f[a2[0] + sx * a2[1] + sxy * a2[2]];
        }
    }
}

void *heat_ptr(const fi_heat *h, int field, int buf) {
    switch (field) {
        case FI_HEAT_T: return h->T[buf];
        case FI_HEAT_T_OLD: return h->To;
        case FI_HEAT_QX: return h->q[0][buf];
        case FI_HEAT_QY: return h->q[1][buf];
        case FI_HEAT_QZ: return h->q[2][buf];
        default: return nullptr;
    }
}

// interior extent of a field: T, T_o Center; q_d Vertex along d
void heat_shape(const fi_heat *h, int field, int ext[3]) {
    for (int e = 0; e < 3; e++) ext[e] = h->d.grid.n[e];
    if (field >= FI_HEAT_QX) ext[field - FI_HEAT_QX] += 1;
}

cudaMemcpy3DParms heat_copy(const fi_heat *h, int field, void *dev, void *host, bool to_dev) {
    int ext[3];
    heat_shape(h, field, ext);
    cudaMemcpy3DParms p{};
    char *base = (char *)dev - kHeatOff * h->esz;
    cudaPitchedPtr dp = make_cudaPitchedPtr(base, (size_t)h->pitch * h->esz, (size_t)h->pitch, (size_t)h->rows);
    cudaPitchedPtr hp = make_cudaPitchedPtr(host, (size_t)ext[0] * h->esz, (size_t)ext[0], (size_t)ext[1]);
    cudaPos dpos = make_cudaPos((size_t)(kHeatOff + 1) * h->esz, 1, 1);
    if (to_dev) {
        p.srcPtr = hp;
        p.dstPtr = dp;
        p.dstPos = dpos;
        p.kind = cudaMemcpyHostToDevice;
    } else {
        p.srcPtr = dp;
        p.srcPos = dpos;
        p.dstPtr = hp;
        p.kind = cudaMemcpyDeviceToHost;
    }
    p.extent = make_cudaExtent((size_t)ext[0] * h->esz, (size_t)ext[1], (size_t)ext[2]);
    return p;
}

template <typename T>
fi_status heat_bcs_t(fi_heat *h) {
    const int *n = h->d.grid.n;
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++)
            if (h->d.kind[d][s] == FI_HEAT_FLUX)
                heat_face<T><<<64, 256, 0, h->stream>>>((T *)h->q[d][h->cur], n[0], n[1], n[2], h->pitch,
                                                         h->pitch * h->rows, d, s, 1, T(h->d.value[d][s]));
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++)
            if (h->d.kind[d][s] == FI_HEAT_VALUE)
                heat_face<T><<<64, 256, 0, h->stream>>>((T *)h->T[h->cur], n[0], n[1], n[2], h->pitch,
                                                         h->pitch * h->rows, d, s, 0, T(h->d.value[d][s]));
    FI_CHECK_CUDA(cudaGetLastError(), "heat boundary faces");
    return FI_OK;
}

template <typename T>
fi_status heat_advance_t(fi_heat *h, int niter, double dt) {
    HeatArgs<T> a{};
    for (int e = 0; e < 3; e++) {
        a.n[e] = h->d.grid.n[e];
        a.D[e] = T(h->d.grid.extent[e] / h->d.grid.n[e]);
        a.iD[e] = T(1) / a.D[e];
        for (int s = 0; s < 2; s++) {
            a.kind[e][s] = h->d.kind[e][s];
            a.val[e][s] = T(h->d.value[e][s]);
        }
    }
    a.sx = h->pitch;
    a.sxy = h->pitch * h->rows;
    a.lam = T(h->d.lambda_rhocp);
    a.dtq = T(h->d.dtau_q);
    a.dtT = T(h->d.dtau_T);
    a.dt = T(dt);
    a.idt = T(1) / a.dt;
    a.To = (const T *)h->To;
    const dim3 blk(32, 8), grd((a.n[0] + 31) / 32, (a.n[1] + 7) / 8, a.n[2]);
    for (int it = 0; it < niter; it++) {
        const int c = h->cur, o = c ^ 1;
        a.T0 = (const T *)h->T[c];
        a.qx0 = (const T *)h->q[0][c];
        a.qy0 = (const T *)h->q[1][c];
        a.qz0 = (const T *)h->q[2][c];
        a.T1 = (T *)h->T[o];
        a.qx1 = (T *)h->q[0][o];
        a.qy1 = (T *)h->q[1][o];
        a.qz1 = (T *)h->q[2][o];
        heat_sweep<T><<<grd, blk, 0, h->stream>>>(a);
        FI_CHECK_CUDA(cudaGetLastError(), "heat sweep");
        h->cur = o;
    }
    return FI_OK;
}

void heat_free(fi_heat *h) {
    auto rel = [&](void *p) {
        if (p) cudaFree((char *)p - kHeatOff * h->esz);
    };
    for (int b = 0; b < 2; b++) {
        rel(h->T[b]);
        for (int d = 0; d < 3; d++) rel(h->q[d][b]);
    }
    rel(h->To);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // namespace
}  // namespace fi

using namespace fi;

extern "C" {

fi_status fi_heat_create(const fi_heat_desc *desc, fi_heat **out) {
    if (!desc || !out) return set_error("bad argument"), FI_ERR_ARG;
    *out = nullptr;
    const fi_grid &g = desc->grid;
    if (g.nd != 3) return set_error("the heat model is 3D (kernels.jl:3-29)"), FI_ERR_UNSUPPORTED;
    for (int k = 0; k < 3; k++)
        if (g.n[k] < 1 || !(g.extent[k] > 0.0)) return set_error("invalid grid"), FI_ERR_ARG;
    for (int k = 0; k < 3; k++)
        for (int s = 0; s < 2; s++)
            if (desc->kind[k][s] != FI_HEAT_VALUE && desc->kind[k][s] != FI_HEAT_FLUX)
                return set_error("boundary kinds must be FI_HEAT_VALUE or FI_HEAT_FLUX"), FI_ERR_ARG;
    if (desc->dtype != FI_F64 && desc->dtype != FI_F32) return set_error("dtype must be FI_F64 or FI_F32"), FI_ERR_ARG;
    fi_heat *h = new fi_heat();
    h->d = *desc;
    h->esz = desc->dtype == FI_F64 ? 8 : 4;
    h->pitch = ((kHeatOff + g.n[0] + 3 + 31) / 32) * 32;
    h->rows = g.n[1] + 3;
    h->elems = (size_t)h->pitch * (size_t)h->rows * (size_t)(g.n[2] + 3);
    cudaError_t e = cudaSetDevice(desc->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    auto alloc = [&](void **p) -> cudaError_t {
        char *raw = nullptr;
        const size_t bytes = (h->elems + 64) * h->esz;
        cudaError_t r = cudaMalloc(&raw, bytes);
        if (r != cudaSuccess) return r;
        r = cudaMemsetAsync(raw, 0, bytes, h->stream);
        *p = raw + kHeatOff * h->esz;
        return r;
    };
    for (int b = 0; b < 2 && e == cudaSuccess; b++) {
        e = alloc(&h->T[b]);
        for (int d = 0; d < 3 && e == cudaSuccess; d++) e = alloc(&h->q[d][b]);
    }
    if (e == cudaSuccess) e = alloc(&h->To);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        fi_status st = cuda_fail(e, "heat model allocation");
        heat_free(h);
        return st;
    }
    *out = h;
    return FI_OK;
}

fi_status fi_heat_destroy(fi_heat *h) {
    if (!h) return FI_OK;
    cudaSetDevice(h->d.device);
    cudaStreamSynchronize(h->stream);
    heat_free(h);
    return FI_OK;
}

fi_status fi_heat_field_size(const fi_heat *h, int32_t field, size_t *count) {
    if (!h || !count || field < FI_HEAT_T || field > FI_HEAT_QZ) return set_error("bad argument"), FI_ERR_ARG;
    int ext[3];
    heat_shape(h, field, ext);
    *count = (size_t)ext[0] * ext[1] * ext[2];
    return FI_OK;
}

fi_status fi_heat_set_field(fi_heat *h, int32_t field, const void *host, size_t nbytes) {
    size_t cnt = 0;
    fi_status st = fi_heat_field_size(h, field, &cnt);
    if (st != FI_OK) return st;
    if (!host || nbytes != cnt * h->esz) return set_error("byte count does not match the field's interior"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(h->d.device), "cudaSetDevice");
    cudaMemcpy3DParms p = heat_copy(h, field, heat_ptr(h, field, h->cur), const_cast<void *>(host), true);
    FI_CHECK_CUDA(cudaMemcpy3DAsync(&p, h->stream), "heat set_field");
    FI_CHECK_CUDA(cudaStreamSynchronize(h->stream), "heat set_field");
    return FI_OK;
}

fi_status fi_heat_get_field(fi_heat *h, int32_t field, void *host, size_t nbytes) {
    size_t cnt = 0;
    fi_status st = fi_heat_field_size(h, field, &cnt);
    if (st != FI_OK) return st;
    if (!host || nbytes != cnt * h->esz) return set_error("byte count does not match the field's interior"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(h->d.device), "cudaSetDevice");
    cudaMemcpy3DParms p = heat_copy(h, field, heat_ptr(h, field, h->cur), host, false);
    FI_CHECK_CUDA(cudaMemcpy3DAsync(&p, h->stream), "heat get_field");
    FI_CHECK_CUDA(cudaStreamSynchronize(h->stream), "heat get_field");
    return FI_OK;
}

fi_status fi_heat_apply_bcs(fi_heat *h) {
    if (!h) return set_error("null model"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(h->d.device), "cudaSetDevice");
    fi_status st = h->esz == 8 ? heat_bcs_t<double>(h) : heat_bcs_t<float>(h);
    if (st != FI_OK) return st;
    FI_CHECK_CUDA(cudaStreamSynchronize(h->stream), "heat boundary faces");
    return FI_OK;
}

fi_status fi_heat_advance(fi_heat *h, int32_t niter, double dt) {
    if (!h || niter < 0 || !(dt > 0.0)) return set_error("bad argument"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(h->d.device), "cudaSetDevice");
    return h->esz == 8 ? heat_advance_t<double>(h, niter, dt) : heat_advance_t<float>(h, niter, dt);
}

fi_status fi_heat_stream(const fi_heat *h, void **stream) {
    if (!h || !stream) return set_error("bad argument"), FI_ERR_ARG;
    *stream = (void *)h->stream;
    return FI_OK;
}

fi_status fi_heat_synchronize(fi_heat *h) {
    if (!h) return set_error("null model"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaStreamSynchronize(h->stream), "heat sync");
    return FI_OK;
}

}  // extern "C"
