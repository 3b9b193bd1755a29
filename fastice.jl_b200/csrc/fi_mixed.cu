// fi_mixed.cu -- element-wise kernels of the mixed-precision defect-correction
// solve (fi_model_solve with FI_SOLVE_MIXED): precision conversion between an
// FP64 model and its FP32 shadow, FP64 accumulation of an FP32 correction, and the
// viscosity refresh η = rheology(τII(τ)) of the nonlinear (Picard) outer step.
//
// The conversion and accumulation kernels run over a field's whole storage box
// (ghosts included): every boundary rule is linear in the field, so ghosts of a
// correction that satisfies homogeneous boundary values add to ghosts of a state
// that satisfies the actual values without breaking them.
#include "fi_device.cuh"

namespace fi {
namespace {

template <typename S, typename D>
__global__ void convert_scale_kernel(const S *__restrict__ src, D *__restrict__ dst, long long n, double scale) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        dst[t] = scale == 1.0 ? D(src[t]) : D(scale * double(src[t]));
}

template <typename D, typename S>
__global__ void accumulate_kernel(D *__restrict__ x, const S *__restrict__ d, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        x[t] += D(d[t]);
}

// out = (D)(a - b), the difference taken in the source precision
template <typename S, typename D>
__global__ void diff_kernel(const S *__restrict__ a, const S *__restrict__ b, D *__restrict__ out, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = D(a[t] - b[t]);
}

// A volume fraction rounded to FP32 for a shadow model whose emptiness threshold
// is thr32 (the smallest float >= 1e-6): values below 1e-6 stay below thr32 and
// the others stay at or above it, so both precisions see the same empty, valid
// and null-space points (rounding to nearest alone could lift a value just under
// 1e-6 onto thr32)
__global__ void mask_to_f32_kernel(const double *__restrict__ src, float *__restrict__ dst, long long n, float thr32) {
    const float below = nextafterf(thr32, 0.0f);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double w = src[t];
        const float r = (float)w;
        dst[t] = w < 1e-6 ? fminf(r, below) : fmaxf(r, thr32);
    }
}

template <typename T>
__device__ __forceinline__ T h(T x) { return T(0.5) * x; }

// η_next at every cell from the current τ (the τII / rheology part of update_V!,
// kernels_3d.jl:215-220, kernels_2d.jl:154-155)
template <typename T, int ND>
__global__ void eta_from_tau_kernel(Geom g, KParams p, Ptrs<T> f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = ND == 3 ? (int)blockIdx.z + 1 : 0;
    if (i > g.n[0] || j > g.n[1]) return;
    const long long sx = g.pitch, sxy = g.sxy;
    const long long I = (long long)i + sx * ((long long)j + g.rows * (long long)k);
    const T *txx = f.txx, *tyy = f.tyy, *txy = f.txy;
    T s2;
    if (ND == 2) {
        T lxy = h(h(txy[I] + txy[I + 1]) + h(txy[I + sx] + txy[I + sx + 1]));
        s2 = T(0.5) * (txx[I] * txx[I] + tyy[I] * tyy[I]) + lxy * lxy;
    } else {
        const T *tzz = f.tzz, *txz = f.txz, *tyz = f.tyz;
        T lxy = h(h(txy[I] + txy[I + 1]) + h(txy[I + sx] + txy[I + sx + 1]));
        T lxz = h(h(txz[I] + txz[I + 1]) + h(txz[I + sxy] + txz[I + sxy + 1]));
        T lyz = h(h(tyz[I] + tyz[I + sx]) + h(tyz[I + sxy] + tyz[I + sxy + sx]));
        s2 = T(0.5) * (txx[I] * txx[I] + tyy[I] * tyy[I] + tzz[I] * tzz[I]) + lxy * lxy + lxz * lxz + lyz * lyz;
    }
    f.eta_next[I] = rheology_s2(p, T(p.rheo_A), T(p.rheo_inv_eta_reg), f.eta_lin, f.A, f.eta[I], I, s2);
}

// largest |value| over several fields' storage boxes; non-negative floats order
// like their bit patterns, so an integer atomicMax of the bits is exact and
// independent of the order of the updates
struct AbsMaxArgs {
    const float *f[8];
    int count;
};
__global__ void absmax_kernel(AbsMaxArgs a, long long n, unsigned *out) {
    float m = 0.0f;
    for (int q = 0; q < a.count; q++)
        for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
            m = fmaxf(m, fabsf(a.f[q][t]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

unsigned grid_1d(long long n) {
    long long b = (n + 255) / 256;
    return (unsigned)(b > 148LL * 32 ? 148LL * 32 : (b < 1 ? 1 : b));
}

}  // namespace

template <typename S, typename D>
cudaError_t launch_convert(const S *src, D *dst, long long n, double scale, cudaStream_t s) {
    convert_scale_kernel<S, D><<<grid_1d(n), 256, 0, s>>>(src, dst, n, scale);
    return cudaGetLastError();
}

template <typename D, typename S>
cudaError_t launch_accumulate(D *x, const S *d, long long n, cudaStream_t s) {
    accumulate_kernel<D, S><<<grid_1d(n), 256, 0, s>>>(x, d, n);
    return cudaGetLastError();
}

cudaError_t launch_mask_to_f32(const double *src, float *dst, long long n, float thr32, cudaStream_t s) {
    mask_to_f32_kernel<<<grid_1d(n), 256, 0, s>>>(src, dst, n, thr32);
    return cudaGetLastError();
}

template <typename S, typename D>
cudaError_t launch_diff(const S *a, const S *b, D *out, long long n, cudaStream_t s) {
    diff_kernel<S, D><<<grid_1d(n), 256, 0, s>>>(a, b, out, n);
    return cudaGetLastError();
}
template cudaError_t launch_diff<double, float>(const double *, const double *, float *, long long, cudaStream_t);

template <typename T>
cudaError_t launch_eta_from_tau(const Geom &g, const KParams &p, const Ptrs<T> &f, cudaStream_t s) {
    dim3 blk(32, 8);
    dim3 grd((g.n[0] + 31) / 32, (g.n[1] + 7) / 8, g.nd == 3 ? g.n[2] : 1);
    if (g.nd == 3) eta_from_tau_kernel<T, 3><<<grd, blk, 0, s>>>(g, p, f);
    else eta_from_tau_kernel<T, 2><<<grd, blk, 0, s>>>(g, p, f);
    return cudaGetLastError();
}

cudaError_t launch_absmax_f32(const float *const *fields, int count, long long n, unsigned *out_bits, cudaStream_t s) {
    AbsMaxArgs a{};
    a.count = count < 8 ? count : 8;
    for (int q = 0; q < a.count; q++) a.f[q] = fields[q];
    cudaError_t e = cudaMemsetAsync(out_bits, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    absmax_kernel<<<grid_1d(n), 256, 0, s>>>(a, n, out_bits);
    return cudaGetLastError();
}

template cudaError_t launch_convert<double, float>(const double *, float *, long long, double, cudaStream_t);
template cudaError_t launch_convert<float, double>(const float *, double *, long long, double, cudaStream_t);
template cudaError_t launch_accumulate<double, float>(double *, const float *, long long, cudaStream_t);
template cudaError_t launch_eta_from_tau<double>(const Geom &, const KParams &, const Ptrs<double> &, cudaStream_t);
template cudaError_t launch_eta_from_tau<float>(const Geom &, const KParams &, const Ptrs<float> &, cudaStream_t);

}  // namespace fi
