// fi_device.cuh -- device helpers shared by the reference-shaped and fused kernels.
#pragma once

#include "fi_internal.h"

namespace fi {

template <typename T>
__device__ __forceinline__ T ipow_dev(T x, int m) {
    // integer exponent as Julia evaluates x^n for an Int n: n == 2 -> x*x, n == 3 -> x*x*x
    if (m == 2) return x * x;
    if (m == 3) return x * x * x;
    if (m == 1) return x;
    if (m == 0) return T(1);
    const int a = m < 0 ? -m : m;
    T r = a == 2 ? x * x : (a == 3 ? x * x * x : (a == 1 ? x : T(pow(double(x), double(a)))));
    return m < 0 ? T(1) / r : r;
}

// rheology(τII, I): src/Physics.jl:11 (linear), :18 (power law), :26
// (viscoplastic regularisation), :46-47 (relaxation of the current viscosity)
template <typename T>
__device__ __forceinline__ T rheology_dev(const KParams &p, const T *eta_lin, const T *Afield, T eta_cur, long long I,
                                          T tII) {
    T inner;
    if (p.rheo_inner == FI_RHEO_LINEAR) {
        inner = p.rheo_eta_is_field ? eta_lin[I] : T(p.rheo_eta);
    } else {
        T A = p.rheo_A_is_field ? Afield[I] : T(p.rheo_A);
        inner = T(0.5) / (A * ipow_dev(tII, p.rheo_n - 1));
    }
    if (p.rheo_has_reg) inner = T(1.0) / (T(1.0) / inner + T(p.rheo_inv_eta_reg));
    if (p.rheo_relax != FI_RELAX_NONE) {
        T a = T(1.0 - p.rheo_rate), b = T(p.rheo_rate);
        if (p.rheo_relax == FI_RELAX_LIN) {
            inner = eta_cur * a + inner * b;
        } else if (p.rheo_relax == FI_RELAX_LOG) {
            inner = T(exp(double(T(log(double(eta_cur))) * a + T(log(double(inner))) * b)));
        } else {
            inner = T(pow(10.0, double(T(log10(double(eta_cur))) * a + T(log10(double(inner))) * b)));
        }
    }
    return inner;
}

// A linear viscosity with neither regularisation nor relaxation: the new
// viscosity is the linear one, whatever the stresses (rheology_dev above).
__device__ __forceinline__ bool linear_unrelaxed(const KParams &p) {
    return p.rheo_inner == FI_RHEO_LINEAR && !p.rheo_has_reg && p.rheo_relax == FI_RELAX_NONE;
}

template <typename T>
__device__ __forceinline__ T gravity_dev(const KParams &p, const T *arr, int c, long long I) {
    return p.g_kind[c] == FI_G_FIELD ? arr[I] : T(p.g_val[c]);
}

// sqrt with IEEE rounding in both precisions
__device__ __forceinline__ double sqrt_dev(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_dev(float x) { return __fsqrt_rn(x); }
__device__ __forceinline__ double div_dev(double a, double b) { return a / b; }
__device__ __forceinline__ float div_dev(float a, float b) { return __fdiv_rn(a, b); }

// Reciprocal by Newton-Raphson iteration r <- r + r (1 - b r) from the hardware
// approximation (PTX rcp.approx.ftz): each step doubles the number of correct
// bits, two steps in FP64 and one in FP32 reach the last bit or so.  Production
// sweeps divide as a * rcp(b) (within a few ulp of the rounded quotient, no
// special-case branches); FI_EXACT_ORDER builds keep the rounded division.
__device__ __forceinline__ double rcp_nr(double b) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    double e = fma(-b, r, 1.0);
    r = fma(r, e, r);
    e = fma(-b, r, 1.0);
    return fma(r, e, r);
}
__device__ __forceinline__ float rcp_nr(float b) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    const float e = fmaf(-b, r, 1.0f);
    return fmaf(r, e, r);
}
template <typename T>
__device__ __forceinline__ T div_fast(T a, T b) {
#ifdef FI_EXACT_ORDER
    return div_dev(a, b);
#else
    return a * rcp_nr(b);
#endif
}
// x / 3 (the deviatoric split); production builds multiply by the rounded 1/3
template <typename T>
__device__ __forceinline__ T third(T x) {
#ifdef FI_EXACT_ORDER
    return x / T(3.0);
#else
    return x * T(1.0 / 3.0);
#endif
}

// η_next from τII² = s2 (rheology(τII) with τII = sqrt(s2)).  Production builds
// evaluate Glen's law with the integer exponent n = 3 as 0.5/(A s2) and its
// viscoplastic regularisation as 1/(2 A s2 + 1/η_reg): the same function without
// the square root and with one division instead of three (a few ulp from the
// reference's rounding sequence).  Builds with FI_EXACT_ORDER keep the
// reference's operation order (sqrt, then the divisions of Physics.jl:18, :26)
// for bit-level comparison with the CPU oracle.
template <typename T>
__device__ __forceinline__ T rheology_s2(const KParams &p, T A_const, T inv_reg, const T *eta_lin, const T *Afield,
                                         T eta_cur, long long I, T s2) {
#ifndef FI_EXACT_ORDER
    if (p.rheo_inner == FI_RHEO_POWER && p.rheo_n == 3 && p.rheo_relax == FI_RELAX_NONE) {
        T A = p.rheo_A_is_field ? Afield[I] : A_const;
        T As2 = A * s2;
        return p.rheo_has_reg ? rcp_nr(T(2.0) * As2 + inv_reg) : div_fast(T(0.5), As2);
    }
#endif
    return rheology_dev(p, eta_lin, Afield, eta_cur, I, sqrt_dev(s2));
}

// immersed-boundary mask components: ccc vvv vcc cvc ccv vvc vcv cvv
enum { W_CCC = 0, W_VVV, W_VCC, W_CVC, W_CCV, W_VVC, W_VCV, W_CVV };

template <typename T>
__device__ __forceinline__ bool small_dev(T w, T thr) {
    return w < thr;
}

// isnullspace: src/Models/ImmersedBoundaryFullStokes/Isothermal/null_spaces.jl:13-37
template <typename T>
__device__ __forceinline__ bool nullspace_dev(const T *const w[8], int comp, long long I, long long sx, long long sxy,
                                              T thr) {
    switch (comp) {
        case W_CCC:
            return small_dev(w[W_VCC][I], thr) || small_dev(w[W_VCC][I + 1], thr) || small_dev(w[W_CVC][I], thr) ||
                   small_dev(w[W_CVC][I + sx], thr) || small_dev(w[W_CCV][I], thr) || small_dev(w[W_CCV][I + sxy], thr);
        case W_VCC:
            return small_dev(w[W_CCC][I - 1], thr) || small_dev(w[W_CCC][I], thr) || small_dev(w[W_VVC][I], thr) ||
                   small_dev(w[W_VVC][I + sx], thr) || small_dev(w[W_VCV][I], thr) || small_dev(w[W_VCV][I + sxy], thr);
        case W_CVC:
            return small_dev(w[W_VVC][I], thr) || small_dev(w[W_VVC][I + 1], thr) || small_dev(w[W_CCC][I - sx], thr) ||
                   small_dev(w[W_CCC][I], thr) || small_dev(w[W_CVV][I], thr) || small_dev(w[W_CVV][I + sxy], thr);
        case W_CCV:
            return small_dev(w[W_VCV][I], thr) || small_dev(w[W_VCV][I + 1], thr) || small_dev(w[W_CVV][I], thr) ||
                   small_dev(w[W_CVV][I + sx], thr) || small_dev(w[W_CCC][I - sxy], thr) || small_dev(w[W_CCC][I], thr);
        case W_VVC:
            return small_dev(w[W_CVC][I - 1], thr) || small_dev(w[W_CVC][I], thr) || small_dev(w[W_VCC][I - sx], thr) ||
                   small_dev(w[W_VCC][I], thr);
        case W_VCV:
            return small_dev(w[W_CCV][I - 1], thr) || small_dev(w[W_CCV][I], thr) || small_dev(w[W_VCC][I - sxy], thr) ||
                   small_dev(w[W_VCC][I], thr);
        case W_CVV:
            return small_dev(w[W_CCV][I - sx], thr) || small_dev(w[W_CCV][I], thr) || small_dev(w[W_CVC][I - sxy], thr) ||
                   small_dev(w[W_CVC][I], thr);
        default:
            return false;
    }
}

// isvalid(a, loc, I) && !isempty(b, loc, I)  (null_spaces.jl:41-43)
template <typename T>
__device__ __forceinline__ bool active_dev(const T *const a[8], const T *const b[8], int comp, long long I, long long sx,
                                           long long sxy, T thr) {
    bool valid = !(nullspace_dev(a, comp, I, sx, sxy, thr) || small_dev(a[comp][I], thr));
    return valid && !small_dev(b[comp][I], thr);
}

// the activity byte at index I: precomputed when the model provides it, else the
// seven predicates of null_spaces.jl:41-43 evaluated here
template <typename T>
__device__ __forceinline__ unsigned ib_flags_at(const Ptrs<T> &f, long long I, long long sx, long long sxy, T thr) {
    if (f.ibf) return __ldg(f.ibf + I);  // read-only while the kernels run
    unsigned b = 0;
    if (active_dev(f.wna, f.wns, W_CCC, I, sx, sxy, thr)) b |= IBF_S_CCC;
    if (active_dev(f.wna, f.wns, W_VVC, I, sx, sxy, thr)) b |= IBF_S_VVC;
    if (active_dev(f.wna, f.wns, W_VCV, I, sx, sxy, thr)) b |= IBF_S_VCV;
    if (active_dev(f.wna, f.wns, W_CVV, I, sx, sxy, thr)) b |= IBF_S_CVV;
    if (active_dev(f.wns, f.wna, W_VCC, I, sx, sxy, thr)) b |= IBF_V_VCC;
    if (active_dev(f.wns, f.wna, W_CVC, I, sx, sxy, thr)) b |= IBF_V_CVC;
    if (active_dev(f.wns, f.wna, W_CCV, I, sx, sxy, thr)) b |= IBF_V_CCV;
    return b;
}

}  // namespace fi
