// fi_model.h -- the model object behind the opaque fi_model handle, shared by
// the translation units that drive a model's device state (fi_api.cu,
// fi_batch.cu).
#pragma once

#include "fi_internal.h"

namespace fi {
constexpr int kState = 10;  // P, txx, tyy, tzz, txy, txz, tyz, Vx, Vy, Vz
}  // namespace fi

struct fi_model {
    using Geom = fi::Geom;
    using KParams = fi::KParams;
    template <typename T>
    using Ptrs = fi::Ptrs<T>;
    static constexpr int kState = fi::kState;

    fi_model_desc d{};
    Geom g{};
    KParams kp{};
    size_t esz = 8;
    size_t elems = 0;
    void *base[FI_FIELD_COUNT] = {};
    void *alt[kState] = {};
    int parity = 0;           // 1: alt[] holds the current P..Vz
    bool eta_swapped = false; // true: base[ETA_NEXT] holds the current eta
    cudaStream_t stream = nullptr;
    double *d_partials = nullptr;
    double *d_out = nullptr;
    double *h_out = nullptr;
    int nblk = 0;
    int path = FI_PATH_REFERENCE;
    int fused_variant = 0;
    int maps_key = -1;  // launch-shape key (fused3d_variant_key) the tensor maps were encoded for
    bool ib = false;
    long long iterations = 0;
    int *d_err = nullptr;  // device error word written by bounded waits
    unsigned char *d_ibf = nullptr;  // immersed-boundary activity byte per grid index (IbFlag bits)
    uint2 *d_blist = nullptr;        // blocks an immersed-boundary update runs once zeros hold (BlockList)
    int *d_bcount = nullptr;
    int n_blist = 0;
    // reference-shaped path: two iterations captured as a CUDA graph, one per η
    // buffer parity at the start of the pair, with the parameters they were captured with
    cudaGraphExec_t pair_graph[2] = {nullptr, nullptr};
    KParams pair_kp[2]{};
    bool ibf_stale = true;           // the volume fractions changed since d_ibf was computed
    // Full immersed-boundary iterations since anything else wrote the state, η or
    // the volume fractions.  After one, inactive strict-interior points of P, τ, V
    // hold zero (boundary batches write only indices 0, 1, n+1, n+2 of their
    // dimension, so they never break it); after two, both η buffers hold the
    // viscosity of every point outside the block list.  A state pointer handed to
    // a caller ends both for good.
    int full_iters = 0;
    bool state_ptr_out = false;
    void *fP = nullptr;    // pressure forcing (defect-correction shadow models only)
    void *d_stage = nullptr;  // staging buffer of set_field (contiguous rows of host data)
    size_t stage_bytes = 0;
    fi_model *shadow = nullptr;  // FP32 model of the mixed-precision solve (created on first use)
    KParams shadow_kp{};         // the shadow's parameters as created (gravity as fields); each solve starts from them
    // TMA maps (128 bytes each) of every buffer the fused sweep reads
    alignas(64) unsigned char map_base[kState][128];
    alignas(64) unsigned char map_alt[kState][128];
    alignas(64) unsigned char map_eta[2][128];  // base[ETA], base[ETA_NEXT]
    // overlapped iteration (fi_model_advance_begin / _end): the second half of an
    // iteration (the tiles away from the split faces) runs on stream2 while the halo
    // moves on `stream`; ev_int marks its end, ev_bnd the end of the first half
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_bnd = nullptr, ev_int = nullptr;
    bool interior_pending = false;  // stream2 work that `stream` has not waited for yet
    int split_begun = -1;           // split dimension of a begun iteration awaiting its second half
    alignas(64) unsigned char pend_maps[18][128];
    unsigned char pend_ptrs[2][sizeof(fi::Ptrs<double>)];  // in / out of the begun iteration
    // trimmed-box maps of the seven stress fields (interior columns of trimmed launch shapes)
    alignas(64) unsigned char tmap_base[7][128];
    alignas(64) unsigned char tmap_alt[7][128];

    bool is_f64() const { return d.dtype == FI_F64; }

    void *cur(int field) const {
        if (field < kState) return parity ? alt[field] : base[field];
        if (field == FI_FIELD_ETA) return eta_swapped ? base[FI_FIELD_ETA_NEXT] : base[FI_FIELD_ETA];
        if (field == FI_FIELD_ETA_NEXT) return eta_swapped ? base[FI_FIELD_ETA] : base[FI_FIELD_ETA_NEXT];
        return base[field];
    }
    void *nxt(int field) const { return parity ? base[field] : alt[field]; }

    template <typename T>
    Ptrs<T> ptrs(bool next_state = false) const {
        Ptrs<T> f{};
        auto S = [&](int fld) { return (T *)(next_state ? nxt(fld) : cur(fld)); };
        f.P = S(FI_FIELD_P);
        f.txx = S(FI_FIELD_TXX);
        f.tyy = S(FI_FIELD_TYY);
        f.tzz = S(FI_FIELD_TZZ);
        f.txy = S(FI_FIELD_TXY);
        f.txz = S(FI_FIELD_TXZ);
        f.tyz = S(FI_FIELD_TYZ);
        f.Vx = S(FI_FIELD_VX);
        f.Vy = S(FI_FIELD_VY);
        f.Vz = S(FI_FIELD_VZ);
        f.eta = (T *)cur(FI_FIELD_ETA);
        f.eta_next = (T *)cur(FI_FIELD_ETA_NEXT);
        f.rP = (T *)base[FI_FIELD_RP];
        f.rVx = (T *)base[FI_FIELD_RVX];
        f.rVy = (T *)base[FI_FIELD_RVY];
        f.rVz = (T *)base[FI_FIELD_RVZ];
        f.gx = (const T *)base[FI_FIELD_GX];
        f.gy = (const T *)base[FI_FIELD_GY];
        f.gz = (const T *)base[FI_FIELD_GZ];
        f.eta_lin = (const T *)base[FI_FIELD_ETA_LIN];
        f.A = (const T *)base[FI_FIELD_A];
        f.fP = (const T *)fP;
        for (int c = 0; c < 8; c++) {
            f.wna[c] = (const T *)base[FI_FIELD_NA_CCC + c];
            f.wns[c] = (const T *)base[FI_FIELD_NS_CCC + c];
        }
        f.ibf = ibf_stale ? nullptr : d_ibf;  // stale bytes are never read: the kernels evaluate the predicates
        return f;
    }
};

// Stages of the FP32-in-FP64 defect correction of an FP64 model (fi_api.cu), shared
// by fi_model_solve (mode MIXED) and fi_batch_solve_mixed:
//   mixed_shadow            the FP32 shadow (created on first use, masks refreshed)
//   mixed_phase_a_begin/end the full problem rounded into the shadow / back
//   mixed_picard            η from the FP64 stresses
//   mixed_correction_begin  projection, FP64 residuals, the shadow's correction problem
//   mixed_correction_end    x += δ
fi_status mixed_shadow(fi_model *m);
fi_status mixed_phase_a_begin(fi_model *m);
fi_status mixed_phase_a_end(fi_model *m);
fi_status mixed_picard(fi_model *m);
fi_status mixed_correction_begin(fi_model *m);
fi_status mixed_correction_end(fi_model *m);
// the boundary batches of the reference-shaped iteration (fi_api.cu) and the refresh of
// an immersed-boundary model's activity bytes and block list when stale
fi::BcBatch model_stress_batch(const fi_model *m, int d);
fi::BcBatch model_velocity_batch(const fi_model *m, int d);
fi_status model_refresh_ibf(fi_model *m);
// allocates the second buffer of every state field a model lacks (fi_api.cu)
fi_status model_ensure_second_state(fi_model *m);
// whether the model stores field f (fi_api.cu)
bool model_field_used(const fi_model *m, int f);
