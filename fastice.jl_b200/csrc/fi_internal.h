// fi_internal.h -- internal types shared by the libfastice_b200 translation units.
//
// Storage: every field of a model lives in one uniform halo box per model:
// (n0+3) x (n1+3) x (n2+3) logical elements (vertex count + one ghost layer on
// each side, for every staggered location), x fastest.  Index (i,j,k) maps to
// field[i + pitch*(j + rows*k)] where the field pointer sits kXOff elements past
// its allocation, and pitch is a multiple of 32: interior index 1 of every row
// starts on a 256-byte (FP64) / 128-byte (FP32) boundary, so a warp storing 32
// consecutive positions of a column tile writes whole 32-byte sectors.  Index 0
// is the left ghost, 1..N_loc the interior (N_loc = n or n+1 per location).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/fastice_b200.h"

namespace fi {

constexpr int kMaxBcOps = 16;
constexpr long long kXOff = 31;  // field pointer offset (elements) inside its allocation
constexpr int kNormSlots = 12;  // per-block partial slots (FI_NORMS_LEN layout)

// geometry as seen by device code
struct Geom {
    int nd;
    int n[3];
    long long pitch;  // elements per x row
    long long rows;   // rows per plane (n1 + 3)
    long long sxy;    // pitch * rows
    long long planes; // n2 + 3 (1 in 2D)
};

// scalar parameters as seen by device code (doubles; kernels convert to T
// exactly as the host would: (T)value)
struct KParams {
    double inv_dx[3];
    double dt_P, dt_tau[6], dt_V[3];
    int g_kind[3];
    double g_val[3];
    int rheo_inner, rheo_eta_is_field, rheo_A_is_field, rheo_n, rheo_has_reg, rheo_relax;
    double rheo_eta, rheo_A, rheo_inv_eta_reg, rheo_rate;
    int bc_kind[3][2];
    double bc_val[3][2][3];
    double small;  // immersed-boundary emptiness threshold (1e-6, or the FP32 value equivalent to it)
    int freeze_eta;  // 1: η is held fixed (no η_next is computed or written)
    int p_forcing;   // 1: the pressure update and r_P carry the forcing field fP (defect correction)
    int skip_zeros;  // 1: the immersed-boundary updates leave inactive points of the strict interior
                     // (index 2..n in every dimension) unwritten: they hold zero since the last
                     // iteration that wrote them (set by the model, never by a caller)
};

// the scalar parameters converted once to the compute type T (the conversion
// (T)value the reference-shaped kernels perform at each use)
template <typename T>
struct TConst {
    T inv_dx[3], dt_P, dt_tau[6], dt_V[3], g_val[3], bc_val[3][2][3];
    T rheo_A, rheo_inv_eta_reg;
};
template <typename T>
inline TConst<T> make_tconst(const KParams &p) {
    TConst<T> q{};
    for (int d = 0; d < 3; d++) {
        q.inv_dx[d] = T(p.inv_dx[d]);
        q.dt_V[d] = T(p.dt_V[d]);
        q.g_val[d] = T(p.g_val[d]);
        for (int s = 0; s < 2; s++)
            for (int c = 0; c < 3; c++) q.bc_val[d][s][c] = T(p.bc_val[d][s][c]);
    }
    q.dt_P = T(p.dt_P);
    for (int k = 0; k < 6; k++) q.dt_tau[k] = T(p.dt_tau[k]);
    q.rheo_A = T(p.rheo_A);
    q.rheo_inv_eta_reg = T(p.rheo_inv_eta_reg);
    return q;
}

// device pointers of one model state (current buffers)
template <typename T>
struct Ptrs {
    T *P, *txx, *tyy, *tzz, *txy, *txz, *tyz;
    T *Vx, *Vy, *Vz;
    T *eta, *eta_next;
    T *rP, *rVx, *rVy, *rVz;
    const T *gx, *gy, *gz;
    const T *eta_lin, *A;
    const T *fP;  // pressure forcing of the defect-correction problem (p_forcing)
    const T *wna[8];
    const T *wns[8];
    // immersed-boundary activity bits per grid index (IbFlag), precomputed from the
    // volume fractions; nullptr: the kernels evaluate the predicates themselves
    const unsigned char *ibf;
};
// bits of the precomputed immersed-boundary activity byte: update_σ! points
// (isvalid(na) && !isempty(ns)) at ccc, vvc, vcv, cvv and update_V! points
// (isvalid(ns) && !isempty(na)) at vcc, cvc, ccv
enum IbFlag { IBF_S_CCC = 1, IBF_S_VVC = 2, IBF_S_VCV = 4, IBF_S_CVV = 8, IBF_V_VCC = 16, IBF_V_CVC = 32, IBF_V_CCV = 64 };

// one boundary-condition operation on a face (see kernel bc_dim_kernel)
enum BcOp { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_PERIODIC = 2 };
struct BcOpDesc {
    void *f;
    int loc[3];
    int side;
    int op;
    double v;
};
struct BcBatch {
    int count;
    int dim;
    int serial;  // set by launch_bc_batch: one thread applies every op in order
    BcOpDesc ops[kMaxBcOps];
};

// smallest float >= 1e-6: for a float w, (w < t) <=> ((double)w < 1e-6), the
// comparison the reference makes after promoting Float32 masks to Float64
inline float small_threshold_f32() {
    float t = 1e-6f;
    if ((double)t < 1e-6) t = std::nextafter(t, 1.0f);
    return t;
}

void set_error(const std::string &msg);
fi_status cuda_fail(cudaError_t e, const char *where);

// Blocks (32·C x 8 points of one z plane, C points per thread) of the
// immersed-boundary launch that must run once the inactive strict interior
// holds zero: those with a point outside the strict interior or next to an
// active one.  Entry: x = block x | block y << 16, y = block z.
struct BlockList {
    const uint2 *ids;
    int count;
};

// one model of a batched immersed-boundary launch: geometry, parameters and the field
// pointers for both roles of its η buffers (f[0]: as when the batch table was built)
template <typename T>
struct IbMember {
    Geom g;
    KParams p;
    Ptrs<T> f[2];
};
// one model's boundary batch of one dimension, for a batched boundary launch
struct BcMember {
    Geom g;
    BcBatch b;
};

// ---- launchers implemented in fi_reference.cu ----
// bl: run only the listed blocks (immersed boundary with KParams::skip_zeros);
// nullptr: the whole vertex-range grid
template <typename T>
cudaError_t launch_update_sigma(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s,
                                const BlockList *bl = nullptr);
template <typename T>
cudaError_t launch_update_V(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s,
                            const BlockList *bl = nullptr);
// the block list of an immersed-boundary model of precision T from its activity
// bytes; *count is device memory, the list unordered
template <typename T>
cudaError_t launch_ib_blocks(const Geom &g, const unsigned char *flags, uint2 *list, int *count, cudaStream_t s);
// number of blocks of the vertex-range grid (the list's capacity)
long long vertex_grid_blocks(const Geom &g);
template <typename T>
cudaError_t launch_compute_residuals(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s);
template <typename T>
cudaError_t launch_compute_tau(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, cudaStream_t s);
// the activity byte of every vertex-range index from the model's volume fractions
template <typename T>
cudaError_t launch_ib_flags(const Geom &g, const KParams &p, const Ptrs<T> &f, unsigned char *flags, cudaStream_t s);
template <typename T>
cudaError_t launch_bc_batch(const Geom &g, const BcBatch &b, cudaStream_t s);
template <typename T>
cudaError_t launch_residual_norms(const Geom &g, const KParams &p, const Ptrs<T> &f, bool ib, double *partials,
                                  int nblocks, double *out_dev, cudaStream_t s);
int norm_blocks(const Geom &g);
// batched immersed-boundary update_σ! (velocity false) or update_V! (true) over work
// items (member, block x | block y << 16, block z, 0)
template <typename T>
cudaError_t launch_ib_batched(const IbMember<T> *members, const uint4 *items, int nitems, int epar, bool velocity,
                              cudaStream_t s);
// batched boundary batches of one dimension; max_a / max_c: the largest face extents
// (storage sizes of the two other dimensions) over the members
template <typename T>
cudaError_t launch_bc_batched(const BcMember *list, int count, int max_a, int max_c, cudaStream_t s);
// work items of member q: its whole block grid (full) or its block list
cudaError_t launch_ib_items(const Geom &g, bool full, const uint2 *list, int count, unsigned q, uint4 *out, bool f32,
                            cudaStream_t s);
long long ib_grid_blocks(const Geom &g, bool f32);
void bc_set_serial(const Geom &g, BcBatch &b);

// ---- fused 3D sweep (fi_fused3d.cu) ----
// P,tau,V read from `in`, written to `out`; eta read from in.eta, eta_next written.
template <typename T>
bool fused3d_supported(const Geom &g, const KParams &p, bool ib);
// maps18: the eleven full-box input tensor maps (P, txx, tyy, tzz, txy, txz, tyz, Vx,
// Vy, Vz, eta) then the trimmed-box maps of the seven stresses, 128 bytes each,
// encoded with fused3d_encode_map for the variant
// part_dim -1: every tile; 0 / 1: the tiles of the split faces along x / y (part 0)
// or every other tile (part 1) -- the two halves of an iteration whose halo
// exchange overlaps the second half
template <typename T>
cudaError_t launch_fused3d(const Geom &g, const KParams &p, const Ptrs<T> &in, const Ptrs<T> &out, const void *maps18,
                           int variant, int *err, cudaStream_t s, int part_dim = -1, int part = 0);
// field: index in the map order above (0..10); trimmed: the interior box of a stress
bool fused3d_encode_map(void *raw_base, const Geom &g, int esz, int variant, int field, bool trimmed, void *map_out);
// generic tiled tensor map (fi_fused3d.cu): nd dims, strides of dims 1..nd-1 in bytes
bool tma_encode(void *raw_base, int nd, const unsigned long long *dims, const unsigned long long *strides,
                const unsigned *box, int esz, void *map_out);
int fused3d_num_variants();
// launch shapes with the same key read through the same tensor maps
int fused3d_variant_key(int v);
// whether launch shape v fits a CTA in precision esz (8 or 4 bytes)
bool fused3d_variant_fits(int v, int esz);
const char *fused3d_variant_name(int v);

// ---- mixed-precision solve helpers (fi_mixed.cu) ----
template <typename S, typename D>
cudaError_t launch_convert(const S *src, D *dst, long long n, double scale, cudaStream_t s);
template <typename D, typename S>
cudaError_t launch_accumulate(D *x, const S *d, long long n, cudaStream_t s);
template <typename S, typename D>
cudaError_t launch_diff(const S *a, const S *b, D *out, long long n, cudaStream_t s);
// FP64 volume fractions to FP32 keeping every emptiness test w < 1e-6 unchanged
cudaError_t launch_mask_to_f32(const double *src, float *dst, long long n, float thr32, cudaStream_t s);
template <typename T>
cudaError_t launch_eta_from_tau(const Geom &g, const KParams &p, const Ptrs<T> &f, cudaStream_t s);
// max |value| over up to 8 FP32 arrays of n elements each, as float bits in *out_bits
cudaError_t launch_absmax_f32(const float *const *fields, int count, long long n, unsigned *out_bits, cudaStream_t s);

// ---- level sets (fi_levelsets.cu) ----
cudaError_t launch_volfrac3d(const Geom &g, const double dx[3], const double *psi, double *const w[8], cudaStream_t s);
cudaError_t launch_volfrac2d(const Geom &g, const double dx[2], const double *psi, double *const w[4], cudaStream_t s);
cudaError_t launch_convert_f64_f32(const double *src, float *dst, long long n, cudaStream_t s);
cudaError_t launch_levelset(const Geom &g3, const double o3[3], const double dx3[3], const int n2[2],
                            const double o2[2], const double dx2[2], long long dem_pitch, const double *dem,
                            const double *R, int has_R, double cutoff, int invert, double *psi, cudaStream_t s);

}  // namespace fi
