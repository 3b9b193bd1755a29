// fi_halo.cu -- halo layers of a subdomain model for a domain split into slabs
// along x or y (the reference's distributed architecture: Chmy.Distributed's
// exchange_halo! of V and η_next after update_V!, Isothermal.jl:103-104).
//
// A slab is an ordinary model (fused sweep) of its own cells whose split dimension
// is declared periodic.  The sweep then treats the faces of that dimension as "ghost values
// come from elsewhere": they recompute the stresses of the ghost layer from the
// ghost velocities (no stress exchange is needed), and they write ghost images of
// their own interior, which the exchange replaces with the neighbours' values.
//
// Layers (index along the split dimension d, n = cells of the slab in d):
//   sent to the low neighbour  : Center-located fields index 1; fields Vertex-located
//                                in d (V_d, the shear stresses with a d component)
//                                nodes 1 and 2
//   sent to the high neighbour : index n (Center and Vertex alike)
//   received from the low      : written at index 0
//   received from the high     : Center index n+1; Vertex nodes n+1 and n+2
// Node n+1 of a slab is node 1 of its high neighbour; after the exchange both hold
// the neighbour-computed value, exactly as the undivided domain would.
//
// A layer is the whole storage plane of the other dimensions (ghosts included),
// so corner ghosts follow the neighbours' images too.  FI_HALO_ITERATION moves V
// and η (the per-iteration exchange); FI_HALO_STATE adds P and τ (once, after the
// initial state is set, so that the ghost stresses start equal to the neighbour's).
#include <algorithm>

#include "fi_model.h"

#define FI_CHECK_CUDA(expr, where)                          \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, where); \
    } while (0)

namespace fi {
namespace {

// Vertex-located in dimension d?
bool vertex_in(int field, int d) {
    switch (field) {
        case FI_FIELD_TXY: return d == 0 || d == 1;
        case FI_FIELD_TXZ: return d == 0 || d == 2;
        case FI_FIELD_TYZ: return d == 1 || d == 2;
        case FI_FIELD_VX: return d == 0;
        case FI_FIELD_VY: return d == 1;
        case FI_FIELD_VZ: return d == 2;
        default: return false;
    }
}

// fields of a halo message of an nd-dimensional model, in message order
int halo_fields_nd(int nd, int what, int *out) {
    static const int order[] = {FI_FIELD_P,   FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TZZ, FI_FIELD_TXY, FI_FIELD_TXZ,
                                FI_FIELD_TYZ, FI_FIELD_VX,  FI_FIELD_VY,  FI_FIELD_VZ,  FI_FIELD_ETA};
    int n = 0;
    for (int f : order) {
        const bool state_only = f <= FI_FIELD_TYZ;
        if (state_only && what != FI_HALO_STATE) continue;
        const bool only_3d = f == FI_FIELD_TZZ || f == FI_FIELD_TXZ || f == FI_FIELD_TYZ || f == FI_FIELD_VZ;
        if (only_3d && nd != 3) continue;
        out[n++] = f;
    }
    return n;
}
int halo_fields(const fi_model *m, int what, int *out) { return halo_fields_nd(m->d.grid.nd, what, out); }

// layer indices along d (n cells of the slab along d): pack toward `side`
// (0 = low neighbour) or unpack from it
int layers_n(int n, int field, int d, int side, bool pack, int *idx) {
    const bool v = vertex_in(field, d);
    if (pack) {
        if (side == 0) {
            idx[0] = 1;
            if (v) idx[1] = 2;
            return v ? 2 : 1;
        }
        idx[0] = n;
        return 1;
    }
    if (side == 0) {
        idx[0] = 0;
        return 1;
    }
    idx[0] = n + 1;
    if (v) idx[1] = n + 2;
    return v ? 2 : 1;
}
int layers(const fi_model *m, int field, int d, int side, bool pack, int *idx) {
    return layers_n(m->d.grid.n[d], field, d, side, pack, idx);
}

// elements of one layer: the storage plane of the other dimensions
long long layer_elems(const fi_model *m, int d) {
    const long long e0 = m->d.grid.n[0] + 3, e1 = m->d.grid.n[1] + 3;
    const long long e2 = m->d.grid.nd == 3 ? m->d.grid.n[2] + 3 : 1;
    return d == 0 ? e1 * e2 : e0 * e2;
}

// the layers of one message: field base and index along d, in message order
// (at most 11 fields, three of them with two layers)
constexpr int kMaxLayers = 16;
struct LayerSet {
    void *field[kMaxLayers];
    int at[kMaxLayers];
};

template <typename T>
__global__ void layers_copy_kernel(LayerSet ls, T *buf, int d, long long pitch, long long rows, int e_other0,
                                   long long planes, bool pack) {
    // layer blockIdx.y of the message: its index ls.at along dimension d; (a, k) run
    // over the other two dims, and the layer's slice of the buffer follows the earlier ones
    const long long total = (long long)e_other0 * planes;
    T *field = (T *)ls.field[blockIdx.y];
    const long long at = ls.at[blockIdx.y];
    T *b = buf + total * blockIdx.y;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long a = t % e_other0, k = t / e_other0;
        const long long I = d == 0 ? at + pitch * (a + rows * k) : a + pitch * (at + rows * k);
        if (pack) b[t] = field[I];
        else field[I] = b[t];
    }
}

// one launch per message: every layer of every field of it
template <typename T>
fi_status halo_move(fi_model *m, int d, int side, int what, void *buf, bool pack) {
    int fl[16];
    const int nf = halo_fields(m, what, fl);
    const long long le = layer_elems(m, d);
    const int e_other0 = d == 0 ? m->d.grid.n[1] + 3 : m->d.grid.n[0] + 3;
    const long long planes = m->d.grid.nd == 3 ? m->d.grid.n[2] + 3 : 1;
    LayerSet ls{};
    int nl_total = 0;
    for (int q = 0; q < nf; q++) {
        int idx[2];
        const int nl = layers(m, fl[q], d, side, pack, idx);
        for (int l = 0; l < nl; l++) {
            if (nl_total == kMaxLayers) return set_error("halo message with too many layers"), FI_ERR_UNSUPPORTED;
            ls.field[nl_total] = m->cur(fl[q]);
            ls.at[nl_total++] = idx[l];
        }
    }
    const int blocks = (int)std::min<long long>((le + 255) / 256, 4096);
    layers_copy_kernel<T><<<dim3(blocks, nl_total), 256, 0, m->stream>>>(ls, (T *)buf, d, m->g.pitch, m->g.rows,
                                                                        e_other0, planes, pack);
    FI_CHECK_CUDA(cudaGetLastError(), pack ? "halo pack" : "halo unpack");
    return FI_OK;
}

// side_moves: the side itself must take part in the exchange (pack / unpack); the
// byte count of a message only needs the dimension to be split (a periodic or halo side)
fi_status halo_check(const fi_model *m, int32_t dim, int32_t side, int32_t what, bool side_moves = true) {
    if (!m) return set_error("null model"), FI_ERR_ARG;
    if (dim < 0 || dim > 1 || dim >= m->d.grid.nd) return set_error("halo dimension must be x (0) or y (1)"), FI_ERR_ARG;
    if (side != 0 && side != 1) return set_error("side must be 0 (low) or 1 (high)"), FI_ERR_ARG;
    if (what != FI_HALO_ITERATION && what != FI_HALO_STATE) return set_error("unknown halo content"), FI_ERR_ARG;
    auto away = [](int k) { return k == FI_BC_PERIODIC || k == FI_BC_HALO; };
    if (side_moves ? !away(m->d.bc[dim][side].kind) : !(away(m->d.bc[dim][0].kind) || away(m->d.bc[dim][1].kind)))
        return set_error("the side of a split dimension must be periodic or a halo side on the subdomain model"),
               FI_ERR_STATE;
    if (m->ib) return set_error("halo exchange of the immersed-boundary model is not covered"), FI_ERR_UNSUPPORTED;
    // the reference-shaped path fills ghost stresses by the boundary copy after
    // update_σ!, so a split would need a second (stress) exchange inside the
    // iteration; the fused sweep recomputes them from the exchanged velocities
    if (m->path != FI_PATH_FUSED)
        return set_error("halo exchange needs the fused sweep (ghost stresses recomputed from the exchanged velocities)"),
               FI_ERR_UNSUPPORTED;
    return FI_OK;
}

}  // namespace
}  // namespace fi

using namespace fi;

extern "C" {

fi_status fi_model_halo_bytes(const fi_model *m, int32_t dim, int32_t side, int32_t what, size_t *bytes) {
    fi_status st = halo_check(m, dim, side, what, false);
    if (st != FI_OK) return st;
    if (!bytes) return set_error("null argument"), FI_ERR_ARG;
    int fl[16];
    const int nf = halo_fields(m, what, fl);
    size_t layers_total = 0;
    for (int q = 0; q < nf; q++) {
        int idx[2];
        layers_total += (size_t)layers(m, fl[q], dim, side, true, idx);
    }
    *bytes = layers_total * (size_t)layer_elems(m, dim) * m->esz;
    return FI_OK;
}

fi_status fi_halo_plan(int32_t nd, const int32_t *n, int32_t dim, int32_t side, int32_t what, int32_t pack,
                       int32_t *fields, int32_t *layer_index, int32_t cap, int32_t *count) {
    if (!n || !count || (nd != 2 && nd != 3) || dim < 0 || dim > 1 || (side != 0 && side != 1) ||
        (what != FI_HALO_ITERATION && what != FI_HALO_STATE) || cap < 0 || (cap > 0 && (!fields || !layer_index)))
        return set_error("bad argument"), FI_ERR_ARG;
    int fl[16];
    const int nf = halo_fields_nd(nd, what, fl);
    int k = 0;
    for (int q = 0; q < nf; q++) {
        int idx[2];
        const int nl = layers_n(n[dim], fl[q], dim, side, pack != 0, idx);
        for (int l = 0; l < nl; l++, k++) {
            if (k < cap) {
                fields[k] = fl[q];
                layer_index[k] = idx[l];
            }
        }
    }
    *count = k;
    if (k > cap && cap > 0) return set_error("plan longer than the arrays given"), FI_ERR_ARG;
    return FI_OK;
}

fi_status fi_model_halo_pack(fi_model *m, int32_t dim, int32_t side, int32_t what, void *dst_dev) {
    fi_status st = halo_check(m, dim, side, what);
    if (st != FI_OK) return st;
    if (!dst_dev) return set_error("null buffer"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    return m->is_f64() ? halo_move<double>(m, dim, side, what, dst_dev, true)
                       : halo_move<float>(m, dim, side, what, dst_dev, true);
}

fi_status fi_model_halo_unpack(fi_model *m, int32_t dim, int32_t side, int32_t what, const void *src_dev) {
    fi_status st = halo_check(m, dim, side, what);
    if (st != FI_OK) return st;
    if (!src_dev) return set_error("null buffer"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    return m->is_f64() ? halo_move<double>(m, dim, side, what, const_cast<void *>(src_dev), false)
                       : halo_move<float>(m, dim, side, what, const_cast<void *>(src_dev), false);
}

}  // extern "C"
