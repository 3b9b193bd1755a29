// fi_api.cu -- C ABI of libfastice_b200: model lifecycle, field I/O, boundary
// batches, the PT iteration driver and the solve loop.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <algorithm>
#include <vector>

#include "fi_model.h"

namespace fi {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

fi_status cuda_fail(cudaError_t e, const char *where) {
    set_error(std::string(where) + ": " + cudaGetErrorString(e));
    return FI_ERR_CUDA;
}

}  // namespace fi

using namespace fi;

#define FI_CHECK_CUDA(expr, where)                 \
    do {                                           \
        cudaError_t e_ = (expr);                   \
        if (e_ != cudaSuccess) return cuda_fail(e_, where); \
    } while (0)

namespace {

// staggered location of each field (0 = Center, 1 = Vertex) per dim
void field_loc(int field, int loc[3]) {
    static const int L[FI_FIELD_COUNT][3] = {
        {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1},  // P, tau
        {1, 0, 0}, {0, 1, 0}, {0, 0, 1},                                            // V
        {0, 0, 0}, {0, 0, 0},                                                       // eta, eta_next
        {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},                                 // residuals
        {1, 0, 0}, {0, 1, 0}, {0, 0, 1},                                            // gravity
        {0, 0, 0}, {0, 0, 0},                                                       // eta_lin, A
        {0, 0, 0}, {1, 1, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1},  // na
        {0, 0, 0}, {1, 1, 1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1},  // ns
    };
    for (int d = 0; d < 3; d++) loc[d] = L[field][d];
}

// field buffers: the field pointer sits kXOff elements past the allocation
cudaError_t field_alloc(void **field_ptr, size_t elems, size_t esz) {
    void *raw = nullptr;
    cudaError_t e = cudaMalloc(&raw, (elems + 64) * esz);
    if (e != cudaSuccess) {
        *field_ptr = nullptr;
        return e;
    }
    *field_ptr = (char *)raw + kXOff * esz;
    return cudaSuccess;
}
void *field_raw(void *field_ptr, size_t esz) { return field_ptr ? (char *)field_ptr - kXOff * esz : nullptr; }
void field_free(void *field_ptr, size_t esz) {
    if (field_ptr) cudaFree(field_raw(field_ptr, esz));
}

}  // namespace

namespace {

fi_status validate(const fi_model_desc *d) {
    if (!d) return set_error("null descriptor"), FI_ERR_ARG;
    const fi_grid &gr = d->grid;
    if (gr.nd != 2 && gr.nd != 3) return set_error("grid.nd must be 2 or 3"), FI_ERR_ARG;
    for (int k = 0; k < gr.nd; k++) {
        if (gr.n[k] < 3) return set_error("grid.n must be >= 3 in every dimension"), FI_ERR_ARG;
        if (!(gr.extent[k] > 0.0)) return set_error("grid.extent must be positive"), FI_ERR_ARG;
    }
    if (d->dtype != FI_F64 && d->dtype != FI_F32) return set_error("dtype must be FI_F64 or FI_F32"), FI_ERR_ARG;
    if (d->immersed && gr.nd != 3)
        return set_error("the immersed-boundary model is 3D only (the reference 2D IB kernels are broken)"),
               FI_ERR_UNSUPPORTED;
    for (int k = 0; k < gr.nd; k++) {
        bool p0 = d->bc[k][0].kind == FI_BC_PERIODIC, p1 = d->bc[k][1].kind == FI_BC_PERIODIC;
        if (p0 != p1) return set_error("a periodic dimension must be periodic on both sides"), FI_ERR_ARG;
        for (int s = 0; s < 2; s++) {
            if (d->bc[k][s].kind < 0 || d->bc[k][s].kind > FI_BC_HALO)
                return set_error("unknown boundary-condition kind"), FI_ERR_ARG;
            if (d->bc[k][s].kind == FI_BC_HALO && (k > 1 || gr.nd != 3 || d->immersed))
                return set_error("halo sides are supported along x or y of 3D FullStokes subdomains"),
                       FI_ERR_UNSUPPORTED;
        }
    }
    const fi_rheology &r = d->rheology;
    if (r.inner != FI_RHEO_LINEAR && r.inner != FI_RHEO_POWER) return set_error("unknown rheology"), FI_ERR_ARG;
    if (r.has_reg && !(r.eta_reg > 0.0)) return set_error("eta_reg must be positive"), FI_ERR_ARG;
    if (r.relax < FI_RELAX_NONE || r.relax > FI_RELAX_LOG10) return set_error("unknown relaxation"), FI_ERR_ARG;
    if (d->path < FI_PATH_AUTO || d->path > FI_PATH_FUSED) return set_error("unknown path"), FI_ERR_ARG;
    return FI_OK;
}

bool field_used(const fi_model *m, int f) {
    const fi_model_desc &d = m->d;
    bool three = d.grid.nd == 3;
    switch (f) {
        case FI_FIELD_TZZ: case FI_FIELD_TXZ: case FI_FIELD_TYZ: case FI_FIELD_VZ: case FI_FIELD_RVZ:
            return three;
        case FI_FIELD_GX: return d.gravity.kind[0] == FI_G_FIELD;
        case FI_FIELD_GY: return d.gravity.kind[1] == FI_G_FIELD;
        case FI_FIELD_GZ: return three && d.gravity.kind[2] == FI_G_FIELD;
        case FI_FIELD_ETA_LIN: return d.rheology.inner == FI_RHEO_LINEAR && d.rheology.eta_is_field;
        case FI_FIELD_A: return d.rheology.inner == FI_RHEO_POWER && d.rheology.A_is_field;
        default:
            if (f >= FI_FIELD_NA_CCC) return d.immersed != 0;
            return true;
    }
}

bool is_residual(int f) { return f >= FI_FIELD_RP && f <= FI_FIELD_RVZ; }

fi_status ensure_residual_arrays(fi_model *m) {
    for (int f = FI_FIELD_RP; f <= FI_FIELD_RVZ; f++) {
        if (!field_used(m, f) || m->base[f]) continue;
        void *p = nullptr;
        cudaError_t e = field_alloc(&p, m->elems, m->esz);
        if (e != cudaSuccess) return set_error("residual field allocation failed"), FI_ERR_OOM;
        FI_CHECK_CUDA(cudaMemsetAsync(field_raw(p, m->esz), 0, (m->elems + 64) * m->esz, m->stream), "memset");
        m->base[f] = p;
    }
    return FI_OK;
}

size_t interior_count(const fi_model *m, int field) {
    int loc[3];
    field_loc(field, loc);
    size_t c = 1;
    for (int k = 0; k < m->d.grid.nd; k++) c *= (size_t)(m->d.grid.n[k] + loc[k]);
    return c;
}

cudaMemcpy3DParms copy_params(const fi_model *m, int field, void *dev, void *host, bool to_dev) {
    int loc[3];
    field_loc(field, loc);
    const int nd = m->d.grid.nd;
    size_t nx = m->d.grid.n[0] + loc[0], ny = m->d.grid.n[1] + loc[1], nz = nd == 3 ? m->d.grid.n[2] + loc[2] : 1;
    cudaMemcpy3DParms p{};
    cudaPitchedPtr hp = make_cudaPitchedPtr(host, nx * m->esz, nx, ny);
    cudaPitchedPtr dp =
        make_cudaPitchedPtr(field_raw(dev, m->esz), (size_t)m->g.pitch * m->esz, (size_t)m->g.pitch, (size_t)m->g.rows);
    cudaPos dpos = make_cudaPos((size_t)(kXOff + 1) * m->esz, 1, nd == 3 ? 1 : 0);
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
    p.extent = make_cudaExtent(nx * m->esz, ny, nz);
    return p;
}

// Host interior -> device halo box.  A pitched 3D copy from host memory runs at
// about half the linear copy rate (rows of a few KB), so the interior goes over
// as linear copies of whole z planes into a staging buffer (at most 64 MB, at
// least one plane, never more than the field), each followed by a kernel that
// writes the rows into the box; both are issued on the model's stream, so one
// buffer suffices.
template <typename E>
__global__ void __launch_bounds__(256) scatter_rows(const E *__restrict__ src, E *__restrict__ dst, int nx, int ny,
                                                    long long pitch, long long rows) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nx) return;
    const long long z = blockIdx.y;
    // rows split over grid.z: a 2D field (one plane) still spreads over many blocks
    for (int y = blockIdx.z; y < ny; y += gridDim.z)
        dst[x + pitch * (y + rows * z)] = src[x + (long long)nx * (y + (long long)ny * z)];
}

fi_status upload_interior(fi_model *m, int field, const void *host) {
    int loc[3];
    field_loc(field, loc);
    const int nd = m->d.grid.nd;
    const int nx = m->d.grid.n[0] + loc[0], ny = m->d.grid.n[1] + loc[1], nz = nd == 3 ? m->d.grid.n[2] + loc[2] : 1;
    const size_t plane = (size_t)nx * ny * m->esz;
    const size_t want = std::max(plane, std::min((size_t)64 << 20, plane * nz));
    if (m->stage_bytes < want) {
        if (m->d_stage) cudaFree(m->d_stage);
        m->d_stage = nullptr, m->stage_bytes = 0;
        if (cudaMalloc(&m->d_stage, want) != cudaSuccess) return cuda_fail(cudaGetLastError(), "staging buffer");
        m->stage_bytes = want;
    }
    const int per = (int)std::min<size_t>(65535, std::max<size_t>(1, m->stage_bytes / plane));  // grid.y limit
    char *dev = (char *)m->cur(field) + (1 + m->g.pitch * (1 + m->g.rows * (nd == 3 ? 1 : 0))) * (long long)m->esz;
    const char *src = (const char *)host;
    for (int z0 = 0; z0 < nz; z0 += per) {
        const int zc = std::min(per, nz - z0);
        FI_CHECK_CUDA(cudaMemcpyAsync(m->d_stage, src + plane * z0, plane * zc, cudaMemcpyHostToDevice, m->stream),
                      "set_field copy");
        char *d = dev + (long long)z0 * m->g.sxy * (long long)m->esz;
        const dim3 grd((nx + 255) / 256, zc, std::max(1, std::min(ny, std::max(1, 4096 / zc))));
        if (m->esz == 8)
            scatter_rows<unsigned long long><<<grd, 256, 0, m->stream>>>(
                (const unsigned long long *)m->d_stage, (unsigned long long *)d, nx, ny, m->g.pitch, m->g.rows);
        else
            scatter_rows<unsigned int><<<grd, 256, 0, m->stream>>>((const unsigned int *)m->d_stage, (unsigned int *)d,
                                                                   nx, ny, m->g.pitch, m->g.rows);
        FI_CHECK_CUDA(cudaGetLastError(), "set_field rows");
    }
    return FI_OK;
}

// ---- boundary-condition batches (boundary_conditions.jl) -------------------
void add_op(BcBatch &b, void *f, int field, int side, int op, double v) {
    BcOpDesc &o = b.ops[b.count++];
    o.f = f;
    field_loc(field, o.loc);
    o.side = side;
    o.op = op;
    o.v = v;
}

// stress batch for dim d (boundary_conditions.jl:26-100, :117)
BcBatch stress_batch(const fi_model *m, int d) {
    BcBatch b{};
    b.dim = d;
    const int nd = m->d.grid.nd;
    for (int s = 0; s < 2; s++) {
        const fi_bc &bc = m->d.bc[d][s];
        if (bc.kind == FI_BC_HALO) continue;  // the neighbour's values arrive by the halo exchange
        if (bc.kind == FI_BC_PERIODIC) {
            if (s == 1) continue;
            int fl3[] = {FI_FIELD_P, FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TZZ, FI_FIELD_TXY, FI_FIELD_TXZ, FI_FIELD_TYZ};
            int fl2[] = {FI_FIELD_P, FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TXY};
            if (nd == 3)
                for (int f : fl3) add_op(b, m->cur(f), f, 0, BC_PERIODIC, 0);
            else
                for (int f : fl2) add_op(b, m->cur(f), f, 0, BC_PERIODIC, 0);
            continue;
        }
        if (bc.kind == FI_BC_VELOCITY) continue;
        const double *c = bc.c;
        if (nd == 2) {
            if (bc.kind == FI_BC_TRACTION) {
                if (d == 0) {
                    add_op(b, m->cur(FI_FIELD_P), FI_FIELD_P, s, BC_DIRICHLET, c[0]);
                    add_op(b, m->cur(FI_FIELD_TXX), FI_FIELD_TXX, s, BC_DIRICHLET, c[0]);
                    add_op(b, m->cur(FI_FIELD_TXY), FI_FIELD_TXY, s, BC_DIRICHLET, c[1]);
                } else {
                    add_op(b, m->cur(FI_FIELD_P), FI_FIELD_P, s, BC_DIRICHLET, c[1]);
                    add_op(b, m->cur(FI_FIELD_TYY), FI_FIELD_TYY, s, BC_DIRICHLET, c[1]);
                    add_op(b, m->cur(FI_FIELD_TXY), FI_FIELD_TXY, s, BC_DIRICHLET, c[0]);
                }
            } else {
                add_op(b, m->cur(FI_FIELD_TXY), FI_FIELD_TXY, s, BC_DIRICHLET, c[1 - d]);
            }
            continue;
        }
        static const int tang[3][2] = {{1, 2}, {0, 2}, {0, 1}};
        static const int shear[3][2] = {{FI_FIELD_TXY, FI_FIELD_TXZ}, {FI_FIELD_TXY, FI_FIELD_TYZ}, {FI_FIELD_TXZ, FI_FIELD_TYZ}};
        static const int diag[3] = {FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TZZ};
        if (bc.kind == FI_BC_TRACTION) {
            add_op(b, m->cur(FI_FIELD_P), FI_FIELD_P, s, BC_DIRICHLET, c[d]);
            add_op(b, m->cur(diag[d]), diag[d], s, BC_DIRICHLET, c[d]);
        }
        add_op(b, m->cur(shear[d][0]), shear[d][0], s, BC_DIRICHLET, c[tang[d][0]]);
        add_op(b, m->cur(shear[d][1]), shear[d][1], s, BC_DIRICHLET, c[tang[d][1]]);
    }
    return b;
}

// velocity batch + eta_next Neumann for dim d (boundary_conditions.jl:104-115, Isothermal.jl:103-104)
BcBatch velocity_batch(const fi_model *m, int d) {
    BcBatch b{};
    b.dim = d;
    const int nd = m->d.grid.nd;
    const int Vf[3] = {FI_FIELD_VX, FI_FIELD_VY, FI_FIELD_VZ};
    for (int s = 0; s < 2; s++) {
        const fi_bc &bc = m->d.bc[d][s];
        if (bc.kind == FI_BC_HALO) continue;
        if (bc.kind == FI_BC_PERIODIC) {
            if (s == 1) continue;
            for (int q = 0; q < nd; q++) add_op(b, m->cur(Vf[q]), Vf[q], 0, BC_PERIODIC, 0);
            add_op(b, m->cur(FI_FIELD_ETA_NEXT), FI_FIELD_ETA_NEXT, 0, BC_PERIODIC, 0);
            continue;
        }
        if (bc.kind == FI_BC_VELOCITY) {
            for (int q = 0; q < nd; q++) add_op(b, m->cur(Vf[q]), Vf[q], s, BC_DIRICHLET, bc.c[q]);
        } else if (bc.kind == FI_BC_SLIP) {
            add_op(b, m->cur(Vf[d]), Vf[d], s, BC_DIRICHLET, bc.c[d]);
        }
        add_op(b, m->cur(FI_FIELD_ETA_NEXT), FI_FIELD_ETA_NEXT, s, BC_NEUMANN, 0);
    }
    return b;
}

BcBatch eta_batch(const fi_model *m, int d, int field) {
    BcBatch b{};
    b.dim = d;
    for (int s = 0; s < 2; s++) {
        const fi_bc &bc = m->d.bc[d][s];
        if (bc.kind == FI_BC_HALO) continue;
        if (bc.kind == FI_BC_PERIODIC) {
            if (s == 0) add_op(b, m->cur(field), field, 0, BC_PERIODIC, 0);
        } else {
            add_op(b, m->cur(field), field, s, BC_NEUMANN, 0);
        }
    }
    return b;
}

BcBatch residual_batch(const fi_model *m, int d) {
    BcBatch b{};
    b.dim = d;
    const int Rf[3] = {FI_FIELD_RVX, FI_FIELD_RVY, FI_FIELD_RVZ};
    for (int s = 0; s < 2; s++) {
        int k = m->d.bc[d][s].kind;
        if (k == FI_BC_TRACTION || k == FI_BC_PERIODIC || k == FI_BC_HALO) continue;
        add_op(b, m->base[Rf[d]], Rf[d], s, BC_DIRICHLET, 0.0);
    }
    return b;
}

template <typename T>
fi_status run_batch(fi_model *m, BcBatch (*mk)(const fi_model *, int)) {
    for (int d = 0; d < m->d.grid.nd; d++) {
        BcBatch b = mk(m, d);
        FI_CHECK_CUDA(launch_bc_batch<T>(m->g, b, m->stream), "boundary batch");
    }
    return FI_OK;
}

template <typename T>
fi_status run_eta_batch(fi_model *m, int field) {
    for (int d = 0; d < m->d.grid.nd; d++) {
        BcBatch b = eta_batch(m, d, field);
        FI_CHECK_CUDA(launch_bc_batch<T>(m->g, b, m->stream), "eta boundary batch");
    }
    return FI_OK;
}

// activity bytes of an immersed-boundary model, recomputed after its volume
// fractions changed (set_field, ω_from_ψ!, a device pointer handed out)
template <typename T>
fi_status refresh_ibf(fi_model *m) {
    if (!m->ib || !m->ibf_stale) return FI_OK;
    FI_CHECK_CUDA(launch_ib_flags<T>(m->g, m->kp, m->ptrs<T>(), m->d_ibf, m->stream), "activity bytes");
    // the block list, in z, y, x order (neighbouring blocks run close in time)
    FI_CHECK_CUDA(cudaMemsetAsync(m->d_bcount, 0, sizeof(int), m->stream), "block count");
    FI_CHECK_CUDA(launch_ib_blocks<T>(m->g, m->d_ibf, m->d_blist, m->d_bcount, m->stream), "block list");
    int cnt = 0;
    FI_CHECK_CUDA(cudaMemcpyAsync(&cnt, m->d_bcount, sizeof(int), cudaMemcpyDeviceToHost, m->stream), "block count");
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "block count");
    std::vector<uint2> ids((size_t)cnt);
    if (cnt > 0) {
        FI_CHECK_CUDA(cudaMemcpy(ids.data(), m->d_blist, cnt * sizeof(uint2), cudaMemcpyDeviceToHost), "block list");
        std::sort(ids.begin(), ids.end(), [](const uint2 &a, const uint2 &b) {
            if (a.y != b.y) return a.y < b.y;
            if ((a.x >> 16) != (b.x >> 16)) return (a.x >> 16) < (b.x >> 16);
            return (a.x & 0xffffu) < (b.x & 0xffffu);
        });
        FI_CHECK_CUDA(cudaMemcpy(m->d_blist, ids.data(), cnt * sizeof(uint2), cudaMemcpyHostToDevice), "block list");
    }
    m->n_blist = cnt;
    // captured iteration pairs hold the old list's launch size
    for (cudaGraphExec_t &g : m->pair_graph)
        if (g) cudaGraphExecDestroy(g), g = nullptr;
    m->ibf_stale = false;
    return FI_OK;
}

// one reference-shaped iteration: update_σ!, stress BCs, update_V!, velocity BCs
template <typename T>
fi_status reference_iteration(fi_model *m) {
    Ptrs<T> f = m->ptrs<T>();
    // once zeros hold, only the blocks with an active or a boundary point run
    const BlockList bl{m->d_blist, m->n_blist};
    // (a relaxed viscosity moves towards its target at every point, so it runs all)
    const bool eta_moves = !m->kp.freeze_eta && m->kp.rheo_relax != FI_RELAX_NONE;
    const BlockList *blp = (m->ib && m->kp.skip_zeros && !m->ibf_stale && m->n_blist > 0 && !eta_moves) ? &bl : nullptr;
    FI_CHECK_CUDA(launch_update_sigma<T>(m->g, m->kp, f, m->ib, m->stream, blp), "update_sigma");
    fi_status st = run_batch<T>(m, stress_batch);
    if (st != FI_OK) return st;
    FI_CHECK_CUDA(launch_update_V<T>(m->g, m->kp, f, m->ib, m->stream, blp), "update_V");
    st = run_batch<T>(m, velocity_batch);
    if (st != FI_OK) return st;
    if (!m->kp.freeze_eta) m->eta_swapped = !m->eta_swapped;
    return FI_OK;
}

// The reference-shaped iteration is 2 + 2·nd launches, most of them small
// boundary batches: on small grids their launch cost exceeds their work.  Two
// iterations bring η / η_next back to their roles, so a pair is captured once as a
// CUDA graph (per starting parity of the η buffers, recaptured when the parameters
// change) and replayed for long advances.
template <typename T>
fi_status reference_pairs(fi_model *m, int pairs) {
    const int e = m->eta_swapped ? 1 : 0;
    if (!m->pair_graph[e] || std::memcmp(&m->pair_kp[e], &m->kp, sizeof(KParams)) != 0) {
        if (m->pair_graph[e]) cudaGraphExecDestroy(m->pair_graph[e]);
        m->pair_graph[e] = nullptr;
        const bool sw = m->eta_swapped;
        FI_CHECK_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
        fi_status st = reference_iteration<T>(m);
        if (st == FI_OK) st = reference_iteration<T>(m);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(m->stream, &g);
        m->eta_swapped = sw;  // capturing ran nothing
        if (st != FI_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        FI_CHECK_CUDA(ce, "graph capture");
        const cudaError_t ie = cudaGraphInstantiate(&m->pair_graph[e], g, 0);
        cudaGraphDestroy(g);
        FI_CHECK_CUDA(ie, "graph instantiate");
        m->pair_kp[e] = m->kp;
    }
    for (int q = 0; q < pairs; q++) FI_CHECK_CUDA(cudaGraphLaunch(m->pair_graph[e], m->stream), "graph launch");
    return FI_OK;
}
constexpr int kPairGraphMin = 8;  // advances of at least this many iterations replay the graph

template <typename T>
fi_status advance_t(fi_model *m, int niter) {
    if (fi_status st = refresh_ibf<T>(m); st != FI_OK) return st;
    if (m->ib && m->path != FI_PATH_FUSED) {
        // the first two iterations after the state changed write every point; later
        // ones skip the zeros of the inactive strict interior and the blocks outside
        // the block list
        m->kp.skip_zeros = 0;
        if (!m->state_ptr_out) {
            while (m->full_iters < 2 && niter > 0) {
                if (fi_status st = reference_iteration<T>(m); st != FI_OK) return st;
                m->iterations++;
                niter--;
                m->full_iters++;
            }
            if (m->full_iters >= 2) m->kp.skip_zeros = 1;
        }
    }
    if (m->path != FI_PATH_FUSED && niter >= kPairGraphMin) {
        const int pairs = niter / 2;
        if (fi_status st = reference_pairs<T>(m, pairs); st != FI_OK) return st;
        m->iterations += 2LL * pairs;
        niter -= 2 * pairs;
    }
    for (int it = 0; it < niter; it++) {
        if (m->path == FI_PATH_FUSED) {
            Ptrs<T> in = m->ptrs<T>(false);
            Ptrs<T> out = m->ptrs<T>(true);
            out.eta = in.eta;
            out.eta_next = in.eta_next;
            alignas(64) unsigned char maps[18][128];
            for (int f = 0; f < kState; f++) std::memcpy(maps[f], m->parity ? m->map_alt[f] : m->map_base[f], 128);
            std::memcpy(maps[10], m->map_eta[m->eta_swapped ? 1 : 0], 128);
            for (int f = 0; f < 7; f++) std::memcpy(maps[11 + f], m->parity ? m->tmap_alt[f] : m->tmap_base[f], 128);
            FI_CHECK_CUDA(launch_fused3d<T>(m->g, m->kp, in, out, maps, m->fused_variant, m->d_err, m->stream),
                          "fused sweep");
            m->parity ^= 1;
            if (!m->kp.freeze_eta) m->eta_swapped = !m->eta_swapped;
        } else {
            fi_status st = reference_iteration<T>(m);
            if (st != FI_OK) return st;
        }
        m->iterations++;
    }
    return FI_OK;
}

fi_status check_err_word(fi_model *m) {
    int h = 0;
    FI_CHECK_CUDA(cudaMemcpy(&h, m->d_err, sizeof(int), cudaMemcpyDeviceToHost), "error word");
    if (h != 0) {
        cudaMemset(m->d_err, 0, sizeof(int));
        set_error("a bounded wait in the fused sweep expired; results of that launch are invalid");
        return (fi_status)h;
    }
    return FI_OK;
}

// (re)encode the tensor maps of every buffer the fused sweep reads, for the
// current variant's tile shape: full boxes of the eleven inputs and trimmed boxes
// of the seven stresses, for both state buffers
fi_status encode_maps(fi_model *m) {
    const int v = m->fused_variant, key = fused3d_variant_key(v), esz = (int)m->esz;
    if (key == m->maps_key) return FI_OK;
    for (int f = 0; f < kState; f++) {
        if (!fused3d_encode_map(field_raw(m->base[f], m->esz), m->g, esz, v, f, false, m->map_base[f]) ||
            !fused3d_encode_map(field_raw(m->alt[f], m->esz), m->g, esz, v, f, false, m->map_alt[f]))
            return set_error("cuTensorMapEncodeTiled failed"), FI_ERR_CUDA;
        if (f < 7 && (!fused3d_encode_map(field_raw(m->base[f], m->esz), m->g, esz, v, f, true, m->tmap_base[f]) ||
                      !fused3d_encode_map(field_raw(m->alt[f], m->esz), m->g, esz, v, f, true, m->tmap_alt[f])))
            return set_error("cuTensorMapEncodeTiled failed"), FI_ERR_CUDA;
    }
    if (!fused3d_encode_map(field_raw(m->base[FI_FIELD_ETA], m->esz), m->g, esz, v, 10, false, m->map_eta[0]) ||
        !fused3d_encode_map(field_raw(m->base[FI_FIELD_ETA_NEXT], m->esz), m->g, esz, v, 10, false, m->map_eta[1]))
        return set_error("cuTensorMapEncodeTiled failed"), FI_ERR_CUDA;
    m->maps_key = key;
    return FI_OK;
}

template <typename T>
fi_status norms_t(fi_model *m, double *out) {
    if (fi_status st = refresh_ibf<T>(m); st != FI_OK) return st;
    Ptrs<T> f = m->ptrs<T>();
    FI_CHECK_CUDA(launch_residual_norms<T>(m->g, m->kp, f, m->ib, m->d_partials, m->nblk, m->d_out, m->stream),
                  "residual norms");
    FI_CHECK_CUDA(cudaMemcpyAsync(m->h_out, m->d_out, FI_NORMS_LEN * sizeof(double), cudaMemcpyDeviceToHost, m->stream),
                  "norms copy");
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "norms sync");
    std::memcpy(out, m->h_out, FI_NORMS_LEN * sizeof(double));
    return check_err_word(m);
}

template <typename T>
fi_status apply_bcs_t(fi_model *m) {
    fi_status st = run_batch<T>(m, stress_batch);
    if (st == FI_OK) st = run_batch<T>(m, velocity_batch);
    if (st == FI_OK) st = run_eta_batch<T>(m, FI_FIELD_ETA);
    return st;
}

template <typename T>
fi_status residuals_t(fi_model *m) {
    fi_status st = ensure_residual_arrays(m);
    if (st != FI_OK) return st;
    if ((st = refresh_ibf<T>(m)) != FI_OK) return st;
    Ptrs<T> f = m->ptrs<T>();
    FI_CHECK_CUDA(launch_compute_residuals<T>(m->g, m->kp, f, m->ib, m->stream), "compute_residuals");
    return run_batch<T>(m, residual_batch);
}

bool fused_ok(const fi_model *m) {
    if (m->d.grid.nd != 3) return false;
    return m->is_f64() ? fused3d_supported<double>(m->g, m->kp, m->ib) : fused3d_supported<float>(m->g, m->kp, m->ib);
}

}  // namespace

BcBatch model_stress_batch(const fi_model *m, int d) { return stress_batch(m, d); }
BcBatch model_velocity_batch(const fi_model *m, int d) { return velocity_batch(m, d); }
fi_status model_refresh_ibf(fi_model *m) { return m->is_f64() ? refresh_ibf<double>(m) : refresh_ibf<float>(m); }

// Second state buffer of every state field, for drivers that double-buffer a
// model whose own path updates in place (the batched 2D sweep); a new buffer
// starts as a copy of the current state, ghosts included.
bool model_field_used(const fi_model *m, int f) { return field_used(m, f); }

fi_status model_ensure_second_state(fi_model *m) {
    for (int f = 0; f < kState; f++) {
        if (!field_used(m, f) || m->alt[f]) continue;
        if (field_alloc(&m->alt[f], m->elems, m->esz) != cudaSuccess) {
            cudaGetLastError();
            set_error("device allocation failed (second state buffer)");
            return FI_ERR_OOM;
        }
        void *dst = field_raw(m->parity ? m->base[f] : m->alt[f], m->esz);
        const void *src = field_raw(m->parity ? m->alt[f] : m->base[f], m->esz);
        FI_CHECK_CUDA(cudaMemcpyAsync(dst, src, (m->elems + 64) * m->esz, cudaMemcpyDeviceToDevice, m->stream),
                      "second state buffer");
    }
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "second state buffer");
    return FI_OK;
}

// An overlapped iteration (fi_model_advance_begin / _end) leaves its second half
// on the model's second stream: every other entry point first orders the model's
// stream after it, and refuses to run between the two halves.
// the rheology and PT-step parameters of a model (set at creation and by fi_model_set_params)
static void set_rheology_dtau(KParams &kp, const fi_rheology &r, const fi_pt_params &dt) {
    kp.dt_P = dt.dt_P;
    for (int k = 0; k < 6; k++) kp.dt_tau[k] = dt.dt_tau[k];
    for (int k = 0; k < 3; k++) kp.dt_V[k] = dt.dt_V[k];
    kp.rheo_inner = r.inner;
    kp.rheo_eta_is_field = r.eta_is_field;
    kp.rheo_A_is_field = r.A_is_field;
    kp.rheo_n = r.n;
    kp.rheo_has_reg = r.has_reg;
    kp.rheo_relax = r.relax;
    kp.rheo_eta = r.eta;
    kp.rheo_A = r.A;
    kp.rheo_inv_eta_reg = r.has_reg ? 1.0 / r.eta_reg : 0.0;  // Physics.jl:22 stores one(η_reg)/η_reg
    kp.rheo_rate = r.rate;
}

static fi_status join_overlap(fi_model *m) {
    if (m->split_begun >= 0)
        return set_error("an overlapped iteration is begun: call fi_model_advance_end first"), FI_ERR_STATE;
    if (m->interior_pending) {
        FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
        FI_CHECK_CUDA(cudaStreamWaitEvent(m->stream, m->ev_int, 0), "join the second half");
        m->interior_pending = false;
    }
    return FI_OK;
}

namespace {
// the two halves of an overlapped fused iteration
template <typename T>
fi_status advance_half(fi_model *m, int dim, int part) {
    if (part == 0) {
        Ptrs<T> in = m->ptrs<T>(false);
        Ptrs<T> out = m->ptrs<T>(true);
        out.eta = in.eta;
        out.eta_next = in.eta_next;
        for (int f = 0; f < kState; f++) std::memcpy(m->pend_maps[f], m->parity ? m->map_alt[f] : m->map_base[f], 128);
        std::memcpy(m->pend_maps[10], m->map_eta[m->eta_swapped ? 1 : 0], 128);
        for (int f = 0; f < 7; f++)
            std::memcpy(m->pend_maps[11 + f], m->parity ? m->tmap_alt[f] : m->tmap_base[f], 128);
        static_assert(sizeof(Ptrs<T>) <= sizeof(m->pend_ptrs[0]), "pending pointers fit");
        std::memcpy(m->pend_ptrs[0], &in, sizeof(in));
        std::memcpy(m->pend_ptrs[1], &out, sizeof(out));
        FI_CHECK_CUDA(launch_fused3d<T>(m->g, m->kp, in, out, m->pend_maps, m->fused_variant, m->d_err, m->stream, dim, 0),
                      "fused sweep (split faces)");
        FI_CHECK_CUDA(cudaEventRecord(m->ev_bnd, m->stream), "event");
        m->parity ^= 1;
        if (!m->kp.freeze_eta) m->eta_swapped = !m->eta_swapped;
        return FI_OK;
    }
    Ptrs<T> in, out;
    std::memcpy(&in, m->pend_ptrs[0], sizeof(in));
    std::memcpy(&out, m->pend_ptrs[1], sizeof(out));
    FI_CHECK_CUDA(cudaStreamWaitEvent(m->stream2, m->ev_bnd, 0), "wait first half");
    FI_CHECK_CUDA(launch_fused3d<T>(m->g, m->kp, in, out, m->pend_maps, m->fused_variant, m->d_err, m->stream2, dim, 1),
                  "fused sweep (interior)");
    FI_CHECK_CUDA(cudaEventRecord(m->ev_int, m->stream2), "event");
    return FI_OK;
}
}  // namespace

extern "C" {

const char *fi_last_error(void) { return g_last_error.c_str(); }
int fi_abi_version(void) { return FI_ABI_VERSION; }

fi_status fi_model_create(const fi_model_desc *desc, fi_model **out) {
    if (!out) return set_error("null output handle"), FI_ERR_ARG;
    *out = nullptr;
    fi_status st = validate(desc);
    if (st != FI_OK) return st;
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0) return set_error("no CUDA device available"), FI_ERR_CUDA;
    if (desc->device < 0 || desc->device >= ndev) return set_error("device ordinal out of range"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(desc->device), "cudaSetDevice");

    fi_model *m = new fi_model();
    m->d = *desc;
    m->esz = desc->dtype == FI_F64 ? 8 : 4;
    m->ib = desc->immersed != 0;
    const fi_grid &gr = desc->grid;
    Geom &g = m->g;
    g.nd = gr.nd;
    for (int k = 0; k < 3; k++) g.n[k] = k < gr.nd ? gr.n[k] : 0;
    g.pitch = ((long long)gr.n[0] + 3 + kXOff + 31) / 32 * 32;
    g.rows = gr.n[1] + 3;
    g.sxy = g.pitch * g.rows;
    g.planes = gr.nd == 3 ? gr.n[2] + 3 : 1;
    m->elems = (size_t)g.sxy * (size_t)g.planes;

    KParams &kp = m->kp;
    for (int k = 0; k < 3; k++) kp.inv_dx[k] = k < gr.nd ? 1.0 / (gr.extent[k] / gr.n[k]) : 0.0;
    for (int k = 0; k < 3; k++) {
        kp.g_kind[k] = desc->gravity.kind[k];
        kp.g_val[k] = desc->gravity.value[k];
    }
    set_rheology_dtau(kp, desc->rheology, desc->dtau);
    for (int k = 0; k < 3; k++)
        for (int s = 0; s < 2; s++) {
            kp.bc_kind[k][s] = k < gr.nd ? desc->bc[k][s].kind : FI_BC_TRACTION;
            for (int c = 0; c < 3; c++) kp.bc_val[k][s][c] = desc->bc[k][s].c[c];
        }
    kp.small = desc->dtype == FI_F64 ? 1e-6 : (double)small_threshold_f32();

    auto fail = [&](fi_status s) {
        fi_model_destroy(m);
        return s;
    };
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "stream create"));

    // kernel path
    int want = desc->path;
    bool fok = fused_ok(m);
    if (want == FI_PATH_FUSED && !fok) {
        set_error("the fused sweep does not cover this problem (3D, FP32/FP64, no z-periodicity, no immersed boundary)");
        return fail(FI_ERR_UNSUPPORTED);
    }
    m->path = (want == FI_PATH_REFERENCE || !fok) ? FI_PATH_REFERENCE : FI_PATH_FUSED;
    for (int k = 0; k < gr.nd; k++)
        for (int s2 = 0; s2 < 2; s2++)
            if (desc->bc[k][s2].kind == FI_BC_HALO && m->path != FI_PATH_FUSED) {
                set_error("a subdomain with halo sides runs the fused sweep (its ghost stresses follow the exchanged velocities)");
                return fail(FI_ERR_UNSUPPORTED);
            }

    const size_t bytes = m->elems * m->esz;
    for (int f = 0; f < FI_FIELD_COUNT; f++) {
        if (!field_used(m, f) || is_residual(f)) continue;
        if (field_alloc(&m->base[f], m->elems, m->esz) != cudaSuccess) {
            cudaGetLastError();
            set_error("device allocation failed (" + std::to_string(bytes) + " bytes per field)");
            return fail(FI_ERR_OOM);
        }
        if (cudaMemsetAsync(field_raw(m->base[f], m->esz), 0, bytes + 64 * m->esz, m->stream) != cudaSuccess)
            return fail(cuda_fail(cudaGetLastError(), "memset"));
    }
    if (m->path == FI_PATH_FUSED) {
        for (int f = 0; f < kState; f++) {
            if (!field_used(m, f)) continue;
            if (field_alloc(&m->alt[f], m->elems, m->esz) != cudaSuccess) {
                cudaGetLastError();
                set_error("device allocation failed (second state buffer)");
                return fail(FI_ERR_OOM);
            }
            if (cudaMemsetAsync(field_raw(m->alt[f], m->esz), 0, bytes + 64 * m->esz, m->stream) != cudaSuccess)
                return fail(cuda_fail(cudaGetLastError(), "memset"));
        }
    }
    if (cudaMalloc(&m->d_err, sizeof(int)) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "error word"));
    if (m->ib && (cudaMalloc(&m->d_ibf, m->elems) != cudaSuccess ||
                  cudaMalloc(&m->d_blist, vertex_grid_blocks(g) * sizeof(uint2)) != cudaSuccess ||
                  cudaMalloc(&m->d_bcount, sizeof(int)) != cudaSuccess))
        return fail(cuda_fail(cudaGetLastError(), "activity bytes"));
    cudaMemsetAsync(m->d_err, 0, sizeof(int), m->stream);
    if (m->path == FI_PATH_FUSED) {
        fi_status es = encode_maps(m);
        if (es != FI_OK) return fail(es);
    }
    m->nblk = norm_blocks(g);
    if (cudaMalloc(&m->d_partials, (size_t)m->nblk * kNormSlots * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&m->d_out, FI_NORMS_LEN * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&m->h_out, FI_NORMS_LEN * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        set_error("norm scratch allocation failed");
        return fail(FI_ERR_OOM);
    }
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "create sync"));
    *out = m;
    return FI_OK;
}

fi_status fi_model_destroy(fi_model *m) {
    if (!m) return FI_OK;
    cudaSetDevice(m->d.device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    if (m->stream2) cudaStreamSynchronize(m->stream2);
    for (int f = 0; f < FI_FIELD_COUNT; f++) field_free(m->base[f], m->esz);
    for (int f = 0; f < kState; f++) field_free(m->alt[f], m->esz);
    if (m->d_err) cudaFree(m->d_err);
    if (m->d_ibf) cudaFree(m->d_ibf);
    if (m->d_blist) cudaFree(m->d_blist);
    if (m->d_bcount) cudaFree(m->d_bcount);
    for (cudaGraphExec_t &g : m->pair_graph)
        if (g) cudaGraphExecDestroy(g);
    field_free(m->fP, m->esz);
    if (m->d_stage) cudaFree(m->d_stage);
    if (m->shadow) fi_model_destroy(m->shadow);
    if (m->d_partials) cudaFree(m->d_partials);
    if (m->d_out) cudaFree(m->d_out);
    if (m->h_out) cudaFreeHost(m->h_out);
    if (m->ev_bnd) cudaEventDestroy(m->ev_bnd);
    if (m->ev_int) cudaEventDestroy(m->ev_int);
    if (m->stream2) cudaStreamDestroy(m->stream2);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return FI_OK;
}

fi_status fi_model_field_size(const fi_model *m, int32_t field, size_t *count) {
    if (!m || !count || field < 0 || field >= FI_FIELD_COUNT) return set_error("bad argument"), FI_ERR_ARG;
    *count = interior_count(m, field);
    return FI_OK;
}

fi_status fi_model_set_field(fi_model *m, int32_t field, const void *host, size_t nbytes) {
    if (!m || !host || field < 0 || field >= FI_FIELD_COUNT) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (!field_used(m, field)) return set_error("field not used by this model"), FI_ERR_ARG;
    if (nbytes != interior_count(m, field) * m->esz) return set_error("byte count does not match the field's interior"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    if (is_residual(field)) {
        fi_status st = ensure_residual_arrays(m);
        if (st != FI_OK) return st;
    }
    fi_status st = upload_interior(m, field, host);
    if (st != FI_OK) return st;
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "set_field sync");
    m->full_iters = 0;
    if (field >= FI_FIELD_NA_CCC) m->ibf_stale = true;
    return FI_OK;
}

fi_status fi_model_get_field(fi_model *m, int32_t field, void *host, size_t nbytes) {
    if (!m || !host || field < 0 || field >= FI_FIELD_COUNT) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (!field_used(m, field)) return set_error("field not used by this model"), FI_ERR_ARG;
    if (nbytes != interior_count(m, field) * m->esz) return set_error("byte count does not match the field's interior"), FI_ERR_ARG;
    if (is_residual(field) && !m->base[field]) return set_error("residuals not computed yet"), FI_ERR_STATE;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    cudaMemcpy3DParms p = copy_params(m, field, m->cur(field), host, false);
    FI_CHECK_CUDA(cudaMemcpy3DAsync(&p, m->stream), "get_field copy");
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "get_field sync");
    return FI_OK;
}

fi_status fi_model_copy_field(fi_model *m, int32_t dst, int32_t src) {
    if (!m || dst < 0 || dst >= FI_FIELD_COUNT || src < 0 || src >= FI_FIELD_COUNT || dst == src)
        return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (!field_used(m, dst) || !field_used(m, src)) return set_error("field not used by this model"), FI_ERR_ARG;
    if (is_residual(dst) || is_residual(src)) return set_error("residual fields are outputs"), FI_ERR_ARG;
    int ld[3], ls[3];
    field_loc(dst, ld);
    field_loc(src, ls);
    if (ld[0] != ls[0] || ld[1] != ls[1] || ld[2] != ls[2])
        return set_error("the two fields have different staggered locations"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    FI_CHECK_CUDA(cudaMemcpyAsync(field_raw(m->cur(dst), m->esz), field_raw(m->cur(src), m->esz),
                                  (m->elems + 64) * m->esz, cudaMemcpyDeviceToDevice, m->stream),
                  "copy_field");
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "copy_field sync");
    m->full_iters = 0;
    if (dst >= FI_FIELD_NA_CCC) m->ibf_stale = true;
    return FI_OK;
}

fi_status fi_model_apply_bcs(fi_model *m) {
    if (!m) return set_error("null model"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    fi_status st = m->is_f64() ? apply_bcs_t<double>(m) : apply_bcs_t<float>(m);
    if (st != FI_OK) return st;
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "apply_bcs sync");
    return FI_OK;
}

fi_status fi_model_advance(fi_model *m, int32_t niter) {
    if (!m || niter < 0) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    return m->is_f64() ? advance_t<double>(m, niter) : advance_t<float>(m, niter);
}

fi_status fi_model_set_params(fi_model *m, const fi_rheology *rheology, const fi_pt_params *dtau) {
    if (!m || !rheology || !dtau) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    const fi_rheology &r = *rheology, &o = m->d.rheology;
    // the fields a rheology reads were allocated for the model's own kinds
    if (r.eta_is_field != o.eta_is_field || r.A_is_field != o.A_is_field)
        return set_error("the new rheology must read the same fields (η, A) as the model's"), FI_ERR_ARG;
    if (r.inner != FI_RHEO_LINEAR && r.inner != FI_RHEO_POWER) return set_error("unknown rheology"), FI_ERR_ARG;
    if (r.has_reg && !(r.eta_reg > 0.0)) return set_error("the regularisation viscosity must be positive"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "sync");
    m->d.rheology = r;
    m->d.dtau = *dtau;
    set_rheology_dtau(m->kp, r, *dtau);
    m->full_iters = 0;  // the viscosity far from the ice may change: every point runs again
    if (m->shadow) {
        // the FP32 shadow of the mixed-precision solve follows (its base parameters too)
        fi_model *s = m->shadow;
        s->d.rheology = r;
        s->d.dtau = *dtau;
        set_rheology_dtau(s->kp, r, *dtau);
        set_rheology_dtau(m->shadow_kp, r, *dtau);
        s->full_iters = 0;
    }
    return FI_OK;
}

fi_status fi_model_advance_begin(fi_model *m, int32_t dim) {
    if (!m || (dim != 0 && dim != 1)) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (m->path != FI_PATH_FUSED) return set_error("an overlapped iteration needs the fused sweep"), FI_ERR_UNSUPPORTED;
    auto away = [](int k) { return k == FI_BC_PERIODIC || k == FI_BC_HALO; };
    if (dim >= m->d.grid.nd || !(away(m->d.bc[dim][0].kind) || away(m->d.bc[dim][1].kind)))
        return set_error("the split dimension needs a periodic or halo side on the subdomain model"), FI_ERR_STATE;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    if (!m->stream2) {
        FI_CHECK_CUDA(cudaStreamCreateWithFlags(&m->stream2, cudaStreamNonBlocking), "second stream");
        FI_CHECK_CUDA(cudaEventCreateWithFlags(&m->ev_bnd, cudaEventDisableTiming), "event");
        FI_CHECK_CUDA(cudaEventCreateWithFlags(&m->ev_int, cudaEventDisableTiming), "event");
    }
    m->full_iters = 0;
    fi_status st = m->is_f64() ? advance_half<double>(m, dim, 0) : advance_half<float>(m, dim, 0);
    if (st == FI_OK) m->split_begun = dim;
    return st;
}

fi_status fi_model_advance_end(fi_model *m) {
    if (!m) return set_error("null model"), FI_ERR_ARG;
    if (m->split_begun < 0) return set_error("no overlapped iteration is begun"), FI_ERR_STATE;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    const int dim = m->split_begun;
    fi_status st = m->is_f64() ? advance_half<double>(m, dim, 1) : advance_half<float>(m, dim, 1);
    if (st != FI_OK) return st;
    m->split_begun = -1;
    m->interior_pending = true;
    m->iterations++;
    return FI_OK;
}

fi_status fi_model_compute_residuals(fi_model *m) {
    if (!m) return set_error("null model"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    return m->is_f64() ? residuals_t<double>(m) : residuals_t<float>(m);
}

fi_status fi_model_residual_norms(fi_model *m, double *out) {
    if (!m || !out) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    return m->is_f64() ? norms_t<double>(m, out) : norms_t<float>(m, out);
}

fi_status fi_model_compute_tau(fi_model *m) {
    if (!m) return set_error("null model"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (m->ib) return set_error("compute_tau of the immersed-boundary model is broken in the reference"), FI_ERR_UNSUPPORTED;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    cudaError_t e = m->is_f64() ? launch_compute_tau<double>(m->g, m->kp, m->ptrs<double>(), false, m->stream)
                                : launch_compute_tau<float>(m->g, m->kp, m->ptrs<float>(), false, m->stream);
    if (e != cudaSuccess) return cuda_fail(e, "compute_tau");
    return FI_OK;
}

fi_status fi_model_device_ptr(fi_model *m, int32_t field, void **dptr) {
    if (!m || !dptr || field < 0 || field >= FI_FIELD_COUNT) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (is_residual(field)) {
        fi_status st = ensure_residual_arrays(m);
        if (st != FI_OK) return st;
    }
    *dptr = m->cur(field);
    // the caller may write volume fractions through the pointer: their activity
    // bytes are recomputed before the next kernel that reads them
    if (field >= FI_FIELD_NA_CCC) m->ibf_stale = true, m->full_iters = 0;
    // the caller may write the state through the pointer at any later time
    if (field < kState) m->state_ptr_out = true;
    return FI_OK;
}

fi_status fi_model_layout(const fi_model *m, size_t *pitch, size_t *rows, size_t *planes) {
    if (!m) return set_error("null model"), FI_ERR_ARG;
    if (pitch) *pitch = (size_t)m->g.pitch;
    if (rows) *rows = (size_t)m->g.rows;
    if (planes) *planes = (size_t)m->g.planes;
    return FI_OK;
}

fi_status fi_model_stream(const fi_model *m, void **stream) {
    if (!m || !stream) return set_error("bad argument"), FI_ERR_ARG;
    *stream = (void *)m->stream;
    return FI_OK;
}

fi_status fi_model_synchronize(fi_model *m) {
    if (!m) return set_error("null model"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "synchronize");
    return check_err_word(m);
}

fi_status fi_model_path(const fi_model *m, int32_t *path) {
    if (!m || !path) return set_error("bad argument"), FI_ERR_ARG;
    *path = m->path;
    return FI_OK;
}

}  // extern "C"

// convergence measure of a norm vector (fi_conv_measure)
static double measure_of(const fi_model *m, const fi_solve_opts *o, const double *norms) {
    if (o->measure == FI_CONV_REL_SLAB) {
        double rv = std::max(norms[1], std::max(norms[2], m->d.grid.nd == 3 ? norms[3] : 0.0));
        double vmax = std::max(norms[8], std::max(norms[9], norms[10]));
        double a = rv / (o->rho_g_inf > 0 ? o->rho_g_inf : 1.0);
        double b = vmax > 0 ? norms[0] * o->length_z / vmax : norms[0];
        return std::max(a, b);
    }
    double meas = norms[0];
    for (int q = 1; q < 4; q++) meas = std::max(meas, norms[q]);
    return meas;
}

// ---- mixed precision: FP32 PT sweeps inside an FP64 defect correction -------------
// The FP32 shadow holds the same grid, boundary kinds and rheology; its gravity
// fields carry -r_V and its pressure forcing r_P during corrections.
static fi_status make_shadow(fi_model *m) {
    if (m->shadow) return FI_OK;
    fi_model_desc d = m->d;
    d.dtype = FI_F32;
    for (int c = 0; c < d.grid.nd; c++) d.gravity.kind[c] = FI_G_FIELD;
    fi_model *s = nullptr;
    fi_status st = fi_model_create(&d, &s);
    if (st != FI_OK) return st;
    if (field_alloc(&s->fP, s->elems, s->esz) != cudaSuccess) {
        fi_model_destroy(s);
        return set_error("forcing allocation failed"), FI_ERR_OOM;
    }
    cudaMemsetAsync(field_raw(s->fP, s->esz), 0, (s->elems + 64) * s->esz, s->stream);
    for (int f : {(int)FI_FIELD_ETA_LIN, (int)FI_FIELD_A})
        if (field_used(m, f)) {
            cudaError_t e = launch_convert<double, float>((const double *)m->base[f], (float *)s->base[f],
                                                          (long long)m->elems, 1.0, s->stream);
            if (e != cudaSuccess) {
                fi_model_destroy(s);
                return cuda_fail(e, "shadow inputs");
            }
        }

    if (s->path == FI_PATH_FUSED && fused3d_num_variants() > 4) {
        s->fused_variant = 4;  // 32x16 tiles: the FP32 shape the autotuner prefers on the slab
        fi_status es = encode_maps(s);
        if (es != FI_OK) {
            fi_model_destroy(s);
            return es;
        }
    }
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
        fi_model_destroy(s);
        return cuda_fail(cudaGetLastError(), "shadow sync");
    }
    m->shadow = s;
    m->shadow_kp = s->kp;
    return FI_OK;
}

template <typename S, typename D>
static fi_status convert_field(void *dst, const void *src, long long n, double scale, cudaStream_t st) {
    cudaError_t e = launch_convert<S, D>((const S *)src, (D *)dst, n, scale, st);
    return e == cudaSuccess ? FI_OK : cuda_fail(e, "convert");
}

// Rounding floor of an FP32 residual evaluation on the shadow: a difference of two
// values of magnitude S over a spacing dx carries an error of about eps32 * S / dx,
// so r_V bottoms out near eps32 * max|P, τ| / dx and r_P near eps32 * max|V| / dx.
// kFloorMargin (measured: the floors of the 3D manufactured solution sit 10-20x
// above the bare estimate at 127^3-255^3) keeps the stop comfortably above them.
constexpr double kFloorMargin = 48.0;
constexpr double kEps32 = 1.1920928955078125e-07;

static fi_status fp32_floors(fi_model *s, const double *nn, double *fl_P, double *fl_V) {
    const float *fs[7];
    int cnt = 0;
    for (int f = FI_FIELD_P; f <= FI_FIELD_TYZ; f++)
        if (field_used(s, f)) fs[cnt++] = (const float *)s->cur(f);
    unsigned *d = reinterpret_cast<unsigned *>(s->d_out);
    FI_CHECK_CUDA(launch_absmax_f32(fs, cnt, (long long)s->elems, d, s->stream), "abs max");
    unsigned bits = 0;
    FI_CHECK_CUDA(cudaMemcpyAsync(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost, s->stream), "abs max copy");
    FI_CHECK_CUDA(cudaStreamSynchronize(s->stream), "abs max sync");
    float smax;
    std::memcpy(&smax, &bits, sizeof(smax));
    double idx = 0.0;
    for (int c = 0; c < s->d.grid.nd; c++) idx = std::max(idx, s->kp.inv_dx[c]);
    const double vmax = std::max(nn[8], std::max(nn[9], nn[10]));
    *fl_V = kFloorMargin * kEps32 * (double)smax * idx;
    *fl_P = kFloorMargin * kEps32 * vmax * idx;
    return FI_OK;
}

// ---- stages of the defect correction, shared by the single-model solve and the
// batched one (fi_batch_solve_mixed) ------------------------------------------------
static const int kGravF[3] = {FI_FIELD_GX, FI_FIELD_GY, FI_FIELD_GZ};
static const int kResVF[3] = {FI_FIELD_RVX, FI_FIELD_RVY, FI_FIELD_RVZ};
static const int kTauF[6] = {FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TZZ, FI_FIELD_TXY, FI_FIELD_TXZ, FI_FIELD_TYZ};

// the shadow's parameters for the full problem (phase A: the model's own gravity and
// boundary values) and for a correction (homogeneous boundary values, frozen η,
// forcing r); built from the shadow's parameters as created (a previous solve leaves
// its last stage's parameters in the shadow)
static KParams mixed_kp(const fi_model *m, bool correction) {
    KParams k = m->shadow_kp;
    if (!correction) {
        for (int c = 0; c < 3; c++) {
            k.g_kind[c] = m->kp.g_kind[c];
            k.g_val[c] = m->kp.g_val[c];
        }
        return k;
    }
    for (int d = 0; d < 3; d++)
        for (int sd = 0; sd < 2; sd++)
            for (int c = 0; c < 3; c++) k.bc_val[d][sd][c] = 0.0;
    k.freeze_eta = 1;
    k.p_forcing = 1;
    return k;
}

// phase A: the FP64 state, viscosity and gravity fields rounded into the shadow,
// which then runs the full problem
fi_status mixed_phase_a_begin(fi_model *m) {
    fi_model *s = m->shadow;
    const long long n = (long long)m->elems;
    fi_status st;
    for (int f = 0; f < kState; f++)
        if (field_used(m, f) && (st = convert_field<double, float>(s->cur(f), m->cur(f), n, 1.0, m->stream)) != FI_OK)
            return st;
    for (int f : {(int)FI_FIELD_ETA, (int)FI_FIELD_ETA_NEXT})
        if ((st = convert_field<double, float>(s->cur(f), m->cur(f), n, 1.0, m->stream)) != FI_OK) return st;
    for (int c = 0; c < m->d.grid.nd; c++)
        if (m->kp.g_kind[c] == FI_G_FIELD &&
            (st = convert_field<double, float>(s->base[kGravF[c]], m->base[kGravF[c]], n, 1.0, m->stream)) != FI_OK)
            return st;
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "mixed sync");
    s->kp = mixed_kp(m, false);
    return FI_OK;
}

// end of phase A: the shadow's state back into the FP64 model
fi_status mixed_phase_a_end(fi_model *m) {
    fi_model *s = m->shadow;
    const long long n = (long long)m->elems;
    fi_status st;
    for (int f = 0; f < kState; f++)
        if (field_used(m, f) && (st = convert_field<float, double>(m->cur(f), s->cur(f), n, 1.0, s->stream)) != FI_OK)
            return st;
    for (int f : {(int)FI_FIELD_ETA, (int)FI_FIELD_ETA_NEXT})
        if ((st = convert_field<float, double>(m->cur(f), s->cur(f), n, 1.0, s->stream)) != FI_OK) return st;
    FI_CHECK_CUDA(cudaStreamSynchronize(s->stream), "mixed sync");
    return FI_OK;
}

// viscosity from the current stresses (Picard step)
fi_status mixed_picard(fi_model *m) {
    Ptrs<double> f = m->ptrs<double>();
    FI_CHECK_CUDA(launch_eta_from_tau<double>(m->g, m->kp, f, m->stream), "eta refresh");
    m->eta_swapped = !m->eta_swapped;
    return run_eta_batch<double>(m, FI_FIELD_ETA);
}

// A correction: projection τ = 2η dev(ε̇(V)) with its BCs (the stresses before it kept
// in the second state buffer), the FP64 residual fields of the projected anchor, and
// the correction problem on the shadow -- frozen η, forcing r_P and -r_V, zero state,
// stresses starting from the constitutive defect.
fi_status mixed_correction_begin(fi_model *m) {
    fi_model *s = m->shadow;
    const long long n = (long long)m->elems;
    const int nd = m->d.grid.nd;
    fi_status st;
    for (int q = 0; q < 6; q++)
        if (field_used(m, kTauF[q]))
            FI_CHECK_CUDA(cudaMemcpyAsync(field_raw(m->nxt(kTauF[q]), m->esz), field_raw(m->cur(kTauF[q]), m->esz),
                                          (m->elems + 64) * m->esz, cudaMemcpyDeviceToDevice, m->stream),
                          "stress copy");
    if ((st = refresh_ibf<double>(m)) != FI_OK) return st;
    FI_CHECK_CUDA(launch_compute_tau<double>(m->g, m->kp, m->ptrs<double>(), m->ib, m->stream), "projection");
    if ((st = run_batch<double>(m, stress_batch)) != FI_OK) return st;
    if ((st = residuals_t<double>(m)) != FI_OK) return st;
    if ((st = convert_field<double, float>(s->cur(FI_FIELD_ETA), m->cur(FI_FIELD_ETA), n, 1.0, m->stream)) != FI_OK)
        return st;
    if ((st = convert_field<double, float>(s->fP, m->base[FI_FIELD_RP], n, 1.0, m->stream)) != FI_OK) return st;
    for (int c = 0; c < nd; c++)
        if ((st = convert_field<double, float>(s->base[kGravF[c]], m->base[kResVF[c]], n, -1.0, m->stream)) != FI_OK)
            return st;
    for (int fl = 0; fl < kState; fl++) {
        if (!field_used(s, fl)) continue;
        FI_CHECK_CUDA(cudaMemsetAsync(field_raw(s->base[fl], s->esz), 0, (s->elems + 64) * s->esz, m->stream), "zero");
        if (s->alt[fl])
            FI_CHECK_CUDA(cudaMemsetAsync(field_raw(s->alt[fl], s->esz), 0, (s->elems + 64) * s->esz, m->stream), "zero");
    }
    for (int q = 0; q < 6; q++)
        if (field_used(m, kTauF[q])) {
            cudaError_t e = launch_diff<double, float>((const double *)m->nxt(kTauF[q]), (const double *)m->cur(kTauF[q]),
                                                       (float *)s->cur(kTauF[q]), n, m->stream);
            if (e != cudaSuccess) return cuda_fail(e, "constitutive defect");
        }
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "mixed sync");
    s->kp = mixed_kp(m, true);
    s->full_iters = 0;
    return FI_OK;
}

// x += δ in FP64
fi_status mixed_correction_end(fi_model *m) {
    fi_model *s = m->shadow;
    const long long n = (long long)m->elems;
    for (int fl = 0; fl < kState; fl++)
        if (field_used(m, fl)) {
            cudaError_t e = launch_accumulate<double, float>((double *)m->cur(fl), (const float *)s->cur(fl), n, m->stream);
            if (e != cudaSuccess) return cuda_fail(e, "accumulate");
        }
    return FI_OK;
}

// the FP32 shadow of an FP64 model (created on first use, masks refreshed)
fi_status mixed_shadow(fi_model *m) {
    if (!m->is_f64()) return set_error("the mixed-precision solve refines an FP64 model"), FI_ERR_ARG;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    fi_status st = make_shadow(m);
    if (st != FI_OK) return st;
    fi_model *s = m->shadow;
    for (int f = FI_FIELD_NA_CCC; f < FI_FIELD_NA_CCC + 16 && m->ib; f++)
        if (field_used(m, f))
            FI_CHECK_CUDA(launch_mask_to_f32((const double *)m->base[f], (float *)s->base[f], (long long)m->elems,
                                             (float)s->kp.small, m->stream),
                          "shadow volume fractions");
    if (m->ib) {
        s->ibf_stale = true, s->full_iters = 0;
        FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "shadow volume fractions");
    }
    return FI_OK;
}

// The reference's driver loop: ncheck iterations, the residual norms, the
// convergence test on the solve's measure; `it0` sweeps already spent (the
// mixed solve's FP32 phase) count against max_iter.
static fi_status solve_plain(fi_model *m, const fi_solve_opts *o, fi_solve_report *rep, int it0) {
    auto t0 = std::chrono::steady_clock::now();
    const bool trace = std::getenv("FI_SOLVE_TRACE") != nullptr;
    int it = it0;
    fi_status st = FI_OK;
    double norms[FI_NORMS_LEN];
    while (it < o->max_iter) {
        int n = o->ncheck;
        if (it + n > o->max_iter) n = o->max_iter - it;
        st = fi_model_advance(m, n);
        if (st != FI_OK) return st;
        it += n;
        st = fi_model_residual_norms(m, norms);
        if (st != FI_OK) return st;
        double meas = measure_of(m, o, norms);
        if (trace) std::fprintf(stderr, "[fi solve] sweeps=%d measure=%.3e\n", it, meas);
        rep->measure = meas;
        std::memcpy(rep->norms, norms, sizeof(norms));
        if (norms[11] != 0.0 || !std::isfinite(meas)) {
            rep->iterations = it;
            set_error("simulation failed: non-finite residual");
            return FI_ERR_DIVERGED;
        }
        if (meas < o->tol) {
            rep->converged = 1;
            break;
        }
    }
    rep->iterations = it;
    rep->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rep->converged ? FI_OK : FI_ERR_TIMEOUT;
}

static fi_status solve_mixed(fi_model *m, const fi_solve_opts *o, fi_solve_report *rep) {
    m->full_iters = 0;  // the solve writes the FP64 state outside its sweeps
    // the shadow, its volume fractions refreshed every solve (the caller may have
    // recomputed them): it sees the FP64 model's empty, valid and null-space points
    fi_status st = mixed_shadow(m);
    if (st != FI_OK) return st;
    fi_model *s = m->shadow;
    const int nd = m->d.grid.nd;
    const double inner_red = o->inner_reduction > 0 ? o->inner_reduction : 1e-3;
    const int inner_max = o->inner_iter > 0 ? o->inner_iter : 50 * o->ncheck;
    // a stage that has not halved its best residual over this many sweeps has stalled
    int window = 0;
    for (int c = 0; c < nd; c++) window = std::max(window, 2 * (m->d.grid.n[c] + 1));
    window = std::max(window, 2 * o->ncheck);
    auto t0 = std::chrono::steady_clock::now();
    double norms[FI_NORMS_LEN];
    int sweeps = 0;
    const bool trace = std::getenv("FI_SOLVE_TRACE") != nullptr;  // per-check progress on stderr

    // FP32 sweeps on the shadow, a check every ncheck, until (a) the FP64 tolerance
    // in the solve's measure (phase A only), (b) the four residual inf-norms drop to
    // target, (c) they reach the FP32 rounding floor (phase A only), (d) the best of
    // them has not halved for `window` sweeps (phase A: not fallen by a fifth for
    // twice that -- a stiff stage of a viscosity continuation converges slowly but
    // steadily), or (e) max_sweeps
    auto stage = [&](bool phase_a, double target, int max_sweeps, const char *what) -> fi_status {
        double best = 1e300;
        int since = 0, done = 0;
        const double gain = phase_a ? 0.8 : 0.5;
        const int win = phase_a ? 2 * window : window;
        double nn[FI_NORMS_LEN];
        s->full_iters = 0;  // the shadow's state was set outside its sweeps
        while (done < max_sweeps && sweeps < o->max_iter) {
            int k = std::min(o->ncheck, o->max_iter - sweeps);
            fi_status e = fi_model_advance(s, k);
            if (e != FI_OK) return e;
            sweeps += k;
            done += k;
            if ((e = fi_model_residual_norms(s, nn)) != FI_OK) return e;
            const double rv = std::max(nn[1], std::max(nn[2], nn[3]));
            const double r = std::max(nn[0], rv);
            if (nn[11] != 0.0 || !std::isfinite(r)) {
                rep->iterations = sweeps;
                return set_error(std::string("simulation failed: non-finite residual in the ") + what), FI_ERR_DIVERGED;
            }
            double fl_P = 0, fl_V = 0;
            if ((e = fp32_floors(s, nn, &fl_P, &fl_V)) != FI_OK) return e;
            if (trace)
                std::fprintf(stderr, "[fi mixed] %s sweeps=%d r=%.3e target=%.3e floors P %.2e V %.2e\n", what, sweeps,
                             r, target, fl_P, fl_V);
            if (phase_a && measure_of(s, o, nn) < o->tol) break;
            if (r <= target) break;
            // the rounding floor ends the full-problem phase; a correction stops at its
            // target or when it stalls (its own floor scales with the correction and
            // would stop it before it has reduced anything)
            if (phase_a && nn[0] <= fl_P && rv <= fl_V) break;
            if (r < gain * best) {
                best = r;
                since = 0;
            } else if ((since += k) >= win) {
                break;
            }
        }
        return FI_OK;
    };

    // ---- phase A: FP32 PT on the full problem down to the FP32 floor
    if ((st = mixed_phase_a_begin(m)) != FI_OK) return st;
    if ((st = stage(true, 0.0, o->max_iter, "fp32 phase")) != FI_OK) return st;
    if ((st = mixed_phase_a_end(m)) != FI_OK) return st;

    // A power law makes η a function of the iterate: the correction below freezes η
    // and an outer step refreshes it from τ (a Picard step), whose slope in log η is
    // 1 - m for the local exponent m = 1 + (n-1)(1 - η/η_reg) where the strain rate
    // is held -- -2 for n = 3, a divergent iteration (and damped to contract, it
    // still needs an outer step per halving, measured far slower than PT).  The
    // FP64 PT iteration, which updates η inside every sweep, finishes such a solve
    // from the FP32 phase's state instead.
    if (m->kp.rheo_inner == FI_RHEO_POWER && m->kp.rheo_n != 1) {
        if (sweeps < o->max_iter) {
            st = solve_plain(m, o, rep, sweeps);
        } else {  // the FP32 phase used every sweep: report the FP64 iterate
            if ((st = norms_t<double>(m, norms)) != FI_OK) return st;
            rep->measure = measure_of(m, o, norms);
            std::memcpy(rep->norms, norms, sizeof(norms));
            rep->converged = rep->measure < o->tol;
            rep->iterations = sweeps;
            st = rep->converged ? FI_OK : FI_ERR_TIMEOUT;
        }
        rep->outer = 0;
        rep->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return st;
    }

    // ---- phase B: FP64 defect correction with FP32 correction sweeps
    //
    // For a fixed viscosity one PT iteration is an affine map x -> M x + c, so PT
    // continued on a correction y from an anchor a follows y -> M y + (M a + c - a).
    // Its pressure and velocity parts are forced by r_P(a) and r_V(a); its stress
    // part carries no forcing once the anchor's stresses are replaced by the
    // viscous law of its velocities (the projection) and the correction's stresses
    // start from the difference the projection removed (the constitutive defect
    // d = τ_a - 2η dev ε̇(V_a), taken in FP64, then rounded).  The FP32 sweeps on y
    // then continue the FP64 iteration instead of restarting it from rest.
    int outer = 0, outer_stale = 0;
    double best_outer = 1e300;
    if ((st = model_ensure_second_state(m)) != FI_OK) return st;
    while (true) {
        if ((st = mixed_picard(m)) != FI_OK) return st;
        // FP64 residual norms of the iterate itself (its own stresses), the quantity
        // the plain solve tests
        if ((st = norms_t<double>(m, norms)) != FI_OK) return st;
        double meas = measure_of(m, o, norms);
        if (trace) std::fprintf(stderr, "[fi mixed] outer=%d sweeps=%d fp64 measure=%.3e\n", outer, sweeps, meas);
        rep->measure = meas;
        std::memcpy(rep->norms, norms, sizeof(norms));
        if (norms[11] != 0.0 || !std::isfinite(meas) || meas > 100.0 * best_outer) {
            rep->iterations = sweeps;
            rep->outer = outer;
            return set_error("simulation failed: the defect correction diverged"), FI_ERR_DIVERGED;
        }
        if (meas < o->tol) {
            rep->converged = 1;
            break;
        }
        if (sweeps >= o->max_iter) break;
        // three outer steps in a row without halving the FP64 measure: the
        // correction no longer reaches the residual (stop, not converged)
        if (meas < 0.5 * best_outer) outer_stale = 0;
        else if (++outer_stale >= 3) break;
        best_outer = std::min(best_outer, meas);
        if ((st = mixed_correction_begin(m)) != FI_OK) return st;
        // target: inner_reduction of r0, but no further than a third of the tolerance
        // (scaled from the solve's measure to the residual inf-norms)
        const double r0 = std::max(std::max(norms[0], norms[1]), std::max(norms[2], norms[3]));
        const double target = std::max(inner_red * r0, meas > 0 ? o->tol / 3.0 * r0 / meas : 0.0);
        if ((st = stage(false, target, inner_max, "correction")) != FI_OK) {
            rep->outer = outer;
            return st;
        }
        if ((st = mixed_correction_end(m)) != FI_OK) return st;
        outer++;
    }
    rep->iterations = sweeps;
    rep->outer = outer;
    rep->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rep->converged ? FI_OK : FI_ERR_TIMEOUT;
}

extern "C" {

fi_status fi_model_solve(fi_model *m, const fi_solve_opts *o, fi_solve_report *rep) {
    if (!m || !o || !rep) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (o->ncheck <= 0 || o->max_iter <= 0) return set_error("ncheck and max_iter must be positive"), FI_ERR_ARG;
    if (o->mode != FI_SOLVE_PLAIN && o->mode != FI_SOLVE_MIXED) return set_error("unknown solve mode"), FI_ERR_ARG;
    std::memset(rep, 0, sizeof(*rep));
    if (o->mode == FI_SOLVE_MIXED) return solve_mixed(m, o, rep);
    return solve_plain(m, o, rep, 0);
}

fi_status fi_model_volfrac_from_levelset(fi_model *m, int32_t group, const double *psi_host) {
    if (!m || !psi_host || (group != 0 && group != 1)) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (!m->ib) return set_error("volume fractions need an immersed-boundary model"), FI_ERR_STATE;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    const Geom &g = m->g;
    const size_t bytes = m->elems * sizeof(double);
    void *dpsi = nullptr;
    void *tmp[8] = {};
    auto cleanup = [&]() {
        field_free(dpsi, sizeof(double));
        for (int c = 0; c < 8; c++) field_free(tmp[c], sizeof(double));
    };
    if (field_alloc(&dpsi, m->elems, sizeof(double)) != cudaSuccess)
        return cleanup(), set_error("allocation failed"), FI_ERR_OOM;
    cudaMemsetAsync(field_raw(dpsi, sizeof(double)), 0, bytes + 64 * sizeof(double), m->stream);
    // dense halo storage (n0+3) x (n1+3) x (n2+3) -> pitched storage
    cudaMemcpy3DParms cp{};
    size_t nx = (size_t)g.n[0] + 3, ny = (size_t)g.n[1] + 3, nz = (size_t)g.planes;
    cp.srcPtr = make_cudaPitchedPtr(const_cast<double *>(psi_host), nx * sizeof(double), nx, ny);
    cp.dstPtr = make_cudaPitchedPtr(field_raw(dpsi, sizeof(double)), (size_t)g.pitch * sizeof(double), (size_t)g.pitch,
                                    (size_t)g.rows);
    cp.dstPos = make_cudaPos((size_t)kXOff * sizeof(double), 0, 0);
    cp.extent = make_cudaExtent(nx * sizeof(double), ny, nz);
    cp.kind = cudaMemcpyHostToDevice;
    if (cudaMemcpy3DAsync(&cp, m->stream) != cudaSuccess) return cleanup(), cuda_fail(cudaGetLastError(), "psi upload");
    double *w[8];
    const int base = group == 0 ? FI_FIELD_NA_CCC : FI_FIELD_NS_CCC;
    for (int c = 0; c < 8; c++) {
        if (m->is_f64()) {
            w[c] = (double *)m->base[base + c];
        } else {
            if (field_alloc(&tmp[c], m->elems, sizeof(double)) != cudaSuccess)
                return cleanup(), set_error("allocation failed"), FI_ERR_OOM;
            cudaMemsetAsync(field_raw(tmp[c], sizeof(double)), 0, bytes + 64 * sizeof(double), m->stream);
            w[c] = (double *)tmp[c];
        }
    }
    double dx[3];
    for (int k = 0; k < 3; k++) dx[k] = m->d.grid.extent[k] / m->d.grid.n[k];
    cudaError_t e = launch_volfrac3d(g, dx, (const double *)dpsi, w, m->stream);
    if (e != cudaSuccess) return cleanup(), cuda_fail(e, "volfrac kernel");
    if (!m->is_f64()) {
        for (int c = 0; c < 8; c++) {
            e = launch_convert_f64_f32(w[c], (float *)m->base[base + c], (long long)m->elems, m->stream);
            if (e != cudaSuccess) return cleanup(), cuda_fail(e, "convert");
        }
    }
    e = cudaStreamSynchronize(m->stream);
    cleanup();
    if (e != cudaSuccess) return cuda_fail(e, "volfrac sync");
    m->ibf_stale = true, m->full_iters = 0;
    return FI_OK;
}

int fi_fused_variant_count(void) { return fused3d_num_variants(); }
const char *fi_fused_variant_name(int32_t variant) { return fused3d_variant_name(variant); }

fi_status fi_model_set_variant(fi_model *m, int32_t variant) {
    if (!m || variant < 0 || variant >= fused3d_num_variants()) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (m->path != FI_PATH_FUSED) return set_error("the model does not run the fused sweep"), FI_ERR_STATE;
    if (!fused3d_variant_fits(variant, (int)m->esz))
        return set_error("this launch shape does not fit a CTA in the model's precision"), FI_ERR_UNSUPPORTED;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    FI_CHECK_CUDA(cudaStreamSynchronize(m->stream), "sync");
    m->fused_variant = variant;
    return encode_maps(m);
}

fi_status fi_model_autotune(fi_model *m, int32_t iters, int32_t *best, double *ms) {
    if (!m || iters <= 0) return set_error("bad argument"), FI_ERR_ARG;
    if (fi_status js = join_overlap(m); js != FI_OK) return js;
    if (m->path != FI_PATH_FUSED) return set_error("the model does not run the fused sweep"), FI_ERR_STATE;
    FI_CHECK_CUDA(cudaSetDevice(m->d.device), "cudaSetDevice");
    cudaEvent_t e0, e1;
    FI_CHECK_CUDA(cudaEventCreate(&e0), "event");
    FI_CHECK_CUDA(cudaEventCreate(&e1), "event");
    int nv = fused3d_num_variants(), bestv = m->fused_variant;
    double bestms = 1e300;
    fi_status st = FI_OK;
    for (int v = 0; v < nv && st == FI_OK; v++) {
        if (!fused3d_variant_fits(v, (int)m->esz)) {
            if (ms) ms[v] = -1.0;  // not offered in this precision
            continue;
        }
        st = fi_model_set_variant(m, v);
        if (st != FI_OK) break;
        st = fi_model_advance(m, 1);  // warm-up of this launch shape
        if (st == FI_ERR_CUDA && cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(m->stream) == cudaSuccess) {
            // the shape could not be launched here (e.g. no room for its cluster); the
            // device is healthy: leave the shape out
            if (ms) ms[v] = -1.0;
            st = FI_OK;
            continue;
        }
        if (st != FI_OK) break;
        cudaEventRecord(e0, m->stream);
        st = fi_model_advance(m, iters);
        cudaEventRecord(e1, m->stream);
        if (st != FI_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            st = cuda_fail(cudaGetLastError(), "autotune sync");
            break;
        }
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        double per = (double)t / iters;
        if (ms) ms[v] = per;
        if (per < bestms) {
            bestms = per;
            bestv = v;
        }
        st = check_err_word(m);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != FI_OK) return st;
    if (best) *best = bestv;
    return fi_model_set_variant(m, bestv);
}

}  // extern "C"
