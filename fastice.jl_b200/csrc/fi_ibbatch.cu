// fi_ibbatch.cu -- several 3D immersed-boundary models advanced by shared launches.
//
// Reference semantics per member: advance_iteration! of the immersed-boundary model
// (src/Models/ImmersedBoundaryFullStokes/Isothermal/Isothermal.jl:100-122): update_σ!,
// the stress boundary batches per dimension, update_V!, the velocity boundary batches,
// the η swap.  A member's iteration here is exactly the one fi_model_advance runs for
// it (the same kernel bodies on the same block list), so its result is the same
// advanced alone or in the batch.
//
// Launches.  One iteration of all members is eight launches whatever their number:
// the masked stress update over a work list that concatenates every member's blocks
// (its block list once the stored zeros hold, else its whole block grid), the three
// stress boundary batches of all members (one launch per dimension, one grid slice per
// member and op), the masked velocity update over the same work list, the three
// velocity boundary batches.  Each block reads its member's geometry, parameters and
// field pointers from a device table into shared memory.  Two iterations (which bring
// the η buffers back to their roles) are captured as one CUDA graph and replayed.
//
// A member whose state was written from outside since its last two full iterations
// (fi_model_set_field, ω_from_ψ!, a new member) runs those iterations alone first,
// exactly as fi_model_advance does, and joins the shared launches from the next call.
// A member whose own launch spans more than kShareBlocks blocks, or the only member
// left to share, advances by fi_model_advance on its own stream.  The shared launches
// wait for the members' streams by events; the members' streams wait for them by the
// `done` event.
#include <algorithm>
#include <cstring>
#include <vector>

#include "fi_model.h"

#define FB_CHECK(expr, where)                                \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, where);  \
    } while (0)

using namespace fi;

struct fi_ib_batch {
    std::vector<fi_model *> models;
    bool f64 = true;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    // the shared-launch table and what it was built from
    std::vector<fi_model *> table_models;
    std::vector<KParams> table_kp;
    std::vector<int> table_eta, table_list, table_nblist;
    void *d_members = nullptr;
    size_t members_cap = 0;
    uint4 *d_items = nullptr;
    long long items_cap = 0;
    int nitems = 0;
    // [9][count]: stress x, y, z; velocity x, y, z with the η roles of the table
    // (epar 0), then with them swapped (epar 1: the η_next Neumann ops follow η_next)
    BcMember *d_bc = nullptr;
    int bc_cap = 0;
    int max_a[3] = {0, 0, 0}, max_c[3] = {0, 0, 0};
    int epar = 0;  // iterations since the table was built, mod 2 (the members' η roles)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};  // a pair of iterations starting at epar 0 / 1
    std::vector<cudaEvent_t> member_ev;               // the members' streams, waited on by the shared launches
};

namespace {

bool eta_moves(const fi_model *m) { return !m->kp.freeze_eta && m->kp.rheo_relax != FI_RELAX_NONE; }

// a member runs alone until its first two full iterations since the state changed are done
bool runs_alone(const fi_model *m) { return !m->state_ptr_out && m->full_iters < 2; }

// the parameters a member's shared iterations use (fi_model_advance's for a member whose
// zeros hold: skipped stores, unless a state pointer was handed out)
KParams member_kp(const fi_model *m) {
    KParams k = m->kp;
    k.skip_zeros = m->state_ptr_out ? 0 : 1;
    return k;
}

bool use_list(const fi_model *m, const KParams &k) {
    return k.skip_zeros && !m->ibf_stale && m->n_blist > 0 && !eta_moves(m);
}

// A member whose launch fills the GPU several times over gains nothing from sharing
// launches (12 glaciers of 48^3-160^3 advanced at 0.99x in FP64 by shared launches,
// measured; 32 of 16^3-48^3 at 4.1x): it advances on its own stream instead, where its
// iterations overlap the other members' and keep the single-model kernels.
constexpr long long kShareBlocks = 2048;  // about two waves of 256-thread blocks at 6-7 per SM
bool too_big_to_share(const fi_model *m, bool f32) {
    return (use_list(m, member_kp(m)) ? (long long)m->n_blist : ib_grid_blocks(m->g, f32)) > kShareBlocks;
}

template <typename P>
cudaError_t regrow(P **ptr, size_t n, size_t *cap) {
    if (n <= *cap && *ptr) return cudaSuccess;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = std::max<size_t>(n, 2 * *cap);
    return cudaMalloc(ptr, std::max<size_t>(*cap, 1) * sizeof(P));
}

void drop_graphs(fi_ib_batch *b) {
    for (cudaGraphExec_t &g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

bool table_current(const fi_ib_batch *b, const std::vector<fi_model *> &shared) {
    if (shared != b->table_models) return false;
    for (size_t q = 0; q < shared.size(); q++) {
        const fi_model *m = shared[q];
        const KParams k = member_kp(m);
        if (std::memcmp(&k, &b->table_kp[q], sizeof(KParams)) != 0) return false;
        const int expect = m->kp.freeze_eta ? b->table_eta[q] : (b->table_eta[q] ^ b->epar);
        if ((int)m->eta_swapped != expect) return false;
        if ((int)use_list(m, k) != b->table_list[q] || m->n_blist != b->table_nblist[q]) return false;
    }
    return true;
}

template <typename T>
fi_status build_table(fi_ib_batch *b, const std::vector<fi_model *> &shared) {
    const int n = (int)shared.size();
    std::vector<IbMember<T>> mem(n);
    std::vector<BcMember> bc((size_t)9 * n);
    long long total = 0;
    std::vector<long long> off(n);
    for (int d = 0; d < 3; d++) b->max_a[d] = b->max_c[d] = 0;
    b->table_kp.resize(n);
    b->table_eta.resize(n);
    b->table_list.resize(n);
    b->table_nblist.resize(n);
    for (int q = 0; q < n; q++) {
        fi_model *m = shared[q];
        IbMember<T> &u = mem[q];
        std::memset(&u, 0, sizeof(u));
        u.g = m->g;
        u.p = member_kp(m);
        u.f[0] = m->ptrs<T>();
        u.f[1] = u.f[0];
        if (!m->kp.freeze_eta) std::swap(u.f[1].eta, u.f[1].eta_next);  // a frozen η keeps its buffer
        const bool list = use_list(m, u.p);
        off[q] = total;
        total += list ? m->n_blist : ib_grid_blocks(m->g, !b->f64);
        b->table_kp[q] = u.p;
        b->table_eta[q] = m->eta_swapped;
        b->table_list[q] = list;
        b->table_nblist[q] = m->n_blist;
        for (int d = 0; d < 3; d++) {
            BcMember &s = bc[(size_t)d * n + q], &v = bc[(size_t)(3 + d) * n + q], &w = bc[(size_t)(6 + d) * n + q];
            s.g = v.g = w.g = m->g;
            s.b = model_stress_batch(m, d);
            v.b = model_velocity_batch(m, d);
            bc_set_serial(m->g, s.b);
            bc_set_serial(m->g, v.b);
            // the same ops one iteration later, when η and η_next have traded buffers
            w.b = v.b;
            for (int o = 0; o < w.b.count; o++)
                if (w.b.ops[o].f == u.f[0].eta_next) w.b.ops[o].f = (void *)u.f[1].eta_next;
            const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
            b->max_a[d] = std::max(b->max_a[d], m->g.n[e1] + 3);
            b->max_c[d] = std::max(b->max_c[d], m->g.n[e2] + 3);
        }
    }
    if (total > (1LL << 31) - 1) return set_error("too many blocks for one shared launch"), FI_ERR_UNSUPPORTED;
    size_t cap_m = b->members_cap;
    FB_CHECK(regrow(reinterpret_cast<IbMember<T> **>(&b->d_members), (size_t)n, &cap_m), "batch table");
    b->members_cap = cap_m;
    size_t cap_i = (size_t)b->items_cap;
    FB_CHECK(regrow(&b->d_items, (size_t)total, &cap_i), "work items");
    b->items_cap = (long long)cap_i;
    size_t cap_b = (size_t)b->bc_cap;
    FB_CHECK(regrow(&b->d_bc, (size_t)9 * n, &cap_b), "boundary table");
    b->bc_cap = (int)cap_b;
    FB_CHECK(cudaMemcpyAsync(b->d_members, mem.data(), sizeof(IbMember<T>) * n, cudaMemcpyHostToDevice, b->stream),
             "batch table");
    // the boundary table is laid out [kind][member] with the member count as stride
    FB_CHECK(cudaMemcpyAsync(b->d_bc, bc.data(), sizeof(BcMember) * 9 * n, cudaMemcpyHostToDevice, b->stream),
             "boundary table");
    for (int q = 0; q < n; q++) {
        fi_model *m = shared[q];
        const bool list = b->table_list[q];
        FB_CHECK(launch_ib_items(m->g, !list, m->d_blist, m->n_blist, (unsigned)q, b->d_items + off[q], !b->f64,
                                 b->stream),
                 "work items");
    }
    FB_CHECK(cudaStreamSynchronize(b->stream), "batch table");
    b->nitems = (int)total;
    b->table_models = shared;
    b->epar = 0;
    drop_graphs(b);
    return FI_OK;
}

template <typename T>
cudaError_t enqueue_iteration(fi_ib_batch *b, int n, int epar) {
    const IbMember<T> *mem = reinterpret_cast<const IbMember<T> *>(b->d_members);
    cudaError_t e = launch_ib_batched<T>(mem, b->d_items, b->nitems, epar, false, b->stream);
    for (int d = 0; d < 3 && e == cudaSuccess; d++)
        e = launch_bc_batched<T>(b->d_bc + (size_t)d * n, n, b->max_a[d], b->max_c[d], b->stream);
    if (e == cudaSuccess) e = launch_ib_batched<T>(mem, b->d_items, b->nitems, epar, true, b->stream);
    for (int d = 0; d < 3 && e == cudaSuccess; d++)
        e = launch_bc_batched<T>(b->d_bc + (size_t)((epar ? 6 : 3) + d) * n, n, b->max_a[d], b->max_c[d], b->stream);
    return e;
}

template <typename T>
fi_status advance_shared(fi_ib_batch *b, const std::vector<fi_model *> &shared, int niter) {
    if (shared.empty() || niter <= 0) return FI_OK;
    if (!table_current(b, shared)) {
        fi_status st = build_table<T>(b, shared);
        if (st != FI_OK) return st;
    }
    const int n = (int)shared.size();
    int left = niter;
    if (left > 0 && b->epar == 1) {  // the graphs start a pair at parity 0
        FB_CHECK(enqueue_iteration<T>(b, n, 1), "shared iteration");
        b->epar = 0;
        left--;
    }
    if (left >= 2) {
        if (!b->graph[0]) {
            cudaGraph_t g = nullptr;
            FB_CHECK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
            cudaError_t ce = enqueue_iteration<T>(b, n, 0);
            if (ce == cudaSuccess) ce = enqueue_iteration<T>(b, n, 1);
            cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
            if (ce != cudaSuccess) return cuda_fail(ce, "graph capture");
            if (ee != cudaSuccess) return cuda_fail(ee, "graph capture");
            cudaError_t ie = cudaGraphInstantiate(&b->graph[0], g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return cuda_fail(ie, "graph instantiate");
        }
        for (; left >= 2; left -= 2) FB_CHECK(cudaGraphLaunch(b->graph[0], b->stream), "graph launch");
    }
    if (left == 1) {
        FB_CHECK(enqueue_iteration<T>(b, n, 0), "shared iteration");
        b->epar = 1;
    }
    for (fi_model *m : shared) {
        m->iterations += niter;
        if (!m->kp.freeze_eta && (niter & 1)) m->eta_swapped = !m->eta_swapped;
    }
    return FI_OK;
}

fi_status validate_ib_member(const fi_ib_batch *b, const fi_model *m) {
    if (!m) return set_error("null model in the batch"), FI_ERR_ARG;
    if (!m->ib || m->d.grid.nd != 3) return set_error("the shared launches take 3D immersed-boundary models"), FI_ERR_UNSUPPORTED;
    if (m->path == FI_PATH_FUSED) return set_error("immersed-boundary members run the reference-shaped path"), FI_ERR_UNSUPPORTED;
    if (m->split_begun >= 0) return set_error("a member has an overlapped iteration begun"), FI_ERR_STATE;
    if (!b->models.empty() && (m->is_f64() != b->f64 || m->d.device != b->device))
        return set_error("all members need one dtype and one device"), FI_ERR_ARG;
    for (const fi_model *o : b->models)
        if (o == m) return set_error("a model appears twice in the batch"), FI_ERR_ARG;
    return FI_OK;
}

}  // namespace

extern "C" {

fi_status fi_ib_batch_create(fi_model *const *models, int32_t count, fi_ib_batch **out) {
    if (!out || count < 0 || (count > 0 && !models)) return set_error("bad argument"), FI_ERR_ARG;
    *out = nullptr;
    fi_ib_batch *b = new fi_ib_batch();
    if (count > 0) {
        b->f64 = models[0] && models[0]->is_f64();
        b->device = models[0] ? models[0]->d.device : 0;
    }
    for (int q = 0; q < count; q++) {
        fi_status st = validate_ib_member(b, models[q]);
        if (st != FI_OK) {
            delete b;
            return st;
        }
        b->models.push_back(models[q]);
    }
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return cuda_fail(cudaGetLastError(), "batch stream");
    }
    *out = b;
    return FI_OK;
}

fi_status fi_ib_batch_destroy(fi_ib_batch *b) {
    if (!b) return FI_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    if (b->d_members) cudaFree(b->d_members);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_bc) cudaFree(b->d_bc);
    if (b->done) cudaEventDestroy(b->done);
    for (cudaEvent_t e : b->member_ev)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return FI_OK;
}

fi_status fi_ib_batch_add(fi_ib_batch *b, fi_model *m) {
    if (!b) return set_error("null batch"), FI_ERR_ARG;
    if (b->models.empty() && m) {
        b->f64 = m->is_f64();
        if (m->d.device != b->device) return set_error("the batch was created on another device"), FI_ERR_ARG;
    }
    fi_status st = validate_ib_member(b, m);
    if (st != FI_OK) return st;
    b->models.push_back(m);
    return FI_OK;
}

fi_status fi_ib_batch_remove(fi_ib_batch *b, fi_model *m) {
    if (!b || !m) return set_error("bad argument"), FI_ERR_ARG;
    auto it = std::find(b->models.begin(), b->models.end(), m);
    if (it == b->models.end()) return set_error("not a member of the batch"), FI_ERR_ARG;
    FB_CHECK(cudaSetDevice(b->device), "cudaSetDevice");
    FB_CHECK(cudaStreamSynchronize(b->stream), "batch sync");
    b->models.erase(it);
    // the table names members by address: a model created later at the same address
    // must not find the old entry current
    b->table_models.clear();
    drop_graphs(b);
    return FI_OK;
}

int32_t fi_ib_batch_size(const fi_ib_batch *b) { return b ? (int32_t)b->models.size() : 0; }

fi_status fi_ib_batch_advance(fi_ib_batch *b, int32_t niter) {
    if (!b || niter < 0) return set_error("bad argument"), FI_ERR_ARG;
    if (b->models.empty() || niter == 0) return FI_OK;
    FB_CHECK(cudaSetDevice(b->device), "cudaSetDevice");
    std::vector<fi_model *> shared;
    fi_status st;
    for (fi_model *m : b->models) {
        if (m->split_begun >= 0) return set_error("a member has an overlapped iteration begun"), FI_ERR_STATE;
        if (runs_alone(m) || too_big_to_share(m, !b->f64)) {
            // its first full iterations since the state changed, or a large member: as
            // fi_model_advance runs them, on the member's own stream
            if ((st = fi_model_advance(m, niter)) != FI_OK) return st;
            continue;
        }
        if (m->ibf_stale) {  // activity bytes and block list (a host round trip)
            FB_CHECK(cudaStreamSynchronize(m->stream), "member stream");
            if ((st = model_refresh_ibf(m)) != FI_OK) return st;
            FB_CHECK(cudaStreamSynchronize(m->stream), "member stream");
            if (too_big_to_share(m, !b->f64)) {
                if ((st = fi_model_advance(m, niter)) != FI_OK) return st;
                continue;
            }
        }
        shared.push_back(m);
    }
    if (shared.size() == 1) {  // nothing to share: the single-model kernels
        if ((st = fi_model_advance(shared[0], niter)) != FI_OK) return st;
        shared.clear();
    }
    // the shared launches wait for what the members' own streams hold (their earlier
    // iterations alone, a set_field)
    if (b->member_ev.size() < shared.size()) {
        const size_t old = b->member_ev.size();
        b->member_ev.resize(shared.size(), nullptr);
        for (size_t q = old; q < shared.size(); q++)
            FB_CHECK(cudaEventCreateWithFlags(&b->member_ev[q], cudaEventDisableTiming), "event");
    }
    for (size_t q = 0; q < shared.size(); q++) {
        FB_CHECK(cudaEventRecord(b->member_ev[q], shared[q]->stream), "event");
        FB_CHECK(cudaStreamWaitEvent(b->stream, b->member_ev[q], 0), "batch stream");
    }
    st = b->f64 ? advance_shared<double>(b, shared, niter) : advance_shared<float>(b, shared, niter);
    if (st != FI_OK) return st;
    if (!shared.empty()) {
        // the members' own streams wait for the shared launches
        FB_CHECK(cudaEventRecord(b->done, b->stream), "event");
        for (fi_model *m : shared) FB_CHECK(cudaStreamWaitEvent(m->stream, b->done, 0), "member stream");
    }
    return FI_OK;
}

fi_status fi_ib_batch_synchronize(fi_ib_batch *b) {
    if (!b) return set_error("null batch"), FI_ERR_ARG;
    FB_CHECK(cudaSetDevice(b->device), "cudaSetDevice");
    FB_CHECK(cudaStreamSynchronize(b->stream), "batch sync");
    for (fi_model *m : b->models) FB_CHECK(cudaStreamSynchronize(m->stream), "member stream");
    return FI_OK;
}

}  // extern "C"
