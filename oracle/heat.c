/*
 * heat.c -- CPU oracle for the pseudo-transient heat-diffusion model
 * (src/Models/Diffusion/Heat/{kernels.jl,boundary_conditions.jl,Heat.jl}).
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the library's heat sweep.  Only
 * tests/ load it; the product never links or calls it.
 *
 * Parity status: UNPINNED.  The reference model does not run as written
 * (Heat.jl:35,43 call `KernelLaunch(...)`, a module, read `model.fields`, which
 * does not exist, and pass `grid` where kernels.jl:3 expects the spacing `Δ`);
 * no reference test or golden output exists.  This restates its evident intent,
 * operation by operation, and is anchored by the steady-state test (a linear
 * profile between two Value sides):
 *   update_q! (kernels.jl:3-17), every index of the vertex range where q_d has
 *     storage (q_d Vertex along d, Center otherwise):
 *       q_d[I] -= (q_d[I] + λ_ρCp * (T[I] - T[I - e_d]) / Δ_d) * Δτ_q
 *   Flux(v) sides (boundary_conditions.jl:17-19, DirichletBC{FullCell}): the
 *     boundary node of q_d = v;
 *   update_T! (kernels.jl:19-29), every cell:
 *       ∇q = (q_x[I+e_x]-q_x[I])/Δx + (q_y[I+e_y]-q_y[I])/Δy + (q_z[I+e_z]-q_z[I])/Δz
 *       T[I] -= ((T[I] - T_o[I]) / Δt + ∇q) * Δτ_T
 *   Value(v) sides (boundary_conditions.jl:10-15, DirichletBC{HalfCell}): the
 *     ghost of T = 2v - T[adjacent cell].
 * Storage: the uniform halo box of the Stokes oracle ((n0+3)(n1+3)(n2+3), x
 * fastest, index 0 = ghost); faces of dim d span the full storage range of the
 * dims before d and the interior of the dims after d; dims x, y, z in order,
 * low side then high side.
 */
#include <stddef.h>

enum { FO_HEAT_VALUE = 0, FO_HEAT_FLUX = 1 };

typedef struct {
    int n[3];
    double dx[3];
    int kind[3][2];     /* FO_HEAT_VALUE / FO_HEAT_FLUX per (dim, side) */
    double value[3][2];
    double lam;         /* λ / (ρ Cp) */
    double dtau_T, dtau_q, dt;
} fo_heat;

#define HEAT_DEF(REAL, SUF)                                                                                         \
    static size_t heat_idx##SUF(const fo_heat *h, int i, int j, int k) {                                            \
        return (size_t)i + (size_t)(h->n[0] + 3) * ((size_t)j + (size_t)(h->n[1] + 3) * (size_t)k);                \
    }                                                                                                               \
    /* set f on the face of dim d, side s: at index `at` along d (Vertex: the node,                                  \
       Center: the ghost, from the adjacent cell) */                                                                 \
    static void heat_face##SUF(const fo_heat *h, REAL *f, int d, int s, int vertex, REAL v) {                        \
        int lo[3], hi[3];                                                                                           \
        for (int e = 0; e < 3; e++) {                                                                               \
            const int nv = h->n[e] + ((vertex && e == d) ? 1 : 0);                                                   \
            if (e < d) { lo[e] = 0; hi[e] = h->n[e] + 2; }                                                          \
            else { lo[e] = 1; hi[e] = nv; }                                                                          \
        }                                                                                                           \
        const int at = vertex ? (s == 0 ? 1 : h->n[d] + 1) : (s == 0 ? 0 : h->n[d] + 1);                            \
        const int adj = s == 0 ? 1 : h->n[d];                                                                       \
        lo[d] = hi[d] = at;                                                                                         \
        for (int k = lo[2]; k <= hi[2]; k++)                                                                        \
            for (int j = lo[1]; j <= hi[1]; j++)                                                                    \
                for (int i = lo[0]; i <= hi[0]; i++) {                                                              \
                    const size_t I = heat_idx##SUF(h, i, j, k);                                                     \
                    if (vertex) {                                                                                   \
                        f[I] = v;                                                                                   \
                    } else {                                                                                        \
                        int a[3] = {i, j, k};                                                                       \
                        a[d] = adj;                                                                                 \
                        f[I] = (REAL)2.0 * v - f[heat_idx##SUF(h, a[0], a[1], a[2])];                               \
                    }                                                                                               \
                }                                                                                                   \
    }                                                                                                               \
    void fo_heat_bc_flux##SUF(const fo_heat *h, REAL *qx, REAL *qy, REAL *qz) {                                      \
        REAL *q[3] = {qx, qy, qz};                                                                                  \
        for (int d = 0; d < 3; d++)                                                                                 \
            for (int s = 0; s < 2; s++)                                                                             \
                if (h->kind[d][s] == FO_HEAT_FLUX) heat_face##SUF(h, q[d], d, s, 1, (REAL)h->value[d][s]);          \
    }                                                                                                               \
    void fo_heat_bc_value##SUF(const fo_heat *h, REAL *T) {                                                          \
        for (int d = 0; d < 3; d++)                                                                                 \
            for (int s = 0; s < 2; s++)                                                                             \
                if (h->kind[d][s] == FO_HEAT_VALUE) heat_face##SUF(h, T, d, s, 0, (REAL)h->value[d][s]);            \
    }                                                                                                               \
    void fo_heat_advance##SUF(const fo_heat *h, REAL *T, const REAL *To, REAL *qx, REAL *qy, REAL *qz, int niter) {  \
        const REAL lam = (REAL)h->lam, dtq = (REAL)h->dtau_q, dtT = (REAL)h->dtau_T, dt = (REAL)h->dt;              \
        const REAL D[3] = {(REAL)h->dx[0], (REAL)h->dx[1], (REAL)h->dx[2]};                                         \
        REAL *q[3] = {qx, qy, qz};                                                                                  \
        const size_t st[3] = {1, (size_t)(h->n[0] + 3), (size_t)(h->n[0] + 3) * (size_t)(h->n[1] + 3)};              \
        for (int it = 0; it < niter; it++) {                                                                        \
            for (int d = 0; d < 3; d++)                                                                             \
                for (int k = 1; k <= h->n[2] + (d == 2); k++)                                                       \
                    for (int j = 1; j <= h->n[1] + (d == 1); j++)                                                   \
                        for (int i = 1; i <= h->n[0] + (d == 0); i++) {                                             \
                            const size_t I = heat_idx##SUF(h, i, j, k);                                             \
                            const REAL dT = lam * (T[I] - T[I - st[d]]) / D[d];                                     \
                            q[d][I] -= (q[d][I] + dT) * dtq;                                                        \
                        }                                                                                           \
            fo_heat_bc_flux##SUF(h, qx, qy, qz);                                                                    \
            for (int k = 1; k <= h->n[2]; k++)                                                                      \
                for (int j = 1; j <= h->n[1]; j++)                                                                  \
                    for (int i = 1; i <= h->n[0]; i++) {                                                            \
                        const size_t I = heat_idx##SUF(h, i, j, k);                                                 \
                        const REAL gq = (qx[I + st[0]] - qx[I]) / D[0] + (qy[I + st[1]] - qy[I]) / D[1] +           \
                                        (qz[I + st[2]] - qz[I]) / D[2];                                             \
                        T[I] -= ((T[I] - To[I]) / dt + gq) * dtT;                                                   \
                    }                                                                                               \
            fo_heat_bc_value##SUF(h, T);                                                                            \
        }                                                                                                           \
    }

HEAT_DEF(double, _f64)
HEAT_DEF(float, _f32)
