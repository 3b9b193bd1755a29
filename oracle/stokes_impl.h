/*
 * stokes_impl.h -- oracle body, instantiated for REAL=double (SUF=_f64) and
 * REAL=float (SUF=_f32).  TEST INFRASTRUCTURE ONLY (see fi_oracle.h).
 *
 * Each function restates one reference kernel, line by line, in Julia's
 * evaluation order (left-to-right products and sums, x^2 as x*x, /3.0 as a true
 * division).  Build with -ffp-contract=off so no fused multiply-add is formed.
 */
#include <math.h>
#include <string.h>
#include <stdlib.h>

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(name, SUF)

#define R(x) ((REAL)(x))

/* location flags: 0 = Center, 1 = Vertex */
static const int F(L_CCC)[3] = {0, 0, 0};
static const int F(L_VVC)[3] = {1, 1, 0};
static const int F(L_VCV)[3] = {1, 0, 1};
static const int F(L_CVV)[3] = {0, 1, 1};
static const int F(L_VCC)[3] = {1, 0, 0};
static const int F(L_CVC)[3] = {0, 1, 0};
static const int F(L_CCV)[3] = {0, 0, 1};

typedef struct {
    size_t sx, sy, sxy;
    int n0, n1, n2;
    int nd;
} F(geom);

static F(geom) F(mkgeom)(const fo_params *p) {
    F(geom) g;
    g.nd = p->nd;
    g.n0 = p->n[0];
    g.n1 = p->n[1];
    g.n2 = p->nd == 3 ? p->n[2] : 0;
    g.sx = (size_t)(p->n[0] + 3);
    g.sy = (size_t)(p->n[1] + 3);
    g.sxy = g.sx * g.sy;
    return g;
}

/* ------------------------------------------------------------------------- */
/* rheology: src/Physics.jl:11 (linear), :18 (power law), :26 (viscoplastic    */
/* regularisation), :46-47 (relaxation, lin/log/log10 scale)                   */
/* ------------------------------------------------------------------------- */
static REAL F(ipow)(REAL x, int m) {
    /* Julia ^(x, n::Int): n==2 -> x*x (compensated, equal to the rounded square),
     * n==3 -> x*x*x */
    if (m == 0) return R(1.0);
    if (m == 1) return x;
    if (m == 2) return x * x;
    if (m == 3) return x * x * x;
    if (m < 0) return R(1.0) / F(ipow)(x, -m);
    return (REAL)pow((double)x, (double)m);
}

static REAL F(rheology)(const fo_params *p, const fo_fields *f, size_t I, REAL tII) {
    REAL inner;
    if (p->rheo_inner == FO_RHEO_LINEAR) {
        inner = f->eta_lin ? ((const REAL *)f->eta_lin)[I] : R(p->rheo_eta_val);
    } else {
        REAL A = f->A_field ? ((const REAL *)f->A_field)[I] : R(p->rheo_A);
        inner = R(0.5) / (A * F(ipow)(tII, p->rheo_n - 1));
    }
    if (p->rheo_has_reg) inner = R(1.0) / (R(1.0) / inner + R(p->rheo_inv_eta_reg));
    if (p->rheo_relax != FO_RELAX_NONE) {
        REAL fld = ((const REAL *)f->eta)[I];
        REAL a = R(1.0 - p->rheo_rate), b = R(p->rheo_rate);
        if (p->rheo_relax == FO_RELAX_LIN) {
            inner = fld * a + inner * b;
        } else if (p->rheo_relax == FO_RELAX_LOG) {
            inner = (REAL)exp((double)((REAL)log((double)fld) * a + (REAL)log((double)inner) * b));
        } else {
            inner = (REAL)pow(10.0, (double)((REAL)log10((double)fld) * a + (REAL)log10((double)inner) * b));
        }
    }
    return inner;
}

static REAL F(gval)(const fo_params *p, const void *arr, int c, size_t I) {
    return p->g_kind[c] == FO_G_ARRAY ? ((const REAL *)arr)[I] : R(p->g_val[c]);
}

/* ------------------------------------------------------------------------- */
/* boundary conditions (adopted Chmy contract, see fi_oracle.h)                */
/* ------------------------------------------------------------------------- */
enum { F(OP_DIRICHLET) = 0, F(OP_NEUMANN) = 1, F(OP_PERIODIC) = 2 };

static void F(face_apply)(const F(geom) *g, REAL *f, const int loc[3], int d, int side, int op, REAL v) {
    int nd = g->nd;
    int n[3] = {g->n0, g->n1, g->n2};
    size_t st[3] = {1, g->sx, g->sxy};
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int e = 0; e < nd; e++) {
        if (e == d) continue;
        if (e < d) { lo[e] = 0; hi[e] = n[e] + 2; }
        else { lo[e] = 1; hi[e] = n[e] + loc[e]; }
    }
    int N = n[d];
    size_t sd = st[d];
    for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
            for (int i = lo[0]; i <= hi[0]; i++) {
                int idx3[3] = {i, j, k};
                idx3[d] = 0;
                size_t B = (size_t)idx3[0] + g->sx * ((size_t)idx3[1] + g->sy * (size_t)idx3[2]);
#define A(q) f[B + (size_t)(q) * sd]
                if (op == F(OP_DIRICHLET)) {
                    REAL two_v = R(2.0) * v;
                    if (loc[d] == 0) {
                        if (side == 0) A(0) = two_v - A(1);
                        else A(N + 1) = two_v - A(N);
                    } else {
                        if (side == 0) A(1) = v;
                        else A(N + 1) = v;
                    }
                } else if (op == F(OP_NEUMANN)) {
                    if (loc[d] == 0) {
                        if (side == 0) A(0) = A(1);
                        else A(N + 1) = A(N);
                    } else {
                        if (side == 0) A(0) = A(2);
                        else A(N + 2) = A(N);
                    }
                } else { /* periodic: both sides at once */
                    if (loc[d] == 0) {
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

/* stress batch: src/Models/FullStokes/Isothermal/boundary_conditions.jl:26-100 */
void F(fo_bc_stress)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    REAL *P = (REAL *)fl->P, *txx = (REAL *)fl->txx, *tyy = (REAL *)fl->tyy, *tzz = (REAL *)fl->tzz;
    REAL *txy = (REAL *)fl->txy, *txz = (REAL *)fl->txz, *tyz = (REAL *)fl->tyz;
    int nd = p->nd;
    for (int d = 0; d < nd; d++) {
        for (int s = 0; s < 2; s++) {
            int kind = p->bc_kind[d][s];
            const double *c = p->bc_val[d][s];
            if (kind == FO_BC_PERIODIC) {
                if (s == 1) continue;
                if (nd == 3) {
                    F(face_apply)(&g, P, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, txx, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, tyy, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, tzz, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, txy, F(L_VVC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, txz, F(L_VCV), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, tyz, F(L_CVV), d, 0, F(OP_PERIODIC), 0);
                } else {
                    F(face_apply)(&g, P, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, txx, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, tyy, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                    F(face_apply)(&g, txy, F(L_VVC), d, 0, F(OP_PERIODIC), 0);
                }
                continue;
            }
            if (kind == FO_BC_VELOCITY) continue; /* :117 EmptyBatch */
            if (nd == 2) {
                /* :26-47 */
                if (kind == FO_BC_TRACTION) {
                    if (d == 0) {
                        F(face_apply)(&g, P, F(L_CCC), 0, s, F(OP_DIRICHLET), R(c[0]));
                        F(face_apply)(&g, txx, F(L_CCC), 0, s, F(OP_DIRICHLET), R(c[0]));
                        F(face_apply)(&g, txy, F(L_VVC), 0, s, F(OP_DIRICHLET), R(c[1]));
                    } else {
                        F(face_apply)(&g, P, F(L_CCC), 1, s, F(OP_DIRICHLET), R(c[1]));
                        F(face_apply)(&g, tyy, F(L_CCC), 1, s, F(OP_DIRICHLET), R(c[1]));
                        F(face_apply)(&g, txy, F(L_VVC), 1, s, F(OP_DIRICHLET), R(c[0]));
                    }
                } else { /* slip: tangential component c[3-D] (1-based) */
                    F(face_apply)(&g, txy, F(L_VVC), d, s, F(OP_DIRICHLET), R(c[1 - d]));
                }
                continue;
            }
            /* 3D, :51-100 */
            if (kind == FO_BC_TRACTION) {
                if (d == 0) {
                    F(face_apply)(&g, P, F(L_CCC), 0, s, F(OP_DIRICHLET), R(c[0]));
                    F(face_apply)(&g, txx, F(L_CCC), 0, s, F(OP_DIRICHLET), R(c[0]));
                    F(face_apply)(&g, txy, F(L_VVC), 0, s, F(OP_DIRICHLET), R(c[1]));
                    F(face_apply)(&g, txz, F(L_VCV), 0, s, F(OP_DIRICHLET), R(c[2]));
                } else if (d == 1) {
                    F(face_apply)(&g, P, F(L_CCC), 1, s, F(OP_DIRICHLET), R(c[1]));
                    F(face_apply)(&g, tyy, F(L_CCC), 1, s, F(OP_DIRICHLET), R(c[1]));
                    F(face_apply)(&g, txy, F(L_VVC), 1, s, F(OP_DIRICHLET), R(c[0]));
                    F(face_apply)(&g, tyz, F(L_CVV), 1, s, F(OP_DIRICHLET), R(c[2]));
                } else {
                    F(face_apply)(&g, P, F(L_CCC), 2, s, F(OP_DIRICHLET), R(c[2]));
                    F(face_apply)(&g, tzz, F(L_CCC), 2, s, F(OP_DIRICHLET), R(c[2]));
                    F(face_apply)(&g, txz, F(L_VCV), 2, s, F(OP_DIRICHLET), R(c[0]));
                    F(face_apply)(&g, tyz, F(L_CVV), 2, s, F(OP_DIRICHLET), R(c[1]));
                }
            } else { /* slip */
                if (d == 0) {
                    F(face_apply)(&g, txy, F(L_VVC), 0, s, F(OP_DIRICHLET), R(c[1]));
                    F(face_apply)(&g, txz, F(L_VCV), 0, s, F(OP_DIRICHLET), R(c[2]));
                } else if (d == 1) {
                    F(face_apply)(&g, txy, F(L_VVC), 1, s, F(OP_DIRICHLET), R(c[0]));
                    F(face_apply)(&g, tyz, F(L_CVV), 1, s, F(OP_DIRICHLET), R(c[2]));
                } else {
                    F(face_apply)(&g, txz, F(L_VCV), 2, s, F(OP_DIRICHLET), R(c[0]));
                    F(face_apply)(&g, tyz, F(L_CVV), 2, s, F(OP_DIRICHLET), R(c[1]));
                }
            }
        }
    }
}

/* velocity batch + eta_next Neumann: boundary_conditions.jl:104-115 and
 * Isothermal.jl:103-104 */
void F(fo_bc_velocity)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    REAL *V[3] = {(REAL *)fl->Vx, (REAL *)fl->Vy, (REAL *)fl->Vz};
    const int *LV[3] = {F(L_VCC), F(L_CVC), F(L_CCV)};
    REAL *en = (REAL *)fl->eta_next;
    int nd = p->nd;
    for (int d = 0; d < nd; d++) {
        for (int s = 0; s < 2; s++) {
            int kind = p->bc_kind[d][s];
            const double *c = p->bc_val[d][s];
            if (kind == FO_BC_PERIODIC) {
                if (s == 1) continue;
                for (int q = 0; q < nd; q++) F(face_apply)(&g, V[q], LV[q], d, 0, F(OP_PERIODIC), 0);
                F(face_apply)(&g, en, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
                continue;
            }
            if (kind == FO_BC_VELOCITY) {
                for (int q = 0; q < nd; q++) F(face_apply)(&g, V[q], LV[q], d, s, F(OP_DIRICHLET), R(c[q]));
            } else if (kind == FO_BC_SLIP) {
                F(face_apply)(&g, V[d], LV[d], d, s, F(OP_DIRICHLET), R(c[d]));
            }
            F(face_apply)(&g, en, F(L_CCC), d, s, F(OP_NEUMANN), 0);
        }
    }
}

/* Neumann (or periodic wrap) on a viscosity field, as drivers do after set!
 * (scripts_future_API/tm_stokes_chmy.jl:280-281) */
void F(fo_bc_eta)(const fo_params *p, REAL *eta) {
    F(geom) g = F(mkgeom)(p);
    for (int d = 0; d < p->nd; d++) {
        for (int s = 0; s < 2; s++) {
            if (p->bc_kind[d][s] == FO_BC_PERIODIC) {
                if (s == 0) F(face_apply)(&g, eta, F(L_CCC), d, 0, F(OP_PERIODIC), 0);
            } else {
                F(face_apply)(&g, eta, F(L_CCC), d, s, F(OP_NEUMANN), 0);
            }
        }
    }
}

/* residual batch: boundary_conditions.jl:120-128 (normal residual Dirichlet(0)
 * except on traction sides) */
static void F(bc_residual)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    REAL *r[3] = {(REAL *)fl->rVx, (REAL *)fl->rVy, (REAL *)fl->rVz};
    const int *LV[3] = {F(L_VCC), F(L_CVC), F(L_CCV)};
    for (int d = 0; d < p->nd; d++)
        for (int s = 0; s < 2; s++) {
            int kind = p->bc_kind[d][s];
            if (kind == FO_BC_TRACTION || kind == FO_BC_PERIODIC) continue;
            F(face_apply)(&g, r[d], LV[d], d, s, F(OP_DIRICHLET), R(0.0));
        }
}

/* ------------------------------------------------------------------------- */
/* FullStokes kernels                                                          */
/* ------------------------------------------------------------------------- */
#define LOOP3(g)                                  \
    for (int k = 1; k <= (g).n2 + 1; k++)         \
        for (int j = 1; j <= (g).n1 + 1; j++)     \
            for (int i = 1; i <= (g).n0 + 1; i++)
#define LOOP2(g)                              \
    for (int j = 1; j <= (g).n1 + 1; j++)     \
        for (int i = 1; i <= (g).n0 + 1; i++)

/* update_sigma!: kernels_3d.jl:3-25 and kernels_2d.jl:3-18 */
void F(fo_update_sigma)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    REAL *P = (REAL *)fl->P, *txx = (REAL *)fl->txx, *tyy = (REAL *)fl->tyy, *txy = (REAL *)fl->txy;
    const REAL *Vx = (const REAL *)fl->Vx, *Vy = (const REAL *)fl->Vy, *eta = (const REAL *)fl->eta;
    const REAL idx = R(p->inv_dx[0]), idy = R(p->inv_dx[1]);
    const REAL dtP = R(p->dt_P), dxx = R(p->dt_tau[0]), dyy = R(p->dt_tau[1]), dxy = R(p->dt_tau[3]);
    const size_t sx = g.sx, sxy = g.sxy;
    if (p->nd == 2) {
#pragma omp parallel for collapse(1) schedule(static)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j;
                REAL exx = (Vx[I + 1] - Vx[I]) * idx;
                REAL eyy = (Vy[I + sx] - Vy[I]) * idy;
                REAL exy = R(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
                REAL divV = exx + eyy;
                REAL etac = eta[I];
                P[I] = P[I] - divV * etac * dtP;
                txx[I] = txx[I] - (txx[I] - R(2.0) * etac * (exx - divV / R(3.0))) * dxx;
                tyy[I] = tyy[I] - (tyy[I] - R(2.0) * etac * (eyy - divV / R(3.0))) * dyy;
                REAL exy_eta = R(0.5) * (R(0.5) * (eta[I - 1 - sx] + eta[I - sx]) + R(0.5) * (eta[I - 1] + eta[I]));
                txy[I] = txy[I] - (txy[I] - R(2.0) * exy_eta * exy) * dxy;
            }
        return;
    }
    REAL *tzz = (REAL *)fl->tzz, *txz = (REAL *)fl->txz, *tyz = (REAL *)fl->tyz;
    const REAL *Vz = (const REAL *)fl->Vz;
    const REAL idz = R(p->inv_dx[2]);
    const REAL dzz = R(p->dt_tau[2]), dxz = R(p->dt_tau[4]), dyz = R(p->dt_tau[5]);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= g.n2 + 1; k++)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                REAL exx = (Vx[I + 1] - Vx[I]) * idx;
                REAL eyy = (Vy[I + sx] - Vy[I]) * idy;
                REAL ezz = (Vz[I + sxy] - Vz[I]) * idz;
                REAL exy = R(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
                REAL exz = R(0.5) * ((Vz[I] - Vz[I - 1]) * idx + (Vx[I] - Vx[I - sxy]) * idz);
                REAL eyz = R(0.5) * ((Vz[I] - Vz[I - sx]) * idy + (Vy[I] - Vy[I - sxy]) * idz);
                REAL divV = exx + eyy + ezz;
                REAL etac = eta[I];
                P[I] = P[I] - divV * etac * dtP;
                txx[I] = txx[I] - (txx[I] - R(2.0) * etac * (exx - divV / R(3.0))) * dxx;
                tyy[I] = tyy[I] - (tyy[I] - R(2.0) * etac * (eyy - divV / R(3.0))) * dyy;
                tzz[I] = tzz[I] - (tzz[I] - R(2.0) * etac * (ezz - divV / R(3.0))) * dzz;
                REAL e_xy = R(0.5) * (R(0.5) * (eta[I - 1 - sx] + eta[I - sx]) + R(0.5) * (eta[I - 1] + eta[I]));
                REAL e_xz = R(0.5) * (R(0.5) * (eta[I - 1 - sxy] + eta[I - sxy]) + R(0.5) * (eta[I - 1] + eta[I]));
                REAL e_yz = R(0.5) * (R(0.5) * (eta[I - sx - sxy] + eta[I - sxy]) + R(0.5) * (eta[I - sx] + eta[I]));
                txy[I] = txy[I] - (txy[I] - R(2.0) * e_xy * exy) * dxy;
                txz[I] = txz[I] - (txz[I] - R(2.0) * e_xz * exz) * dxz;
                tyz[I] = tyz[I] - (tyz[I] - R(2.0) * e_yz * eyz) * dyz;
            }
}

/* update_V!: kernels_3d.jl:27-40 and kernels_2d.jl:20-29.  The 2D reference
 * interpolates eta to location(V.x) for both components and omits the grid
 * argument (kernels_2d.jl:24-25); the evident intent, lerp to location(V.y) for
 * V.y, is restated here. */
void F(fo_update_V)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    const REAL *P = (const REAL *)fl->P, *txx = (const REAL *)fl->txx, *tyy = (const REAL *)fl->tyy;
    const REAL *txy = (const REAL *)fl->txy, *eta = (const REAL *)fl->eta;
    REAL *Vx = (REAL *)fl->Vx, *Vy = (REAL *)fl->Vy, *en = (REAL *)fl->eta_next;
    const REAL idx = R(p->inv_dx[0]), idy = R(p->inv_dx[1]);
    const REAL dVx = R(p->dt_V[0]), dVy = R(p->dt_V[1]);
    const size_t sx = g.sx, sxy = g.sxy;
    if (p->nd == 2) {
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j;
                REAL gx = F(gval)(p, fl->gx, 0, I), gy = F(gval)(p, fl->gy, 1, I);
                REAL ex = R(0.5) * (eta[I - 1] + eta[I]);
                REAL ey = R(0.5) * (eta[I - sx] + eta[I]);
                Vx[I] = Vx[I] + (-(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy - gx) / ex * dVx;
                Vy[I] = Vy[I] + (-(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx - gy) / ey * dVy;
                REAL lxy = R(0.5) * (R(0.5) * (txy[I] + txy[I + 1]) + R(0.5) * (txy[I + sx] + txy[I + sx + 1]));
                REAL tII = (REAL)sqrt((double)(R(0.5) * (txx[I] * txx[I] + tyy[I] * tyy[I]) + lxy * lxy));
                en[I] = F(rheology)(p, fl, I, tII);
            }
        return;
    }
    const REAL *tzz = (const REAL *)fl->tzz, *txz = (const REAL *)fl->txz, *tyz = (const REAL *)fl->tyz;
    REAL *Vz = (REAL *)fl->Vz;
    const REAL idz = R(p->inv_dx[2]), dVz = R(p->dt_V[2]);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= g.n2 + 1; k++)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                REAL gx = F(gval)(p, fl->gx, 0, I), gy = F(gval)(p, fl->gy, 1, I), gz = F(gval)(p, fl->gz, 2, I);
                REAL ex = R(0.5) * (eta[I - 1] + eta[I]);
                REAL ey = R(0.5) * (eta[I - sx] + eta[I]);
                REAL ez = R(0.5) * (eta[I - sxy] + eta[I]);
                Vx[I] = Vx[I] + (-(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy +
                                 (txz[I + sxy] - txz[I]) * idz - gx) / ex * dVx;
                Vy[I] = Vy[I] + (-(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx +
                                 (tyz[I + sxy] - tyz[I]) * idz - gy) / ey * dVy;
                Vz[I] = Vz[I] + (-(P[I] - P[I - sxy]) * idz + (tzz[I] - tzz[I - sxy]) * idz + (txz[I + 1] - txz[I]) * idx +
                                 (tyz[I + sx] - tyz[I]) * idy - gz) / ez * dVz;
                REAL lxy = R(0.5) * (R(0.5) * (txy[I] + txy[I + 1]) + R(0.5) * (txy[I + sx] + txy[I + sx + 1]));
                REAL lxz = R(0.5) * (R(0.5) * (txz[I] + txz[I + 1]) + R(0.5) * (txz[I + sxy] + txz[I + sxy + 1]));
                REAL lyz = R(0.5) * (R(0.5) * (tyz[I] + tyz[I + sx]) + R(0.5) * (tyz[I + sxy] + tyz[I + sxy + sx]));
                REAL s = R(0.5) * (txx[I] * txx[I] + tyy[I] * tyy[I] + tzz[I] * tzz[I]) + lxy * lxy + lxz * lxz + lyz * lyz;
                REAL tII = (REAL)sqrt((double)s);
                en[I] = F(rheology)(p, fl, I, tII);
            }
}

static void F(swap_eta)(fo_fields *fl) {
    void *t = fl->eta;
    fl->eta = fl->eta_next;
    fl->eta_next = t;
}

/* advance_iteration!: src/Models/FullStokes/Isothermal/Isothermal.jl:91-112 */
void F(fo_advance)(const fo_params *p, fo_fields *fl, int niter) {
    for (int it = 0; it < niter; it++) {
        F(fo_update_sigma)(p, fl);
        F(fo_bc_stress)(p, fl);
        F(fo_update_V)(p, fl);
        F(fo_bc_velocity)(p, fl);
        F(swap_eta)(fl);
    }
}

/* compute_residuals!: kernels_3d.jl:66-75, kernels_2d.jl:46-54, Isothermal.jl:114-125 */
void F(fo_compute_residuals)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    const REAL *P = (const REAL *)fl->P, *txx = (const REAL *)fl->txx, *tyy = (const REAL *)fl->tyy;
    const REAL *txy = (const REAL *)fl->txy, *Vx = (const REAL *)fl->Vx, *Vy = (const REAL *)fl->Vy;
    REAL *rP = (REAL *)fl->rP, *rVx = (REAL *)fl->rVx, *rVy = (REAL *)fl->rVy;
    const REAL idx = R(p->inv_dx[0]), idy = R(p->inv_dx[1]);
    const size_t sx = g.sx, sxy = g.sxy;
    if (p->nd == 2) {
#pragma omp parallel for schedule(static)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j;
                REAL gx = F(gval)(p, fl->gx, 0, I), gy = F(gval)(p, fl->gy, 1, I);
                rP[I] = (Vx[I + 1] - Vx[I]) * idx + (Vy[I + sx] - Vy[I]) * idy;
                rVx[I] = -(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy - gx;
                rVy[I] = -(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx - gy;
            }
    } else {
        const REAL *tzz = (const REAL *)fl->tzz, *txz = (const REAL *)fl->txz, *tyz = (const REAL *)fl->tyz;
        const REAL *Vz = (const REAL *)fl->Vz;
        REAL *rVz = (REAL *)fl->rVz;
        const REAL idz = R(p->inv_dx[2]);
#pragma omp parallel for schedule(static)
        for (int k = 1; k <= g.n2 + 1; k++)
            for (int j = 1; j <= g.n1 + 1; j++)
                for (int i = 1; i <= g.n0 + 1; i++) {
                    size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                    REAL gx = F(gval)(p, fl->gx, 0, I), gy = F(gval)(p, fl->gy, 1, I), gz = F(gval)(p, fl->gz, 2, I);
                    rP[I] = (Vx[I + 1] - Vx[I]) * idx + (Vy[I + sx] - Vy[I]) * idy + (Vz[I + sxy] - Vz[I]) * idz;
                    rVx[I] = -(P[I] - P[I - 1]) * idx + (txx[I] - txx[I - 1]) * idx + (txy[I + sx] - txy[I]) * idy +
                             (txz[I + sxy] - txz[I]) * idz - gx;
                    rVy[I] = -(P[I] - P[I - sx]) * idy + (tyy[I] - tyy[I - sx]) * idy + (txy[I + 1] - txy[I]) * idx +
                             (tyz[I + sxy] - tyz[I]) * idz - gy;
                    rVz[I] = -(P[I] - P[I - sxy]) * idz + (tzz[I] - tzz[I - sxy]) * idz + (txz[I + 1] - txz[I]) * idx +
                             (tyz[I + sx] - tyz[I]) * idy - gz;
                }
    }
    F(bc_residual)(p, fl);
}

/* Norms over each field's interior (scripts_future_API/tm_stokes_mpi_wip.jl:21-22
 * take norms of interior(A)). */
static void F(norms_from_arrays)(const fo_params *p, fo_fields *fl, double *out) {
    F(geom) g = F(mkgeom)(p);
    const REAL *arr[4] = {(const REAL *)fl->rP, (const REAL *)fl->rVx, (const REAL *)fl->rVy, (const REAL *)fl->rVz};
    const int *locs[4] = {F(L_CCC), F(L_VCC), F(L_CVC), F(L_CCV)};
    const REAL *V[3] = {(const REAL *)fl->Vx, (const REAL *)fl->Vy, (const REAL *)fl->Vz};
    int nf = p->nd == 3 ? 4 : 3;
    for (int q = 0; q < FO_NORMS_LEN; q++) out[q] = 0.0;
    for (int q = 0; q < nf; q++) {
        const int *L = locs[q];
        int hk = p->nd == 3 ? g.n2 + L[2] : 0, lk = p->nd == 3 ? 1 : 0;
        double mx = 0.0, ss = 0.0, vm = 0.0;
        for (int k = lk; k <= hk; k++)
            for (int j = 1; j <= g.n1 + L[1]; j++)
                for (int i = 1; i <= g.n0 + L[0]; i++) {
                    size_t I = (size_t)i + g.sx * (size_t)j + g.sxy * (size_t)k;
                    double r = (double)arr[q][I];
                    double a = fabs(r);
                    if (!(a <= mx)) mx = a; /* propagates NaN */
                    ss += r * r;
                    if (q > 0) {
                        double v = fabs((double)V[q - 1][I]);
                        if (!(v <= vm)) vm = v;
                    }
                }
        out[q] = mx;
        out[4 + q] = sqrt(ss);
        if (q > 0) out[8 + q - 1] = vm;
    }
}

void F(fo_residual_norms)(const fo_params *p, fo_fields *fl, double *out) {
    F(fo_compute_residuals)(p, fl);
    F(norms_from_arrays)(p, fl, out);
}

/* compute_tau!: kernels_3d.jl:44-64, kernels_2d.jl:33-44 */
void F(fo_compute_tau)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    REAL *txx = (REAL *)fl->txx, *tyy = (REAL *)fl->tyy, *txy = (REAL *)fl->txy;
    const REAL *Vx = (const REAL *)fl->Vx, *Vy = (const REAL *)fl->Vy, *eta = (const REAL *)fl->eta;
    const REAL idx = R(p->inv_dx[0]), idy = R(p->inv_dx[1]);
    const size_t sx = g.sx, sxy = g.sxy;
    if (p->nd == 2) {
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j;
                REAL exx = (Vx[I + 1] - Vx[I]) * idx;
                REAL eyy = (Vy[I + sx] - Vy[I]) * idy;
                REAL exy = R(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
                REAL divV = exx + eyy;
                txx[I] = R(2.0) * eta[I] * (exx - divV / R(3.0));
                tyy[I] = R(2.0) * eta[I] * (eyy - divV / R(3.0));
                REAL e_xy = R(0.5) * (R(0.5) * (eta[I - 1 - sx] + eta[I - sx]) + R(0.5) * (eta[I - 1] + eta[I]));
                txy[I] = R(2.0) * e_xy * exy;
            }
        return;
    }
    REAL *tzz = (REAL *)fl->tzz, *txz = (REAL *)fl->txz, *tyz = (REAL *)fl->tyz;
    const REAL *Vz = (const REAL *)fl->Vz;
    const REAL idz = R(p->inv_dx[2]);
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= g.n2 + 1; k++)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                REAL exx = (Vx[I + 1] - Vx[I]) * idx;
                REAL eyy = (Vy[I + sx] - Vy[I]) * idy;
                REAL ezz = (Vz[I + sxy] - Vz[I]) * idz;
                REAL exy = R(0.5) * ((Vy[I] - Vy[I - 1]) * idx + (Vx[I] - Vx[I - sx]) * idy);
                REAL exz = R(0.5) * ((Vz[I] - Vz[I - 1]) * idx + (Vx[I] - Vx[I - sxy]) * idz);
                REAL eyz = R(0.5) * ((Vz[I] - Vz[I - sx]) * idy + (Vy[I] - Vy[I - sxy]) * idz);
                REAL divV = exx + eyy + ezz;
                txx[I] = R(2.0) * eta[I] * (exx - divV / R(3.0));
                tyy[I] = R(2.0) * eta[I] * (eyy - divV / R(3.0));
                tzz[I] = R(2.0) * eta[I] * (ezz - divV / R(3.0));
                REAL e_xy = R(0.5) * (R(0.5) * (eta[I - 1 - sx] + eta[I - sx]) + R(0.5) * (eta[I - 1] + eta[I]));
                REAL e_xz = R(0.5) * (R(0.5) * (eta[I - 1 - sxy] + eta[I - sxy]) + R(0.5) * (eta[I - 1] + eta[I]));
                REAL e_yz = R(0.5) * (R(0.5) * (eta[I - sx - sxy] + eta[I - sxy]) + R(0.5) * (eta[I - sx] + eta[I]));
                txy[I] = R(2.0) * e_xy * exy;
                txz[I] = R(2.0) * e_xz * exz;
                tyz[I] = R(2.0) * e_yz * eyz;
            }
}

/* ------------------------------------------------------------------------- */
/* Immersed-boundary FullStokes (3D):                                          */
/* src/Models/ImmersedBoundaryFullStokes/Isothermal/kernels_3d.jl and          */
/* null_spaces.jl.  Mask components: 0 ccc 1 vvv 2 vcc 3 cvc 4 ccv 5 vvc 6 vcv  */
/* 7 cvv.  Threshold 1e-6 is compared in double (Julia promotes Float32).      */
/* ------------------------------------------------------------------------- */
#define W_CCC 0
#define W_VVV 1
#define W_VCC 2
#define W_CVC 3
#define W_CCV 4
#define W_VVC 5
#define W_VCV 6
#define W_CVV 7

#define SMALL(w) ((double)(w) < 1e-6)

/* isnullspace: null_spaces.jl:13-37; left/right: :3-11 */
static int F(nullspace)(const REAL *const w[8], int comp, size_t I, size_t sx, size_t sxy) {
    switch (comp) {
    case W_CCC: /* generic, all dims: flipped comps vcc/cvc/ccv at i, i+1 */
        return SMALL(w[W_VCC][I]) || SMALL(w[W_VCC][I + 1]) || SMALL(w[W_CVC][I]) || SMALL(w[W_CVC][I + sx]) ||
               SMALL(w[W_CCV][I]) || SMALL(w[W_CCV][I + sxy]);
    case W_VCC: /* x: ccc at i-1,i; y: vvc at j,j+1; z: vcv at k,k+1 */
        return SMALL(w[W_CCC][I - 1]) || SMALL(w[W_CCC][I]) || SMALL(w[W_VVC][I]) || SMALL(w[W_VVC][I + sx]) ||
               SMALL(w[W_VCV][I]) || SMALL(w[W_VCV][I + sxy]);
    case W_CVC:
        return SMALL(w[W_VVC][I]) || SMALL(w[W_VVC][I + 1]) || SMALL(w[W_CCC][I - sx]) || SMALL(w[W_CCC][I]) ||
               SMALL(w[W_CVV][I]) || SMALL(w[W_CVV][I + sxy]);
    case W_CCV:
        return SMALL(w[W_VCV][I]) || SMALL(w[W_VCV][I + 1]) || SMALL(w[W_CVV][I]) || SMALL(w[W_CVV][I + sx]) ||
               SMALL(w[W_CCC][I - sxy]) || SMALL(w[W_CCC][I]);
    case W_VVC: /* :24-27, dims x and y only */
        return SMALL(w[W_CVC][I - 1]) || SMALL(w[W_CVC][I]) || SMALL(w[W_VCC][I - sx]) || SMALL(w[W_VCC][I]);
    case W_VCV: /* :29-32, dims x and z */
        return SMALL(w[W_CCV][I - 1]) || SMALL(w[W_CCV][I]) || SMALL(w[W_VCC][I - sxy]) || SMALL(w[W_VCC][I]);
    case W_CVV: /* :34-37, dims y and z */
        return SMALL(w[W_CCV][I - sx]) || SMALL(w[W_CCV][I]) || SMALL(w[W_CVC][I - sxy]) || SMALL(w[W_CVC][I]);
    default:
        return 0;
    }
}

/* isvalid(a, loc, I) && !isempty(b, loc, I): kernels_3d.jl:6,26,32,38,50,56,62 */
static int F(active)(const REAL *const a[8], const REAL *const b[8], int comp, size_t I, size_t sx, size_t sxy) {
    int valid = !(F(nullspace)(a, comp, I, sx, sxy) || SMALL(a[comp][I]));
    return valid && !SMALL(b[comp][I]);
}

/* IB update_sigma!: kernels_3d.jl:3-44 */
void F(fo_ib_update_sigma)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    REAL *P = (REAL *)fl->P, *txx = (REAL *)fl->txx, *tyy = (REAL *)fl->tyy, *tzz = (REAL *)fl->tzz;
    REAL *txy = (REAL *)fl->txy, *txz = (REAL *)fl->txz, *tyz = (REAL *)fl->tyz;
    const REAL *Vx = (const REAL *)fl->Vx, *Vy = (const REAL *)fl->Vy, *Vz = (const REAL *)fl->Vz;
    const REAL *eta = (const REAL *)fl->eta;
    const REAL *const *na = (const REAL *const *)fl->wna, *const *ns = (const REAL *const *)fl->wns;
    const REAL idx = R(p->inv_dx[0]), idy = R(p->inv_dx[1]), idz = R(p->inv_dx[2]);
    const REAL dtP = R(p->dt_P), dxx = R(p->dt_tau[0]), dyy = R(p->dt_tau[1]), dzz = R(p->dt_tau[2]);
    const REAL dxy = R(p->dt_tau[3]), dxz = R(p->dt_tau[4]), dyz = R(p->dt_tau[5]);
    const size_t sx = g.sx, sxy = g.sxy;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= g.n2 + 1; k++)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                if (F(active)(na, ns, W_CCC, I, sx, sxy)) {
                    REAL exx = (ns[W_VCC][I + 1] * Vx[I + 1] - ns[W_VCC][I] * Vx[I]) * idx;
                    REAL eyy = (ns[W_CVC][I + sx] * Vy[I + sx] - ns[W_CVC][I] * Vy[I]) * idy;
                    REAL ezz = (ns[W_CCV][I + sxy] * Vz[I + sxy] - ns[W_CCV][I] * Vz[I]) * idz;
                    REAL divV = exx + eyy + ezz;
                    REAL etac = eta[I];
                    P[I] = P[I] - divV * etac * dtP;
                    txx[I] = txx[I] - (txx[I] - R(2.0) * etac * (exx - divV / R(3.0))) * dxx;
                    tyy[I] = tyy[I] - (tyy[I] - R(2.0) * etac * (eyy - divV / R(3.0))) * dyy;
                    tzz[I] = tzz[I] - (tzz[I] - R(2.0) * etac * (ezz - divV / R(3.0))) * dzz;
                } else {
                    P[I] = R(0.0);
                    txx[I] = R(0.0);
                    tyy[I] = R(0.0);
                    tzz[I] = R(0.0);
                }
                if (F(active)(na, ns, W_VVC, I, sx, sxy)) {
                    REAL exy = R(0.5) * ((ns[W_CVC][I] * Vy[I] - ns[W_CVC][I - 1] * Vy[I - 1]) * idx +
                                         (ns[W_VCC][I] * Vx[I] - ns[W_VCC][I - sx] * Vx[I - sx]) * idy);
                    REAL e_xy = R(0.5) * (R(0.5) * (eta[I - 1 - sx] + eta[I - sx]) + R(0.5) * (eta[I - 1] + eta[I]));
                    txy[I] = txy[I] - (txy[I] - R(2.0) * e_xy * exy) * dxy;
                } else {
                    txy[I] = R(0.0);
                }
                if (F(active)(na, ns, W_VCV, I, sx, sxy)) {
                    REAL exz = R(0.5) * ((ns[W_CCV][I] * Vz[I] - ns[W_CCV][I - 1] * Vz[I - 1]) * idx +
                                         (ns[W_VCC][I] * Vx[I] - ns[W_VCC][I - sxy] * Vx[I - sxy]) * idz);
                    REAL e_xz = R(0.5) * (R(0.5) * (eta[I - 1 - sxy] + eta[I - sxy]) + R(0.5) * (eta[I - 1] + eta[I]));
                    txz[I] = txz[I] - (txz[I] - R(2.0) * e_xz * exz) * dxz;
                } else {
                    txz[I] = R(0.0);
                }
                if (F(active)(na, ns, W_CVV, I, sx, sxy)) {
                    REAL eyz = R(0.5) * ((ns[W_CCV][I] * Vz[I] - ns[W_CCV][I - sx] * Vz[I - sx]) * idy +
                                         (ns[W_CVC][I] * Vy[I] - ns[W_CVC][I - sxy] * Vy[I - sxy]) * idz);
                    REAL e_yz = R(0.5) * (R(0.5) * (eta[I - sx - sxy] + eta[I - sxy]) + R(0.5) * (eta[I - sx] + eta[I]));
                    tyz[I] = tyz[I] - (tyz[I] - R(2.0) * e_yz * eyz) * dyz;
                } else {
                    tyz[I] = R(0.0);
                }
            }
}

/* IB update_V!: kernels_3d.jl:46-74 */
void F(fo_ib_update_V)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    const REAL *P = (const REAL *)fl->P, *txx = (const REAL *)fl->txx, *tyy = (const REAL *)fl->tyy;
    const REAL *tzz = (const REAL *)fl->tzz, *txy = (const REAL *)fl->txy, *txz = (const REAL *)fl->txz;
    const REAL *tyz = (const REAL *)fl->tyz, *eta = (const REAL *)fl->eta;
    REAL *Vx = (REAL *)fl->Vx, *Vy = (REAL *)fl->Vy, *Vz = (REAL *)fl->Vz, *en = (REAL *)fl->eta_next;
    const REAL *const *na = (const REAL *const *)fl->wna, *const *ns = (const REAL *const *)fl->wns;
    const REAL idx = R(p->inv_dx[0]), idy = R(p->inv_dx[1]), idz = R(p->inv_dx[2]);
    const REAL dVx = R(p->dt_V[0]), dVy = R(p->dt_V[1]), dVz = R(p->dt_V[2]);
    const size_t sx = g.sx, sxy = g.sxy;
    const REAL *wc = na[W_CCC], *wvvc = na[W_VVC], *wvcv = na[W_VCV], *wcvv = na[W_CVV];
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= g.n2 + 1; k++)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                REAL gx = F(gval)(p, fl->gx, 0, I), gy = F(gval)(p, fl->gy, 1, I), gz = F(gval)(p, fl->gz, 2, I);
                if (F(active)(ns, na, W_VCC, I, sx, sxy)) {
                    REAL ex = R(0.5) * (eta[I - 1] + eta[I]);
                    Vx[I] = Vx[I] + (-(wc[I] * P[I] - wc[I - 1] * P[I - 1]) * idx + (wc[I] * txx[I] - wc[I - 1] * txx[I - 1]) * idx +
                                     (wvvc[I + sx] * txy[I + sx] - wvvc[I] * txy[I]) * idy +
                                     (wvcv[I + sxy] * txz[I + sxy] - wvcv[I] * txz[I]) * idz - gx) /
                                        ex / ns[W_VCC][I] * dVx;
                } else {
                    Vx[I] = R(0.0);
                }
                if (F(active)(ns, na, W_CVC, I, sx, sxy)) {
                    REAL ey = R(0.5) * (eta[I - sx] + eta[I]);
                    Vy[I] = Vy[I] + (-(wc[I] * P[I] - wc[I - sx] * P[I - sx]) * idy + (wc[I] * tyy[I] - wc[I - sx] * tyy[I - sx]) * idy +
                                     (wvvc[I + 1] * txy[I + 1] - wvvc[I] * txy[I]) * idx +
                                     (wcvv[I + sxy] * tyz[I + sxy] - wcvv[I] * tyz[I]) * idz - gy) /
                                        ey / ns[W_CVC][I] * dVy;
                } else {
                    Vy[I] = R(0.0);
                }
                if (F(active)(ns, na, W_CCV, I, sx, sxy)) {
                    REAL ez = R(0.5) * (eta[I - sxy] + eta[I]);
                    Vz[I] = Vz[I] + (-(wc[I] * P[I] - wc[I - sxy] * P[I - sxy]) * idz + (wc[I] * tzz[I] - wc[I - sxy] * tzz[I - sxy]) * idz +
                                     (wvcv[I + 1] * txz[I + 1] - wvcv[I] * txz[I]) * idx +
                                     (wcvv[I + sx] * tyz[I + sx] - wcvv[I] * tyz[I]) * idy - gz) /
                                        ez / ns[W_CCV][I] * dVz;
                } else {
                    Vz[I] = R(0.0);
                }
                REAL lxy = R(0.5) * (R(0.5) * (txy[I] + txy[I + 1]) + R(0.5) * (txy[I + sx] + txy[I + sx + 1]));
                REAL lxz = R(0.5) * (R(0.5) * (txz[I] + txz[I + 1]) + R(0.5) * (txz[I + sxy] + txz[I + sxy + 1]));
                REAL lyz = R(0.5) * (R(0.5) * (tyz[I] + tyz[I + sx]) + R(0.5) * (tyz[I + sxy] + tyz[I + sxy + sx]));
                REAL s = R(0.5) * (txx[I] * txx[I] + tyy[I] * tyy[I] + tzz[I] * tzz[I]) + lxy * lxy + lxz * lxz + lyz * lyz;
                REAL tII = (REAL)sqrt((double)s);
                en[I] = F(rheology)(p, fl, I, tII);
            }
}

/* IB advance_iteration!: ImmersedBoundaryFullStokes/Isothermal/Isothermal.jl:100-122 */
void F(fo_ib_advance)(const fo_params *p, fo_fields *fl, int niter) {
    for (int it = 0; it < niter; it++) {
        F(fo_ib_update_sigma)(p, fl);
        F(fo_bc_stress)(p, fl);
        F(fo_ib_update_V)(p, fl);
        F(fo_bc_velocity)(p, fl);
        F(swap_eta)(fl);
    }
}

/* IB compute_residuals!: kernels_3d.jl:118-143 */
void F(fo_ib_compute_residuals)(const fo_params *p, fo_fields *fl) {
    F(geom) g = F(mkgeom)(p);
    const REAL *P = (const REAL *)fl->P, *txx = (const REAL *)fl->txx, *tyy = (const REAL *)fl->tyy;
    const REAL *tzz = (const REAL *)fl->tzz, *txy = (const REAL *)fl->txy, *txz = (const REAL *)fl->txz;
    const REAL *tyz = (const REAL *)fl->tyz;
    const REAL *Vx = (const REAL *)fl->Vx, *Vy = (const REAL *)fl->Vy, *Vz = (const REAL *)fl->Vz;
    REAL *rP = (REAL *)fl->rP, *rVx = (REAL *)fl->rVx, *rVy = (REAL *)fl->rVy, *rVz = (REAL *)fl->rVz;
    const REAL *const *na = (const REAL *const *)fl->wna, *const *ns = (const REAL *const *)fl->wns;
    const REAL idx = R(p->inv_dx[0]), idy = R(p->inv_dx[1]), idz = R(p->inv_dx[2]);
    const size_t sx = g.sx, sxy = g.sxy;
    const REAL *wc = na[W_CCC], *wvvc = na[W_VVC], *wvcv = na[W_VCV], *wcvv = na[W_CVV];
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= g.n2 + 1; k++)
        for (int j = 1; j <= g.n1 + 1; j++)
            for (int i = 1; i <= g.n0 + 1; i++) {
                size_t I = (size_t)i + sx * (size_t)j + sxy * (size_t)k;
                REAL gx = F(gval)(p, fl->gx, 0, I), gy = F(gval)(p, fl->gy, 1, I), gz = F(gval)(p, fl->gz, 2, I);
                if (F(active)(na, ns, W_CCC, I, sx, sxy))
                    rP[I] = (ns[W_VCC][I + 1] * Vx[I + 1] - ns[W_VCC][I] * Vx[I]) * idx +
                            (ns[W_CVC][I + sx] * Vy[I + sx] - ns[W_CVC][I] * Vy[I]) * idy +
                            (ns[W_CCV][I + sxy] * Vz[I + sxy] - ns[W_CCV][I] * Vz[I]) * idz;
                else
                    rP[I] = R(0.0);
                if (F(active)(ns, na, W_VCC, I, sx, sxy))
                    rVx[I] = -(wc[I] * P[I] - wc[I - 1] * P[I - 1]) * idx + (wc[I] * txx[I] - wc[I - 1] * txx[I - 1]) * idx +
                             (wvvc[I + sx] * txy[I + sx] - wvvc[I] * txy[I]) * idy +
                             (wvcv[I + sxy] * txz[I + sxy] - wvcv[I] * txz[I]) * idz - gx;
                else
                    rVx[I] = R(0.0);
                if (F(active)(ns, na, W_CVC, I, sx, sxy))
                    rVy[I] = -(wc[I] * P[I] - wc[I - sx] * P[I - sx]) * idy + (wc[I] * tyy[I] - wc[I - sx] * tyy[I - sx]) * idy +
                             (wvvc[I + 1] * txy[I + 1] - wvvc[I] * txy[I]) * idx +
                             (wcvv[I + sxy] * tyz[I + sxy] - wcvv[I] * tyz[I]) * idz - gy;
                else
                    rVy[I] = R(0.0);
                if (F(active)(ns, na, W_CCV, I, sx, sxy))
                    rVz[I] = -(wc[I] * P[I] - wc[I - sxy] * P[I - sxy]) * idz + (wc[I] * tzz[I] - wc[I - sxy] * tzz[I - sxy]) * idz +
                             (wvcv[I + 1] * txz[I + 1] - wvcv[I] * txz[I]) * idx +
                             (wcvv[I + sx] * tyz[I + sx] - wcvv[I] * tyz[I]) * idy - gz;
                else
                    rVz[I] = R(0.0);
            }
    F(bc_residual)(p, fl);
}

void F(fo_ib_residual_norms)(const fo_params *p, fo_fields *fl, double *out) {
    F(fo_ib_compute_residuals)(p, fl);
    F(norms_from_arrays)(p, fl, out);
}

#undef SMALL
#undef W_CCC
#undef W_VVV
#undef W_VCC
#undef W_CVC
#undef W_CCV
#undef W_VVC
#undef W_VCV
#undef W_CVV
#undef LOOP3
#undef LOOP2
#undef R
#undef F
#undef CAT
#undef CAT_
