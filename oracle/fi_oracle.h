/*
 * fi_oracle.h -- CPU oracle for the FastIce pseudo-transient Stokes path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (PTsolvers/FastIce.jl v0.3.3) used as the checker for the CUDA
 * library.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference leg may load it.  The product never links or calls it.
 *
 * Parity status: PARTIALLY PINNED.  Grid geometry (sizes, spacing, coordinates)
 * is pinned against the reference's own test/test_chmy_grids.jl.  The stencil
 * operators, interpolation and boundary-condition ghost rules live in the
 * un-vendored third-party package Chmy.jl 0.1 (no patch version pinned; its
 * Manifest.toml is git-ignored by the reference), which is absent here, so their
 * exact floating-point order is "parity unpinned" and is fixed by the adopted
 * contract below, anchored by manufactured-solution O(h^2) convergence tests.
 *
 * Adopted Chmy contract (restated from Chmy's published semantics):
 *  - every field is stored with one ghost layer: index 0 and N_loc+1, where
 *    N_loc = n (Center) or n+1 (Vertex) per dimension; storage is a uniform
 *    (n0+3) x (n1+3) [x (n2+3)] box for every location, x fastest;
 *  - vertex i sits at origin+(i-1)*dx, centre i at origin+(i-1/2)*dx;
 *  - d/dx of a Vertex-in-x field at index i: (f[i+1]-f[i])*inv_dx;
 *    d/dx of a Center-in-x field at index i: (f[i]-f[i-1])*inv_dx;
 *  - lerp C->V uses {i-1,i}, V->C uses {i,i+1}, each 1-D step is 0.5*(a+b),
 *    and multi-dimensional lerps interpolate x first, then y, then z;
 *  - kernels run over the vertex-sized index range 1..n+1 in every dimension
 *    and write every field at that index (so centre fields get values written
 *    into their right ghost; those values are overwritten by boundary
 *    conditions or never read by interior points);
 *  - Dirichlet(v) on a field Center in the normal dim sets ghost = 2*v - f[adj];
 *    on a field Vertex in the normal dim sets the boundary node = v;
 *    Neumann() sets ghost = f[adj] (Center) or f[0]=f[2], f[n+2]=f[n] (Vertex);
 *  - boundary conditions are applied dimension by dimension (x, y, z), left
 *    side then right side; a face of dim d spans the full storage range of the
 *    dims before d and the interior range of the dims after d;
 *  - periodic dims (never exercised by the reference) wrap ghosts:
 *    Center f[0]=f[n], f[n+1]=f[1]; Vertex f[n+1]=f[1], f[0]=f[n], f[n+2]=f[2];
 *    stresses wrap after the stress update, velocities and eta_next after the
 *    velocity update.
 */
#ifndef FI_ORACLE_H
#define FI_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* boundary-condition kinds, per (dim, side); mirror
 * src/Models/FullStokes/Isothermal/boundary_conditions.jl:1-13 */
enum { FO_BC_SLIP = 0, FO_BC_TRACTION = 1, FO_BC_VELOCITY = 2, FO_BC_PERIODIC = 3 };

/* rheology (src/Physics.jl): inner law, optional viscoplastic cap, optional relaxation */
enum { FO_RHEO_LINEAR = 0, FO_RHEO_POWER = 1 };
enum { FO_RELAX_NONE = 0, FO_RELAX_LIN = 1, FO_RELAX_LOG = 2, FO_RELAX_LOG10 = 3 };

/* gravity component kinds: ZeroField / ValueField / array (FunctionField sampled) */
enum { FO_G_VALUE = 0, FO_G_ARRAY = 1 };

typedef struct {
    int nd;                /* 2 or 3 */
    int n[3];              /* cells per dim (n[2] ignored in 2D) */
    double inv_dx[3];      /* inverse spacing per dim */
    int bc_kind[3][2];     /* [dim][side] */
    double bc_val[3][2][3];/* [dim][side][component] */
    /* PT pseudo-time steps (solver_params.dtau): Pr, tau{xx,yy,zz,xy,xz,yz}, V{x,y,z} */
    double dt_P;
    double dt_tau[6];
    double dt_V[3];
    /* gravity (rho*g) per component */
    int g_kind[3];
    double g_val[3];
    /* rheology */
    int rheo_inner;        /* FO_RHEO_LINEAR / FO_RHEO_POWER */
    double rheo_eta_val;   /* LinearViscousRheology constant (used when eta_lin is NULL) */
    double rheo_A;         /* PowerLawRheology A (used when A_field is NULL) */
    int rheo_n;            /* PowerLawRheology exponent (Int) */
    int rheo_has_reg;      /* ViscoplasticRegularisation wrapper */
    double rheo_inv_eta_reg;
    int rheo_relax;        /* FO_RELAX_* wrapper: field = current eta */
    double rheo_rate;
} fo_params;

/* Field bundle.  All arrays use the uniform halo storage described above.
 * 2D problems leave tzz, txz, tyz, Vz, gz NULL. */
typedef struct {
    void *P, *txx, *tyy, *tzz, *txy, *txz, *tyz;
    void *Vx, *Vy, *Vz;
    void *eta, *eta_next;
    void *rVx, *rVy, *rVz, *rP;         /* residual arrays (compute_residuals) */
    const void *gx, *gy, *gz;           /* gravity arrays when g_kind == FO_G_ARRAY */
    const void *eta_lin;                /* linear rheology field, or NULL */
    const void *A_field;                /* power-law A field, or NULL */
    /* immersed-boundary masks, 8 components each: ccc vvv vcc cvc ccv vvc vcv cvv */
    const void *wna[8], *wns[8];
} fo_fields;

#define FO_DECL(SUF, REAL)                                                                   \
    void fo_update_sigma##SUF(const fo_params *p, fo_fields *f);                             \
    void fo_update_V##SUF(const fo_params *p, fo_fields *f);                                 \
    void fo_bc_stress##SUF(const fo_params *p, fo_fields *f);                                \
    void fo_bc_velocity##SUF(const fo_params *p, fo_fields *f);                              \
    void fo_bc_eta##SUF(const fo_params *p, REAL *eta);                                      \
    void fo_advance##SUF(const fo_params *p, fo_fields *f, int niter);                       \
    void fo_compute_residuals##SUF(const fo_params *p, fo_fields *f);                        \
    void fo_residual_norms##SUF(const fo_params *p, fo_fields *f, double *out);              \
    void fo_compute_tau##SUF(const fo_params *p, fo_fields *f);                              \
    void fo_ib_update_sigma##SUF(const fo_params *p, fo_fields *f);                          \
    void fo_ib_update_V##SUF(const fo_params *p, fo_fields *f);                              \
    void fo_ib_advance##SUF(const fo_params *p, fo_fields *f, int niter);                    \
    void fo_ib_compute_residuals##SUF(const fo_params *p, fo_fields *f);                     \
    void fo_ib_residual_norms##SUF(const fo_params *p, fo_fields *f, double *out);

FO_DECL(_f64, double)
FO_DECL(_f32, float)

/* number of doubles written by fo_residual_norms_*: inf-norms of rP, rVx, rVy, rVz,
 * L2 norms (sqrt of sum of squares) of the same, and max|Vx|,|Vy|,|Vz| */
#define FO_NORMS_LEN 12

/* level sets and volume fractions (FP64 only, setup path) */
void fo_volfrac3d(const int n[3], const double dx[3], const double *psi, double *w[8]);
void fo_volfrac2d(const int n[2], const double dx[2], const double *psi, double *w[4]);
double fo_vol_box3(const double psi[8], const double d[3]);
double fo_vol_box2(const double psi[4], const double d[2]);
void fo_levelset_from_dem(const int n3[3], const double o3[3], const double dx3[3],
                          const int n2[2], const double o2[2], const double dx2[2],
                          const double *dem, const double *R, double cutoff, double *psi);
void fo_invert_levelset(const int n3[3], double *psi);
void fo_neumann_vertex3(const int n3[3], double *psi);

#ifdef __cplusplus
}
#endif
#endif
