/*
 * fastice_b200.h -- C ABI of libfastice_b200, a B200 (sm_100a) implementation of
 * the FastIce.jl pseudo-transient (PT) Stokes iteration.
 *
 * The ABI is shaped for a Julia `ccall` shim that keeps FastIce's API: plain C
 * types, opaque handles and host pointers; no CUDA, torch or C++ types cross
 * it.  Each entry point names the reference (PTsolvers/FastIce.jl v0.3.3)
 * function it replaces.  All functions return an fi_status; fi_last_error()
 * gives the message of the last failure on the calling thread.
 *
 * Data layout.  A model owns its device fields.  Host arrays passed to
 * fi_model_set_field / fi_model_get_field hold a field's interior in Julia
 * column-major order (x fastest), sized by the field's staggered location:
 * n per Center dimension and n+1 per Vertex dimension -- exactly
 * `Array(interior(field))` on the Julia side.
 *
 * Threading.  One CUDA stream per model.  fi_model_advance is asynchronous;
 * functions returning host data synchronise the model's stream.  A model may be
 * used by one thread at a time; distinct models are independent.
 */
#ifndef FASTICE_B200_H
#define FASTICE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FI_ABI_VERSION 1

/* ---- status codes (Julia exceptions in the reference, e.g. the
 *      error("simulation failed") of scripts_future_API/tm_stokes_chmy.jl:104-106) */
typedef enum {
    FI_OK = 0,
    FI_ERR_ARG = 1,         /* invalid argument or descriptor */
    FI_ERR_OOM = 2,         /* device or host allocation failed, or over budget */
    FI_ERR_DIVERGED = 3,    /* non-finite residual */
    FI_ERR_TIMEOUT = 4,     /* iteration budget or bounded wait exhausted */
    FI_ERR_CUDA = 5,        /* CUDA runtime error */
    FI_ERR_UNSUPPORTED = 6, /* valid request the library does not implement */
    FI_ERR_STATE = 7        /* call not valid in the object's current state */
} fi_status;

typedef enum { FI_F64 = 0, FI_F32 = 1 } fi_dtype;

/* ---- boundary conditions: BoundaryCondition{Slip|Traction|Velocity}(components...)
 *      src/Models/FullStokes/Isothermal/boundary_conditions.jl:1-13.  PERIODIC is
 *      an extension (both sides of a dim must be PERIODIC). */
typedef enum { FI_BC_SLIP = 0, FI_BC_TRACTION = 1, FI_BC_VELOCITY = 2, FI_BC_PERIODIC = 3, FI_BC_HALO = 4 } fi_bc_kind;
/* FI_BC_HALO: the side of a subdomain whose ghost layer comes from its neighbour
 * (the reference's distributed boundary, exchanged by Chmy.Distributed); x or y only,
 * fused sweep only; the other side of that dimension may be a physical boundary */

typedef struct {
    int32_t kind;   /* fi_bc_kind */
    double c[3];    /* components (x, y, z) */
} fi_bc;

/* ---- grid: Chmy UniformGrid(arch; origin, extent, dims) */
typedef struct {
    int32_t nd;        /* 2 or 3 */
    int32_t n[3];      /* cells per dimension */
    double origin[3];
    double extent[3];
} fi_grid;

/* ---- rheology: src/Physics.jl.  inner law, optionally wrapped by
 *      ViscoplasticRegularisation (:20-26) and then by Relaxation (:28-47, the
 *      relaxed field being the model's current viscosity). */
typedef enum { FI_RHEO_LINEAR = 0, FI_RHEO_POWER = 1 } fi_rheo_inner;
typedef enum { FI_RELAX_NONE = 0, FI_RELAX_LIN = 1, FI_RELAX_LOG = 2, FI_RELAX_LOG10 = 3 } fi_relax;

typedef struct {
    int32_t inner;         /* fi_rheo_inner */
    int32_t eta_is_field;  /* LinearViscousRheology(field): values via FI_FIELD_ETA_LIN */
    double eta;            /* LinearViscousRheology(constant) */
    int32_t A_is_field;    /* PowerLawRheology(A field): values via FI_FIELD_A */
    double A;              /* PowerLawRheology A (constant) */
    int32_t n;             /* PowerLawRheology exponent (integer) */
    int32_t has_reg;       /* wrap in ViscoplasticRegularisation(., eta_reg) */
    double eta_reg;
    int32_t relax;         /* fi_relax */
    double rate;
} fi_rheology;

/* ---- gravity (rho*g) per component: ZeroField/ValueField (value) or a field
 *      sampled at the velocity component's location (FunctionField), set with
 *      FI_FIELD_GX/GY/GZ. */
typedef enum { FI_G_VALUE = 0, FI_G_FIELD = 1 } fi_gravity_kind;

typedef struct {
    int32_t kind[3];
    double value[3];
} fi_gravity;

/* ---- PT pseudo-time steps: solver_params.Δτ = (Pr, τ = (xx, yy, zz, xy, xz, yz),
 *      V = (x, y, z)), scripts_future_API/stokes_manufactured_solution_free_slip_2D.jl:67-77 */
typedef struct {
    double dt_P;
    double dt_tau[6];
    double dt_V[3];
} fi_pt_params;

/* kernel-path selection (fi_model_desc.path) */
typedef enum {
    FI_PATH_AUTO = 0,      /* fused single-pass sweep where supported, else reference-shaped */
    FI_PATH_REFERENCE = 1, /* reference-shaped: update_sigma, BC batch, update_V, BC batch */
    FI_PATH_FUSED = 2      /* fused sweep; FI_ERR_UNSUPPORTED if the problem is not covered */
} fi_path;

/* ---- model: IsothermalFullStokesModel(; arch, grid, boundary_conditions,
 *      gravity, rheology, solver_params) (FullStokes/Isothermal/Isothermal.jl:60-89)
 *      and IsothermalImmersedBoundaryFullStokesModel(; ..., level_sets)
 *      (ImmersedBoundaryFullStokes/Isothermal/Isothermal.jl:63-98). */
typedef struct {
    fi_grid grid;
    fi_bc bc[3][2];          /* [dim][side]: boundary_conditions = (x=(l,r), y=..., z=...) */
    fi_gravity gravity;
    fi_rheology rheology;
    fi_pt_params dtau;
    int32_t dtype;           /* fi_dtype */
    int32_t immersed;        /* 1: immersed-boundary model (3D only), masks via FI_FIELD_NA_* / NS_* */
    int32_t path;            /* fi_path */
    int32_t device;          /* CUDA device ordinal */
} fi_model_desc;

typedef struct fi_model fi_model;

/* field identifiers (model.stress.P, model.stress.τ.xx, ..., model.velocity.V.x,
 * model.viscosity.η, model.residual.r_P, model.field_masks.na.ccc, ...) */
typedef enum {
    FI_FIELD_P = 0, FI_FIELD_TXX, FI_FIELD_TYY, FI_FIELD_TZZ, FI_FIELD_TXY, FI_FIELD_TXZ, FI_FIELD_TYZ,
    FI_FIELD_VX, FI_FIELD_VY, FI_FIELD_VZ,
    FI_FIELD_ETA, FI_FIELD_ETA_NEXT,
    FI_FIELD_RP, FI_FIELD_RVX, FI_FIELD_RVY, FI_FIELD_RVZ,
    FI_FIELD_GX, FI_FIELD_GY, FI_FIELD_GZ,
    FI_FIELD_ETA_LIN, FI_FIELD_A,
    FI_FIELD_NA_CCC, FI_FIELD_NA_VVV, FI_FIELD_NA_VCC, FI_FIELD_NA_CVC,
    FI_FIELD_NA_CCV, FI_FIELD_NA_VVC, FI_FIELD_NA_VCV, FI_FIELD_NA_CVV,
    FI_FIELD_NS_CCC, FI_FIELD_NS_VVV, FI_FIELD_NS_VCC, FI_FIELD_NS_CVC,
    FI_FIELD_NS_CCV, FI_FIELD_NS_VVC, FI_FIELD_NS_VCV, FI_FIELD_NS_CVV,
    FI_FIELD_COUNT
} fi_field;

/* length of the fi_model_residual_norms output: [0..3] inf-norms of r_P, r_Vx,
 * r_Vy, r_Vz; [4..7] L2 norms of the same; [8..10] max |Vx|, |Vy|, |Vz|;
 * [11] 1.0 if any value was non-finite. */
#define FI_NORMS_LEN 12

const char *fi_last_error(void);
int fi_abi_version(void);

/* IsothermalFullStokesModel(...) / IsothermalImmersedBoundaryFullStokesModel(...):
 * allocates every field on the device, zero-filled. */
fi_status fi_model_create(const fi_model_desc *desc, fi_model **out);
fi_status fi_model_destroy(fi_model *m);

/* set!(field, array) / Array(interior(field)): interior values, x fastest, in the
 * model's dtype; nbytes must equal the field's interior size times sizeof(dtype).
 * set_field stages the upload through a device buffer that the model keeps until
 * it is destroyed (at most 64 MB, at least one z plane, at most one field). */
fi_status fi_model_set_field(fi_model *m, int32_t field, const void *host, size_t nbytes);
fi_status fi_model_get_field(fi_model *m, int32_t field, void *host, size_t nbytes);
/* set!(dst, src) between two fields of the model at the same staggered location,
 * on the device (the drivers' η_next = η before iterating, tm_stokes_chmy.jl:277-278):
 * the whole halo box, ghosts included. */
fi_status fi_model_copy_field(fi_model *m, int32_t dst, int32_t src);
/* interior element count of a field (n or n+1 per dim by location) */
fi_status fi_model_field_size(const fi_model *m, int32_t field, size_t *count);

/* New rheology parameters and PT steps for the next iterations (the model's
 * `rheology` and `solver_params`, Isothermal.jl:27-35; a continuation driver changes
 * them between solves, e.g. raising a viscosity cap stage by stage).  The new
 * rheology must read the same fields as the model's (eta_is_field, A_is_field); the
 * state is kept; the mixed-precision shadow, if any, follows. */
fi_status fi_model_set_params(fi_model *m, const fi_rheology *rheology, const fi_pt_params *dtau);

/* Ghost fill that drivers do after set!: stress and velocity BC batches and
 * Neumann on η / η_next (tm_stokes_chmy.jl:273-281). */
fi_status fi_model_apply_bcs(fi_model *m);

/* advance_iteration!(model, t, Δt) repeated niter times
 * (FullStokes/Isothermal/Isothermal.jl:91-112; IB: Isothermal.jl:100-122).
 * Asynchronous on the model's stream. */
fi_status fi_model_advance(fi_model *m, int32_t niter);

/* compute_residuals!(model) (Isothermal.jl:114-125): writes r_P and r_V fields. */
fi_status fi_model_compute_residuals(fi_model *m);

/* compute_residuals!(model) followed by norm(r, Inf) / norm(r, 2) of every
 * component (tm_stokes_chmy.jl:286-290), fused: no residual field is written.
 * Synchronises; out has FI_NORMS_LEN doubles. */
fi_status fi_model_residual_norms(fi_model *m, double *out);

/* compute_τ! helper (kernels_3d.jl:44-64, kernels_2d.jl:33-44): τ = 2η dev(ε̇). */
fi_status fi_model_compute_tau(fi_model *m);

/* Driver loop (tm_stokes_chmy.jl:283-305): advance, every ncheck iterations take
 * the residual norms, stop when the convergence measure drops below tol or after
 * max_iter iterations.  FI_ERR_DIVERGED on a non-finite residual. */
typedef enum { FI_CONV_ABS_INF = 0, FI_CONV_REL_SLAB = 1 } fi_conv_measure;
typedef enum { FI_SOLVE_PLAIN = 0, FI_SOLVE_MIXED = 1 } fi_solve_mode;

typedef struct {
    int32_t max_iter;
    int32_t ncheck;
    double tol;
    int32_t measure;        /* fi_conv_measure */
    double rho_g_inf;       /* FI_CONV_REL_SLAB: ||ρg||∞ */
    double length_z;        /* FI_CONV_REL_SLAB: L_z */
    int32_t mode;           /* fi_solve_mode: MIXED = FP32 sweeps in FP64 defect correction;
                               with a power-law rheology the FP32 phase is followed by FP64
                               sweeps (the plain iteration) instead of frozen-η corrections */
    int32_t inner_iter;     /* MIXED: most FP32 sweeps per correction (0: 50 * ncheck) */
    double inner_reduction; /* MIXED: stop a correction once its residual dropped by this
                               factor (0: 1e-3) or stopped halving for 2(n+1) sweeps */
} fi_solve_opts;

typedef struct {
    int32_t iterations;     /* PT sweeps (all precisions) */
    int32_t outer;          /* defect-correction steps (MIXED) */
    double measure;         /* final convergence measure */
    double norms[FI_NORMS_LEN];
    double seconds;         /* wall time of the solve */
    int32_t converged;
} fi_solve_report;

fi_status fi_model_solve(fi_model *m, const fi_solve_opts *opts, fi_solve_report *rep);

/* swap-free view of the model state for callers that manage device memory:
 * device pointer of a field's storage (uniform halo box, see fi_model_layout).
 * The caller may write through it at any later time, so for an immersed-boundary
 * model a pointer to P, τ or V turns off for good the iterations' skipping of
 * zeros already stored at inactive points (results are the same either way). */
fi_status fi_model_device_ptr(fi_model *m, int32_t field, void **dptr);
/* storage box: pitch (elements per x row, >= n0+3), rows per plane (n1+3),
 * planes (n2+3, 1 in 2D); index (i,j,k) -> i + pitch*(j + rows*k), 0 = ghost. */
fi_status fi_model_layout(const fi_model *m, size_t *pitch, size_t *rows, size_t *planes);
/* cudaStream_t of the model, as void* */
fi_status fi_model_stream(const fi_model *m, void **stream);
fi_status fi_model_synchronize(fi_model *m);
/* which kernel path the model runs (fi_path, never AUTO) */
fi_status fi_model_path(const fi_model *m, int32_t *path);

/* Launch shape of the fused sweep: tile width and height, z-block depth,
 * thread-block cluster shape and trimmed interior boxes.  A shape that does not
 * fit a CTA in the model's precision is rejected by fi_model_set_variant with
 * FI_ERR_UNSUPPORTED.  fi_model_autotune times every shape offered in the model's
 * precision for `iters` iterations on the model itself (so the model advances
 * like warm-up iterations), keeps the fastest and writes its index and the
 * per-variant milliseconds per iteration to best / ms (-1 for shapes not offered;
 * ms may be NULL, else it needs fi_fused_variant_count() slots).  No counterpart
 * in the reference (its launch shape is fixed by Chmy's Launcher). */
int fi_fused_variant_count(void);
const char *fi_fused_variant_name(int32_t variant);
fi_status fi_model_set_variant(fi_model *m, int32_t variant);
fi_status fi_model_autotune(fi_model *m, int32_t iters, int32_t *best, double *ms);

/* Device-side view of a model state for callers that own the field memory:
 * device pointers to index (0,0,0) of each field's uniform halo box (x fastest,
 * index (i,j,k) at ptr[i + pitch*(j + (n1+3)*k)], ghosts included), in the
 * model's dtype.  fi_model_device_ptr / fi_model_layout give a model's own view. */
typedef struct {
    const void *P, *txx, *tyy, *tzz, *txy, *txz, *tyz;
    const void *Vx, *Vy, *Vz;
    const void *g[3];   /* gravity fields where gravity.kind[c] == FI_G_FIELD, else NULL */
    const void *na[8];  /* immersed-boundary masks (immersed models only), else NULL */
    const void *ns[8];
    size_t pitch;       /* elements per x row, >= n0 + 3 */
} fi_state_view;

/* Residual norms that allocate nothing.  No counterpart in the reference: it is
 * fi_model_residual_norms for callers that cannot allocate device memory -- a
 * host program whose device memory belongs to another runtime's allocator,
 * services that fix their device memory at start-up and forbid allocation
 * afterwards.  It computes the same FI_NORMS_LEN values for the
 * state in `state` (problem described by `desc`; desc->path and device are
 * ignored, the current device is used) into the caller's device buffer out_dev,
 * asynchronously on `stream` (a cudaStream_t, NULL for the default stream).
 * Per-block partial sums live in a static device array of 2048 slots (192 KiB,
 * held by every device that loads the library until the process exits); the
 * reduction is a grid-stride loop over at most 148 * 8 blocks, the model's own
 * block count, so any grid fits and the norms equal fi_model_residual_norms' bit
 * for bit (a launch needing more slots would be rejected with FI_ERR_ARG).  The
 * first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) and caches it for the process; make that first call
 * before any stream capture, and do not call it on a device after
 * cudaDeviceReset.  All calls on a device share the array: calls that overlap
 * on the GPU race and must be serialised by the caller. */
fi_status fi_residual_norms_noalloc(const fi_model_desc *desc, const fi_state_view *state, double *out_dev,
                                    void *stream);

/* ---- batched 2D solves -------------------------------------------------------
 * Many independent 2D models advanced together: one persistent launch per PT
 * iteration strides over a device-side work list of the tiles of the instances
 * still iterating; every ncheck iterations an FP64 check, per-instance
 * retirement and work-list compaction run on the device, and the check-to-check
 * step replays as one CUDA graph.  No counterpart in the reference, which runs one
 * model per driver loop (scripts_future_API/tm_stokes_chmy.jl:283-305); each
 * instance follows advance_iteration! of its own model.
 *
 * Members: 2D IsothermalFullStokesModel handles of one dtype and device, linear
 * rheology without regularisation or relaxation, no periodic sides.  The batch
 * holds each member's viscosity fixed at its current η (linear rheology: the
 * rheology's viscosity with Neumann ghosts, as after the reference's first η
 * swap).  The models must outlive the batch; batch calls synchronise the
 * members' streams first, and each member's state and iteration count are
 * updated in place.
 *
 * Measure of an instance (FP64 arithmetic on the stored state): the cell-scaled
 * relative residual max(||r_V||∞ h / max|P, τ|, ||r_P||∞ h / max|V|), h the
 * smallest grid spacing, over the points the residual boundary batch leaves free. */
typedef struct fi_batch fi_batch;

typedef enum {
    FI_ITEM_ACTIVE = 0,    /* still iterating (never reported by fi_batch_solve) */
    FI_ITEM_CONVERGED = 1, /* measure < tol */
    FI_ITEM_STALLED = 2,   /* the measure did not halve for `window` iterations */
    FI_ITEM_DIVERGED = 3,  /* non-finite residual or state */
    FI_ITEM_MAXITER = 4    /* max_iter iterations */
} fi_batch_item_status;

typedef struct {
    int32_t max_iter;   /* per instance */
    int32_t ncheck;     /* iterations between checks (even) */
    double tol;         /* on the measure above */
    int32_t use_graph;  /* 1: replay the check-to-check step as a CUDA graph */
    int32_t window;     /* stall window in iterations (0: never stall) */
} fi_batch_opts;

typedef struct {
    int32_t iterations;
    int32_t status;     /* fi_batch_item_status */
    double measure;     /* at the last check */
} fi_batch_item;

/* count >= 1: the first member fixes the batch's dtype and device */
fi_status fi_batch_create(fi_model *const *models, int32_t count, fi_batch **out);
fi_status fi_batch_destroy(fi_batch *b);
/* membership between steps (continuous batching): a new member starts its own
 * solve (iteration count 0) at the next step; removing a member leaves its state
 * as the batch last wrote it */
fi_status fi_batch_add(fi_batch *b, fi_model *m);
fi_status fi_batch_remove(fi_batch *b, fi_model *m);
int32_t fi_batch_size(const fi_batch *b);
/* niter PT iterations of every member (no checks) */
fi_status fi_batch_advance(fi_batch *b, int32_t niter);
/* restart every member's solve and iterate until all retire; items has one entry
 * per member, in order;
 * seconds (may be NULL) receives the wall time */
fi_status fi_batch_solve(fi_batch *b, const fi_batch_opts *opts, fi_batch_item *items, double *seconds);
/* at most max_rounds check-to-check steps of the members still iterating, without
 * resetting anyone's solve; items (may be NULL) gets every member's state, in
 * membership order; nactive (may be NULL) the members still iterating */
fi_status fi_batch_step(fi_batch *b, const fi_batch_opts *opts, int32_t max_rounds, fi_batch_item *items,
                        int32_t *nactive);
/* current measure of every member (count doubles) */
fi_status fi_batch_measure(fi_batch *b, double *out);
/* FP32 PT sweeps inside an FP64 defect correction, batched: the members (FP64
 * models) keep the solution and the FP64 residuals; their FP32 shadows run every
 * sweep as one batch -- first the full problems to the measure 2e-4 (above the
 * FP32 rounding floor; the stall window ends a member that meets its floor
 * first), then, per outer step, the correction
 * problems of the members whose FP64 measure is still >= tol (forcing r_P and
 * -r_V of the projected iterate, homogeneous boundary values), each to the
 * relative measure inner_tol (0: 1e-3), added to the FP64 state.  A member stops
 * when its FP64 measure drops below tol (CONVERGED), after three outer steps that
 * did not halve it (STALLED) or after max_iter FP32 sweeps (MAXITER); items get
 * the FP32 sweeps, the status and the last FP64 measure.  The mixed-precision
 * solve applied to the batch; no counterpart in the reference. */
fi_status fi_batch_solve_mixed(fi_batch *b, const fi_batch_opts *opts, double inner_tol, fi_batch_item *items,
                               double *seconds);
/* tile shapes of the batched sweep; autotune times each for `iters` iterations on
 * the batch itself (the members advance by (2 + iters) * count_of_variants) */
int fi_batch_variant_count(void);
const char *fi_batch_variant_name(int32_t variant);
fi_status fi_batch_set_variant(fi_batch *b, int32_t variant);
fi_status fi_batch_autotune(fi_batch *b, int32_t iters, int32_t *best, double *ms);

/* ---- batched 3D immersed-boundary iterations ------------------------------------
 * Several 3D immersed-boundary models (one dtype, one device, reference-shaped path)
 * advanced by shared launches: one iteration of every member is eight launches --
 * the masked update_σ! over a work list that concatenates the members' blocks (each
 * member's block list once its stored zeros hold), the stress boundary batches of
 * all members per dimension, the masked update_V!, the velocity boundary batches --
 * and pairs of iterations replay as one CUDA graph.  Each member's iteration is the
 * one fi_model_advance runs for it, so its result is the same alone or in the batch;
 * a member whose state changed runs its first two full iterations alone, and a member
 * whose launch already spans more than 2048 blocks (about two waves) always advances
 * alone on its own stream, overlapping the others.  The models
 * must outlive the batch; after fi_ib_batch_advance each member's stream is ordered
 * after the shared launches.  No counterpart in the reference, which runs one model
 * per driver loop (scripts_future_API/tm_stokes_chmy.jl:283-305). */
typedef struct fi_ib_batch fi_ib_batch;
fi_status fi_ib_batch_create(fi_model *const *models, int32_t count, fi_ib_batch **out);
fi_status fi_ib_batch_destroy(fi_ib_batch *b);
fi_status fi_ib_batch_add(fi_ib_batch *b, fi_model *m);
fi_status fi_ib_batch_remove(fi_ib_batch *b, fi_model *m);
int32_t fi_ib_batch_size(const fi_ib_batch *b);
/* niter iterations of every member */
fi_status fi_ib_batch_advance(fi_ib_batch *b, int32_t niter);
fi_status fi_ib_batch_synchronize(fi_ib_batch *b);

/* ---- subdomains: halo layers of a domain split into slabs ---------------------
 * Replaces the halo exchange of the reference's distributed architecture
 * (Chmy.Distributed exchange_halo! of V and η_next after update_V!,
 * src/Models/FullStokes/Isothermal/Isothermal.jl:103-104).  A slab is a model of
 * its own cells whose split dimension (x or y) has a periodic pair of sides (a ring
 * of slabs over a periodic domain) or a FI_BC_HALO side toward every neighbour (a
 * chain of slabs: the outer sides keep their physical conditions); after each PT
 * iteration the caller moves the halo messages between neighbouring slabs (over
 * NCCL, MPI or a device copy) and unpacks them, replacing the ghost images the
 * sweep wrote.  Messages are device buffers in the model's dtype.
 *   fi_model_halo_bytes(m, dim, side, what, &b): size of the message packed toward
 *       `side` (0 = low neighbour, 1 = high neighbour); the neighbour unpacks it
 *       from its opposite side (any side of a split dimension: a chain's end slab
 *       sizes the buffer it receives into from the side it sends toward)
 *   fi_model_halo_pack(m, dim, side, what, dst): fill that message (on the model's stream)
 *   fi_model_halo_unpack(m, dim, side, what, src): write the message received from
 *       the neighbour on `side` into the ghost layers (on the model's stream)
 * what: FI_HALO_ITERATION (V, η: after every iteration) or FI_HALO_STATE (P, τ, V,
 * η: once, after the initial state is set).  Slabs run the fused sweep (it recomputes
 * the ghost stresses from the exchanged velocities); reference-shaped and
 * immersed-boundary models are rejected with FI_ERR_UNSUPPORTED.  Each pack or
 * unpack is one launch.  Where either dimension may be split, y is the cheaper one:
 * its layers are whole rows, while x layers take one value per row (at 511^3 FP64
 * about 44 against 156 us of pack and unpack per iteration). */
typedef enum { FI_HALO_ITERATION = 0, FI_HALO_STATE = 1 } fi_halo_what;
fi_status fi_model_halo_bytes(const fi_model *m, int32_t dim, int32_t side, int32_t what, size_t *bytes);
fi_status fi_model_halo_pack(fi_model *m, int32_t dim, int32_t side, int32_t what, void *dst_dev);
fi_status fi_model_halo_unpack(fi_model *m, int32_t dim, int32_t side, int32_t what, const void *src_dev);
/* One PT iteration of a slab in two halves, so that its halo exchange overlaps
 * the second (the reference hides the exchange behind the interior with
 * outer_width, FullStokes/Isothermal/Isothermal.jl:72-76,101-107):
 *   fi_model_advance_begin(m, dim): the tiles of the split faces (the layers the
 *     slab sends and the ghost images it writes) on the model's stream; the model's
 *     state is the new one from here on (its other points still being written);
 *   then pack, exchange and unpack on the model's stream;
 *   fi_model_advance_end(m): every other tile, on a second stream of the model,
 *     after the first half; it runs while the halo moves.
 * Every other entry point (and the next begin) first waits for the second half;
 * between begin and end only the halo entry points may be called (FI_ERR_STATE
 * otherwise).  Fused sweep only, split dimension declared periodic. */
fi_status fi_model_advance_begin(fi_model *m, int32_t dim);
fi_status fi_model_advance_end(fi_model *m);
/* The layer plan of those messages, host only (no device, no model): for an
 * nd-dimensional slab of n cells, the (field, layer index along dim) pairs of the
 * message packed toward `side` (pack != 0) or unpacked from it, in message order;
 * each pair is one whole storage plane of the other dimensions.  *count gets the
 * plan's length (pass cap = 0 to query it).  The layer rules of Chmy.Distributed's
 * exchange for the fields the reference exchanges; no counterpart of its own in
 * the reference (its halo layout is implicit in Chmy). */
fi_status fi_halo_plan(int32_t nd, const int32_t *n, int32_t dim, int32_t side, int32_t what, int32_t pack,
                       int32_t *fields, int32_t *layer_index, int32_t cap, int32_t *count);

/* ---- heat diffusion (src/Models/Diffusion/Heat/) -------------------------------
 * HeatDiffusionModel(; grid, boundary_conditions, physics, iter_params) and
 * advance_iteration!(model, t, Δt) (Heat.jl:26-61, kernels.jl:3-29): the
 * pseudo-transient flux q and the implicit temperature step, one fused sweep per
 * iteration.  Boundary kinds BoundaryCondition{Value}(v) (T ghost 2v - T) and
 * BoundaryCondition{Flux}(v) (q on the boundary face = v), per (dim, side) in the
 * order west/east, south/north, bottom/top.  Fields are interiors, x fastest: T and
 * T_o n0 x n1 x n2, q_d with n_d + 1 faces along d.  3D only, as the reference. */
typedef enum { FI_HEAT_VALUE = 0, FI_HEAT_FLUX = 1 } fi_heat_bc_kind;
typedef enum { FI_HEAT_T = 0, FI_HEAT_T_OLD = 1, FI_HEAT_QX = 2, FI_HEAT_QY = 3, FI_HEAT_QZ = 4 } fi_heat_field;
typedef struct {
    fi_grid grid;
    int32_t kind[3][2];    /* fi_heat_bc_kind */
    double value[3][2];
    double lambda_rhocp;   /* physics λ / (ρ Cp) */
    double dtau_T, dtau_q; /* iter_params.Δτ.T, iter_params.Δτ.q */
    int32_t dtype;         /* fi_dtype */
    int32_t device;
} fi_heat_desc;
typedef struct fi_heat fi_heat;
fi_status fi_heat_create(const fi_heat_desc *desc, fi_heat **out);
fi_status fi_heat_destroy(fi_heat *h);
fi_status fi_heat_field_size(const fi_heat *h, int32_t field, size_t *count);
fi_status fi_heat_set_field(fi_heat *h, int32_t field, const void *host, size_t nbytes);
fi_status fi_heat_get_field(fi_heat *h, int32_t field, void *host, size_t nbytes);
/* the Flux faces of q, then the Value ghosts of T (after set_field, as the drivers' _apply_bcs!) */
fi_status fi_heat_apply_bcs(fi_heat *h);
/* niter PT iterations of the implicit step of length dt (asynchronous on the model's stream) */
fi_status fi_heat_advance(fi_heat *h, int32_t niter, double dt);
fi_status fi_heat_synchronize(fi_heat *h);
/* cudaStream_t of the heat model, as void* */
fi_status fi_heat_stream(const fi_heat *h, void **stream);

/* ---- level sets and volume fractions (setup path) --------------------------- */

/* ω_from_ψ!(arch, launch, ω, ψ, grid) (LevelSets/volume_fractions_kernels.jl:101-110):
 * psi is the level set at grid vertices in halo storage of a model's grid
 * ((n0+3) x (n1+3) x (n2+3), x fastest, ghosts filled); writes the model's
 * mask group (0 = na, 1 = ns), all 8 components (4 in 2D is not supported). */
fi_status fi_model_volfrac_from_levelset(fi_model *m, int32_t group, const double *psi_host);

/* compute_levelset_from_dem!(arch, launch, Ψ, dem, dem_grid2D, grid, R)
 * (LevelSets/compute_levelsets.jl:21-25) followed by invert_levelset! when
 * invert != 0 (:32-35).  dem: vertex values of the 2D DEM grid in halo storage
 * ((m0+3) x (m1+3), x fastest, valid up to index m+2); R: row-major 3x3 or NULL
 * (identity).  psi_host receives the 3D vertex level set in halo storage. */
fi_status fi_levelset_from_dem(const fi_grid *grid3, const fi_grid *dem_grid2, const double *dem_host,
                               const double *R, int32_t invert, double *psi_host, int32_t device);

/* Standalone ω_from_ψ! on host arrays (3D: 8 outputs ccc vvv vcc cvc ccv vvc
 * vcv cvv; 2D: 4 outputs cc vv vc cv), halo storage, FP64. */
fi_status fi_volfrac(const fi_grid *grid, const double *psi_host, double **w_host, int32_t device);

#ifdef __cplusplus
}
#endif
#endif /* FASTICE_B200_H */
