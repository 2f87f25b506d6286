/*
 * ablate_fv.h -- C ABI of the B200 finite-volume right-hand-side backend.
 *
 * This library replaces, for one PETSc rank, the discontinuous and continuous flux loops that
 * ablate::finiteVolume::FiniteVolumeSolver::ComputeRHSFunction runs
 * (src/finiteVolume/finiteVolumeSolver.cpp:233-291 in ABLATE 0.13.03):
 *
 *   CellInterpolant::ComputeRHS        src/finiteVolume/cellInterpolant.cpp:43-140
 *     ComputeFieldGradients + limiter  src/finiteVolume/cellInterpolant.cpp:282-497
 *     ComputeFluxSourceTerms           src/finiteVolume/cellInterpolant.cpp:499-639
 *   FaceInterpolant::ComputeRHS        src/finiteVolume/faceInterpolant.cpp:262-448
 *   NavierStokesTransport::AdvectionFlux / DiffusionFlux
 *                                      src/finiteVolume/processes/navierStokesTransport.cpp:99-207, 454-532
 *   SpeciesTransport::AdvectionFlux / DiffusionSpeciesFlux / DiffusionEnergyFlux
 *                                      src/finiteVolume/processes/speciesTransport.cpp:112-341
 *   the aux update run before it       src/solver/cellSolver.cpp:62-135
 *
 * Everything crossing this boundary is plain C: pointers, sizes and status codes. No C++ exception
 * crosses it. Every entry point returns ABL_OK (0) or a negative ABL_ERR_* code; the text of the last
 * error of the calling thread is returned by abl_last_error_string().
 *
 * Data layout (identical to the PETSc local vectors ABLATE hands to its flux functions):
 *   state     U[n_cells][nc],  nc  = 2 + dim + n_species:  rho, rhoE, rho*u[dim], rho*Y[n_species]
 *             (the "euler" field then the "densityYi" field, src/finiteVolume/compressibleFlowFields.cpp:12-29)
 *   residual  F[n_cells][nc], same layout; the backend ADDS into it (locF is zeroed by the caller,
 *             src/solver/timeStepper.cpp:363) and only touches owned cells.
 *   aux       A[n_cells][naux], naux = 1 + dim + n_species: T, u[dim], Y[n_species]
 * All floating point values are IEEE binary64.
 */
#ifndef ABLATE_FV_H
#define ABLATE_FV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------------- */
#define ABL_OK 0
#define ABL_ERR_INVALID_ARGUMENT -1 /* bad pointer, size, enum or mesh descriptor                   */
#define ABL_ERR_CUDA -2             /* a CUDA runtime call failed                                   */
#define ABL_ERR_NAN -3              /* a NaN or Inf appeared in the residual (device status word)  */
#define ABL_ERR_EOS_NOT_CONVERGED -4 /* the mixture temperature iteration hit its iteration cap     */
#define ABL_ERR_RIEMANN_NOT_CONVERGED -5 /* exact Riemann p* iteration failed                       */
#define ABL_ERR_OUT_OF_MEMORY -6
#define ABL_ERR_UNSUPPORTED -7      /* configuration not supported by this build                   */
#define ABL_ERR_NO_DEVICE -8        /* no CUDA device visible                                       */

/* ---- enums ------------------------------------------------------------------------------------ */
/* fluxCalculator::FluxCalculator implementations (src/finiteVolume/fluxCalculator/) */
#define ABL_FLUX_OFF 0     /* offFlux.cpp:2-9     */
#define ABL_FLUX_AVERAGE 1 /* averageFlux.cpp:2-11 */
#define ABL_FLUX_AUSM 2    /* ausm.cpp:2-43       */
#define ABL_FLUX_AUSMPUP 3 /* ausmpUp.cpp:5-96    */
#define ABL_FLUX_RIEMANN 4 /* riemann.cpp:6-36 + riemannSolver.cpp:7-187 */

/* fluxCalculator::Direction (src/finiteVolume/fluxCalculator/fluxCalculator.hpp:12) */
#define ABL_DIR_NA 0
#define ABL_DIR_LEFT 1
#define ABL_DIR_RIGHT 2

/* eos::EOS implementations */
#define ABL_EOS_PERFECT_GAS 0 /* src/eos/perfectGas.cpp                                    */
#define ABL_EOS_NASA7 1       /* src/eos/tChem.cpp (TChem NASA-7 thermodynamics, no kinetics) */

/* eos::ThermodynamicProperty (src/eos/eos.hpp:14-24), same order */
#define ABL_PROP_PRESSURE 0
#define ABL_PROP_TEMPERATURE 1
#define ABL_PROP_INTERNAL_SENSIBLE_ENERGY 2
#define ABL_PROP_SENSIBLE_ENTHALPY 3
#define ABL_PROP_CV 4
#define ABL_PROP_CP 5
#define ABL_PROP_SPEED_OF_SOUND 6
#define ABL_PROP_SPECIES_SENSIBLE_ENTHALPY 7
#define ABL_PROP_DENSITY 8

/* eos::transport::TransportModel implementations */
#define ABL_TRANSPORT_NONE 0
#define ABL_TRANSPORT_CONSTANT 1       /* src/eos/transport/constant.cpp   */
#define ABL_TRANSPORT_SUTHERLAND 2     /* src/eos/transport/sutherland.cpp */
#define ABL_TRANSPORT_CONSTANT_LEWIS 3 /* k = mu*cp/Pr, D = k/(rho*cp*Le); no reference counterpart */

/* PetscFV type of the conserved fields */
#define ABL_RECON_UPWIND 0        /* PETSCFVUPWIND: first order, no gradients         */
#define ABL_RECON_LEASTSQUARES 1  /* PETSCFVLEASTSQUARES: LSQ gradient + limiter      */

/* PetscLimiter types (symmetric Berger-Aftosmis-Murman form, f = 1/2 du/(grad u . dx)) */
#define ABL_LIMITER_NONE 0
#define ABL_LIMITER_ZERO 1
#define ABL_LIMITER_MINMOD 2
#define ABL_LIMITER_VANLEER 3
#define ABL_LIMITER_VANALBADA 4
#define ABL_LIMITER_SIN 5

/* cell kinds inside one rank's local mesh */
#define ABL_CELL_OWNED 0      /* residual written here                                          */
#define ABL_CELL_BOUNDARY 1   /* DMPlex FV ghost cell behind a boundary face (ghost label 1)   */
#define ABL_CELL_HALO 2       /* owned by another rank; gradient computed here, no residual    */
#define ABL_CELL_HALO_OUTER 3 /* owned by another rank; state only (second halo layer)          */

/* precision of abl_fv_rhs */
#define ABL_PRECISION_FP64 0
#define ABL_PRECISION_MIXED 1 /* FP32 reconstruction/flux arithmetic, FP64 e=E/rho-|u|^2/2, T solve and accumulation.
                                With species a mixed request runs the FP64 kernels, unless ABL_FV_MIXED_SPECIES=1
                                is set at abl_fv_create (instances up to 9 species) */
/* or'ed into the precision argument of abl_fv_rhs: F = RHS(U) instead of F += RHS(U) (for a caller
 * whose residual vector holds nothing else; saves reading F) */
#define ABL_RHS_OVERWRITE 0x100

/* ---- descriptors ------------------------------------------------------------------------------ */
/* One rank's local mesh: what DMPlex + DMPlexComputeGeometryFVM hold for the FV solver.
 * face_cells is the face support (left, right); the area-weighted normal points left -> right
 * (PetscFVFaceGeom.normal). Cells of kind ABL_CELL_BOUNDARY have exactly one face. */
typedef struct abl_mesh_desc {
    int32_t dim;                  /* 1, 2 or 3 */
    int32_t n_cells;              /* all local cells, including boundary ghost and halo cells */
    int32_t n_faces;
    const int32_t* face_cells;    /* [n_faces][2] */
    const double* face_normal;    /* [n_faces][3] area-weighted normal (unused components 0) */
    const double* face_centroid;  /* [n_faces][3] */
    const double* cell_centroid;  /* [n_cells][3] */
    const double* cell_volume;    /* [n_cells] */
    const uint8_t* cell_kind;     /* [n_cells] ABL_CELL_*; NULL: every cell owned */
    const double* face_shift;     /* [n_faces][3] periodic image shift: the right cell's centroid seen from
                                     the left cell is cell_centroid[right] + face_shift (and the face centroid,
                                     given in the left cell's frame, is face_centroid - face_shift in the right
                                     cell's frame); NULL: no periodic faces */
} abl_mesh_desc;

/* Process configuration: what NavierStokesTransport / SpeciesTransport register in Setup
 * (src/finiteVolume/processes/navierStokesTransport.cpp:35-97, speciesTransport.cpp:35-96). */
typedef struct abl_physics_desc {
    int32_t eos;             /* ABL_EOS_* */
    double gamma;            /* perfect gas: specific heat ratio (default 1.4) */
    double r_gas;            /* perfect gas: gas constant J/(kg K) (default 287) */
    int32_t n_species;       /* densityYi components, 0..128; 0 = no species field. Instances with their
                                loops unrolled: (1, 0), (2, 0), (2, 2), (2, 3), (3, 0), (3, 2), (3, 5),
                                (3, 9) (every entry point); 16 species in 1D, 2D and 3D (RHS, JVP, aux);
                                with run-time loops, 64 species in 3D (RHS, JVP, aux) and 128 species in
                                1D, 2D and 3D (RHS, aux). Any other
                                count runs in the smallest instance that holds it, its species after zero-state
                                padding species (results unchanged; the RHS, JVP, VJP and aux entry points
                                translate the rows). An entry point the instance does not compile returns
                                ABL_ERR_UNSUPPORTED: the VJP above 9 species (3 in 2D, none with species in
                                1D), the JVP above 16 (64 in 3D), the ghost, step, CFL, normalisation and functional
                                entry points for counts other than the exact ones */
    const double* nasa7;     /* [n_species][15]: T_mid, low a1..a7, high a1..a7 (cp/R = a1 + a2 T + ... ) */
    const double* mw;        /* [n_species] molar mass kg/kmol */

    int32_t flux;            /* ABL_FLUX_*; ABL_FLUX_OFF with advection = 0 disables advection */
    double ausmpup_minf;     /* AusmpUp mInf (0 = fa = 1) */
    double pgs_alpha;        /* pressure gradient scaling alpha (1 = none) */

    int32_t reconstruction;  /* ABL_RECON_* (both conserved fields use the same PetscFV) */
    int32_t limiter;         /* ABL_LIMITER_* */
    double max_lim_grad;     /* CellInterpolant maxLimGrad (default 1e10) */

    int32_t transport;       /* ABL_TRANSPORT_* */
    double k, mu, diff;      /* constant model values; for CONSTANT_LEWIS: mu, prandtl in k, lewis in diff */

    int32_t advection;          /* NavierStokesTransport::AdvectionFlux registered */
    int32_t diffusion;          /* NavierStokesTransport::DiffusionFlux registered */
    int32_t species_advection;  /* SpeciesTransport::AdvectionFlux registered */
    int32_t species_diffusion;  /* SpeciesTransport::DiffusionSpeciesFlux + DiffusionEnergyFlux registered */
    const double* species_diff; /* [n_species] per-species diffusivities D_k of the Constant model given one
                                   value per species, which registers DiffusionSpeciesFluxVariableDiffusionCoefficient
                                   and DiffusionEnergyFluxVariableDiffusionCoefficient instead
                                   (src/finiteVolume/processes/speciesTransport.cpp:64-75, 154-194, 230-261);
                                   ABL_TRANSPORT_CONSTANT only. NULL: the scalar diff */
    int32_t species_advection_compact; /* the species advection of CompactCompressibleNSSpeciesTransport::AdvectionFlux
                                          (compactCompressibleNSSpeciesTransport.cpp:162-271): where the flux calculator
                                          gives no direction (NA), rho Y_k is carried as
                                          (rho Y_L + rho Y_R) / (rho_L + rho_R) instead of the right state */
} abl_physics_desc;

typedef struct abl_fv abl_fv; /* opaque handle: one mesh + physics resident on one device */

/* ---- library ---------------------------------------------------------------------------------- */
const char* abl_last_error_string(void);
int abl_version(void);
int abl_device_count(int* count);

/* ---- handle lifecycle ------------------------------------------------------------------------- */
/* Upload the mesh, the geometry and the least-squares weights (built here, once, from the geometry as
 * BuildGradientReconstruction_Internal and LeastSquaresAverage::Generate do:
 * src/finiteVolume/cellInterpolant.cpp:641-715, src/finiteVolume/stencils/leastSquaresAverage.cpp:5-155)
 * to device `device`. Replaces the lazy CellInterpolant/FaceInterpolant construction at
 * src/finiteVolume/finiteVolumeSolver.cpp:241-243, 269-271. */
int abl_fv_create(const abl_mesh_desc* mesh, const abl_physics_desc* physics, int device, abl_fv** out);
int abl_fv_destroy(abl_fv* fv);
int abl_fv_sizes(const abl_fv* fv, int32_t* nc, int32_t* naux, int32_t* n_cells, int32_t* n_faces);
/* The device layout abl_fv_create chose (no reference counterpart: PETSc stores one geometry record per
 * face and one weight set per cell). Tile face geometry records and per-cell cone weight sequences that
 * repeat bit for bit (a structured block) are stored once and read through a per-face / per-cell index
 * when there are at most 4096 distinct ones and at most 1/8 of the records; results are bitwise the
 * same. 0 = one record per face / cone entry. The environment variable ABL_FV_RECORD_TABLES=0, read at
 * create, keeps one record per face and cone entry. */
int abl_fv_record_classes(const abl_fv* fv, int32_t* weight_classes, int32_t* geometry_classes);

/* The RHS kernel layout of a handle: whether the fused one-pass kernel runs the FP64 and the mixed RHS
 * (it does where one tile's staged rows, gradients and face fluxes fit in shared memory; otherwise the
 * gradient pass and the tile flux pass run), how many distinct tile tables it holds, and the largest
 * number of cells one tile stages (its cells and two rings of neighbours). No counterpart in the
 * reference: a diagnostic of this backend. */
int abl_fv_fused_info(const abl_fv* fv, int32_t* fp64, int32_t* mixed, int32_t* classes, int32_t* max_ext);

/* ---- the hot path ----------------------------------------------------------------------------- */
/* F += RHS(U) for owned cells, device pointers, on `stream` (a cudaStream_t; NULL = legacy stream).
 * Runs the aux update (T, velocity, Y for every local cell, T guess = the resident aux T), the
 * gradient/limiter pass and the flux passes. Replaces CellSolver::UpdateAuxFields +
 * FiniteVolumeSolver::ComputeRHSFunction (src/solver/cellSolver.cpp:62-135,
 * src/finiteVolume/finiteVolumeSolver.cpp:233-291). */
int abl_fv_rhs(abl_fv* fv, double time, const double* U_dev, double* F_dev, int precision, void* stream);

/* Same with host pointers (the plain PETSc Vec case): copies U in, runs abl_fv_rhs, adds into F. The
 * copies run on the handle's own streams, overlapped with the kernels (F's rows in chunks, each sent
 * back as soon as its tiles are done); the call returns when F_host holds the result. Only the owned
 * rows of F travel when they are one contiguous range. Pinned host memory makes the copies asynchronous.
 * A handle serves one call at a time (no two threads on one handle). */
int abl_fv_rhs_host(abl_fv* fv, double time, const double* U_host, double* F_host, int precision);

/* abl_fv_rhs in two phases, so that a partitioned run moves its halo while the device computes. Phase
 * ABL_RHS_PHASE_INTERIOR reads no halo row (ABL_CELL_HALO, ABL_CELL_HALO_OUTER): it updates the aux
 * fields of the other cells and the gradients of the cells whose stencils hold no halo cell. Phase
 * ABL_RHS_PHASE_REST, issued after the halo rows are current, does the rest and adds the residual into
 * F. The two calls on one stream equal one abl_fv_rhs call bit for bit; the caller may write the halo
 * rows of U between them (the exchange of DMGlobalToLocal, src/solver/timeStepper.cpp:343-344, moved
 * beside the interior work). Kernels that do not split (the fused kernel, a padded species count) run
 * entirely in the second phase. */
#define ABL_RHS_PHASE_INTERIOR 0
#define ABL_RHS_PHASE_REST 1
int abl_fv_rhs_phase(abl_fv* fv, double time, const double* U_dev, double* F_dev, int precision, int phase, void* stream);

/* Forward tangent (JVP) of abl_fv_rhs at FP64: dF += J(U) dU for owned cells, and F += RHS(U) when F
 * is not NULL. The RHS kernels are evaluated on dual numbers (value + one directional derivative), so
 * every branch (limiter min, flux splittings, upwind choice) is the primal one and its derivative is
 * that of the active branch; the mixture temperature's derivative comes from the implicit-function
 * theorem on e_s(T, Y) = e. The reference's counterpart is PETSc's finite-difference Jacobian-vector
 * product through the same RHS (MatMFFD on TSComputeRHSFunction). */
int abl_fv_jvp(abl_fv* fv, double time, const double* U_dev, const double* dU_dev, double* F_dev, double* dF_dev, void* stream);

/* Tangent mode of the following abl_fv_jvp calls. ABL_JVP_EXACT (the default) differentiates every
 * branch it takes, the limiter factor included. ABL_JVP_FROZEN_LIMITER holds each limiter factor at
 * its value (its derivative, which carries 1/(grad . dx) terms and jumps where the minimising face
 * changes, is dropped): the Jacobian a matrix-free Newton-Krylov step uses to stay well conditioned on
 * limited schemes. abl_fv_vjp is the transpose of the exact tangent in either mode. */
#define ABL_JVP_EXACT 0
#define ABL_JVP_FROZEN_LIMITER 1
int abl_fv_set_jvp_mode(abl_fv* fv, int mode);
int abl_fv_jvp_host(abl_fv* fv, double time, const double* U_host, const double* dU_host, double* F_host, double* dF_host);

/* Adjoint (vector-Jacobian product) of abl_fv_rhs at FP64: Ubar += J(U)^T Fbar. Fbar is read on owned
 * cells (the rows the RHS writes); Ubar receives every cell, boundary ghosts and halos included, since
 * their values enter the owned residuals. It is the transpose of the abl_fv_jvp tangent (same active
 * branches). Only the forward gradients are stored; the limiter, EOS decode and fluxes are recomputed.
 * The reference has no adjoint; it would form J^T only through a finite-difference Jacobian
 * (SNESComputeJacobianDefaultColor / MatMFFD) of ComputeRHSFunction (finiteVolumeSolver.cpp:233-291). */
int abl_fv_vjp(abl_fv* fv, double time, const double* U_dev, const double* Fbar_dev, double* Ubar_dev, void* stream);
int abl_fv_vjp_host(abl_fv* fv, double time, const double* U_host, const double* Fbar_host, double* Ubar_host);

/* Aux fields (T, u, Y). With the NASA-7 mixture EOS every abl_fv_rhs updates them (the resident T is
 * also the next secant guess); with a perfect gas the RHS recomputes them on the fly and they are
 * refreshed only by abl_fv_update_aux. set_aux sets the temperature guess used by the next update. */
int abl_fv_update_aux(abl_fv* fv, const double* U_dev, void* stream);
int abl_fv_update_aux_host(abl_fv* fv, const double* U_host);
int abl_fv_get_aux(abl_fv* fv, double* aux_host);
int abl_fv_set_aux(abl_fv* fv, const double* aux_host);

/* Device status word accumulated since the last call: ABL_OK or the first ABL_ERR_* a kernel saw. */
int abl_fv_status(abl_fv* fv);

/* Per-kernel device timing of abl_fv_rhs: with profiling on, each call records CUDA events between its
 * launches; profile_read returns the durations of the last call (n <= 7 entries, ms[i] and the kernel
 * name in names[32*i], NUL-terminated). */
int abl_fv_profile(abl_fv* fv, int enable);
int abl_fv_profile_read(abl_fv* fv, int32_t* n, float* ms, char* names);

/* Number of kernel launches one abl_fv_rhs call makes at `precision` (for launch accounting). */
int abl_fv_launch_count(const abl_fv* fv, int precision, int32_t* launches);

/* ---- point functions (device batches; used for known-answer tests of the device physics) --------- */
/* Flux calculator over n faces: the FluxCalculatorFunction signature
 * (src/finiteVolume/fluxCalculator/fluxCalculator.hpp:13-14) applied element-wise on the device. */
int abl_flux_calculator_batch(int kind, double minf, double pgs_alpha, double gamma, int64_t n, const double* uL, const double* aL,
                              const double* rhoL, const double* pL, const double* uR, const double* aR, const double* rhoR,
                              const double* pR, double* mass_flux, double* p12, int32_t* direction);

/* ThermodynamicTemperatureFunction / ThermodynamicFunction of `property` for n conserved states
 * conserved[n][nc] with dim = nc - 2 - n_species. If T_in is non-NULL it is the temperature argument
 * (the *TemperatureFunction variant); otherwise T is computed first (guess 300 K, as TChem does).
 * out[n][property size]. */
int abl_eos_batch(const abl_physics_desc* physics, int dim, int property, int64_t n, const double* conserved,
                  const double* T_in, double* out);

/* Allocation-free variant of abl_eos_batch for states already on the device. No counterpart in the
 * reference. abl_eos_batch copies host arrays and the species tables into device buffers it allocates
 * and frees on every call; a caller whose device memory is reserved by a pool allocator (PETSc's or
 * PyTorch's) may be unable to allocate at all, and one evaluating properties inside a time step cannot
 * afford the device-wide synchronisation every cudaFree implies. This entry point calls no cudaMalloc,
 * cudaFree or allocating library routine: conserved_dev[n][nc], T_dev[n] (or NULL) and out_dev[n][property
 * size] are the caller's device buffers, and the NASA-7 tables and the status word live in a 16 KiB
 * file-scope device array of the library (held by every GPU that loads it until exit), which limits
 * n_species to 64 (abl_eos_batch takes up to 128); more are rejected with ABL_ERR_INVALID_ARGUMENT.
 * Work is ordered on `stream`; the call waits for it to finish to return the status.
 * Every call, n = 0 included, first looks up the array's device address on the current device. That
 * lookup may load the library's device code on first use (CUDA loads modules lazily by default), which
 * needs device memory: make one call with n = 0 on each device before a pool allocator reserves the
 * memory. The call copies the tables from host memory and synchronises `stream`, so it must not be made
 * while `stream` is being captured into a CUDA graph. Every call reuses the same array: calls that
 * overlap on the GPU (other streams, other host threads) race on it. */
int abl_eos_batch_noalloc(const abl_physics_desc* physics, int dim, int property, int64_t n, const double* conserved_dev,
                          const double* T_dev, double* out_dev, void* stream);

/* ---- the steps around the RHS in a time step ------------------------------------------------------ */

/* Ghost-cell boundary conditions (the Ghost / EssentialGhost update functions the reference applies
 * through DMPlexInsertBoundaryValuesRiemann before every RHS: src/solver/solver.cpp:50-102,
 * src/finiteVolume/boundaryConditions/ghost.cpp:17-28, essentialGhost.cpp:5-22). The reference takes an
 * arbitrary host callback per boundary; on the device the common conditions are built in. */
#define ABL_BC_OUTFLOW 0     /* ghost = interior (zero gradient)                                      */
#define ABL_BC_DIRICHLET 1   /* ghost = value; with enforce_at_face, 2 value - interior (EssentialGhost) */
#define ABL_BC_SLIP_WALL 2   /* ghost = interior with the normal momentum reversed                    */
#define ABL_BC_NOSLIP_WALL 3 /* ghost = interior with the momentum reversed (zero velocity at the face)  */
#define ABL_BC_MAX_COMPONENTS 16
typedef struct abl_bc {
    int32_t kind;
    int32_t enforce_at_face;
    double value[ABL_BC_MAX_COMPONENTS]; /* conserved state [rho, rhoE, rho u, rhoY] for ABL_BC_DIRICHLET */
} abl_bc;

/* Conditions table and, for every cell, the index of its condition (read for ABL_CELL_BOUNDARY cells
 * only; cell_bc may be NULL: every ghost takes entry 0). Until the first call every ghost is outflow. */
int abl_fv_set_boundary(abl_fv* fv, int32_t n_bc, const abl_bc* table, const int32_t* cell_bc);
/* Fill the ghost rows of U_dev from their interior neighbours (before every RHS evaluation). */
int abl_fv_fill_ghosts(abl_fv* fv, double time, double* U_dev, void* stream);

/* Tangent of the fill on a perturbation dU_dev (in place): every ghost row becomes dG/du times its
 * interior neighbour's row (the condition values are constants: a plain Dirichlet ghost gets 0). */
int abl_fv_fill_ghosts_jvp(abl_fv* fv, double* dU_dev, void* stream);

/* Adjoint of the fill on adjoint rows Ubar_dev (in place): each ghost row's adjoint is added to its
 * interior neighbour through (dG/du)^T and the ghost row is cleared; value_bar_host[n_bc][16] (may be
 * NULL) accumulates the adjoint of every condition's value[] (ABL_BC_DIRICHLET only; the other kinds
 * take no value). Sums run in a fixed order: the same inputs give the same bits. With abl_fv_vjp and
 * abl_fv_rk_stage this is the reverse of abl_fv_step, for gradients of a functional of the marched state
 * with respect to the initial state and the boundary values. No reference counterpart: the reference
 * has no adjoint of its boundary conditions. */
int abl_fv_fill_ghosts_vjp(abl_fv* fv, double* Ubar_dev, double* value_bar_host, void* stream);

/* Pressure functional J(U) = sum_j w_j p(U_{c_j}) over distinct cells c_j (for the pressure integrated
 * over a wall patch: the cells next to the wall faces, w = face area; a no-slip ghost mirrors only the
 * momentum, so the wall-face pressure is the cell's). set_ registers the cells and weights (host
 * arrays, validated: in range, no cell twice). The evaluation returns J in *J_host and, when Ubar_dev
 * is not NULL, adds w_j dp/dU into Ubar_dev's rows (the reverse of the EOS decode, NASA-7 included). */
int abl_fv_set_pressure_functional(abl_fv* fv, int32_t n, const int32_t* cells, const double* weights);
int abl_fv_pressure_functional(abl_fv* fv, const double* U_dev, double* J_host, double* Ubar_dev, void* stream);

/* CFL time step of NavierStokesTransport::ComputeCflTimeStep (navierStokesTransport.cpp:209-278):
 * min over owned cells of cfl * 2 r_min / (a / alpha + sum_d |u_d|), r_min the smallest cell-centroid to
 * face-centroid distance, a the speed of sound at T(U) (guess 300 K), alpha the pressure-gradient
 * scaling. Waits for `stream`; *dt_host receives this rank's minimum (reduce over ranks with MIN). */
int abl_fv_cfl_dt(abl_fv* fv, const double* U_dev, double cfl, double* dt_host, void* stream);

/* Mass-fraction clipping of SpeciesTransport::NormalizeSpecies (speciesTransport.cpp:343-403) on the
 * owned rows; a no-op without species. */
int abl_fv_normalize_species(abl_fv* fv, double* U_dev, void* stream);

/* One stage of a Runge-Kutta step on the owned rows: Uout = a U0 + b (Us + dt F) (a == 0 drops U0). */
int abl_fv_rk_stage(abl_fv* fv, double a, const double* U0_dev, double b, const double* Us_dev, double dt, const double* F_dev,
                    double* Uout_dev, void* stream);

/* One explicit step, in place on U_dev. ABL_STEP_EULER is PETSc's default explicit TS (forward Euler),
 * which the reference's shock-tube tests run; ABL_STEP_SSPRK3 the three-stage strong-stability-
 * preserving Runge-Kutta scheme (Shu-Osher form). Every stage fills the ghosts and evaluates the RHS at
 * `precision`; the species are normalised after the step and the ghosts refilled. Single domain (a
 * partitioned run exchanges halos between the stages and drives abl_fv_rk_stage itself). The step size
 * policy (CFL step of the state the previous step started from, exact final time) is the caller's; see
 * abl_fv_cfl_dt. */
#define ABL_STEP_EULER 0
#define ABL_STEP_SSPRK3 1
int abl_fv_step(abl_fv* fv, int scheme, double time, double dt, double* U_dev, int precision, void* stream);

/* The same step with dt = the CFL step of U_dev's state (abl_fv_cfl_dt, this rank's minimum) computed
 * and used on the device: nothing returns to the host, so consecutive steps queue back to back on
 * `stream` (and can be captured in a CUDA graph). When time_dev is not NULL, dt is added to *time_dev
 * (a device double). Single domain: a partitioned run needs the minimum over ranks first. */
int abl_fv_step_cfl(abl_fv* fv, int scheme, double cfl, double* U_dev, int precision, double* time_dev, void* stream);

/* State download and upload for output and restart. The reference saves the TS solution vector (the
 * rank's owned cells, in local order: the DM's global vector) through PetscViewerHDF5 in its
 * Hdf5Serializer monitor and reads it back on restart (src/io/hdf5Serializer.cpp:54-160,
 * src/finiteVolume/finiteVolumeSolver.cpp:398-442). With the state resident on the GPU, download_owned
 * copies the owned rows of a device array with `width` doubles per cell (the state, nc; the aux
 * fields, naux) into host[n_owned][width], ascending local cell order, ready for VecView on that
 * global vector; upload_owned writes such an array back into the owned rows (ghost and halo rows are
 * the caller's: fill them and exchange halos after a restart). Both wait for `stream`. */
int abl_fv_download_owned(abl_fv* fv, const double* src_dev, int width, double* host, void* stream);
int abl_fv_upload_owned(abl_fv* fv, const double* host, int width, double* dst_dev, void* stream);

/* Halo exchange between ranks of a partitioned mesh (the pack and unpack of DMGlobalToLocal's PetscSF
 * broadcast of the state to ghost/overlap cells, src/solver/timeStepper.cpp:343-344). Row i of a
 * width-column FP64 array is copied to or from a contiguous message buffer on `stream`:
 *   gather:  dst[i][:] = src[idx[i]][:]   (pack the owned rows a neighbour needs)
 *   scatter: dst[idx[i]][:] = src[i][:]   (unpack a neighbour's rows into the halo rows)
 * All pointers are device pointers; the message travels between the calls (NCCL or peer copies). */
int abl_rows_gather(const double* src_dev, int width, const int32_t* idx_dev, int64_t n, double* dst_dev, void* stream);
int abl_rows_scatter(const double* src_dev, int width, const int32_t* idx_dev, int64_t n, double* dst_dev, void* stream);

/* The adjoint of the exchange: dst[idx[i]][:] += src[i][:] (the indices of one call distinct). A rank
 * sends the adjoint of its halo rows back to their owners, which add them into the owned rows, one
 * peer after another in a fixed order (the transpose of DMGlobalToLocal, a LocalToGlobal with
 * ADD_VALUES: src/solver/timeStepper.cpp:379-380). */
int abl_rows_scatter_add(const double* src_dev, int width, const int32_t* idx_dev, int64_t n, double* dst_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ABLATE_FV_H */
