/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY. CPU restatement of ABLATE's finite-volume RHS path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load this library, and only
 * as the checker or as the timed CPU baseline -- never as part of the product path.
 *
 * Parity anchor: every function cites the reference file:line it restates (ABLATE 0.13.03). The
 * restatement is pinned against the reference's own unit-test vectors (tests/golden/*.json, made
 * by tests/golden/make_golden.py from the reference test sources). The PETSc pieces the reference
 * calls but does not contain (PetscFVComputeGradient least squares, PetscLimiterLimit,
 * DMPlexComputeGeometryFVM) and TChem's NASA-7 functions are restated from their published
 * algorithms; the PETSc LSQ gradient is pinned by exactness on linear fields, the limiter forms by
 * the reference's least-squares convergence orders, the NASA-7 functions by the gri30 known answers.
 */
#ifndef ABLATE_ORACLE_H
#define ABLATE_ORACLE_H
#include <stdint.h>
#include "../include/ablate_fv.h"

#ifdef __cplusplus
extern "C" {
#endif

/* flux calculator batch, same meaning as abl_flux_calculator_batch; returns 0 or -5 (Riemann non-convergence) */
int orc_flux_calculator_batch(int kind, double minf, double pgs_alpha, double gamma, int64_t n, const double* uL, const double* aL,
                              const double* rhoL, const double* pL, const double* uR, const double* aR, const double* rhoR,
                              const double* pR, double* mass_flux, double* p12, int32_t* direction);

/* EOS batch, same meaning as abl_eos_batch */
int orc_eos_batch(const abl_physics_desc* physics, int dim, int property, int64_t n, const double* conserved, const double* T_in,
                  double* out);

/* NavierStokesTransport::CompressibleFlowComputeStressTensor (navierStokesTransport.cpp:510-532) */
int orc_stress_tensor(int dim, double mu, const double* grad_vel, double* tau);

/* NavierStokesTransport::AdvectionFlux for one face (navierStokesTransport.cpp:99-207); normal[dim] is the
 * area-weighted normal, fieldL/R the euler field, TL/TR the aux temperature, flux[2+dim] out. */
int orc_ns_advection_flux(const abl_physics_desc* physics, int dim, const double* normal, const double* fieldL, const double* fieldR,
                          double TL, double TR, double* flux);
/* SpeciesTransport::AdvectionFlux for one face (speciesTransport.cpp:263-341), or the species part of
 * CompactCompressibleNSSpeciesTransport::AdvectionFlux when physics->species_advection_compact; fieldL/R
 * the euler + densityYi fields, flux[n_species] out. */
int orc_species_advection_flux(const abl_physics_desc* physics, int dim, const double* normal, const double* fieldL, const double* fieldR,
                               double TL, double TR, double* flux);

/* PetscLimiterLimit restatement for the ABL_LIMITER_* kinds */
double orc_limiter(int kind, double f);

/* Least-squares face weights fg->grad[2][3] (BuildGradientReconstruction_Internal, cellInterpolant.cpp:641-715):
 * out[n_faces][2][3]. Boundary faces get zero weights. */
int orc_lsq_face_weights(const abl_mesh_desc* mesh, double* out);

/* The full RHS: aux update over every local cell (cellSolver.cpp:62-135), then
 * FiniteVolumeSolver::ComputeRHSFunction (finiteVolumeSolver.cpp:233-291) adding into F for owned cells.
 * aux[n_cells][naux] is in/out (in: temperature guess; out: updated aux). threads > 1 runs the
 * per-cell/per-face loops with OpenMP using an owner-computes scatter (deterministic). */
int orc_rhs(const abl_mesh_desc* mesh, const abl_physics_desc* physics, const double* U, double* aux, double* F, int threads);

/* The same split into the one-time setup (LSQ weights, face stencils: what the reference's interpolant
 * constructors do) and the per-evaluation work. The descriptors must outlive the handle. */
void* orc_create(const abl_mesh_desc* mesh, const abl_physics_desc* physics);
int orc_run(void* handle, const double* U, double* aux, double* F, int threads);
void orc_destroy(void* handle);

/* last error text */
const char* orc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
