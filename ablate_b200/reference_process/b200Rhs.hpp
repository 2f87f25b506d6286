// b200Rhs.hpp -- the reference-side drop-in: an ablate::finiteVolume::processes::Process that registers
// one RHSArbitraryFunction computing the finite-volume RHS on a B200 through the C ABI of
// include/ablate_fv.h.
//
// It plugs into ABLATE the way its own processes do (src/finiteVolume/processes/process.hpp:7-20):
// Setup registers the function with FiniteVolumeSolver::RegisterRHSFunction(RHSArbitraryFunction, ctx)
// (src/finiteVolume/finiteVolumeSolver.hpp:32, 155), which ComputeRHSFunction calls after the
// interpolants (src/finiteVolume/finiteVolumeSolver.cpp:285-287); Initialize uploads the local mesh once.
// The physics is read from the reference's own configuration objects:
//   eos::PerfectGas                 GetSpecificHeatRatio(), GetGasConstant(), GetSpeciesVariables()
//   eos::TChem                      GetSpeciesVariables(), GetSpeciesMolecularMass(); its NASA-7 tables are
//                                   private to TChem and come from Options::nasa7 (T_mid, low a1..a7, high
//                                   a1..a7 per species, the mechanism file's "thermo" blocks)
//   fluxCalculator::Ausm, AusmpUp, Riemann, AverageFlux, OffFlux   by type; AusmpUp keeps mInf and its
//                                   pressure-gradient scaling private, so they come from Options
//   eos::transport::Constant        its public GetTransportFunction() evaluated once (k, mu, and D or one
//                                   D per species)
//   eos::transport::Sutherland      by type
// Which fluxes to compute (the NavierStokesTransport / SpeciesTransport / compact process
// registrations) and the PetscFV reconstruction and limiter of the fields come from Options.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "ablate_fv.h"
#include "eos/eos.hpp"
#include "eos/transport/transportModel.hpp"
#include "finiteVolume/finiteVolumeSolver.hpp"
#include "finiteVolume/fluxCalculator/fluxCalculator.hpp"
#include "finiteVolume/processes/process.hpp"

namespace ablate::finiteVolume::processes {

class B200Rhs : public Process {
   public:
    struct Options {
        bool advection = true, diffusion = true, speciesAdvection = true, speciesDiffusion = true;
        bool compactSpeciesAdvection = false;  // CompactCompressibleNSSpeciesTransport's averaged species advection
        std::string reconstruction = "leastsquares";  // petscfv_type of the euler / densityYi fields
        std::string limiter = "none";                  // petsclimiter_type
        double maxLimGrad = 1e10;                      // CompressibleFlowSolver's maxLimGrad
        double mInf = 0.0;                             // AusmpUp reference Mach number
        double pgsAlpha = 1.0;                         // AusmpUp pressure-gradient scaling factor
        std::vector<double> nasa7;                     // TChem: [n_species][15]
        int precision = ABL_PRECISION_FP64;            // ABL_PRECISION_FP64 or ABL_PRECISION_MIXED
        int device = 0;
    };

    // The local mesh of the solver's DM in the descriptor's layout (filled once in Initialize). The
    // arrays are owned here; desc points into them.
    struct LocalMesh {
        int dim = 0, nCells = 0, nFaces = 0;
        std::vector<int32_t> faceCells;
        std::vector<double> faceNormal, faceCentroid, cellCentroid, cellVolume, faceShift;
        std::vector<uint8_t> cellKind;
        abl_mesh_desc Descriptor() const;
    };

    B200Rhs(std::shared_ptr<eos::EOS> eos, std::shared_ptr<fluxCalculator::FluxCalculator> fluxCalculator,
            std::shared_ptr<eos::transport::TransportModel> transport, Options options);
    ~B200Rhs() override;
    B200Rhs(const B200Rhs&) = delete;
    B200Rhs& operator=(const B200Rhs&) = delete;

    void Setup(FiniteVolumeSolver& flow) override;
    void Initialize(FiniteVolumeSolver& flow) override;

    // The descriptor the configuration objects map to (valid for the life of this object).
    const abl_physics_desc& Physics() const { return physics; }

    // The registered function: F += RHS(X) on the rank's local vectors, through abl_fv_rhs_host
    // (with device vectors a caller would use abl_fv_rhs on VecCUDAGetArray pointers instead).
    static PetscErrorCode ComputeRhs(const FiniteVolumeSolver& flow, DM dm, PetscReal time, Vec locX, Vec locF, void* ctx);

   private:
    std::shared_ptr<eos::EOS> eos;
    std::shared_ptr<fluxCalculator::FluxCalculator> fluxCalculator;
    std::shared_ptr<eos::transport::TransportModel> transport;
    Options options;
    abl_physics_desc physics{};
    std::vector<double> nasa7, mw, speciesDiff;  // storage the descriptor points into
    LocalMesh mesh;
    abl_fv* fv = nullptr;
};

// The solver's local mesh (its DM after DMPlexComputeGeometryFVM): implemented with DMPlex calls in an
// ABLATE build (face support, PetscFVFaceGeom / PetscFVCellGeom, the FV ghost label, periodic shifts),
// by a test stand-in elsewhere.
B200Rhs::LocalMesh GetLocalMesh(const FiniteVolumeSolver& flow);

}  // namespace ablate::finiteVolume::processes
