// b200Rhs.cpp -- the B200Rhs process (declared in b200Rhs.hpp): the reference's configuration objects
// mapped onto abl_physics_desc, the RHSArbitraryFunction registration, and the RHS call through the C ABI.
#include "b200Rhs.hpp"

#include <algorithm>
#include <stdexcept>

#include "eos/perfectGas.hpp"
#include "eos/tChem.hpp"
#include "eos/transport/constant.hpp"
#include "eos/transport/sutherland.hpp"
#include "finiteVolume/fluxCalculator/ausm.hpp"
#include "finiteVolume/fluxCalculator/ausmpUp.hpp"
#include "finiteVolume/fluxCalculator/averageFlux.hpp"
#include "finiteVolume/fluxCalculator/offFlux.hpp"
#include "finiteVolume/fluxCalculator/riemann.hpp"

namespace ablate::finiteVolume::processes {

namespace {

int LimiterCode(const std::string& name) {
    // PetscLimiter type names (petsclimiter_type)
    if (name == "none" || name.empty()) return ABL_LIMITER_NONE;
    if (name == "zero") return ABL_LIMITER_ZERO;
    if (name == "minmod") return ABL_LIMITER_MINMOD;
    if (name == "vanleer") return ABL_LIMITER_VANLEER;
    if (name == "vanalbada") return ABL_LIMITER_VANALBADA;
    if (name == "sin") return ABL_LIMITER_SIN;
    throw std::invalid_argument("B200Rhs: limiter '" + name + "' has no device counterpart");
}

int ReconstructionCode(const std::string& name) {
    // PetscFV type names (petscfv_type)
    if (name == "upwind") return ABL_RECON_UPWIND;
    if (name == "leastsquares") return ABL_RECON_LEASTSQUARES;
    throw std::invalid_argument("B200Rhs: PetscFV type '" + name + "' has no device counterpart");
}

// value of a transport property through the model's public function (null function: inactive, 0)
std::vector<double> TransportValue(const eos::transport::TransportModel& model, eos::transport::TransportProperty property) {
    const eos::ThermodynamicFunction fn = model.GetTransportFunction(property, {});
    std::vector<double> out((size_t)std::max<PetscInt>(fn.propertySize, 1), 0.0);
    if (fn.function) {
        // the Constant model ignores the conserved state
        const std::vector<PetscReal> conserved(64, 0.0);
        if (fn.function(conserved.data(), out.data(), fn.context.get()) != 0) throw std::runtime_error("B200Rhs: transport function failed");
    }
    return out;
}

}  // namespace

abl_mesh_desc B200Rhs::LocalMesh::Descriptor() const {
    abl_mesh_desc d{};
    d.dim = dim;
    d.n_cells = nCells;
    d.n_faces = nFaces;
    d.face_cells = faceCells.data();
    d.face_normal = faceNormal.data();
    d.face_centroid = faceCentroid.data();
    d.cell_centroid = cellCentroid.data();
    d.cell_volume = cellVolume.data();
    d.cell_kind = cellKind.empty() ? nullptr : cellKind.data();
    d.face_shift = faceShift.empty() ? nullptr : faceShift.data();
    return d;
}

B200Rhs::B200Rhs(std::shared_ptr<eos::EOS> eosIn, std::shared_ptr<fluxCalculator::FluxCalculator> fluxIn,
                 std::shared_ptr<eos::transport::TransportModel> transportIn, Options optionsIn)
    : eos(std::move(eosIn)), fluxCalculator(std::move(fluxIn)), transport(std::move(transportIn)), options(std::move(optionsIn)) {
    if (!eos) throw std::invalid_argument("B200Rhs: an EOS is required");
    const std::vector<std::string>& species = eos->GetSpeciesVariables();
    const int ns = (int)species.size();
    physics.n_species = ns;

    // equation of state
    if (auto perfectGas = std::dynamic_pointer_cast<eos::PerfectGas>(eos)) {
        physics.eos = ABL_EOS_PERFECT_GAS;
        physics.gamma = perfectGas->GetSpecificHeatRatio();
        physics.r_gas = perfectGas->GetGasConstant();
    } else if (auto tChem = std::dynamic_pointer_cast<eos::TChem>(eos)) {
        physics.eos = ABL_EOS_NASA7;
        const std::map<std::string, double> masses = tChem->GetSpeciesMolecularMass();
        mw.resize(ns);
        for (int k = 0; k < ns; k++) mw[k] = masses.at(species[k]);
        if (options.nasa7.size() != 15 * (size_t)ns)
            throw std::invalid_argument("B200Rhs: the TChem EOS needs 15 NASA-7 coefficients per species in Options::nasa7");
        nasa7 = options.nasa7;
        physics.nasa7 = nasa7.data();
        physics.mw = mw.data();
    } else {
        throw std::invalid_argument("B200Rhs: the EOS must be eos::PerfectGas or eos::TChem");
    }

    // flux calculator
    if (!fluxCalculator || std::dynamic_pointer_cast<fluxCalculator::OffFlux>(fluxCalculator)) {
        physics.flux = ABL_FLUX_OFF;
    } else if (std::dynamic_pointer_cast<fluxCalculator::Ausm>(fluxCalculator)) {
        physics.flux = ABL_FLUX_AUSM;
    } else if (std::dynamic_pointer_cast<fluxCalculator::AusmpUp>(fluxCalculator)) {
        physics.flux = ABL_FLUX_AUSMPUP;
        physics.ausmpup_minf = options.mInf;
        physics.pgs_alpha = options.pgsAlpha;
    } else if (std::dynamic_pointer_cast<fluxCalculator::Riemann>(fluxCalculator)) {
        physics.flux = ABL_FLUX_RIEMANN;
    } else if (std::dynamic_pointer_cast<fluxCalculator::AverageFlux>(fluxCalculator)) {
        physics.flux = ABL_FLUX_AVERAGE;
    } else {
        throw std::invalid_argument("B200Rhs: the flux calculator has no device counterpart");
    }

    // reconstruction of the conserved fields
    physics.reconstruction = ReconstructionCode(options.reconstruction);
    physics.limiter = LimiterCode(options.limiter);
    physics.max_lim_grad = options.maxLimGrad;

    // transport
    if (!transport) {
        physics.transport = ABL_TRANSPORT_NONE;
    } else if (std::dynamic_pointer_cast<eos::transport::Sutherland>(transport)) {
        physics.transport = ABL_TRANSPORT_SUTHERLAND;
    } else if (std::dynamic_pointer_cast<eos::transport::Constant>(transport)) {
        physics.transport = ABL_TRANSPORT_CONSTANT;
        physics.k = TransportValue(*transport, eos::transport::TransportProperty::Conductivity)[0];
        physics.mu = TransportValue(*transport, eos::transport::TransportProperty::Viscosity)[0];
        const std::vector<double> diff = TransportValue(*transport, eos::transport::TransportProperty::Diffusivity);
        if (diff.size() == 1) {
            physics.diff = diff[0];
        } else {
            // one diffusivity per species: SpeciesTransport registers the VariableDiffusionCoefficient fluxes
            if ((int)diff.size() != ns) throw std::invalid_argument("B200Rhs: the diffusivity vector must have one entry per species");
            speciesDiff = diff;
            physics.species_diff = speciesDiff.data();
        }
    } else {
        throw std::invalid_argument("B200Rhs: the transport model has no device counterpart");
    }

    // the fluxes the replaced processes register
    physics.advection = options.advection;
    physics.diffusion = options.diffusion;
    physics.species_advection = ns > 0 && options.speciesAdvection;
    physics.species_diffusion = ns > 0 && options.speciesDiffusion;
    physics.species_advection_compact = options.compactSpeciesAdvection;
}

B200Rhs::~B200Rhs() {
    if (fv) abl_fv_destroy(fv);
}

void B200Rhs::Setup(FiniteVolumeSolver& flow) { flow.RegisterRHSFunction(ComputeRhs, this); }

void B200Rhs::Initialize(FiniteVolumeSolver& flow) {
    mesh = GetLocalMesh(flow);
    const abl_mesh_desc desc = mesh.Descriptor();
    if (fv) abl_fv_destroy(fv);
    fv = nullptr;
    if (abl_fv_create(&desc, &physics, options.device, &fv) != ABL_OK) {
        fv = nullptr;
        throw std::runtime_error(std::string("B200Rhs: ") + abl_last_error_string());
    }
}

PetscErrorCode B200Rhs::ComputeRhs(const FiniteVolumeSolver&, DM, PetscReal time, Vec locX, Vec locF, void* ctx) {
    PetscFunctionBeginUser;
    auto* self = static_cast<B200Rhs*>(ctx);
    if (!self->fv) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_WRONGSTATE, "B200Rhs: the process was not initialized");
    const PetscScalar* x = nullptr;
    PetscScalar* f = nullptr;
    PetscCall(VecGetArrayRead(locX, &x));
    PetscCall(VecGetArray(locF, &f));
    int rc = abl_fv_rhs_host(self->fv, time, x, f, self->options.precision);
    if (rc == ABL_OK) rc = abl_fv_status(self->fv);  // device conditions: NaN, EOS iteration cap, Riemann
    PetscCall(VecRestoreArray(locF, &f));
    PetscCall(VecRestoreArrayRead(locX, &x));
    if (rc != ABL_OK) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_LIB, "B200 RHS failed (%d): %s", rc, abl_last_error_string());
    PetscFunctionReturn(PETSC_SUCCESS);
}

}  // namespace ablate::finiteVolume::processes
