// TEST INFRASTRUCTURE ONLY: eos::PerfectGas with the public accessors of the reference's
// src/eos/perfectGas.hpp:93-99, 130 (gamma, R and the species list).
#pragma once
#include "eos/eos.hpp"
namespace ablate::eos {
class PerfectGas : public EOS {
    PetscReal gamma, rGas;
    std::vector<std::string> species;

   public:
    PerfectGas(PetscReal gamma, PetscReal rGas, std::vector<std::string> species = {}) : gamma(gamma), rGas(rGas), species(std::move(species)) {}
    [[nodiscard]] PetscReal GetSpecificHeatRatio() const { return gamma; }
    [[nodiscard]] PetscReal GetGasConstant() const { return rGas; }
    [[nodiscard]] const std::vector<std::string>& GetSpeciesVariables() const override { return species; }
};
}  // namespace ablate::eos
