// TEST INFRASTRUCTURE ONLY: eos::TChem with the public accessors of the reference's src/eos/tChem.hpp:105
// and tChemBase.hpp:96 (species list, molar masses); the mechanism itself is not modelled.
#pragma once
#include "eos/eos.hpp"
namespace ablate::eos {
class TChem : public EOS {
    std::vector<std::string> species;
    std::vector<double> masses;

   public:
    TChem(std::vector<std::string> species, std::vector<double> masses) : species(std::move(species)), masses(std::move(masses)) {}
    [[nodiscard]] const std::vector<std::string>& GetSpeciesVariables() const override { return species; }
    [[nodiscard]] std::map<std::string, double> GetSpeciesMolecularMass() const {
        std::map<std::string, double> m;
        for (size_t k = 0; k < species.size(); k++) m[species[k]] = masses[k];
        return m;
    }
};
}  // namespace ablate::eos
