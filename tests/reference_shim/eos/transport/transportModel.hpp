// TEST INFRASTRUCTURE ONLY: eos::transport::TransportModel as declared in the reference's
// src/eos/transport/transportModel.hpp (TransportProperty, GetTransportFunction).
#pragma once
#include "eos/eos.hpp"
namespace ablate::eos::transport {
enum class TransportProperty { Conductivity, Viscosity, Diffusivity };
class TransportModel {
   public:
    virtual ~TransportModel() = default;
    [[nodiscard]] virtual ThermodynamicFunction GetTransportFunction(TransportProperty property, const std::vector<domain::Field>& fields) const = 0;
};
}  // namespace ablate::eos::transport
