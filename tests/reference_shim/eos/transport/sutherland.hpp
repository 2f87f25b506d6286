// TEST INFRASTRUCTURE ONLY: eos::transport::Sutherland, identified by type only.
#pragma once
#include "eos/transport/transportModel.hpp"
namespace ablate::eos::transport {
class Sutherland : public TransportModel {
   public:
    [[nodiscard]] ThermodynamicFunction GetTransportFunction(TransportProperty, const std::vector<domain::Field>&) const override { return {}; }
};
}  // namespace ablate::eos::transport
