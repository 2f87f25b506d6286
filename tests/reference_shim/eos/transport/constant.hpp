// TEST INFRASTRUCTURE ONLY: eos::transport::Constant: constant k, mu and one diffusivity or one per
// species, returned by its transport functions (the behaviour of the reference's
// src/eos/transport/constant.cpp; inactive when all are zero).
#pragma once
#include "eos/transport/transportModel.hpp"
namespace ablate::eos::transport {
class Constant : public TransportModel {
    bool active;
    double k, mu;
    std::vector<double> diff;
    static PetscErrorCode Scalar(const PetscReal*, PetscReal* property, void* ctx) {
        *property = *static_cast<double*>(ctx);
        return 0;
    }
    static PetscErrorCode Vector(const PetscReal*, PetscReal* property, void* ctx) {
        const auto* v = static_cast<std::vector<double>*>(ctx);
        for (size_t i = 0; i < v->size(); i++) property[i] = (*v)[i];
        return 0;
    }

   public:
    Constant(double k, double mu, double diff) : active(k != 0 || mu != 0 || diff != 0), k(k), mu(mu), diff({diff}) {}
    Constant(double k, double mu, std::vector<double> diff) : active(k != 0 || mu != 0 || !diff.empty()), k(k), mu(mu), diff(std::move(diff)) {}
    [[nodiscard]] ThermodynamicFunction GetTransportFunction(TransportProperty property, const std::vector<domain::Field>&) const override {
        if (!active) return {};
        switch (property) {
            case TransportProperty::Conductivity: return {Scalar, std::make_shared<double>(k), 1};
            case TransportProperty::Viscosity: return {Scalar, std::make_shared<double>(mu), 1};
            default:
                if (diff.size() == 1) return {Scalar, std::make_shared<double>(diff[0]), 1};
                return {Vector, std::make_shared<std::vector<double>>(diff), (PetscInt)diff.size()};
        }
    }
};
}  // namespace ablate::eos::transport
