// TEST INFRASTRUCTURE ONLY: the FiniteVolumeSolver members a process uses to register an arbitrary RHS
// function (the reference's src/finiteVolume/finiteVolumeSolver.hpp:32, 155), and ComputeRHSFunction's
// call of the registered functions (finiteVolumeSolver.cpp:285-287). The local mesh that an ABLATE build
// reads from its DM is held here as plain arrays.
#pragma once
#include <petsc.h>

#include <utility>
#include <vector>

#include "ablate_fv.h"

namespace ablate::finiteVolume {
class FiniteVolumeSolver {
   public:
    using RHSArbitraryFunction = PetscErrorCode (*)(const FiniteVolumeSolver&, DM dm, PetscReal time, Vec locXVec, Vec locFVec, void* ctx);
    void RegisterRHSFunction(RHSArbitraryFunction function, void* context) { rhsArbitraryFunctions.emplace_back(function, context); }
    // every registered function in order, adding into locF
    PetscErrorCode ComputeRHSFunction(PetscReal time, Vec locX, Vec locF) const {
        for (const auto& [fn, ctx] : rhsArbitraryFunctions) {
            PetscErrorCode e = fn(*this, nullptr, time, locX, locF, ctx);
            if (e) return e;
        }
        return PETSC_SUCCESS;
    }
    std::vector<std::pair<RHSArbitraryFunction, void*>> rhsArbitraryFunctions;
    // the stand-in's local mesh (what DMPlex and DMPlexComputeGeometryFVM hold in an ABLATE build)
    abl_mesh_desc mesh{};
};
}  // namespace ablate::finiteVolume
