// TEST INFRASTRUCTURE ONLY: finiteVolume::processes::Process as declared in the reference's
// src/finiteVolume/processes/process.hpp:7-20.
#pragma once
#include "finiteVolume/finiteVolumeSolver.hpp"
namespace ablate::finiteVolume::processes {
class Process {
   public:
    virtual ~Process() = default;
    virtual void Setup(ablate::finiteVolume::FiniteVolumeSolver& fv) = 0;
    virtual void Initialize(ablate::finiteVolume::FiniteVolumeSolver& fv) {}
};
}  // namespace ablate::finiteVolume::processes
