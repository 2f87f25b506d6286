/* TEST INFRASTRUCTURE ONLY: see petsc.h in this directory. */
#pragma once
#include "petsc.h"
