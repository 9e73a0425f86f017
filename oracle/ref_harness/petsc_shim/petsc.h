#pragma once
#include "petsc_shim_impl.h"
