// Project-written stand-in (test infrastructure only).
#pragma once
#include "fixed_size_tensor.hpp"
namespace MATH::MATRIX_T {}
