#pragma once
#include "MathUtils.hpp"
