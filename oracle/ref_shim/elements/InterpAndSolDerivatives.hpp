// Shim: the interpolation record lives in the shared element shim.
#pragma once
#include "element_shim_common.hpp"
