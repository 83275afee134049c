// Shim: the include path the diffusion elements use for hexQuadPoint.hpp.
#pragma once
#include "../../hexQuadPoint.hpp"
