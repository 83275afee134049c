// Shim: the include path the 2D elasticity element uses for quadQuadPoint.hpp.
#pragma once
#include "../../quadQuadPoint.hpp"
