// Shim: the part of the interpolation record the heat-transfer material
// reads (the temperature gradient at a point), for the material library.
#pragma once

struct InterpAndSolDerivatives {
  double p_u1_x1 = 0.0, p_u1_x2 = 0.0, p_u1_x3 = 0.0;
};
