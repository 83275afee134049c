// Shim: matrix.cpp includes its header by its own directory's name.
#pragma once
#include "math/matrix.hpp"
