// Shim: the reference's utility.h pulls in headers it does not ship; the
// elasticity element needs only its macros (utility_defines.h, which the
// reference does ship) and the standard headers those macros expand into.
#pragma once
#include <algorithm>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "utility/utility_defines.h"
