// Shim: what equation.cpp uses from the reference's utility.h (its macros
// come from the reference's own utility_defines.h); the helper functions are
// defined in ref_equations_api.cpp.
#pragma once
#include <algorithm>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "utility/utility_defines.h"
#include "verbose_level.hpp"

int getLineAndTokenize(std::istream* inStream, char* terminateString, char* tokenList[], int& numberOfTokens);
void displayTime(const char* message, std::ostream& outStream);
std::ifstream* openFileForInput(char* filename);

// Before C++11 a stream inserted into another printed through its void*
// conversion (non-null while good); equation.cpp logs its input streams so.
inline std::ostream& operator<<(std::ostream& os, const std::ifstream& in) {
  return os << (in ? static_cast<const void*>(&in) : static_cast<const void*>(0));
}
