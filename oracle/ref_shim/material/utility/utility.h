// Shim: the two input helpers elastic.cpp calls (their definitions are in
// ref_material_api.cpp) and the reference's own utility macros.
#pragma once
#include <algorithm>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "utility/utility_defines.h"

int getLineAndTokenize(std::istream* inStream, char* terminateString, char* tokenList[], int& numberOfTokens);
void banner(char* string, std::ostream& outStream);
