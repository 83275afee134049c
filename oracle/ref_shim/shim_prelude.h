// Force-included before each reference translation unit compiled into
// oracle/_ref.  The reference ships no headers; these shims declare just what
// gauss.cpp and shape.cpp need so they compile unmodified.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
using namespace std;
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
