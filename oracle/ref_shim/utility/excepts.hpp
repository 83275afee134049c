// Shim: the reference's error-handling macros, reduced to what sparse.cpp,
// largeMatrix.cpp, equation.cpp and addeqn.cpp need (fatal errors and range
// violations abort the test program).
#pragma once
#include <cstdlib>
#include <iostream>
#define CreateErrorHandler(cls)
#define WhoClass(x)
#define WhoMethod(x)
#define DeleteWhoMethod(x)
#define DEBUG3(x)
#define Assert(x) do { if (!(x)) { std::cerr << "allocation failed\n"; std::abort(); } } while (0)
#define FatalError(msg) do { std::cerr << (msg) << '\n'; std::abort(); } while (0)
#define Warning(msg) (std::cerr << (msg) << '\n')
#define RangeCheck(lo, v, hi) \
  do { if ((v) < (lo) || (v) > (hi)) { std::cerr << "range check failed: " << (v) << '\n'; std::abort(); } } while (0)
