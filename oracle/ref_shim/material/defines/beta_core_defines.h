// Shim: the reference's core defines header includes a header it does not
// ship; elastic.cpp needs none of its declarations.
#pragma once
#define TEMPERATURE 0
#define MOISTURE 1
#define LINEAR 0
#define GEOMETRIC_NONLINEAR 1
