// Shim: the reference's precompiled-header include resolves here.
#pragma once
#include <cmath>
#include <iostream>
