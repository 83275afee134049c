// Shim: ElasticityElement3D.cpp includes the tensor header but calls nothing
// from it.
#pragma once
