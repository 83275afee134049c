// adapter_check.cpp -- drives the GPU path through BETA's own interfaces, in
// the order BasicModel / Equations call them (BasicModel.cpp:1022-1033,
// 1169-1220; equation.cpp:1288-1405):
//   assembler->allocateAndInitialize; makeAssignments; matrix->allocate;
//   assembler->assembleK; b = load + pseudo-load (prescribed on restrained
//   dofs); matrix->solve(b, x0) -> x in b; matrix->vectorProduct.
// Reads a model written by tests/test_adapters.py, writes the solution and
// probes of the matrix interface.  Exit status: 0 ok, 2 beta_gpu::Error.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>

#include "beta_gpu_adapters.hpp"

template <typename T>
static void rd(std::ifstream& f, std::vector<T>& v, size_t n) {
  v.resize(n);
  f.read(reinterpret_cast<char*>(v.data()), sizeof(T) * n);
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: adapter_check model.bin out.bin\n");
    return 1;
  }
  std::ifstream f(argv[1], std::ios::binary);
  int hdr[12];
  double tol;
  f.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
  f.read(reinterpret_cast<char*>(&tol), sizeof(tol));
  const int kind = hdr[0], ndim = hdr[1], nnode = hdr[2], nelem = hdr[3], nnpe = hdr[4], ndpn = hdr[5],
            order = hdr[6], ngroups = hdr[7], nparams = hdr[8], precision = hdr[9], rule = hdr[10], maxit = hdr[11];
  const int n = nnode * ndpn;
  std::vector<double> xyz, params, presc, load;
  std::vector<int> conn;
  std::vector<unsigned char> rest;
  rd(f, xyz, (size_t)nnode * ndim);
  rd(f, conn, (size_t)nelem * nnpe);
  rd(f, params, (size_t)ngroups * nparams);
  rd(f, rest, (size_t)n);
  rd(f, presc, (size_t)n);
  rd(f, load, (size_t)n);
  if (!f) {
    std::fprintf(stderr, "short model file\n");
    return 1;
  }
  std::vector<int> first(nnode);
  for (int i = 0; i < nnode; ++i) first[i] = ndpn * i;  // Node::setNumDofPerNode, node-major
  try {
    beta_gpu::Context ctx(0);
    beta_gpu::ModelArrays m;
    m.kind = kind; m.ndim = ndim; m.nnode = nnode; m.nelem = nelem; m.nnpe = nnpe; m.ndof_per_node = ndpn;
    m.integration_order = order; m.xyz = xyz.data(); m.conn = conn.data(); m.first_dof = first.data();
    m.ngroups = ngroups; m.nparams = nparams; m.group_params = params.data(); m.elem_group = nullptr;
    m.restrained = rest.data(); m.prescribed = presc.data(); m.load = load.data();

    beta_gpu::GPUAssembler assembler(ctx, precision);
    beta_gpu::GPUPCGMatrix A(ctx, n);
    beta_gpu::LargeMatrix& K = A;
    beta_gpu::BasicAssembler& as = assembler;
    as.allocateAndInitialize(m);
    as.makeAssignments(n);
    K.allocate();
    K.setSOLUTION_EPSILON(tol);
    K.setMAX_NUMBER_ITERATIONS(maxit);
    A.options().stop_rule = rule;
    K.zeroYourself();
    as.assembleK(nullptr);
    if (K.CheckAndFixZeroDiagonal() != 0) return 3;
    // Equations::solve's right-hand side
    std::vector<double> pseudo(n), b(n);
    assembler.pseudoLoad(pseudo.data());
    for (int i = 0; i < n; ++i) b[i] = rest[i] ? presc[i] : load[i] + pseudo[i];
    K.solve(b.data(), nullptr);  // x in b
    // probes: y = A 1, and the diagonal through operator()
    std::vector<double> ones(n, 1.0), y(n, 0.0), diag(n, 0.0);
    K.vectorProduct(y.data(), ones.data());
    for (int i = 0; i < n; ++i) diag[i] = K(i, i);
    std::ofstream o(argv[2], std::ios::binary);
    const int it = A.lastStats().iterations;
    o.write(reinterpret_cast<const char*>(&it), sizeof(it));
    o.write(reinterpret_cast<const char*>(b.data()), sizeof(double) * n);
    o.write(reinterpret_cast<const char*>(y.data()), sizeof(double) * n);
    o.write(reinterpret_cast<const char*>(diag.data()), sizeof(double) * n);
    o.write(reinterpret_cast<const char*>(pseudo.data()), sizeof(double) * n);
  } catch (const beta_gpu::Error& e) {
    std::fprintf(stderr, "beta_gpu::Error %d: %s\n", e.status(), e.what());
    return 2;
  }
  return 0;
}
