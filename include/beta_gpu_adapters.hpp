/* beta_gpu_adapters.hpp -- BETA's own assembler and matrix interfaces over
 * the C ABI (header-only C++17).
 *
 * BETA plugs a global matrix in through `LargeMatrix` (chosen by a storage
 * token in Equations::setStorageMethod / CreateMatrix, equation.cpp:36-140,
 * 1021-1103) and an assembler through `BasicAssembler` (chosen in
 * BasicModel::createAssembler, BasicModel.cpp:1642-1657).  The reference tree
 * does not ship those class headers, so the two interfaces are declared here
 * with the reference's method names and argument meaning (sparse.cpp:41-48,
 * 80-99, 114-242, 243-248, 452-495; largeMatrix.cpp:43-79;
 * BasicAssembler.cpp:10-35; SerialAssembler.cpp:9-89), and a BETA build
 * derives its `GpuPcgMatrix` / `GpuAssembler` from these adapters.
 *
 *   GPUPCGMatrix : LargeMatrix   -- storage token GPUPCG
 *   GPUAssembler : BasicAssembler -- ParallelAssembly GPU
 *
 * Both share one `Context` (one device context per model, as one Equations
 * object owns one matrix).  Where the reference calls FatalError / exit(1)
 * (sparse.cpp:225-229, largeMatrix.cpp:43-79, BasicElement.cpp:116-130) the
 * adapters throw beta_gpu::Error with the C ABI's status and message.
 */
#pragma once
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "beta_gpu.h"

namespace beta_gpu {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

// ---- the reference's interfaces ---------------------------------------------
// LargeMatrix (sparse.cpp / largeMatrix.cpp): a symmetric global matrix stored
// as its lower triangle, i >= j.
class LargeMatrix {
 public:
  virtual ~LargeMatrix() {}
  virtual double& operator()(int i, int j) = 0;
  virtual void specifyNonZeroLocation(int I, int J) = 0;
  virtual void allocate() = 0;
  virtual void zeroYourself() = 0;
  // Solves A x = b; on return b holds x (sparse.cpp:114-242).  x0: initial guess or null.
  virtual void solve(double* b, double* x0) = 0;
  virtual void vectorProduct(double* y, double* x) = 0;  // y = A x
  virtual void setMAX_NUMBER_ITERATIONS(int n) = 0;
  virtual void setSOLUTION_EPSILON(double eps) = 0;
  virtual int CheckAndFixZeroDiagonal() = 0;
};

// What BasicAssembler::allocateAndInitialize reads from a BasicModel: the
// mesh, the material groups (one group per element when properties vary per
// element, Factory_Material.cpp:30-47) and the Equations' restraints,
// prescribed values and nodal loads (equation.cpp:306-341, 851-868).
struct ModelArrays {
  int kind = 0;  // BETA_GPU_QUAD4_PSTRESS, BETA_GPU_HEX8_ELASTIC, BETA_GPU_HEX8_HEAT, BETA_GPU_QUAD4_HEAT
  int ndim = 0, nnode = 0, nelem = 0, nnpe = 0, ndof_per_node = 0, integration_order = 2;
  const double* xyz = nullptr;     // nnode*ndim
  const int* conn = nullptr;       // nelem*nnpe, BETA local node order
  const int* first_dof = nullptr;  // nnode (Node::firstDof, node-major)
  int ngroups = 0, nparams = 0;
  const double* group_params = nullptr;  // ngroups*nparams in readModuli / PlaneStress::read order
  const int* elem_group = nullptr;       // nelem, or null for one group per element
  const unsigned char* restrained = nullptr;  // ndof
  const double* prescribed = nullptr;         // ndof
  const double* load = nullptr;               // ndof
};

// BasicAssembler (BasicAssembler.cpp, SerialAssembler.cpp).  u: the current
// solution the element updates read (null for a linear K).
class BasicAssembler {
 public:
  virtual ~BasicAssembler() {}
  virtual void allocateAndInitialize(const ModelArrays& model) = 0;
  virtual void makeAssignments(int nDof) = 0;
  virtual void assembleK(double* u) = 0;
  virtual void assembleKandF(double* u) = 0;
  virtual void assembleInitialF() = 0;
  virtual void postAssemblyOperations() = 0;
};

// ---- the B200 implementations -------------------------------------------------
class Context {
 public:
  explicit Context(int device = 0) {
    check(beta_gpu_create(&ctx_, device), "beta_gpu_create");
  }
  ~Context() { beta_gpu_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  beta_gpu_ctx* get() const { return ctx_; }
  void check(int rc, const char* what) const {
    if (rc == BETA_GPU_OK) return;
    std::string msg = std::string(what) + ": ";
    const char* e = ctx_ ? beta_gpu_last_error(ctx_) : nullptr;
    msg += (e && *e) ? e : "error";
    throw Error(rc, msg);
  }
  int ndof = 0;
  long long nnz_lower = 0;
  int precision = BETA_GPU_FP32;  // precision of the last assembly of K
  bool assembled = false;

 private:
  beta_gpu_ctx* ctx_ = nullptr;
};

// GPUAssembler: the Gauss-point loops and the scatter run on the device.
class GPUAssembler : public BasicAssembler {
 public:
  // precision: BETA_GPU_FP32 (for the mixed-precision solve) or BETA_GPU_FP64
  GPUAssembler(Context& c, int precision = BETA_GPU_FP32) : c_(c), precision_(precision) {}

  void allocateAndInitialize(const ModelArrays& m) override {
    beta_gpu_ctx* x = c_.get();
    c_.check(beta_gpu_mesh_upload(x, m.kind, m.ndim, m.nnode, m.xyz, m.nelem, m.nnpe, m.conn, m.first_dof,
                                  m.ndof_per_node, m.integration_order),
             "allocateAndInitialize (mesh)");
    c_.check(beta_gpu_materials_upload(x, m.ngroups, m.nparams, m.group_params, m.elem_group),
             "allocateAndInitialize (materials)");
    c_.ndof = m.nnode * m.ndof_per_node;
    restrained_ = m.restrained;
    prescribed_ = m.prescribed;
    load_ = m.load;
  }
  // Restraints, prescribed values and loads go to the device, then the
  // structure (pattern, colouring, element->slot map) is built.
  void makeAssignments(int nDof) override {
    if (nDof != c_.ndof) throw Error(BETA_GPU_ERR_ARG, "makeAssignments: dof count differs from the mesh");
    c_.check(beta_gpu_bc_upload(c_.get(), restrained_, prescribed_, load_), "makeAssignments (restraints)");
    c_.check(beta_gpu_build_pattern(c_.get(), &c_.nnz_lower), "makeAssignments (structure)");
  }
  void assembleK(double*) override {
    c_.check(beta_gpu_assemble(c_.get(), BETA_GPU_ASM_K, precision_, 0.0, 1.0), "assembleK");
    c_.precision = precision_;
    c_.assembled = true;
  }
  // K, and the internal force f = sum_e K_e u_e into f (ndof, host).
  void assembleKandF(double* u) override {
    assembleK(u);
    if (u && f_) c_.check(beta_gpu_internal_force(c_.get(), u, f_), "assembleKandF");
  }
  void assembleInitialF() override {}
  void postAssemblyOperations() override {}
  void setForceTarget(double* f) { f_ = f; }
  // The pseudo-load Equations::addMatrix accumulates for the symmetric
  // elimination, F[I] -= K_IJ u_J over restrained J (equation.cpp:499-503),
  // here from the FP64 matrix-free operator: out = -(K u_ext) on free dofs,
  // 0 on restrained ones (u_ext = prescribed values on restrained dofs).
  void pseudoLoad(double* out) {
    const int n = c_.ndof;
    std::vector<double> u(n, 0.0), f(n, 0.0);
    for (int i = 0; i < n; ++i) u[i] = restrained_ && restrained_[i] && prescribed_ ? prescribed_[i] : 0.0;
    c_.check(beta_gpu_internal_force(c_.get(), u.data(), f.data()), "pseudoLoad");
    for (int i = 0; i < n; ++i) out[i] = restrained_ && restrained_[i] ? 0.0 : -f[i];
  }

 private:
  Context& c_;
  int precision_;
  const unsigned char* restrained_ = nullptr;
  const double* prescribed_ = nullptr;
  const double* load_ = nullptr;
  double* f_ = nullptr;
};

// GPUPCGMatrix: storage and solve on the device.  The sparsity comes from the
// mesh, so specifyNonZeroLocation is a no-op and allocate() builds nothing
// new; operator() reads a host mirror of the assembled lower triangle (the
// device matrix is written by the assembler, not through this operator).
class GPUPCGMatrix : public LargeMatrix {
 public:
  GPUPCGMatrix(Context& c, int numberOfEquations) : c_(c), n_(numberOfEquations) {
    opts_.mode = BETA_GPU_MODE_MPIR;
    opts_.precond = BETA_GPU_PRECOND_BLOCK_JACOBI;
    opts_.stop_rule = BETA_GPU_STOP_REF;  // sqrt(r.r / x.x) < eps, sparse.cpp:202-223
    opts_.maxit = 10000;                  // sparse.cpp:22-23
    opts_.tol = 1e-4;
    opts_.inner_tol = 0.01;
    opts_.max_outer = 60;
    opts_.use_last_solution = 0;
    opts_.check_every = 0;
    opts_.reserved = 0;
  }
  double& operator()(int i, int j) override {
    if (i < j) throw Error(BETA_GPU_ERR_ARG, "LargeMatrix stores the lower triangle (i >= j)");
    mirror();
    for (long long k = rp_[i]; k < rp_[i + 1]; ++k)
      if (col_[k] == j) return val_[k];
    zero_ = 0.0;
    return zero_;  // not in the pattern
  }
  void specifyNonZeroLocation(int, int) override {}
  void allocate() override {
    if (n_ != c_.ndof) throw Error(BETA_GPU_ERR_ARG, "allocate: equation count differs from the mesh");
  }
  void zeroYourself() override { have_mirror_ = false; }  // every assembly starts from zero
  void solve(double* b, double* x0) override {
    c_.check(c_.assembled ? BETA_GPU_OK : BETA_GPU_ERR_STATE, "solve: assemble K first");
    opts_.mode = c_.precision == BETA_GPU_FP64 ? BETA_GPU_MODE_FP64 : BETA_GPU_MODE_MPIR;
    const int rc = beta_gpu_solve_rhs(c_.get(), b, x0, &opts_, &stats_);
    if (rc == BETA_GPU_MAXIT) throw Error(rc, "Solution not converged...");  // sparse.cpp:225-229
    c_.check(rc, "solve");
    c_.check(beta_gpu_download(c_.get(), b), "solve (download)");
  }
  void vectorProduct(double* y, double* x) override {
    c_.check(beta_gpu_matvec(c_.get(), c_.precision, x, y), "vectorProduct");
  }
  void setMAX_NUMBER_ITERATIONS(int n) override { opts_.maxit = n; }
  void setSOLUTION_EPSILON(double eps) override { opts_.tol = eps; }
  // Negative or zero diagonals are reported by the assembly itself
  // (BETA_GPU_ERR_NEGDIAG / BETA_GPU_ERR_ZERODIAG thrown from assembleK or
  // solve), so nothing is left to fix here.
  int CheckAndFixZeroDiagonal() override { return 0; }

  // Beyond the reference interface: the stop rule, mode and last statistics.
  beta_gpu_solve_opts& options() { return opts_; }
  const beta_gpu_solve_stats& lastStats() const { return stats_; }

 private:
  void mirror() {
    if (have_mirror_) return;
    rp_.assign(n_ + 1, 0);
    col_.assign(c_.nnz_lower, 0);
    val_.assign(c_.nnz_lower, 0.0);
    c_.check(beta_gpu_pattern_lower(c_.get(), rp_.data(), col_.data()), "operator() (pattern)");
    c_.check(beta_gpu_matrix_lower_values(c_.get(), c_.precision, val_.data(), nullptr), "operator() (values)");
    have_mirror_ = true;
  }
  Context& c_;
  int n_;
  beta_gpu_solve_opts opts_{};
  beta_gpu_solve_stats stats_{};
  bool have_mirror_ = false;
  std::vector<long long> rp_;
  std::vector<int> col_;
  std::vector<double> val_;
  double zero_ = 0.0;
};

}  // namespace beta_gpu
