/*
 * beta_gpu.h -- C ABI of the B200 element-assembly + PCG path for BETA.
 *
 * This library replaces, behind BETA's own interfaces, the hot path
 *   SerialAssembler/ESA_Assembler::assembleK  (beta/assemblers/SerialAssembler.cpp:35-59,
 *                                              beta/assemblers/ESA_Assembler.cpp:9-68)
 *   Element::update("K"|"F"|"KM")             (beta/elements/3D/ElasticityElement3D.cpp:1032-1051,
 *                                              beta_ext/diffusion/element/HeatTransferElement3DTransient.cpp:707-767)
 *   Equations::addMatrix / specifyNonZeroLocation / solve
 *                                             (beta/math/equation/equation.cpp:445-562, 1216-1267, 1288-1405)
 *   SymmetricSparseMatrix::solve / vectorProduct (beta/math/equation/sparse.cpp:114-242, 452-478)
 * with hand-written sm_100a kernels.  Every call is plain C: host pointers,
 * sizes and opaque handles; no CUDA or framework types cross the boundary
 * except in the explicitly device-pointer entry points, whose names say so.
 *
 * Conventions
 *   - Every function returns an int status (BETA_GPU_OK == 0).  Nothing calls
 *     exit(); beta_gpu_last_error() returns a message for the last failure.
 *   - Host pointers are only read (or written) during the call.
 *   - All device work of a context runs on the context's own stream, in order.
 *   - DOF numbering is BETA's: dof(node, j) = first_dof[node] + j
 *     (BasicElement::calculateDofList, beta/elements/BasicElement.cpp:49-68;
 *     Node::setNumDofPerNode, beta/mesh/node.cpp:158-227).  The block
 *     layouts require the uniform node-major numbering first_dof[i] = ndpn*i
 *     that "SetNumDofPerNode <n> all" produces.
 */
#ifndef BETA_GPU_H
#define BETA_GPU_H

#if defined(__GNUC__)
#define BETA_GPU_API __attribute__((visibility("default")))
#else
#define BETA_GPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  BETA_GPU_OK = 0,
  BETA_GPU_ERR_ARG = 1,          /* bad argument / size                                  */
  BETA_GPU_ERR_CUDA = 2,         /* CUDA runtime error (message in last_error)           */
  BETA_GPU_ERR_STATE = 3,        /* call out of order (e.g. solve before assemble)       */
  BETA_GPU_MAXIT = 4,            /* PCG hit max iterations (sparse.cpp:225-229)          */
  BETA_GPU_BREAKDOWN = 5,        /* p.Ap <= 0 or non-finite scalar in PCG                */
  BETA_GPU_ERR_NEGDIAG = 6,      /* element/global diagonal <= 0 (BasicElement.cpp:116-130) */
  BETA_GPU_ERR_ZERODIAG = 7,     /* zero global diagonal (largeMatrix.cpp:43-79)         */
  BETA_GPU_ERR_OOM = 8,          /* device allocation failed                             */
  BETA_GPU_REJECTED = 9,         /* admission refused (HBM budget)                       */
  BETA_GPU_TIMEOUT = 10,         /* bounded device wait expired                          */
  BETA_GPU_ERR_NOT_FINITE = 11,  /* NaN/Inf in inputs                                    */
  BETA_GPU_ERR_LOAD_ON_RESTRAINED = 12, /* equation.cpp:858-861                          */
  BETA_GPU_ERR_UNSUPPORTED = 13, /* layout or element kind not supported                 */
  BETA_GPU_ERR_TOO_LARGE = 14    /* size above a fixed capacity (see the no-alloc solver) */
};

/* ---- element / material kinds ------------------------------------------ */
enum {
  /* ElasticityElement2D quad4 + PlaneStress material: 4 params per group
     (E11, E22, nu12, G12) as PlaneStress::read takes them (pStress.cpp:49-85). */
  BETA_GPU_QUAD4_PSTRESS = 1,
  /* ElasticityElement3D hex8 + ElasticMaterial "readModuli": 9 params per group
     (E11, E22, E33, nu12, nu23, nu13, G12, G23, G13) (elastic.cpp:335-370). */
  BETA_GPU_HEX8_ELASTIC = 2,
  /* HeatTransferElement3Dtransient hex8 + HeatTransferMaterial: 4 params per
     group (k11, k22, k33, capacity c) (heatTransferMaterial.cpp:89-92). */
  BETA_GPU_HEX8_HEAT = 3,
  /* HeatTransferElement2Dtransient quad4 (HeatTransferElement2DTransient.cpp:
     67-108) + the same material and 4 params; k11 and k22 act in the plane
     (k12 = 0 for the unrotated orthotropic material), unit thickness.  Single
     systems only (steady solves and beta_gpu_heat_run), not batches. */
  BETA_GPU_QUAD4_HEAT = 4
};

/* ---- what to assemble (Element::update action letters) ------------------ */
enum {
  BETA_GPU_ASM_K = 1,      /* "K": stiffness / conductivity                           */
  BETA_GPU_ASM_MBAR = 2,   /* "KM" + formK_s: Mbar = (a1*K + M)/dt (DiffusionModel.cpp:322-347) */
  BETA_GPU_ASM_TANGENT = 3 /* "K" with analysisType GEOMETRIC_NONLINEAR at the current solution
                              (hex8 elasticity; ElasticityElement3D.cpp:84-119, 560-641)          */
};

/* ---- precision of the assembled matrix ---------------------------------- */
enum {
  BETA_GPU_FP64 = 0,       /* scalar FP64 sliced-ELL (plain FP64 PCG)                  */
  BETA_GPU_FP32 = 1        /* node-block FP32 sliced-ELL (mixed-precision inner PCG)   */
};

/* ---- solver options ------------------------------------------------------ */
enum {
  BETA_GPU_MODE_FP64 = 0,  /* plain FP64 Jacobi-PCG on the FP64 matrix                 */
  BETA_GPU_MODE_MPIR = 1   /* FP32 inner PCG + FP64 matrix-free outer residual/update  */
};
enum {
  BETA_GPU_PRECOND_JACOBI = 0,       /* z = r / diag (sparse.cpp:165, 192)            */
  BETA_GPU_PRECOND_BLOCK_JACOBI = 1  /* z = inv(D_node) r, per-node ndpn x ndpn block */
};
enum {
  BETA_GPU_STOP_REF = 0,   /* sqrt(r.r / x.x) < tol, the reference rule (sparse.cpp:202-223) */
  BETA_GPU_STOP_RB = 1     /* ||b - A x|| / ||b|| < tol                                      */
};

typedef struct beta_gpu_solve_opts {
  int mode;          /* BETA_GPU_MODE_*                                              */
  int precond;       /* BETA_GPU_PRECOND_* (MPIR inner solve; FP64 mode uses JACOBI) */
  int stop_rule;     /* BETA_GPU_STOP_*                                              */
  int maxit;         /* max PCG iterations (FP64) / max total inner iterations (MPIR) */
  double tol;        /* outer tolerance (FP64: PCG tolerance)                        */
  double inner_tol;  /* MPIR: relative residual reduction of each inner solve         */
  int max_outer;     /* MPIR: max refinement steps                                   */
  int use_last_solution; /* start from the previous solution (Equations::lastSolution) */
  int check_every;   /* host convergence poll interval in iterations (0 = default)   */
  int reserved;
} beta_gpu_solve_opts;

typedef struct beta_gpu_solve_stats {
  int status;             /* BETA_GPU_OK / MAXIT / BREAKDOWN ...                    */
  int iterations;         /* total PCG iterations (MPIR: sum of inner iterations)   */
  int outer_iterations;   /* MPIR refinement steps                                  */
  int reserved;
  double final_norm;      /* last value of the stop-rule quantity                   */
  double true_rel_residual; /* ||b - A x|| / ||b|| in FP64 at exit                  */
  double ms_solve;        /* device time of the solve (CUDA events)                 */
  double ms_spmv_avg;     /* average device time of one SpMV launch (if measured)   */
} beta_gpu_solve_stats;

typedef struct beta_gpu_ctx beta_gpu_ctx;

/* ---- lifetime ----------------------------------------------------------- */
/* Creates a context bound to CUDA device `device` with its own stream. */
BETA_GPU_API int beta_gpu_create(beta_gpu_ctx** ctx, int device);
BETA_GPU_API int beta_gpu_destroy(beta_gpu_ctx* ctx);
BETA_GPU_API const char* beta_gpu_last_error(const beta_gpu_ctx* ctx);
/* Library/ABI version: major*10000 + minor*100 + patch. */
BETA_GPU_API int beta_gpu_version(void);

/* Runs the context's device work on a caller-owned cudaStream_t (passed as
 * void*; NULL restores the context's own stream).  The caller keeps the
 * stream alive while the context uses it. */
BETA_GPU_API int beta_gpu_set_stream(beta_gpu_ctx* ctx, void* stream);
/* Cumulative counters since creation: out[0] kernel launches, out[1] bytes
 * copied host->device, out[2] bytes copied device->host.  n <= 3. */
BETA_GPU_API int beta_gpu_counters(const beta_gpu_ctx* ctx, long long* out, int n);

/* ---- model upload (BasicMesh::ReadMesh / SetElementProperty / loads) ----- */
/* Every upload copies its host input before it returns (the caller may reuse
 * the buffer at once): pinned inputs directly, pageable ones of 4 MiB or more
 * through a 64 MiB pinned staging buffer allocated once per device and kept
 * for the process, shared by the contexts on that device. */
/* Mesh: ndim 2|3, xyz[nnode*ndim] (node-major), conn[nelem*nnpe] in BETA
 * local node order (BasicElement.cpp:464-467, 518-525), first_dof[nnode].
 * `kind` fixes the element formulation; `integration_order` is the Gauss order
 * per direction (IsoElement::setIntegrationOrder, isoElement.cpp:463-478). */
BETA_GPU_API int beta_gpu_mesh_upload(beta_gpu_ctx* ctx, int kind, int ndim, int nnode, const double* xyz,
                         int nelem, int nnpe, const int* conn, const int* first_dof,
                         int ndof_per_node, int integration_order);

/* Materials as groups (BasicModel::SetElementProperty, BasicModel.cpp:682-748):
 * group_params[ngroups*nparams] (nparams per kind, see above) and
 * elem_group[nelem] (NULL: group index = element index). */
BETA_GPU_API int beta_gpu_materials_upload(beta_gpu_ctx* ctx, int ngroups, int nparams,
                              const double* group_params, const int* elem_group);

/* Boundary conditions over ndof dofs (Equations::setRestraint/setSolution/
 * addLoadToEqn, equation.cpp:306-341, 851-868): restrained[ndof] (0/1),
 * prescribed[ndof] (used where restrained), load[ndof] (nodal loads). */
BETA_GPU_API int beta_gpu_bc_upload(beta_gpu_ctx* ctx, const unsigned char* restrained,
                       const double* prescribed, const double* load);

/* ---- structure ---------------------------------------------------------- */
/* Builds the node graph, element colouring, element->slot map and the
 * sliced-ELL layouts (Equations::specifyNonZeroLocation + allocate,
 * equation.cpp:1216-1280; sparse.cpp:479-495).  Returns the number of stored
 * lower-triangle entries of the reference layout in *nnz_lower. */
BETA_GPU_API int beta_gpu_build_pattern(beta_gpu_ctx* ctx, long long* nnz_lower);

/* Column storage of the FP32 node-block matrix (no counterpart in the
 * reference, whose matrices are FP64 compressed rows).  run = 3 (the default)
 * lets the build store one column index per run of up to three consecutive
 * node columns, the 9 runs of 3 that a 27-block row of a lexicographically
 * numbered hex mesh holds, when that makes the FP32 matrix at least 5 %
 * smaller (e.g. 216 -> 144 bytes per row with one dof per node); run = 1
 * keeps one index per block.  The values, and every sum of the solves, are
 * the same either way.  Takes effect at the next beta_gpu_build_pattern (a
 * built pattern is dropped when the value changes). */
BETA_GPU_API int beta_gpu_set_block_runs(beta_gpu_ctx* ctx, int run);
/* FP64 element matrices of the hex8 diffusion operator kept on the device (no
 * counterpart in the reference, which integrates its elements at every
 * assembly).  With on = 1 (the default) the first FP64 operator use after a
 * mesh, material or pattern change integrates K_e and M_e of every element
 * once (72 doubles per element, built only when they fit in a quarter of the
 * free device memory), and the FP64 residuals of mixed-precision solves and
 * the transient right-hand sides read them instead of integrating again;
 * on = 0 integrates at every use.  Results agree to rounding. */
BETA_GPU_API int beta_gpu_set_operator_cache(beta_gpu_ctx* ctx, int on);
/* The layout built: out[0] run length (1 or 3), out[1] value chunks of 32
 * blocks, out[2] column indices the SpMV reads (4 bytes each), out[3] bytes
 * of values and columns, out[4] 1 when the runs are in their compact form (a
 * slice of 32 rows whose runs all sit at the same offsets from their rows --
 * one inside an x-row of a structured mesh -- stores those offsets once, not
 * 32 columns per run: 21 % less matrix with one dof per node on a
 * 256x256x64 slab).  n <= 5.  BETA_GPU_ERR_STATE before the pattern is
 * built. */
BETA_GPU_API int beta_gpu_block_layout(const beta_gpu_ctx* ctx, long long* out, int n);

/* Exports the lower-triangle pattern exactly as SymmetricSparseMatrix stores
 * it: row_ptr[ndof+1], col[nnz_lower], columns ascending, diagonal last. */
BETA_GPU_API int beta_gpu_pattern_lower(beta_gpu_ctx* ctx, long long* row_ptr, int* col);

/* Host-only form of the structure step (no device needed): the reference's
 * lower-triangle pattern for a mesh and restraint mask.  Call with
 * row_ptr == col == NULL to get *nnz_lower, then again with row_ptr[ndof+1]
 * and col[*nnz_lower].  Same layout as beta_gpu_pattern_lower. */
BETA_GPU_API int beta_gpu_pattern_lower_host(int nnode, int nelem, int nnpe, int ndof_per_node,
                                             const int* conn, const int* first_dof,
                                             const unsigned char* restrained, long long* nnz_lower,
                                             long long* row_ptr, int* col);

/* ---- assembly ------------------------------------------------------------ */
/* Assembles the global matrix in `precision` (zeroMatrix + element loop +
 * addMatrix).  what = BETA_GPU_ASM_K (static) or BETA_GPU_ASM_MBAR with
 * a1 = alpha*dt (DiffusionModel.cpp:745-746).  In FP64 the pseudo-load of
 * restrained columns is formed as Equations::addMatrix does. */
BETA_GPU_API int beta_gpu_assemble(beta_gpu_ctx* ctx, int what, int precision, double dt, double alpha);

/* Exports the assembled lower-triangle values in the pattern_lower order (FP32
 * values are widened) and, for FP64 assembly, the pseudo-load vector. */
BETA_GPU_API int beta_gpu_matrix_lower_values(beta_gpu_ctx* ctx, int precision, double* vals,
                                 double* pseudo_load);

/* Equations::setReplaceZeroDiagonal_Option, the ReplaceZeroDiagonal command
 * (equation.cpp:1819-1823), as LargeMatrix::CheckAndFixZeroDiagonal applies
 * it when a solve starts (largeMatrix.cpp:43-79, sparse.cpp:127): with value
 * 0 (the default) a zero global diagonal is refused (BETA_GPU_ERR_ZERODIAG,
 * where the reference exits); with any other value every zero diagonal of
 * the assembled matrix the solve uses (FP64, or FP32 for mixed precision,
 * whose FP64 residual operator gets the same entry) becomes value before the
 * solve, and stays so until the next assembly.  A negative diagonal below the
 * first zero one is refused either way (BETA_GPU_ERR_NEGDIAG). */
BETA_GPU_API int beta_gpu_set_zero_diagonal(beta_gpu_ctx* ctx, double value);

/* ---- solve --------------------------------------------------------------- */
/* Equations::solve: right-hand side = load + pseudo-load on free dofs,
 * prescribed values on restrained dofs; then PCG per opts.  The solution stays
 * on the device until beta_gpu_download. */
BETA_GPU_API int beta_gpu_solve(beta_gpu_ctx* ctx, const beta_gpu_solve_opts* opts,
                   beta_gpu_solve_stats* stats);
BETA_GPU_API int beta_gpu_download(beta_gpu_ctx* ctx, double* u);
/* LargeMatrix::solve(b, x0) on the assembled system (sparse.cpp:114-242):
 * b (host, ndof) is the eliminated right-hand side -- load + pseudo-load on
 * free dofs, the prescribed value on restrained ones, as Equations::solve
 * forms it (equation.cpp:1288-1405) -- and x0 (host, ndof, may be NULL) the
 * initial guess.  Same opts, stats and status as beta_gpu_solve; the solution
 * is read with beta_gpu_download. */
BETA_GPU_API int beta_gpu_solve_rhs(beta_gpu_ctx* ctx, const double* b, const double* x0,
                                    const beta_gpu_solve_opts* opts, beta_gpu_solve_stats* stats);

/* y = A x with the assembled matrix of `precision` (SymmetricSparseMatrix::
 * vectorProduct, sparse.cpp:452-478), host vectors of length ndof. */
BETA_GPU_API int beta_gpu_matvec(beta_gpu_ctx* ctx, int precision, const double* x, double* y);

/* Internal force f = K_e u summed over elements in FP64, matrix-free
 * (BasicModel::CalculateResidual, BasicModel.cpp:1035-1061, without the
 * restrained-row skip): host u[ndof] -> host f[ndof]. */
BETA_GPU_API int beta_gpu_internal_force(beta_gpu_ctx* ctx, const double* u, double* f);

/* ---- mesh files ------------------------------------------------------------ */
/* BETA's mesh files, text (BasicMesh::ReadMesh, BasicMesh.cpp:79-190, with the
 * processCommands / setCoordinateReadOption block) or binary (ReadMeshBinary,
 * :192-268).  Returns xyz (nnode x ndim) and the connectivity as 0-based node
 * indices in BETA's local order (node numbers may start at 0 or 1), elements
 * in ascending element number; all elements must share nnpe
 * (BETA_GPU_ERR_UNSUPPORTED otherwise).  Call with xyz/conn NULL for the
 * sizes, then with arrays.  Host only. */
BETA_GPU_API int beta_gpu_read_mesh(const char* path, int binary, int* ndim, int* nnode, int* nelem, int* nnpe,
                                    double* xyz, int* conn);
/* Writes a mesh in the same layouts, numbering nodes and elements from
 * first_number (0 or 1). */
BETA_GPU_API int beta_gpu_write_mesh(const char* path, int binary, int ndim, int nnode, const double* xyz, int nelem,
                                     int nnpe, const int* conn, int first_number);

/* ---- material groups of an input deck -------------------------------------- */
/* The body of a setElementMaterial block (BasicModel::ProcessSetElementProperty,
 * BasicModel.cpp:682-775): lines "first last increment group" or
 * "all group", blank/tab separated, with // and slash-star comments, ended
 * by a line "end" (any case) or a negative first element.  Sets
 * elem_group[e] for the elements named (others keep their value), in line
 * order; *nlines (may be NULL) receives the number of lines applied.
 * BETA_GPU_ERR_ARG for a malformed line, last >= nelem (the reference
 * accepts last == numElements and writes past its element array), a line of
 * 2-3 tokens that is not "all" (the reference reads undefined values), or an
 * unpaired comment.  The map feeds beta_gpu_materials_upload's elem_group.
 * Host only. */
BETA_GPU_API int beta_gpu_parse_element_groups(const char* text, int nelem, int* elem_group, int* nlines);

/* ---- surface flux loads ---------------------------------------------------- */
/* SurfaceLoad::applyTo (beta/BCs/SurfaceLoad.cpp:16-255) without its
 * shared-memory coupling: for each of nsurf surface faces (node ids into the
 * model's nodes, nodes_per_face 4 or 8 = quadrilateral, 6 = triangle, node
 * orders of shape.cpp's shapeQuad4 / shapeQuad8 / shapeTri6) the nodal flux
 * is interpolated to the integration points (3x3 Gauss on quadrilaterals,
 * 7 points on triangles), scaled by |dx/dxi x dx/deta| and its consistent
 * nodal loads are ADDED to load[first_dof[node]] (the node's first dof, as
 * the reference does).  xyz: nnode x 3.  Host only. */
BETA_GPU_API int beta_gpu_surface_flux_load(int nsurf, int nodes_per_face, const int* face_conn, int nnode,
                                            const double* xyz, const double* nodal_flux, const int* first_dof,
                                            int ndof, double* load);

/* ---- system exchange formats -------------------------------------------- */
/* The lower triangle of a symmetric matrix (SymmetricSparseMatrix order: rows
 * ascending, columns ascending, diagonal last) in BETA's dump layouts, for
 * cross-checks against external solvers:
 *   ADDRESS_LOWER  printMatrixAddressFormat (sparse.cpp:295-325)
 *   ADDRESS_UPPER  printMatrixAddressFormatUpper (sparse.cpp:263-293)
 *   COMPRESSED_ROW printCompressedRowFormat (sparse.cpp:327-355)
 *   CSR_ASCII      writeCSRMatrixInASCII / readCSRMatrixInASCII (SparseMatrixUtility.cpp:11-26, 60-78)
 *   CSR_BINARY     writeCSRMatrixInBinary / readCSRMatrixInBinary (SparseMatrixUtility.cpp:28-58)
 * The CSR files hold the lower triangle's 0-based row pointers and columns as
 * 32-bit ints (BETA_GPU_ERR_TOO_LARGE beyond 2^31-1 entries).  Host only. */
#define BETA_GPU_FMT_ADDRESS_LOWER 1
#define BETA_GPU_FMT_ADDRESS_UPPER 2
#define BETA_GPU_FMT_COMPRESSED_ROW 3
#define BETA_GPU_FMT_CSR_ASCII 4
#define BETA_GPU_FMT_CSR_BINARY 5
BETA_GPU_API int beta_gpu_write_lower(const char* path, int format, int n, const long long* row_ptr, const int* col,
                                      const double* val);
/* Reads a file written in `format`: call with row_ptr/col/val NULL for n and
 * nnz, then with arrays of n+1, nnz, nnz. */
BETA_GPU_API int beta_gpu_read_lower(const char* path, int format, int* n, long long* nnz, long long* row_ptr,
                                     int* col, double* val);
/* Writes the assembled matrix of `precision` (FP32 values widened). */
BETA_GPU_API int beta_gpu_export_matrix(beta_gpu_ctx* ctx, int precision, int format, const char* path);

/* ---- post-solve element outputs ------------------------------------------- */
/* ElasticityElement3D::getVolAvgValues (ElasticityElement3D.cpp:417-558) for
 * every element of an elasticity mesh, in FP64 on the device: per element
 * [volume, int stress dV (ns), int strain dV (ns), strain energy], ns = 6
 * (hex8: xx,yy,zz,xy,yz,xz, engineering shear) or 3 (quad4 plane stress:
 * xx,yy,xy; unit thickness).  u: host displacements (ndof) or NULL for the
 * last solution.  per_element: nelem*(2ns+2) or NULL; totals: 2ns+2 sums over
 * the mesh in element order or NULL (volume averages = totals / volume). */
BETA_GPU_API int beta_gpu_element_outputs(beta_gpu_ctx* ctx, const double* u, double* per_element, double* totals);

/* ---- transient diffusion (DiffusionModel::DoTransientNonLinearAnalysis) -- */
/* Sets u_s (host, ndof) as the current field. */
BETA_GPU_API int beta_gpu_heat_set_state(beta_gpu_ctx* ctx, const double* u0);
/* Runs nsteps steps of size dt with the generalized-alpha family (alpha=1:
 * backward Euler), assembling Mbar = (a1 K + M)/dt once (linear conductivity)
 * and solving Mbar du = -(a1+a2) K u_s / dt per step (DiffusionModel.cpp:743-818).
 * Every step after the first starts its solve from the previous step's
 * increment (beta_gpu_heat_set_state forgets it).
 * With BETA_GPU_STOP_RB a mixed-precision step stops at
 * ||r|| <= tol * max(||b||, ||(M/dt) u_s||): the increment's right-hand side b
 * shrinks as the field smooths, the new state's does not, and both systems
 * have the same residual. */
BETA_GPU_API int beta_gpu_heat_run(beta_gpu_ctx* ctx, double dt, double alpha, int nsteps,
                      const beta_gpu_solve_opts* opts, beta_gpu_solve_stats* last_step_stats,
                      int* total_iterations);
BETA_GPU_API int beta_gpu_heat_get_state(beta_gpu_ctx* ctx, double* u);

/* ---- device-pointer solver (LargeMatrix::solve on caller-owned storage) --- */
/* Jacobi-PCG on a caller-provided full (both-triangle) CSR matrix in device
 * memory: A x = b, x holds the initial guess on entry and the solution on
 * exit.  Scratch (Krylov vectors and reduction partials) is allocated by the
 * call with cudaMalloc and freed before return.  Stop rule and tolerance as in
 * beta_gpu_solve_opts.  Runs on the legacy default stream when stream == 0,
 * otherwise on the given cudaStream_t (passed as void*). */
BETA_GPU_API int beta_gpu_csr_pcg_device(int n, const int* d_row_ptr, const int* d_col, const double* d_val,
                            const double* d_b, double* d_x, int stop_rule, double tol, int maxit,
                            void* stream, beta_gpu_solve_stats* stats);

/* ---- batched systems in one persistent launch ----------------------------- */
/* No single counterpart in the reference, which solves one model per run
 * (BasicModel::DoAnalysis, BasicModel.cpp:1169-1220); each system goes through
 * the same path: structure (equation.cpp:1216-1267), FP32 assembly
 * (SerialAssembler.cpp:35-59 + equation.cpp:445-562) and the solve of
 * sparse.cpp:114-242, here in mixed precision with FP64 residual replacement.
 *
 * A batch owns a device pool of hbm_budget_bytes.  beta_gpu_batch_add builds a
 * system's structure on the host and copies it into the pool, or returns
 * BETA_GPU_REJECTED when the pool has no room (admission by HBM budget).
 * beta_gpu_batch_run assembles and solves every unfinished system in one
 * persistent launch (a replayed CUDA graph).  iters_per_launch > 0 bounds the PCG iterations each system
 * gets per launch, so a serving loop can admit and retire systems between
 * launches; the Krylov state stays in the pool.  Big systems are solved by
 * gangs of CTAs (SMs) meeting at software barriers, small ones by single
 * CTAs; every sum has a fixed order, so a system's result does not depend on
 * the mix or the gang size.  Stop rule: ||b-Au||/||b||
 * (opts->tol); opts->inner_tol is the residual-replacement factor.  Batched
 * diffusion systems are steady (conductivity only). */
typedef struct beta_gpu_batch beta_gpu_batch;
BETA_GPU_API int beta_gpu_batch_create(beta_gpu_batch** batch, int device, long long hbm_budget_bytes,
                                       int max_systems);
BETA_GPU_API int beta_gpu_batch_destroy(beta_gpu_batch* batch);
BETA_GPU_API const char* beta_gpu_batch_last_error(const beta_gpu_batch* batch);
BETA_GPU_API int beta_gpu_batch_add(beta_gpu_batch* batch, int kind, int ndim, int nnode, const double* xyz,
                                    int nelem, int nnpe, const int* conn, const int* first_dof, int ndof_per_node,
                                    int integration_order, int ngroups, int nparams, const double* group_params,
                                    const int* elem_group, const unsigned char* restrained,
                                    const double* prescribed, const double* load, int* sys_id);
/* One system for beta_gpu_batch_add_many: the arguments of beta_gpu_batch_add. */
typedef struct beta_gpu_system {
  int kind, ndim, nnode, nelem, nnpe, ndof_per_node, integration_order, ngroups, nparams, reserved;
  const double* xyz;
  const int* conn;
  const int* first_dof;
  const double* group_params;
  const int* elem_group;
  const unsigned char* restrained;
  const double* prescribed;
  const double* load;
} beta_gpu_system;
/* Adds `count` systems: their structures are built on up to `host_threads`
 * host threads (0 = all cores), then they are copied into the pool in order.
 * sys_ids[i] receives the id, or -(status) for a system that was not added
 * (bad input, or BETA_GPU_REJECTED when the pool is full).  Returns
 * BETA_GPU_OK when every system was added, else the first failing status. */
BETA_GPU_API int beta_gpu_batch_add_many(beta_gpu_batch* batch, int count, const beta_gpu_system* systems,
                                         int host_threads, int* sys_ids);
BETA_GPU_API int beta_gpu_batch_run(beta_gpu_batch* batch, const beta_gpu_solve_opts* opts, int iters_per_launch,
                                    int* n_unfinished);
/* Status/iterations of one system; u (ndof, may be NULL) receives its current
 * solution.  stats->ms_solve: device time spent on the system so far (the wall
 * time of the CTAs that solved it, summed over launches). */
BETA_GPU_API int beta_gpu_batch_result(beta_gpu_batch* batch, int sys_id, double* u,
                                       beta_gpu_solve_stats* stats);
BETA_GPU_API int beta_gpu_batch_remove(beta_gpu_batch* batch, int sys_id);
/* Launch shape: threads per CTA (256, 512 or 1024 (the default); one CTA per
 * SM) and gang sizing.  A system gets about gang_boost x (its share of the
 * batch's work: FP32 matrix values x expected iterations) of the CTAs, as one
 * gang, when that is at least 2; the other systems are solved by single CTAs.
 * gang_boost 0: every system on one CTA.
 * The result of a system does not depend on either choice. */
BETA_GPU_API int beta_gpu_batch_tune(beta_gpu_batch* batch, int threads_per_cta, int gang_boost);
/* Times every launch shape (threads per CTA, gang boost) on the current
 * systems for `budget` iterations each (budget 0: complete solves, which also
 * measures the tail of the largest systems), resets the systems to unsolved
 * afterwards and keeps the shape with the least time per unit of work. */
BETA_GPU_API int beta_gpu_batch_autotune(beta_gpu_batch* batch, const beta_gpu_solve_opts* opts, int budget,
                                         int* threads_per_cta, int* gang_boost);
/* Precision per system.  The FP32 matrix of a batch system is kept in
 * row-sum form: each diagonal block holds the block row sum of the FP64
 * operator and the product is formed from differences, so rounding the
 * entries to FP32 leaves the rigid-body (low-energy) modes exact.  A system
 * whose FP32 inner solve needs more than iters_per_cycle iterations for one
 * residual-replacement cycle (a drop of ||r|| by inner_tol) continues with
 * FP64 vectors and arithmetic on the same FP32 matrix, with the same FP64
 * reliable updates (stats->reserved = 1 in beta_gpu_batch_result): FP32
 * Krylov recurrences lose their convergence rate on ill-conditioned systems
 * such as long plates.  0: never.  Default 500.  The choice depends only on
 * the system. */
BETA_GPU_API int beta_gpu_batch_set_switch(beta_gpu_batch* batch, int iters_per_cycle);
/* Time slice of a launch (0 to 60 s; 0, the default: off).  With a slice, a
 * launch stops every system after the iteration in which the slice ends (on
 * top of the iteration budget of beta_gpu_batch_run), and no CTA starts a new
 * system after it; the systems a launch did not reach go first in the next.
 * A big system then no longer holds every other one for its whole budget.
 * Stopping and resuming leave the results unchanged. */
BETA_GPU_API int beta_gpu_batch_set_slice(beta_gpu_batch* batch, long long slice_us);
/* Failure-path test hook.  Sets the longest wait at a gang barrier (1 ms to
 * 10 s; default 2 s) and, with phantom != 0, plans the first gang of the next
 * launch one CTA larger than the CTAs it is given, so its first barrier can
 * only end by running out of time: that launch stops and returns
 * BETA_GPU_TIMEOUT, its unfinished systems restart from scratch on the next
 * beta_gpu_batch_run, the context stays usable, and the hook clears itself.
 * Not for production use. */
BETA_GPU_API int beta_gpu_batch_test_barrier(beta_gpu_batch* batch, long long limit_ns, int phantom);
/* The batch engine's CTA planner, exposed for inspection: for nsys systems
 * sorted by stored FP32 matrix values (largest first) with their 32-node
 * slice counts, fills gang_ctas[0..g) with the CTAs of each gang a launch of
 * `ctas` CTAs would form and returns g (systems 0..g-1 are solved by gangs,
 * the rest by single CTAs), or -BETA_GPU_ERR_ARG.  Host only. */
BETA_GPU_API int beta_gpu_gang_plan(int nsys, const long long* matrix_values, const int* slices, int ctas,
                                    int threads_per_cta, int gang_boost, int* gang_ctas);
/* Marks every system unsolved: its next launch assembles and solves it again
 * from the data already in the pool (repeat solves without re-upload). */
BETA_GPU_API int beta_gpu_batch_reset(beta_gpu_batch* batch);
/* out[0] live systems, out[1] pool bytes in use, out[2] pool bytes, out[3]
 * launches, out[4] bytes host->device, out[5] bytes device->host, out[6]
 * device time of the last launch in ns (CUDA events on the batch's stream),
 * out[7] gangs and out[8] CTAs in gangs in the last launch, out[9] threads
 * per CTA, out[10] gang boost, out[11] device time the systems' groups spent
 * on them (ns, summed over systems, removed ones included), out[12] of which
 * in setup (assembly, factors, first residual), out[13] of which in reliable
 * updates (FP64 residual replacements), out[14] inner iterations in all;
 * n <= 15. */
BETA_GPU_API int beta_gpu_batch_info(const beta_gpu_batch* batch, long long* out, int n);

/* ---- continuous-batching server ------------------------------------------ */
/* No counterpart in the reference (one model per process run).  A server owns
 * a batch and one worker thread.  beta_gpu_server_submit checks a system and
 * builds its structure on the calling thread, then queues it; the worker
 * admits queued systems in arrival order while the HBM pool has room, runs
 * bounded launches of iters_per_launch iterations over every admitted system
 * (new systems join between launches, with their assembly inside the launch)
 * and retires finished ones to host memory.  A request that does not fit into
 * an empty pool ends REJECTED.  Every system is solved exactly as
 * beta_gpu_batch_run solves it, so its result does not depend on what else is
 * in flight. */
#define BETA_GPU_REQ_QUEUED 0
#define BETA_GPU_REQ_RUNNING 1
#define BETA_GPU_REQ_DONE 2
#define BETA_GPU_REQ_REJECTED 3
#define BETA_GPU_REQ_CANCELLED 4
#define BETA_GPU_REQ_FAILED 5
typedef struct beta_gpu_server beta_gpu_server;
/* threads_per_cta / gang_boost as in beta_gpu_batch_tune; 0 / -1 keep the defaults. */
BETA_GPU_API int beta_gpu_server_create(beta_gpu_server** server, int device, long long hbm_budget_bytes,
                                        int max_systems, const beta_gpu_solve_opts* opts, int iters_per_launch,
                                        int threads_per_cta, int gang_boost);
/* Stops the worker after its current launch; unfinished requests are dropped. */
BETA_GPU_API int beta_gpu_server_destroy(beta_gpu_server* server);
BETA_GPU_API const char* beta_gpu_server_last_error(const beta_gpu_server* server);
/* Same system arguments as beta_gpu_batch_add; input errors return at once. */
BETA_GPU_API int beta_gpu_server_submit(beta_gpu_server* server, int kind, int ndim, int nnode, const double* xyz,
                                        int nelem, int nnpe, const int* conn, const int* first_dof,
                                        int ndof_per_node, int integration_order, int ngroups, int nparams,
                                        const double* group_params, const int* elem_group,
                                        const unsigned char* restrained, const double* prescribed,
                                        const double* load, long long* request_id);
/* Waits up to wait_ms for the request to reach a final state (DONE, REJECTED,
 * CANCELLED, FAILED), then reports its state, ndof, stats (stats->status is
 * the solve status once final, BETA_GPU_ERR_STATE before) and latency from
 * submit to completion in ms (-1 before).  u (ndof doubles, may be NULL)
 * receives the solution of a DONE request.  release != 0 forgets a final
 * request.  Returns BETA_GPU_ERR_ARG for an unknown id. */
BETA_GPU_API int beta_gpu_server_poll(beta_gpu_server* server, long long request_id, int wait_ms, int* state,
                                      int* ndof, double* u, beta_gpu_solve_stats* stats, double* latency_ms,
                                      int release);
/* Time slice of each launch, as beta_gpu_batch_set_slice (0, the default:
 * iters_per_launch alone bounds a launch); takes effect at the next launch.
 * With a slice, a running launch ends it early (after at least 2 ms) when
 * requests that arrived meanwhile have all been admitted, or -- for a launch
 * issued while no request waited -- when one of its requests finishes, so new
 * work and finished results wait about one iteration, not the rest of the
 * slice; with a backlog the slice runs out.  Gang plans keep a few CTAs (the
 * small systems' share of the work, 1 to 1/8 of the CTAs) for systems solved
 * by one CTA, so a small request next to big ones starts at once. */
BETA_GPU_API int beta_gpu_server_set_slice(beta_gpu_server* server, long long slice_us);
/* Queued requests end CANCELLED before admission, running ones after the current launch. */
BETA_GPU_API int beta_gpu_server_cancel(beta_gpu_server* server, long long request_id);
/* out[0] submitted, [1] done, [2] rejected, [3] failed, [4] cancelled,
 * [5] queued, [6] running, [7] launches, [8] pool bytes in use, [9] pool
 * bytes, [10] device microseconds of the launches (CUDA events), [11] bytes
 * host->device, [12] bytes device->host, [13] device time the retired
 * systems' groups spent on them (ns, summed over systems), [14] of which in
 * setup, [15] of which in reliable updates, [16] their inner iterations;
 * n <= 17. */
BETA_GPU_API int beta_gpu_server_stats(beta_gpu_server* server, long long* out, int n);

/* ---- geometric-nonlinear Newton loop (hex8 elasticity) ------------------- */
/* BasicModel::iterate (BasicModel.cpp:1244-1381) with the element in its
 * GEOMETRIC_NONLINEAR form: Green-Lagrange strain, B with the
 * displacement-gradient terms, the initial-stress term in the tangent
 * (ElasticityElement3D.cpp:84-160, 560-641). */
typedef struct beta_gpu_newton_opts {
  double max_residual;       /* stop when max |load - f_int| over free dofs < this (the reference's
                                maxAllowableResidual; 0: its default 1e-10)                       */
  int max_newton;            /* Newton solves at most (0: the reference's 400)                    */
  int use_last_solution;     /* start from the context's solution, else from the prescribed values */
  beta_gpu_solve_opts solve; /* each step: MODE_FP64 -- FP64 tangent, the reference's PCG from the
                                current solution as initial guess (solve.stop_rule, tol, maxit);
                                MODE_MPIR -- FP32 tangent, block-Jacobi PCG reducing the FP32
                                residual by solve.inner_tol (0: 1e-3), refined by the next FP64
                                residual (an inexact Newton)                                       */
} beta_gpu_newton_opts;

typedef struct beta_gpu_newton_stats {
  int status;            /* BETA_GPU_OK, MAXIT, BREAKDOWN or a linear solve's error      */
  int iterations;        /* Newton solves done                                            */
  int linear_iterations; /* PCG iterations in all                                         */
  int reserved;
  double max_residual;   /* max |R| over free dofs at exit                                */
} beta_gpu_newton_stats;

/* Runs the loop; the solution stays on the device (beta_gpu_download).
 * history (may be NULL): max |R| at each iteration, max_newton + 1 entries. */
BETA_GPU_API int beta_gpu_newton(beta_gpu_ctx* ctx, const beta_gpu_newton_opts* opts,
                                 beta_gpu_newton_stats* stats, double* history);
/* The context's current solution from host memory (BasicModel::
 * readDisplacementsIntoCurrentSolution, BasicModel.cpp:1230-1242: a Newton
 * loop restarted from saved displacements); the tangent assembly and a
 * Newton loop with use_last_solution start from it. */
BETA_GPU_API int beta_gpu_set_solution(beta_gpu_ctx* ctx, const double* u);
/* The geometric-nonlinear internal force f(u) (getGlobalForces with "F",
 * BasicModel.cpp:1063-1110, without the restraint mapping); host vectors. */
BETA_GPU_API int beta_gpu_internal_force_nonlinear(beta_gpu_ctx* ctx, const double* u, double* f);

/* ---- allocation-free variant of beta_gpu_csr_pcg_device ------------------ */
/* No counterpart in the reference (BETA's solvers allocate their work vectors
 * with new[] on every call, sparse.cpp:139-159).
 *
 * Some callers cannot let a library call cudaMalloc: an application that hands
 * nearly all of HBM to its own memory pool at start-up (a framework's caching
 * allocator, a serving loop sized to the card) would see the allocation fail
 * or fragment its pool, and cudaMalloc/cudaFree also synchronize the device,
 * stalling the caller's other streams.  This entry point allocates nothing: its
 * scratch (Krylov vectors r, p, q, 1/diag, reduction partials and solver state)
 * lives in one fixed device array inside the library, of
 * BETA_GPU_NOALLOC_SCRATCH_BYTES (about 8.1 MiB), which every GPU that loads
 * the library keeps until the process exits.
 *
 * Same arguments, algorithm and results as beta_gpu_csr_pcg_device, except:
 *   - n may not exceed BETA_GPU_NOALLOC_MAX_ROWS; larger systems return
 *     BETA_GPU_ERR_TOO_LARGE before any device work;
 *   - the first call on a device sets the array up there (loads the library's
 *     module on that device and looks up the array's device address): make
 *     that device current first, and make the first call before any stream
 *     capture.  Every call looks the address up again (cheap after the first),
 *     so a cudaDeviceReset between calls leaves no stale address behind;
 *   - all calls share the one array: calls that overlap on the GPU (other
 *     streams, other host threads) race and corrupt each other -- serialize them;
 *   - stats->ms_solve is not measured (0).
 * The caller still owns and passes the matrix, b and x. */
#define BETA_GPU_NOALLOC_MAX_ROWS 262144
#define BETA_GPU_NOALLOC_MAX_BLOCKS 2048
#define BETA_GPU_NOALLOC_SCRATCH_BYTES \
  (8 * (4 * (BETA_GPU_NOALLOC_MAX_ROWS) + 4 * (BETA_GPU_NOALLOC_MAX_BLOCKS) + 8) + 256)
BETA_GPU_API int beta_gpu_csr_pcg_device_noalloc(int n, const int* d_row_ptr, const int* d_col,
                                                 const double* d_val, const double* d_b, double* d_x,
                                                 int stop_rule, double tol, int maxit, void* stream,
                                                 beta_gpu_solve_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* BETA_GPU_H */
