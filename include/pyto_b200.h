/*
 * pyto_b200.h -- C ABI of the B200 voxel hex8 structural-FEA library.
 *
 * One shared library (libpyto_b200.so) built for sm_100a.  Every entry point
 * takes plain pointers and sizes; device pointers are CUDA global-memory
 * pointers of the calling process's current device, `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Calls are stream-ordered and
 * return a status code; none aborts the process.  The library never allocates
 * device memory: entry points that need scratch take a caller-provided
 * workspace whose size is given by pyto_workspace_bytes().
 *
 * Connectivity is implicit.  A grid of nelx*nely*nelz box elements of size
 * (hx,hy,hz) numbers nodes  n = ix + (nelx+1)*(iy + (nely+1)*iz),
 * elements e = ex + nelx*(ey + nely*ez) and DOFs 3n+{0,1,2} (x,y,z), element
 * corners in the order (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),
 * (1,1,1),(0,1,1) -- exactly PyTO's HexMesher.grid_mesh / createEdofMatStructural
 * numbering (src/hex_mesher.py:72-169, :1080-1095).
 *
 * Each declaration names the PyTO (UW-ERSL/PyTO) interface it replaces.
 */
#ifndef PYTO_B200_H
#define PYTO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PYTO_OK 0
#define PYTO_NOT_CONVERGED 1     /* iteration cap reached; result is the last iterate */
#define PYTO_ERR_ARG (-1)        /* invalid argument (null pointer, bad size, bad Ke) */
#define PYTO_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define PYTO_ERR_WORKSPACE (-3)  /* workspace missing or too small */
#define PYTO_ERR_BREAKDOWN (-4)  /* Krylov breakdown: p.Kp <= 0 or a non-finite scalar */
#define PYTO_ERR_TOO_LARGE (-5)  /* size beyond a fixed limit of the entry point */

/* ---- matvec / filter modes ---------------------------------------------- */
#define PYTO_MASK_IN 1   /* treat fixed DOFs of the input vector as zero */
#define PYTO_MASK_OUT 2  /* write zero to fixed DOFs of the output vector */

#define PYTO_FILTER_RAW 0      /* y = H x                                  */
#define PYTO_FILTER_DENSITY 1  /* y = (H x) / Hs                           */
#define PYTO_FILTER_CHAIN 2    /* y = H^T (x / Hs)        (hs required)    */
#define PYTO_FILTER_SENS 3     /* y = H (w .* x) / Hs ./ w  (w required)   */
#define PYTO_FILTER_HS 4       /* y = Hs = H 1                             */

/* ---- workspace kinds for pyto_workspace_bytes ---------------------------- */
#define PYTO_WS_REDUCE 0  /* reductions of matvec/energy/stress (dot, compliance, p-norm) */
#define PYTO_WS_PCG 1     /* pyto_pcg_solve                                               */
#define PYTO_WS_DPCG 2    /* pyto_dpcg_setup / pyto_dpcg_solve (coarse inverse is separate) */
#define PYTO_WS_OC 3      /* pyto_oc_update                                               */
#define PYTO_WS_DPCG_MIXED 4  /* pyto_dpcg_setup / pyto_dpcg_mixed_solve                      */

/* The operator: grid + the element stiffness matrix, plus the data derived
 * from Ke that the kernels use (Ke rotated into the 8x8 Hadamard corner basis,
 * where a box hex8 Ke splits into eight 3x3 blocks, and the corner diagonal). */
typedef struct pyto_operator {
  int32_t nelx, nely, nelz;
  int32_t tune;          /* per-grid matvec tile variants (the autotuner's choice): bits 0-7 =
                            FP64 variant + 1, bits 8-15 = FP32 variant + 1; 0 = library default */
  double hx, hy, hz;
  double E, nu;          /* material of Ke (stress recovery uses them) */
  double ke[576];        /* 24x24 Ke, row-major, reference DOF order */
  double khat[8][3][3];  /* parity-class blocks of Phi Ke Phi^T / 64 */
  double kdiag[3];       /* Ke[3a+c][3a+c], equal for every corner a */
} pyto_operator_t;

typedef struct pyto_solve_cfg {
  double rtol;          /* relative tolerance of the stopping rule */
  int32_t max_iters;    /* iteration cap */
  int32_t stop_rule;    /* 0: ||r||_2 < rtol ||b||_2 (scipy cg); 1: sqrt(r.z / r0.z0) <= rtol (PyTO DPCG);
                           2 (pyto_dpcg_solve only): FP64 residual replacement, see there */
  int32_t check_every;  /* host polls convergence every this many iterations (>=1) */
  int32_t x0_given;     /* 1: u holds the initial guess on entry; 0: start from zero (the deflated
                           solvers: from the coarse solution); honoured by pyto_pcg_solve and by the
                           residual-replacement deflated solvers (stop rule 2, mixed) */
} pyto_solve_cfg_t;

typedef struct pyto_solve_status {
  int32_t converged;    /* 1 if the stopping rule was met */
  int32_t iters;        /* Krylov iterations performed */
  int32_t breakdown;    /* 1 if p.Kp <= 0 or a scalar became non-finite */
  int32_t reserved;
  double rel_res;       /* stopping quantity at exit */
  double true_rel_res;  /* ||b - K u||_2 / ||b||_2 recomputed in FP64 at exit */
} pyto_solve_status_t;

/* Sparse coarse solver of a deflation space (nested dissection; see pyto_coarse_nd_plan). */
typedef struct pyto_coarse_nd pyto_coarse_nd_t;

/* Deflation space: node groups with rigid-body modes about the group centre.
 * modes = 6: columns [tx,ty,tz,rx,ry,rz] per group (src/deflation.py:386-457);
 * modes = 3: translations only.  All pointers are device pointers. */
typedef struct pyto_deflation {
  int32_t ngroups;
  int32_t modes;               /* 3 or 6 */
  const int32_t* node_group;   /* [nnodes] group of each node (16-byte aligned) */
  const int32_t* group_ptr;    /* [ngroups+1] CSR offsets of group_nodes */
  const int32_t* group_nodes;  /* [nnodes] node ids sorted by group */
  const double* group_center;  /* [ngroups*3] centroid of each group */
  double* coarse_inv;          /* [nc*nc], nc = ngroups*modes: written by pyto_dpcg_setup */
  double shift;                /* diagonal shift added to W^T K W */
  int32_t shift_relative;      /* 1: shift scales the mean diagonal; 0: absolute (PyTO: 1e-10) */
  int32_t max_group_nodes;     /* largest group (nodes) */
  const int32_t* group_box;    /* [ngroups*6] element index box touching the group:
                                  ex0,ex1,ey0,ey1,ez0,ez1 (inclusive) */
  const int32_t* nbr_ptr;      /* [ngroups+1] CSR offsets of nbr_list */
  const int32_t* nbr_list;     /* groups sharing an element with each group (incl. itself), ascending */
  int32_t max_nbr;             /* largest neighbour list (<= 128) */
  int32_t bel_count;           /* entries of bel_list (0: read from bel_ptr[ngroups] when needed) */
  /* Optional boundary element lists (NULL: the solver applies K to z with a full
   * matvec before restricting, as src/deflation.py:560-566 does).  A rigid mode of
   * a group is in the null space of every element whose 8 corners lie in that
   * group and are free, so W_f^T K z only needs, per group, the elements with a
   * corner in the group and a corner in another group or on a fixed DOF; the
   * lists must be rebuilt when the fixed DOFs change. */
  const int32_t* bel_ptr;      /* [ngroups+1] CSR offsets of bel_list */
  const int32_t* bel_list;     /* boundary elements of each group, ascending element ids */
  /* Optional per-entry metadata of bel_list (NULL: derived on the fly from node_group and
   * the mask): bits 0-7 = corner k of the entry's element lies in the entry's group,
   * bit 8 = the element has a fixed DOF.  Rebuilt with the lists. */
  const uint16_t* bel_meta;    /* [bel_count] */
  /* Optional sparse coarse solver (NULL: the dense coarse_inv).  When set (a plan bound
   * to its device buffer), pyto_dpcg_setup assembles W_f^T K_ff W_f block-sparse and
   * factors it by nested dissection, and pyto_dpcg_solve / pyto_dpcg_mixed_solve apply
   * that factorisation; coarse_inv may then be NULL.  Needs the boundary lists. */
  pyto_coarse_nd_t* coarse_nd;
} pyto_deflation_t;

/* ---- version / workspace ------------------------------------------------- */
int pyto_version(void);
/* sizeof of this library's ABI structs, for bindings to check their layout:
 * 0 pyto_operator_t, 1 pyto_solve_cfg_t, 2 pyto_solve_status_t, 3 pyto_deflation_t,
 * 4 pyto_batch_item_t, 5 pyto_thermal_t; 0 for other values.  No reference counterpart. */
size_t pyto_struct_size(int which);
/* Description of the last CUDA call of this thread that failed inside the library
 * (file:line, the call, the CUDA error); "" if none.  No reference counterpart. */
const char* pyto_last_error(void);
/* Number of kernel launches this library has issued in the process so far (no
 * reference counterpart: instrumentation of the launch count). */
long long pyto_launch_count(void);
/* Select the tile variant of a kernel (no reference counterpart: the tile
 * choice of the project's autotuner).  PYTO_KERNEL_MATVEC variants 0..3 (tile kernel,
 * default 2) and 8..10 (chunk-staged kernel: node-plane rows copied as 16-byte chunks,
 * faces and pending accumulators in registers; bitwise-equal results); PYTO_KERNEL_MATVEC32
 * variants 0..5, 8..11, 12..14 (chunk-staged, two element rows per thread), 15..17
 * (the same with the two rows as packed FP32x2 lanes) and 18, 19 (packed, element core
 * specialised to the block structure of an isotropic box / cube Ke, default 18; other
 * Ke run variant 16's kernel).  The chunk-staged
 * variants need u and the mask 16-byte aligned and otherwise run the tile kernel.
 * Process-wide; not thread-safe against concurrent launches. */
#define PYTO_KERNEL_MATVEC 0
#define PYTO_KERNEL_MATVEC32 1
#define PYTO_KERNEL_GRAPHS 2   /* variant 1 (default): deflated PCG iteration chunks replayed as
                                  CUDA graphs; 0: launched one kernel at a time */
int pyto_tune(int kernel, int variant);
/* Bytes of workspace for a call of the given kind on this operator (for
 * PYTO_WS_DPCG: up to 65536 groups; coarse sizes up to 24576 with the dense coarse inverse). */
size_t pyto_workspace_bytes(const pyto_operator_t* op, int kind);

/* ---- element matrices and operator set-up (host only, no GPU work) ------- */
/* 24x24 Ke of a box hex8, 2x2x2 Gauss, isotropic (E, nu).
 * Replaces hex_element_stiffness.hex8_stiffness_matrix_structural
 * (src/hex_element_stiffness.py:232-286). */
int pyto_ke_hex8(double E, double nu, double hx, double hy, double hz, double* ke_out);
/* Fill *op.  ke may be NULL (then Ke = pyto_ke_hex8(E, nu, h)); a given Ke must have
 * the reflection symmetry of a box hex8 or PYTO_ERR_ARG is returned.  Replaces the
 * Ke / COO-index set-up of HexStructuralFEA.__init__ (src/hex_structural_fea.py:21-52). */
int pyto_operator_init(pyto_operator_t* op, int32_t nelx, int32_t nely, int32_t nelz,
                       double hx, double hy, double hz, double E, double nu, const double* ke);

/* ---- material model -------------------------------------------------------- */
/* s = emin + x^p (1-emin), ds = p x^(p-1) (1-emin) (ds may be NULL); active (may be
 * NULL) zeroes s and ds of inactive elements.  Replaces
 * get_structural_material_model_scaling / _sensitivity (src/topopt_material_model.py:76-139). */
int pyto_simp(const double* x, const uint8_t* active, int64_t n, double penal, double emin,
              double* s, double* ds, void* stream);

/* ---- boundary conditions ------------------------------------------------------ */
/* mask[n] bit c set <=> DOF 3n+c is fixed.  mask is cleared first; its pointer must be
 * 4-byte aligned and the buffer must hold nnodes bytes rounded up to a multiple of 4
 * (bits are set with 32-bit atomics).  Out-of-range DOF ids are ignored.
 * Replaces BC.fixed_dofs / free_dofs (src/bound_cond.py:9-37). */
int pyto_bc_mask(const pyto_operator_t* op, const int64_t* fixed_dofs, int64_t n_fixed,
                 uint8_t* mask, void* stream);

/* ---- operator application ------------------------------------------------------- */
/* y = K(s) u, matrix-free, with Dirichlet masking per `mode` (PYTO_MASK_IN|PYTO_MASK_OUT
 * gives the reduced operator K_ff of impose_dirichlet_bc, src/bound_cond.py:40-70, on
 * full-length vectors).  If dot is non-NULL, *dot (device) = sum(u_masked . y); this
 * needs a PYTO_WS_REDUCE workspace.  Replaces the COO assembly + CSR SpMV of
 * HexStructuralFEA.solve / linear_solvers.solve (src/hex_structural_fea.py:87-102,
 * src/linear_solvers.py:136-202). */
int pyto_matvec(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* u,
                double* y, int mode, double* dot, void* ws, size_t ws_bytes, void* stream);

/* FP32 form of pyto_matvec (FP32 s, u, y; FP32 arithmetic on the FP32 Hadamard-basis
 * element blocks; the optional dot is accumulated in FP64).  The operator of the
 * inner cycles of pyto_dpcg_mixed_solve; no counterpart in the reference, which
 * assembles K in FP64 only. */
int pyto_matvec_f32(const pyto_operator_t* op, const float* s, const uint8_t* mask, const float* u,
                    float* y, int mode, double* dot, void* ws, size_t ws_bytes, void* stream);
/* FP32 tile variants 4 and 5 run the element contraction on the tensor cores (tcgen05,
 * BF16 split hi/lo operands, FP32 accumulation in TMEM).  Their waits are bounded; this
 * returns 1 if a wait ever gave up (never expected), 0 otherwise (synchronous; reset != 0
 * clears the flag).  No reference counterpart. */
int pyto_tensor_core_status(int reset);
/* pyto_matvec with a non-NULL dot, for callers that cannot allocate device memory
 * (plugins whose host owns every allocation, loops where allocation is forbidden after
 * start-up).  No counterpart in the reference.  The cross-block scratch is a fixed
 * array inside the library (~64 KB held on every GPU that loads it until process
 * exit); launches needing more than 8192 matvec blocks return PYTO_ERR_TOO_LARGE.  The
 * first call on a device looks up the array's device address and should precede any
 * stream capture; calls that overlap on the GPU race on the shared array.  The address
 * is kept for the life of the process: after a cudaDeviceReset (or any reset of the
 * device's primary context) this entry point must not be called again in that process. */
int pyto_matvec_dot_noalloc(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                            const double* u, double* y, int mode, double* dot, void* stream);
/* Jacobi data: diag(K)[3n+c] = kdiag[c] * sum_{e ni n} s_e.  Writes winv[n] = 1/sum s
 * and flags[n] = mask bits | (clamp bits << 3), clamp bit c set when |diag| < 1e-12 (then
 * the preconditioner is 1, src/linear_solvers.py:71-87).  diag_out (may be NULL) gets the
 * full diagonal [3*nnodes]. */
int pyto_jacobi(const pyto_operator_t* op, const double* s, const uint8_t* mask, double* winv,
                uint8_t* flags, double* diag_out, void* stream);

/* ---- solvers -------------------------------------------------------------------- */
/* Jacobi PCG on the reduced system K_ff u_f = b_f (src/linear_solvers.py:164-168).
 * b is full length; fixed entries are ignored.  u: solution, fixed entries set to 0. */
int pyto_pcg_solve(const pyto_operator_t* op, const double* s, const uint8_t* mask, const double* b,
                   double* u, const pyto_solve_cfg_t* cfg, pyto_solve_status_t* status, void* ws,
                   size_t ws_bytes, void* stream);
/* Build (W_f^T K_ff W_f + shift I)^-1 into defl->coarse_inv (dense FP64 sweep inversion on
 * the GPU).  Replaces the WKW set-up of deflatedPCG_CPU (src/deflation.py:513-521). */
int pyto_dpcg_setup(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                    pyto_deflation_t* defl, void* ws, size_t ws_bytes, void* stream);
/* Deflated PCG (src/deflation.py:504-584): coarse start, p0 = z - W mu, per iteration
 * one coarse correction; stopping rule per cfg (0: scipy, 1: PyTO).  cfg->stop_rule = 2
 * selects FP64 residual replacement: the recurrence of rule 0, but whenever ||r|| has
 * dropped 100-fold the coarse part of the true residual is removed and r is replaced by
 * b - K u; converged when ||b - K u|| <= rtol ||b|| (robust at tight tolerances where the
 * recurrence alone drifts).  b and u must be 16-byte aligned.  With
 * boundary lists in defl, W_f^T K z is formed from the group-boundary elements instead
 * of a second full matvec per iteration.  Replaces DeflationSolver.deflatedPCG. */
int pyto_dpcg_solve(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                    const pyto_deflation_t* defl, const double* b, double* u,
                    const pyto_solve_cfg_t* cfg, pyto_solve_status_t* status, void* ws,
                    size_t ws_bytes, void* stream);

/* Mixed-precision deflated PCG with reliable updates.  The Krylov recurrence runs
 * on FP32 vectors with the FP32 operator (FP64 dot-product reductions and scalars,
 * the FP64 coarse inverse of pyto_dpcg_setup); the solution is held in FP64.  The
 * start is the FP64 coarse solve u = W E^-1 W_f^T b.  Whenever the FP32 recursive
 * residual has dropped by `delta` (0 < delta < 1) since the last update, or meets
 * cfg->rtol, the FP32 iterate is added to u in FP64 and the residual is replaced by
 * b - K u computed in FP64; the search direction is kept, so no Krylov information
 * is discarded.  Convergence is ||b - K u|| <= cfg->rtol ||b||, tested in FP64.
 * cfg->max_iters caps the FP32 iterations; status->reserved returns the number of
 * FP64 residual updates.  Needs a PYTO_WS_DPCG_MIXED workspace.  Replaces
 * DeflationSolver.deflatedPCG (src/deflation.py:504-584) where FP64 accuracy is
 * required at lower cost. */
int pyto_dpcg_mixed_solve(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                          const pyto_deflation_t* defl, const double* b, double* u,
                          const pyto_solve_cfg_t* cfg, double delta, pyto_solve_status_t* status,
                          void* ws, size_t ws_bytes, void* stream);

/* ---- building blocks of a deflated PCG split across ranks --------------------------- */
/* No reference counterpart: PyTO solves on one host.  These are the pieces of
 * DeflationSolver.deflatedPCG (src/deflation.py:504-584) for a grid cut into slabs of node
 * planes, one slab per rank; the host composes them between its collectives (halo
 * exchange of the slab's boundary planes before each operator application, sums over
 * ranks of the dot products, of the restricted coarse vectors and of the coarse matrix).
 * A rank marks its halo nodes as fixed (all 3 bits) in `mask`, so outputs, dots and
 * restrictions cover its own nodes only.  All vectors are FP64 on the slab's grid. */
/* defl->coarse_inv = W_f^T K(s) W_f (dense nc x nc, no shift, not inverted: the sum over
 * ranks of each rank's elements gives the global matrix).  PYTO_WS_DPCG workspace. */
int pyto_coarse_assemble(const pyto_operator_t* op, const double* s, const uint8_t* mask,
                         pyto_deflation_t* defl, void* ws, size_t ws_bytes, void* stream);
/* defl->coarse_inv: E on entry, (sym(E) + shift I)^-1 on exit (vanishing rows -> identity,
 * shift as in pyto_dpcg_setup).  PYTO_WS_DPCG workspace. */
int pyto_coarse_invert(const pyto_operator_t* op, pyto_deflation_t* defl, void* ws, size_t ws_bytes,
                       void* stream);
/* v[nc] = W_f^T y over the nodes whose DOFs `mask` leaves free (deterministic order).
 * PYTO_WS_DPCG workspace. */
int pyto_coarse_restrict(const pyto_operator_t* op, const pyto_deflation_t* defl, const uint8_t* mask,
                         const double* y, double* v, void* ws, size_t ws_bytes, void* stream);
/* mu = defl->coarse_inv v (dense FP64 GEMV). */
int pyto_coarse_apply(const pyto_deflation_t* defl, const double* v, double* mu, void* stream);
/* p = a z + b p - W mu on free DOFs, 0 on fixed ones (z may be NULL: a z = 0). */
int pyto_coarse_prolong(const pyto_operator_t* op, const pyto_deflation_t* defl, const uint8_t* mask,
                        const double* mu, double a, const double* z, double b, double* p, void* stream);
/* x += alpha p (when p and x are given), r -= alpha q (when q is given), z = M r (Jacobi
 * data of pyto_jacobi: winv, flags), and dots[0] = r.r, dots[1] = r.z over the free DOFs
 * (device, deterministic).  p and x are both given or both NULL.  PYTO_WS_REDUCE
 * workspace. */
int pyto_cg_update(const pyto_operator_t* op, const double* winv, const uint8_t* flags, double alpha,
                   const double* p, const double* q, double* x, double* r, double* z, double* dots, void* ws,
                   size_t ws_bytes, void* stream);

/* ---- sparse coarse solver: nested dissection on a box grid of groups ----------------- */
/* The reference densifies W^T K W and solves it with a direct solver per iteration
 * (src/deflation.py:517-521, 577); a dense coarse matrix limits the coarse space to a few
 * thousand unknowns (82,944 for 4x4x4-element aggregates with 3 translations on a
 * 192x96x96 grid would be 55 GB).  For groups on a regular gx x gy x gz box grid (group
 * id = ix + gx (iy + gy iz), every neighbour within one box in each direction: the
 * element-box aggregates of create_deflation_groups_box and the reference's node-box
 * partition of a grid mesh), W^T K W is block-sparse with at most 27 neighbour blocks per
 * group.  It is factored by nested dissection on that grid: boxes of groups are split
 * recursively by separator planes (leaves: boxes of at most `leaf` groups); each tree node
 * holds a dense frontal matrix over its own unknowns and its boundary (the groups around
 * its box, all in ancestor separators); the node's own unknowns are eliminated by a
 * blocked Gauss-Jordan sweep, and the Schur complement on its boundary is added into the
 * parent's front.  A solve runs the tree up (frontal right-hand sides) and down (GEMVs
 * with the stored -A_ss^-1 and A_bs A_ss^-1).  All sums are in a fixed order: the
 * factorisation and the solves are bitwise reproducible.  No reference counterpart
 * beyond the direct coarse solve it replaces. */
/* Host-only planning (no GPU work).  nbr_ptr / nbr_list: host copies of the deflation's
 * neighbour lists (pyto_deflation_t.nbr_ptr / nbr_list).  NULL on invalid arguments or a
 * neighbour list that does not match the box grid (pyto_last_error says which). */
pyto_coarse_nd_t* pyto_coarse_nd_plan(int32_t gx, int32_t gy, int32_t gz, int32_t modes, int32_t leaf,
                                      const int32_t* nbr_ptr, const int32_t* nbr_list);
/* Device bytes of the plan (index tables, the block-sparse coarse matrix, frontal matrices,
 * their sweep scratch).  info (may be NULL) receives [0] tree nodes, [1] tree depth,
 * [2] largest front (unknowns), [3] factorisation flops, [4] bytes read per solve. */
size_t pyto_coarse_nd_bytes(const pyto_coarse_nd_t* plan, double* info);
/* Bind the plan to a caller-owned device buffer of pyto_coarse_nd_bytes bytes (256-byte
 * aligned) and copy the index tables into it (stream-ordered; the plan's host tables must
 * stay alive until the copy has run: keep the plan until the stream is synchronised). */
int pyto_coarse_nd_bind(pyto_coarse_nd_t* plan, void* dev_buf, size_t bytes, void* stream);
/* mu[nc] = (W_f^T K_ff W_f + shift I)^-1 v with the factorisation of the last
 * pyto_dpcg_setup (nc = groups x modes, both device vectors). */
int pyto_coarse_nd_solve(const pyto_coarse_nd_t* plan, const double* v, double* mu, void* stream);
void pyto_coarse_nd_free(pyto_coarse_nd_t* plan);

/* ---- batched solves in one CUDA graph ---------------------------------------------- */
/* One independent deflated PCG problem of a batch (no reference counterpart: PyTO
 * solves one problem per call).  op and defl are read when the batch is created; the
 * device buffers (s, mask, b, u, the deflation arrays, ws) are read at every launch,
 * so rewriting s and b and launching again solves new designs and load cases.  defl
 * needs its boundary lists with bel_count set; each item needs its own PYTO_WS_DPCG
 * workspace; b and u 16-byte aligned.  Items may share one deflation space (several load
 * cases of one design: same op, s and mask, different b and u): the first of them builds
 * the coarse inverse and the others wait for it. */
typedef struct pyto_batch_item {
  const pyto_operator_t* op;
  const double* s;
  const uint8_t* mask;
  pyto_deflation_t* defl;
  const double* b;
  double* u;
  void* ws;
  size_t ws_bytes;
} pyto_batch_item_t;
typedef struct pyto_batch* pyto_batch_t;
/* Capture every item's coarse set-up and deflated PCG (cfg: stop rule 0 or 1) into one
 * CUDA graph: one concurrent branch per item, the iterations of each in a conditional
 * WHILE node driven by the device-side stopping flag (ends on convergence, breakdown
 * or cfg->max_iters).  Nothing runs at creation (the capture uses a private stream;
 * `stream` is not used). */
int pyto_batch_create(const pyto_batch_item_t* items, int n, const pyto_solve_cfg_t* cfg,
                      pyto_batch_t* out, void* stream);
/* One graph launch: coarse set-up and solve of every item, no host round trips. */
int pyto_batch_launch(pyto_batch_t b, void* stream);
/* status[n] of the last launch (synchronises the stream); returns the worst status. */
int pyto_batch_status(pyto_batch_t b, pyto_solve_status_t* status, void* stream);
int pyto_batch_destroy(pyto_batch_t b);

/* ---- objectives and sensitivities ------------------------------------------------ */
/* ce[e] = u_e^T Ke v_e (u == v gives the element energy of compliance).  If s != NULL and
 * total != NULL, *total (device) = sum_e s_e ce_e (needs PYTO_WS_REDUCE workspace).
 * Replaces the gather + GEMM of compute_compliance_and_gradient
 * (src/topopt_obj_cons_sensitivities.py:148-179, :279-282, :308-311). */
int pyto_elem_energy(const pyto_operator_t* op, const double* u, const double* v, const double* s,
                     double* ce, double* total, void* ws, size_t ws_bytes, void* stream);
/* Centroid strain, stress = x^q D eps, von Mises, strain energy 0.5 eps.sigma
 * (src/hex_structural_fea.py:152-234).  strain/stress [ne*6] and sed may be NULL. */
int pyto_stress(const pyto_operator_t* op, const double* u, const double* x, double q,
                double* strain, double* stress, double* vm, double* sed, void* stream);
/* sum_e vm_e^P into *sum_out (device); needs PYTO_WS_REDUCE workspace. */
int pyto_pnorm_sum(const pyto_operator_t* op, const double* vm, double P, double* sum_out,
                   void* ws, size_t ws_bytes, void* stream);
/* p-norm adjoint pieces (src/topopt_obj_cons_sensitivities.py:238-266): with
 * dpn = (sum vm^P)^(1/P-1) read from *dpn_dev, T1[e] = dpn q x^(q-1) vm^(P-1) DvmDs.D.B.u_e
 * and the adjoint load g = sum_e x^q dpn vm^(P-1) B^T D^T DvmDs (node-owned gather,
 * no atomics).  x is clamped below at 1e-12 as in the reference.  tvec is scratch of
 * [ne*6] doubles. */
int pyto_pnorm_adjoint(const pyto_operator_t* op, const double* u, const double* x, double q,
                       double P, const double* dpn_dev, double* T1, double* g, double* tvec,
                       void* stream);

/* ---- density filter and OC update ---------------------------------------------- */
/* Linear hat filter H_ij = (r - d_ij)/r, d_ij <= r, r = rel_radius * hx, applied as a
 * grid stencil (src/topopt_filters.py:8-38; density filter src/topopt_mma.py:255-258,
 * chain rule :341-345; OC sensitivity filter src/topopt_ocm.py:239).  hs is needed by
 * PYTO_FILTER_CHAIN, w by PYTO_FILTER_SENS; both may be NULL otherwise.  active (may be
 * NULL) restricts H to active elements (inactive outputs are 0). */
int pyto_filter(const pyto_operator_t* op, double rel_radius, int mode, const double* x,
                const double* w, const double* hs, const uint8_t* active, double* y, void* stream);
/* Symmetry / extrusion map F of the element field of a full box grid (no active mask):
 * y = F(x o pre) / post (pre, post may be NULL; y must not alias x).  kind
 * PYTO_SYM_MIRROR: F x = (x + x[mirror about the mid-plane normal to axis]) / 2
 * (createX/Y/ZSymmetryFilter, src/topopt_filters.py:292-393); PYTO_SYM_EXTRUDE: the
 * reference's extrusion average along axis, whose lines are visited from their first
 * element, which joins its line twice (createX/Y/ZExtrudeFilter, src/topopt_filters.py:
 * 595-716).  Both maps are symmetric.  The composed filter H = H_s F_1 F_2 ... of
 * createFilters (src/topopt_common.py:127-159) applies them before pyto_filter. */
#define PYTO_SYM_MIRROR 0
#define PYTO_SYM_EXTRUDE 1
int pyto_symmetry_filter(const pyto_operator_t* op, int kind, int axis, const double* x, const double* pre,
                         const double* post, double* y, void* stream);
/* y = x o mul / (div1 o div2) over n entries (each factor may be NULL); the elementwise
 * step of the composed filters.  No reference counterpart (numpy broadcasting there). */
int pyto_vec_scale(int64_t n, const double* x, const double* mul, const double* div1, const double* div2,
                   double* y, void* stream);
/* One OC update with bisection on the volume multiplier (src/topopt_ocm.py:244-283),
 * the same bisection sequence as the reference.  x is updated in place; *change_out
 * (device) = max |x_new - x_old|.  dc is the filtered objective gradient.  With an active
 * mask (may be NULL) only its n_active elements are updated and counted in the volume. */
int pyto_oc_update(const pyto_operator_t* op, double* x, const double* dc, const uint8_t* active,
                   long long n_active, double volfrac, double move, double xmin, double xmax,
                   double* change_out, void* ws, size_t ws_bytes, void* stream);

/* ---- MMA update of the density-based optimiser ------------------------------------- */
/* One subproblem of the method of moving asymptotes (K. Svanberg's 2007 mmasub/subsolv,
 * the algorithm of the third-party mmasub that src/mmaWrapper.py:91-94 calls) on the
 * device, for n design variables and 1 <= m <= 4 constraints f_j(x) <= 0, in one
 * cooperative kernel.  Device arrays: x (in: the current design, out: the subproblem's
 * solution), xold1, xold2 (the two previous designs; may be NULL while iter <= 2),
 * xmin, xmax (per-variable bounds, or NULL: xmin_s / xmax_s), df0dx [n], dfdx [m][n],
 * low, upp (the asymptotes, updated), dual_out (may be NULL: y[m], z, lam[m], mu[m], zet,
 * s[m], Newton steps).  Host arrays: fval, a, c, d [m].  The workspace also keeps the
 * subproblem state read by pyto_mma_kkt.  No reference counterpart in this library's
 * other entry points: PyTO's MMA runs on the host. */
size_t pyto_mma_workspace_bytes(int64_t n, int m);
int pyto_mma_update(int64_t n, int m, int iter, double* x, const double* xold1, const double* xold2,
                    const double* xmin, const double* xmax, double xmin_s, double xmax_s, const double* df0dx,
                    const double* fval, const double* dfdx, double* low, double* upp, double a0, const double* a,
                    const double* c, const double* d, double move, double* dual_out, void* ws, size_t ws_bytes,
                    void* stream);
/* KKT residual of the original problem at the last update's solution, with the
 * gradients evaluated there (kktcheck of the same package): kkt_out[0] = its 2-norm,
 * kkt_out[1] = its max |.| (host doubles; synchronises the stream). */
int pyto_mma_kkt(int64_t n, int m, const double* x, const double* xmin, const double* xmax, double xmin_s,
                 double xmax_s, const double* df0dx, const double* fval, const double* dfdx, double a0,
                 const double* a, const double* c, const double* d, double* kkt_out, void* ws, size_t ws_bytes,
                 void* stream);

/* ---- thermal hex8 (one temperature DOF per node) ----------------------------------- */
/* Grid + the 8x8 conduction matrix of a box element.  For a box element Ke[a][b] depends
 * only on which coordinates of corners a and b differ: kxor[d] with d = bits(a) ^ bits(b),
 * bits = the corner's (x, y, z) offsets as bits 0, 1, 2. */
typedef struct pyto_thermal {
  int32_t nelx, nely, nelz, pad;
  double hx, hy, hz;
  double k;          /* conductivity of Ke */
  double ke[64];     /* 8x8 Ke, row-major, reference corner order */
  double kxor[8];    /* Ke as a function of the differing offset bits */
} pyto_thermal_t;
/* 8x8 conduction Ke of a box hex8, 2x2x2 Gauss.  Replaces
 * hex_element_stiffness.hex8_stiffness_matrix_thermal (src/hex_element_stiffness.py:340-385). */
int pyto_ke_hex8_thermal(double k, double hx, double hy, double hz, double* ke_out);
/* Fill *t (ke may be NULL: Ke = pyto_ke_hex8_thermal(k, h)); a given Ke without the box
 * symmetry is refused (PYTO_ERR_ARG).  Replaces the set-up of HexThermalFEA.__init__
 * (src/hex_thermal_fea.py:19-52). */
int pyto_thermal_init(pyto_thermal_t* t, int32_t nelx, int32_t nely, int32_t nelz, double hx, double hy,
                      double hz, double k, const double* ke);
/* mask[n] = 1 for the fixed-temperature nodes (nnodes bytes, cleared first). */
int pyto_thermal_mask(const pyto_thermal_t* t, const int64_t* fixed_nodes, int64_t n_fixed, uint8_t* mask,
                      void* stream);
/* Bytes of workspace of pyto_thermal_pcg_solve (also enough for the dot / total
 * reductions of pyto_thermal_matvec and pyto_thermal_energy). */
size_t pyto_thermal_workspace_bytes(const pyto_thermal_t* t);
/* T-field operator y = K(s) u with masking per mode (as pyto_matvec); optional *dot =
 * u_masked . y.  Replaces the COO assembly of HexThermalFEA.solve (src/hex_thermal_fea.py:69-117). */
int pyto_thermal_matvec(const pyto_thermal_t* t, const double* s, const uint8_t* mask, const double* u, double* y,
                        int mode, double* dot, void* ws, size_t ws_bytes, void* stream);
/* Jacobi PCG on the reduced thermal system (scipy cg semantics, src/linear_solvers.py:164-168);
 * stop rules 0 and 1 as pyto_pcg_solve. */
int pyto_thermal_pcg_solve(const pyto_thermal_t* t, const double* s, const uint8_t* mask, const double* b,
                           double* u, const pyto_solve_cfg_t* cfg, pyto_solve_status_t* status, void* ws,
                           size_t ws_bytes, void* stream);
/* ce[e] = u_e^T Ke v_e (v NULL: v = u); with total: *total = sum s_e ce_e (device).  Replaces
 * the thermal branch of compute_compliance_and_gradient (src/topopt_obj_cons_sensitivities.py:148-179). */
int pyto_thermal_energy(const pyto_thermal_t* t, const double* u, const double* v, const double* s, double* ce,
                        double* total, void* ws, size_t ws_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PYTO_B200_H */
