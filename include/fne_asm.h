/*
 * fne_asm.h -- C ABI of libfne_asm.so: element energy / gradient / Hessian
 * assembly for the nonlinear-energy minimisers of Beremi/fenics_nonlinear_energies,
 * on one NVIDIA B200 (sm_100a).
 *
 * Plain pointers and sizes only.  Every function returns an fne_status; on
 * failure fne_last_error() gives a thread-local message.  Device pointers
 * are CUDA global-memory pointers of the current device; ``stream`` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   fne_layout_build     build_global_layout + select_permutation('none'|'block_xyz')
 *                        src/core/petsc/reordered_element_base.py:183-200, 380-506
 *                        (+ petsc_ownership_range, src/core/petsc/dof_partition.py:27-55)
 *   fne_create           ReorderedElementAssemblerBase._make_local_element_kernels
 *                        (:922-923; per-family implementations
 *                        src/problems/plaplace/jax_petsc/reordered_element_assembler.py:30-65,
 *                        src/problems/ginzburg_landau/jax_petsc/reordered_element_assembler.py:54-91,
 *                        src/problems/hyperelasticity/jax_petsc/reordered_element_assembler.py:55-101,
 *                        src/problems/slope_stability/jax_petsc/reordered_element_assembler.py:152-243)
 *                        together with _build_scatter_data (:1464-1534)
 *   fne_eval ENERGY      energy_fn (:1579-1611): sum_e w_e e_e - f.u
 *   fne_eval GRAD        gradient_fn (:1613-1633): grad_local[owned_local_pos] - f_owned
 *   fne_eval HESS        assemble_hessian_element (:1733-1762): the (E,n,n) Hessian stack
 *                        plus the np.add.at scatter into the owned COO values,
 *                        in layout.owned_rows/owned_cols order
 *   fne_set_dirichlet    update_dirichlet (:1560-1566)
 *   fne_destroy          cleanup (:1777-1783)
 *   fne_layout_build_device  fne_layout_build on the GPU (same arrays)
 *   fne_hvp*             matrix-free Mohr-Coulomb operator,
 *                        src/problems/slope_stability/jax_petsc/reordered_element_assembler.py:335-440, 527-562
 *   fne_cg_*             the Newton step's KSP solve on the assembled matrix (Jacobi CG),
 *                        src/core/petsc/scalar_problem_driver.py:154-226
 */
#ifndef FNE_ASM_H
#define FNE_ASM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FNE_OK = 0,
  FNE_EINVAL = 1,   /* bad argument                                    */
  FNE_ECUDA = 2,    /* a CUDA runtime call failed                      */
  FNE_EBOUNDS = 3,  /* an index or size outside the supported range    */
  FNE_ETIMEOUT = 4, /* a bounded device wait gave up                   */
  FNE_ENOMEM = 5,   /* host or device allocation failed                */
  FNE_ELAYOUT = 6   /* COO pattern does not match the element graph    */
} fne_status;

typedef enum {
  FNE_PLAPLACE = 1,        /* P1 triangles, scalar, (1/p)|grad u|^p      */
  FNE_GINZBURG_LANDAU = 2, /* P1 triangles, scalar, eps/2|grad u|^2+W(u) */
  FNE_NEOHOOKEAN = 3,      /* P1 tetrahedra, 3 dofs per node            */
  FNE_MOHR_COULOMB = 4,    /* Pk triangles, plane strain, 2 dofs/node   */
  FNE_MOHR_COULOMB_3D = 5  /* P1 / P2 / P4 tetrahedra, 3 dofs/node      */
} fne_family;

typedef enum { FNE_FP64 = 0, FNE_FP32 = 1 } fne_precision;

typedef enum { FNE_REORDER_NONE = 0, FNE_REORDER_BLOCK_XYZ = 1 } fne_reorder;

enum { FNE_ENERGY = 1, FNE_GRAD = 2, FNE_HESS = 4 };

/* ---------------------------------------------------------------------------
 * Layout (host side, C++).  Replaces build_global_layout for the
 * global-adjacency branch.  The COO pattern is iperm[adjacency CSR nonzero()]
 * restricted to owned rows; when adj_indptr is NULL the adjacency is the
 * free-DOF element-pair graph of ``elems`` (what the reference's mesh
 * builders store).
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t n_total;              /* length of the full DOF vector              */
  int64_t n_free;               /* number of free DOFs                        */
  const int64_t* freedofs;      /* [n_free] total-DOF ids, ascending          */
  int64_t n_elem;
  int32_t ndof_e;               /* DOFs per element (npe * block_size)        */
  const int64_t* elems;         /* [n_elem * ndof_e] total-DOF connectivity   */
  int32_t block_size;
  int32_t reorder;              /* fne_reorder                                */
  int64_t n_nodes;              /* rows of coords                             */
  int32_t dim;                  /* columns of coords                          */
  const double* coords;         /* [n_nodes * dim] (block_xyz only)           */
  const int64_t* perm_override; /* [n_free] or NULL                           */
  const int64_t* adj_indptr;    /* [n_free+1] or NULL                         */
  const int64_t* adj_indices;   /* [nnz] or NULL                              */
  int32_t comm_rank, comm_size;
} fne_layout_desc;

typedef struct fne_layout fne_layout;

int fne_layout_build(const fne_layout_desc* desc, fne_layout** out);
/* The same layout built on the current CUDA device, array for array
 * identical: stable radix sorts of the blocks' coordinates (z, y, x) and a
 * radix sort + unique of the element DOF-pair keys row * n_free + col.
 * Inputs are host arrays, checked as fne_layout_build checks them; the
 * arrays stay in device memory until fne_layout_copy (D2H) and
 * fne_layout_free.  Needs about 16 * n_elem * ndof_e^2 bytes of device
 * memory for the pair keys when no adjacency is given. */
int fne_layout_build_device(const fne_layout_desc* desc, fne_layout** out);
/* Sizes of the arrays fne_layout_copy fills. */
int fne_layout_sizes(const fne_layout* lay, int64_t* n_free, int64_t* lo, int64_t* hi,
                     int64_t* nnz_total, int64_t* nnz_owned, int64_t* n_elem);
/* Any output pointer may be NULL.  perm/iperm [n_free]; total_to_free_reord
 * [n_total]; coo_rows/cols [nnz_total]; owned_rows/cols [nnz_owned];
 * elem_owner [n_elem] (-1 = element without free DOF). */
int fne_layout_copy(const fne_layout* lay, int64_t* perm, int64_t* iperm,
                    int64_t* total_to_free_reord, int64_t* coo_rows, int64_t* coo_cols,
                    int64_t* owned_rows, int64_t* owned_cols, int64_t* elem_owner);
void fne_layout_free(fne_layout* lay);

/* ---------------------------------------------------------------------------
 * Assembler handle.  Holds device copies of the element data and the
 * precomputed element -> nonzero gather plan; immutable after creation
 * except for the Dirichlet values.
 * ------------------------------------------------------------------------- */
typedef struct {
  int32_t family;               /* fne_family                                 */
  int32_t precision;            /* fne_precision: arithmetic of grad/Hessian  */
  int32_t hess_fp32;            /* FP32 mode only: 1 = Hessian values float32 */
  int64_t n_elem;
  int32_t npe;                  /* nodes per element                          */
  int32_t block_size;           /* DOFs per node                              */
  const int64_t* elems;         /* [n_elem * npe*block_size] total DOFs       */
  int64_t n_total;
  const int64_t* total_to_free_reord; /* [n_total], -1 = Dirichlet            */
  int64_t n_free, lo, hi;       /* owned reordered range [lo, hi)             */
  int64_t nnz;                  /* owned COO entries                          */
  const int64_t* owned_rows;    /* [nnz] reordered row ids (output order)     */
  const int64_t* owned_cols;    /* [nnz] reordered column ids                 */
  const double* energy_weights; /* [n_elem] 0/1, or NULL = 1 where any free   */
  int32_t nq;                   /* quadrature points (Mohr-Coulomb)           */
  /* family element arrays, float64:
   *   p-Laplace / GL : e0 = dvx [E*3], e1 = dvy [E*3], e2 = vol [E]
   *   Neo-Hookean    : e0 = dphix [E*4], e1 = dphiy, e2 = dphiz, e3 = vol [E]
   *   Mohr-Coulomb   : affine form of the reference's elem_B / quad_weight
   *                    (elem_B[e,q] = rows (xx, yy, xy) of the basis
   *                    gradients J_e^-T grad(phi_a)(xi_q); quad_weight[e,q]
   *                    = |det J_e| w_q):
   *                    e0 = J_e^-1 row-major [E*4], e1 = |det J_e| [E],
   *                    or, with s[6] = 1 (P2 only), the isoparametric map's
   *                    e0 = J_eq^-1 [E*nq*4], e1 = |det J_eq| [E*nq] per
   *                    quadrature point (the reference's P2 operators,
   *                    src/problems/slope_stability/support/mesh.py:530-567),
   *                    e2 = eps_p_old [E*nq*3] or NULL (zero),
   *                    e3 = reference tables [dhat1 (nq*np) | dhat2 (nq*np) | w (nq)],
   *                    npe = np (3, 6 or 15), block_size = 2, nq = 1, 7 or 19 */
  const double* e0;
  const double* e1;
  const double* e2;
  const double* e3;
  /*   Mohr-Coulomb 3-D (SlopeStability3DReorderedElementAssembler,
   *                    src/problems/slope_stability_3d/jax_petsc/
   *                    reordered_element_assembler.py:189-206): the
   *                    reference's per-element, per-quadrature-point arrays
   *                    e0 = dphix, e1 = dphiy, e2 = dphiz [E*nq*npe],
   *                    e3 = [E*nq*6] (quad_weight, c_bar_q, sin_phi_q,
   *                    shear_q, bulk_q, lame_q) per point,
   *                    npe = 4, 10 or 35, block_size = 3, nq <= 16
   *                    (P1, P2) or nq <= 32 (P4)                          */
  /* scalars:
   *   p-Laplace : s[0] = p
   *   GL        : s[0] = eps, s[1..9] = ip (3x3 row-major), s[10..12] = w
   *   Neo-Hook. : s[0] = C1, s[1] = D1, s[2] = use_abs_det (0/1)
   *   M-C       : s[0] = E, s[1] = nu, s[2] = phi_deg, s[3] = cohesion,
   *               s[4] = reg, s[5] = elastic (0/1),
   *               s[6] = geometry per quadrature point (0/1, see e0/e1)
   *   M-C 3-D   : s[0] = the density's guard constant (0: 1e-15),
   *               s[5] = elastic (0/1)                                       */
  double s[16];
  const double* dirichlet;      /* [n_total] full DOF vector (Dirichlet part) */
  const double* rhs_owned;      /* [hi-lo] load vector f (reordered), or NULL */
  int32_t dirichlet_only_energy;/* 1: add the energy of elements without any
                                 * free DOF (Ginzburg-Landau assembler,
                                 * src/problems/ginzburg_landau/jax_petsc/
                                 * reordered_element_assembler.py:34-52, 96-97) */
  int32_t kernel_variant;       /* P1 triangles: 0 = automatic (banded
                                 * sweep); 1 = row-gather; 2 = incidence-
                                 * parallel; 3 = banded sweep with shared-
                                 * memory atomics (push; not bit-reproducible);
                                 * 7 = banded sweep; 8 = persistent row-cluster
                                 * kernel (TMA-staged; the banded sweep when
                                 * the mesh does not fit its packed format).
                                 * P1 tets: 0 = row-gather with automatic lanes
                                 * per row; 1 = row-gather, one lane per row;
                                 * 2 = element-parallel pass + node-block
                                 * gather; 4 / 5 / 6 = row-gather with 2 / 4 / 8
                                 * lanes per row.
                                 * Mohr-Coulomb: 0 = automatic (tcgen05 tensor
                                 * cores for FP32 P2/P4, FP64 DMMA tensor cores
                                 * for FP64 P2/P4, CUDA cores for P1);
                                 * 1 = CUDA cores only.                        */
} fne_desc;

typedef struct fne_handle fne_handle;

typedef struct {
  int64_t n_rows;       /* owned rows (= hi - lo)                              */
  int64_t nnz;          /* owned COO entries                                   */
  int64_t n_elem;       /* elements with at least one owned DOF                */
  int64_t n_incidences; /* (row-node, element) pairs in the gather plan        */
  int64_t device_bytes; /* device memory the handle owns                       */
  int32_t max_row_len;
  int32_t kernel_variant; /* 1 row-gather (triangles), 2 row-gather (tets),
                           * 3 incidence-parallel, 4 banded sweep,
                           * 5 Mohr-Coulomb CUDA cores, 6 Mohr-Coulomb tcgen05,
                           * 7 element-parallel tets + node-block gather,
                           * 8 banded sweep, push variant,
                           * 9 Mohr-Coulomb FP64 DMMA (mma.sync f64),
                           * 10 row clusters (P1 triangles),
                           * 11 3-D Mohr-Coulomb point-tile element kernel +
                           * node-block gather */
  int32_t row_lanes;      /* lanes per output row of the tet row kernel, else 1 */
} fne_info;

int fne_create(const fne_desc* desc, fne_handle** out);
int fne_info_get(const fne_handle* h, fne_info* info);
/*
 * Matrix-free Hessian products (Mohr-Coulomb handles), replacing the
 * reference's prepare_matrix_free_operator / matrix_free_mult /
 * matrix_free_get_diagonal (src/problems/slope_stability/jax_petsc/
 * reordered_element_assembler.py:335-562, mode "matfree_element").
 *   fne_hvp_prepare: linearize at u (device, [n_free] full reordered free
 *     vector): stores the weighted consistent tangent of every quadrature
 *     point (n_elem * nq * 6 values; allocated on the first call).
 *   fne_hvp: y[owned] = H(u) x, x a device [n_free] tangent (its Dirichlet
 *     components are zero by construction), y device [hi - lo].
 *   fne_hvp_diagonal: diag[owned] = the diagonal of H(u).
 * Stream-ordered; FNE_EINVAL for other families or before a prepare.
 */
int fne_hvp_prepare(fne_handle* h, const double* u, void* stream);
int fne_hvp(fne_handle* h, const double* x, double* y, void* stream);
int fne_hvp_diagonal(fne_handle* h, double* diag, void* stream);
/*
 * Synchronous read of the handle's device status word (kernels that wait on
 * the tensor core, or on their own bulk copies into shared memory -- the
 * Mohr-Coulomb tensor-core kernel and the P1-triangle row-cluster kernel --
 * record a bounded wait that gave up there instead of hanging).  FNE_OK, or
 * FNE_ETIMEOUT (the word is then cleared).  No counterpart in the reference,
 * whose element kernels run on the CPU.
 */
int fne_check_device_status(fne_handle* h);
/*
 * The same status without a device synchronisation: every pass of those
 * kernels ends with a stream-ordered copy of the word into pinned host memory, and
 * this reads that copy.  Call it after synchronising the stream of the pass
 * (the assembler callbacks do so after each pass).  FNE_OK, or FNE_ETIMEOUT
 * (both copies are then cleared).  No counterpart in the reference.
 */
int fne_poll_device_status(fne_handle* h);
/*
 * Polls of the tensor-core kernel's per-tile MMA-completion wait before it
 * gives up (records FNE_ETIMEOUT, drains its own MMAs with the full bound,
 * frees its tensor memory and returns), or of the row-cluster kernel's waits
 * for its staging copies (records FNE_ETIMEOUT, waits for its own copies
 * with the full bound, writes no output and makes the energy NaN); polls < 0
 * restores the default (2^22).  0 makes every pass give up at once: how the
 * tests exercise the timeout path without a fault.  FNE_EINVAL for a handle
 * without either kernel.  No counterpart in the reference.
 */
int fne_set_wait_limit(fne_handle* h, int64_t polls);
/* Replace the Dirichlet values; ``dirichlet`` is a host array [n_total]. */
int fne_set_dirichlet(fne_handle* h, const double* dirichlet);
/*
 * One fused pass.  u: device [n_free] full reordered free vector (on one
 * rank this is the owned vector).  flags: FNE_ENERGY|FNE_GRAD|FNE_HESS.
 *   energy (device, 1 double)   sum_e w_e e_e - f.u_owned      (FP64 always)
 *   grad   (device, hi-lo doubles) owned gradient minus f
 *   hess   (device, nnz values)  owned COO values, float64, or float32 when
 *                                the handle was created with hess_fp32 = 1
 * Outputs for flags not set may be NULL.  Stream-ordered; no allocation.
 */
int fne_eval(fne_handle* h, const double* u, int flags, double* energy, double* grad,
             void* hess, void* stream);
/* Host convenience: same pass with host buffers (copies in and out). */
int fne_eval_host(fne_handle* h, const double* u_host, int flags, double* energy_host,
                  double* grad_host, void* hess_host);
int fne_destroy(fne_handle* h);

/*
 * No counterpart in the reference.  FP64 energy of P1-triangle p-Laplace /
 * Ginzburg-Landau elements WITHOUT any device allocation: for callers whose
 * device memory belongs to someone else -- a framework whose caching
 * allocator already holds the GPU's memory, or a solver that forbids
 * allocation once it is set up -- and who therefore cannot let a library
 * call cudaMalloc (fne_create allocates the element records and its scratch).
 * The caller passes every input and the output as device arrays:
 *   codes   [n_elem*3] int32 gather codes: >= 0 index into u, < 0 the
 *           Dirichlet entry -1-code of ``dirichlet``
 *   dvx, dvy [n_elem*3], vol [n_elem] float64 (the reference's element arrays)
 *   weights [n_elem] 0/1 energy weights, or NULL (all 1)
 *   params  HOST array laid out like fne_desc.s (p; or eps, ip[9], w[3])
 *   rhs     [n_owned] load vector or NULL; subtracts rhs . u[lo:lo+n_owned]
 *   energy  device double receiving sum_e w_e e_e - rhs.u
 * Scratch: a fixed device array inside libfne_asm.so (1024 FP64 partial sums
 * and a ticket, ~8 KB per GPU, held until the process exits); the grid is
 * capped at 1024 CTAs, so any n_elem up to 2^31-1 fits and larger sizes are
 * rejected with FNE_EBOUNDS.  Every call looks the array's device address up
 * with cudaGetSymbolAddress on the current device (so an address made stale
 * by cudaDeviceReset is never reused); the first call on a device may load
 * the library's device code, so make that first call before any stream
 * capture.  All calls share the array and it keeps the last call's contents
 * (the ticket is cleared by each call): calls that overlap on the GPU (other
 * streams, other threads) race and must be serialised by the caller.  No
 * cudaMalloc, cudaFree or allocating library routine is called.
 */
int fne_energy_p1tri_noalloc(int32_t family, int64_t n_elem, const int32_t* codes, const double* dvx,
                             const double* dvy, const double* vol, const double* weights, const double* u,
                             const double* dirichlet, const double* params, const double* rhs,
                             int64_t n_owned, int64_t lo, double* energy, void* stream);

/* ---------------------------------------------------------------------------
 * Newton linear solve on the device: Jacobi-preconditioned CG on the owned
 * COO Hessian.  Replaces, for single-GPU Newton runs, the KSP solve the
 * reference drives with the assembled matrix
 * (core/petsc/scalar_problem_driver.py:154-226: ksp.setOperators,
 * ksp.setTolerances(rtol, max_it), ksp.solve, ksp.getIterationNumber;
 * hyperelasticity/jax_petsc/solver.py:257-330 the same).  Every iteration
 * runs on the device (two kernels, in-kernel fixed-order reductions); the
 * host reads the solver state once per CUDA graph of `chunk` iterations.
 * ------------------------------------------------------------------------- */
typedef struct fne_cg fne_cg;
/* Square n x n pattern from the COO entries (rows[k], cols[k]), 0-based local
 * indices in [0, n) (host arrays, e.g. owned_rows - lo and owned_cols of a
 * one-rank layout); the CSR order keeps the COO order within a row.
 * vals_fp32 = 1 stores FP32 values (the FP32-Hessian assemblers' output),
 * 0 FP64; the arithmetic is FP64 either way.  FNE_EBOUNDS for an entry
 * outside the block.  Allocates all device memory the solves use. */
int fne_cg_create(int32_t n, int64_t nnz, const int64_t* rows, const int64_t* cols, int32_t vals_fp32,
                  int32_t chunk, fne_cg** out);
/* Takes the matrix values in COO order (device pointer, float or double as
 * created) and the Jacobi scaling 1/|a_ii| (1 for a missing, zero or NaN
 * diagonal).  Stream-ordered. */
int fne_cg_set_matrix(fne_cg* cg, const void* coo_vals, void* stream);
/* Solves A x = b (device pointers, FP64, length n) from x = 0.  Stops at the
 * first iterate with ||r|| <= rtol ||b||, at a non-positive curvature p.Ap
 * (returning the last iterate, or b itself at the first iteration), or after
 * maxit iterations.  *its = iterations taken (1 for the first-iteration
 * curvature stop, 0 for b = 0); *reason = 0 converged, 1 non-positive
 * curvature, 2 iteration limit, 3 zero right-hand side.  Synchronises the
 * stream once per `chunk` iterations; a handle runs one solve at a time. */
int fne_cg_solve(fne_cg* cg, const double* b, double* x, double rtol, int32_t maxit, int32_t* its, int32_t* reason,
                 void* stream);
int fne_cg_destroy(fne_cg* cg);

/* ---------------------------------------------------------------------------
 * Learned Newton warm start (no counterpart in the reference).  Kernels of a
 * small MLP over nodal features: BF16 operands, FP32 accumulation / master
 * weights.  All pointers are device pointers; BF16 arrays are passed as void*.
 * ------------------------------------------------------------------------- */
/* C[m, n] = sum_k A(m, k) B(k, n) + beta C[m, n], A(m, k) = A[m*sam + k*sak],
 * B(k, n) = B[k*sbk + n*sbn] (BF16), C row-major with leading dimension ldc
 * (FP32).  5th-generation tensor cores (tcgen05.mma kind::f16, FP32
 * accumulator in tensor memory), 128 x 128 (N > 32) or 128 x 32 tiles.
 * The MMA-completion waits are bounded: a CTA that gives up writes nothing
 * and sets the status fne_gemm_check_status reports. */
int fne_gemm_bf16(int M, int N, int K, const void* A, int64_t sam, int64_t sak, const void* B, int64_t sbk,
                  int64_t sbn, float* C, int64_t ldc, float beta, void* stream);
/* Synchronous read of the GEMM's status: FNE_OK, or FNE_ETIMEOUT when a wait
 * gave up since the last call (the status is then cleared). */
int fne_gemm_check_status(void);
/* Polls of each MMA-completion wait of later fne_gemm_bf16 calls; < 0
 * restores the default (2^22); 0 makes every tile give up at once (how the
 * tests exercise the timeout path without a fault). */
int fne_gemm_set_wait_limit(int64_t polls);
/* Z += bias (per column); H = silu(Z) (act = 1) or Z (act = 0); H32 / H16 may be NULL. */
int fne_mlp_bias_act(int64_t rows, int cols, float* Z, const float* bias, int act, float* H32, void* H16,
                     void* stream);
/* dZ = dH * silu'(Z) (act = 1) or dH (act = 0); dZ32 / dZ16 may be NULL. */
int fne_mlp_act_bwd(int64_t n, const float* Z, const float* dH, int act, float* dZ32, void* dZ16, void* stream);
/* out[c] = sum_r X[r, c] (FP64 accumulation, fixed order). */
int fne_mlp_colsum(int64_t rows, int cols, const float* X, float* out, void* stream);
/* One Adam step on FP32 parameters (bias-corrected with ``step`` >= 1);
 * writes the BF16 copy p16 when it is not NULL. */
int fne_mlp_adam(int64_t n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                 int step, void* p16, void* stream);
int fne_mlp_cast_bf16(int64_t n, const float* x, void* y, void* stream);

const char* fne_last_error(void);
const char* fne_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FNE_ASM_H */
