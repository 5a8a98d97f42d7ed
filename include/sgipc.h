/*
 * sgipc.h — C ABI of the B200-native per-Newton-iteration linear system of StiffGIPC.
 *
 * The reference has no C ABI; its C++ class interfaces are the API this header
 * replaces.  Every entry point below names the reference interface it stands in for.
 *
 * Conventions (all entry points):
 *   - return an SgipcStatus; nothing aborts or exits the process;
 *   - array arguments marked [dev] are caller-owned device pointers, [host] host ones;
 *   - `stream` is a cudaStream_t passed as void* (0 = legacy default stream); all work
 *     is stream-ordered and no entry point synchronises the device unless it returns a
 *     host-side scalar (documented per call);
 *   - one host thread per context, as the reference uses one host thread per GIPC
 *     object (StiffGIPC/gl_main.cu:100-108);
 *   - vectors of 3D points are packed double3 (x0,y0,z0,x1,...), 3x3 blocks are row-major.
 */
#ifndef SGIPC_H_
#define SGIPC_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum SgipcStatus {
    SGIPC_OK            = 0,
    SGIPC_CUDA_ERROR    = 1,  /* a CUDA runtime call or kernel launch failed */
    SGIPC_NOT_CONVERGED = 2,  /* PCG hit its iteration cap (reference: 0.3*dof, pcg_solver.cu:168) */
    SGIPC_BREAKDOWN     = 3,  /* p^T A p <= 0 or a non-finite scalar inside PCG */
    SGIPC_BAD_INPUT     = 4,  /* null pointer, negative count, index out of range, NaN input */
    SGIPC_CAPACITY      = 5,  /* more pairs/blocks than the context was created for */
    SGIPC_NOT_READY     = 6   /* a call whose prerequisite (assemble, mas_build) has not run */
} SgipcStatus;

typedef enum SgipcPrecision {
    SGIPC_FP64  = 0,  /* FP64 matrix, vectors and MAS domain inverses ("plain FP64 MAS-PCG") */
    SGIPC_MIXED = 1,  /* FP32 matrix copy, FP32 MAS and inner PCG; FP64 residual refinement */
    SGIPC_REF   = 2   /* the reference's shipping mix: FP64 matrix/PCG, FP32 MAS inverses */
} SgipcPrecision;

typedef enum SgipcCriterion {
    SGIPC_CRIT_RZ   = 0,  /* |r.z| <= tol * r0.z0, checked before the update (pcg_solver.cu:232) */
    SGIPC_CRIT_TRUE = 1   /* ||b - A x||_2 <= tol * ||b||_2 */
} SgipcCriterion;

/* Static topology, given once at context creation [host or dev: each array may be a host,
 * pinned, managed or device pointer; device arrays, as device_TetraData keeps them, are read
 * back once].  Mirrors what StiffGIPC's init reads: the tet/triangle/hinge connectivity
 * (device_TetraData, StiffGIPC/device_fem_data.cuh:17-78) and the MAS neighbour CSR + part
 * maps (MASPreconditioner::initPreconditioner_Neighbor, StiffGIPC/MASPreconditioner.cu:2264). */
typedef struct SgipcTopology {
    int32_t         vertex_num;
    int32_t         tet_num;
    int32_t         tri_num;
    int32_t         tri_edge_num;
    int32_t         soft_num;
    const uint32_t* tetrahedras;          /* uint4[tet_num] */
    const uint32_t* triangles;            /* uint3[tri_num] */
    const uint32_t* tri_edges;            /* uint2[tri_edge_num] */
    const int32_t*  tri_edge_adj_vertex;  /* int2[tri_edge_num], -1 = boundary hinge */
    const uint32_t* targetIndex;          /* uint32[soft_num] */
    /* MAS partition: positions padded to a multiple of 16 (partId_map_real = -1 on padding) */
    int32_t         part_map_size;
    const int32_t*  partId_map_real;      /* int[part_map_size] */
    const int32_t*  real_map_partId;      /* int[vertex_num] */
    const uint32_t* neighborStart;        /* uint[vertex_num + 1] (CSR; the reference keeps start+num) */
    const uint32_t* neighborList;         /* uint[neighborStart[vertex_num]] */
    /* capacities of the per-Newton contact inputs */
    int32_t         max_pairs;
    int32_t         max_ground;
    int32_t         max_fric_pairs;
    int32_t         max_fric_ground;
    int32_t         max_rhs;              /* right-hand sides batched in one adjoint solve (>= 1) */
} SgipcTopology;

/* Per-Newton FEM state [dev]; field names follow device_TetraData. */
typedef struct SgipcFemData {
    const double*   vertexes;             /* double3[V]  current iterate x */
    const double*   o_vertexes;           /* double3[V]  start-of-step positions (friction) */
    const double*   rest_vertexes;        /* double3[V]  rest positions (mollifier eps) */
    const double*   xTilta;               /* double3[V]  inertial target */
    const double*   masses;               /* double[V] */
    const int32_t*  BoundaryType;         /* int[V], 0 = free */
    const double*   DmInverses;           /* Matrix3x3d[T] row-major */
    const double*   volum;                /* double[T] */
    const double*   lengthRate;           /* double[T]  4*mu/3 */
    const double*   volumeRate;           /* double[T]  lambda + 5*mu/6 */
    const double*   triDmInverses;        /* Matrix2x2d[F] row-major */
    const double*   area;                 /* double[F]  area * thickness */
    const double*   quad_bending_Q;       /* Matrix4d[Eh] (column-major, as Eigen stores it) */
    const double*   targetVert;           /* double3[soft_num] */
} SgipcFemData;

/* Contact inputs of one Newton iteration [dev].  Encodings as produced by the
 * reference's LBVH queries (StiffGIPC/mlbvh.cu:560-1059). */
typedef struct SgipcContacts {
    const int32_t*  pairs;                /* int4[pair_num] */
    int32_t         pair_num;
    const uint32_t* ground_pairs;         /* uint[ground_num] vertex ids near the ground */
    int32_t         ground_num;
    /* lagged friction set-up (_calFrictionLastH_DistAndTan, StiffGIPC/GIPC.cu:8388) */
    const int32_t*  fric_pairs;           /* int4[fric_num] */
    const double*   fric_lambda;          /* double[fric_num] lagged normal force */
    const double*   fric_coord;           /* double2[fric_num] closest-point coordinates */
    const double*   fric_basis;           /* Matrix3x2d[fric_num] row-major tangent basis */
    int32_t         fric_num;
    const uint32_t* fric_gd_pairs;        /* uint[fric_gd_num] */
    const double*   fric_gd_lambda;       /* double[fric_gd_num] */
    int32_t         fric_gd_num;
} SgipcContacts;

/* Scalars of the Newton system (the GIPC members read by computeGradientAndHessian). */
typedef struct SgipcParams {
    double dt;               /* IPC_dt */
    double dHat;             /* squared barrier distance (GIPC.cu:8602) */
    double kappa;            /* barrier stiffness */
    double fDhat;            /* friction d-hat, squared (GIPC.cu:8603); eps_f^2 = fDhat*dt^2 */
    double frictionRate;     /* mu for pair friction */
    double gd_frictionRate;  /* mu for ground friction */
    double ground_offset;    /* plane n.x = offset, n = +y (GIPC.cu:8541-8549) */
    double stretchStiff;     /* cloth membrane */
    double shearStiff;
    double strainRate;
    double bendStiff;
    double motionRate;       /* soft constraint stiffness */
    double softRate;         /* soft constraint rate (squared inside) */
} SgipcParams;

typedef struct SgipcSolveStats {
    int32_t iterations;          /* PCG iterations (inner iterations summed in MIXED mode) */
    int32_t refinements;         /* outer refinement steps (MIXED) */
    double  rz0;                 /* r0.z0 */
    double  rz;                  /* final r.z */
    double  rel_residual;        /* ||b - A x|| / ||b|| recomputed in FP64 */
    int32_t status;              /* SgipcStatus of the solve */
} SgipcSolveStats;

typedef struct SgipcCtx SgipcCtx;

/* ---- context ------------------------------------------------------------------------ */

/* Builds the static symmetric-upper BSR pattern of the FEM topology (tets, triangles,
 * hinges, mass diagonal), the element -> slot maps and the MAS level-0 tables, and
 * allocates every workspace.  Replaces GIPC::init's triplet buffers (GIPC.cu:8593-8640),
 * MASPreconditioner::initPreconditioner_Neighbor/_Matrix (MASPreconditioner.cu:2264-2330)
 * and PCGSolver's vectors (pcg_solver.cu:158-172).  Synchronises the device. */
SgipcStatus sgipc_create(const SgipcTopology* topo, int device, SgipcCtx** out);
SgipcStatus sgipc_destroy(SgipcCtx* ctx);
const char* sgipc_status_string(SgipcStatus s);
/* Last CUDA error text recorded on the context (empty if none). */
const char* sgipc_last_error(const SgipcCtx* ctx);
/* How long a grid-barrier wait inside the persistent PCG solve and the one-launch MAS
 * hierarchy build may last, in polls of the arrival counter (0 = the defaults, about 2 s;
 * new; the reference synchronises on the host and has no device waits).  A wait that runs
 * out raises the kernel's abort word, every CTA leaves, and the call returns
 * SGIPC_CUDA_ERROR with a message, the context staying usable.  A watchdog for hosts that
 * must bound a call's time; 1 makes nearly every wait run out. */
SgipcStatus sgipc_set_wait_limit(SgipcCtx* ctx, int64_t polls);

/* ---- assembly (GIPC::computeGradientAndHessian, StiffGIPC/GIPC.cu:10110-10344) -------- */

/* Full assembly: kinetic gradient, barrier, friction, ground, soft constraints, stable
 * Neo-Hookean tets, cloth membrane, quadratic bending, Dirichlet zeroing and the mass
 * diagonal, written straight into the context's BSR (static part) and contact BCOO
 * (dynamic part), plus the right-hand side b = fb + shape_grads with Dirichlet rows
 * zeroed (FEMLinearSubsystem::assemble, fem_linear_subsystem.cu:56-84).  Stream-ordered.
 * It also starts the MAS hierarchy for con's pairs on the context's own stream, beside the
 * assembly (the hierarchy needs the contact graph, not the matrix), and scatters the static
 * blocks into its domains there once they are assembled; the next
 * sgipc_mas_build / sgipc_solve given the same pair array and count uses it, so the pair
 * array must stay unchanged until that call. */
SgipcStatus sgipc_assemble(SgipcCtx* ctx, const SgipcFemData* fem, const SgipcContacts* con,
                           const SgipcParams* prm, void* stream);

/* GIPC::calBarrierGradientAndHessian (GIPC.cu:9112): barrier gradient added into
 * grad [dev double3[V]] and barrier blocks written into the contact BCOO. */
SgipcStatus sgipc_barrier_grad_hess(SgipcCtx* ctx, const SgipcFemData* fem,
                                    const SgipcContacts* con, const SgipcParams* prm,
                                    double* grad, void* stream);
/* GIPC::calFrictionGradient + calFrictionHessian (GIPC.cu:9164-9217). */
SgipcStatus sgipc_friction_grad_hess(SgipcCtx* ctx, const SgipcFemData* fem,
                                     const SgipcContacts* con, const SgipcParams* prm,
                                     double* grad, void* stream);
/* femEnergy.cu:1719 _calculate_fem_gradient_hessian: SNK gradient added into grad and
 * element blocks gathered into the static BSR values. */
SgipcStatus sgipc_fem_grad_hess(SgipcCtx* ctx, const SgipcFemData* fem, const SgipcParams* prm,
                                double* grad, void* stream);

/* Copy the assembled upper block matrix out as merged, sorted BCOO (static + contact,
 * duplicates summed) [host arrays of capacity cap blocks].  Synchronises.  For parity
 * tests and checkpoints: the layout of GIPCTripletMatrix after Converter::convert. */
SgipcStatus sgipc_export_bcoo(SgipcCtx* ctx, int32_t cap, int32_t* rows, int32_t* cols,
                              double* vals, int32_t* count);
/* Right-hand side b [dev double[3n]] of the last assembly. */
SgipcStatus sgipc_get_rhs(SgipcCtx* ctx, double* b, void* stream);
/* GIPC::computeEnergy (GIPC.cu:10520-10580), the line-search objective, for the FEM part at
 * fem->vertexes: kinetic + dt^2 (tets + triangles + hinges) + soft constraints + barrier +
 * kappa ground + frictionRate friction + gd_frictionRate ground friction, with the per-term
 * reductions of Energy_Add_Reduction_Algorithm (GIPC.cu:10347-10518).  Each term is summed
 * in a fixed order, so the result is the same on every run.  *energy receives the total;
 * terms (optional, host, double[9]) the nine parts in that order.  Needs no assembly first;
 * synchronises the stream. */
SgipcStatus sgipc_compute_energy(SgipcCtx* ctx, const SgipcFemData* fem, const SgipcContacts* con,
                                 const SgipcParams* prm, double* energy, double* terms, void* stream);
/* GIPC::self_largestFeasibleStepSize (GIPC.cu:8880-8914; per candidate
 * _reduct_min_selfTimeStep_to_double GIPC.cu:7052 with the additive CCD of ACCD.cu:373-535):
 * the largest step alpha <= 1 along -move_dir (the reference's moveDir) that keeps every
 * candidate pair apart by the fraction 1 - slackness of its current distance.  pairs:
 * int32[4] per candidate, x < 0 for point -x-1 against triangle (y, z, w), else edge (x, y)
 * against edge (z, w).  x, move_dir: device double3 per vertex; toi (optional, device,
 * double[npairs]) receives each candidate's time of impact.  Returns SGIPC_BAD_INPUT for a
 * vertex index outside the context's vertices.  Synchronises the stream. */
SgipcStatus sgipc_self_step_size(SgipcCtx* ctx, const double* x, const double* move_dir, const int32_t* pairs,
                                 int32_t npairs, double slackness, double* alpha, double* toi, void* stream);
/* GIPC::ground_largestFeasibleStepSize (GIPC.cu:8986-9025; per vertex
 * _reduct_min_groundTimeStep_to_double GIPC.cu:6902): the step bound of the vertices verts
 * against the plane y = ground_offset (normal +y), alpha = 1 / max(1, move_dir_y / ((y -
 * offset) slackness)) over the vertices with move_dir_y > 0.  Synchronises the stream. */
SgipcStatus sgipc_ground_step_size(SgipcCtx* ctx, const double* x, const double* move_dir, const uint32_t* verts,
                                   int32_t nverts, double ground_offset, double slackness, double* alpha,
                                   void* stream);
/* GIPC::cfl_largestSpeed (GIPC.cu:8916-8944; per vertex _reduct_max_cfl_to_double
 * GIPC.cu:7157): the largest |move_dir| over the vertices verts (0 for none), from which
 * the reference bounds the step by sqrt(dHat) / (2 speed).  Synchronises the stream. */
SgipcStatus sgipc_cfl_largest_speed(SgipcCtx* ctx, const double* move_dir, const uint32_t* verts, int32_t nverts,
                                    double* speed, void* stream);
/* GIPC::step_forward (GIPC.cu:9637; _stepForward :7937): the line search's trial positions
 * x = x_base - alpha move_dir for the vertices with boundary_type 0 (all of them when
 * move_boundary is nonzero); the others keep their x.  Device double3 arrays of the
 * context's vertices; x may not alias x_base.  Stream-ordered. */
SgipcStatus sgipc_step_forward(SgipcCtx* ctx, double* x, const double* x_base, const double* move_dir,
                               const int32_t* boundary_type, double alpha, int32_t move_boundary, void* stream);

/* ---- operators --------------------------------------------------------------------- */

/* y = A x with the assembled symmetric matrix (Spmv::warp_reduce_sym_spmv, spmv.cu:8). */
SgipcStatus sgipc_spmv(SgipcCtx* ctx, const double* x, double* y, void* stream);

/* MASPreconditioner::setPreconditioner_bcoo (MASPreconditioner.cu:2180): per-Newton
 * hierarchy with contact connectivity, domain matrices and their inverses. */
SgipcStatus sgipc_mas_build(SgipcCtx* ctx, const SgipcContacts* con, SgipcPrecision prec,
                            void* stream);
/* MASPreconditioner::preconditioning (MASPreconditioner.cu:2221): z = M^-1 r. */
SgipcStatus sgipc_mas_apply(SgipcCtx* ctx, const double* r, double* z, void* stream);
/* The same z = M^-1 r, for callers that may not allocate device memory during a call (a
 * host whose pool owns every device allocation, or a loop where an allocation's implicit
 * synchronisation is not allowed).  No counterpart in the reference.  It allocates nothing:
 * its two work vectors live in one fixed array compiled into the library, 3 MiB on every
 * device that loads it, kept until the process exits, serving hierarchies of at most 65536
 * clusters (sgipc_mas_info's total); larger ones return SGIPC_CAPACITY with a message.  The
 * first call on a device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture.  All calls on a device share the array:
 * calls whose work overlaps on the GPU (other streams, other contexts) race and must be
 * ordered by the caller. */
SgipcStatus sgipc_mas_apply_noalloc(SgipcCtx* ctx, const double* r, double* z, void* stream);
/* Host copy of the level structure: levels, per-level node counts, total clusters. */
SgipcStatus sgipc_mas_info(SgipcCtx* ctx, int32_t* levelnum, int32_t* level_counts /*[8]*/,
                           int32_t* total_clusters);
/* Host copy of the per-vertex coarse node table (global cluster index of each vertex at
 * levels 1..levelnum-1, int[V*(levelnum-1)]) for hierarchy parity tests. */
SgipcStatus sgipc_mas_export_tables(SgipcCtx* ctx, int32_t* table);

/* Host copy of the MAS domain inverses, total_clusters/16 dense row-major 48x48 blocks
 * (FP64; FP32-built inverses are widened), in the order of the global cluster index —
 * the contents of MASPreconditioner::d_inverseMatMas / d_precondMatMas
 * (MASPreconditioner.cuh:44-45) unpacked.  For checkpoints and parity tests. */
SgipcStatus sgipc_mas_export_domains(SgipcCtx* ctx, double* inverses);

/* Restriction of r [dev double3[V]] to every level, R [host double[3*total_clusters]]
 * indexed by global cluster (__buildMultiLevelR_optimized_new, MASPreconditioner.cu:729).
 * Synchronises.  For parity tests of the restriction operator. */
SgipcStatus sgipc_mas_restrict(SgipcCtx* ctx, const double* r, double* R);

/* ---- solve ------------------------------------------------------------------------- */

/* PCGSolver::pcg (pcg_solver.cu:174-267) on the assembled system: x [dev] = A^-1 b.
 * max_iter <= 0 selects the reference cap 0.3*dof.  Fills stats [host]; synchronises. */
SgipcStatus sgipc_pcg_solve(SgipcCtx* ctx, SgipcPrecision prec, SgipcCriterion crit,
                            double tol, int32_t max_iter, const double* b, double* x,
                            SgipcSolveStats* stats, void* stream);

/* Batched PCG on nrhs right-hand sides sharing A and M (b, x: [dev] nrhs x 3n, rhs-major). */
SgipcStatus sgipc_pcg_solve_batched(SgipcCtx* ctx, SgipcPrecision prec, SgipcCriterion crit,
                                    double tol, int32_t max_iter, int32_t nrhs,
                                    const double* b, double* x, SgipcSolveStats* stats,
                                    void* stream);

/* GIPC::calculateMovingDirection (GIPC.cu:10581-10592): MAS build + PCG on the
 * assembled system, move_dir [dev double3[V]] = dx.  Synchronises (returns stats). */
SgipcStatus sgipc_solve(SgipcCtx* ctx, const SgipcContacts* con, SgipcPrecision prec,
                        SgipcCriterion crit, double tol, int32_t max_iter, double* move_dir,
                        SgipcSolveStats* stats, void* stream);

/* ---- adjoint (new; no counterpart in the reference) --------------------------------- */

/* Parameter derivatives of the gradient g(x; E, v0) at the assembled state, contracted
 * with nrhs adjoint vectors lambda [dev nrhs x 3V]:
 *   dLdE  [dev nrhs x T]  = -lambda^T dg/dE_t   (stable Neo-Hookean, per tet)
 *   dLdv0 [dev nrhs x 3V] = +dt * m_i * lambda_i (g_kin = M(x - x_prev - dt v0 - dt^2 g))
 * poisson: Poisson ratio used to split E into (lengthRate, volumeRate). */
SgipcStatus sgipc_adjoint_param_grads(SgipcCtx* ctx, const SgipcFemData* fem,
                                      const SgipcParams* prm, double poisson, int32_t nrhs,
                                      const double* lambda, double* dLdE, double* dLdv0,
                                      void* stream);

/* ---- affine bodies (ABDSystem / ABDPreconditioner) ----------------------------------- */

/* Static description of the affine bodies [host], what ABDSystem::init derives
 * (StiffGIPC/abd_system/abd_system.cu:50-140).  Body b owns the block rows 4b..4b+3 of the
 * global system (translation p, then the rows a1, a2, a3 of its affine matrix); FEM rows
 * follow at 4 * body_num.  ABD points are numbered body by body (non-decreasing
 * point_body), as the reference's unique points are. */
typedef struct SgipcAbdTopology {
    int32_t        body_num;
    int32_t        point_num;           /* ABD points */
    const int32_t* point_body;          /* int[point_num]  unique_point_id_to_body_id */
    const double*  x_bar;               /* double3[point_num]  ABDJacobi::x_bar */
    const double*  dyadic_mass;         /* double[13 * body_num]: m, m x_bar (3), m x_bar x_bar^T (9,
                                         * row-major) -- ABDJacobiDyadicMass */
    const double*  volume;              /* double[body_num] */
    const int32_t* boundary_type;       /* int[body_num]: 0 free, 1 fixed (BodyBoundaryType) */
    int32_t        max_abd_blocks;      /* capacity: ABD-ABD point blocks per call */
    int32_t        max_fem_blocks;      /* capacity: ABD-FEM point blocks per call */
} SgipcAbdTopology;

typedef struct SgipcAbdCtx SgipcAbdCtx;

SgipcStatus sgipc_abd_create(const SgipcAbdTopology* topo, int device, SgipcAbdCtx** out);
SgipcStatus sgipc_abd_destroy(SgipcAbdCtx* ctx);
const char* sgipc_abd_last_error(const SgipcAbdCtx* ctx);

/* ABDSystem::setup_abd_system_gradient_hessian (setup_abd_system_gradient_and_hessian.cu:
 * 162-181, 200-610): per body the kinetic term M (q - q_tilde) with the dyadic mass and the
 * orthogonality potential kappa * volume * dt^2 * V_perp(q) (abd_energy.inl:9-127, its 9x9
 * Hessian projected to PSD); point barrier gradients mapped to bodies with J^T
 * (point_grad [dev double3[point_num]], may be null); point-space contact blocks mapped to
 * body space: ABD-ABD blocks [dev] (rows, cols = ABD point ids, row <= col, row-major 3x3)
 * to J_i^T H J_j, ABD-FEM blocks (rows = ABD point, cols = FEM-local vertex) to J_i^T H in
 * column 4 * body_num + col (zeroed where fem_boundary [dev int per FEM vertex, may be
 * null] is non-zero).  Fixed bodies: zero gradient, mass-only Hessian, zero contact
 * blocks.  Writes body_grad [dev double[12 * body_num]] and keeps the merged upper
 * body-space BCOO in the context. */
SgipcStatus sgipc_abd_grad_hess(SgipcAbdCtx* ctx, const double* q, const double* q_tilde, double kappa,
                                double dt, const double* point_grad, int32_t abd_blocks,
                                const int32_t* abd_rows, const int32_t* abd_cols, const double* abd_vals,
                                int32_t fem_blocks, const int32_t* fem_rows, const int32_t* fem_cols,
                                const double* fem_vals, const int32_t* fem_boundary, double* body_grad,
                                void* stream);
/* Host copy of the merged upper body-space blocks of the last sgipc_abd_grad_hess (block
 * rows < 4 * body_num; columns >= 4 * body_num are FEM rows).  Synchronises. */
SgipcStatus sgipc_abd_export_bcoo(SgipcAbdCtx* ctx, int32_t cap, int32_t* rows, int32_t* cols,
                                  double* vals, int32_t* count);
/* ABDPreconditioner::assemble (abd_preconditioner.cu:15-38, _cal_abd_system_preconditioner
 * setup_abd_system_gradient_and_hessian.cu:612-655): the inverse of every body's 12x12
 * diagonal block of the assembled body-space matrix. */
SgipcStatus sgipc_abd_precond_build(SgipcAbdCtx* ctx, void* stream);
/* ABDPreconditioner::apply: z_b = P_b^-1 r_b, r and z [dev double[12 * body_num]]. */
SgipcStatus sgipc_abd_precond_apply(SgipcAbdCtx* ctx, const double* r, double* z, void* stream);

/* The class partition of the contact terms (GIPC::partitionContactHessian, GIPC.cu:9932-10108,
 * with the contact gradient of the ABD points) for a context whose vertices [abd_first, nv)
 * are the points of affine bodies, marked Dirichlet in fem->BoundaryType so that sgipc_assemble
 * keeps only the FEM-FEM parts of the contact terms in its matrix.  The barrier, friction and
 * ground terms of `con` are evaluated at fem->vertexes; their blocks that touch an ABD point
 * are written in slot order to the caller's device arrays: ABD-ABD blocks (rows, cols = ABD
 * point ids counted from abd_first, row <= col, row-major 3x3) and ABD-FEM blocks (rows = ABD
 * point id, cols = FEM vertex, the block in that orientation), up to cap of each, with their
 * counts on the host; point_grad [dev double3[nv - abd_first], may be null] receives the
 * contact gradient at the ABD points.  These are the inputs of sgipc_abd_grad_hess.
 * Synchronises; SGIPC_CAPACITY when a count exceeds cap (the count is still returned). */
SgipcStatus sgipc_contact_partition(SgipcCtx* ctx, const SgipcFemData* fem, const SgipcContacts* con,
                                    const SgipcParams* prm, int32_t abd_first, int32_t cap, int32_t* abd_rows,
                                    int32_t* abd_cols, double* abd_vals, int32_t* abd_count, int32_t* fem_rows,
                                    int32_t* fem_cols, double* fem_vals, int32_t* fem_count, double* point_grad,
                                    void* stream);

/* ---- barrier stiffness (kappa) adaptation ----------------------------------------------- */

/* GIPC::initKappa with suggestKappa and upperBoundKappa (GIPC.cu:9850-9929): with contact
 * pairs, kappa = -(g_c . g_E) / (g_c . g_c) where g_E is the kinetic, tet elastic and soft-
 * constraint gradient and g_c the barrier and ground gradient at kappa = 1 (both at
 * fem->vertexes), raised to the suggested minimum minKappaCoef * meanMass / (4e-16 bbox^2
 * H_b) and bounded by 100 times it (meanMass 0: without it).  kappa [host, in/out] keeps its
 * value without pairs.  Uses the context's element gradient scratch: call it before
 * sgipc_assemble, as the reference does.  Synchronises. */
SgipcStatus sgipc_init_kappa(SgipcCtx* ctx, const SgipcFemData* fem, const SgipcContacts* con,
                             const SgipcParams* prm, double mean_mass, double bbox_diag2, double min_kappa_coef,
                             double* kappa, void* stream);
/* GIPC::computeCloseGroundVal / computeSelfCloseVal (GIPC.cu:8776, 9219): records the ground
 * vertices of con [dev] whose squared distance to the plane y = ground_offset, and the pairs
 * whose squared distance, is below dtol (the reference's dTol = 1e-18 bbox^2), with those
 * values, at x [dev].  counts [host int[2], may be null]: ground vertices and pairs recorded.
 * Synchronises. */
SgipcStatus sgipc_close_record(SgipcCtx* ctx, const double* x, const SgipcContacts* con, double dtol,
                               double ground_offset, int32_t* counts, void* stream);
/* GIPC::checkCloseGroundVal || checkSelfCloseVal (GIPC.cu:8794, 9230): *changed = 1 when a
 * recorded ground vertex or pair is closer at x [dev] than when it was recorded (the caller
 * then doubles kappa and bounds it, GIPC::postLineSearch GIPC.cu:10777-10806).  Synchronises. */
SgipcStatus sgipc_close_check(SgipcCtx* ctx, const double* x, double ground_offset, int32_t* changed,
                              void* stream);

/* ---- the global FEM + ABD system ------------------------------------------------------- */

/* GlobalLinearSystem::solve_linear_system + distribute_solution (global_linear_system.cu:
 * 8-166, gipc/gipc.cu:42-70) with the ABD and FEM subsystems: PCGSolver::pcg
 * (pcg_solver.cu:174-267, FP64 vectors) on the global vector [12 * body_num ABD DOFs |
 * 3 * n FEM DOFs].  A = the FEM context's assembled matrix on the FEM rows plus the ABD
 * context's merged body-space blocks (body rows and body x FEM coupling) with their
 * transposes; M = the ABD block Jacobi (sgipc_abd_precond_build) on the body rows and the
 * FEM context's MAS (sgipc_mas_build; FP64 or FP32 inverses as built) on the FEM rows.
 * b, x [dev double[12 * body_num + 3 n]]; abd_point_dx [dev double3[point_num], may be
 * null] receives J(x_bar) dq of every ABD point.  max_iter <= 0: 0.3 x DOFs.  Returns
 * SGIPC_NOT_READY unless both systems are assembled and both preconditioners built.
 * Synchronises (one read-back of the loop's device-side state per iteration). */
SgipcStatus sgipc_global_pcg_solve(SgipcCtx* fem, SgipcAbdCtx* abd, SgipcCriterion crit, double tol,
                                   int32_t max_iter, const double* b, double* x, double* abd_point_dx,
                                   SgipcSolveStats* stats, void* stream);

/* ---- contact pairs and the lagged friction set-up -------------------------------------- */

/* Collision surface [dev]: the surface points, triangles (uint3) and edges (uint2) the
 * contact-pair search reads (GIPC's _surfVerts, bvh_f._faces, bvh_e._edges).  Every vertex
 * of a triangle or an edge must be a surface point. */
typedef struct SgipcSurface {
    const uint32_t* surf_verts;
    int32_t         surf_vert_num;
    const uint32_t* faces;
    int32_t         face_num;
    const uint32_t* edges;
    int32_t         edge_num;
} SgipcSurface;

/* GIPC::buildCP (GIPC.cu:9065-9083: the LBVH queries _selfQuery_vf / _selfQuery_ee with
 * _checkPTintersection / _checkEEintersection, mlbvh.cu:534-1059, 1306-1742, and
 * _GroundCollisionDetect GIPC.cu:6433): every surface point within sqrt(dHat) of a triangle
 * and every edge pair within it, at positions x [dev double3[V]], mollifier thresholds from
 * rest [dev double3[V]].  A pair is tested when its vertices belong to different bodies or
 * the body id is -1 (body_id [dev int[V]]; -1 everywhere collides every body with itself),
 * shares no vertex, and not all of its vertices have boundary type >= 2 (boundary_type [dev
 * int[V]], may be null).  Writes [dev] pairs int4[cap] in the reference encoding, ccd_pairs
 * int4[cap] (the point with the whole triangle, or the two edges), mat_index int[cap] (rank
 * among the pairs of the same size), cp_num uint[5] (total, 0, two-, three-, four-vertex
 * pairs), ground_pairs uint[ground_cap] (surface points with (y - ground_offset)^2 <= dHat,
 * normal +y) and gp_num uint[1]; h_cp_num [host uint[5]] and h_gp_num [host] receive the
 * counts, as the reference copies h_cpNum / h_gpNum.  The order is deterministic:
 * point-triangle pairs by surface point then triangle, then edge-edge pairs by edge then
 * other edge.  SGIPC_CAPACITY (counts reported, pairs unwritten) when cap or ground_cap is
 * too small; cap must stay below 2^21.  Synchronises the stream. */
SgipcStatus sgipc_build_cp(SgipcCtx* ctx, const double* x, const double* rest, const SgipcSurface* surf,
                           const int32_t* body_id, const int32_t* boundary_type, double dHat, double ground_offset,
                           int32_t cap, int32_t* pairs, int32_t* ccd_pairs, int32_t* mat_index, uint32_t* cp_num,
                           int32_t ground_cap, uint32_t* ground_pairs, uint32_t* gp_num, uint32_t* h_cp_num,
                           uint32_t* h_gp_num, void* stream);

/* The lagged friction set-up of a frame (_calFrictionLastH_DistAndTan / _calFrictionLastH_gd,
 * GIPC.cu:8362-8499, called from GIPC.cu:8660-8696), at the frame's positions x [dev]: for
 * every pair [dev int4[pair_num]] that is not mollified, in input order, the pair, its lagged
 * normal force, closest-point coordinates (double2) and tangent basis (3 x 2 row-major) into
 * fric_pairs / fric_lambda / fric_coord / fric_basis [dev, pair_num entries at most];
 * cp_num_last [dev uint[5]] = (kept pairs, 0, point-point, point-edge, point-triangle and
 * edge-edge); and for the ground pairs [dev uint[ground_num]] their vertices and normal forces
 * (fric_gd_pairs, fric_gd_lambda).  A pair or ground pair naming a vertex outside the mesh is
 * left out and sets cp_num_last[1].  h_cp_num_last [host uint[5], may be null] receives the
 * counts (then the call synchronises the stream, and returns SGIPC_BAD_INPUT for such a pair). */
SgipcStatus sgipc_friction_setup(SgipcCtx* ctx, const double* x, const int32_t* pairs, int32_t pair_num,
                                 const uint32_t* ground_pairs, int32_t ground_num, double dHat, double kappa,
                                 double ground_offset, int32_t* fric_pairs, double* fric_lambda, double* fric_coord,
                                 double* fric_basis, uint32_t* cp_num_last, uint32_t* fric_gd_pairs,
                                 double* fric_gd_lambda, uint32_t* h_cp_num_last, void* stream);

/* ---- instrumentation (the reference's gipc::Timer / cudaEvent phase timers,
 *      StiffGIPC/gipc/utils/timer.h:19-136, GIPC.cu:10854-10964) ----------------------- */

/* Number of this library's kernels launched on the context since creation (library
 * kernels such as CUB sorts excluded; a persistent PCG solve counts as one launch, a
 * graph-resident PCG loop by the iteration bodies it executed).  Synchronises. */
SgipcStatus sgipc_launch_count(SgipcCtx* ctx, int64_t* launches);

/* Re-launch one hot kernel `reps` times on `stream` against the context's current state,
 * bracketed by CUDA events on that stream, and return its average duration [ms] and the
 * algorithmic bytes one launch must move.  Names: "snk", "gather_blocks", "barrier",
 * "friction", "spmv64", "spmv32", "mas_scatter", "mas_invert", "mas_domain64",
 * "mas_domain32", and "pcg32" / "pcg64" (one whole persistent PCG solve of the last
 * right-hand side to the 1e-4 r.z criterion, with FP32 / FP64 vectors; the MAS must have
 * been built in that precision).  Leaves the assembled system and the MAS state as they were (the
 * MAS kernels rebuild what they overwrite).  Synchronises. */
SgipcStatus sgipc_time_kernel(SgipcCtx* ctx, const char* name, int32_t reps, void* stream,
                              float* avg_ms, double* bytes_per_launch);

/* Phase profile of one persistent PCG solve (the reference's per-phase gipc::Timer, here
 * inside the one-kernel solve): runs one solve of the last assembled right-hand side to the
 * 1e-4 r.z criterion ("pcg32" / "pcg64": FP32 / FP64 vectors, one right-hand side;
 * "pcg32x4" / "pcg64x4": four copies of it interleaved, as the adjoint's batched solve) with
 * every CTA recording the device clock (%globaltimer, ns) when it arrives at and leaves each
 * grid barrier.  stamps [host uint64, (grid capacity) x max_epochs x 2 + max_epochs]: entry
 * [(cta * max_epochs + e) * 2 + {0, 1}] = arrival at / departure from barrier e (e = 0: the
 * kernel's start and the end of its shared-memory loads; later epochs past the solve's last
 * barrier stay 0), then at [capacity * max_epochs * 2 + e] the phase that ends at barrier e
 * (1 init, 2 MAS domain solves, 3 coarser-level solves, 4 prolongation, 5 SpMV, 6 update and
 * restriction, 7-10 the mixed solve's refinement epilogue).  *grid receives the CTAs of the
 * launch, *epochs the barriers recorded.  The grid capacity is 2 x the device's SM count.
 * Allocates and frees a device buffer, and synchronises.  SGIPC_NOT_READY when the device
 * runs the per-phase-kernel graph instead. */
SgipcStatus sgipc_profile_pcg(SgipcCtx* ctx, const char* name, int32_t max_epochs, uint64_t* stamps,
                              int32_t* grid, int32_t* epochs, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SGIPC_H_ */
