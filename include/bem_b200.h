/*
 * bem_b200.h — C ABI of the B200 (sm_100a) GMRES + FMM Laplace boundary-value solver.
 *
 * Drop-in for the reference's GMRES-FMM branch of BEM_BVP::solve()
 * (bem/BEM_solveBVP.hpp:565-630 -> solveGMRES, bem/BEM_solveBVP_GMRES_FMM.hpp:3056-3506):
 * mesh, boundary types and known phi/phin in; phi/phin per DOF out.
 * Conventions follow the reference's Metal plugins (bem/metal_m2l/metal_m2l.h:23-130):
 * opaque context, create() returns NULL on failure, int status (0 = success), no C++
 * exceptions cross this boundary, plain pointers and sizes only.
 *
 * All arrays are HOST memory unless a function name ends in _device.
 * Units: coordinates and known values are physical; the solver applies the reference's
 * coordinate scaling internally (x' = x/L, L = bounding-box diagonal) and returns
 * physical values.
 */
#ifndef BEM_B200_H
#define BEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define BEM_OK 0
#define BEM_ERR_INVALID_ARGUMENT -1
#define BEM_ERR_OUT_OF_MEMORY -2
#define BEM_ERR_NOT_CONVERGED -3
#define BEM_ERR_NAN -4
#define BEM_ERR_DEVICE -5
#define BEM_ERR_NOT_READY -6
#define BEM_ERR_UNSUPPORTED -7

/* DOF kinds (bem/BEM_setBoundaryTypes.hpp:29-100):
 *   0: Dirichlet key (p, null): phi known, phin unknown
 *   1: Neumann key  (p, null) or (p, f): phin known, phi unknown
 *   2: Neumann key (p, f) of a CORNER point: phi unknown and constrained to the point's
 *      Dirichlet phi (constraint row A v = phi, BEM_solveBVP_GMRES_FMM.hpp:100-108, 2031-2047) */
#define BEM_DOF_DIRICHLET 0
#define BEM_DOF_NEUMANN 1
#define BEM_DOF_CORNER_NEUMANN 2

typedef struct bem_gpu_ctx bem_gpu_ctx;

/* Solver options.  Replaces the reference's globals fmm_max_level, fmm_bucket_max_points,
 * g_mac_theta, solver_tol, solver_max_iter (bem/main_time_domain.cpp:52-62) and the
 * compile-time expansion order of B_poles (bem/BEM_solveBVP.hpp:563). */
typedef struct {
  int32_t expansion_order;   /* p, 1..12 (reference default 10) */
  double mac_theta;          /* MAC parameter theta (0.25) */
  int32_t leaf_max_elements; /* a bucket splits while it holds more elements than this */
  int32_t max_level;         /* deepest octree level (7) */
  double tol;                /* absolute GMRES tolerance on the scaled system (solver_tol) */
  int32_t max_iter;          /* GMRES iteration cap (solver_max_iter) */
  int32_t device;            /* CUDA device ordinal */
  int32_t tol_relative;      /* 0: stop at |A x - b| <= tol (reference semantics); 1: at <= tol*|b| */
  int32_t preconditioner;    /* 0: none (reference default); 1: right Jacobi from the near-field diagonal;
                                2: right near-field polynomial -- D^-1 p(A_near D^-1), p the GMRES
                                polynomial (harmonic Ritz roots) of a poly_degree-step Arnoldi run on
                                A_near D^-1; the device counterpart of the reference's near-field
                                ILU/Schwarz preconditioners (bem/BEM_solveBVP_GMRES_FMM.hpp:215-1050);
                                3: right near-block -- block Jacobi over the DOFs of each near block's
                                targets (the reference's additive Schwarz, :899-1013, with bucket
                                cores and no overlap), inverses formed at set-up */
  int32_t precision;         /* 0: FP64 throughout; 1: mixed -- GMRES corrections use the tensor-core
                                M2L (FP16 split operands, FP32 accumulate), FP64 outer refinement on the
                                true residual, same stopping test; needs p <= 12 */
  int32_t poly_degree;       /* preconditioner 2: polynomial degree 1..24 (0: 8) */
  int32_t tree_on_host;      /* 0: the octree is grown on the device (tree.cu), 1: on the host; same tree */
  int32_t tc_item_pairs;     /* mixed: pairs per tensor-core M2L work item, 1..128 (p <= 10) or 1..80;
                                0: autotuned (once per process and problem class; the result does not
                                depend on it) */
  int32_t overlap_near;      /* 1 (bem_gpu_default_opts) = the near-field sums of A.x run on a
                                second stream while the FMM passes run, the rows after both; 0 = the
                                near sums after the FMM passes on one stream */
  double refine_rtol;        /* mixed: each inner GMRES cycle on the low-precision operator stops at
                                max(tol, refine_rtol * |r|) before the FP64 residual update (0: 1e-6) */
  int32_t tc_deterministic;  /* mixed: 0 = the tensor-core M2L adds each pair's translated expansion into
                                its target's FP32 accumulator in L2 (fast; the summation order, and so the
                                last bits, vary between runs); 1 = per-pair partials summed in a fixed
                                order (bit-reproducible, one more pass over HBM) */
} bem_gpu_opts;

/* One boundary-value problem.  The DOF table is what the reference's setNodeFaceIndices()
 * produces (one DOF per (point, face-or-null) key); bem_gpu_build_dofs() derives it from
 * the face flags with the reference's rules. */
typedef struct {
  int32_t n_points;
  const double* X;               /* [3*n_points] */
  int32_t n_faces;
  const int32_t* tri;            /* [3*n_faces], outward orientation */
  const uint8_t* face_dirichlet; /* [n_faces] 1 = Dirichlet (free surface), 0 = Neumann */
  int32_t n_dof;
  const int32_t* dof_point;      /* [n_dof] */
  const int32_t* dof_face;       /* [n_dof] face id or -1 */
  const int32_t* dof_kind;       /* [n_dof] BEM_DOF_* */
  const int32_t* face_dof;       /* [3*n_faces] DOF used by each face vertex (pf2Index) */
} bem_bvp_desc;

typedef struct {
  int32_t iterations;     /* GMRES iterations (Arnoldi steps) */
  int32_t converged;      /* 1 if the true residual reached tol */
  double residual;        /* last true residual |A x - b| (scaled system) */
  double residual_est;    /* last Givens estimate */
  double time_setup_s;    /* wall time of setup (tree, lists, near weights, diagonal) */
  double time_solve_s;    /* wall time of the GMRES solve */
  int64_t nnz_near;       /* cached near-field weights */
  int64_t m2l_pairs;      /* box pairs in the M2L lists */
  int32_t n_nodes;        /* non-empty octree nodes */
  int32_t n_leaves;
  int32_t matvecs;        /* FP64 operator applications in this solve */
  int32_t matvecs_lo;     /* tensor-core (mixed precision) operator applications */
  double time_device_s;   /* CUDA-event time of the device work of setup + solve */
  int64_t h2d_bytes;      /* host->device bytes of setup + solve */
  int64_t d2h_bytes;      /* device->host bytes of setup + solve */
  int64_t kernel_launches;/* kernels launched by setup + solve (graph nodes counted) */
  double time_plan_s;     /* host part of the set-up: tree, lists, near-field sparsity */
  double time_upload_s;   /* host->device copies of the set-up */
  double time_setup_device_s; /* device part of the set-up (near weights, tables, diagonal) */
  double rhs_norm;        /* |b| of the scaled system (the reference's right-hand side -(A 0 - b)) */
  double tol_abs;         /* absolute tolerance the solve stopped at (tol, or tol*|b| with tol_relative) */
} bem_gpu_stats;

/* 1 if a CUDA device of compute capability 10.x is visible. */
int bem_gpu_is_available(void);

/* Default options: p=10, theta=0.25, 30 elements per leaf, 7 levels, tol 1e-9, 500 iterations. */
void bem_gpu_default_opts(bem_gpu_opts* opts);

/* Create a solver context on opts->device; NULL on failure. */
bem_gpu_ctx* bem_gpu_create(const bem_gpu_opts* opts);
void bem_gpu_destroy(bem_gpu_ctx* ctx);
const char* bem_gpu_last_error(const bem_gpu_ctx* ctx);

/* DOF table from face flags (setNodeFaceIndices + setIsMultipleNode,
 * bem/BEM_setBoundaryTypes.hpp:134-254, 434-441, 555-562).  Output arrays hold up to
 * n_points + 3*n_faces entries (face_dof: 3*n_faces; point_flags: n_points, bits
 * 1=Neumann 2=Dirichlet 4=CORNER 8=multiple node, may be NULL).  Returns n_dof (>= 0) or
 * a negative status.  Host-only; needs no GPU. */
int bem_gpu_build_dofs(int32_t n_points, const double* X, int32_t n_faces, const int32_t* tri, const uint8_t* face_dirichlet,
                       int32_t* dof_point, int32_t* dof_face, int32_t* dof_kind, int32_t* face_dof, uint8_t* point_flags);

/* Geometry set-up for one BVP: scaling, element sources, octree, interaction lists,
 * L2P targets, near-field weights and the rigid-mode diagonal.  Replaces the part of
 * solveGMRES() before solveSystemGMRES (BEM_solveBVP_GMRES_FMM.hpp:3056-3447). */
int bem_gpu_setup(bem_gpu_ctx* ctx, const bem_bvp_desc* desc);

/* Set-up at new coordinates of the mesh of the last set-up (a Runge-Kutta stage or time step:
 * same faces, boundary types and DOF tables, moved points), as the reference's solveGMRES does
 * when the topology is unchanged (bem/BEM_solveBVP_GMRES_FMM.hpp:3125-3346): the octree is
 * regrown in the root bucket of the previous set-up (a fresh root only if an element centroid
 * left it), lists, sources, near-field weights and the rigid-mode diagonal are recomputed.
 * What came out unchanged stays on the device: returns 2 (tree, lists and L2P targets kept:
 * only the geometry is uploaded; near-field weights, P2M operator and diagonal recomputed),
 * 1 (tree and lists kept, near-field blocks rebuilt), 0 (full set-up; also without a previous
 * set-up or for another mesh) or a negative error code.  Either way the operator is the one a
 * full set-up builds in that root bucket, bit for bit. */
int bem_gpu_setup_refresh(bem_gpu_ctx* ctx, const bem_bvp_desc* desc);

/* Solve with known boundary values (physical units; phi for Dirichlet DOFs, phin for
 * Neumann and corner-Neumann DOFs).  x0: initial guess of the unknowns in the same units
 * (phin for Dirichlet DOFs, phi for the others), e.g. the previous stage's solution as the
 * reference starts from the current boundary values (BEM_solveBVP_GMRES_FMM.hpp:3450-3454);
 * NULL for a zero initial guess.  out_phi and
 * out_phin get every DOF's phi and phin (known values copied through).  Replaces
 * solveSystemGMRES + the unscaling in solveGMRES (BEM_solveBVP_GMRES_FMM.hpp:2007-2649,
 * 3462-3486).  Returns BEM_OK, or BEM_ERR_NOT_CONVERGED with the outputs still written. */
int bem_gpu_solve(bem_gpu_ctx* ctx, const double* known, const double* x0, double* out_phi, double* out_phin, bem_gpu_stats* stats);

/* setup + solve. */
int bem_gpu_solve_bvp(bem_gpu_ctx* ctx, const bem_bvp_desc* desc, const double* known, const double* x0, double* out_phi,
                      double* out_phin, bem_gpu_stats* stats);

/* Operator rows for per-DOF phi/phin in scaled units (compute_Ax_minus_b,
 * BEM_solveBVP_GMRES_FMM.hpp:34-158): Av[i] = GPhin - (GnPhi + diag_i phi_i), or phi_i on
 * corner-Neumann rows. */
int bem_gpu_apply(bem_gpu_ctx* ctx, const double* phi, const double* phin, double* Av);

/* Near + far integrals per point, GPhin = int G phin, GnPhi = int dG/dn phi
 * (target4FMM::integrateNearField + integrateFarField, lib_multipole_expansion.hpp:1143-1150,
 * 1273-1302).  Arrays of n_points. */
int bem_gpu_point_integrals(bem_gpu_ctx* ctx, const double* phi, const double* phin, double* GPhin, double* GnPhi);

/* Unknown-space mat-vec on device buffers: y = A x (x, y: n_dof doubles on the device),
 * on the context's stream (return_A_dot_v, BEM_solveBVP_GMRES_FMM.hpp:2124-2155). */
int bem_gpu_matvec_device(bem_gpu_ctx* ctx, const double* d_x, double* d_y);

/* Same mat-vec as bem_gpu_matvec_device, but the call allocates nothing: the M2L pair
 * slots live in a 32 MiB area that is part of the library's device image (one per device,
 * reserved when the module loads).  For callers that must not allocate device memory while
 * applying the operator.  Limit: m2l_pairs * 2 * (p+1)(p+2)/2 * 16 bytes <= 32 MiB, else
 * BEM_ERR_UNSUPPORTED with the sizes in bem_gpu_last_error.  It always applies the FP64
 * operator, also on a mixed-precision context (opts.precision = 1).  The area's device address
 * is looked up once per context, during its first bem_gpu_setup with its device current (no
 * allocation), so the call itself does no lookup; it restores the caller's current device
 * before returning.  Calls that overlap on one device race on the shared area and must be
 * ordered by the caller.  No
 * counterpart in the reference (its operator allocates per call,
 * BEM_solveBVP_GMRES_FMM.hpp:2124-2155). */
int bem_gpu_matvec_device_noalloc(bem_gpu_ctx* ctx, const double* d_x, double* d_y);

/* Device bytes a context's buffers hold now (they keep their size across set-ups), and an
 * estimate of a BVP's device bytes from its sizes alone (no GPU needed), for admission control.
 * No counterpart in the reference. */
int64_t bem_gpu_device_bytes(const bem_gpu_ctx* ctx);
int64_t bem_gpu_estimate_bytes(const bem_gpu_opts* opts, const bem_bvp_desc* desc);

/* Introspection for parity tests. */
int bem_gpu_get_diag(bem_gpu_ctx* ctx, double* diag);                 /* [n_dof] */
double bem_gpu_scale_factor(const bem_gpu_ctx* ctx);                  /* L */
int bem_gpu_near_row(bem_gpu_ctx* ctx, int32_t point, int32_t cap, int32_t* dof, double* wG, double* wGn);
int bem_gpu_face_leaf(bem_gpu_ctx* ctx, int32_t* level, double* corner); /* [n_faces], [3*n_faces] */
int bem_gpu_tree_stats(bem_gpu_ctx* ctx, int64_t* out /*[10]: nodes, leaves, depth, added, m2l pairs, near pairs, nnz, near blocks, M2L chunks, M2L translation groups*/);
/* Near-field block sizes of the A.x kernel: out[6] = stored FP64 weights (sum over blocks of
 * targets x DOF columns), FP32 weights (rows padded to 4 columns), DOF columns gathered (sum
 * over blocks), blocks, targets, DOFs. */
int bem_gpu_near_stats(bem_gpu_ctx* ctx, int64_t* out /*[6]*/);

/* Host-only inspection of the set-up plan (no GPU needed): builds the octree, lists and
 * near-field sparsity for desc with opts and reports, per face, the level and lower corner
 * of the leaf bucket holding it (-1 if none), plus stats[10] as bem_gpu_tree_stats. */
int bem_plan_inspect(const bem_gpu_opts* opts, const bem_bvp_desc* desc, int32_t* face_level, double* face_corner, int64_t* stats);
/* Host check of the refresh path (no device needed): plans desc0, then desc1 as a refresh of
 * it, once taking over the unchanged structure and once rebuilding it in the same root.
 * out[0] = 1 if the root bucket was kept, out[1] = the structure taken over (as the return
 * value of bem_gpu_setup_refresh), out[2] = number of plan arrays in which the two desc1 plans
 * differ (0 expected). */
int bem_plan_refresh_inspect(const bem_gpu_opts* opts, const bem_bvp_desc* desc0, const bem_bvp_desc* desc1, int64_t* out);

/* The octree grown on the device against the host's growth of the same BVP (both bit-exact
 * restatements of the reference's Buckets::generateTree and list traversal): out[0] = 1 if the
 * device grew the tree, + 2 if it built the interaction lists,
 * out[1] = number of plan arrays that differ (0 expected), out[2] = buckets, out[3] = elements
 * a child refused (the reference's InsideQ edge case).  Needs a device. */
int bem_gpu_tree_check(const bem_gpu_opts* opts, const bem_bvp_desc* desc, int64_t* out);

/* Mat-vec stage timing with CUDA events on the context stream, averaged over repeats:
 * stage_ms = [p2m, m2m, m2l, l2l, near+l2p+rows, whole graph-launched mat-vec]. */
int bem_gpu_profile_matvec(bem_gpu_ctx* ctx, int repeats, double* stage_ms /*[6]*/);

/* Batch / asynchronous solving (the reference solves one BVP per call; BEM_BVP::solve(),
 * bem/BEM_solveBVP.hpp:565-630).  A batch owns n_workers contexts (one CUDA stream and one
 * host thread each) created with *opts; submitted problems queue FIFO and the next free
 * worker runs bem_gpu_solve_bvp on it, so one problem's host set-up overlaps another's GPU
 * work and the GPU work of different workers overlaps on the device.  The caller keeps every
 * array of the submitted problem (desc arrays, known, outputs, stats) alive and untouched
 * until its ticket polls done.  bem_gpu_batch_poll returns the solve's status (as
 * bem_gpu_solve_bvp), or BEM_ERR_NOT_READY while it is pending and wait == 0; a finished
 * ticket keeps its status (poll it any number of times) until bem_gpu_batch_release drops it.
 * bem_gpu_batch_last_error gives the message of the calling thread's last poll (messages are
 * per thread, so pollers on different threads do not see each other's). */
typedef struct bem_gpu_batch bem_gpu_batch;
bem_gpu_batch* bem_gpu_batch_create(const bem_gpu_opts* opts, int32_t n_workers);
int bem_gpu_batch_submit(bem_gpu_batch* batch, const bem_bvp_desc* desc, const double* known, double* out_phi, double* out_phin,
                         bem_gpu_stats* stats, int64_t* ticket);
int bem_gpu_batch_poll(bem_gpu_batch* batch, int64_t ticket, int32_t wait);
int bem_gpu_batch_release(bem_gpu_batch* batch, int64_t ticket);   /* forget a finished ticket; NOT_READY if unknown or pending */
/* Admission by device memory: the queue's head request starts only while the bytes the worker
 * contexts hold (each replaced, for the worker taking the request, by the larger of its own and
 * the request's bem_gpu_estimate_bytes) stay within `bytes`; an idle worker whose buffers keep
 * the head out gives them back.  A request above the budget alone ends with
 * BEM_ERR_OUT_OF_MEMORY.  0 = no limit (the default). */
int bem_gpu_batch_set_budget(bem_gpu_batch* batch, int64_t bytes);
/* A whole Runge-Kutta time-stepping chain of a BEM-MEL simulation as one request: n_steps steps
 * of 4 stages, each a set-up at the stage positions (bem_gpu_setup first, then
 * bem_gpu_setup_refresh), a solve warm-started from the previous stage's solution, and the MEL
 * stage update (bem_gpu_mel_stage, dt, gravity) whose positions and point phi give the next
 * stage's geometry and Dirichlet values (bem/main_time_domain.cpp:1071-2600); Neumann values stay
 * as given.  point_flags as bem_gpu_build_dofs.  Outputs the positions [3*n_points] and point phi
 * [n_points] at the end; stats sums the chain's solves (iterations, times, operator
 * applications; converged = every solve converged). */
int bem_gpu_batch_submit_chain(bem_gpu_batch* batch, const bem_bvp_desc* desc, const uint8_t* point_flags, const double* known,
                               int32_t n_steps, double dt, double gravity, double* out_X, double* out_phi_point,
                               bem_gpu_stats* stats, int64_t* ticket);
/* out[6]: requests admitted, admissions that had to wait for device memory, worker contexts
 * recreated to give memory back, device bytes held (or reserved) by the workers now, the
 * budget, requests queued. */
int bem_gpu_batch_stats(bem_gpu_batch* batch, int64_t* out);
const char* bem_gpu_batch_last_error(const bem_gpu_batch* batch);  /* message of this thread's last polled failure */
void bem_gpu_batch_destroy(bem_gpu_batch* batch);                  /* finishes queued problems first */

/* Mixed-Eulerian-Lagrangian stage update (the step that follows each BVP solve of a BEM-MEL
 * time step; set_u_potential_BEM, DphiDt_damped, pushPhi, pushPosition:
 * bem/BEM_calculateVelocities.hpp:1027-1044, lib/include/Network.hpp:224-235,
 * bem/main_time_domain.cpp:2410-2510).  Physical units.  The surface is the BVP's mesh with its
 * DOF table and solution: phi / phin per DOF as bem_gpu_solve returns them, face_dof as
 * bem_gpu_build_dofs, point_flags bits 1 all-Neumann, 2 all-Dirichlet, 4 CORNER. */
typedef struct {
  int32_t n_points;
  const double* X; /* [n_points*3] current positions */
  int32_t n_faces;
  const int32_t* tri;            /* [n_faces*3] */
  const uint8_t* face_dirichlet; /* [n_faces] */
  const uint8_t* point_flags;    /* [n_points] */
  int32_t n_dof;
  const int32_t* face_dof; /* [n_faces*3] DOF of each face vertex */
  const double* phi;       /* [n_dof] */
  const double* phin;      /* [n_dof] */
} bem_mel_surface;
typedef struct bem_gpu_mel bem_gpu_mel;
bem_gpu_mel* bem_gpu_mel_create(int32_t device);
void bem_gpu_mel_destroy(bem_gpu_mel* mel);
const char* bem_gpu_mel_last_error(const bem_gpu_mel* mel);
/* phi per point (storePhiPhin: all-Neumann points average their face DOFs by area,
 * bem/BEM_setBoundaryTypes.hpp:967-983) and velocity u = grad phi per point (gradPhi(p),
 * bem/BEM_BoundaryValues.hpp:500-563: per adjacent face the surface gradient of the linear
 * interpolant plus phin times the normal, fitted by area-weighted least squares as
 * optimalVector does, lib/include/rootFinding.hpp:119-205).  out_phi_point may be NULL. */
int bem_gpu_mel_velocity(bem_gpu_mel* mel, const bem_mel_surface* s, double* out_phi_point, double* out_u);
/* RK4 stage `stage` (0..3) of step dt: u as above, Dphi/Dt = -|u|^2/2 - gravity z + u_node.u
 * - gamma (phi - phi_ref) on points that are not all-Neumann (u_node [n_points*3] defaults to u
 * when NULL, damping [n_points*2] = (gamma, phi_ref) to 0 when NULL), then phi (those points) and
 * X (all points) advance as RungeKuttaCommon::push with steps = 4
 * (lib/include/integrationOfODE.hpp:227-300).  rk_* is the caller's RK state, in and out: stage
 * 0 sets rk_X0 / rk_phi0 from the current state, rk_acc* hold the weighted sums of f dt.
 * out_u and out_dphidt may be NULL. */
int bem_gpu_mel_stage(bem_gpu_mel* mel, const bem_mel_surface* s, int32_t stage, double dt, double gravity, const double* u_node,
                      const double* damping, double* rk_X0, double* rk_phi0, double* rk_accX, double* rk_accphi, double* out_X,
                      double* out_phi, double* out_u, double* out_dphidt);
/* Known values of the phi_t boundary-value problem that a floating-body step solves with the
 * same operator (setPhiPhin_t, bem/BEM_setBoundaryTypes.hpp:858-935), per DOF of the table
 * (dof_point / dof_face / dof_kind as bem_gpu_build_dofs):
 *   Dirichlet DOF: phi_t = -|u|^2/2 - gravity z (aphiat(0), lib/include/Network.hpp:971-976);
 *   Neumann DOF on face F: phin_t = 0 on a face of no body (face_body[F] = -1), else, for the
 *     rigid body b = face_body[F] with bodies[15 b ..] = centre (3), velocity (3), angular
 *     velocity (3), acceleration (3), angular acceleration (3) (RigidBodyDynamics.hpp:84-89),
 *     phint_Neumann(p, F) (bem/BEM_BoundaryValues.hpp:701-728): n.a + (Omega x n).(v - u)
 *     - (B v).H0 with the body's velocity v and acceleration a at the point, the face basis
 *     B = {n, s0, s1} (OrthogonalBasis, :307-315) and H0 the first row of HessianOfPhi (:653-672);
 *   Neumann point DOF (dof_face -1): the area-weighted mean over the point's Neumann faces
 *     (phint_Neumann(p), :751-779).
 * u: point velocities [3 n_points], NULL to compute them from the surface's solution as
 * bem_gpu_mel_velocity does.  Physical units; out_known [n_dof] is the `known` argument of the
 * phi_t solve (bem_gpu_solve on the same set-up): its result is phin_t on Dirichlet DOFs and
 * phi_t on the others. */
int bem_gpu_mel_phit_known(bem_gpu_mel* mel, const bem_mel_surface* s, const int32_t* dof_point, const int32_t* dof_face,
                           const int32_t* dof_kind, const int32_t* face_body, int32_t n_bodies, const double* bodies, double gravity,
                           const double* u, double* out_known);

/* Mixed precision (context set up with opts.precision = 1).  No reference counterpart: the
 * reference's M2L is FP64 only (lib/include/moments.hpp:732-764).
 * bem_gpu_matvec_device_mixed: y = A_lo x on device buffers (tensor-core M2L, everything
 *   else FP64), on the context's stream — the correction operator of the mixed solve.
 * bem_gpu_profile_matvec_mixed: stage times of that operator, the layout above followed by
 *   the three kernels of its M2L alone: [6] expand, [7] tensor-core contraction, [8] reduce,
 *   and [9] the near-field sums alone (the FP32 near-weight stream of stage [4], no rows).
 * bem_gpu_check_device_status: BEM_ERR_DEVICE if a bounded device-side wait of the
 *   tensor-core M2L gave up since set-up (the results of that launch are invalid). */
int bem_gpu_matvec_device_mixed(bem_gpu_ctx* ctx, const double* d_x, double* d_y);
int bem_gpu_profile_matvec_mixed(bem_gpu_ctx* ctx, int repeats, double* stage_ms /*[10]*/);
int bem_gpu_check_device_status(bem_gpu_ctx* ctx);
/* Iteration limit of the tensor-core M2L's device-side pipeline waits (a kernel argument;
 * default 2^22 tries, a fraction of a second).  For testing failure detection: with a small
 * limit the waits give up, the kernel drains its own copies and MMAs in flight (with the
 * default limit), records the failure and returns, so bem_gpu_check_device_status reports
 * BEM_ERR_DEVICE while the context stays usable.  tries < 0 restores the default; the call
 * clears the recorded failure and recaptures the operator graphs. */
int bem_gpu_set_wait_limit(bem_gpu_ctx* ctx, int64_t tries);

/* Near-field polynomial preconditioner (opts.preconditioner = 2).
 * bem_gpu_poly_roots: the roots formed by the last set-up, in the order they are applied (a
 *   conjugate pair a +- bi is one entry with im = b > 0); returns the number of entries, 0 when
 *   none could be formed (the solve then uses the Jacobi scaling alone), or an error code.
 * bem_harmonic_ritz_values: host helper -- harmonic Ritz values of a (k+1) x k Arnoldi
 *   Hessenberg matrix (row-major, leading dimension ldh, k <= 32); 0 or -1. */
int bem_gpu_poly_roots(bem_gpu_ctx* ctx, int32_t cap, double* re, double* im);

/* Tensor-core M2L work-item size of a mixed context: *pairs_in_use, and the 4 candidates with
 * their contraction-kernel times (ms; zeros if never tuned in this process).  Returns 1 if the
 * last set-up ran the tuning, 0 if it used a cached or forced size. */
int bem_gpu_tc_tuning(bem_gpu_ctx* ctx, int32_t* pairs_in_use, int32_t* candidates /*[4]*/, double* ms /*[4]*/);

/* Set-up time by part (seconds) of the last set-up: [0] element sources, [1] octree, [2] lists,
 * [3] element order and node arrays, [4] M2L grouping, [5] near-field blocks, [6] DOF incidence
 * (host plan), [7] uploads, [8] device set-up; [9] = 1 if the octree was grown on the device
 * + 2 if the lists were built there; [10..15] the host time of the uploads by step: node and
 * level arrays, near blocks and element/tree arrays, tensor-core work items, P2M operator
 * lists, remaining arrays (the copies are asynchronous; the device part follows them in
 * stream order); [15] the near-field quadrature's part of [8]. */
int bem_gpu_setup_phases(bem_gpu_ctx* ctx, double* out /*[16]*/);
int bem_harmonic_ritz_values(int32_t k, const double* H, int32_t ldh, double* re, double* im);

/* FP64 FMA throughput of the device (TFLOP/s), measured by a short probe kernel. */
double bem_gpu_fp64_peak_tflops(int32_t device);

#ifdef __cplusplus
}
#endif
#endif /* BEM_B200_H */
