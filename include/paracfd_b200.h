/*
 * paracfd_b200.h -- C ABI of the B200-native ParaCFD per-timestep solver path.
 *
 * The boundary sits exactly where the reference hands host topology to its device
 * classes: a caller builds (or imports) the static 2:1 brick hierarchy and the
 * composite cut-cell pressure system once, passes them here as flat arrays, and then
 * drives projection / cell-momentum / surface-load work that stays resident in HBM.
 *
 * Reference interfaces replaced (paths inside the ParaCFD project):
 *   pcfd_system_create            DeviceAmrFields + DeviceCompositeAmrProjection +
 *                                 DeviceCompositeCellMomentumTransport constructors
 *                                 (src/core/fluid/external_aero_core.cpp:220-228; the topology
 *                                 consumed is CompositeAmrPressureSystem, amr_pressure.h:193-260,
 *                                 and AmrHierarchy, amr_grid.h:86-118)
 *   pcfd_pressure_apply           DeviceCompositeAmrPressureOperator::apply / apply_orthogonal
 *                                 (src/core/fluid/amr_pressure.h:299-300)
 *   pcfd_pressure_diagonal        CompositeAmrPressureSystem::diagonal_cpu (amr_pressure.h:259)
 *   pcfd_pressure_precondition    DeviceCompositeAmrPressureSolver::apply_preconditioner
 *                                 (amr_pressure.h:405)
 *   pcfd_pressure_solve           DeviceCompositeAmrPressureSolver::solve (amr_pressure.h:363)
 *   pcfd_projection_divergence    DeviceCompositeAmrProjection::compute_divergence (amr_pressure.h:475)
 *   pcfd_projection_rhs           DeviceCompositeAmrProjection::build_projection_rhs (amr_pressure.h:476)
 *   pcfd_projection_correct       DeviceCompositeAmrProjection::correct_fluxes (amr_pressure.h:477)
 *   pcfd_projection_project       DeviceCompositeAmrProjection::project (amr_pressure.h:478)
 *   pcfd_set/get_* state          DeviceAmrFields::upload/download, upload/download_special_fluxes,
 *                                 upload_pressure, DeviceCompositeCellMomentumTransport::
 *                                 upload_state/download_state (amr_fields.h:57-58,
 *                                 amr_pressure.h:462-483, amr_advection.h:286-287)
 *
 * Conventions: every entry point returns a pcfd_status; on failure
 * pcfd_last_error_message() (thread-local) says why.  No exception crosses the ABI.
 * "_host" entry points take caller-owned host buffers and copy in/out (they synchronise);
 * "_device" entry points take device pointers on the system's stream.  Array sizes are
 * stated in the comments: S = storage_size (pressure DOF slots, covered bricks included),
 * B = total brick slots over all levels (S = B * bs^3), F = B * (bs+1) * bs^2 faces per
 * component.  A system object is used by one host thread at a time.
 */
#ifndef PARACFD_B200_H
#define PARACFD_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pcfd_status {
    PCFD_OK = 0,
    PCFD_INVALID_ARG = 1,
    PCFD_CUDA_ERROR = 2,
    PCFD_NOT_CONVERGED = 3,
    PCFD_TOPOLOGY_UNRESOLVED = 4,
    PCFD_OUT_OF_MEMORY = 5,
    PCFD_TIMEOUT = 6,
    PCFD_INTERNAL = 7
} pcfd_status;

/* Brick flags, bit-identical to BrickFlags (amr_grid.h:27-32). */
enum {
    PCFD_BRICK_XMIN = 1u << 0, PCFD_BRICK_XMAX = 1u << 1, PCFD_BRICK_YMIN = 1u << 2,
    PCFD_BRICK_YMAX = 1u << 3, PCFD_BRICK_ZMIN = 1u << 4, PCFD_BRICK_ZMAX = 1u << 5,
    PCFD_BRICK_EMBEDDED_BOUNDARY = 1u << 6, PCFD_BRICK_COVERED = 1u << 7
};

/* One AMR level (AmrLevel + BrickMetadata, amr_grid.h:34-64). */
typedef struct pcfd_level {
    double h;                    /* cell size of this level */
    int32_t brick_count;         /* bricks stored on this level, covered ones included */
    int32_t level_offset;        /* first pressure DOF of this level (= brick slot * bs^3) */
    const int32_t* coord;        /* [brick_count][3] integer brick coordinates */
    const double* origin;        /* [brick_count][3] world origin of the brick */
    const int32_t* neighbors;    /* [brick_count][6] same-level neighbour (-x,+x,-y,+y,-z,+z), -1 none */
    const uint32_t* flags;       /* [brick_count] PCFD_BRICK_* */
    const int32_t* children;     /* [brick_count][8] fine children or -1; may be NULL on the finest level */
} pcfd_level;

/* Compact pressure connections: CoarseFinePressureConnection (amr_pressure.h:101-121), SoA. */
typedef struct pcfd_connections {
    int32_t count;
    const int32_t* coarse_dof;
    const int32_t* fine_dof;
    const double* open_area;
    const double* centre_distance;
    const double* normal_distance;
    const int8_t* axis;
    const int8_t* direction;            /* +1: coarse_dof is the lower-axis side */
    const double* face_centroid;        /* [count][3] */
    const double* orthogonal_gradient_factor;
    const int32_t* lower_gradient_node;
    const int32_t* upper_gradient_node;
    const double* nonorthogonal_correction; /* [count][3] */
    const double* upper_gradient_weight;
} pcfd_connections;

/* RegularPressureCorrection (amr_pressure.h:141-155), SoA. */
typedef struct pcfd_regular_corrections {
    int32_t count;
    const int32_t* lower_dof;
    const int32_t* upper_dof;
    const int32_t* level;
    const int32_t* brick;
    const int32_t* ijk;                 /* [count][3] positive-face index in the owning brick */
    const int8_t* axis;
    const double* open_area;
    const double* two_point_delta;
    const int32_t* lower_gradient_node;
    const int32_t* upper_gradient_node;
    const double* nonorthogonal_correction; /* [count][3] */
    const double* upper_gradient_weight;
} pcfd_regular_corrections;

/* CompositeSurfacePressurePatch (amr_pressure.h:156-165), SoA. */
typedef struct pcfd_surface_patches {
    int32_t count;
    const double* area;
    const double* centroid;             /* [count][3] */
    const double* normal;               /* [count][3], minus -> plus */
    const int32_t* plus_dof;
    const int32_t* minus_dof;
} pcfd_surface_patches;

/* CompositeBoundaryPressureFace (amr_pressure.h:166-170), SoA. */
typedef struct pcfd_boundary_faces {
    int32_t count;
    const int32_t* dof;
    const double* outward_area;         /* [count][3] */
    const double* centroid;             /* [count][3] */
} pcfd_boundary_faces;

/* Complete static topology: AmrHierarchy + CompositeAmrPressureSystem. */
typedef struct pcfd_topology {
    int32_t brick_size;
    int32_t level_count;
    const pcfd_level* levels;
    double domain_lo[3], domain_hi[3];
    int32_t storage_size;
    int32_t pressure_outlet_xmax;
    const uint8_t* active;                  /* [S] */
    const uint8_t* freestream_connected;    /* [S] may be NULL (treated as active) */
    const uint8_t* cut_face_mask;           /* [S] +X/+Y/+Z suppression bits */
    const double* volume;                   /* [S] */
    const double* centroid;                 /* [S][3] */
    const int32_t* preconditioner_aggregate;/* [S] level-0 aggregate DOF or -1 */
    pcfd_connections coarse_fine;
    pcfd_connections embedded;
    pcfd_regular_corrections regular;
    int32_t gradient_node_count;            /* compact WLS pressure-gradient stencil */
    const int32_t* gradient_dof;            /* [nodes] */
    const int32_t* gradient_offset;         /* [nodes+1] */
    const int32_t* gradient_neighbour;      /* [nnz] */
    const double* gradient_weight;          /* [nnz][3] */
    int32_t gauge_count;
    const int32_t* gauge_dof;
    const double* gauge_coefficient;
    pcfd_surface_patches patches;
    pcfd_boundary_faces boundary_faces;
    int32_t retained_count;                 /* face_state_retained_dofs */
    const int32_t* retained_dofs;
} pcfd_topology;

/* Precision of the multigrid preconditioner inside the FP64 outer Krylov solve. */
typedef enum pcfd_mg_precision {
    PCFD_MG_FP64 = 0,   /* reference-equivalent arithmetic (parity mode) */
    PCFD_MG_FP32 = 1    /* FP32 smoother/coarse levels, FP64 outer recurrence */
} pcfd_mg_precision;

typedef struct pcfd_options {
    int32_t mg_precision;            /* pcfd_mg_precision */
    int32_t device;                  /* CUDA device ordinal */
    void* stream;                    /* cudaStream_t or NULL for a library-owned stream */
    double momentum_min_volume_fraction; /* AmrConfig::min_volume_fraction (small-cell groups) */
    int32_t disable_fused_smoother;  /* 1: run the preconditioner's fine level as separate
                                        operator/vector launches (same sweeps, reference order) */
    int32_t mg_cycle;                /* pcfd_mg_cycle */
    int32_t gmres_restart;           /* columns per GCRO/LGMRES cycle, 1..24; 0: the reference's 24 */
    int32_t mg_stage_sweeps;         /* composite cycle: smoothing steps before and after each stage's
                                        coarse correction, 1..16; 0: 6 */
    int32_t mg_block_iterations;     /* composite cycle: 0 = the reference's two Jacobi pre-sweeps on
                                        the fine level; k = 1..64: instead, k Chebyshev iterations of
                                        each brick's own diagonal block solve in shared memory */
    int32_t mg_stage_chebyshev;      /* composite stages: r = 2..1000: Chebyshev polynomial smoothing of
                                        D^-1 A on [2 / r, 2]; 1 = damped Jacobi (w = 2/3); 0: r = 30 */
    int32_t mg_fine_chebyshev;       /* composite cycle's fine sweeps: r = 2..1000: the two pre- and two
                                        post-sweeps take the Chebyshev-Richardson step sizes of
                                        [2 / r, 2]; 1 = damped Jacobi (w = 2/3); 0: r = 10 */
    int32_t gmres_delayed;           /* 1: GCRO/LGMRES columns orthogonalised by delayed CGS2 (one dot
                                        and one update pass over the basis per column; the previous
                                        basis vector reorthogonalised in the same passes); 0: CGS2
                                        (three passes) */
    int32_t gmres_recycle;           /* recycled (U, C = A U) pairs kept between solves: 1..3; -1: none;
                                        0: the reference's 3 */
    int32_t mg_stage_fp16;           /* 1: with the composite cycle and the FP32 multigrid, the stage
                                        matrices (all but the coarsest) store their off-diagonal
                                        coefficients in FP16; vectors, diagonals and sums stay FP32 or
                                        wider.  0: FP32 */
    int32_t mg_stage_csr;            /* 1: keep the composite cycle's first stage as CSR rows; 0: with 8^3
                                        bricks, its brick-structured form (64 rows per brick, face
                                        neighbours found from the row index, the same couplings) */
} pcfd_options;

/* Coarse-correction weighting of the multigrid cycle.  The aggregation coarse operators are
 * Galerkin products with piecewise-constant transfer, which over-weight the coarse problem (by 2
 * per 2x2x2 coarsening of a uniform Laplacian, 8^l for the reference's direct aggregation of a
 * level-l cell into its level-0 cell); the corrected cycle scales the prolonged corrections by 2
 * (fine <- level-0 aggregates) and 1.5 (between lattice levels).  Same smoother, transfers and
 * coarse matrices.  On the 2- and 3-level wing grids (1-5 M cells) it cuts the cold-start
 * iterations to 1e-8 by 25-40 %; on the 4-level 16 M-cell grid it does not help, so the
 * reference cycle stays the default. */
typedef enum pcfd_mg_cycle {
    PCFD_MG_CYCLE_REFERENCE = 0,     /* the reference's cycle (amr_pressure.cu:1103-1154) */
    PCFD_MG_CYCLE_CORRECTED = 1,     /* over-corrected prolongation */
    PCFD_MG_CYCLE_COMPOSITE = 2      /* composite-grid stages instead of the level-0 lattice: stage k
                                        holds one cell per 2^k-wide block of same-level cells of every
                                        AMR level (Galerkin operators, prolongations weighted 2,
                                        mg_stage_sweeps Chebyshev steps per stage, an explicit inverse
                                        on the last stage of at most 512 cells): 3.8x fewer iterations
                                        than the reference cycle on the 4-level 16 M-cell wing grid.
                                        Needs 8^3 bricks and the fused fine level; with the FP32
                                        multigrid the stages and the fine sweeps are float, the Krylov
                                        vectors and the operator stay FP64. */
} pcfd_mg_cycle;

/* AmrGpuSolveResult (amr_pressure.h:337-351), trimmed to what the solver reports. */
typedef struct pcfd_solve_result {
    int32_t iterations;
    double relative_residual;
    int32_t converged;
    int32_t preconditioner_applications;
    int32_t recycle_rejections;
    int32_t fallback_solves;     /* no reference counterpart: 1 when a solve under the learned
                                    preconditioner did not converge and the multigrid solve from its
                                    last iterate finished it (iterations count both) */
} pcfd_solve_result;

/* Physical case and solver settings used by the time step (ParagliderConfig's freestream and
 * solver blocks, src/core/paraglider_config.h:10-58, and ExternalAeroExecutionOptions,
 * src/core/fluid/external_aero_core.h:106-120). */
typedef struct pcfd_case {
    double speed;                    /* freestream speed along +X [m/s] */
    double rho;                      /* density [kg/m^3] */
    double nu;                       /* kinematic viscosity [m^2/s] */
    double cfl;
    double smagorinsky_cs;
    double projection_tolerance;     /* relative residual of the pressure solve */
    int32_t projection_max_iterations;
    int32_t smooth_wall;             /* apply the Spalding smooth-wall model */
    int32_t pressure_impulse;        /* apply the projected pressure traction to cell momentum */
} pcfd_case;

/* ExternalAeroStepStats (external_aero_core.h:61-83), device-timed. */
typedef struct pcfd_step_stats {
    double dt;
    double physical_time;
    double max_abs_velocity;         /* max |cell velocity component| before the step */
    double max_abs_special_velocity; /* max |2:1 tile or EB aperture velocity| before the step */
    double max_outflow_rate;         /* conservative CFL rate [1/s] */
    double cfl_velocity;
    double effective_cfl;
    double max_diffusion_rate;
    int32_t diffusion_substeps;
    pcfd_solve_result pressure;
    double step_ms;                  /* CUDA-event time of the whole step on the system stream */
    double projection_ms;
} pcfd_step_stats;

typedef struct pcfd_system pcfd_system;

const char* pcfd_last_error_message(void);
const char* pcfd_version(void);

/* ---- preprocessing: closed wing surface -> brick hierarchy + composite system ------------
 * Replaces AmrHierarchy::build_static (amr_grid.cpp:222-261) and the composite pressure
 * builder (build_composite_amr_pressure_system, amr_pressure.cpp:247-301 with its finalisation
 * :24-189).  With solid != 0 the cells whose centres lie inside the closed, outward-oriented
 * surface become solid and every fluid/solid face a wall patch (a Cartesian stand-in for the
 * reference's polyhedral cut-cell atlas, build_amr_embedded_boundary_atlas, amr_eb.h:69-70). */
typedef struct pcfd_mesh {
    int64_t vertex_count;
    const double* positions;         /* [vertex_count][3] metres */
    int64_t triangle_count;
    const uint32_t* indices;         /* [triangle_count][3] */
} pcfd_mesh;

typedef struct pcfd_amr_config {     /* AmrConfig subset (paraglider_config.h:27-43) */
    double domain_lo[3], domain_hi[3];   /* requested flow domain (padded to whole bricks) */
    double base_cell_size;
    int32_t max_levels;
    int32_t brick_size;
    double wing_refinement_distance;
    double surface_refinement_distance;
    double wake_length;
    double wake_radius;
    int32_t anchor_y_min;            /* half-wing symmetry plane at Y-min */
} pcfd_amr_config;

typedef struct pcfd_built_topology pcfd_built_topology;
/* Fills *view with arrays owned by *out (valid until pcfd_topology_free). */
pcfd_status pcfd_topology_build(const pcfd_mesh* surface, const pcfd_amr_config* config, int32_t solid,
                                pcfd_built_topology** out, pcfd_topology* view);
void pcfd_topology_free(pcfd_built_topology* topology);
const char* pcfd_builder_last_error(void);

/* Topology upload + device allocation (all static arrays copied; caller may free inputs). */
pcfd_status pcfd_system_create(const pcfd_topology* topology, const pcfd_options* options,
                               pcfd_system** out);
void pcfd_system_destroy(pcfd_system* system);
/* Sizes: storage_size, brick slots, faces per component, coarse/fine and EB connection counts. */
pcfd_status pcfd_system_sizes(const pcfd_system* system, int64_t* storage_size, int64_t* bricks,
                              int64_t* faces_per_component, int64_t* coarse_fine_count,
                              int64_t* embedded_count);
pcfd_status pcfd_system_synchronize(pcfd_system* system);

/* ---- pressure operator (FP64) -------------------------------------------------------- */
/* out = A p (orthogonal != 0: two-point part only, as apply_orthogonal). p, out: [S]. */
pcfd_status pcfd_pressure_apply_host(pcfd_system* system, const double* p, double* out,
                                     int32_t orthogonal);
pcfd_status pcfd_pressure_apply_device(pcfd_system* system, const double* d_p, double* d_out,
                                       int32_t orthogonal);
/* No reference counterpart.  The same operator as pcfd_pressure_apply_device, but the call
 * allocates nothing: the WLS-gradient scratch is a static device array of at most 262,144
 * gradient nodes (6 MiB), shared by all systems on the device; systems with more nodes get
 * PCFD_INVALID_ARG for the full operator.  For callers that cannot allocate at call time
 * (device memory reserved by another pool, allocator-free loops).  The first full-operator
 * call through a system looks up the scratch address (no allocation) and should come before any
 * stream capture; calls overlapping in time race on the scratch. */
pcfd_status pcfd_pressure_apply_device_noalloc(pcfd_system* system, const double* d_p, double* d_out,
                                               int32_t orthogonal);
/* Jacobi diagonal used by the smoother (diagonal_cpu semantics). diag: [S]. */
pcfd_status pcfd_pressure_diagonal_host(pcfd_system* system, double* diag);
/* z = M^-1 r with the reference-structured V-cycle (FP64 or FP32 per options). [S]. */
pcfd_status pcfd_pressure_precondition_host(pcfd_system* system, const double* r, double* z);
/* Solve A x = b. warm_start != 0 keeps x as the initial guess. x, b: [S]. */
pcfd_status pcfd_pressure_solve_host(pcfd_system* system, double* x, const double* b,
                                     double tolerance, int32_t max_iterations, int32_t warm_start,
                                     pcfd_solve_result* result);

/* ---- resident flow state (FP32 fields, FP64 pressure) --------------------------------- */
/* Faces in brick-slot order, per brick (bs+1)*bs*bs for u ((k*bs+j)*(bs+1)+i), bs*(bs+1)*bs
 * for v ((k*(bs+1)+j)*bs+i), bs*bs*(bs+1) for w ((k*bs+j)*bs+i).  u, v, w: [F]. */
pcfd_status pcfd_set_faces_host(pcfd_system* system, const float* u, const float* v, const float* w);
pcfd_status pcfd_get_faces_host(pcfd_system* system, float* u, float* v, float* w);
/* Compact special velocities: coarse/fine tiles [count_cf], EB apertures [count_eb]. */
pcfd_status pcfd_set_special_host(pcfd_system* system, const float* coarse_fine, const float* embedded);
pcfd_status pcfd_get_special_host(pcfd_system* system, float* coarse_fine, float* embedded);
/* FP64 solve pressure [S]; the FP32 shadow is refreshed from it. */
pcfd_status pcfd_set_pressure_host(pcfd_system* system, const double* p);
pcfd_status pcfd_get_pressure_host(pcfd_system* system, double* p);
pcfd_status pcfd_get_pressure_shadow_host(pcfd_system* system, float* p32);

/* ---- projection ------------------------------------------------------------------------- */
/* divergence [S] (FP32) = integrated aperture flux / volume. */
pcfd_status pcfd_projection_divergence_host(pcfd_system* system, float* divergence);
/* rhs [S] (FP64) = -(rho/dt) * integrated aperture flux. */
pcfd_status pcfd_projection_rhs_host(pcfd_system* system, double rho, double dt, double* rhs);
/* Gradient correction of all face kinds from the resident FP64 pressure. */
pcfd_status pcfd_projection_correct(pcfd_system* system, double rho, double dt);
/* build rhs -> solve -> (if converged) shadow, correct, divergence. */
pcfd_status pcfd_projection_project(pcfd_system* system, double rho, double dt, double tolerance,
                                    int32_t max_iterations, int32_t warm_start,
                                    pcfd_solve_result* result);

/* No reference counterpart.  keep != 0: every projection saves its solver start (warm-start
 * pressure, recycled GCRO subspace) on the device; resolve solves the last projection's system
 * again from that start with the current preconditioner and returns its device time (CUDA
 * events on the system stream) -- the same right-hand side and start for every preconditioner
 * being compared. */
pcfd_status pcfd_projection_keep_start(pcfd_system* system, int32_t keep);

/* No reference counterpart.  Initial guess of the step projections, which the reference
 * warm-starts from the last pressure (mode 0, the default).  Mode 1 starts from the linear
 * extrapolation 2 p_n - p_(n-1) of the last two converged step pressures, mode 2 from the
 * quadratic 3 p_n - 3 p_(n-1) + p_(n-2) of the last three; with fewer converged pressures
 * (after initialization, pcfd_set_pressure_host or a projection that did not converge) the
 * highest order they allow.  The solve still ends at the same relative residual; only its start
 * moves. */
pcfd_status pcfd_core_set_initial_guess(pcfd_system* system, int32_t mode);
pcfd_status pcfd_projection_resolve(pcfd_system* system, double tolerance, int32_t max_iterations, double* ms,
                                    pcfd_solve_result* result);

/* ---- cell momentum (DeviceCompositeCellMomentumTransport, amr_advection.h:269-405) ---------- */
/* Collocated FP32 control-volume velocity [S] per component. */
pcfd_status pcfd_momentum_set_state_host(pcfd_system* system, const float* x, const float* y, const float* z);
pcfd_status pcfd_momentum_get_state_host(pcfd_system* system, float* x, float* y, float* z);
/* MUSCL/minmod conservative transport (step, amr_advection.h:292-293). */
pcfd_status pcfd_momentum_transport(pcfd_system* system, double dt, double freestream_speed, int32_t external_aero);
/* Smagorinsky viscosity + sub-cycled explicit diffusion (diffuse_smagorinsky, amr_advection.h:297). */
pcfd_status pcfd_momentum_smagorinsky(pcfd_system* system, double nu, double cs, double dt, double* rate,
                                      int32_t* substeps);
/* Implicit Spalding smooth wall (apply_smooth_fabric_wall_model, amr_advection.h:300). */
pcfd_status pcfd_momentum_smooth_wall(pcfd_system* system, double dt, double nu);
/* Per wall side (patch plus side, then minus side, in patch order) force/density [3*sides]. */
pcfd_status pcfd_momentum_wall_forces_host(pcfd_system* system, float* force_per_density, int64_t* sides);
/* Pressure traction of the resident FP32 pressure shadow (apply_projected_pressure_gradient,
 * amr_advection.h:304; physical_boundaries=0 gives apply_pressure_impulse(...,false)). */
pcfd_status pcfd_momentum_pressure_impulse(pcfd_system* system, double dt, double rho, int32_t physical_boundaries,
                                           int32_t redistribute);
/* Cell -> face normal velocities (reconstruct_fluxes, amr_advection.h:307). */
pcfd_status pcfd_momentum_reconstruct_fluxes(pcfd_system* system);
/* External aerodynamic face conditions (DeviceAmrFields::apply_external_aero_boundaries, amr_fields.h:63). */
pcfd_status pcfd_apply_external_boundaries(pcfd_system* system, double freestream_speed);
/* out[0] max |cell velocity|, out[1] max outflow rate [1/s], out[2] max |special velocity|. */
pcfd_status pcfd_momentum_cfl(pcfd_system* system, int32_t external_aero, double out[3]);

/* ---- time step (ExternalAeroCore, external_aero_core.h:124-182) ------------------------------ */
/* Sets the case.  A changed flow case (speed, rho, nu, cfl, Smagorinsky constant, wall or impulse
 * switch) needs pcfd_core_initialize again; a call that changes only the projection tolerance or
 * iteration budget keeps the initialized state and the physical time. */
pcfd_status pcfd_core_configure(pcfd_system* system, const pcfd_case* config);
/* Freestream state, reconstruction, first projection (ExternalAeroCore::initialize). */
pcfd_status pcfd_core_initialize(pcfd_system* system, pcfd_step_stats* stats);
/* One time step (ExternalAeroCore::step): CFL, transport, LES diffusion, wall, reconstruction,
 * boundaries, projection, pressure traction.  Time advances only when the solve converged. */
pcfd_status pcfd_core_step(pcfd_system* system, pcfd_step_stats* stats);
/* X-min inflow profile (generalises ExternalAeroCore's uniform u = speed on the XMIN faces,
 * external_aero_core.cpp:290 / amr_advection.cu external-boundary kernel).  The layout is one
 * normal velocity per boundary face: face (j, k) of the n-th non-covered brick carrying
 * PCFD_BRICK_XMIN (all levels, coarsest first, brick order) sits at n*bs*bs + k*bs + j.
 * pcfd_core_inflow_layout returns the face count and, if brick_slots is non-NULL, the global
 * brick slot of each of those bricks ([face_count / bs^2]).  set_inflow with count 0 (and any
 * pointer) returns to the uniform freestream; otherwise count must equal the face count. */
pcfd_status pcfd_core_inflow_layout(pcfd_system* system, int64_t* face_count, int32_t* brick_slots);
pcfd_status pcfd_core_set_inflow_host(pcfd_system* system, const float* normal_velocity, int64_t count);

/* Integrated surface loads (AerodynamicLoads, src/core/aero_loads.h:33-53). */
typedef struct pcfd_loads {
    double pressure_force[3], pressure_moment[3];
    double viscous_force[3], viscous_moment[3];
    double total_force[3], total_moment[3];
    double cl, cd, cs;               /* NaN unless reference_area > 0 and the case is configured */
} pcfd_loads;
/* compute_pressure_loads (+ accumulate_viscous_loads when include_viscous) of the resident
 * pressure shadow and wall forces (aero_loads.cpp:183-204); device FP64 sums, 12-double readback. */
pcfd_status pcfd_core_loads(pcfd_system* system, double pressure_reference, const double moment_origin[3],
                            double reference_area, int32_t include_viscous, pcfd_loads* out);

/* ExternalAeroConservationStats (external_aero_core.h:84-92). */
typedef struct pcfd_conservation_stats {
    double max_abs_divergence;             /* 1/s */
    double volume_weighted_rms_divergence; /* 1/s */
    double worst_control_volume;           /* m^3 at max_abs_divergence (first DOF on ties) */
    double max_integrated_flux_error;      /* m^3/s, one control volume */
    double absolute_integrated_flux_error; /* sum |divergence * volume|, m^3/s */
    double net_integrated_flux_error;      /* sum divergence * volume, m^3/s */
} pcfd_conservation_stats;
/* ExternalAeroCore::conservation_stats (external_aero_core.cpp:347-356) of the resident divergence
 * (left by the last projection, or by pcfd_projection_divergence_host): device FP64 reductions,
 * six doubles read back. */
pcfd_status pcfd_core_conservation_stats(pcfd_system* system, pcfd_conservation_stats* out);

/* ---- launch-shape autotuner ---------------------------------------------------------------- */
/* No reference counterpart.  Times each candidate persistent-grid size of the brick pipeline (the
 * fused fine-level multigrid and structured-operator kernels: 1 .. the occupancy limit, at most 8
 * resident CTAs per SM) on this system's bricks -- the FP64 structured operator plus one fine sweep,
 * CUDA events over `iterations` launches -- and keeps the fastest for the system's later launches. */
typedef struct pcfd_autotune_report {
    int32_t candidates;
    int32_t ctas_per_sm[8];
    double apply_ms[8];
    double sweep_ms[8];
    int32_t chosen;                  /* resident CTAs per SM now used */
} pcfd_autotune_report;
pcfd_status pcfd_autotune(pcfd_system* system, int32_t iterations, pcfd_autotune_report* report);
/* Sets the brick pipeline's resident CTAs per SM (1..8; launches never exceed what the kernels'
 * launch bounds keep resident).  No result depends on it. */
pcfd_status pcfd_set_pipeline_ctas(pcfd_system* system, int32_t ctas_per_sm);

/* ---- point location and headless slices ---------------------------------------------------- */
/* DeviceAmrLocator::locate_points (amr_fields.cu:131-168, 244-249): for each point of d_points
 * [count][3] (FP32, device) the finest non-covered brick containing it, d_locations [count][5] =
 * level, brick (index within its level), i, j, k (device); level = brick = -1 for a point outside
 * every brick.  Same FP32 arithmetic as the reference, so the same answer at brick and cell edges. */
pcfd_status pcfd_locate_points_device(pcfd_system* system, const float* d_points, int32_t count, int32_t* d_locations);
/* Headless slice of the resident state (in place of the reference GUI's OpenGL slice,
 * src/gui/slice_field.cu:147-261): nu x nv samples at origin + (a + 1/2)/nu edge_u + (b + 1/2)/nv
 * edge_v, point located as above, each the value of the finest active cell containing it (NaN
 * where none).  field: 0 |cell velocity|, 1/2/3 cell velocity x/y/z, 4 pressure (FP32 shadow).
 * out [nv][nu] (host). */
pcfd_status pcfd_sample_slice_host(pcfd_system* system, const double origin[3], const double edge_u[3],
                                   const double edge_v[3], int32_t nu, int32_t nv, int32_t field, float* out);

/* ---- staggered MAC momentum mode ---------------------------------------------------------- */
/* Momentum path of pcfd_core_initialize / pcfd_core_step (ExternalAeroExecutionOptions::
 * conservative_cell_momentum, external_aero_core.h:108-113). */
typedef enum pcfd_momentum_mode {
    PCFD_MOMENTUM_CELL = 0,   /* conservative cell momentum (the reference's default) */
    PCFD_MOMENTUM_MAC = 1     /* staggered MAC faces: needs pcfd_mac_set_links */
} pcfd_momentum_mode;
/* Selects the momentum path; the core needs pcfd_core_initialize again afterwards. */
pcfd_status pcfd_core_set_momentum_mode(pcfd_system* system, int32_t mode);
/* The reference's non-default momentum path, DeviceAmrAdvection (amr_advection.cu:1652-1690), on
 * the resident face velocities (pcfd_set_faces_host / pcfd_get_faces_host, compact per-brick
 * layout).  Link bytes per face [F] each (host), the caller's geometry preprocessing as in the
 * DeviceAmrAdvection constructor: bits 0..5 the open -x,+x,-y,+y,-z,+z same-side links, bit 6 the
 * near-fabric band; faces away from the fabric 0x3f. */
pcfd_status pcfd_mac_set_links(pcfd_system* system, const uint8_t* links_u, const uint8_t* links_v, const uint8_t* links_w);
/* DeviceAmrAdvection::advect (amr_advection.cu:1663-1671): MacCormack semi-Lagrangian advection of
 * every face of every level over dt (FP32, dt rounded to FP32), band faces by the limited MUSCL
 * update; faces of covered bricks become 0.  Needs the links. */
pcfd_status pcfd_mac_advect(pcfd_system* system, double dt);
/* DeviceAmrAdvection::diffuse_smagorinsky (amr_advection.cu:1683-1690): Smagorinsky eddy viscosity
 * per cell, then one explicit face-diffusion step (nu + mean nut across the face; band faces: nu
 * along their open links). */
pcfd_status pcfd_mac_diffuse_smagorinsky(pcfd_system* system, double nu, double cs, double dt);
/* DeviceCompositeAmrProjection::transport_embedded_apertures(dt, nu, cs, false) (amr_pressure.cu:
 * 1868-1911), the MAC step's transport of the compact embedded face velocities (special slots
 * after the coarse/fine ones): node means over apertures and regular carrier faces, LS gradients,
 * bounded MUSCL along same-axis aperture chains, pairwise Smagorinsky momentum exchange scattered
 * back to apertures and carrier faces.  FP32 atomics, as the reference. */
pcfd_status pcfd_mac_transport_apertures(pcfd_system* system, double dt, double nu, double cs);
/* The cell eddy viscosity [S] (host, FP32) of the last pcfd_mac_diffuse_smagorinsky. */
pcfd_status pcfd_mac_eddy_viscosity_host(pcfd_system* system, float* nut);

/* ---- instrumentation ---------------------------------------------------------------------- */
/* Average device time of one launch sequence of `which` (0 full apply, 1 orthogonal apply,
 * 2 preconditioner, 3 divergence, 4 flux correction, 5 FP64 dot, 6/7/8 preconditioner
 * pre-smoothing / coarse correction / post-smoothing of the separate-launch cycle, 9/14/15 one
 * GCRO column orthogonalisation against 3 recycled + 13/5/24 basis vectors, 10/11/12/13 the
 * fused cycle's pre-smoothing / restriction / aggregation hierarchy / prolongation +
 * post-smoothing, 16 the learned network on every brick, 17 one Chebyshev smoothing step of the
 * composite cycle's first stage, 18 one delayed-CGS2 column against 13 basis vectors), measured with CUDA events on the system stream over
 * `iterations` back-to-back repetitions on resident scratch vectors. */
pcfd_status pcfd_time_kernel(pcfd_system* system, int32_t which, int32_t iterations, double* ms_per_launch);
/* Device-timeline markers on the system stream (slots 0..7) for whole-job timing. */
pcfd_status pcfd_event_record(pcfd_system* system, int32_t slot);
pcfd_status pcfd_event_elapsed(pcfd_system* system, int32_t start_slot, int32_t stop_slot, double* ms);
/* Per-launch device time of one instrumented region inside the real time step: begin arms
 * `capacity` CUDA event pairs recorded on the system stream around every launch of `region`;
 * end waits for them, writes up to `capacity` per-launch times (ms) and the count, and disarms. */
enum {
    PCFD_PROFILE_STRUCTURED_APPLY = 0,   /* brick-tiled FP64 7-point operator kernel */
    PCFD_PROFILE_PRECONDITIONER = 1,     /* one whole multigrid preconditioner application */
    PCFD_PROFILE_STAGE_SMOOTH = 2,       /* one smoothing step of the composite cycle's first stage
                                            (its stage chain runs uncaptured while this is armed) */
    PCFD_PROFILE_DCGS_COLUMN = 3         /* bytes only (pcfd_profile_begin refuses it): one delayed-CGS2
                                            column against 13 basis vectors, the sequence that
                                            pcfd_time_kernel 18 times */
};
/* Algorithmic bytes of one launch of a profiled region (each element read once and written once):
 * region 0 17 B per slot of a non-covered brick; region 2 per stage row its rhs, x, diagonal,
 * direction read and write and next iterate, then in CSR form the row offset and per stored
 * coupling its column index and coefficient, in brick-structured form the row's packed face
 * coefficients, per rest coupling its column index and coefficient and per 4^3 block its six
 * neighbour blocks; region 3 per entry of the Krylov vectors' sweep (the non-covered bricks' slots
 * and the fragments) 258 B: the dot pass reads the 13 basis vectors, v and w (8 B each) and the
 * active flag, the update pass reads them again and writes v and the next vector.  0 for
 * region 1. */
pcfd_status pcfd_profile_bytes(pcfd_system* system, int32_t region, double* bytes_per_launch);
/* 1 when the composite cycle's first stage runs in brick-structured form (64 rows per 8^3 brick,
 * face neighbours found from the row index), 0 when it runs as CSR or the cycle is not composite. */
pcfd_status pcfd_stage_brick_structured(pcfd_system* system, int32_t* structured);
/* 1 when the preconditioner's fine level runs as fused brick kernels (8^3 bricks whose
 * level-0 aggregates follow the brick geometry), 0 when it runs as separate launches. */
pcfd_status pcfd_preconditioner_fused(pcfd_system* system, int32_t* fused);
/* Number of this library's kernels launched on the system's stream since creation. */
pcfd_status pcfd_launch_count(pcfd_system* system, int64_t* launches);
pcfd_status pcfd_profile_begin(pcfd_system* system, int32_t region, int32_t capacity);
pcfd_status pcfd_profile_end(pcfd_system* system, double* ms_per_launch, int32_t capacity, int32_t* launches);

/* ---- learned preconditioner (no reference counterpart) ------------------------------
 * A brick-local 3-D U-Net (8^3/4^3/2^3 levels, 16/32/64 channels, 3x3x3 BF16 tensor-core
 * convolutions with FP32 accumulation, ReLU, 1x1x1 head) maps D^-1 r / s and the active mask
 * of every non-covered brick to z / s (s = RMS of D^-1 r over the brick's active cells); the DOFs
 * after the structured slots (EB fragments) take one damped Jacobi step.  It is trained on
 * (r, multigrid preconditioner output) brick pairs that the solver harvests from its own
 * preconditioner calls.  The definition is oracle/unet.py; parameters are FP32 in the flat order
 * enc0, enc1, bottleneck, dec1 (up, skip), dec0 (up, skip) ([27][cout][cin] each), head [16]. */
typedef enum pcfd_preconditioner {
    PCFD_PRECONDITIONER_MULTIGRID = 0,   /* the multigrid V-cycle of pcfd_options (default) */
    PCFD_PRECONDITIONER_LEARNED = 1,     /* the U-Net, then one damped Jacobi sweep */
    PCFD_PRECONDITIONER_JACOBI = 2,      /* z = D^-1 r: the method without the network or the V-cycle */
    PCFD_PRECONDITIONER_LEARNED_MULTIGRID = 3 /* the composite cycle (PCFD_MG_CYCLE_COMPOSITE) with the
                                            U-Net in place of its fine pre-sweeps */
} pcfd_preconditioner;
/* Solves under either learned kind run flexible GCRO/LGMRES; one that does not converge is
 * finished by the multigrid solve from its last iterate (pcfd_solve_result.fallback_solves). */
pcfd_status pcfd_set_preconditioner(pcfd_system* system, int32_t kind);
pcfd_status pcfd_learned_parameter_count(int64_t* count);
/* Replaces the FP32 master parameters (and resets the optimiser); count = parameter count.
 * Before the first call a system uses He-normal weights from a fixed seed. */
pcfd_status pcfd_learned_set_parameters(pcfd_system* system, const float* parameters, int64_t count);
pcfd_status pcfd_learned_get_parameters(pcfd_system* system, float* parameters, int64_t count);
/* Training target of a harvested brick: the multigrid preconditioner's output on it, or the
 * solution of the brick's own diagonal block A_B z = r_B (conjugate gradients in the harvest
 * kernel; the part of the correction a brick-local network can represent, since it depends on
 * the brick's residual alone). */
enum {
    PCFD_LEARNED_TARGET_MULTIGRID = 0,
    PCFD_LEARNED_TARGET_BRICK_SOLVE = 1
};
/* From now on every multigrid preconditioner application of this system stores bricks_per_pair
 * randomly chosen bricks (input, mask, target) until capacity_pairs applications are stored.
 * The store is one per process (on the first harvesting system's device) and shared by all
 * systems, so pairs harvested on several grids accumulate; a call with another capacity,
 * bricks_per_pair or target starts an empty store. */
pcfd_status pcfd_learned_harvest_begin(pcfd_system* system, int32_t capacity_pairs, int32_t bricks_per_pair,
                                       uint64_t seed, int32_t target);
/* Stops harvesting (the store is kept for training); samples = stored bricks. */
pcfd_status pcfd_learned_harvest_stop(pcfd_system* system, int64_t* samples);
/* `steps` Adam steps (cosine decay from learning_rate to a tenth) on random batches of the
 * harvested bricks; final_loss = mean loss of the last min(steps, 50) steps. */
pcfd_status pcfd_learned_train(pcfd_system* system, int32_t steps, int32_t batch, double learning_rate,
                               uint64_t seed, double* final_loss);
/* Forward and backward pass on host samples: inputs [samples][512][2] (D^-1 r / s, mask),
 * targets [samples][512]; zhat [samples][512] = net output, loss, gradients [parameter count]
 * (may be NULL).  For checking the kernels against the oracle. */
pcfd_status pcfd_learned_evaluate_host(pcfd_system* system, int32_t samples, const float* inputs, const float* targets,
                                       float* zhat, double* loss, float* gradients);
/* z = learned preconditioner applied to r (device vectors [S]). */
pcfd_status pcfd_learned_apply_device(pcfd_system* system, const double* d_r, double* d_z);
/* No reference counterpart.  Limit of each tensor-core completion wait of the network kernels
 * (default 2 s): a wait that runs out makes the call return PCFD_TIMEOUT after the kernel has
 * drained its own MMAs and freed its tensor memory, and the system stays usable.
 * idle_barrier_once != 0 makes the first wait of the next network convolution poll a barrier that
 * nothing completes, so it runs out: the fault-path check of the tests (no GPU fault involved). */
pcfd_status pcfd_learned_set_wait(pcfd_system* system, double seconds, int32_t idle_barrier_once);

#ifdef __cplusplus
}
#endif
#endif
