/*
 * ref_shim.h -- flat C entry points into the reference ParaCFD host code, compiled from the
 * reference's own sources into oracle/_ref/libparacfd_ref.so.  TEST INFRASTRUCTURE ONLY:
 * the product never links this; tests and the CPU-baseline arm use it as the checker.
 */
#ifndef PCFD_REF_SHIM_H
#define PCFD_REF_SHIM_H
#include <stdint.h>
#include "../include/paracfd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { REF_CASE_BOX = 0, REF_CASE_NACA_SLAB = 1, REF_CASE_NACA_WING = 2, REF_CASE_BOX_CROPPED = 3 };

typedef struct ref_case_params {
    int32_t kind;            /* REF_CASE_* */
    int32_t naca_digits;     /* e.g. 12 for 0012, 4412 */
    int32_t section_points;  /* polygon points per surface */
    int32_t max_levels;
    int32_t brick_size;
    double base_cell_size;
    double chord;
    double span;             /* full span of the wing (NACA_WING) / slab width (NACA_SLAB) */
    double aoa_deg;
    double domain_lo[3], domain_hi[3];   /* explicit flow domain for the NACA cases */
    double surface_refinement_distance;
    double wing_refinement_distance;
    double wake_length, wake_radius;
    double min_volume_fraction;
} ref_case_params;

void ref_default_params(int32_t kind, ref_case_params* params);
/* Builds hierarchy -> EB atlas -> composite pressure system with the reference code. */
void* ref_case_create(const ref_case_params* params);
void ref_case_destroy(void* handle);
const char* ref_last_error(void);
/* Fills a topology view whose arrays live inside the handle. */
int ref_case_topology(void* handle, pcfd_topology* out);
/* The case's reference objects (AmrHierarchy, CompositeAmrPressureSystem, ParagliderConfig), for
 * C++ drivers compiled against the reference headers (oracle/adapter/adapter_probe.cpp). */
int ref_case_objects(void* handle, const void** hierarchy, const void** system, const void** config);
/* The reference's DeviceAmrLocator::locate_points (its GPU code) on the case's hierarchy:
 * points [count][3] (host), out5 [count][5] = level, brick, i, j, k (host).  Needs a GPU. */
int ref_locate_points(void* handle, const float* points, int64_t count, int32_t* out5);
/* Summary numbers: [levels, storage, active dofs, coarse_fine, embedded, regular corr,
 * gradient nodes, gauges, patches, boundary faces, unresolved cells, retained] */
int ref_case_summary(void* handle, int64_t* out12);
/* Per level: coarsest-first brick count and active brick count, [levels][2]. */
int ref_case_level_counts(void* handle, int64_t* out);

/* Reference host operators (FP64), DOF-indexed vectors of length S. */
int ref_apply_cpu(void* handle, const double* p, double* out);
int ref_diagonal_cpu(void* handle, double* diag);
/* Faces in the compact per-brick layout of paracfd_b200.h; special velocities in double. */
int ref_divergence_cpu(void* handle, const float* u, const float* v, const float* w,
                       const double* cf, const double* eb, double* divergence);
int ref_rhs_cpu(void* handle, const float* u, const float* v, const float* w,
                const double* cf, const double* eb, double rho, double dt, double* rhs);
/* In/out faces and special velocities. */
int ref_correct_fluxes_cpu(void* handle, const double* pressure, double rho, double dt,
                           float* u, float* v, float* w, double* cf, double* eb);
int ref_pressure_gradients_cpu(void* handle, const double* pressure, double* gradient3);

/* Cell-momentum host twins (reference amr_advection.cu:874-1100).  State x,y,z: FP32 [S], in/out. */
int ref_transport_cpu(void* handle, const float* u, const float* v, const float* w, const double* cf,
                      const double* eb, double dt, int external, double freestream, float* x, float* y, float* z);
int ref_smagorinsky_viscosity_cpu(void* handle, const float* x, const float* y, const float* z, double nu,
                                  double cs, double* viscosity);
int ref_diffuse_smagorinsky_cpu(void* handle, double nu, double cs, double dt, float* x, float* y, float* z);
int ref_diffuse_cpu(void* handle, double nu, double dt, float* x, float* y, float* z);
/* forces: 3 per wall side in patch order (plus side then minus side); returns side count in *sides */
int ref_wall_cpu(void* handle, double nu, double dt, double rho, float* x, float* y, float* z, double* forces,
                 int64_t* sides);
int ref_impulse_cpu(void* handle, const double* pressure, double dt, double rho, int physical, float* x, float* y,
                    float* z);
/* faces (compact layout) and special velocities are outputs; faces start from the given values */
int ref_reconstruct_cpu(void* handle, const float* x, const float* y, const float* z, float* u, float* v, float* w,
                        double* cf, double* eb);
int ref_outflow_rate_cpu(void* handle, const float* u, const float* v, const float* w, const double* cf,
                         const double* eb, int external, double* rate);

/* The smooth-wall twin on a copy of the state x,y,z, then compute_pressure_loads of `pressure` and
 * accumulate_viscous_loads of the wall's patch loads (aero_loads.cpp:183-204), as
 * ExternalAeroCore::aerodynamic_loads combines them: out = [Fp(3), Mp(3), Fv(3), Mv(3)]. */
int ref_wall_loads_cpu(void* handle, double nu, double dt, double rho, const float* x, const float* y, const float* z,
                       const double* pressure, double pressure_reference, const double* origin, double* out12);
/* compute_pressure_loads (aero_loads.cpp:183-195) of a DOF pressure vector: out = [F(3), M(3)]. */
int ref_pressure_loads(void* handle, const double* pressure, double pressure_reference, const double* origin,
                       double* out6);

/* Hierarchy from an arbitrary closed mesh (AmrHierarchy::build_static on the given requested
 * domain) and the composite pressure system WITHOUT an embedded-boundary atlas (the reference's
 * build_composite_amr_pressure_system(hierarchy) overload). */
void* ref_case_from_mesh(const double* positions, int64_t vertices, const uint32_t* indices, int64_t triangles,
                         const double* domain_lo, const double* domain_hi, double base_cell_size, int32_t max_levels,
                         int32_t brick_size, double wing_refinement_distance, double surface_refinement_distance,
                         double wake_length, double wake_radius);

/* The same with the reference's cut-cell embedded boundary: the closed mesh is the solid (its
 * discrete inside test), then build_amr_embedded_boundary_atlas and the atlas overload of
 * build_composite_amr_pressure_system, with ExternalAeroCore's atlas options
 * (external_aero_core.cpp:97-103). */
void* ref_case_from_mesh_eb(const double* positions, int64_t vertices, const uint32_t* indices, int64_t triangles,
                            const double* domain_lo, const double* domain_hi, double base_cell_size,
                            int32_t max_levels, int32_t brick_size, double wing_refinement_distance,
                            double surface_refinement_distance, double wake_length, double wake_radius,
                            double min_volume_fraction);

typedef struct ref_core_case {
    double speed, rho, nu, cfl, smagorinsky_cs, projection_tolerance;
    int32_t projection_max_iterations;
} ref_core_case;

/* Import a flat topology (e.g. one built by paracfd_b200's own preprocessing) into the
 * reference's AmrHierarchy + CompositeAmrPressureSystem objects, so its host twins and device
 * classes run on exactly that grid.  No mesh/atlas is attached. */
void* ref_import_topology(const pcfd_topology* topology);
/* The reference's device classes (DeviceAmrFields, DeviceCompositeAmrProjection,
 * DeviceCompositeCellMomentumTransport) driven with ExternalAeroCore's initialize/step sequence
 * (external_aero_core.cpp:245-328) on any case handle (fixture or imported). */
void* ref_device_core_create(void* case_handle, const ref_core_case* config, double min_volume_fraction);
void ref_device_core_destroy(void* core);
/* The same with the staggered MAC momentum path (the smooth fabric wall on or off); faces of its
 * fields in the compact per-brick layout. */
void* ref_device_core_create_mac(void* case_handle, const ref_core_case* config, int32_t smooth_wall);
int ref_device_core_faces(void* core, float* u, float* v, float* w);
int ref_device_core_initialize(void* core, double* stats6);
int ref_device_core_step(void* core, double* stats6);

/* Cell-momentum state [S] (FP32) and the FP32 pressure shadow widened to double [S]. */
int ref_device_core_state(void* core, float* x, float* y, float* z, double* pressure);

/* The reference's staggered MAC momentum path (DeviceAmrAdvection on DeviceAmrFields,
 * amr_advection.cu:1652-1690) on a case with a surface; faces [B][(bs+1) bs^2] per component in the
 * compact per-brick layout, nut [S].  ref_mac_links: the constructor's per-face link bytes. */
int ref_mac_links(void* case_handle, double protection_cells, uint8_t* links_u, uint8_t* links_v, uint8_t* links_w);
void* ref_mac_create(void* case_handle, double protection_cells);
void ref_mac_destroy(void* mac);
int ref_mac_set_faces(void* mac, const float* u, const float* v, const float* w);
int ref_mac_advect(void* mac, double dt);
int ref_mac_diffuse_smagorinsky(void* mac, double nu, double cs, double dt);
int ref_mac_state(void* mac, float* u, float* v, float* w, float* nut);
/* Special (coarse/fine, embedded) face velocities of the MAC objects' projection, and its
 * transport_embedded_apertures(dt, nu, cs, false). */
int ref_mac_set_special(void* mac, const double* coarse_fine, const double* embedded);
int ref_mac_transport_apertures(void* mac, double dt, double nu, double cs);
int ref_mac_special(void* mac, double* coarse_fine, double* embedded);

/* The reference's own GPU path (ExternalAeroCore on the fixture), for the sm_100a baseline arm. */
void* ref_core_create(void* case_handle, const ref_core_case* config);
void ref_core_destroy(void* core);
/* stats: [dt, gpu_step_ms, projection_ms, iterations, converged, residual] */
int ref_core_initialize(void* core, double* stats6);
int ref_core_step(void* core, double* stats6);
/* Cell-momentum state [S] (FP32) and the FP32 pressure shadow widened to double [S]. */
int ref_core_state(void* core, float* x, float* y, float* z, double* pressure);

#ifdef __cplusplus
}
#endif
#endif
