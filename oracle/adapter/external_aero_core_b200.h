// external_aero_core_b200.h -- the reference-side adapter: what a ParaCFD maintainer adds beside
// ExternalAeroCore (src/core/fluid/external_aero_core.h:124-182) to run the per-step solver path
// on paracfd_b200.  The reference keeps its own preprocessing (AmrHierarchy::build_static, the
// cut-cell atlas, build_composite_amr_pressure_system); the adapter flattens the hierarchy and
// composite system into a pcfd_topology and drives the C ABI of include/paracfd_b200.h.
//
// Compiled here against the reference headers (oracle/Makefile, target `adapter`): the test
// harness's topology export (oracle/ref_shim.cpp) is this TopologyView, and
// oracle/adapter/adapter_probe.cpp runs ExternalAeroCoreB200 beside the reference's own
// ExternalAeroCore in a GPU test.  Link: -lparacfd_b200 -lcudart.
#pragma once

#include "paracfd_b200.h"

#include "core/aero_loads.h"
#include "core/fluid/amr_grid.h"
#include "core/fluid/amr_pressure.h"
#include "core/fluid/external_aero_core.h"
#include "core/paraglider_config.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace paracfd_b200_adapter
{
    using namespace paracfd::core;

    // pcfd_topology over a reference hierarchy + composite system.  Per-brick metadata, the edge
    // lists and the Vec3d arrays are flattened into owned arrays; the system's plain vectors
    // (active, masks, volume, aggregates, WLS CSR indices) are borrowed, so the system must outlive
    // every use of `topology` (pcfd_system_create copies what it keeps).
    class TopologyView
    {
    public:
        pcfd_topology topology{};

        TopologyView(const AmrHierarchy& hierarchy, const CompositeAmrPressureSystem& system)
        {
            const auto& levels = hierarchy.levels();
            const int L = int(levels.size());
            levels_.resize(L);
            coord_.resize(L); neighbors_.resize(L); children_.resize(L); origin_.resize(L); flags_.resize(L);
            for (int l = 0; l < L; ++l)
            {
                const AmrLevel& lev = levels[l];
                for (const BrickMetadata& b : lev.bricks)
                {
                    coord_[l].insert(coord_[l].end(), {b.coord.x, b.coord.y, b.coord.z});
                    origin_[l].insert(origin_[l].end(), {b.origin.x, b.origin.y, b.origin.z});
                    for (int f = 0; f < 6; ++f) neighbors_[l].push_back(b.same_level_neighbor[f]);
                    for (int c = 0; c < 8; ++c) children_[l].push_back(b.children[c]);
                    flags_[l].push_back(b.flags);
                }
                pcfd_level& v = levels_[l];
                v.h = lev.h;
                v.brick_count = int32_t(lev.bricks.size());
                v.level_offset = system.level_offset[l];
                v.coord = coord_[l].data();
                v.origin = origin_[l].data();
                v.neighbors = neighbors_[l].data();
                v.flags = flags_[l].data();
                v.children = children_[l].data();
            }
            for (const Vec3d& c : system.centroid) centroid_.insert(centroid_.end(), {c.x, c.y, c.z});
            flatten(system.coarse_fine, cf_);
            flatten(system.embedded, eb_);
            for (const auto& r : system.regular_pressure_corrections)
            {
                rc_lower_.push_back(r.lower_dof); rc_upper_.push_back(r.upper_dof);
                rc_level_.push_back(r.level); rc_brick_.push_back(r.brick);
                rc_ijk_.insert(rc_ijk_.end(), {r.i, r.j, r.k});
                rc_axis_.push_back(r.axis); rc_area_.push_back(r.open_area); rc_delta_.push_back(r.two_point_delta);
                rc_lower_node_.push_back(r.lower_gradient_node); rc_upper_node_.push_back(r.upper_gradient_node);
                for (int a = 0; a < 3; ++a) rc_correction_.push_back(r.nonorthogonal_correction[a]);
                rc_weight_.push_back(r.upper_gradient_weight);
            }
            for (const Vec3d& w : system.pressure_gradient_weight) gradient_weight_.insert(gradient_weight_.end(), {w.x, w.y, w.z});
            for (const auto& g : system.gauges) { gauge_dof_.push_back(g.dof); gauge_coefficient_.push_back(g.coefficient); }
            for (const auto& p : system.surface_patches)
            {
                patch_area_.push_back(p.area);
                patch_centroid_.insert(patch_centroid_.end(), {p.centroid.x, p.centroid.y, p.centroid.z});
                patch_normal_.insert(patch_normal_.end(), {p.normal.x, p.normal.y, p.normal.z});
                patch_plus_.push_back(p.plus_dof); patch_minus_.push_back(p.minus_dof);
            }
            for (const auto& f : system.boundary_faces)
            {
                bf_dof_.push_back(f.dof);
                bf_area_.insert(bf_area_.end(), {f.outward_area.x, f.outward_area.y, f.outward_area.z});
                bf_centroid_.insert(bf_centroid_.end(), {f.centroid.x, f.centroid.y, f.centroid.z});
            }
            retained_.assign(system.face_state_retained_dofs.begin(), system.face_state_retained_dofs.end());

            pcfd_topology& t = topology;
            std::memset(&t, 0, sizeof(t));
            t.brick_size = system.brick_size;
            t.level_count = L;
            t.levels = levels_.data();
            for (int a = 0; a < 3; ++a) { t.domain_lo[a] = hierarchy.domain().lo[a]; t.domain_hi[a] = hierarchy.domain().hi[a]; }
            t.storage_size = system.storage_size;
            t.pressure_outlet_xmax = system.pressure_outlet_xmax ? 1 : 0;
            t.active = system.active.data();
            t.freestream_connected = system.freestream_connected.data();
            t.cut_face_mask = system.cut_face_mask.data();
            t.volume = system.volume.data();
            t.centroid = centroid_.data();
            t.preconditioner_aggregate = system.preconditioner_aggregate.data();
            t.coarse_fine = view(cf_);
            t.embedded = view(eb_);
            pcfd_regular_corrections& r = t.regular;
            r.count = int32_t(rc_lower_.size());
            r.lower_dof = rc_lower_.data(); r.upper_dof = rc_upper_.data(); r.level = rc_level_.data();
            r.brick = rc_brick_.data(); r.ijk = rc_ijk_.data(); r.axis = rc_axis_.data();
            r.open_area = rc_area_.data(); r.two_point_delta = rc_delta_.data();
            r.lower_gradient_node = rc_lower_node_.data(); r.upper_gradient_node = rc_upper_node_.data();
            r.nonorthogonal_correction = rc_correction_.data(); r.upper_gradient_weight = rc_weight_.data();
            t.gradient_node_count = int32_t(system.pressure_gradient_dof.size());
            t.gradient_dof = system.pressure_gradient_dof.data();
            t.gradient_offset = system.pressure_gradient_offset.data();
            t.gradient_neighbour = system.pressure_gradient_neighbour.data();
            t.gradient_weight = gradient_weight_.data();
            t.gauge_count = int32_t(gauge_dof_.size());
            t.gauge_dof = gauge_dof_.data();
            t.gauge_coefficient = gauge_coefficient_.data();
            t.patches.count = int32_t(patch_area_.size());
            t.patches.area = patch_area_.data(); t.patches.centroid = patch_centroid_.data();
            t.patches.normal = patch_normal_.data(); t.patches.plus_dof = patch_plus_.data();
            t.patches.minus_dof = patch_minus_.data();
            t.boundary_faces.count = int32_t(bf_dof_.size());
            t.boundary_faces.dof = bf_dof_.data(); t.boundary_faces.outward_area = bf_area_.data();
            t.boundary_faces.centroid = bf_centroid_.data();
            t.retained_count = int32_t(retained_.size());
            t.retained_dofs = retained_.data();
        }
        TopologyView(const TopologyView&) = delete;
        TopologyView& operator=(const TopologyView&) = delete;

    private:
        struct Edges
        {
            std::vector<int32_t> coarse, fine, lower_node, upper_node;
            std::vector<double> area, centre, normal_distance, face_centroid, factor, correction, weight;
            std::vector<int8_t> axis, direction;
        };
        static void flatten(const std::vector<CoarseFinePressureConnection>& in, Edges& out)
        {
            for (const auto& e : in)
            {
                out.coarse.push_back(e.coarse_dof);
                out.fine.push_back(e.fine_dof);
                out.area.push_back(e.open_area);
                out.centre.push_back(e.centre_distance);
                out.normal_distance.push_back(e.normal_distance);
                out.axis.push_back(e.axis);
                out.direction.push_back(e.direction);
                for (int a = 0; a < 3; ++a) out.face_centroid.push_back(e.face_centroid[a]);
                out.factor.push_back(e.orthogonal_gradient_factor);
                out.lower_node.push_back(e.lower_gradient_node);
                out.upper_node.push_back(e.upper_gradient_node);
                for (int a = 0; a < 3; ++a) out.correction.push_back(e.nonorthogonal_correction[a]);
                out.weight.push_back(e.upper_gradient_weight);
            }
        }
        static pcfd_connections view(Edges& c)
        {
            pcfd_connections v{};
            v.count = int32_t(c.coarse.size());
            v.coarse_dof = c.coarse.data(); v.fine_dof = c.fine.data(); v.open_area = c.area.data();
            v.centre_distance = c.centre.data(); v.normal_distance = c.normal_distance.data();
            v.axis = c.axis.data(); v.direction = c.direction.data(); v.face_centroid = c.face_centroid.data();
            v.orthogonal_gradient_factor = c.factor.data(); v.lower_gradient_node = c.lower_node.data();
            v.upper_gradient_node = c.upper_node.data(); v.nonorthogonal_correction = c.correction.data();
            v.upper_gradient_weight = c.weight.data();
            return v;
        }

        std::vector<pcfd_level> levels_;
        std::vector<std::vector<int32_t>> coord_, neighbors_, children_;
        std::vector<std::vector<double>> origin_;
        std::vector<std::vector<uint32_t>> flags_;
        std::vector<double> centroid_;
        Edges cf_, eb_;
        std::vector<int32_t> rc_lower_, rc_upper_, rc_level_, rc_brick_, rc_ijk_, rc_lower_node_, rc_upper_node_;
        std::vector<int8_t> rc_axis_;
        std::vector<double> rc_area_, rc_delta_, rc_correction_, rc_weight_;
        std::vector<double> gradient_weight_;
        std::vector<int32_t> gauge_dof_;
        std::vector<double> gauge_coefficient_;
        std::vector<double> patch_area_, patch_centroid_, patch_normal_;
        std::vector<int32_t> patch_plus_, patch_minus_;
        std::vector<int32_t> bf_dof_;
        std::vector<double> bf_area_, bf_centroid_;
        std::vector<int32_t> retained_;
    };

    // ExternalAeroCore's stepping surface (initialize, step, pressure/aerodynamic loads, state
    // downloads) on paracfd_b200.  Errors follow the reference's convention: exceptions, with
    // non-convergence reported in the stats (physical time advances only on convergence).
    class ExternalAeroCoreB200
    {
    public:
        ExternalAeroCoreB200(const AmrHierarchy& hierarchy, const CompositeAmrPressureSystem& system,
                             const ParagliderConfig& config, int device = 0)
            : config_(config), storage_(system.storage_size)
        {
            TopologyView view(hierarchy, system);
            pcfd_options options{};
            options.mg_precision = PCFD_MG_FP32;
            options.device = device;
            options.stream = nullptr;
            options.momentum_min_volume_fraction = config.amr.min_volume_fraction;
            options.mg_cycle = PCFD_MG_CYCLE_COMPOSITE;     // PCFD_MG_CYCLE_REFERENCE: the reference's cycle
            options.gmres_delayed = 1;
            options.gmres_recycle = -1;
            options.mg_stage_fp16 = 1;
            check(pcfd_system_create(&view.topology, &options, &handle_));
            pcfd_case c{};
            c.speed = config.freestream.speed;
            c.rho = config.freestream.rho;
            c.nu = config.freestream.nu;
            c.cfl = config.solver.cfl;
            c.smagorinsky_cs = config.solver.smagorinsky_cs;
            c.projection_tolerance = config.solver.projection_tolerance;
            c.projection_max_iterations = config.solver.projection_max_iterations;
            c.smooth_wall = 1;
            c.pressure_impulse = 1;
            check(pcfd_core_configure(handle_, &c));
        }
        ~ExternalAeroCoreB200() { pcfd_system_destroy(handle_); }
        ExternalAeroCoreB200(const ExternalAeroCoreB200&) = delete;
        ExternalAeroCoreB200& operator=(const ExternalAeroCoreB200&) = delete;

        ExternalAeroStepStats initialize()
        {
            pcfd_step_stats s{};
            const int status = pcfd_core_initialize(handle_, &s);
            if (status != PCFD_OK && status != PCFD_NOT_CONVERGED) check(status);
            return convert(s);
        }
        ExternalAeroStepStats step()
        {
            pcfd_step_stats s{};
            const int status = pcfd_core_step(handle_, &s);
            if (status != PCFD_OK && status != PCFD_NOT_CONVERGED) check(status);
            return convert(s);
        }
        AerodynamicLoads pressure_loads(double reference_pressure = 0.0) const { return loads(reference_pressure, false); }
        AerodynamicLoads aerodynamic_loads(double reference_pressure = 0.0) const { return loads(reference_pressure, true); }
        void download_pressure(std::vector<double>& pressure) const
        {
            pressure.resize(std::size_t(storage_));
            check(pcfd_get_pressure_host(handle_, pressure.data()));
        }
        bool download_cell_momentum_state(CompositeCellMomentumState& state) const
        {
            const std::size_t n = std::size_t(storage_);
            std::vector<float> x(n), y(n), z(n);
            check(pcfd_momentum_get_state_host(handle_, x.data(), y.data(), z.data()));
            state.x.assign(x.begin(), x.end());
            state.y.assign(y.begin(), y.end());
            state.z.assign(z.begin(), z.end());
            return true;
        }
        pcfd_system* handle() const { return handle_; }

    private:
        static void check(int status)
        {
            if (status != PCFD_OK) throw std::runtime_error(std::string("paracfd_b200: ") + pcfd_last_error_message());
        }
        static ExternalAeroStepStats convert(const pcfd_step_stats& s)
        {
            ExternalAeroStepStats o;
            o.dt = s.dt;
            o.physical_time = s.physical_time;
            o.projection_ms = s.projection_ms;
            o.gpu_step_ms = s.step_ms;
            o.max_abs_velocity = std::max(s.max_abs_velocity, s.max_abs_special_velocity);
            o.max_abs_regular_velocity = s.max_abs_velocity;
            o.max_abs_special_velocity = s.max_abs_special_velocity;
            o.max_diffusion_rate = s.max_diffusion_rate;
            o.cfl_velocity = s.cfl_velocity;
            o.effective_cfl = s.effective_cfl;
            o.diffusion_substeps = s.diffusion_substeps;
            o.pressure.converged = s.pressure.converged != 0;
            o.pressure.iterations = s.pressure.iterations;
            o.pressure.relative_residual = s.pressure.relative_residual;
            o.les_applied = true;
            o.embedded_transport_applied = true;
            o.smooth_fabric_wall_applied = true;
            o.conservative_cell_momentum = true;
            return o;
        }
        AerodynamicLoads loads(double reference_pressure, bool viscous) const
        {
            pcfd_loads l{};
            const Vec3d& o = config_.reference.moment_origin;
            const double origin[3] = {o.x, o.y, o.z};
            check(pcfd_core_loads(handle_, reference_pressure, origin, config_.reference.area, viscous ? 1 : 0, &l));
            AerodynamicLoads out;
            out.pressure_force = {l.pressure_force[0], l.pressure_force[1], l.pressure_force[2]};
            out.pressure_moment = {l.pressure_moment[0], l.pressure_moment[1], l.pressure_moment[2]};
            out.pressure_drag = out.pressure_force.x;
            out.pressure_side = out.pressure_force.y;
            out.pressure_lift = out.pressure_force.z;
            if (viscous)
            {
                out.viscous_force = {l.viscous_force[0], l.viscous_force[1], l.viscous_force[2]};
                out.viscous_moment = {l.viscous_moment[0], l.viscous_moment[1], l.viscous_moment[2]};
                out.total_force = {l.total_force[0], l.total_force[1], l.total_force[2]};
                out.total_moment = {l.total_moment[0], l.total_moment[1], l.total_moment[2]};
                out.viscous_drag = out.viscous_force.x; out.viscous_side = out.viscous_force.y; out.viscous_lift = out.viscous_force.z;
                out.drag = out.total_force.x; out.side = out.total_force.y; out.lift = out.total_force.z;
                out.viscous_loads_valid = true;
            }
            if (config_.reference.area > 0 && std::isfinite(l.cl))
            {
                out.force_coefficients_valid = true;
                if (viscous) { out.cl = l.cl; out.cd = l.cd; out.cs = l.cs; }
                else { out.cl_pressure = l.cl; out.cd_pressure = l.cd; out.cs_pressure = l.cs; }
            }
            return out;
        }

        ParagliderConfig config_;
        pcfd_system* handle_ = nullptr;
        int storage_ = 0;
    };
}
