// ref_shim.cpp -- exposes the reference ParaCFD preprocessing and host parity operators
// through flat C entry points.  Test infrastructure only (see ref_shim.h).  Everything that
// computes here is the reference's own code (AmrHierarchy::build_static,
// build_amr_embedded_boundary_atlas, build_composite_amr_pressure_system, apply_cpu,
// diagonal_cpu, composite_amr_*_cpu); this file only builds analytic fixtures, in the
// pattern of the reference's tools/physics_contract_probe.cpp:19-67, and converts layouts.
#include "ref_shim.h"
#include "adapter/external_aero_core_b200.h"

#include "core/fluid/amr_eb.h"
#include "core/fluid/amr_fields.h"
#include "core/fluid/amr_pressure.h"
#include "core/fluid/amr_advection.h"
#include "core/fluid/external_aero_core.h"
#include "core/geometry/mesh_clip.h"
#include "core/geometry/model_placement.h"
#include "core/paraglider_config.h"

#include <algorithm>
#include <chrono>
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

using namespace paracfd::core;

namespace
{
    thread_local std::string g_error;

    // ---- analytic fixtures ------------------------------------------------------------
    // Axis-aligned box solid of half extents `half` under a rigid placement (the
    // reference's manufactured-contract fixture, tools/physics_contract_probe.cpp:39-67).
    TriMesh box_mesh(Vec3d half)
    {
        TriMesh mesh;
        for (int vertex = 0; vertex < 8; ++vertex)
            for (int axis = 0; axis < 3; ++axis)
            {
                const double value = (vertex & (1 << axis)) ? half[axis] : -half[axis];
                mesh.positions_fp64.push_back(value);
                mesh.positions.push_back(float(value));
                mesh.normals.push_back(0);
            }
        const int faces[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
        for (int face = 0; face < 6; ++face)
            for (int t = 0; t < 2; ++t)
            {
                for (int corner : {0, t + 1, t + 2}) mesh.indices.push_back(faces[face][corner]);
                mesh.source_face_ids.push_back(face);
            }
        for (int axis = 0; axis < 3; ++axis)
        {
            mesh.bbox_min[axis] = float(-half[axis]);
            mesh.bbox_max[axis] = float(half[axis]);
        }
        return mesh;
    }

    class PlacedBox final : public ClosedSolidGeometry
    {
        Vec3d half_;
        ModelPlacement inverse_;
        Aabb3d bounds_;

    public:
        PlacedBox(Vec3d half, const ModelPlacement& placement) : half_(half)
        {
            if (!inverse_placement(placement, inverse_)) throw std::runtime_error("invalid box placement");
            for (int vertex = 0; vertex < 8; ++vertex)
            {
                Vec3d p;
                placement.apply((vertex & 1) ? half.x : -half.x, (vertex & 2) ? half.y : -half.y,
                                (vertex & 4) ? half.z : -half.z, p.x, p.y, p.z);
                bounds_.expand(p);
            }
        }
        const Aabb3d& bounds() const override { return bounds_; }
        void classify_points(const Vec3d* points, std::size_t count, double tolerance,
                             ClosedSolidPointLocation* locations) const override
        {
            for (std::size_t q = 0; q < count; ++q)
            {
                Vec3d p;
                inverse_.apply(points[q].x, points[q].y, points[q].z, p.x, p.y, p.z);
                double distance = -1e30;
                for (int axis = 0; axis < 3; ++axis) distance = std::max(distance, std::abs(p[axis]) - half_[axis]);
                locations[q] = distance > tolerance ? ClosedSolidPointLocation::outside
                             : (distance < -tolerance ? ClosedSolidPointLocation::inside
                                                       : ClosedSolidPointLocation::boundary);
            }
        }
    };

    // NACA 4-digit section (published thickness/camber formulas; the closed trailing edge
    // uses -0.1036 for the x^4 coefficient).  Returns a closed polygon in (x, z), counter-
    // clockwise, starting at the trailing edge along the upper surface.
    std::vector<std::array<double, 2>> naca_polygon(int digits, int points_per_side, double chord)
    {
        const double m = (digits / 1000) / 100.0, p = ((digits / 100) % 10) / 10.0, t = (digits % 100) / 100.0;
        auto evaluate = [&](double x, bool upper) {
            const double yt = 5 * t * (0.2969 * std::sqrt(x) - 0.1260 * x - 0.3516 * x * x + 0.2843 * x * x * x - 0.1036 * x * x * x * x);
            double yc = 0, slope = 0;
            if (m > 0 && p > 0)
            {
                if (x < p) { yc = m / (p * p) * (2 * p * x - x * x); slope = 2 * m / (p * p) * (p - x); }
                else { yc = m / ((1 - p) * (1 - p)) * ((1 - 2 * p) + 2 * p * x - x * x); slope = 2 * m / ((1 - p) * (1 - p)) * (p - x); }
            }
            const double theta = std::atan(slope);
            if (upper) return std::array<double, 2>{(x - yt * std::sin(theta)) * chord, (yc + yt * std::cos(theta)) * chord};
            return std::array<double, 2>{(x + yt * std::sin(theta)) * chord, (yc - yt * std::cos(theta)) * chord};
        };
        std::vector<std::array<double, 2>> polygon;
        const double pi = std::acos(-1.0);
        for (int q = 0; q < points_per_side; ++q)   // upper: TE -> LE
        {
            const double beta = pi * (1.0 - double(q) / points_per_side);
            polygon.push_back(evaluate(0.5 * (1 - std::cos(beta)), true));
        }
        for (int q = 0; q < points_per_side; ++q)   // lower: LE -> TE (TE point shared once)
        {
            const double beta = pi * double(q) / points_per_side;
            polygon.push_back(evaluate(0.5 * (1 - std::cos(beta)), false));
        }
        polygon[0] = {chord, 0.0};
        return polygon;   // upper TE..LE then lower LE..(just before TE): counter-clockwise in (x,z)?
    }

    double polygon_signed_area(const std::vector<std::array<double, 2>>& poly)
    {
        double a = 0;
        for (std::size_t q = 0; q < poly.size(); ++q)
        {
            const auto& p0 = poly[q];
            const auto& p1 = poly[(q + 1) % poly.size()];
            a += p0[0] * p1[1] - p1[0] * p0[1];
        }
        return 0.5 * a;
    }

    // Extruded section along +Y between y0 and y1, placed by `place` (section (x,z) -> world).
    // Caps are emitted when `caps` is set.  The solid below classifies against the same polygon.
    struct SectionPlacement
    {
        double cos_a = 1, sin_a = 0, pivot_x = 0, pivot_z = 0, tx = 0, tz = 0;
        void to_world(double x, double z, double& wx, double& wz) const
        {
            const double dx = x - pivot_x, dz = z - pivot_z;
            wx = pivot_x + tx + cos_a * dx + sin_a * dz;
            wz = pivot_z + tz - sin_a * dx + cos_a * dz;
        }
        void to_section(double wx, double wz, double& x, double& z) const
        {
            const double dx = wx - pivot_x - tx, dz = wz - pivot_z - tz;
            x = pivot_x + cos_a * dx - sin_a * dz;
            z = pivot_z + sin_a * dx + cos_a * dz;
        }
    };

    TriMesh extruded_mesh(const std::vector<std::array<double, 2>>& poly, const SectionPlacement& place,
                          double y0, double y1, bool caps)
    {
        TriMesh mesh;
        const int n = int(poly.size());
        auto push = [&](double x, double y, double z) {
            double wx, wz;
            place.to_world(x, z, wx, wz);
            mesh.positions_fp64.insert(mesh.positions_fp64.end(), {wx, y, wz});
            mesh.positions.insert(mesh.positions.end(), {float(wx), float(y), float(wz)});
            mesh.normals.insert(mesh.normals.end(), {0.f, 0.f, 0.f});
        };
        for (int q = 0; q < n; ++q) push(poly[q][0], y0, poly[q][1]);
        for (int q = 0; q < n; ++q) push(poly[q][0], y1, poly[q][1]);
        // Polygon is CCW in (x,z); with +Y out of the (z,x) plane the outward side normal
        // of edge (a->b) for a solid to the left follows from the winding below.
        for (int q = 0; q < n; ++q)
        {
            const uint32_t a0 = q, b0 = (q + 1) % n, a1 = n + q, b1 = n + (q + 1) % n;
            mesh.indices.insert(mesh.indices.end(), {a0, a1, b1, a0, b1, b0});
            mesh.source_face_ids.push_back(0);
            mesh.source_face_ids.push_back(0);
        }
        if (caps)
        {
            // fan around vertex 0 (convex enough for a fan? not in general) -> use centre point
            double cx = 0, cz = 0;
            for (auto& p : poly) { cx += p[0]; cz += p[1]; }
            cx /= n; cz /= n;
            const uint32_t c0 = uint32_t(mesh.positions.size() / 3);
            push(cx, y0, cz);
            const uint32_t c1 = c0 + 1;
            push(cx, y1, cz);
            for (int q = 0; q < n; ++q)
            {
                const uint32_t a = q, b = (q + 1) % n;
                mesh.indices.insert(mesh.indices.end(), {c0, b, a});
                mesh.source_face_ids.push_back(1);
                mesh.indices.insert(mesh.indices.end(), {c1, uint32_t(n + a), uint32_t(n + b)});
                mesh.source_face_ids.push_back(2);
            }
        }
        // Make the winding outward: compute signed volume and flip if negative.
        double volume = 0;
        for (std::size_t t = 0; t < mesh.indices.size() / 3; ++t)
        {
            const double* p0 = &mesh.positions_fp64[3 * mesh.indices[3 * t]];
            const double* p1 = &mesh.positions_fp64[3 * mesh.indices[3 * t + 1]];
            const double* p2 = &mesh.positions_fp64[3 * mesh.indices[3 * t + 2]];
            volume += p0[0] * (p1[1] * p2[2] - p1[2] * p2[1]) - p0[1] * (p1[0] * p2[2] - p1[2] * p2[0]) +
                      p0[2] * (p1[0] * p2[1] - p1[1] * p2[0]);
        }
        if (volume < 0)
            for (std::size_t t = 0; t < mesh.indices.size() / 3; ++t) std::swap(mesh.indices[3 * t + 1], mesh.indices[3 * t + 2]);
        float bmin[3] = {1e30f, 1e30f, 1e30f}, bmax[3] = {-1e30f, -1e30f, -1e30f};
        for (std::size_t v = 0; v < mesh.positions.size() / 3; ++v)
            for (int a = 0; a < 3; ++a)
            {
                bmin[a] = std::min(bmin[a], mesh.positions[3 * v + a]);
                bmax[a] = std::max(bmax[a], mesh.positions[3 * v + a]);
            }
        for (int a = 0; a < 3; ++a) { mesh.bbox_min[a] = bmin[a]; mesh.bbox_max[a] = bmax[a]; }
        return mesh;
    }

    class ExtrudedSection final : public ClosedSolidGeometry
    {
        std::vector<std::array<double, 2>> poly_;
        SectionPlacement place_;
        double y0_, y1_;
        bool finite_;
        Aabb3d bounds_;

    public:
        ExtrudedSection(std::vector<std::array<double, 2>> poly, SectionPlacement place, double y0, double y1, bool finite)
            : poly_(std::move(poly)), place_(place), y0_(y0), y1_(y1), finite_(finite)
        {
            for (auto& p : poly_)
            {
                double wx, wz;
                place_.to_world(p[0], p[1], wx, wz);
                bounds_.expand(Vec3d{wx, y0_, wz});
                bounds_.expand(Vec3d{wx, y1_, wz});
            }
        }
        const Aabb3d& bounds() const override { return bounds_; }
        void classify_points(const Vec3d* points, std::size_t count, double tolerance,
                             ClosedSolidPointLocation* locations) const override
        {
            const int n = int(poly_.size());
            for (std::size_t q = 0; q < count; ++q)
            {
                double x, z;
                place_.to_section(points[q].x, points[q].z, x, z);
                bool inside = false;
                double d2 = 1e300;
                for (int e = 0, f = n - 1; e < n; f = e++)
                {
                    const double xa = poly_[f][0], za = poly_[f][1], xb = poly_[e][0], zb = poly_[e][1];
                    if (((zb > z) != (za > z)) && (x < (xa - xb) * (z - zb) / (za - zb) + xb)) inside = !inside;
                    const double ex = xb - xa, ez = zb - za, len2 = ex * ex + ez * ez;
                    double s = len2 > 0 ? ((x - xa) * ex + (z - za) * ez) / len2 : 0;
                    s = std::clamp(s, 0.0, 1.0);
                    const double dx = x - (xa + s * ex), dz = z - (za + s * ez);
                    d2 = std::min(d2, dx * dx + dz * dz);
                }
                double signed_distance = inside ? -std::sqrt(d2) : std::sqrt(d2);
                if (finite_)
                {
                    const double y = points[q].y;
                    const double dy = std::max(y0_ - y, y - y1_);   // >0 outside the span
                    if (signed_distance < 0) signed_distance = std::max(signed_distance, dy);
                    else if (dy > 0) signed_distance = std::sqrt(signed_distance * signed_distance + dy * dy);
                }
                locations[q] = signed_distance > tolerance ? ClosedSolidPointLocation::outside
                             : (signed_distance < -tolerance ? ClosedSolidPointLocation::inside
                                                              : ClosedSolidPointLocation::boundary);
            }
        }
    };

    // ---- case object --------------------------------------------------------------------
    struct RefCase
    {
        ParagliderConfig config;
        TriMesh wing;
        std::unique_ptr<TriangleBvh> bvh;
        ClosedSolidGeometryPtr solid;
        AmrHierarchy hierarchy;
        AmrEmbeddedBoundaryAtlas atlas;
        CompositeAmrPressureSystem system;
        // the flattened pcfd_topology (the adapter's view of hierarchy + system)
        std::unique_ptr<paracfd_b200_adapter::TopologyView> view;
    };

    void export_case(RefCase& rc)
    {
        rc.view = std::make_unique<paracfd_b200_adapter::TopologyView>(rc.hierarchy, rc.system);
    }

    // Compact per-brick face layout <-> reference ghosted AmrHostFields.
    std::size_t u_compact(int bs, std::size_t slot, int i, int j, int k) { return slot * std::size_t((bs + 1) * bs * bs) + std::size_t((k * bs + j) * (bs + 1) + i); }
    std::size_t v_compact(int bs, std::size_t slot, int i, int j, int k) { return slot * std::size_t((bs + 1) * bs * bs) + std::size_t((k * (bs + 1) + j) * bs + i); }
    std::size_t w_compact(int bs, std::size_t slot, int i, int j, int k) { return slot * std::size_t((bs + 1) * bs * bs) + std::size_t((k * bs + j) * bs + i); }

    void to_host_fields(const RefCase& rc, const float* u, const float* v, const float* w, AmrHostFields& fields)
    {
        const int bs = rc.system.brick_size;
        for (int l = 0; l < int(rc.hierarchy.levels().size()); ++l)
        {
            auto& lv = fields.levels()[l];
            const auto& lay = lv.layout;
            const int nb = int(rc.hierarchy.levels()[l].bricks.size());
            const std::size_t slot0 = std::size_t(rc.system.level_offset[l]) / std::size_t(bs * bs * bs);
            for (int b = 0; b < nb; ++b)
                for (int k = 0; k < bs; ++k)
                    for (int j = 0; j < bs; ++j)
                        for (int i = 0; i <= bs; ++i)
                        {
                            lv.u[lay.u_index(b, i, j, k)] = u[u_compact(bs, slot0 + b, i, j, k)];
                            lv.v[lay.v_index(b, j, i, k)] = v[v_compact(bs, slot0 + b, j, i, k)];
                            lv.w[lay.w_index(b, j, k, i)] = w[w_compact(bs, slot0 + b, j, k, i)];
                        }
        }
    }
    void from_host_fields(const RefCase& rc, const AmrHostFields& fields, float* u, float* v, float* w)
    {
        const int bs = rc.system.brick_size;
        for (int l = 0; l < int(rc.hierarchy.levels().size()); ++l)
        {
            const auto& lv = fields.levels()[l];
            const auto& lay = lv.layout;
            const int nb = int(rc.hierarchy.levels()[l].bricks.size());
            const std::size_t slot0 = std::size_t(rc.system.level_offset[l]) / std::size_t(bs * bs * bs);
            for (int b = 0; b < nb; ++b)
                for (int k = 0; k < bs; ++k)
                    for (int j = 0; j < bs; ++j)
                        for (int i = 0; i <= bs; ++i)
                        {
                            u[u_compact(bs, slot0 + b, i, j, k)] = lv.u[lay.u_index(b, i, j, k)];
                            v[v_compact(bs, slot0 + b, j, i, k)] = lv.v[lay.v_index(b, j, i, k)];
                            w[w_compact(bs, slot0 + b, j, k, i)] = lv.w[lay.w_index(b, j, k, i)];
                        }
        }
    }

    CompositeAmrFluxes special_from(const RefCase& rc, const double* cf, const double* eb)
    {
        CompositeAmrFluxes f = make_zero_composite_fluxes(rc.system);
        for (std::size_t q = 0; q < f.coarse_fine_velocity.size(); ++q) f.coarse_fine_velocity[q] = cf ? cf[q] : 0.0;
        for (std::size_t q = 0; q < f.embedded_velocity.size(); ++q) f.embedded_velocity[q] = eb ? eb[q] : 0.0;
        return f;
    }

    template <class F> int guarded(F&& f)
    {
        try { f(); return 0; }
        catch (const std::exception& e) { g_error = e.what(); return 1; }
        catch (...) { g_error = "unknown exception"; return 1; }
    }
}

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

void ref_default_params(int32_t kind, ref_case_params* p)
{
    std::memset(p, 0, sizeof(*p));
    p->kind = kind;
    p->naca_digits = 12;
    p->section_points = 48;
    p->max_levels = 2;
    p->brick_size = 8;
    p->base_cell_size = 0.125;
    p->chord = 1.0;
    p->span = 2.0;
    p->aoa_deg = 4.0;
    p->surface_refinement_distance = 0.2;
    p->wing_refinement_distance = 0.2;
    p->wake_length = 0.5;
    p->wake_radius = 0.5;
    p->min_volume_fraction = 0.005;
    if (kind == REF_CASE_NACA_SLAB)
    {
        // Single uniform level over 4c x 2c x 2c (chord 1): the plain-method case, scaled by
        // base_cell_size (1/32 gives 128 x 64 x 64 cells).
        p->max_levels = 1;
        p->base_cell_size = 1.0 / 32.0;
        p->domain_lo[0] = -1.0; p->domain_lo[1] = -1.0; p->domain_lo[2] = -1.0;
        p->domain_hi[0] = 3.0; p->domain_hi[1] = 1.0; p->domain_hi[2] = 1.0;
        p->min_volume_fraction = 0.25;
    }
}

void* ref_case_create(const ref_case_params* p)
{
    RefCase* rc = nullptr;
    const int status = guarded([&] {
        auto owned = std::make_unique<RefCase>();
        RefCase& c = *owned;
        ParagliderConfig& config = c.config;
        config.amr.brick_size = p->brick_size;
        config.amr.max_levels = p->max_levels;
        config.amr.base_cell_size = p->base_cell_size;
        config.amr.wing_refinement_distance = p->wing_refinement_distance;
        config.amr.surface_refinement_distance = p->surface_refinement_distance;
        config.amr.wake_length = p->wake_length;
        config.amr.wake_radius = p->wake_radius;
        config.amr.min_volume_fraction = p->min_volume_fraction;
        Aabb3d domain;
        if (p->kind == REF_CASE_BOX || p->kind == REF_CASE_BOX_CROPPED)
        {
            // tools/physics_contract_probe.cpp:110-138 (box and --cropped variants)
            const bool cropped = p->kind == REF_CASE_BOX_CROPPED;
            const Vec3d half{0.6, 0.8, 0.18};
            TriMesh source = box_mesh(half);
            config.freestream.speed = 2;
            config.domain = {1.25, 1.25, 1.25, 1.25, false};
            const double pitch = 0.31, yaw = cropped ? 0 : 0.17, cp = std::cos(pitch), sp = std::sin(pitch),
                         ca = std::cos(yaw), sa = std::sin(yaw);
            const double rotation[9] = {ca * cp, -sa, ca * sp, sa * cp, ca, sa * sp, -sp, 0, cp};
            std::copy(rotation, rotation + 9, config.placement.m);
            if (cropped)
            {
                source = clip_mesh_to_axis_slab(source, 1, -0.25, 0.25);
                config.domain.lateral_margin = 0;
                config.amr.base_cell_size = 0.0625;
                config.amr.max_levels = 1;
            }
            config.placement = frame_wing_for_external_domain(source, config.placement, config.domain.upstream_margin,
                config.domain.lateral_margin, config.domain.vertical_margin, config.amr.base_cell_size * config.amr.brick_size);
            c.wing = placed_mesh(source, config.placement);
            c.solid = std::make_shared<PlacedBox>(half, config.placement);
            domain = automatic_flow_domain(c.wing, config.domain);
        }
        else
        {
            auto poly = naca_polygon(p->naca_digits, p->section_points, p->chord);
            if (polygon_signed_area(poly) < 0) std::reverse(poly.begin(), poly.end());
            SectionPlacement place;
            const double a = p->aoa_deg * std::acos(-1.0) / 180.0;
            place.cos_a = std::cos(a); place.sin_a = std::sin(a);
            place.pivot_x = 0.25 * p->chord; place.pivot_z = 0;
            // centre the placed section vertically on z = 0
            double zmin = 1e300, zmax = -1e300, xmin = 1e300, xmax = -1e300;
            for (const auto& pt : poly)
            {
                double wx, wz;
                place.to_world(pt[0], pt[1], wx, wz);
                zmin = std::min(zmin, wz); zmax = std::max(zmax, wz); xmin = std::min(xmin, wx); xmax = std::max(xmax, wx);
            }
            place.tz = -0.5 * (zmin + zmax);
            const bool slab = p->kind == REF_CASE_NACA_SLAB;
            const double half_span = 0.5 * p->span;
            if (slab)
            {
                // Section extruded beyond the slab and clipped at the side walls (slip walls
                // meet the solid): same construction as the reference's cropped contract.
                TriMesh longer = extruded_mesh(poly, place, -half_span - 0.5, half_span + 0.5, true);
                c.wing = clip_mesh_to_axis_slab(longer, 1, p->domain_lo[1], p->domain_hi[1]);
                c.solid = std::make_shared<ExtrudedSection>(poly, place, -1e9, 1e9, false);
            }
            else
            {
                c.wing = extruded_mesh(poly, place, -half_span, half_span, true);
                c.solid = std::make_shared<ExtrudedSection>(poly, place, -half_span, half_span, true);
            }
            // Express the requested box as the reference's automatic-domain margins so that
            // ExternalAeroCore, which always derives its domain from them, builds this grid too.
            config.domain.upstream_margin = double(c.wing.bbox_min[0]) - p->domain_lo[0];
            // (1e-9 short of the box so the brick-count ceil cannot round up by one brick)
            config.domain.downstream_margin = p->domain_hi[0] - double(c.wing.bbox_max[0]) - 1e-9;
            config.domain.lateral_margin = slab ? 0.0 : 0.5 * ((p->domain_hi[1] - p->domain_lo[1]) - (double(c.wing.bbox_max[1]) - double(c.wing.bbox_min[1])) - 1e-9);
            config.domain.vertical_margin = 0.5 * ((p->domain_hi[2] - p->domain_lo[2]) - (double(c.wing.bbox_max[2]) - double(c.wing.bbox_min[2])) - 1e-9);
            config.domain.half_wing_symmetry = false;
            domain = automatic_flow_domain(c.wing, config.domain);
        }
        c.bvh = std::make_unique<TriangleBvh>(c.wing);
        c.hierarchy = AmrHierarchy::build_static(domain, c.wing, *c.bvh, config.amr, config.domain.half_wing_symmetry);
        EmbeddedBoundaryBuildOptions eb;
        eb.min_volume_fraction = config.amr.min_volume_fraction;
        eb.retain_signed_bracketed_small_roots_for_face_state = true;
        eb.min_aperture_area_fraction = config.amr.min_aperture_area_fraction;
        eb.closed_solid = c.solid;
        c.atlas = build_amr_embedded_boundary_atlas(c.hierarchy, c.wing, *c.bvh, eb);
        if (!c.atlas.ready_for_flow())
            throw std::runtime_error("reference EB atlas has " + std::to_string(c.atlas.unresolved_count()) + " unresolved cells");
        CompositeAmrPressureBuildOptions options;
        options.pressure_outlet_xmax = true;
        c.system = build_composite_amr_pressure_system(c.hierarchy, c.atlas, options);
        c.system.hierarchy = &c.hierarchy;
        export_case(c);
        rc = owned.release();
    });
    return status == 0 ? rc : nullptr;
}

void ref_case_destroy(void* handle) { delete static_cast<RefCase*>(handle); }

int ref_case_topology(void* handle, pcfd_topology* out)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        *out = c.view->topology;
    });
}
int ref_case_objects(void* handle, const void** hierarchy, const void** system, const void** config)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        if (hierarchy) *hierarchy = &c.hierarchy;
        if (system) *system = &c.system;
        if (config) *config = &c.config;
    });
}
int ref_locate_points(void* handle, const float* points, int64_t count, int32_t* out5)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        if (count <= 0) return;
        DeviceAmrLocator locator(c.hierarchy);
        GpuAmrPoint* d_points = nullptr;
        GpuBrickLocation* d_out = nullptr;
        auto ok = [](cudaError_t e, const char* what) { if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e)); };
        ok(cudaMalloc(&d_points, size_t(count) * sizeof(GpuAmrPoint)), "points");
        ok(cudaMalloc(&d_out, size_t(count) * sizeof(GpuBrickLocation)), "locations");
        std::vector<GpuAmrPoint> host(static_cast<size_t>(count));
        for (int64_t q = 0; q < count; ++q) host[size_t(q)] = {points[3 * q], points[3 * q + 1], points[3 * q + 2]};
        ok(cudaMemcpy(d_points, host.data(), host.size() * sizeof(GpuAmrPoint), cudaMemcpyHostToDevice), "upload points");
        locator.locate_points(d_points, d_out, int(count));
        std::vector<GpuBrickLocation> result(static_cast<size_t>(count));
        ok(cudaMemcpy(result.data(), d_out, result.size() * sizeof(GpuBrickLocation), cudaMemcpyDeviceToHost), "download locations");
        cudaFree(d_points);
        cudaFree(d_out);
        for (int64_t q = 0; q < count; ++q)
        {
            const GpuBrickLocation& r = result[size_t(q)];
            out5[5 * q] = r.level; out5[5 * q + 1] = r.brick; out5[5 * q + 2] = r.i; out5[5 * q + 3] = r.j; out5[5 * q + 4] = r.k;
        }
    });
}
int ref_case_summary(void* handle, int64_t* o)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        const auto& s = c.system;
        int64_t active = 0;
        for (auto a : s.active) active += a ? 1 : 0;
        o[0] = int64_t(c.hierarchy.levels().size()); o[1] = s.storage_size; o[2] = active;
        o[3] = int64_t(s.coarse_fine.size()); o[4] = int64_t(s.embedded.size());
        o[5] = int64_t(s.regular_pressure_corrections.size()); o[6] = int64_t(s.pressure_gradient_dof.size());
        o[7] = int64_t(s.gauges.size()); o[8] = int64_t(s.surface_patches.size());
        o[9] = int64_t(s.boundary_faces.size()); o[10] = int64_t(c.atlas.unresolved_count());
        o[11] = int64_t(s.face_state_retained_dofs.size());
    });
}

int ref_case_level_counts(void* handle, int64_t* o)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        for (std::size_t l = 0; l < c.hierarchy.levels().size(); ++l)
        {
            o[2 * l] = int64_t(c.hierarchy.levels()[l].bricks.size());
            o[2 * l + 1] = int64_t(c.hierarchy.levels()[l].active_bricks);
        }
    });
}

int ref_apply_cpu(void* handle, const double* p, double* out)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        std::vector<double> in(p, p + c.system.storage_size), result;
        c.system.apply_cpu(in, result);
        std::copy(result.begin(), result.end(), out);
    });
}

int ref_diagonal_cpu(void* handle, double* diag)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        std::vector<double> d;
        c.system.diagonal_cpu(d);
        std::copy(d.begin(), d.end(), diag);
    });
}

int ref_divergence_cpu(void* handle, const float* u, const float* v, const float* w, const double* cf,
                       const double* eb, double* divergence)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        AmrHostFields fields(c.hierarchy);
        to_host_fields(c, u, v, w, fields);
        std::vector<double> div;
        composite_amr_divergence_cpu(c.system, fields, special_from(c, cf, eb), div);
        std::copy(div.begin(), div.end(), divergence);
    });
}

int ref_rhs_cpu(void* handle, const float* u, const float* v, const float* w, const double* cf,
                const double* eb, double rho, double dt, double* rhs)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        AmrHostFields fields(c.hierarchy);
        to_host_fields(c, u, v, w, fields);
        std::vector<double> r;
        composite_amr_projection_rhs_cpu(c.system, fields, special_from(c, cf, eb), rho, dt, r);
        std::copy(r.begin(), r.end(), rhs);
    });
}

int ref_correct_fluxes_cpu(void* handle, const double* pressure, double rho, double dt, float* u, float* v,
                           float* w, double* cf, double* eb)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        AmrHostFields fields(c.hierarchy);
        to_host_fields(c, u, v, w, fields);
        CompositeAmrFluxes special = special_from(c, cf, eb);
        std::vector<double> p(pressure, pressure + c.system.storage_size);
        composite_amr_correct_fluxes_cpu(c.system, p, rho, dt, fields, special);
        from_host_fields(c, fields, u, v, w);
        if (cf) std::copy(special.coarse_fine_velocity.begin(), special.coarse_fine_velocity.end(), cf);
        if (eb) std::copy(special.embedded_velocity.begin(), special.embedded_velocity.end(), eb);
    });
}

int ref_pressure_gradients_cpu(void* handle, const double* pressure, double* gradient3)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        std::vector<double> p(pressure, pressure + c.system.storage_size);
        const auto g = composite_pressure_gradients_cpu(c.system, p);
        for (std::size_t q = 0; q < g.size(); ++q)
            for (int a = 0; a < 3; ++a) gradient3[3 * q + a] = g[q][a];
    });
}


}  // extern "C"

namespace
{
    CompositeCellMomentumState state_from(const RefCase& c, const float* x, const float* y, const float* z)
    {
        CompositeCellMomentumState st;
        const int n = c.system.storage_size;
        st.x.assign(x, x + n); st.y.assign(y, y + n); st.z.assign(z, z + n);
        return st;
    }
    void state_to(const CompositeCellMomentumState& st, float* x, float* y, float* z)
    {
        std::copy(st.x.begin(), st.x.end(), x); std::copy(st.y.begin(), st.y.end(), y); std::copy(st.z.begin(), st.z.end(), z);
    }
    struct RefCore
    {
        RefCase* owner = nullptr;
        std::unique_ptr<ExternalAeroCore> core;
    };
    void fill_stats(const ExternalAeroStepStats& s, double* o)
    {
        o[0] = s.dt; o[1] = s.gpu_step_ms; o[2] = s.projection_ms; o[3] = s.pressure.iterations;
        o[4] = s.pressure.converged ? 1 : 0; o[5] = s.pressure.relative_residual;
    }
}

extern "C" {

int ref_transport_cpu(void* handle, const float* u, const float* v, const float* w, const double* cf, const double* eb,
                      double dt, int external, double freestream, float* x, float* y, float* z)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        AmrHostFields fields(c.hierarchy);
        to_host_fields(c, u, v, w, fields);
        CompositeCellMomentumState st = state_from(c, x, y, z);
        conservative_composite_cell_momentum_cpu(c.system, fields, special_from(c, cf, eb), dt, st, external != 0, freestream);
        state_to(st, x, y, z);
    });
}

int ref_smagorinsky_viscosity_cpu(void* handle, const float* x, const float* y, const float* z, double nu, double cs, double* viscosity)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        const auto vis = composite_cell_smagorinsky_viscosity_cpu(c.system, state_from(c, x, y, z), nu, cs);
        std::copy(vis.begin(), vis.end(), viscosity);
    });
}

int ref_diffuse_smagorinsky_cpu(void* handle, double nu, double cs, double dt, float* x, float* y, float* z)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        CompositeCellMomentumState st = state_from(c, x, y, z);
        diffuse_composite_cell_momentum_smagorinsky_cpu(c.system, nu, cs, dt, st);
        state_to(st, x, y, z);
    });
}

int ref_diffuse_cpu(void* handle, double nu, double dt, float* x, float* y, float* z)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        CompositeCellMomentumState st = state_from(c, x, y, z);
        diffuse_composite_cell_momentum_cpu(c.system, nu, dt, st);
        state_to(st, x, y, z);
    });
}

int ref_wall_cpu(void* handle, double nu, double dt, double rho, float* x, float* y, float* z, double* forces, int64_t* sides)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        CompositeCellMomentumState st = state_from(c, x, y, z);
        const auto loads = apply_composite_cell_smooth_fabric_wall_cpu(c.system, nu, dt, rho, st);
        state_to(st, x, y, z);
        if (sides) *sides = int64_t(loads.size());
        if (forces)
            for (std::size_t q = 0; q < loads.size(); ++q)
                for (int a = 0; a < 3; ++a) forces[3 * q + a] = loads[q].force[a];
    });
}

int ref_wall_loads_cpu(void* handle, double nu, double dt, double rho, const float* x, const float* y, const float* z,
                       const double* pressure, double pref, const double* origin, double* out12)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        CompositeCellMomentumState st = state_from(c, x, y, z);
        const auto wall = apply_composite_cell_smooth_fabric_wall_cpu(c.system, nu, dt, rho, st);
        std::vector<double> p(pressure, pressure + c.system.storage_size);
        FreestreamConfig fs;
        fs.rho = rho;
        AeroReferenceConfig rf;
        rf.moment_origin = {origin[0], origin[1], origin[2]};
        // (ExternalAeroCore::aerodynamic_loads: pressure loads, then the wall model's patch loads)
        auto loads = compute_pressure_loads(c.system, p, c.wing.triangle_count() + 1, fs, rf, pref);
        accumulate_viscous_loads(loads, wall, fs, rf);
        for (int a = 0; a < 3; ++a)
        {
            out12[a] = loads.pressure_force[a];
            out12[3 + a] = loads.pressure_moment[a];
            out12[6 + a] = loads.viscous_force[a];
            out12[9 + a] = loads.viscous_moment[a];
        }
    });
}

int ref_impulse_cpu(void* handle, const double* pressure, double dt, double rho, int physical, float* x, float* y, float* z)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        CompositeCellMomentumState st = state_from(c, x, y, z);
        std::vector<double> p(pressure, pressure + c.system.storage_size);
        apply_composite_cell_pressure_impulse_cpu(c.system, p, dt, rho, st, physical != 0);
        state_to(st, x, y, z);
    });
}

int ref_reconstruct_cpu(void* handle, const float* x, const float* y, const float* z, float* u, float* v, float* w, double* cf, double* eb)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        AmrHostFields fields(c.hierarchy);
        to_host_fields(c, u, v, w, fields);
        CompositeAmrFluxes fluxes;
        reconstruct_composite_cell_fluxes_cpu(c.system, state_from(c, x, y, z), fields, fluxes);
        from_host_fields(c, fields, u, v, w);
        if (cf) std::copy(fluxes.coarse_fine_velocity.begin(), fluxes.coarse_fine_velocity.end(), cf);
        if (eb) std::copy(fluxes.embedded_velocity.begin(), fluxes.embedded_velocity.end(), eb);
    });
}

int ref_outflow_rate_cpu(void* handle, const float* u, const float* v, const float* w, const double* cf, const double* eb,
                         int external, double* rate)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        AmrHostFields fields(c.hierarchy);
        to_host_fields(c, u, v, w, fields);
        *rate = composite_cell_max_outflow_rate_cpu(c.system, fields, special_from(c, cf, eb), external != 0);
    });
}

int ref_pressure_loads(void* handle, const double* pressure, double pref, const double* origin, double* out)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(handle);
        std::vector<double> p(pressure, pressure + c.system.storage_size);
        FreestreamConfig fs;
        AeroReferenceConfig rf;
        rf.moment_origin = {origin[0], origin[1], origin[2]};
        const auto loads = compute_pressure_loads(c.system, p, c.wing.triangle_count() + 1, fs, rf, pref);
        for (int a = 0; a < 3; ++a) { out[a] = loads.pressure_force[a]; out[3 + a] = loads.pressure_moment[a]; }
    });
}

}  // extern "C"

namespace
{
    // Closed-solid classification by the reference's own discrete test on the same triangle
    // shell (TriangleBvh::classify_closed_point, three-ray parity with a solid-angle fallback).
    // The reference's STEP solid answers classify_discrete_points exactly this way
    // (occt_closed_solid.cpp:46-58), and the cut-cell builder only asks that question
    // (solid_embedded_boundary.cpp:831, 1062; amr_eb.cpp:109).
    class DiscreteMeshSolid final : public ClosedSolidGeometry
    {
        const TriangleBvh* bvh_;
        Aabb3d bounds_;

    public:
        DiscreteMeshSolid(const TriMesh& mesh, const TriangleBvh* bvh) : bvh_(bvh)
        {
            for (std::size_t q = 0; q < mesh.vertex_count(); ++q)
            {
                const auto p = mesh.vertex_position_double(q);
                bounds_.expand(Vec3d{p[0], p[1], p[2]});
            }
        }
        const Aabb3d& bounds() const override { return bounds_; }
        void classify_points(const Vec3d* points, std::size_t count, double tolerance,
                             ClosedSolidPointLocation* locations) const override
        {
            for (std::size_t q = 0; q < count; ++q)
            {
                const auto location = bvh_->classify_closed_point(points[q], tolerance);
                locations[q] = location == ClosedMeshPointLocation::inside ? ClosedSolidPointLocation::inside
                             : (location == ClosedMeshPointLocation::outside ? ClosedSolidPointLocation::outside
                                                                             : ClosedSolidPointLocation::boundary);
            }
        }
    };

    RefCase* case_from_mesh(const double* positions, int64_t vertices, const uint32_t* indices, int64_t triangles,
                            const double* lo, const double* hi, double h, int32_t levels, int32_t bs,
                            double wing_distance, double surface_distance, double wake_length, double wake_radius,
                            bool cut_cells, double min_volume_fraction)
    {
        auto owned = std::make_unique<RefCase>();
        RefCase& c = *owned;
        TriMesh mesh;
        float bmin[3] = {1e30f, 1e30f, 1e30f}, bmax[3] = {-1e30f, -1e30f, -1e30f};
        for (int64_t v = 0; v < vertices; ++v)
            for (int a = 0; a < 3; ++a)
            {
                const double x = positions[3 * v + a];
                mesh.positions_fp64.push_back(x);
                mesh.positions.push_back(float(x));
                mesh.normals.push_back(0.f);
                bmin[a] = std::min(bmin[a], float(x));
                bmax[a] = std::max(bmax[a], float(x));
            }
        for (int64_t t = 0; t < triangles; ++t)
        {
            for (int k = 0; k < 3; ++k) mesh.indices.push_back(indices[3 * t + k]);
            mesh.source_face_ids.push_back(0);
        }
        for (int a = 0; a < 3; ++a) { mesh.bbox_min[a] = bmin[a]; mesh.bbox_max[a] = bmax[a]; }
        c.wing = mesh;
        c.bvh = std::make_unique<TriangleBvh>(c.wing);
        c.config.amr.base_cell_size = h;
        c.config.amr.max_levels = levels;
        c.config.amr.brick_size = bs;
        c.config.amr.wing_refinement_distance = wing_distance;
        c.config.amr.surface_refinement_distance = surface_distance;
        c.config.amr.wake_length = wake_length;
        c.config.amr.wake_radius = wake_radius;
        c.config.amr.min_volume_fraction = min_volume_fraction;
        Aabb3d domain;
        domain.lo = {lo[0], lo[1], lo[2]};
        domain.hi = {hi[0], hi[1], hi[2]};
        c.hierarchy = AmrHierarchy::build_static(domain, c.wing, *c.bvh, c.config.amr, false);
        if (cut_cells)
        {
            // external_aero_core.cpp:97-103: the constructor's atlas options.
            c.solid = std::make_shared<DiscreteMeshSolid>(c.wing, c.bvh.get());
            EmbeddedBoundaryBuildOptions eb;
            eb.min_volume_fraction = c.config.amr.min_volume_fraction;
            eb.retain_signed_bracketed_small_roots_for_face_state = true;
            eb.min_aperture_area_fraction = c.config.amr.min_aperture_area_fraction;
            eb.closed_solid = c.solid;
            c.atlas = build_amr_embedded_boundary_atlas(c.hierarchy, c.wing, *c.bvh, eb);
            if (!c.atlas.ready_for_flow())
            {
                std::string why;
                int shown = 0;
                for (const auto& level : c.atlas.levels)
                    for (const auto& problem : level.topology.unresolved)
                        if (shown++ < 3)
                        {
                            const Vec3d at = level.topology.grid.cell_centroid(problem.parent_cell);
                            why += "; level " + std::to_string(level.level) + " at (" + std::to_string(at.x) + "," +
                                   std::to_string(at.y) + "," + std::to_string(at.z) + "): " + problem.reason;
                        }
                throw std::runtime_error("reference EB atlas has " + std::to_string(c.atlas.unresolved_count()) +
                                         " unresolved cells" + why);
            }
            CompositeAmrPressureBuildOptions options;
            options.pressure_outlet_xmax = true;
            c.system = build_composite_amr_pressure_system(c.hierarchy, c.atlas, options);
        }
        else
            c.system = build_composite_amr_pressure_system(c.hierarchy, true);
        c.system.hierarchy = &c.hierarchy;
        export_case(c);
        return owned.release();
    }
}

extern "C" {

void* ref_case_from_mesh(const double* positions, int64_t vertices, const uint32_t* indices, int64_t triangles,
                         const double* lo, const double* hi, double h, int32_t levels, int32_t bs, double wing_distance,
                         double surface_distance, double wake_length, double wake_radius)
{
    RefCase* rc = nullptr;
    guarded([&] {
        rc = case_from_mesh(positions, vertices, indices, triangles, lo, hi, h, levels, bs, wing_distance,
                            surface_distance, wake_length, wake_radius, false, 0.25);
    });
    return rc;
}

void* ref_case_from_mesh_eb(const double* positions, int64_t vertices, const uint32_t* indices, int64_t triangles,
                            const double* lo, const double* hi, double h, int32_t levels, int32_t bs,
                            double wing_distance, double surface_distance, double wake_length, double wake_radius,
                            double min_volume_fraction)
{
    RefCase* rc = nullptr;
    guarded([&] {
        rc = case_from_mesh(positions, vertices, indices, triangles, lo, hi, h, levels, bs, wing_distance,
                            surface_distance, wake_length, wake_radius, true, min_volume_fraction);
    });
    return rc;
}

void* ref_import_topology(const pcfd_topology* t)
{
    RefCase* rc = nullptr;
    guarded([&] {
        auto owned = std::make_unique<RefCase>();
        RefCase& c = *owned;
        const int bs = t->brick_size;
        const double h0 = t->levels[0].h;
        Aabb3d domain;
        domain.lo = {t->domain_lo[0], t->domain_lo[1], t->domain_lo[2]};
        // a hair inside the padded box so the brick count is not rounded up
        domain.hi = {t->domain_hi[0] - 1e-9, t->domain_hi[1] - 1e-9, t->domain_hi[2] - 1e-9};
        c.hierarchy = AmrHierarchy::uniform(domain, h0, bs, 1);
        auto& levels = c.hierarchy.levels();
        levels.assign(t->level_count, {});
        for (int l = 0; l < t->level_count; ++l)
        {
            const pcfd_level& src = t->levels[l];
            AmrLevel& lev = levels[l];
            lev.level = l;
            lev.h = src.h;
            lev.bricks.resize(src.brick_count);
            for (int b = 0; b < src.brick_count; ++b)
            {
                BrickMetadata& m = lev.bricks[b];
                m.level = l;
                m.coord = {src.coord[3 * b], src.coord[3 * b + 1], src.coord[3 * b + 2]};
                m.origin = {src.origin[3 * b], src.origin[3 * b + 1], src.origin[3 * b + 2]};
                m.h = src.h;
                for (int f = 0; f < 6; ++f) m.same_level_neighbor[f] = src.neighbors[6 * b + f];
                if (src.children)
                    for (int k = 0; k < 8; ++k) m.children[k] = src.children[8 * b + k];
                m.flags = src.flags[b];
                if (m.active()) ++lev.active_bricks;
            }
        }
        CompositeAmrPressureSystem& s = c.system;
        s.hierarchy = &c.hierarchy;
        s.brick_size = bs;
        s.storage_size = t->storage_size;
        s.pressure_outlet_xmax = t->pressure_outlet_xmax != 0;
        const int n = t->storage_size;
        for (int l = 0; l < t->level_count; ++l) s.level_offset.push_back(t->levels[l].level_offset);
        s.active.assign(t->active, t->active + n);
        s.freestream_connected = t->freestream_connected ? std::vector<unsigned char>(t->freestream_connected, t->freestream_connected + n) : s.active;
        s.cut_face_mask.assign(t->cut_face_mask, t->cut_face_mask + n);
        s.volume.assign(t->volume, t->volume + n);
        s.centroid.resize(n);
        for (int q = 0; q < n; ++q) s.centroid[q] = {t->centroid[3 * q], t->centroid[3 * q + 1], t->centroid[3 * q + 2]};
        s.preconditioner_aggregate.assign(t->preconditioner_aggregate, t->preconditioner_aggregate + n);
        auto conn = [](const pcfd_connections& in, std::vector<CoarseFinePressureConnection>& out) {
            out.resize(in.count);
            for (int e = 0; e < in.count; ++e)
            {
                auto& o = out[e];
                o.coarse_dof = in.coarse_dof[e]; o.fine_dof = in.fine_dof[e]; o.open_area = in.open_area[e];
                o.centre_distance = in.centre_distance[e]; o.normal_distance = in.normal_distance[e];
                o.axis = in.axis[e]; o.direction = in.direction[e];
                o.face_centroid = {in.face_centroid[3 * e], in.face_centroid[3 * e + 1], in.face_centroid[3 * e + 2]};
                o.orthogonal_gradient_factor = in.orthogonal_gradient_factor[e];
                o.lower_gradient_node = in.lower_gradient_node[e]; o.upper_gradient_node = in.upper_gradient_node[e];
                o.nonorthogonal_correction = {in.nonorthogonal_correction[3 * e], in.nonorthogonal_correction[3 * e + 1], in.nonorthogonal_correction[3 * e + 2]};
                o.upper_gradient_weight = in.upper_gradient_weight[e];
            }
        };
        conn(t->coarse_fine, s.coarse_fine);
        conn(t->embedded, s.embedded);
        s.regular_pressure_corrections.resize(t->regular.count);
        for (int e = 0; e < t->regular.count; ++e)
        {
            auto& o = s.regular_pressure_corrections[e];
            const pcfd_regular_corrections& r = t->regular;
            o.lower_dof = r.lower_dof[e]; o.upper_dof = r.upper_dof[e]; o.level = r.level[e]; o.brick = r.brick[e];
            o.i = r.ijk[3 * e]; o.j = r.ijk[3 * e + 1]; o.k = r.ijk[3 * e + 2]; o.axis = r.axis[e];
            o.open_area = r.open_area[e]; o.two_point_delta = r.two_point_delta[e];
            o.lower_gradient_node = r.lower_gradient_node[e]; o.upper_gradient_node = r.upper_gradient_node[e];
            o.nonorthogonal_correction = {r.nonorthogonal_correction[3 * e], r.nonorthogonal_correction[3 * e + 1], r.nonorthogonal_correction[3 * e + 2]};
            o.upper_gradient_weight = r.upper_gradient_weight[e];
        }
        const int nodes = t->gradient_node_count;
        s.pressure_gradient_dof.assign(t->gradient_dof, t->gradient_dof + nodes);
        s.pressure_gradient_offset.assign(t->gradient_offset, t->gradient_offset + (nodes ? nodes + 1 : 0));
        const int nnz = nodes ? t->gradient_offset[nodes] : 0;
        s.pressure_gradient_neighbour.assign(t->gradient_neighbour, t->gradient_neighbour + nnz);
        s.pressure_gradient_weight.resize(nnz);
        for (int q = 0; q < nnz; ++q) s.pressure_gradient_weight[q] = {t->gradient_weight[3 * q], t->gradient_weight[3 * q + 1], t->gradient_weight[3 * q + 2]};
        s.pressure_gradient_rank.assign(nodes, 3);
        s.pressure_gradient_ring.assign(nodes, 1);
        for (int g = 0; g < t->gauge_count; ++g) s.gauges.push_back({t->gauge_dof[g], t->gauge_coefficient[g]});
        for (int p = 0; p < t->patches.count; ++p)
        {
            CompositeSurfacePressurePatch o;
            o.area = t->patches.area[p];
            o.centroid = {t->patches.centroid[3 * p], t->patches.centroid[3 * p + 1], t->patches.centroid[3 * p + 2]};
            o.normal = {t->patches.normal[3 * p], t->patches.normal[3 * p + 1], t->patches.normal[3 * p + 2]};
            o.plus_dof = t->patches.plus_dof[p];
            o.minus_dof = t->patches.minus_dof[p];
            s.surface_patches.push_back(o);
        }
        for (int f = 0; f < t->boundary_faces.count; ++f)
        {
            CompositeBoundaryPressureFace o;
            o.dof = t->boundary_faces.dof[f];
            o.outward_area = {t->boundary_faces.outward_area[3 * f], t->boundary_faces.outward_area[3 * f + 1], t->boundary_faces.outward_area[3 * f + 2]};
            o.centroid = {t->boundary_faces.centroid[3 * f], t->boundary_faces.centroid[3 * f + 1], t->boundary_faces.centroid[3 * f + 2]};
            s.boundary_faces.push_back(o);
        }
        s.face_state_retained_dofs.assign(t->retained_dofs, t->retained_dofs + t->retained_count);
        s.face_state_retained_small_root_count = s.face_state_retained_dofs.size();
        export_case(c);
        rc = owned.release();
    });
    return rc;
}

namespace
{
    struct RefDeviceCore
    {
        RefCase* c = nullptr;
        ref_core_case cfg{};
        std::unique_ptr<DeviceAmrFields> fields;
        std::unique_ptr<DeviceCompositeAmrProjection> projection;
        std::unique_ptr<DeviceCompositeCellMomentumTransport> momentum;
        std::unique_ptr<DeviceAmrAdvection> advection;     // staggered MAC mode (no cell momentum)
        bool smooth_wall = false;                           // MAC mode: the projection's smooth fabric wall
        bool initialized = false;
        double time = 0;
    };
    double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b)
    {
        return std::chrono::duration<double, std::milli>(b - a).count();
    }
}

void* ref_device_core_create(void* case_handle, const ref_core_case* cfg, double min_volume_fraction)
{
    RefDeviceCore* out = nullptr;
    guarded([&] {
        auto core = std::make_unique<RefDeviceCore>();
        core->c = static_cast<RefCase*>(case_handle);
        core->cfg = *cfg;
        RefCase& c = *core->c;
        core->fields = std::make_unique<DeviceAmrFields>(c.hierarchy);
        core->projection = std::make_unique<DeviceCompositeAmrProjection>(c.system, *core->fields);
        core->momentum = std::make_unique<DeviceCompositeCellMomentumTransport>(c.system, *core->fields, min_volume_fraction);
        out = core.release();
    });
    return out;
}

// The same with the staggered MAC momentum path (ExternalAeroExecutionOptions::
// conservative_cell_momentum = false, the smooth fabric wall as asked): DeviceAmrAdvection with
// the constructor's 2.5-cell fabric protection instead of the cell-momentum transport.
void* ref_device_core_create_mac(void* case_handle, const ref_core_case* cfg, int32_t smooth_wall)
{
    RefDeviceCore* out = nullptr;
    guarded([&] {
        auto core = std::make_unique<RefDeviceCore>();
        core->c = static_cast<RefCase*>(case_handle);
        core->cfg = *cfg;
        RefCase& c = *core->c;
        if (!c.bvh) throw std::invalid_argument("the MAC mode needs a case with a surface");
        core->fields = std::make_unique<DeviceAmrFields>(c.hierarchy);
        core->projection = std::make_unique<DeviceCompositeAmrProjection>(c.system, *core->fields);
        core->advection = std::make_unique<DeviceAmrAdvection>(c.hierarchy, *c.bvh, 2.5, &c.system);
        core->smooth_wall = smooth_wall != 0;
        out = core.release();
    });
    return out;
}

int ref_device_core_faces(void* handle, float* u, float* v, float* w)
{
    return guarded([&] {
        RefDeviceCore& k = *static_cast<RefDeviceCore*>(handle);
        AmrHostFields host(k.c->hierarchy);
        k.fields->download(host);
        from_host_fields(*k.c, host, u, v, w);
    });
}

void ref_device_core_destroy(void* core) { delete static_cast<RefDeviceCore*>(core); }

// ExternalAeroCore::initialize (external_aero_core.cpp:245-302) on the imported grid.
int ref_device_core_initialize(void* handle, double* stats)
{
    return guarded([&] {
        RefDeviceCore& k = *static_cast<RefDeviceCore*>(handle);
        RefCase& c = *k.c;
        const CompositeAmrPressureSystem& s = c.system;
        const Real speed = Real(k.cfg.speed);
        CompositeCellMomentumState state;
        state.x.assign(s.storage_size, Real(0)); state.y.assign(s.storage_size, Real(0)); state.z.assign(s.storage_size, Real(0));
        for (int q = 0; q < s.storage_size; ++q) if (s.active[q] && s.freestream_connected[q]) state.x[q] = speed;
        AmrHostFields fields(c.hierarchy);
        CompositeAmrFluxes fluxes;
        reconstruct_composite_cell_fluxes_cpu(s, state, fields, fluxes);
        const int bs = s.brick_size;
        for (int l = 0; l < int(c.hierarchy.levels().size()); ++l)
        {
            const AmrLevel& level = c.hierarchy.levels()[l];
            AmrHostLevelFields& values = fields.levels()[l];
            for (int b = 0; b < int(level.bricks.size()); ++b)
            {
                const BrickMetadata& m = level.bricks[b];
                if (!m.active()) continue;
                for (int kk = 0; kk < bs; ++kk)
                    for (int j = 0; j < bs; ++j)
                    {
                        if (m.flags & BRICK_XMIN) { const int d = s.dof(l, b, 0, j, kk); values.u[values.layout.u_index(b, 0, j, kk)] = s.active[d] && s.freestream_connected[d] ? speed : Real(0); }
                        if (m.flags & BRICK_XMAX) { const int d = s.dof(l, b, bs - 1, j, kk); values.u[values.layout.u_index(b, bs, j, kk)] = s.active[d] && s.freestream_connected[d] ? speed : Real(0); }
                    }
            }
        }
        k.fields->upload(fields);
        k.projection->upload_special_fluxes(fluxes);
        if (k.momentum)
        {
            k.momentum->upload_state(state);
            k.momentum->reconstruct_fluxes(k.projection->coarse_fine_velocity_device(), k.projection->embedded_velocity_device());
        }
        k.fields->apply_external_aero_boundaries(speed);
        const double maximum = std::max(1e-9, std::abs(k.cfg.speed)), dt = k.cfg.cfl * c.hierarchy.finest_cell_size() / maximum;
        const auto t0 = std::chrono::steady_clock::now();
        if (k.advection) k.projection->sync_coarse_fine_from_fields();   // project(false, dt) with its default sync
        const AmrGpuSolveResult r = k.projection->project(Real(k.cfg.rho), Real(dt), k.cfg.projection_tolerance, k.cfg.projection_max_iterations, false);
        if (r.converged && k.momentum) k.momentum->apply_projected_pressure_gradient(k.projection->pressure(), Real(dt), Real(k.cfg.rho));
        const auto t1 = std::chrono::steady_clock::now();
        k.initialized = r.converged;
        stats[0] = dt; stats[1] = ms_between(t0, t1); stats[2] = stats[1]; stats[3] = r.iterations; stats[4] = r.converged; stats[5] = r.relative_residual;
    });
}

// ExternalAeroCore::step (external_aero_core.cpp:304-328), conservative cell momentum, wall on.
int ref_device_core_step(void* handle, double* stats)
{
    return guarded([&] {
        RefDeviceCore& k = *static_cast<RefDeviceCore*>(handle);
        if (!k.initialized) throw std::logic_error("reference device core needs a converged initialization");
        RefCase& c = *k.c;
        const auto t0 = std::chrono::steady_clock::now();
        const double h = c.hierarchy.finest_cell_size();
        if (k.advection)
        {
            // ExternalAeroCore::step, MAC branch (external_aero_core.cpp:304-311, 321-325)
            const double mass_flux = k.fields->max_abs_velocity(), special = k.projection->max_abs_special_velocity(),
                         eb_rate = k.projection->max_embedded_cfl_rate();
            (void)special;
            const double cfl_rate = std::max({1e-9, std::abs(k.cfg.speed) / h, mass_flux / h, eb_rate}), dt_value = k.cfg.cfl / cfl_rate;
            const Real dt = Real(dt_value), nu = Real(k.cfg.nu), cs = Real(k.cfg.smagorinsky_cs), speed = Real(k.cfg.speed), rho = Real(k.cfg.rho);
            k.advection->advect(*k.fields, dt);
            k.advection->diffuse_smagorinsky(*k.fields, nu, cs, dt);
            k.fields->apply_external_aero_boundaries(speed);
            k.projection->transport_embedded_apertures(dt, nu, cs, false);
            if (k.smooth_wall) k.projection->apply_smooth_fabric_wall_model(dt, nu);
            const auto p0 = std::chrono::steady_clock::now();
            k.projection->sync_coarse_fine_from_fields();
            const AmrGpuSolveResult r = k.projection->project(rho, dt, k.cfg.projection_tolerance, k.cfg.projection_max_iterations, true);
            const auto p1 = std::chrono::steady_clock::now();
            if (r.converged) k.time += dt_value;
            cudaDeviceSynchronize();
            const auto t1 = std::chrono::steady_clock::now();
            stats[0] = dt_value; stats[1] = ms_between(t0, t1); stats[2] = ms_between(p0, p1); stats[3] = r.iterations; stats[4] = r.converged; stats[5] = r.relative_residual;
            return;
        }
        const double rate = k.momentum->max_outflow_rate(k.projection->coarse_fine_velocity_device(), k.projection->embedded_velocity_device(), true);
        (void)k.fields->max_abs_velocity();
        (void)k.momentum->max_abs_velocity();
        (void)k.projection->max_abs_special_velocity();
        (void)k.projection->max_embedded_cfl_rate();
        const double cfl_rate = std::max({1e-9, std::abs(k.cfg.speed) / h, rate}), dt_value = k.cfg.cfl / cfl_rate;
        const Real dt = Real(dt_value), nu = Real(k.cfg.nu), cs = Real(k.cfg.smagorinsky_cs), speed = Real(k.cfg.speed), rho = Real(k.cfg.rho);
        k.momentum->step(k.projection->coarse_fine_velocity_device(), k.projection->embedded_velocity_device(), dt, true, speed);
        k.momentum->diffuse_smagorinsky(nu, cs, dt);
        k.momentum->apply_smooth_fabric_wall_model(dt, nu);
        k.momentum->reconstruct_fluxes(k.projection->coarse_fine_velocity_device(), k.projection->embedded_velocity_device());
        k.fields->apply_external_aero_boundaries(speed);
        const auto p0 = std::chrono::steady_clock::now();
        const AmrGpuSolveResult r = k.projection->project(rho, dt, k.cfg.projection_tolerance, k.cfg.projection_max_iterations, true);
        const auto p1 = std::chrono::steady_clock::now();
        if (r.converged) { k.momentum->apply_projected_pressure_gradient(k.projection->pressure(), dt, rho); k.time += dt_value; }
        cudaDeviceSynchronize();
        const auto t1 = std::chrono::steady_clock::now();
        stats[0] = dt_value; stats[1] = ms_between(t0, t1); stats[2] = ms_between(p0, p1); stats[3] = r.iterations; stats[4] = r.converged; stats[5] = r.relative_residual;
    });
}

namespace
{
    // The reference's staggered MAC momentum objects on one case (amr_advection.cu:1652-1690).
    struct RefMac
    {
        RefCase* c = nullptr;
        std::unique_ptr<DeviceAmrFields> fields;
        std::unique_ptr<DeviceAmrAdvection> advection;
        std::unique_ptr<DeviceCompositeAmrProjection> projection;
    };
    Vec3d mac_face_centre(const BrickMetadata& brick, double h, int component, int i, int j, int k)
    {
        return brick.origin + Vec3d{(i + (component == 0 ? 0.0 : 0.5)) * h, (j + (component == 1 ? 0.0 : 0.5)) * h,
                                    (k + (component == 2 ? 0.0 : 0.5)) * h};
    }
}

// The per-face link bytes of the DeviceAmrAdvection constructor (amr_advection.cu:1655-1659):
// every face 0x3f; in a brick whose box grown by protection_cells * h meets the surface, a face
// within that distance of it takes 0x40 plus, when it is off the surface, one bit per axis
// direction whose h-long segment does not cross the surface; then the interface links that the
// composite momentum coupling replaces (build_momentum_interface_replaced_links) are cleared.
// Compact per-brick face layout.
int ref_mac_links(void* case_handle, double protection_cells, uint8_t* lu, uint8_t* lv, uint8_t* lw)
{
    return guarded([&] {
        RefCase& c = *static_cast<RefCase*>(case_handle);
        if (!c.bvh) throw std::invalid_argument("MAC links need a case with a surface");
        const int bs = c.system.brick_size;
        const std::size_t per = std::size_t((bs + 1) * bs * bs);
        const std::vector<AmrMacFaceDirectionalLink> replaced = build_momentum_interface_replaced_links(c.system);
        uint8_t* out[3] = {lu, lv, lw};
        auto compact = [&](int component, std::size_t slot, int i, int j, int k) {
            return component == 0 ? u_compact(bs, slot, i, j, k) : (component == 1 ? v_compact(bs, slot, i, j, k) : w_compact(bs, slot, i, j, k));
        };
        for (int l = 0; l < int(c.hierarchy.levels().size()); ++l)
        {
            const AmrLevel& level = c.hierarchy.levels()[l];
            const std::size_t slot0 = std::size_t(c.system.level_offset[l]) / std::size_t(bs * bs * bs);
            for (int comp = 0; comp < 3; ++comp) std::fill(out[comp] + slot0 * per, out[comp] + (slot0 + level.bricks.size()) * per, uint8_t(0x3f));
            const double radius = protection_cells * level.h;
            for (int b = 0; b < int(level.bricks.size()); ++b)
            {
                const BrickMetadata& record = level.bricks[b];
                if (!record.active()) continue;
                const Aabb3d grown{{record.origin.x - radius, record.origin.y - radius, record.origin.z - radius},
                                   {record.origin.x + bs * level.h + radius, record.origin.y + bs * level.h + radius,
                                    record.origin.z + bs * level.h + radius}};
                if (c.bvh->query_aabb(grown).empty()) continue;
                for (int comp = 0; comp < 3; ++comp)
                {
                    const int ni = comp == 0 ? bs + 1 : bs, nj = comp == 1 ? bs + 1 : bs, nk = comp == 2 ? bs + 1 : bs;
                    for (int k = 0; k < nk; ++k)
                        for (int j = 0; j < nj; ++j)
                            for (int i = 0; i < ni; ++i)
                            {
                                const Vec3d point = mac_face_centre(record, level.h, comp, i, j, k);
                                const double distance = c.bvh->distance(point, radius);
                                if (!std::isfinite(distance)) continue;
                                uint8_t links = 0x40;
                                if (distance > 1e-7 * level.h)
                                    for (int axis = 0; axis < 3; ++axis)
                                        for (int direction = -1; direction <= 1; direction += 2)
                                        {
                                            Vec3d other = point;
                                            other[axis] += direction * level.h;
                                            if (!c.bvh->intersect_segment(point, other, 1e-7, 1.0 - 1e-7).hit)
                                                links |= uint8_t(1u << (2 * axis + (direction > 0)));
                                        }
                                out[comp][compact(comp, slot0 + b, i, j, k)] = links;
                            }
                }
            }
            for (const AmrMacFaceDirectionalLink& link : replaced)
                if (link.face.level == l)
                    out[link.face.component][compact(link.face.component, slot0 + link.face.brick, link.face.i, link.face.j, link.face.k)] &=
                        uint8_t(~(1u << (2 * link.transport_axis + (link.direction > 0))));
        }
    });
}

void* ref_mac_create(void* case_handle, double protection_cells)
{
    RefMac* out = nullptr;
    guarded([&] {
        auto m = std::make_unique<RefMac>();
        m->c = static_cast<RefCase*>(case_handle);
        if (!m->c->bvh) throw std::invalid_argument("MAC advection needs a case with a surface");
        m->fields = std::make_unique<DeviceAmrFields>(m->c->hierarchy);
        m->advection = std::make_unique<DeviceAmrAdvection>(m->c->hierarchy, *m->c->bvh, protection_cells, &m->c->system);
        m->projection = std::make_unique<DeviceCompositeAmrProjection>(m->c->system, *m->fields);
        out = m.release();
    });
    return out;
}

void ref_mac_destroy(void* mac) { delete static_cast<RefMac*>(mac); }

int ref_mac_set_faces(void* mac, const float* u, const float* v, const float* w)
{
    return guarded([&] {
        RefMac& m = *static_cast<RefMac*>(mac);
        AmrHostFields host(m.c->hierarchy);
        to_host_fields(*m.c, u, v, w, host);
        m.fields->upload(host);
    });
}

int ref_mac_advect(void* mac, double dt)
{
    return guarded([&] {
        RefMac& m = *static_cast<RefMac*>(mac);
        m.advection->advect(*m.fields, Real(dt));
    });
}

int ref_mac_diffuse_smagorinsky(void* mac, double nu, double cs, double dt)
{
    return guarded([&] {
        RefMac& m = *static_cast<RefMac*>(mac);
        m.advection->diffuse_smagorinsky(*m.fields, Real(nu), Real(cs), Real(dt));
    });
}

int ref_mac_set_special(void* mac, const double* coarse_fine, const double* embedded)
{
    return guarded([&] {
        RefMac& m = *static_cast<RefMac*>(mac);
        m.projection->upload_special_fluxes(special_from(*m.c, coarse_fine, embedded));
    });
}

// DeviceCompositeAmrProjection::transport_embedded_apertures (amr_pressure.cu:1868-1911) as the
// MAC step calls it (no molecular fabric wall)
int ref_mac_transport_apertures(void* mac, double dt, double nu, double cs)
{
    return guarded([&] {
        RefMac& m = *static_cast<RefMac*>(mac);
        m.projection->transport_embedded_apertures(Real(dt), Real(nu), Real(cs), false);
    });
}

int ref_mac_special(void* mac, double* coarse_fine, double* embedded)
{
    return guarded([&] {
        RefMac& m = *static_cast<RefMac*>(mac);
        CompositeAmrFluxes f;
        m.projection->download_special_fluxes(f);
        std::copy(f.coarse_fine_velocity.begin(), f.coarse_fine_velocity.end(), coarse_fine);
        std::copy(f.embedded_velocity.begin(), f.embedded_velocity.end(), embedded);
    });
}

int ref_mac_state(void* mac, float* u, float* v, float* w, float* nut)
{
    return guarded([&] {
        RefMac& m = *static_cast<RefMac*>(mac);
        AmrHostFields host(m.c->hierarchy);
        m.fields->download(host);
        from_host_fields(*m.c, host, u, v, w);
        if (nut)
        {
            const int bs = m.c->system.brick_size;
            for (int l = 0; l < int(m.c->hierarchy.levels().size()); ++l)
            {
                const auto& lv = host.levels()[l];
                const std::size_t slot0 = std::size_t(m.c->system.level_offset[l]) / std::size_t(bs * bs * bs);
                for (int b = 0; b < int(m.c->hierarchy.levels()[l].bricks.size()); ++b)
                    for (int k = 0; k < bs; ++k)
                        for (int j = 0; j < bs; ++j)
                            for (int i = 0; i < bs; ++i)
                                nut[(slot0 + b) * std::size_t(bs * bs * bs) + std::size_t((k * bs + j) * bs + i)] = lv.nut[lv.layout.cell_index(b, i, j, k)];
            }
        }
    });
}

void* ref_core_create(void* case_handle, const ref_core_case* cfg)
{
    RefCore* out = nullptr;
    guarded([&] {
        RefCase& c = *static_cast<RefCase*>(case_handle);
        auto core = std::make_unique<RefCore>();
        core->owner = &c;
        ParagliderConfig config = c.config;
        config.freestream.speed = cfg->speed;
        config.freestream.rho = cfg->rho;
        config.freestream.nu = cfg->nu;
        config.solver.cfl = cfg->cfl;
        config.solver.smagorinsky_cs = cfg->smagorinsky_cs;
        config.solver.projection_tolerance = cfg->projection_tolerance;
        config.solver.projection_max_iterations = cfg->projection_max_iterations;
        ExternalAeroExecutionOptions options;
        options.closed_solid = c.solid;
        core->core = std::make_unique<ExternalAeroCore>(c.wing, *c.bvh, config, options);
        out = core.release();
    });
    return out;
}

void ref_core_destroy(void* core) { delete static_cast<RefCore*>(core); }

int ref_core_initialize(void* core, double* stats)
{
    return guarded([&] { fill_stats(static_cast<RefCore*>(core)->core->initialize(), stats); });
}

int ref_core_step(void* core, double* stats)
{
    return guarded([&] { fill_stats(static_cast<RefCore*>(core)->core->step(), stats); });
}

int ref_device_core_state(void* handle, float* x, float* y, float* z, double* pressure)
{
    return guarded([&] {
        RefDeviceCore& k = *static_cast<RefDeviceCore*>(handle);
        if (k.momentum)
        {
            CompositeCellMomentumState st;
            k.momentum->download_state(st);
            state_to(st, x, y, z);
        }
        if (pressure)
        {
            std::vector<Real> p;
            k.projection->download_pressure(p);
            for (std::size_t q = 0; q < p.size(); ++q) pressure[q] = double(p[q]);
        }
    });
}
int ref_core_state(void* core, float* x, float* y, float* z, double* pressure)
{
    return guarded([&] {
        ExternalAeroCore& c = *static_cast<RefCore*>(core)->core;
        CompositeCellMomentumState st;
        if (!c.download_cell_momentum_state(st)) throw std::runtime_error("reference core has no cell momentum");
        state_to(st, x, y, z);
        if (pressure)
        {
            std::vector<double> p;
            c.download_pressure(p);
            std::copy(p.begin(), p.end(), pressure);
        }
    });
}

}  // extern "C"
