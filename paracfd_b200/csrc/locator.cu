// locator.cu -- finest-brick point location on the device and headless slice sampling of the
// resident state.
//
// Location follows the reference's DeviceAmrLocator::locate_points (src/core/fluid/amr_fields.cu:
// 131-168, 200-249) in the same FP32 arithmetic: a point outside the domain box is not located;
// otherwise the levels are tried finest first, the point's brick coordinate at a level is
// floor((p - domain_lo) / (brick_size * h)), a brick that exists and is not covered takes the
// point, and the cell index inside it is floor((p - brick_origin) / h) clamped to the brick.  The
// reference finds the brick coordinate in a per-level open-addressed hash; here each level keeps a
// dense brick-index grid over the bounding box of its brick coordinates (one load per level).
//
// Slice sampling replaces the reference GUI's OpenGL slice (a graphics path): nu x nv points on a
// plane, each taking the value of the finest active cell that contains it, written to a buffer.
#include "locator.h"
#include "momentum.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace pcfd
{
    namespace
    {
        __global__ void locate_kernel(LocatorView v, const float* __restrict__ points, int count, int* __restrict__ out)
        {
            const int q = blockIdx.x * blockDim.x + threadIdx.x;
            if (q < count) locate_one(v, points[3 * q], points[3 * q + 1], points[3 * q + 2], out + 5 * q);
        }

        // field: 0 |v|, 1..3 v_x, v_y, v_z, 4 pressure (FP32 shadow)
        __global__ void slice_kernel(LocatorView v, double ox, double oy, double oz, double ux, double uy, double uz, double vx,
            double vy, double vz, int nu, int nv, int field, const uint8_t* __restrict__ active, const float* __restrict__ x,
            const float* __restrict__ y, const float* __restrict__ z, const float* __restrict__ p, float* __restrict__ out)
        {
            const int q = blockIdx.x * blockDim.x + threadIdx.x;
            if (q >= nu * nv) return;
            const int a = q % nu, b = q / nu;
            const double sa = (a + 0.5) / nu, sb = (b + 0.5) / nv;
            int where[5];
            locate_one(v, float(ox + sa * ux + sb * vx), float(oy + sa * uy + sb * vy), float(oz + sa * uz + sb * vz), where);
            float value = __int_as_float(0x7fc00000);   // NaN: no active cell
            if (where[0] >= 0)
            {
                const LocatorLevel lev = v.levels[where[0]];
                const int bs = v.brick_size;
                const int64_t dof = (int64_t(lev.slot0) + where[1]) * bs * bs * bs + (int64_t(where[4]) * bs + where[3]) * bs + where[2];
                if (active[dof])
                {
                    if (field == 0) value = sqrtf(x[dof] * x[dof] + y[dof] * y[dof] + z[dof] * z[dof]);
                    else if (field == 1) value = x[dof];
                    else if (field == 2) value = y[dof];
                    else if (field == 3) value = z[dof];
                    else value = p[dof];
                }
            }
            out[q] = value;
        }
    }

    struct LocatorState
    {
        DBuf<int> grid;
        DBuf<float4> record;
        DBuf<uint32_t> flags;
        DBuf<LocatorLevel> levels;
        LocatorView view{};
    };

    void build_locator(System& s, const pcfd_topology& t)
    {
        auto* L = new LocatorState();
        s.locator = L;
        const int levels = t.level_count;
        std::vector<LocatorLevel> host(static_cast<size_t>(levels));
        std::vector<int> grid;
        std::vector<float4> record;
        std::vector<uint32_t> flags;
        std::vector<size_t> grid_at(static_cast<size_t>(levels)), record_at(static_cast<size_t>(levels));
        int slot0 = 0;
        for (int l = 0; l < levels; ++l)
        {
            const pcfd_level& lev = t.levels[l];
            LocatorLevel& out = host[size_t(l)];
            int lo[3] = {std::numeric_limits<int>::max(), std::numeric_limits<int>::max(), std::numeric_limits<int>::max()};
            int hi[3] = {std::numeric_limits<int>::min(), std::numeric_limits<int>::min(), std::numeric_limits<int>::min()};
            for (int b = 0; b < lev.brick_count; ++b)
                for (int a = 0; a < 3; ++a)
                {
                    lo[a] = std::min(lo[a], lev.coord[3 * b + a]);
                    hi[a] = std::max(hi[a], lev.coord[3 * b + a]);
                }
            if (!lev.brick_count) lo[0] = lo[1] = lo[2] = 0, hi[0] = hi[1] = hi[2] = -1;
            out.min_x = lo[0]; out.min_y = lo[1]; out.min_z = lo[2];
            out.nx = hi[0] - lo[0] + 1; out.ny = hi[1] - lo[1] + 1; out.nz = hi[2] - lo[2] + 1;
            const int64_t cells = int64_t(out.nx) * out.ny * out.nz;
            require(cells <= int64_t(1) << 30, "locator: brick lattice of a level too large");
            grid_at[size_t(l)] = grid.size();
            grid.resize(grid.size() + size_t(cells), -1);
            int* g = grid.data() + grid_at[size_t(l)];
            for (int b = 0; b < lev.brick_count; ++b)
            {
                const int64_t at = (int64_t(lev.coord[3 * b + 2] - lo[2]) * out.ny + (lev.coord[3 * b + 1] - lo[1])) * out.nx +
                                   (lev.coord[3 * b] - lo[0]);
                require(g[at] < 0, "locator: two bricks share a coordinate");
                g[at] = b;
            }
            record_at[size_t(l)] = record.size();
            for (int b = 0; b < lev.brick_count; ++b)
            {
                record.push_back(make_float4(float(lev.origin[3 * b]), float(lev.origin[3 * b + 1]), float(lev.origin[3 * b + 2]),
                                             float(lev.h)));
                flags.push_back(lev.flags[b]);
            }
            out.brick_count = lev.brick_count;
            out.slot0 = slot0;
            out.h = float(lev.h);
            slot0 += lev.brick_count;
        }
        L->grid.upload(grid);
        L->record.upload(record);
        L->flags.upload(flags);
        for (int l = 0; l < levels; ++l)
        {
            host[size_t(l)].grid = L->grid.p + grid_at[size_t(l)];
            host[size_t(l)].record = L->record.p + record_at[size_t(l)];
            host[size_t(l)].flags = L->flags.p + record_at[size_t(l)];
        }
        L->levels.upload(host);
        LocatorView& v = L->view;
        v.levels = L->levels.p;
        v.level_count = levels;
        v.brick_size = t.brick_size;
        for (int a = 0; a < 3; ++a) { v.lo[a] = float(t.domain_lo[a]); v.hi[a] = float(t.domain_hi[a]); }
    }

    const LocatorView& locator_view(const System& s)
    {
        require(s.locator != nullptr, "locator not built");
        return static_cast<const LocatorState*>(s.locator)->view;
    }

    void destroy_locator(System& s)
    {
        delete static_cast<LocatorState*>(s.locator);
        s.locator = nullptr;
    }

    void locate_points(System& s, const float* points, int count, int* out)
    {
        require(s.locator != nullptr, "locator not built");
        if (count <= 0) return;
        const LocatorState& L = *static_cast<LocatorState*>(s.locator);
        locate_kernel<<<blocks_for(count), kThreads, 0, launch_stream(s)>>>(L.view, points, count, out);
        cuda_check(cudaGetLastError(), "locate points");
    }

    void sample_slice(System& s, const double origin[3], const double edge_u[3], const double edge_v[3], int nu, int nv, int field,
                      float* device_out)
    {
        require(s.locator != nullptr, "locator not built");
        require(nu > 0 && nv > 0 && int64_t(nu) * nv <= (int64_t(1) << 28), "slice: 1..2^28 samples");
        require(field >= 0 && field <= 4, "slice: field must be 0..4");
        const LocatorState& L = *static_cast<LocatorState*>(s.locator);
        Momentum& m = momentum_of(s);
        slice_kernel<<<blocks_for(int64_t(nu) * nv), kThreads, 0, launch_stream(s)>>>(
            L.view, origin[0], origin[1], origin[2], edge_u[0], edge_u[1], edge_u[2], edge_v[0], edge_v[1], edge_v[2], nu, nv, field,
            s.active, m.x, m.y, m.z, s.pressure32, device_out);
        cuda_check(cudaGetLastError(), "slice sampling");
    }
}
