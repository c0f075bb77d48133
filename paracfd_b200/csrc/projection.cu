// projection.cu -- aperture/volume-weighted divergence, projection RHS and the aperture-weighted
// gradient flux correction of every face kind (regular brick faces, 2:1 coarse/fine tiles, EB
// apertures, WLS non-orthogonal terms).
//
// Semantics: composite_amr_divergence_cpu / composite_amr_projection_rhs_cpu /
// composite_amr_correct_fluxes_cpu (reference src/core/fluid/amr_pressure.cpp:479-496) and the
// device bridge DeviceCompositeAmrProjection (src/core/fluid/amr_pressure.cu:255-351, 2021-2095).
// FP32 face velocities; geometry (areas, volumes, WLS weights) and every flux sum stay FP64, and
// each corrected face is rounded to FP32 once.  The reference's float atomics for the 2:1 group
// means are replaced by a deterministic per-group gather.
#include "pcfd_internal.h"

#include <algorithm>
#include <map>
#include <unordered_map>

namespace pcfd
{
    namespace
    {
        __device__ inline float face_value(const float* u, const float* v, const float* w, int bs, int axis, int64_t slot, int i, int j, int k)
        {
            return axis == 0 ? u[u_face(bs, slot, i, j, k)] : (axis == 1 ? v[v_face(bs, slot, i, j, k)] : w[w_face(bs, slot, i, j, k)]);
        }
        __device__ inline float* face_ptr(float* u, float* v, float* w, int bs, int axis, int64_t slot, int i, int j, int k)
        {
            return axis == 0 ? u + u_face(bs, slot, i, j, k) : (axis == 1 ? v + v_face(bs, slot, i, j, k) : w + w_face(bs, slot, i, j, k));
        }

        // Net outward integrated flux of every regular cell, gather form (one writer per cell).
        __global__ void structured_integrated_flux_kernel(const int* __restrict__ brick_list, int brick_count, int bs,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const uint32_t* __restrict__ flags,
            const double* __restrict__ level_h, const uint8_t* __restrict__ active, const uint8_t* __restrict__ cut,
            const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w, double* __restrict__ integrated)
        {
            const int c3 = bs * bs * bs;
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(brick_count) * c3) return;
            const int slot = brick_list[int(work) / c3], local = int(work) % c3;
            const int i = local % bs, j = (local / bs) % bs, k = local / (bs * bs);
            const int64_t a = int64_t(slot) * c3 + local;
            if (!active[a]) { integrated[a] = 0.0; return; }
            const double h = level_h[brick_level[slot]], area = h * h;
            double net = 0.0;
            for (int axis = 0; axis < 3; ++axis)
            {
                int q[3] = {i, j, k};
                int64_t upper = -1;
                if (++q[axis] < bs) upper = int64_t(slot) * c3 + (q[2] * bs + q[1]) * bs + q[0];
                else
                {
                    const int n = nbr[slot * 6 + 2 * axis + 1];
                    if (n >= 0) { q[axis] = 0; upper = int64_t(n) * c3 + (q[2] * bs + q[1]) * bs + q[0]; }
                }
                if (upper >= 0 && active[upper] && !(cut[a] & (1u << axis)))
                {
                    int f[3] = {i, j, k};
                    ++f[axis];
                    net += double(face_value(u, v, w, bs, axis, slot, f[0], f[1], f[2])) * area;
                }
                q[0] = i; q[1] = j; q[2] = k;
                int64_t lower = -1;
                int lower_slot = slot;
                if (--q[axis] >= 0) lower = int64_t(slot) * c3 + (q[2] * bs + q[1]) * bs + q[0];
                else
                {
                    lower_slot = nbr[slot * 6 + 2 * axis];
                    if (lower_slot >= 0) { q[axis] = bs - 1; lower = int64_t(lower_slot) * c3 + (q[2] * bs + q[1]) * bs + q[0]; }
                }
                if (lower >= 0 && active[lower] && !(cut[lower] & (1u << axis)))
                {
                    int f[3] = {q[0], q[1], q[2]};
                    ++f[axis];
                    net -= double(face_value(u, v, w, bs, axis, lower_slot, f[0], f[1], f[2])) * area;
                }
            }
            if ((flags[slot] & PCFD_BRICK_XMIN) && i == 0) net -= double(u[u_face(bs, slot, 0, j, k)]) * area;
            if ((flags[slot] & PCFD_BRICK_XMAX) && i == bs - 1) net += double(u[u_face(bs, slot, bs, j, k)]) * area;
            integrated[a] = net;
        }

        // The same integrated flux for 8^3 bricks, one CTA per non-covered brick (two cells per
        // thread): the brick's active and cut bytes and its neighbour slots staged in shared
        // memory, 32-bit index arithmetic, and the per-cell terms added in the order above, so the
        // result is bit-identical.
        __global__ void __launch_bounds__(256) brick_integrated_flux_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const uint32_t* __restrict__ flags,
            const double* __restrict__ level_h, const uint8_t* __restrict__ active, const uint8_t* __restrict__ cut,
            const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w, double* __restrict__ integrated)
        {
            constexpr int bs = 8, c3 = 512;
            __shared__ uint8_t act[c3], cm[c3];
            __shared__ int nb[6];
            const int slot = brick_list[blockIdx.x];
            const int64_t first = int64_t(slot) * c3;
            if (threadIdx.x < 6) nb[threadIdx.x] = nbr[slot * 6 + threadIdx.x];
            for (int c = threadIdx.x; c < c3; c += 256)
            {
                act[c] = active[first + c];
                cm[c] = cut[first + c];
            }
            __syncthreads();
            const double h = level_h[brick_level[slot]], area = h * h;
            const uint32_t fl = flags[slot];
            const float* comp[3] = {u, v, w};
            for (int half = 0; half < 2; ++half)
            {
                const int local = threadIdx.x + 256 * half;
                const int i = local & 7, j = (local >> 3) & 7, k = local >> 6;
                const int64_t a = first + local;
                if (!act[local]) { integrated[a] = 0.0; continue; }
                const int ijk[3] = {i, j, k};
                const int stride[3] = {1, 8, 64};
                double net = 0.0;
                for (int axis = 0; axis < 3; ++axis)
                {
                    // + face (a -> upper)
                    bool upper_active = false;
                    if (ijk[axis] < bs - 1) upper_active = act[local + stride[axis]];
                    else if (nb[2 * axis + 1] >= 0) upper_active = active[int64_t(nb[2 * axis + 1]) * c3 + local - (bs - 1) * stride[axis]];
                    if (upper_active && !(cm[local] & (1u << axis)))
                    {
                        int f[3] = {i, j, k};
                        ++f[axis];
                        net += double(comp[axis][axis == 0 ? u_face(bs, slot, f[0], f[1], f[2])
                                                           : (axis == 1 ? v_face(bs, slot, f[0], f[1], f[2]) : w_face(bs, slot, f[0], f[1], f[2]))]) * area;
                    }
                    // - face (lower -> a), read from the lower cell's brick
                    int lower_slot = -1, lower_local = 0;
                    bool lower_active = false;
                    uint8_t lower_cut = 0;
                    if (ijk[axis] > 0)
                    {
                        lower_slot = slot;
                        lower_local = local - stride[axis];
                        lower_active = act[lower_local];
                        lower_cut = cm[lower_local];
                    }
                    else if (nb[2 * axis] >= 0)
                    {
                        lower_slot = nb[2 * axis];
                        lower_local = local + (bs - 1) * stride[axis];
                        const int64_t lq = int64_t(lower_slot) * c3 + lower_local;
                        lower_active = active[lq];
                        lower_cut = cut[lq];
                    }
                    if (lower_slot >= 0 && lower_active && !(lower_cut & (1u << axis)))
                    {
                        int f[3] = {lower_local & 7, (lower_local >> 3) & 7, lower_local >> 6};
                        ++f[axis];
                        net -= double(comp[axis][axis == 0 ? u_face(bs, lower_slot, f[0], f[1], f[2])
                                                           : (axis == 1 ? v_face(bs, lower_slot, f[0], f[1], f[2])
                                                                        : w_face(bs, lower_slot, f[0], f[1], f[2]))]) * area;
                    }
                }
                if ((fl & PCFD_BRICK_XMIN) && i == 0) net -= double(u[u_face(bs, slot, 0, j, k)]) * area;
                if ((fl & PCFD_BRICK_XMAX) && i == bs - 1) net += double(u[u_face(bs, slot, bs, j, k)]) * area;
                integrated[a] = net;
            }
        }

        __global__ void zero_tail_kernel(double* x, int64_t begin, int64_t end)
        {
            const int64_t q = begin + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q < end) x[q] = 0.0;
        }

        __global__ void special_integrated_flux_kernel(const int* __restrict__ incident_dof, const int* __restrict__ incident_offset,
            const int* __restrict__ incident_edge, const int8_t* __restrict__ incident_sign, int incident_dofs,
            const double* __restrict__ area, const float* __restrict__ velocity, double* __restrict__ integrated)
        {
            const int node = blockIdx.x * blockDim.x + threadIdx.x;
            if (node >= incident_dofs) return;
            double sum = 0.0;
            for (int q = incident_offset[node]; q < incident_offset[node + 1]; ++q)
            {
                const int e = incident_edge[q];
                sum += double(incident_sign[q]) * (double(velocity[e]) * area[e]);
            }
            integrated[incident_dof[node]] += sum;
        }

        __global__ void normalize_kernel(const double* __restrict__ integrated, const double* __restrict__ volume,
            const uint8_t* __restrict__ active, double rho_over_dt, float* __restrict__ divergence, double* __restrict__ rhs, int64_t n)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= n) return;
            if (active[q] && volume[q] > 0.0)
            {
                divergence[q] = float(integrated[q] / volume[q]);
                if (rhs) rhs[q] = -rho_over_dt * integrated[q];
            }
            else
            {
                divergence[q] = 0.0f;
                if (rhs) rhs[q] = 0.0;
            }
        }

        // u_f -= (dt/rho) (p_b - p_a)/h on every open regular face, mirrored into the neighbour
        // brick's copy of a shared face; outlet face: u += (dt/rho) p_a / (h/2).
        template <int kBS>
        __global__ void structured_correction_kernel(const int* __restrict__ brick_list, int brick_count, int bs_arg,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const uint32_t* __restrict__ flags,
            const double* __restrict__ level_h, const uint8_t* __restrict__ active, const uint8_t* __restrict__ cut,
            const double* __restrict__ p, double scale, int outlet, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            const int c3 = bs * bs * bs;
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(brick_count) * c3) return;
            const int slot = brick_list[int(work) / c3], local = int(work) % c3;
            const int i = local % bs, j = (local / bs) % bs, k = local / (bs * bs);
            const int64_t a = int64_t(slot) * c3 + local;
            if (!active[a]) return;
            const double h = level_h[brick_level[slot]], pa = p[a];
            const uint8_t cm = cut[a];
            // every axis's upper cell, its activity and pressure and the face value are loaded
            // before any face is written, so the loads of the three axes are in flight together
            int64_t upper[3];
            int n[3];
            float* face[3];
            bool open[3];
            double pu[3];
            float fv[3];
#pragma unroll
            for (int axis = 0; axis < 3; ++axis)
            {
                int q[3] = {i, j, k};
                upper[axis] = -1;
                n[axis] = -1;
                if (++q[axis] < bs) upper[axis] = int64_t(slot) * c3 + (q[2] * bs + q[1]) * bs + q[0];
                else
                {
                    n[axis] = nbr[slot * 6 + 2 * axis + 1];
                    if (n[axis] >= 0) { q[axis] = 0; upper[axis] = int64_t(n[axis]) * c3 + (q[2] * bs + q[1]) * bs + q[0]; }
                }
                int f[3] = {i, j, k};
                ++f[axis];
                face[axis] = face_ptr(u, v, w, bs, axis, slot, f[0], f[1], f[2]);
                open[axis] = !(cm & (1u << axis)) && upper[axis] >= 0;
                pu[axis] = open[axis] ? p[upper[axis]] : 0.0;
                fv[axis] = open[axis] ? *face[axis] : 0.0f;
                open[axis] = open[axis] && active[upper[axis]];
            }
#pragma unroll
            for (int axis = 0; axis < 3; ++axis)
            {
                if (!open[axis]) continue;
                const float corrected = float(double(fv[axis]) - scale * (pu[axis] - pa) / h);
                *face[axis] = corrected;
                if (n[axis] >= 0)
                {
                    int m[3] = {i, j, k};
                    m[axis] = 0;
                    *face_ptr(u, v, w, bs, axis, n[axis], m[0], m[1], m[2]) = corrected;
                }
            }
            if (outlet && (flags[slot] & PCFD_BRICK_XMAX) && i == bs - 1)
            {
                float* f = u + u_face(bs, slot, bs, j, k);
                *f = float(double(*f) + scale * pa / (0.5 * h));
            }
        }

        __global__ void gradient_kernel(const int* __restrict__ dof, const int* __restrict__ offset, const int* __restrict__ neighbour,
            const double* __restrict__ weight, const double* __restrict__ p, double* __restrict__ gradient, int nodes)
        {
            const int node = blockIdx.x * blockDim.x + threadIdx.x;
            if (node >= nodes) return;
            const double centre = p[dof[node]];
            double gx = 0, gy = 0, gz = 0;
            for (int q = offset[node]; q < offset[node + 1]; ++q)
            {
                const double d = p[neighbour[q]] - centre;
                gx += weight[3 * q] * d;
                gy += weight[3 * q + 1] * d;
                gz += weight[3 * q + 2] * d;
            }
            gradient[3 * node] = gx;
            gradient[3 * node + 1] = gy;
            gradient[3 * node + 2] = gz;
        }

        __device__ inline double skew_derivative(const double* gradient, int ln, int un, const double* corr, double uw)
        {
            if (ln < 0 || un < 0) return 0.0;
            const double lw = 1.0 - uw;
            double d = 0.0;
            for (int c = 0; c < 3; ++c) d += corr[c] * (lw * gradient[3 * ln + c] + uw * gradient[3 * un + c]);
            return d;
        }

        __global__ void regular_correction_kernel(const int64_t* __restrict__ face, const int64_t* __restrict__ mirror,
            const int8_t* __restrict__ axis, const int* __restrict__ lower, const int* __restrict__ upper,
            const int* __restrict__ lower_node, const int* __restrict__ upper_node, const double* __restrict__ delta,
            const double* __restrict__ correction, const double* __restrict__ upper_weight, const double* __restrict__ gradient,
            const double* __restrict__ p, double scale, int count, float* u, float* v, float* w)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= count) return;
            const double derivative = delta[e] * (p[upper[e]] - p[lower[e]]) +
                                      skew_derivative(gradient, lower_node[e], upper_node[e], correction + 3 * e, upper_weight[e]);
            float* values = axis[e] == 0 ? u : (axis[e] == 1 ? v : w);
            const float corrected = float(double(values[face[e]]) - scale * derivative);
            values[face[e]] = corrected;
            if (mirror[e] >= 0) values[mirror[e]] = corrected;
        }

        __global__ void special_correction_kernel(const int* __restrict__ lower, const int* __restrict__ upper,
            const double* __restrict__ factor, const int* __restrict__ lower_node, const int* __restrict__ upper_node,
            const double* __restrict__ correction, const double* __restrict__ upper_weight, const double* __restrict__ gradient,
            const uint8_t* __restrict__ active, const double* __restrict__ p, double scale, int count, float* velocity)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= count) return;
            const int a = lower[e], b = upper[e];
            if (!active[a] || !active[b]) return;
            double derivative = (p[b] - p[a]) * factor[e];
            if (gradient) derivative += skew_derivative(gradient, lower_node[e], upper_node[e], correction + 3 * e, upper_weight[e]);
            velocity[e] = float(double(velocity[e]) - scale * derivative);
        }

        // 2:1 tiles: fine face <- tile velocity; coarse face <- area-weighted mean of its tiles.
        __global__ void coarse_fine_scatter_kernel(const int* __restrict__ group_offset, const int* __restrict__ group_member,
            const int64_t* __restrict__ group_face, const int8_t* __restrict__ group_axis, const int64_t* __restrict__ fine_face,
            const int8_t* __restrict__ axis, const double* __restrict__ area, const float* __restrict__ velocity, int groups,
            float* u, float* v, float* w)
        {
            const int g = blockIdx.x * blockDim.x + threadIdx.x;
            if (g >= groups) return;
            double sum = 0.0, total = 0.0;
            for (int q = group_offset[g]; q < group_offset[g + 1]; ++q)
            {
                const int e = group_member[q];
                const float value = velocity[e];
                float* faces = axis[e] == 0 ? u : (axis[e] == 1 ? v : w);
                faces[fine_face[e]] = value;
                sum += area[e] * double(value);
                total += area[e];
            }
            if (total > 0.0)
            {
                float* faces = group_axis[g] == 0 ? u : (group_axis[g] == 1 ? v : w);
                faces[group_face[g]] = float(sum / total);
            }
        }

        __global__ void convert_pressure_kernel(const double* p, float* p32, int64_t n)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q < n) p32[q] = float(p[q]);
        }
    }

    void build_projection(System& s, const pcfd_topology& t)
    {
        const int cf = t.coarse_fine.count, eb = t.embedded.count, nc = cf + eb;
        s.cf_count = cf;
        s.eb_count = eb;
        std::vector<int> lower(nc), upper(nc), lnode(nc), unode(nc);
        std::vector<double> area(nc), factor(nc), corr(size_t(nc) * 3), weight(nc);
        for (int e = 0; e < nc; ++e)
        {
            const pcfd_connections& c = e < cf ? t.coarse_fine : t.embedded;
            const int q = e < cf ? e : e - cf;
            const bool forward = c.direction[q] > 0;
            lower[e] = forward ? c.coarse_dof[q] : c.fine_dof[q];
            upper[e] = forward ? c.fine_dof[q] : c.coarse_dof[q];
            area[e] = c.open_area[q];
            const double f = c.orthogonal_gradient_factor[q];
            factor[e] = f > 0 ? f : (c.normal_distance[q] > 0 ? 1.0 / c.normal_distance[q] : 0.0);
            lnode[e] = c.lower_gradient_node[q];
            unode[e] = c.upper_gradient_node[q];
            for (int a = 0; a < 3; ++a) corr[3 * e + a] = c.nonorthogonal_correction[3 * q + a];
            weight[e] = c.upper_gradient_weight[q];
        }
        s.special_lower.upload(lower); s.special_upper.upload(upper); s.special_area.upload(area);
        s.special_factor.upload(factor); s.special_lower_node.upload(lnode); s.special_upper_node.upload(unode);
        s.special_correction.upload(corr); s.special_upper_weight.upload(weight);
        s.special.alloc(size_t(nc));

        struct Incident { int dof, edge; int8_t sign; };
        std::vector<Incident> inc;
        for (int e = 0; e < nc; ++e)
        {
            const int a = lower[e], b = upper[e];
            if (a < 0 || b < 0 || a >= s.S || b >= s.S || a == b || !t.active[a] || !t.active[b]) continue;
            inc.push_back({a, e, 1});
            inc.push_back({b, e, -1});
        }
        std::sort(inc.begin(), inc.end(), [](const Incident& a, const Incident& b) {
            if (a.dof != b.dof) return a.dof < b.dof;
            if (a.edge != b.edge) return a.edge < b.edge;
            return a.sign < b.sign;
        });
        std::vector<int> idof, ioff, iedge;
        std::vector<int8_t> isign;
        for (size_t q = 0; q < inc.size(); ++q)
        {
            if (q == 0 || inc[q].dof != inc[q - 1].dof) { idof.push_back(inc[q].dof); ioff.push_back(int(q)); }
            iedge.push_back(inc[q].edge);
            isign.push_back(inc[q].sign);
        }
        ioff.push_back(int(inc.size()));
        s.special_incident_dofs = int(idof.size());
        s.special_incident_dof.upload(idof); s.special_incident_offset.upload(ioff);
        s.special_incident_edge.upload(iedge); s.special_incident_sign.upload(isign);

        // regular correction face addresses
        const int bs = s.bs;
        const pcfd_regular_corrections& rc = t.regular;
        std::vector<int64_t> face(rc.count), mirror(rc.count, -1);
        std::vector<int8_t> raxis(rc.count);
        for (int e = 0; e < rc.count; ++e)
        {
            const int l = rc.level[e], brick = rc.brick[e], ax = rc.axis[e];
            const int i = rc.ijk[3 * e], j = rc.ijk[3 * e + 1], k = rc.ijk[3 * e + 2];
            const int64_t slot = s.level_slot0[l] + brick;
            face[e] = axis_face(bs, ax, slot, i, j, k);
            raxis[e] = int8_t(ax);
            const int coordinate = ax == 0 ? i : (ax == 1 ? j : k);
            if (coordinate == bs)
            {
                const int nb = t.levels[l].neighbors[brick * 6 + 2 * ax + 1];
                if (nb >= 0)
                {
                    int m[3] = {i, j, k};
                    m[ax] = 0;
                    mirror[e] = axis_face(bs, ax, s.level_slot0[l] + nb, m[0], m[1], m[2]);
                }
            }
        }
        s.reg_face.upload(face); s.reg_mirror.upload(mirror); s.reg_axis.upload(raxis);

        // coarse/fine tile groups (key: coarse DOF, axis, side), reference amr_pressure.cu:1752-1767
        if (cf)
        {
            const int c3 = s.bs3;
            auto face_address = [&](int dof, int ax, bool positive) -> int64_t {
                if (dof < 0 || dof >= s.structured) throw Error(PCFD_INVALID_ARG, "coarse/fine DOF has no regular face");
                const int slot = dof / c3, local = dof % c3;
                int c[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
                c[ax] += positive ? 1 : 0;
                return axis_face(bs, ax, slot, c[0], c[1], c[2]);
            };
            std::vector<int64_t> fine_face(cf), group_face;
            std::vector<int8_t> cf_axis(cf), group_axis;
            std::vector<int> group_of(cf);
            std::unordered_map<uint64_t, int> groups;
            for (int e = 0; e < cf; ++e)
            {
                const int ax = t.coarse_fine.axis[e], dir = t.coarse_fine.direction[e];
                fine_face[e] = face_address(t.coarse_fine.fine_dof[e], ax, dir < 0);
                cf_axis[e] = int8_t(ax);
                const uint64_t key = (uint64_t(uint32_t(t.coarse_fine.coarse_dof[e])) << 3) | (uint64_t(ax) << 1) | uint64_t(dir > 0);
                auto found = groups.find(key);
                int id;
                if (found == groups.end())
                {
                    id = int(group_face.size());
                    groups.emplace(key, id);
                    group_face.push_back(face_address(t.coarse_fine.coarse_dof[e], ax, dir > 0));
                    group_axis.push_back(int8_t(ax));
                }
                else id = found->second;
                group_of[e] = id;
            }
            s.cf_groups = int(group_face.size());
            std::vector<int> goff(size_t(s.cf_groups) + 1, 0), gmem(cf);
            for (int e = 0; e < cf; ++e) ++goff[group_of[e] + 1];
            for (int g = 0; g < s.cf_groups; ++g) goff[g + 1] += goff[g];
            std::vector<int> cursor = goff;
            for (int e = 0; e < cf; ++e) gmem[cursor[group_of[e]]++] = e;
            s.cf_fine_face.upload(fine_face); s.cf_axis.upload(cf_axis); s.cf_group_face.upload(group_face);
            s.cf_group_axis.upload(group_axis); s.cf_group_offset.upload(goff); s.cf_group_member.upload(gmem);
        }
    }

    void launch_integrated_flux(System& s)
    {
        if (s.active_bricks)
        {
            if (s.bs == 8)
                brick_integrated_flux_kernel<<<s.active_bricks, 256, 0, launch_stream(s)>>>(
                    s.active_brick_list, s.brick_level, s.brick_nbr, s.brick_flags, s.d_level_h, s.active, s.cut_face_mask, s.u, s.v,
                    s.w, s.integrated);
            else
                structured_integrated_flux_kernel<<<blocks_for(int64_t(s.active_bricks) * s.bs3), kThreads, 0, launch_stream(s)>>>(
                    s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr, s.brick_flags, s.d_level_h, s.active,
                    s.cut_face_mask, s.u, s.v, s.w, s.integrated);
        }
        if (s.S > s.structured)
            zero_tail_kernel<<<blocks_for(s.S - s.structured), kThreads, 0, launch_stream(s)>>>(s.integrated, s.structured, s.S);
        if (s.special_incident_dofs)
            special_integrated_flux_kernel<<<blocks_for(s.special_incident_dofs), kThreads, 0, launch_stream(s)>>>(
                s.special_incident_dof, s.special_incident_offset, s.special_incident_edge, s.special_incident_sign,
                s.special_incident_dofs, s.special_area, s.special, s.integrated);
        cuda_check(cudaGetLastError(), "integrated flux");
    }

    void launch_normalize(System& s, double rho_over_dt, bool with_rhs)
    {
        normalize_kernel<<<blocks_for(s.S), kThreads, 0, launch_stream(s)>>>(s.integrated, s.volume, s.active, rho_over_dt, s.divergence,
                                                                    with_rhs ? s.rhs.p : nullptr, s.S);
        cuda_check(cudaGetLastError(), "normalize divergence");
    }

    void launch_correct_fluxes(System& s, double rho, double dt)
    {
        const double scale = dt / rho;
        if (s.active_bricks)
            (s.bs == 8 ? structured_correction_kernel<8> : structured_correction_kernel<0>)<<<blocks_for(int64_t(s.active_bricks) * s.bs3), kThreads, 0, launch_stream(s)>>>(
                s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr, s.brick_flags, s.d_level_h, s.active,
                s.cut_face_mask, s.pressure, scale, s.outlet ? 1 : 0, s.u, s.v, s.w);
        IrregularOperator& o = s.irr;
        if (o.gradient_nodes)
            gradient_kernel<<<blocks_for(o.gradient_nodes), kThreads, 0, launch_stream(s)>>>(o.grad_dof, o.grad_offset, o.grad_neighbour,
                                                                                   o.grad_weight, s.pressure, o.gradient, o.gradient_nodes);
        if (o.regular_count)
            regular_correction_kernel<<<blocks_for(o.regular_count), kThreads, 0, launch_stream(s)>>>(
                s.reg_face, s.reg_mirror, s.reg_axis, o.reg_lower, o.reg_upper, o.reg_lower_node, o.reg_upper_node, o.reg_delta,
                o.reg_correction, o.reg_upper_weight, o.gradient_nodes ? o.gradient.p : nullptr, s.pressure, scale, o.regular_count,
                s.u, s.v, s.w);
        const int nc = s.cf_count + s.eb_count;
        if (nc)
            special_correction_kernel<<<blocks_for(nc), kThreads, 0, launch_stream(s)>>>(
                s.special_lower, s.special_upper, s.special_factor, s.special_lower_node, s.special_upper_node, s.special_correction,
                s.special_upper_weight, o.gradient_nodes ? o.gradient.p : nullptr, s.active, s.pressure, scale, nc, s.special);
        if (s.cf_groups)
            coarse_fine_scatter_kernel<<<blocks_for(s.cf_groups), kThreads, 0, launch_stream(s)>>>(
                s.cf_group_offset, s.cf_group_member, s.cf_group_face, s.cf_group_axis, s.cf_fine_face, s.cf_axis, s.special_area,
                s.special, s.cf_groups, s.u, s.v, s.w);
        cuda_check(cudaGetLastError(), "correct fluxes");
    }

    // ==================================================================================
    // conservation statistics of the resident divergence (ExternalAeroCore::conservation_stats,
    // external_aero_core.cpp:347-356): over active DOFs with positive volume, the largest
    // |divergence| and its control volume (first DOF on ties), the largest |divergence * V|,
    // sum |divergence * V|, sum divergence * V and the volume-weighted RMS divergence.  FP64 sums
    // over a fixed grid with fixed-order trees: deterministic run to run.
    // ==================================================================================
    namespace
    {
        constexpr int kStatBlocks = 592, kStatThreads = 256, kStatSums = 5;
        struct StatMax { double value; int64_t index; };
        __device__ inline StatMax better(StatMax a, StatMax b)
        {
            if (b.value > a.value || (b.value == a.value && b.index >= 0 && (a.index < 0 || b.index < a.index))) return b;
            return a;
        }

        // sums: [max |div V|, sum |div V|, sum div V, sum div^2 V, sum V]
        __global__ void __launch_bounds__(kStatThreads) conservation_partial_kernel(const float* __restrict__ divergence,
            const double* __restrict__ volume, const uint8_t* __restrict__ active, int64_t n, double* __restrict__ partial,
            double* __restrict__ partial_max, int64_t* __restrict__ partial_index)
        {
            __shared__ double sums[kStatSums][kStatThreads];
            __shared__ StatMax best[kStatThreads];
            double s[kStatSums] = {0, 0, 0, 0, 0};
            StatMax m{0.0, -1};
            for (int64_t q = int64_t(blockIdx.x) * kStatThreads + threadIdx.x; q < n; q += int64_t(gridDim.x) * kStatThreads)
            {
                if (!active[q] || !(volume[q] > 0.0)) continue;
                const double value = double(divergence[q]), v = volume[q], integrated = value * v;
                m = better(m, StatMax{fabs(value), q});
                s[0] = fmax(s[0], fabs(integrated));
                s[1] += fabs(integrated);
                s[2] += integrated;
                s[3] += value * value * v;
                s[4] += v;
            }
            for (int k = 0; k < kStatSums; ++k) sums[k][threadIdx.x] = s[k];
            best[threadIdx.x] = m;
            __syncthreads();
            for (int stride = kStatThreads / 2; stride > 0; stride >>= 1)
            {
                if (threadIdx.x < stride)
                {
                    sums[0][threadIdx.x] = fmax(sums[0][threadIdx.x], sums[0][threadIdx.x + stride]);
                    for (int k = 1; k < kStatSums; ++k) sums[k][threadIdx.x] += sums[k][threadIdx.x + stride];
                    best[threadIdx.x] = better(best[threadIdx.x], best[threadIdx.x + stride]);
                }
                __syncthreads();
            }
            if (threadIdx.x == 0)
            {
                for (int k = 0; k < kStatSums; ++k) partial[blockIdx.x * kStatSums + k] = sums[k][0];
                partial_max[blockIdx.x] = best[0].value;
                partial_index[blockIdx.x] = best[0].index;
            }
        }

        // out: [max |div|, rms, worst volume, max |div V|, sum |div V|, sum div V]
        __global__ void __launch_bounds__(kStatThreads) conservation_final_kernel(const double* __restrict__ partial,
            const double* __restrict__ partial_max, const int64_t* __restrict__ partial_index, int blocks,
            const double* __restrict__ volume, double* __restrict__ out)
        {
            __shared__ double sums[kStatSums][kStatThreads];
            __shared__ StatMax best[kStatThreads];
            double s[kStatSums] = {0, 0, 0, 0, 0};
            StatMax m{0.0, -1};
            for (int b = threadIdx.x; b < blocks; b += kStatThreads)
            {
                s[0] = fmax(s[0], partial[b * kStatSums]);
                for (int k = 1; k < kStatSums; ++k) s[k] += partial[b * kStatSums + k];
                m = better(m, StatMax{partial_max[b], partial_index[b]});
            }
            for (int k = 0; k < kStatSums; ++k) sums[k][threadIdx.x] = s[k];
            best[threadIdx.x] = m;
            __syncthreads();
            for (int stride = kStatThreads / 2; stride > 0; stride >>= 1)
            {
                if (threadIdx.x < stride)
                {
                    sums[0][threadIdx.x] = fmax(sums[0][threadIdx.x], sums[0][threadIdx.x + stride]);
                    for (int k = 1; k < kStatSums; ++k) sums[k][threadIdx.x] += sums[k][threadIdx.x + stride];
                    best[threadIdx.x] = better(best[threadIdx.x], best[threadIdx.x + stride]);
                }
                __syncthreads();
            }
            if (threadIdx.x == 0)
            {
                out[0] = best[0].value;
                out[1] = sums[4][0] > 0.0 ? sqrt(sums[3][0] / sums[4][0]) : 0.0;
                out[2] = best[0].index >= 0 ? volume[best[0].index] : 0.0;
                out[3] = sums[0][0];
                out[4] = sums[1][0];
                out[5] = sums[2][0];
            }
        }
    }

    void conservation_stats(System& s, double out[6])
    {
        DBuf<double>& scratch = s.conservation_scratch;
        DBuf<int64_t>& where = s.conservation_index;
        if (!scratch.p)
        {
            scratch.alloc(size_t(kStatBlocks) * (kStatSums + 1) + 8);
            where.alloc(size_t(kStatBlocks));
        }
        const int grid = std::max(1, std::min(kStatBlocks, int((int64_t(s.S) + kStatThreads - 1) / kStatThreads)));
        double* partial = scratch.p;
        double* partial_max = partial + size_t(kStatBlocks) * kStatSums;
        double* result = partial_max + kStatBlocks;
        conservation_partial_kernel<<<grid, kStatThreads, 0, launch_stream(s)>>>(s.divergence, s.volume, s.active, s.S, partial,
                                                                                 partial_max, where);
        conservation_final_kernel<<<1, kStatThreads, 0, launch_stream(s)>>>(partial, partial_max, where, grid, s.volume, result);
        cuda_check(cudaGetLastError(), "conservation statistics");
        cuda_check(cudaMemcpyAsync(out, result, 6 * sizeof(double), cudaMemcpyDeviceToHost, s.stream), "conservation readback");
        cuda_check(cudaStreamSynchronize(s.stream), "conservation readback");
    }

    void launch_convert_pressure(System& s)
    {
        convert_pressure_kernel<<<blocks_for(s.S), kThreads, 0, launch_stream(s)>>>(s.pressure, s.pressure32, s.S);
        cuda_check(cudaGetLastError(), "convert pressure");
    }
}
