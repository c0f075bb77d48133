// mac_apertures.cu -- transport of the compact embedded-boundary face velocities in the staggered
// MAC momentum mode (DeviceCompositeAmrProjection::transport_embedded_apertures without the
// molecular fabric wall, src/core/fluid/amr_pressure.cu:352-540, 1868-1911; preprocessing of the
// projection's constructor, :1766-1791).
//
// The embedded (cut) apertures are not MAC faces of any brick: each is an edge of a graph whose
// nodes are the pressure DOFs on either side.  One step:
//   1. node velocities per component: area-weighted means of the incident apertures of that axis
//      and of the regular MAC faces around the node ("carriers");
//   2. a least-squares gradient per node and component from the node-mean differences along the
//      edges (per-node 3x3 pseudoinverse set up once in FP64, applied in FP32);
//   3. per aperture a bounded MUSCL update along its chain of same-axis apertures (upstream,
//      upstream-of-upstream, downstream found once at setup by nearest face centroid), a
//      tangential correction from the node gradients, and the pair's Smagorinsky diffusion rate;
//   4. conservative pairwise diffusion of node momentum (dual masses area / (2 gradient factor))
//      along the edges, scattered back to the apertures and, half each, to the carrier faces.
// All accumulations are FP32 atomics, as in the reference, so sums can differ in their last bits
// from run to run; the test tolerance says so.
#include "pcfd_internal.h"
#include "pseudoinverse3.h"

#include <algorithm>
#include <cstring>
#include <cmath>
#include <limits>
#include <unordered_map>
#include <vector>

namespace pcfd
{
    namespace
    {
        // compact-aperture helpers (the reference's detail:: functions, amr_pressure.h:21-97)
        __device__ inline float cmin(float a, float b) { return a < b ? a : b; }
        __device__ inline float cmax(float a, float b) { return a > b ? a : b; }
        __device__ inline float cabs(float a) { return a < 0.0f ? -a : a; }
        __device__ inline float cminmod(float a, float b) { return a * b <= 0.0f ? 0.0f : (cabs(a) < cabs(b) ? a : b); }
        __device__ inline float strain_squared(const float* g)
        {
            const float sxx = g[0], syy = g[4], szz = g[8];
            const float sxy = 0.5f * (g[1] + g[3]), sxz = 0.5f * (g[2] + g[6]), syz = 0.5f * (g[5] + g[7]);
            return 2.0f * (sxx * sxx + syy * syy + szz * szz + 2.0f * (sxy * sxy + sxz * sxz + syz * syz));
        }
        // bounded MUSCL update along the aperture chain (complete chain), else the first-order
        // update from the upstream node; clamped to the values it was built from
        __device__ inline float chain_update(float current, float lower, float upper, float up, float up2, float down, float courant,
                                             float diffusion, bool complete)
        {
            float lo = cmin(current, cmin(lower, upper)), hi = cmax(current, cmax(lower, upper));
            float advected;
            if (complete)
            {
                const float delta = current - up;
                const float slope = cminmod(delta, down - current), up_slope = cminmod(up - up2, delta);
                advected = current - courant * delta - 0.5f * courant * (1.0f - courant) * (slope - up_slope);
                lo = cmin(lo, cmin(up, cmin(up2, down)));
                hi = cmax(hi, cmax(up, cmax(up2, down)));
            }
            else
            {
                const float node_up = current >= 0.0f ? lower : upper;
                advected = current + courant * (node_up - current);
            }
            const float candidate = advected + diffusion * (lower + upper - 2.0f * current);
            return cmax(lo, cmin(hi, candidate));
        }
        __device__ inline float tangential_update(float normal, float current, float lower, float upper, const float* advector,
                                                  const float* gradient, int component, float dt)
        {
            float rate = 0.0f;
            for (int a = 0; a < 3; ++a)
                if (a != component) rate += advector[a] * gradient[component * 3 + a];
            const float candidate = normal - dt * rate;
            const float lo = cmin(normal, cmin(current, cmin(lower, upper))), hi = cmax(normal, cmax(current, cmax(lower, upper)));
            return cmax(lo, cmin(hi, candidate));
        }

        // ---- graph arrays on the device ----
        struct ApertureGraph
        {
            int edges, nodes, carriers, offset;          // offset: first embedded slot of the special arrays
            const int *node_a, *node_b, *negative, *positive;
            const int8_t *axis, *direction;              // per embedded edge
            const float *area, *factor, *length;         // FP32 as the reference's device copies
            const float *ls_displacement, *ls_weight, *inverse;
            const int* carrier_node;
            const int64_t* carrier_face;                 // face index in the component's array
            const int8_t* carrier_axis;
            const float *carrier_area, *carrier_mass;
            float *sum, *weight, *gradient, *scratch, *rate, *advected, *delta, *count;
        };
        struct FaceFields
        {
            float* c[3];
        };

        __global__ void carrier_mean_kernel(ApertureGraph g, FaceFields f)
        {
            const int q = blockIdx.x * blockDim.x + threadIdx.x;
            if (q >= g.carriers) return;
            const int slot = g.carrier_node[q] * 3 + g.carrier_axis[q];
            atomicAdd(g.sum + slot, g.carrier_area[q] * f.c[g.carrier_axis[q]][g.carrier_face[q]]);
            atomicAdd(g.weight + slot, g.carrier_area[q]);
        }
        __global__ void aperture_mean_kernel(ApertureGraph g, const float* velocity)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int c = g.axis[e], a = g.node_a[e] * 3 + c, b = g.node_b[e] * 3 + c;
            const float weighted = g.area[e] * velocity[g.offset + e];
            atomicAdd(g.sum + a, weighted);
            atomicAdd(g.sum + b, weighted);
            atomicAdd(g.weight + a, g.area[e]);
            atomicAdd(g.weight + b, g.area[e]);
        }
        __global__ void gradient_rhs_kernel(ApertureGraph g)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int a = g.node_a[e], b = g.node_b[e];
            for (int c = 0; c < 3; ++c)
            {
                const float wa = g.weight[a * 3 + c], wb = g.weight[b * 3 + c], w = g.ls_weight[e * 3 + c];
                if (!(wa > 0.0f && wb > 0.0f && w > 0.0f)) continue;
                const float delta = g.sum[b * 3 + c] / wb - g.sum[a * 3 + c] / wa;
                for (int d = 0; d < 3; ++d)
                {
                    const float contribution = w * g.ls_displacement[e * 9 + c * 3 + d] * delta;
                    atomicAdd(g.gradient + a * 9 + c * 3 + d, contribution);
                    atomicAdd(g.gradient + b * 9 + c * 3 + d, contribution);
                }
            }
        }
        __global__ void gradient_solve_kernel(ApertureGraph g)
        {
            const int node = blockIdx.x * blockDim.x + threadIdx.x;
            if (node >= g.nodes) return;
            for (int c = 0; c < 3; ++c)
            {
                float rhs[3];
                for (int q = 0; q < 3; ++q) rhs[q] = g.gradient[node * 9 + c * 3 + q];
                for (int row = 0; row < 3; ++row)
                {
                    float value = 0.0f;
                    for (int col = 0; col < 3; ++col) value += g.inverse[node * 27 + c * 9 + row * 3 + col] * rhs[col];
                    g.gradient[node * 9 + c * 3 + row] = value;
                }
            }
        }
        __global__ void aperture_transport_kernel(ApertureGraph g, const float* velocity, float dt, float nu, float cs)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int c = g.axis[e], first = g.node_a[e], second = g.node_b[e];
            const int lower = g.direction[e] > 0 ? first : second, upper = g.direction[e] > 0 ? second : first;
            const float current = velocity[g.offset + e];
            const float lw = g.weight[lower * 3 + c], uw = g.weight[upper * 3 + c];
            const float lower_value = lw > 0.0f ? g.sum[lower * 3 + c] / lw : current;
            const float upper_value = uw > 0.0f ? g.sum[upper * 3 + c] / uw : current;
            const float d = fmaxf(g.length[e], 1e-12f);
            float gradient[9], advector[3];
            for (int vc = 0; vc < 3; ++vc)
            {
                const float aw = g.weight[lower * 3 + vc], bw = g.weight[upper * 3 + vc];
                float value = 0.0f, samples = 0.0f;
                if (aw > 0.0f) { value += g.sum[lower * 3 + vc] / aw; samples += 1.0f; }
                if (bw > 0.0f) { value += g.sum[upper * 3 + vc] / bw; samples += 1.0f; }
                advector[vc] = samples > 0.0f ? value / samples : 0.0f;
            }
            advector[c] = current;
            for (int q = 0; q < 9; ++q) gradient[q] = 0.5f * (g.gradient[lower * 9 + q] + g.gradient[upper * 9 + q]);
            const float normal_rate = fabsf(upper_value - lower_value) / d;
            const float strain = fmaxf(sqrtf(fmaxf(0.0f, strain_squared(gradient))), normal_rate);
            const float length = cs * d, eddy = length * length * strain;
            g.rate[e] = (nu + eddy) / (d * d);
            const float courant = fminf(1.0f, fabsf(current) * dt / d);
            const bool positive = current >= 0.0f;
            const int up = positive ? g.negative[e] : g.positive[e], down = positive ? g.positive[e] : g.negative[e];
            const int up2 = up >= 0 ? (positive ? g.negative[up] : g.positive[up]) : -1;
            const bool complete = up >= 0 && up2 >= 0 && down >= 0;
            const float vu = complete ? velocity[g.offset + up] : current, vu2 = complete ? velocity[g.offset + up2] : current,
                        vd = complete ? velocity[g.offset + down] : current;
            const float normal = chain_update(current, lower_value, upper_value, vu, vu2, vd, courant, 0.0f, complete);
            g.scratch[e] = tangential_update(normal, current, lower_value, upper_value, advector, gradient, c, dt);
        }
        __global__ void dual_momentum_kernel(ApertureGraph g)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int c = g.axis[e], a = g.node_a[e] * 3 + c, b = g.node_b[e] * 3 + c;
            const float mass = 0.5f * g.area[e] / fmaxf(g.factor[e], 1e-12f), weighted = mass * g.advected[e];
            atomicAdd(g.sum + a, weighted);
            atomicAdd(g.sum + b, weighted);
            atomicAdd(g.weight + a, mass);
            atomicAdd(g.weight + b, mass);
        }
        __global__ void carrier_momentum_kernel(ApertureGraph g, FaceFields f)
        {
            const int q = blockIdx.x * blockDim.x + threadIdx.x;
            if (q >= g.carriers) return;
            const int slot = g.carrier_node[q] * 3 + g.carrier_axis[q];
            const float m = 0.5f * g.carrier_mass[q], u = f.c[g.carrier_axis[q]][g.carrier_face[q]];
            atomicAdd(g.sum + slot, m * u);
            atomicAdd(g.weight + slot, m);
        }
        __global__ void neighbour_count_kernel(ApertureGraph g)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int a = g.node_a[e], b = g.node_b[e];
            for (int c = 0; c < 3; ++c)
            {
                const int sa = a * 3 + c, sb = b * 3 + c;
                if (g.weight[sa] > 0.0f && g.weight[sb] > 0.0f)
                {
                    atomicAdd(g.count + sa, 1.0f);
                    atomicAdd(g.count + sb, 1.0f);
                }
            }
        }
        __global__ void exchange_kernel(ApertureGraph g, float dt)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int a = g.node_a[e], b = g.node_b[e];
            for (int c = 0; c < 3; ++c)
            {
                const int sa = a * 3 + c, sb = b * 3 + c;
                const float ma = g.weight[sa], mb = g.weight[sb];
                if (!(ma > 0.0f && mb > 0.0f)) continue;
                const float degree = fmaxf(1.0f, fmaxf(g.count[sa], g.count[sb]));
                const float theta = fminf(0.25f, dt * g.rate[e]) / degree;
                const float ua = g.sum[sa] / ma, ub = g.sum[sb] / mb;
                const float transfer = theta * (ma * mb / (ma + mb)) * (ub - ua);
                atomicAdd(g.delta + sa, transfer);
                atomicAdd(g.delta + sb, -transfer);
            }
        }
        __global__ void apply_to_apertures_kernel(ApertureGraph g, float* velocity)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int c = g.axis[e], sa = g.node_a[e] * 3 + c, sb = g.node_b[e] * 3 + c;
            const float wa = g.weight[sa], wb = g.weight[sb];
            const float du_a = wa > 0.0f ? g.delta[sa] / wa : 0.0f, du_b = wb > 0.0f ? g.delta[sb] / wb : 0.0f;
            velocity[g.offset + e] = g.advected[e] + 0.5f * (du_a + du_b);
        }
        __global__ void apply_to_carriers_kernel(ApertureGraph g, FaceFields f)
        {
            const int q = blockIdx.x * blockDim.x + threadIdx.x;
            if (q >= g.carriers) return;
            const int slot = g.carrier_node[q] * 3 + g.carrier_axis[q];
            if (!(g.weight[slot] > 0.0f)) return;
            atomicAdd(f.c[g.carrier_axis[q]] + g.carrier_face[q], 0.5f * g.delta[slot] / g.weight[slot]);
        }
    }

    namespace
    {
        // coarse/fine special velocities from the fine side's regular face (the reference's
        // sync_coarse_fine_from_fields, amr_pressure.cu:340-342, 1864-1867)
        __global__ void sync_coarse_fine_kernel(const int64_t* face, const int8_t* axis, int count, FaceFields f, float* special)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e < count) special[e] = f.c[axis[e]][face[e]];
        }
        // max over [0, n) of |value[i]| / divisor[i] (divisor null: 1), as a non-negative float
        // kept in the bits of an unsigned int (monotone for non-negative floats)
        __global__ void max_ratio_kernel(const float* value, const float* divisor, int64_t n, unsigned int* out)
        {
            __shared__ float shared[8];
            float m = 0.0f;
            for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
                m = fmaxf(m, divisor ? fabsf(value[i]) / fmaxf(divisor[i], 1e-12f) : fabsf(value[i]));
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0) shared[threadIdx.x >> 5] = m;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                for (int w = 1; w < int(blockDim.x >> 5); ++w) m = fmaxf(m, shared[w]);
                atomicMax(out, __float_as_uint(m));
            }
        }
    }

    // ---- MAC smooth fabric wall (DeviceCompositeAmrProjection::apply_smooth_fabric_wall_model,
    // amr_pressure.cu:418-535, 1913-1960; preprocessing :1796-1830): node velocities of the wall
    // cells from their apertures (dual masses) and regular carrier faces, the Spalding-law wall
    // drag k (I - n n^T) per surface patch, an implicit 3x3 Cholesky solve per node, and the
    // velocity change scattered half to each aperture endpoint and carrier face.
    namespace
    {
        struct WallGraph
        {
            int nodes, patches, carriers, edges, offset;
            const int *edge_a, *edge_b, *patch_node, *carrier_node;
            const int8_t *axis, *carrier_axis;
            const float *area, *factor, *normal, *patch_area, *distance, *carrier_mass;
            const int64_t* carrier_face;
            float *sum, *weight, *delta, *matrix, *coefficient;
        };
        __device__ inline float wall_friction_velocity(float speed, float distance, float nu)
        {
            // Spalding's law as u+ y+(u+) = Re_y, 36 bisections of u+ on [0, 80]
            if (!(speed > 0.0f) || !(distance > 0.0f) || !(nu > 0.0f)) return 0.0f;
            const float reynolds = speed * distance / nu, kappa = 0.41f, coefficient = 0.1185998568f;
            float lower = 0.0f, upper = 80.0f;
            for (int it = 0; it < 36; ++it)
            {
                const float uplus = 0.5f * (lower + upper), xk = kappa * uplus, x2 = xk * xk, x3 = x2 * xk;
                const float remainder = xk < 0.5f ? x2 * x2 * (1.0f / 24.0f + xk * (1.0f / 120.0f) + x2 * (1.0f / 720.0f))
                                                  : expf(xk) - 1.0f - xk - 0.5f * x2 - x3 * (1.0f / 6.0f);
                const float yplus = uplus + coefficient * remainder;
                if (uplus * yplus < reynolds) lower = uplus;
                else upper = uplus;
            }
            return speed / fmaxf(0.5f * (lower + upper), 1e-12f);
        }
        __global__ void wall_aperture_velocity_kernel(WallGraph g, const float* velocity)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int c = g.axis[e], a = g.edge_a[e], b = g.edge_b[e];
            const float mass = 0.5f * g.area[e] / fmaxf(g.factor[e], 1e-12f), weighted = mass * velocity[g.offset + e];
            if (a >= 0) { atomicAdd(g.sum + a * 3 + c, weighted); atomicAdd(g.weight + a * 3 + c, mass); }
            if (b >= 0) { atomicAdd(g.sum + b * 3 + c, weighted); atomicAdd(g.weight + b * 3 + c, mass); }
        }
        __global__ void wall_carrier_velocity_kernel(WallGraph g, FaceFields f)
        {
            const int q = blockIdx.x * blockDim.x + threadIdx.x;
            if (q >= g.carriers) return;
            const int slot = g.carrier_node[q] * 3 + g.carrier_axis[q];
            const float m = 0.5f * g.carrier_mass[q], u = f.c[g.carrier_axis[q]][g.carrier_face[q]];
            atomicAdd(g.sum + slot, m * u);
            atomicAdd(g.weight + slot, m);
        }
        __global__ void wall_matrix_kernel(WallGraph g, float nu)
        {
            const int p = blockIdx.x * blockDim.x + threadIdx.x;
            if (p >= g.patches) return;
            const int target = g.patch_node[p];
            float velocity[3];
            for (int c = 0; c < 3; ++c)
            {
                const int slot = target * 3 + c;
                velocity[c] = g.weight[slot] > 0.0f ? g.sum[slot] / g.weight[slot] : 0.0f;
            }
            const float* n = g.normal + 3 * p;
            const float un = velocity[0] * n[0] + velocity[1] * n[1] + velocity[2] * n[2];
            const float tangent[3] = {velocity[0] - un * n[0], velocity[1] - un * n[1], velocity[2] - un * n[2]};
            const float speed = sqrtf(fmaxf(0.0f, tangent[0] * tangent[0] + tangent[1] * tangent[1] + tangent[2] * tangent[2]));
            float k = 0.0f;
            if (speed > 0.0f)
            {
                const float friction = wall_friction_velocity(speed, g.distance[p], nu);
                k = g.patch_area[p] * friction * friction / speed;
            }
            g.coefficient[p] = k;
            if (!(k > 0.0f)) return;
            float* a = g.matrix + 6 * target;
            atomicAdd(a, k * (1.0f - n[0] * n[0]));
            atomicAdd(a + 1, -k * n[0] * n[1]);
            atomicAdd(a + 2, -k * n[0] * n[2]);
            atomicAdd(a + 3, k * (1.0f - n[1] * n[1]));
            atomicAdd(a + 4, -k * n[1] * n[2]);
            atomicAdd(a + 5, k * (1.0f - n[2] * n[2]));
        }
        // I + dt M^-1/2 K M^-1/2 is symmetric positive definite (every patch adds k (I - n n^T),
        // k >= 0): a Cholesky solve gives a dissipative wall impulse without a wall time-step limit
        __global__ void wall_solve_kernel(WallGraph g, float dt)
        {
            const int node = blockIdx.x * blockDim.x + threadIdx.x;
            if (node >= g.nodes) return;
            const float* k = g.matrix + 6 * node;
            float root[3], old[3], rhs[3];
            for (int c = 0; c < 3; ++c)
            {
                const int slot = node * 3 + c;
                root[c] = sqrtf(fmaxf(0.0f, g.weight[slot]));
                old[c] = g.weight[slot] > 0.0f ? g.sum[slot] / g.weight[slot] : 0.0f;
                rhs[c] = root[c] * old[c];
            }
            auto scaled = [&](int a, int b, float value) { return root[a] > 0.0f && root[b] > 0.0f ? dt * value / (root[a] * root[b]) : 0.0f; };
            const float a00 = 1.0f + scaled(0, 0, k[0]), a01 = scaled(0, 1, k[1]), a02 = scaled(0, 2, k[2]), a11 = 1.0f + scaled(1, 1, k[3]),
                        a12 = scaled(1, 2, k[4]), a22 = 1.0f + scaled(2, 2, k[5]);
            const float l00 = sqrtf(a00), l10 = a01 / l00, l20 = a02 / l00;
            const float l11 = sqrtf(a11 - l10 * l10), l21 = (a12 - l20 * l10) / l11;
            const float l22 = sqrtf(a22 - l20 * l20 - l21 * l21);
            const float y0 = rhs[0] / l00, y1 = (rhs[1] - l10 * y0) / l11, y2 = (rhs[2] - l20 * y0 - l21 * y1) / l22;
            const float s2 = y2 / l22, s1 = (y1 - l21 * s2) / l11, s0 = (y0 - l10 * s1 - l20 * s2) / l00;
            const float solved[3] = {s0, s1, s2};
            for (int c = 0; c < 3; ++c) g.delta[node * 3 + c] = root[c] > 0.0f ? solved[c] / root[c] - old[c] : 0.0f;
        }
        __global__ void wall_apply_apertures_kernel(WallGraph g, float* velocity)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= g.edges) return;
            const int c = g.axis[e], a = g.edge_a[e], b = g.edge_b[e];
            float delta = 0.0f;
            if (a >= 0) delta += 0.5f * g.delta[a * 3 + c];
            if (b >= 0) delta += 0.5f * g.delta[b * 3 + c];
            velocity[g.offset + e] += delta;
        }
        __global__ void wall_apply_carriers_kernel(WallGraph g, FaceFields f)
        {
            const int q = blockIdx.x * blockDim.x + threadIdx.x;
            if (q >= g.carriers) return;
            atomicAdd(f.c[g.carrier_axis[q]] + g.carrier_face[q], 0.5f * g.delta[g.carrier_node[q] * 3 + g.carrier_axis[q]]);
        }
    }

    // ---- setup (the projection constructor's EB transport preprocessing) ----
    struct ApertureState
    {
        int edges = 0, nodes = 0, carriers = 0, offset = 0;
        DBuf<int64_t> cf_face;                  // per coarse/fine connection: the fine side's regular face
        DBuf<int8_t> cf_axis;
        DBuf<unsigned int> maximum;
        // MAC smooth wall
        int wall_nodes = 0, wall_patches = 0, wall_carriers = 0;
        DBuf<int> wall_edge_a, wall_edge_b, wall_patch_node, wall_carrier_node;
        DBuf<int8_t> wall_carrier_axis;
        DBuf<float> wall_normal, wall_area, wall_distance, wall_carrier_mass;
        DBuf<int64_t> wall_carrier_face;
        DBuf<float> wall_sum, wall_weight, wall_delta, wall_matrix, wall_coefficient;
        WallGraph wall_graph() const
        {
            return WallGraph{wall_nodes, wall_patches, wall_carriers, edges, offset, wall_edge_a, wall_edge_b, wall_patch_node,
                             wall_carrier_node, axis, wall_carrier_axis, area, factor, wall_normal, wall_area, wall_distance,
                             wall_carrier_mass, wall_carrier_face, wall_sum, wall_weight, wall_delta, wall_matrix, wall_coefficient};
        }
        DBuf<int> node_a, node_b, negative, positive, carrier_node;
        DBuf<int8_t> axis, direction, carrier_axis;
        DBuf<float> area, factor, length, ls_displacement, ls_weight, inverse, carrier_area, carrier_mass;
        DBuf<int64_t> carrier_face;
        DBuf<float> sum, weight, gradient, scratch, rate, advected, delta, count;
        ApertureGraph graph() const
        {
            return ApertureGraph{edges, nodes, carriers, offset, node_a, node_b, negative, positive, axis, direction, area, factor, length,
                                 ls_displacement, ls_weight, inverse, carrier_node, carrier_face, carrier_axis, carrier_area, carrier_mass,
                                 sum, weight, gradient, scratch, rate, advected, delta, count};
        }
    };

    namespace
    {
        // the two-point gradient factor of a compact connection (the projection's own rule)
        double gradient_factor(const pcfd_connections& c, int e)
        {
            const double f = c.orthogonal_gradient_factor[e];
            return f > 0 ? f : (c.normal_distance[e] > 0 ? 1.0 / c.normal_distance[e] : 0.0);
        }
    }

    namespace
    {
        // structured location of a DOF: level, brick, slot; false for EB fragments
        bool locate_dof(const pcfd_topology& t, int dof, int& level, int& brick, int& local, int& slot)
        {
            const int c3 = t.brick_size * t.brick_size * t.brick_size;
            for (int l = 0, at = 0; l < t.level_count; at += t.levels[l].brick_count, ++l)
            {
                const int begin = t.levels[l].level_offset, end = begin + t.levels[l].brick_count * c3;
                if (dof >= begin && dof < end)
                {
                    level = l;
                    brick = (dof - begin) / c3;
                    local = (dof - begin) % c3;
                    slot = at + brick;
                    return true;
                }
            }
            return false;
        }
        // the regular faces between a structured DOF and its active same-level neighbours that are
        // not cut: f(axis, sign, other DOF, face index) for each
        template <class F> void regular_faces(const pcfd_topology& t, int dof, F&& f)
        {
            int level, brick, local, slot;
            if (!locate_dof(t, dof, level, brick, local, slot)) return;
            const pcfd_level& lev = t.levels[level];
            if (lev.flags[brick] & PCFD_BRICK_COVERED) return;
            const int bs = t.brick_size, c3 = bs * bs * bs;
            const int ijk[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
            for (int a = 0; a < 3; ++a)
                for (int sign = -1; sign <= 1; sign += 2)
                {
                    int c[3] = {ijk[0], ijk[1], ijk[2]}, other = -1;
                    c[a] += sign;
                    if (c[a] >= 0 && c[a] < bs) other = lev.level_offset + brick * c3 + (c[2] * bs + c[1]) * bs + c[0];
                    else
                    {
                        const int ob = lev.neighbors[brick * 6 + 2 * a + (sign > 0)];
                        if (ob >= 0 && !(lev.flags[ob] & PCFD_BRICK_COVERED))
                        {
                            c[a] = sign > 0 ? 0 : bs - 1;
                            other = lev.level_offset + ob * c3 + (c[2] * bs + c[1]) * bs + c[0];
                        }
                    }
                    if (other < 0 || !t.active[other]) continue;
                    const int lower = sign > 0 ? dof : other;
                    if (t.cut_face_mask[lower] & (1u << a)) continue;
                    int fc[3] = {ijk[0], ijk[1], ijk[2]};
                    fc[a] += sign > 0;
                    f(a, sign, other, axis_face(bs, a, slot, fc[0], fc[1], fc[2]), level, brick, ijk);
                }
        }

        void build_wall(ApertureState& st, const pcfd_topology& t)
        {
            const pcfd_surface_patches& P = t.patches;
            if (!P.count) return;
            std::unordered_map<int, int> node_of;
            std::vector<int> node_dof;
            auto wall_node = [&](int dof) {
                if (dof < 0 || dof >= t.storage_size || !t.active[dof]) return;
                if (node_of.count(dof)) return;
                node_of.emplace(dof, int(node_dof.size()));
                node_dof.push_back(dof);
            };
            for (int p = 0; p < P.count; ++p) { wall_node(P.plus_dof[p]); wall_node(P.minus_dof[p]); }
            std::vector<int> patch_node;
            std::vector<float> normal, area, distance;
            for (int p = 0; p < P.count; ++p)
            {
                const double* nv = P.normal + 3 * p;
                const double len = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
                require(P.area[p] >= 0 && len > 0, "invalid fabric wall patch geometry");
                const double un[3] = {nv[0] / len, nv[1] / len, nv[2] / len};
                for (int dof : {P.plus_dof[p], P.minus_dof[p]})
                {
                    auto it = node_of.find(dof);
                    if (it == node_of.end()) continue;
                    const double volume = t.volume[dof];
                    double d = 0.0;
                    for (int k = 0; k < 3; ++k) d += (t.centroid[3 * size_t(dof) + k] - P.centroid[3 * p + k]) * un[k];
                    d = std::abs(d);
                    const double scale = std::cbrt(std::max(0.0, volume));
                    require(volume > 0 && d > std::max(1e-14, scale * 1e-10), "fabric wall patch has zero same-side centroid distance");
                    patch_node.push_back(it->second);
                    for (int k = 0; k < 3; ++k) normal.push_back(float(un[k]));
                    area.push_back(float(P.area[p]));
                    distance.push_back(float(d));
                }
            }
            const pcfd_connections& eb = t.embedded;
            std::vector<int> ea(size_t(std::max(1, eb.count)), -1), eb_(size_t(std::max(1, eb.count)), -1);
            for (int e = 0; e < eb.count; ++e)
            {
                auto a = node_of.find(eb.coarse_dof[e]), b = node_of.find(eb.fine_dof[e]);
                if (a != node_of.end()) ea[size_t(e)] = a->second;
                if (b != node_of.end()) eb_[size_t(e)] = b->second;
            }
            std::vector<int> carrier_node;
            std::vector<int64_t> carrier_face;
            std::vector<int8_t> carrier_axis;
            std::vector<float> carrier_mass;
            for (int n = 0; n < int(node_dof.size()); ++n)
            {
                const int dof = node_dof[size_t(n)];
                regular_faces(t, dof, [&](int a, int, int other, int64_t face, int, int, const int*) {
                    carrier_node.push_back(n);
                    carrier_face.push_back(face);
                    carrier_axis.push_back(int8_t(a));
                    carrier_mass.push_back(float(0.5 * (t.volume[dof] + t.volume[other])));
                });
            }
            st.wall_nodes = int(node_dof.size());
            st.wall_patches = int(patch_node.size());
            st.wall_carriers = int(carrier_node.size());
            st.wall_edge_a.upload(ea);
            st.wall_edge_b.upload(eb_);
            st.wall_patch_node.upload(patch_node.empty() ? std::vector<int>(1, 0) : patch_node);
            st.wall_normal.upload(normal.empty() ? std::vector<float>(3, 0.0f) : normal);
            st.wall_area.upload(area.empty() ? std::vector<float>(1, 0.0f) : area);
            st.wall_distance.upload(distance.empty() ? std::vector<float>(1, 0.0f) : distance);
            st.wall_carrier_node.upload(carrier_node.empty() ? std::vector<int>(1, 0) : carrier_node);
            st.wall_carrier_face.upload(carrier_face.empty() ? std::vector<int64_t>(1, 0) : carrier_face);
            st.wall_carrier_axis.upload(carrier_axis.empty() ? std::vector<int8_t>(1, 0) : carrier_axis);
            st.wall_carrier_mass.upload(carrier_mass.empty() ? std::vector<float>(1, 0.0f) : carrier_mass);
            const size_t n = size_t(std::max(1, st.wall_nodes));
            st.wall_sum.alloc(n * 3); st.wall_weight.alloc(n * 3); st.wall_delta.alloc(n * 3); st.wall_matrix.alloc(n * 6);
            st.wall_coefficient.alloc(size_t(std::max(1, st.wall_patches)));
        }
    }

    void build_apertures(System& s, const pcfd_topology& t)
    {
        auto* st = new ApertureState();
        s.apertures = st;
        const pcfd_connections& eb = t.embedded;
        const int E = eb.count, S = t.storage_size, bs = t.brick_size, c3 = bs * bs * bs;
        st->edges = E;
        st->offset = t.coarse_fine.count;
        st->maximum.alloc(1);
        {
            // the fine cell's face toward the coarse side (direction > 0: the coarse DOF is on the lower side)
            const pcfd_connections& cf = t.coarse_fine;
            std::vector<int64_t> face(size_t(std::max(1, cf.count)), 0);
            std::vector<int8_t> ax(size_t(std::max(1, cf.count)), 0);
            for (int e = 0; e < cf.count; ++e)
            {
                const int dof = cf.fine_dof[e], a = cf.axis[e];
                int level = -1, brick = 0, local = 0, slot0 = 0;
                for (int l = 0, at = 0; l < t.level_count; at += t.levels[l].brick_count, ++l)
                {
                    const int begin = t.levels[l].level_offset, end = begin + t.levels[l].brick_count * c3;
                    if (dof >= begin && dof < end) { level = l; brick = (dof - begin) / c3; local = (dof - begin) % c3; slot0 = at; break; }
                }
                require(level >= 0, "coarse/fine connection without a regular fine face");
                int f[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
                f[a] += cf.direction[e] < 0;
                face[size_t(e)] = axis_face(bs, a, slot0 + brick, f[0], f[1], f[2]);
                ax[size_t(e)] = int8_t(a);
            }
            st->cf_face.upload(face);
            st->cf_axis.upload(ax);
        }
        build_wall(*st, t);
        if (!E) return;
        struct V3 { double x[3] = {0, 0, 0}; };
        // graph nodes in order of first appearance
        std::unordered_map<int, int> node_of;
        std::vector<int> node_dof, na(static_cast<size_t>(E)), nb(static_cast<size_t>(E));
        auto node = [&](int dof) {
            auto it = node_of.find(dof);
            if (it != node_of.end()) return it->second;
            const int id = int(node_dof.size());
            node_of.emplace(dof, id);
            node_dof.push_back(dof);
            return id;
        };
        std::vector<float> length(static_cast<size_t>(E)), area(static_cast<size_t>(E)), factor(static_cast<size_t>(E));
        std::vector<int8_t> axis(static_cast<size_t>(E)), direction(static_cast<size_t>(E));
        for (int e = 0; e < E; ++e)
        {
            na[size_t(e)] = node(eb.coarse_dof[e]);
            nb[size_t(e)] = node(eb.fine_dof[e]);
            const double sa = std::cbrt(std::max(0.0, t.volume[eb.coarse_dof[e]])), sb = std::cbrt(std::max(0.0, t.volume[eb.fine_dof[e]]));
            length[size_t(e)] = float(std::max(eb.centre_distance[e], 0.5 * (sa + sb)));
            area[size_t(e)] = float(eb.open_area[e]);
            factor[size_t(e)] = float(gradient_factor(eb, e));
            axis[size_t(e)] = eb.axis[e];
            direction[size_t(e)] = eb.direction[e];
        }
        const int N = int(node_dof.size());
        st->nodes = N;
        // per node and component: weighted position of the velocity samples
        std::vector<V3> position(size_t(N) * 3);
        std::vector<double> sample_weight(size_t(N) * 3, 0.0);
        auto add_sample = [&](int n, int c, const double* p, double w) {
            V3& q = position[size_t(n) * 3 + c];
            for (int a = 0; a < 3; ++a) q.x[a] += p[a] * w;
            sample_weight[size_t(n) * 3 + c] += w;
        };
        for (int e = 0; e < E; ++e)
        {
            add_sample(na[size_t(e)], eb.axis[e], eb.face_centroid + 3 * e, eb.open_area[e]);
            add_sample(nb[size_t(e)], eb.axis[e], eb.face_centroid + 3 * e, eb.open_area[e]);
        }
        // same-axis aperture chains through shared nodes: the nearest face centroid that extends
        // the aperture in the required direction
        std::vector<std::vector<int>> incident(static_cast<size_t>(N));
        for (int e = 0; e < E; ++e)
        {
            incident[size_t(na[size_t(e)])].push_back(e);
            incident[size_t(nb[size_t(e)])].push_back(e);
        }
        auto lower_node = [&](int e) { return eb.direction[e] > 0 ? na[size_t(e)] : nb[size_t(e)]; };
        auto upper_node = [&](int e) { return eb.direction[e] > 0 ? nb[size_t(e)] : na[size_t(e)]; };
        auto extension = [&](int e, int shared, bool negative) {
            int best = -1;
            double best_distance = std::numeric_limits<double>::infinity();
            const int a = eb.axis[e];
            for (int cand : incident[size_t(shared)])
            {
                if (cand == e || eb.axis[cand] != a) continue;
                if (negative ? upper_node(cand) != shared : lower_node(cand) != shared) continue;
                const double delta = eb.face_centroid[3 * cand + a] - eb.face_centroid[3 * e + a];
                if (negative ? delta >= -1e-12 : delta <= 1e-12) continue;
                double d2 = 0.0;
                for (int k = 0; k < 3; ++k)
                {
                    const double dk = eb.face_centroid[3 * cand + k] - eb.face_centroid[3 * e + k];
                    d2 += dk * dk;
                }
                if (d2 < best_distance) { best_distance = d2; best = cand; }
            }
            return best;
        };
        std::vector<int> negative(static_cast<size_t>(E)), positive(static_cast<size_t>(E));
        for (int e = 0; e < E; ++e)
        {
            negative[size_t(e)] = extension(e, lower_node(e), true);
            positive[size_t(e)] = extension(e, upper_node(e), false);
        }
        // carriers: the regular MAC faces between a structured node and its active same-level
        // neighbours (not cut), with their velocity samples at the face position
        std::vector<int> carrier_node;
        std::vector<int64_t> carrier_face;
        std::vector<int8_t> carrier_axis;
        std::vector<float> carrier_area, carrier_mass;
        require(t.level_count <= 64, "aperture transport: at most 64 levels");
        int slot0_of_level[64] = {};
        for (int l = 1; l < t.level_count && l < 64; ++l) slot0_of_level[l] = slot0_of_level[l - 1] + t.levels[l - 1].brick_count;
        for (int n = 0; n < N; ++n)
        {
            const int dof = node_dof[size_t(n)];
            if (dof < 0 || dof >= S || !t.active[dof]) continue;
            int level = -1, brick = -1, local = -1;
            for (int l = 0; l < t.level_count; ++l)
            {
                const int begin = t.levels[l].level_offset, end = begin + t.levels[l].brick_count * c3;
                if (dof >= begin && dof < end) { level = l; brick = (dof - begin) / c3; local = (dof - begin) % c3; break; }
            }
            if (level < 0) continue;
            const pcfd_level& lev = t.levels[level];
            if (lev.flags[brick] & PCFD_BRICK_COVERED) continue;
            const int ijk[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
            const double h = lev.h;
            for (int a = 0; a < 3; ++a)
                for (int sign = -1; sign <= 1; sign += 2)
                {
                    int c[3] = {ijk[0], ijk[1], ijk[2]}, other = -1;
                    c[a] += sign;
                    if (c[a] >= 0 && c[a] < bs) other = lev.level_offset + brick * c3 + (c[2] * bs + c[1]) * bs + c[0];
                    else
                    {
                        const int ob = lev.neighbors[brick * 6 + 2 * a + (sign > 0)];
                        if (ob >= 0 && !(lev.flags[ob] & PCFD_BRICK_COVERED))
                        {
                            c[a] = sign > 0 ? 0 : bs - 1;
                            other = lev.level_offset + ob * c3 + (c[2] * bs + c[1]) * bs + c[0];
                        }
                    }
                    if (other < 0 || !t.active[other]) continue;
                    const int lower = sign > 0 ? dof : other;
                    if (t.cut_face_mask[lower] & (1u << a)) continue;
                    int f[3] = {ijk[0], ijk[1], ijk[2]};
                    f[a] += sign > 0;
                    carrier_node.push_back(n);
                    carrier_face.push_back(axis_face(bs, a, slot0_of_level[level] + brick, f[0], f[1], f[2]));
                    carrier_axis.push_back(int8_t(a));
                    carrier_area.push_back(float(h * h));
                    carrier_mass.push_back(float(0.5 * (t.volume[dof] + t.volume[other])));
                    double p[3];
                    for (int k = 0; k < 3; ++k) p[k] = lev.origin[3 * brick + k] + (ijk[k] + 0.5) * h;
                    p[a] = lev.origin[3 * brick + a] + (ijk[a] + (sign > 0 ? 1 : 0)) * h;
                    add_sample(n, a, p, h * h);
                }
        }
        // least-squares gradients: per edge and component the displacement between the two
        // nodes' mean sample positions, weighted by area / distance^2
        for (int q = 0; q < N * 3; ++q)
            if (sample_weight[size_t(q)] > 0)
                for (int k = 0; k < 3; ++k) position[size_t(q)].x[k] = position[size_t(q)].x[k] / sample_weight[size_t(q)];
        std::vector<float> ls_displacement(size_t(E) * 9, 0.0f), ls_weight(size_t(E) * 3, 0.0f), inverse(size_t(N) * 27, 0.0f);
        std::vector<double> normal(size_t(N) * 27, 0.0);
        for (int e = 0; e < E; ++e)
            for (int c = 0; c < 3; ++c)
            {
                const int a = na[size_t(e)], b = nb[size_t(e)];
                const size_t sa = size_t(a) * 3 + c, sb = size_t(b) * 3 + c;
                if (!(sample_weight[sa] > 0 && sample_weight[sb] > 0)) continue;
                double d[3], d2 = 0.0;
                for (int k = 0; k < 3; ++k) { d[k] = position[sb].x[k] - position[sa].x[k]; d2 += d[k] * d[k]; }
                if (!(d2 > 1e-20)) continue;
                const double w = eb.open_area[e] / d2;
                ls_weight[size_t(e) * 3 + c] = float(w);
                for (int k = 0; k < 3; ++k) ls_displacement[size_t(e) * 9 + c * 3 + k] = float(d[k]);
                for (int endpoint : {a, b})
                    for (int r = 0; r < 3; ++r)
                        for (int col = 0; col < 3; ++col) normal[size_t(endpoint) * 27 + c * 9 + r * 3 + col] += w * d[r] * d[col];
            }
        // inverses: modes below 1e-4 of the largest eigenvalue dropped (FP32 application)
        for (int n = 0; n < N; ++n)
            for (int c = 0; c < 3; ++c)
            {
                double inv[9];
                pseudoinverse3(normal.data() + size_t(n) * 27 + c * 9, inv, 16, 1e-4);
                for (int q = 0; q < 9; ++q) inverse[size_t(n) * 27 + c * 9 + q] = float(inv[q]);
            }
        st->carriers = int(carrier_node.size());
        st->node_a.upload(na); st->node_b.upload(nb); st->negative.upload(negative); st->positive.upload(positive);
        st->axis.upload(axis); st->direction.upload(direction);
        st->area.upload(area); st->factor.upload(factor); st->length.upload(length);
        st->ls_displacement.upload(ls_displacement); st->ls_weight.upload(ls_weight); st->inverse.upload(inverse);
        st->carrier_node.upload(carrier_node.empty() ? std::vector<int>(1, 0) : carrier_node);
        st->carrier_face.upload(carrier_face.empty() ? std::vector<int64_t>(1, 0) : carrier_face);
        st->carrier_axis.upload(carrier_axis.empty() ? std::vector<int8_t>(1, 0) : carrier_axis);
        st->carrier_area.upload(carrier_area.empty() ? std::vector<float>(1, 0.0f) : carrier_area);
        st->carrier_mass.upload(carrier_mass.empty() ? std::vector<float>(1, 0.0f) : carrier_mass);
        st->sum.alloc(size_t(N) * 3); st->weight.alloc(size_t(N) * 3); st->gradient.alloc(size_t(N) * 9);
        st->delta.alloc(size_t(N) * 3); st->count.alloc(size_t(N) * 3);
        st->scratch.alloc(size_t(E)); st->rate.alloc(size_t(E)); st->advected.alloc(size_t(E));
    }

    void destroy_apertures(System& s)
    {
        delete static_cast<ApertureState*>(s.apertures);
        s.apertures = nullptr;
    }

    // DeviceCompositeAmrProjection::transport_embedded_apertures(dt, nu, cs, false) on the
    // system's special and face velocities
    void mac_transport_apertures(System& s, float dt, float nu, float cs)
    {
        require(s.apertures != nullptr, "aperture transport not set up");
        ApertureState& st = *static_cast<ApertureState*>(s.apertures);
        if (!st.edges) return;
        const ApertureGraph g = st.graph();
        const FaceFields f{{s.u.p, s.v.p, s.w.p}};
        cudaStream_t stream = launch_stream(s);
        const size_t n3 = size_t(st.nodes) * 3 * sizeof(float);
        cuda_check(cudaMemsetAsync(st.sum.p, 0, n3, stream), "clear aperture sums");
        cuda_check(cudaMemsetAsync(st.weight.p, 0, n3, stream), "clear aperture weights");
        cuda_check(cudaMemsetAsync(st.gradient.p, 0, 3 * n3, stream), "clear aperture gradients");
        const int ge = blocks_for(st.edges), gc = blocks_for(std::max(1, st.carriers)), gn = blocks_for(st.nodes);
        if (st.carriers) carrier_mean_kernel<<<gc, kThreads, 0, stream>>>(g, f);
        aperture_mean_kernel<<<ge, kThreads, 0, stream>>>(g, s.special.p);
        gradient_rhs_kernel<<<ge, kThreads, 0, stream>>>(g);
        gradient_solve_kernel<<<gn, kThreads, 0, stream>>>(g);
        aperture_transport_kernel<<<ge, kThreads, 0, stream>>>(g, s.special.p, dt, nu, cs);
        // the transported state is kept; diffusion then exchanges node momentum pairwise
        cuda_check(cudaMemcpyAsync(st.advected.p, st.scratch.p, size_t(st.edges) * sizeof(float), cudaMemcpyDeviceToDevice, stream),
                   "keep transported apertures");
        cuda_check(cudaMemsetAsync(st.sum.p, 0, n3, stream), "clear aperture momentum");
        cuda_check(cudaMemsetAsync(st.weight.p, 0, n3, stream), "clear aperture masses");
        cuda_check(cudaMemsetAsync(st.delta.p, 0, n3, stream), "clear aperture deltas");
        cuda_check(cudaMemsetAsync(st.count.p, 0, n3, stream), "clear aperture neighbour counts");
        dual_momentum_kernel<<<ge, kThreads, 0, stream>>>(g);
        if (st.carriers) carrier_momentum_kernel<<<gc, kThreads, 0, stream>>>(g, f);
        neighbour_count_kernel<<<ge, kThreads, 0, stream>>>(g);
        exchange_kernel<<<ge, kThreads, 0, stream>>>(g, dt);
        apply_to_apertures_kernel<<<ge, kThreads, 0, stream>>>(g, s.special.p);
        if (st.carriers) apply_to_carriers_kernel<<<gc, kThreads, 0, stream>>>(g, f);
        cuda_check(cudaGetLastError(), "aperture transport");
    }

    void mac_sync_coarse_fine(System& s)
    {
        ApertureState& st = *static_cast<ApertureState*>(s.apertures);
        if (!st.offset) return;
        const FaceFields f{{s.u.p, s.v.p, s.w.p}};
        sync_coarse_fine_kernel<<<blocks_for(st.offset), kThreads, 0, launch_stream(s)>>>(st.cf_face, st.cf_axis, st.offset, f, s.special.p);
        cuda_check(cudaGetLastError(), "coarse/fine sync");
    }

    namespace
    {
        float device_max(System& s, unsigned int* slot, const float* value, const float* divisor, int64_t n)
        {
            cuda_check(cudaMemsetAsync(slot, 0, sizeof(unsigned int), s.stream), "clear maximum");
            if (n > 0)
                max_ratio_kernel<<<int(std::min<int64_t>(592, (n + kThreads - 1) / kThreads)), kThreads, 0, launch_stream(s)>>>(value, divisor, n, slot);
            unsigned int bits = 0;
            cuda_check(cudaMemcpyAsync(&bits, slot, sizeof(bits), cudaMemcpyDeviceToHost, s.stream), "read maximum");
            cuda_check(cudaStreamSynchronize(s.stream), "maximum");
            float out;
            std::memcpy(&out, &bits, sizeof(out));
            return out;
        }
    }

    // max |v| / transport length over the embedded apertures (max_embedded_cfl_rate)
    float mac_embedded_cfl_rate(System& s)
    {
        ApertureState& st = *static_cast<ApertureState*>(s.apertures);
        if (!st.edges) return 0.0f;
        return device_max(s, st.maximum, s.special.p + st.offset, st.length, st.edges);
    }
    float mac_max_special_speed(System& s)
    {
        ApertureState& st = *static_cast<ApertureState*>(s.apertures);
        return device_max(s, st.maximum, s.special.p, nullptr, int64_t(st.offset) + st.edges);
    }

    // DeviceCompositeAmrProjection::apply_smooth_fabric_wall_model (the MAC step's wall)
    void mac_smooth_wall(System& s, float dt, float nu)
    {
        ApertureState& st = *static_cast<ApertureState*>(s.apertures);
        require(dt > 0.0f && nu > 0.0f, "smooth fabric wall timestep/viscosity");
        if (!st.wall_nodes || !st.wall_patches) return;
        WallGraph g = st.wall_graph();
        const FaceFields f{{s.u.p, s.v.p, s.w.p}};
        cudaStream_t stream = launch_stream(s);
        const size_t n3 = size_t(st.wall_nodes) * 3 * sizeof(float);
        cuda_check(cudaMemsetAsync(st.wall_sum.p, 0, n3, stream), "clear wall sums");
        cuda_check(cudaMemsetAsync(st.wall_weight.p, 0, n3, stream), "clear wall weights");
        cuda_check(cudaMemsetAsync(st.wall_delta.p, 0, n3, stream), "clear wall deltas");
        cuda_check(cudaMemsetAsync(st.wall_matrix.p, 0, 2 * n3, stream), "clear wall matrices");
        if (st.edges) wall_aperture_velocity_kernel<<<blocks_for(st.edges), kThreads, 0, stream>>>(g, s.special.p);
        if (st.wall_carriers) wall_carrier_velocity_kernel<<<blocks_for(st.wall_carriers), kThreads, 0, stream>>>(g, f);
        wall_matrix_kernel<<<blocks_for(st.wall_patches), kThreads, 0, stream>>>(g, nu);
        wall_solve_kernel<<<blocks_for(st.wall_nodes), kThreads, 0, stream>>>(g, dt);
        if (st.edges) wall_apply_apertures_kernel<<<blocks_for(st.edges), kThreads, 0, stream>>>(g, s.special.p);
        if (st.wall_carriers) wall_apply_carriers_kernel<<<blocks_for(st.wall_carriers), kThreads, 0, stream>>>(g, f);
        cuda_check(cudaGetLastError(), "MAC smooth wall");
    }
}
