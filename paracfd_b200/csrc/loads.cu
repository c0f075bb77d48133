// loads.cu -- surface-load integration on the device (reference compute_pressure_loads,
// src/core/aero_loads.cpp:183-195, and accumulate_viscous_loads, :197-204).
//
// Per wall patch: two-sided wall pressure p + grad(p).(x_patch - x_cv) reconstructed with the
// FP64 WLS stencil from the FP32 pressure shadow (as the reference does after its download),
// force n (p_minus - p_plus) A and moment about the reference origin; viscous patch forces come
// from the smooth-wall model.  All sums are FP64 with a fixed-grid deterministic tree, so the
// only D2H traffic per call is 12 doubles instead of the whole pressure field.
#include "momentum.h"

namespace pcfd
{
    namespace
    {
        constexpr int kLoadBlocks = 148;

        __device__ inline double block_sum_d(double v, double* shared)
        {
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            __syncthreads();
            if (lane == 0) shared[warp] = v;
            __syncthreads();
            v = threadIdx.x < (blockDim.x >> 5) ? shared[threadIdx.x] : 0.0;
            if (warp == 0)
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            return v;
        }

        __device__ inline double wall_pressure(int dof, const double* point, const float* p, const int* pnode, const int* goff,
                                               const int* gnbr, const double* gw, const double* centroid, double pref)
        {
            if (dof < 0) return pref;
            const double centre = double(p[dof]);
            double value = centre;
            const int n = pnode[dof];
            if (n >= 0)
            {
                double g[3] = {0, 0, 0};
                for (int q = goff[n]; q < goff[n + 1]; ++q)
                {
                    const double d = double(p[gnbr[q]]) - centre;
                    g[0] += gw[3 * q] * d; g[1] += gw[3 * q + 1] * d; g[2] += gw[3 * q + 2] * d;
                }
                for (int c = 0; c < 3; ++c) value += g[c] * (point[c] - centroid[3 * dof + c]);
            }
            return value;
        }

        __global__ void __launch_bounds__(256) loads_partial_kernel(int patches, const double* __restrict__ area,
            const double* __restrict__ pcentroid, const double* __restrict__ normal, const int* __restrict__ plus,
            const int* __restrict__ minus, const float* __restrict__ p, const int* __restrict__ pnode, const int* __restrict__ goff,
            const int* __restrict__ gnbr, const double* __restrict__ gw, const double* __restrict__ centroid, double pref,
            double ox, double oy, double oz, int sides, const float* __restrict__ side_force, const int* __restrict__ side_patch,
            double rho, double* __restrict__ partial)
        {
            __shared__ double shared[8];
            double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            const int stride = gridDim.x * blockDim.x;
            for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < patches; q += stride)
            {
                const double* c = pcentroid + 3 * q;
                const double pp = wall_pressure(plus[q], c, p, pnode, goff, gnbr, gw, centroid, pref);
                const double pm = wall_pressure(minus[q], c, p, pnode, goff, gnbr, gw, centroid, pref);
                const double scale = (pm - pp) * area[q];
                const double f[3] = {normal[3 * q] * scale, normal[3 * q + 1] * scale, normal[3 * q + 2] * scale};
                const double r[3] = {c[0] - ox, c[1] - oy, c[2] - oz};
                acc[0] += f[0]; acc[1] += f[1]; acc[2] += f[2];
                acc[3] += r[1] * f[2] - r[2] * f[1]; acc[4] += r[2] * f[0] - r[0] * f[2]; acc[5] += r[0] * f[1] - r[1] * f[0];
            }
            for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < sides; s += stride)
            {
                const double f[3] = {rho * double(side_force[3 * s]), rho * double(side_force[3 * s + 1]), rho * double(side_force[3 * s + 2])};
                const double* c = pcentroid + 3 * side_patch[s];
                const double r[3] = {c[0] - ox, c[1] - oy, c[2] - oz};
                acc[6] += f[0]; acc[7] += f[1]; acc[8] += f[2];
                acc[9] += r[1] * f[2] - r[2] * f[1]; acc[10] += r[2] * f[0] - r[0] * f[2]; acc[11] += r[0] * f[1] - r[1] * f[0];
            }
            for (int k = 0; k < 12; ++k)
            {
                const double v = block_sum_d(acc[k], shared);
                if (threadIdx.x == 0) partial[12 * blockIdx.x + k] = v;
            }
        }

        __global__ void __launch_bounds__(256) loads_final_kernel(const double* __restrict__ partial, int blocks, double* __restrict__ out)
        {
            __shared__ double shared[8];
            for (int k = 0; k < 12; ++k)
            {
                double v = 0.0;
                for (int b = threadIdx.x; b < blocks; b += blockDim.x) v += partial[12 * b + k];
                v = block_sum_d(v, shared);
                if (threadIdx.x == 0) out[k] = v;
            }
        }
    }

    struct LoadsState
    {
        int patches = 0;
        DBuf<double> area, centroid_p, normal, dof_centroid, partial, result;
        DBuf<int> plus, minus, pnode, side_patch;
        double* pinned = nullptr;
        ~LoadsState() { if (pinned) cudaFreeHost(pinned); }
    };

    void build_loads(System& s, const pcfd_topology& t)
    {
        auto* L = new LoadsState();
        s.loads = L;
        const pcfd_surface_patches& P = t.patches;
        L->patches = P.count;
        L->area.upload(std::vector<double>(P.area, P.area + P.count));
        L->centroid_p.upload(std::vector<double>(P.centroid, P.centroid + size_t(P.count) * 3));
        L->normal.upload(std::vector<double>(P.normal, P.normal + size_t(P.count) * 3));
        L->plus.upload(std::vector<int>(P.plus_dof, P.plus_dof + P.count));
        L->minus.upload(std::vector<int>(P.minus_dof, P.minus_dof + P.count));
        std::vector<int> pnode(size_t(s.S), -1);
        for (int n = 0; n < t.gradient_node_count; ++n) pnode[t.gradient_dof[n]] = n;
        L->pnode.upload(pnode);
        L->dof_centroid.upload(std::vector<double>(t.centroid, t.centroid + size_t(s.S) * 3));
        // wall sides are emitted patch by patch (plus side, then minus side) for active sides
        std::vector<int> side_patch;
        for (int q = 0; q < P.count; ++q)
        {
            if (P.plus_dof[q] >= 0 && t.active[P.plus_dof[q]]) side_patch.push_back(q);
            if (P.minus_dof[q] >= 0 && t.active[P.minus_dof[q]]) side_patch.push_back(q);
        }
        L->side_patch.upload(side_patch);
        L->partial.alloc(size_t(kLoadBlocks) * 12);
        L->result.alloc(12);
        cuda_check(cudaMallocHost(&L->pinned, 12 * sizeof(double)), "pinned loads");
    }

    void destroy_loads(System& s)
    {
        delete static_cast<LoadsState*>(s.loads);
        s.loads = nullptr;
    }

    void compute_loads(System& s, double pref, const double origin[3], double rho, bool viscous, double out[12])
    {
        LoadsState& L = *static_cast<LoadsState*>(s.loads);
        Momentum& m = momentum_of(s);
        const IrregularOperator& o = s.irr;
        const int sides = viscous ? m.nW : 0;
        loads_partial_kernel<<<kLoadBlocks, 256, 0, launch_stream(s)>>>(
            L.patches, L.area, L.centroid_p, L.normal, L.plus, L.minus, s.pressure32, L.pnode, o.grad_offset, o.grad_neighbour,
            o.grad_weight, L.dof_centroid, pref, origin[0], origin[1], origin[2], sides, m.w_force, L.side_patch, rho, L.partial);
        loads_final_kernel<<<1, 256, 0, launch_stream(s)>>>(L.partial, kLoadBlocks, L.result);
        cuda_check(cudaMemcpyAsync(L.pinned, L.result, 12 * sizeof(double), cudaMemcpyDeviceToHost, s.stream), "loads readback");
        cuda_check(cudaStreamSynchronize(s.stream), "loads");
        for (int k = 0; k < 12; ++k) out[k] = L.pinned[k];
    }
}
