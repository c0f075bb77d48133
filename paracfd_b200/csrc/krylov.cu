// krylov.cu -- fused block vector kernels for the flexible GCRO/LGMRES orthogonalisation.
//
// The reference orthogonalises each new Krylov column by modified Gram-Schmidt run twice
// (src/core/fluid/amr_pressure.cu:1390-1698): one active-masked dot, one host read and one axpy
// per basis vector and pass, so column j costs ~2(j+1) synchronising dots and ~5(j+1) passes
// over 19 M-entry FP64 vectors at 16 M cells.  Here the same projection is classical
// Gram-Schmidt applied twice (CGS2), which is mathematically the same projector and
// numerically at least as orthogonal, with every pass a single sweep over the vectors:
//   block_dot     h = Q^T w and w.w                          (reads |Q| + 1 vectors)
//   block_update  w -= Q h, y += sign * U h_U, then h' = Q^T w (reads |Q| + |U| + 2, writes 2)
// Coefficients stay on the device between passes; the host reads them once per column.
// All reductions are deterministic: fixed grid, fixed per-block order, fixed final tree.
#include "pcfd_internal.h"

#include <algorithm>

namespace pcfd
{
    namespace
    {
        constexpr int kBlocks = 592;   // 4 CTAs per SM on 148 SMs
        constexpr int kThreadsBlock = 256;
        constexpr int kStride = kMaxSet + 1;

        __device__ inline double warp_sum(double v)
        {
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            return v;
        }

        // Sums acc[0..count] over the block into partial[blockIdx.x * kStride + j].
        template <int M>
        __device__ inline void block_store(double (&acc)[M + 1], int count, double* partial)
        {
            __shared__ double shared[kThreadsBlock / 32][M + 1];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
            for (int j = 0; j <= M; ++j)
            {
                const double v = warp_sum(acc[j]);
                if (lane == 0) shared[warp][j] = v;
            }
            __syncthreads();
            if (threadIdx.x <= count)
            {
                const int j = threadIdx.x == count ? M : threadIdx.x;   // the norm lives in slot M
                double v = 0.0;
#pragma unroll
                for (int w = 0; w < kThreadsBlock / 32; ++w) v += shared[w][j];
                partial[int64_t(blockIdx.x) * kStride + threadIdx.x] = v;
            }
        }

        // Vectors are processed as pairs (16-byte loads): n2 = padded length / 2, every vector
        // 16-byte aligned, padding entries inactive.
        template <int M>
        __global__ void __launch_bounds__(kThreadsBlock) block_dot_kernel(VecSet Q, const double* __restrict__ w,
            const uint8_t* __restrict__ active, int64_t n2, double* __restrict__ partial)
        {
            double acc[M + 1];
#pragma unroll
            for (int j = 0; j <= M; ++j) acc[j] = 0.0;
            const int count = Q.count;
            for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n2; q += int64_t(gridDim.x) * blockDim.x)
            {
                const uchar2 a = reinterpret_cast<const uchar2*>(active)[q];
                double2 wq = reinterpret_cast<const double2*>(w)[q];
#pragma unroll
                for (int j = 0; j < M; ++j)
                    if (j < count)
                    {
                        const double2 v = reinterpret_cast<const double2*>(Q.v[j])[q];
                        acc[j] += a.x ? v.x * wq.x : 0.0;
                        acc[j] += a.y ? v.y * wq.y : 0.0;
                    }
                acc[M] += a.x ? wq.x * wq.x : 0.0;
                acc[M] += a.y ? wq.y * wq.y : 0.0;
            }
            block_store<M>(acc, count, partial);
        }

        // mode 0: update only; 1: + w'.w'; 2: + Q^T w' and w'.w'.  Inactive entries are left
        // untouched and contribute nothing.
        template <int M, int kMode>
        __global__ void __launch_bounds__(kThreadsBlock) block_update_kernel(VecSet Q, const double* __restrict__ h, double* __restrict__ w,
            VecSet U, double sign, double* __restrict__ y, const uint8_t* __restrict__ active, int64_t n2, double* __restrict__ partial)
        {
            __shared__ double coefficient[M];
            double acc[M + 1];
#pragma unroll
            for (int j = 0; j <= M; ++j) acc[j] = 0.0;
            const int count = Q.count, ucount = U.count;
            if (threadIdx.x < M) coefficient[threadIdx.x] = threadIdx.x < count ? h[threadIdx.x] : 0.0;
            __syncthreads();
            for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n2; q += int64_t(gridDim.x) * blockDim.x)
            {
                const uchar2 a = reinterpret_cast<const uchar2*>(active)[q];
                // up to 16 basis pairs stay in registers for the dot pass; wider sets re-read
                // them (the lines were just fetched, so the second read is served by L2)
                constexpr int kKeep = M <= 16 ? M : 1;
                double2 qv[kKeep];
                const double2 w0 = reinterpret_cast<const double2*>(w)[q];
                double2 wq = w0;
#pragma unroll
                for (int j = 0; j < M; ++j)
                    if (j < count)
                    {
                        const double2 v = reinterpret_cast<const double2*>(Q.v[j])[q];
                        if (M <= 16) qv[j % kKeep] = v;
                        wq.x -= coefficient[j] * v.x;
                        wq.y -= coefficient[j] * v.y;
                    }
                wq.x = a.x ? wq.x : w0.x;
                wq.y = a.y ? wq.y : w0.y;
                reinterpret_cast<double2*>(w)[q] = wq;
                if (ucount)
                {
                    const double2 y0 = reinterpret_cast<const double2*>(y)[q];
                    double2 yq = y0;
#pragma unroll
                    for (int j = 0; j < M; ++j)
                        if (j < ucount)
                        {
                            const double2 u = reinterpret_cast<const double2*>(U.v[j])[q];
                            yq.x += sign * coefficient[j] * u.x;
                            yq.y += sign * coefficient[j] * u.y;
                        }
                    yq.x = a.x ? yq.x : y0.x;
                    yq.y = a.y ? yq.y : y0.y;
                    reinterpret_cast<double2*>(y)[q] = yq;
                }
                if (kMode == 2)
                {
#pragma unroll
                    for (int j = 0; j < M; ++j)
                        if (j < count)
                        {
                            const double2 v = M <= 16 ? qv[j % kKeep] : reinterpret_cast<const double2*>(Q.v[j])[q];
                            acc[j] += a.x ? v.x * wq.x : 0.0;
                            acc[j] += a.y ? v.y * wq.y : 0.0;
                        }
                }
                if (kMode >= 1)
                {
                    acc[M] += a.x ? wq.x * wq.x : 0.0;
                    acc[M] += a.y ? wq.y * wq.y : 0.0;
                }
            }
            if (kMode >= 1) block_store<M>(acc, kMode == 2 ? count : 0, partial);
        }

        // out[j] = sum over blocks of partial[b * kStride + j], j <= count (fixed order).
        __global__ void __launch_bounds__(256) block_final_kernel(const double* __restrict__ partial, int blocks, int count,
                                                                  double* __restrict__ out)
        {
            __shared__ double shared[8];
            for (int j = 0; j <= count; ++j)
            {
                double v = 0.0;
                for (int b = threadIdx.x; b < blocks; b += blockDim.x) v += partial[int64_t(b) * kStride + j];
                v = warp_sum(v);
                if ((threadIdx.x & 31) == 0) shared[threadIdx.x >> 5] = v;
                __syncthreads();
                if (threadIdx.x == 0)
                {
                    double t = 0.0;
                    for (int w = 0; w < 8; ++w) t += shared[w];
                    out[j] = t;
                }
                __syncthreads();
            }
        }

        __global__ void combine_kernel(VecSet Z, Coefficients c, double* __restrict__ y, int accumulate,
                                       const uint8_t* __restrict__ active, int64_t n)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= n) return;
            if (!active[q]) { if (!accumulate) y[q] = 0.0; return; }
            double v = accumulate ? y[q] : 0.0;
            for (int j = 0; j < Z.count; ++j) v += c.value[j] * Z.v[j][q];
            y[q] = v;
        }

        __global__ void scale_by_inverse_norm_kernel(double* __restrict__ dst, const double* __restrict__ src,
                                                     const double* __restrict__ norm2, const uint8_t* __restrict__ active, int64_t n)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= n) return;
            const double a = 1.0 / sqrt(fmax(0.0, norm2[0]));
            dst[q] = active[q] ? a * src[q] : 0.0;
        }

        // Grid of a block kernel; it depends only on the device, so the reduction order is fixed.
        template <class K> int resident_grid(K kernel)
        {
            // 4 CTAs per SM: at the register budget of the widest instantiation two are resident at
            // a time and the 16-byte loads keep enough bytes in flight either way.
            (void)kernel;
            int device = 0, sms = 0;
            cuda_check(cudaGetDevice(&device), "device");
            cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
            return std::max(1, std::min(kBlocks, 4 * sms));
        }

        template <int M> int launch_dot(System& s, const VecSet& Q, const double* w)
        {
            const int grid = resident_grid(block_dot_kernel<M>);
            block_dot_kernel<M><<<grid, kThreadsBlock, 0, launch_stream(s)>>>(Q, w, s.active, s.Sp / 2, s.block_partial);
            return grid;
        }
        template <int M, int kMode>
        int launch_update(System& s, const VecSet& Q, const double* h, double* w, const VecSet& U, double sign, double* y)
        {
            const int grid = resident_grid(block_update_kernel<M, kMode>);
            block_update_kernel<M, kMode><<<grid, kThreadsBlock, 0, launch_stream(s)>>>(Q, h, w, U, sign, y, s.active, s.Sp / 2,
                                                                                        s.block_partial);
            return grid;
        }
        template <int kMode>
        int dispatch_update(System& s, const VecSet& Q, const double* h, double* w, const VecSet& U, double sign, double* y)
        {
            const int m = std::max(Q.count, U.count);
            if (m <= 4) return launch_update<4, kMode>(s, Q, h, w, U, sign, y);
            if (m <= 8) return launch_update<8, kMode>(s, Q, h, w, U, sign, y);
            if (m <= 16) return launch_update<16, kMode>(s, Q, h, w, U, sign, y);
            return launch_update<32, kMode>(s, Q, h, w, U, sign, y);
        }
    }

    namespace
    {
        void require_aligned(const VecSet& set, const char* what)
        {
            for (int j = 0; j < set.count; ++j) require(aligned16(set.v[j]), what);
        }
    }

    void block_dot(System& s, const VecSet& Q, const double* w, double* out)
    {
        require(Q.count >= 0 && Q.count <= kMaxSet, "block dot: too many vectors");
        require(aligned16(w), "block dot: vector not 16-byte aligned");
        require_aligned(Q, "block dot: vector not 16-byte aligned");
        int grid;
        if (Q.count <= 4) grid = launch_dot<4>(s, Q, w);
        else if (Q.count <= 8) grid = launch_dot<8>(s, Q, w);
        else if (Q.count <= 16) grid = launch_dot<16>(s, Q, w);
        else grid = launch_dot<32>(s, Q, w);
        block_final_kernel<<<1, 256, 0, launch_stream(s)>>>(s.block_partial, grid, Q.count, out);
    }

    void block_update(System& s, const VecSet& Q, const double* h, double* w, const VecSet& U, double sign, double* y, int mode,
                      double* out)
    {
        require(Q.count <= kMaxSet && U.count <= Q.count, "block update: invalid vector sets");
        require(aligned16(w) && (!U.count || aligned16(y)), "block update: vector not 16-byte aligned");
        require_aligned(Q, "block update: vector not 16-byte aligned");
        require_aligned(U, "block update: vector not 16-byte aligned");
        int grid;
        if (mode == 0) grid = dispatch_update<0>(s, Q, h, w, U, sign, y);
        else if (mode == 1) grid = dispatch_update<1>(s, Q, h, w, U, sign, y);
        else grid = dispatch_update<2>(s, Q, h, w, U, sign, y);
        if (mode >= 1)
            block_final_kernel<<<1, 256, 0, launch_stream(s)>>>(s.block_partial, grid, mode == 2 ? Q.count : 0, out);
    }

    void block_combine(System& s, const VecSet& Z, const Coefficients& c, double* y, bool accumulate)
    {
        require(Z.count <= kMaxSet, "block combine: too many vectors");
        combine_kernel<<<blocks_for(s.S), kThreads, 0, launch_stream(s)>>>(Z, c, y, accumulate ? 1 : 0, s.active, s.S);
    }

    void scale_by_inverse_norm(System& s, double* dst, const double* src, const double* norm2)
    {
        scale_by_inverse_norm_kernel<<<blocks_for(s.S), kThreads, 0, launch_stream(s)>>>(dst, src, norm2, s.active, s.S);
    }
}
