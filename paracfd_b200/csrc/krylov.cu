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
// All reductions are deterministic: a grid fixed per kernel and device (one wave of resident CTAs),
// fixed per-block order, fixed final tree.
#include "pcfd_internal.h"

#include <algorithm>
#include <mutex>
#include <unordered_map>

namespace pcfd
{
    namespace
    {
        constexpr int kThreadsBlock = 256;
        constexpr int kStride = kMaxSet + 1;
        constexpr int kLanes = 4;                              // lanes per element pair
        constexpr int kPairsPerWarp = 32 / kLanes;             // 8
        constexpr int kPairsPerPass = kPairsPerWarp * (kThreadsBlock / 32);   // 64 pairs per CTA pass

        __device__ inline double warp_sum(double v)
        {
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            return v;
        }

        // The DOF range swept by the block kernels: the non-covered bricks (one 512-entry brick
        // per CTA iteration, 256 threads x one 16-byte pair) followed by the EB-fragment tail
        // [structured, padded length) in 512-entry chunks.  Covered-brick slots hold no DOF and
        // are skipped.  Every vector is 16-byte aligned; padding entries are inactive.
        struct Sweep
        {
            const int* bricks;
            int64_t brick_count, items, structured, padded;
            __device__ int64_t base(int64_t item) const
            {
                return item < brick_count ? int64_t(bricks[item]) * 512 : structured + (item - brick_count) * 512;
            }
        };

        // ---- split-lane block kernels (CGS2, three passes) ------------------------------------------
        // Four lanes share one element pair (16 bytes of every vector): lane l handles pair
        // (l & 7) of an 8-pair warp segment and vectors [V * (l >> 3), V * (l >> 3) + V), V = 1, 2,
        // 4 or 8 for up to 4, 8, 16 or 32 vectors.  Each basis entry is loaded exactly once and a
        // thread holds only V loads and V + 1 accumulators, so registers stay low and many warps
        // keep loads in flight.  The four partial updates of an entry are combined as
        // ((q0 + q1) + (q2 + q3)) on every lane, so the four lanes hold the same bits; the dot
        // partials are reduced per quarter and then over the block in fixed order.
        __device__ inline double quarter_total(double v)
        {
            const int pair = threadIdx.x & 7;
            const double q0 = __shfl_sync(0xffffffffu, v, pair), q1 = __shfl_sync(0xffffffffu, v, pair + 8);
            const double q2 = __shfl_sync(0xffffffffu, v, pair + 16), q3 = __shfl_sync(0xffffffffu, v, pair + 24);
            return (q0 + q1) + (q2 + q3);
        }
        __device__ inline double segment_sum(double v)
        {
            for (int o = 4; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, 8);
            return v;
        }

        // sums acc[u] of vector V*quarter + u and the norm (kept by quarter 0) into partial[block][j]
        template <int V>
        __device__ inline void block_store(double (&acc)[V + 1], int count, double* partial)
        {
            __shared__ double shared[kThreadsBlock / 32][kMaxSet + 1];
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, quarter = lane >> 3;
#pragma unroll
            for (int u = 0; u <= V; ++u)
            {
                const double v = segment_sum(acc[u]);
                if ((lane & 7) == 0)
                {
                    if (u < V) shared[warp][V * quarter + u] = v;
                    else if (quarter == 0) shared[warp][kMaxSet] = v;
                }
            }
            __syncthreads();
            if (threadIdx.x <= count)
            {
                const int j = threadIdx.x == count ? kMaxSet : threadIdx.x;
                double v = 0.0;
#pragma unroll
                for (int w = 0; w < kThreadsBlock / 32; ++w) v += shared[w][j];
                partial[int64_t(blockIdx.x) * kStride + threadIdx.x] = v;
            }
        }

        // kMode -1: h = Q^T w and w.w (w unchanged)
        //        0: w -= Q h, y += sign * U h[0..|U|)
        //        1: as 0, then w.w
        //        2: as 0, then Q^T w and w.w
        template <int V, int kMode>
        __global__ void __launch_bounds__(kThreadsBlock, V >= 8 ? 2 : 1) block_kernel(VecSet Q, const double* __restrict__ h, double* __restrict__ w,
            VecSet U, double sign, double* __restrict__ y, const uint8_t* __restrict__ active, Sweep range, double* __restrict__ partial)
        {
            __shared__ double coefficient[kMaxSet];
            double acc[V + 1];
#pragma unroll
            for (int u = 0; u <= V; ++u) acc[u] = 0.0;
            const int count = Q.size(), ucount = U.size();
            const int lane = threadIdx.x & 31, quarter = lane >> 3;
            if (kMode >= 0)
            {
                if (threadIdx.x < kMaxSet) coefficient[threadIdx.x] = threadIdx.x < count ? h[threadIdx.x] : 0.0;
                __syncthreads();
            }
            const int seg_pair = ((threadIdx.x >> 5) * kPairsPerWarp) + (lane & 7);   // 0..63
            for (int64_t item = blockIdx.x; item < range.items; item += gridDim.x)
            {
                const int64_t base = range.base(item);
#pragma unroll 1
                for (int sub = 0; sub < 256 / kPairsPerPass; ++sub)
                {
                    // every lane runs the shuffles below; a pair past the end only loads nothing
                    const int64_t e = base + 2 * (seg_pair + kPairsPerPass * sub);
                    const bool valid = e < range.padded;
                    const int64_t q = valid ? e >> 1 : 0;
                    const uchar2 a = valid ? reinterpret_cast<const uchar2*>(active)[q] : make_uchar2(0, 0);
                    const double2 w0 = valid ? reinterpret_cast<const double2*>(w)[q] : make_double2(0.0, 0.0);
                    double2 v[V];
#pragma unroll
                    for (int u = 0; u < V; ++u)
                    {
                        const int j = V * quarter + u;
                        v[u] = valid && j < count ? reinterpret_cast<const double2*>(Q.vec(j))[q] : make_double2(0.0, 0.0);
                    }
                    double2 wq = w0;
                    if (kMode >= 0)
                    {
                        double px = 0.0, py = 0.0;
#pragma unroll
                        for (int u = 0; u < V; ++u)
                        {
                            px += coefficient[V * quarter + u] * v[u].x;
                            py += coefficient[V * quarter + u] * v[u].y;
                        }
                        const double sx = quarter_total(px), sy = quarter_total(py);
                        wq.x = a.x ? w0.x - sx : w0.x;
                        wq.y = a.y ? w0.y - sy : w0.y;
                        if (quarter == 0 && valid) reinterpret_cast<double2*>(w)[q] = wq;
                        if (ucount)
                        {
                            double ux = 0.0, uy = 0.0;
#pragma unroll
                            for (int u = 0; u < V; ++u)
                            {
                                const int j = V * quarter + u;
                                if (valid && j < ucount)
                                {
                                    const double2 uv = reinterpret_cast<const double2*>(U.vec(j))[q];
                                    ux += sign * coefficient[j] * uv.x;
                                    uy += sign * coefficient[j] * uv.y;
                                }
                            }
                            const double tx = quarter_total(ux), ty = quarter_total(uy);
                            if (quarter == 0 && valid)
                            {
                                const double2 y0 = reinterpret_cast<const double2*>(y)[q];
                                reinterpret_cast<double2*>(y)[q] = make_double2(a.x ? y0.x + tx : y0.x, a.y ? y0.y + ty : y0.y);
                            }
                        }
                    }
                    if (kMode == -1 || kMode == 2)
                    {
#pragma unroll
                        for (int u = 0; u < V; ++u)
                        {
                            acc[u] += a.x ? v[u].x * wq.x : 0.0;
                            acc[u] += a.y ? v[u].y * wq.y : 0.0;
                        }
                    }
                    if (kMode != 0 && quarter == 0)
                    {
                        acc[V] += a.x ? wq.x * wq.x : 0.0;
                        acc[V] += a.y ? wq.y * wq.y : 0.0;
                    }
                }
            }
            if (kMode != 0) block_store<V>(acc, kMode == 1 ? 0 : count, partial);
        }

        // out[j] = sum over blocks of partial[b * kStride + j], j <= count (fixed order).
        __global__ void __launch_bounds__(256) block_final_kernel(const double* __restrict__ partial, int blocks, int count,
                                                                  double* __restrict__ out)
        {
            // thread partials over b = t, t + 256, ..., a warp tree, then the 8 warps in order; no
            // barrier inside the loop over j, so the sums' loads overlap
            __shared__ double shared[8][kStride];
#pragma unroll 4
            for (int j = 0; j <= count; ++j)
            {
                double v = 0.0;
                for (int b = threadIdx.x; b < blocks; b += blockDim.x) v += partial[int64_t(b) * kStride + j];
                v = warp_sum(v);
                if ((threadIdx.x & 31) == 0) shared[threadIdx.x >> 5][j] = v;
            }
            __syncthreads();
            if (threadIdx.x <= count)
            {
                double t = 0.0;
                for (int w = 0; w < 8; ++w) t += shared[w][threadIdx.x];
                out[threadIdx.x] = t;
            }
        }

        // y (+)= Z c on the active entries of the swept range (inactive entries 0 when not
        // accumulating); one CTA iteration per brick, one pair per thread.
        __global__ void __launch_bounds__(256) combine_kernel(VecSet Z, Coefficients c, double* __restrict__ y, int accumulate,
                                                               const uint8_t* __restrict__ active, Sweep range)
        {
            for (int64_t item = blockIdx.x; item < range.items; item += gridDim.x)
            {
                const int64_t e = range.base(item) + 2 * threadIdx.x;
                if (e >= range.padded) continue;
                const uchar2 a = reinterpret_cast<const uchar2*>(active)[e >> 1];
                double2 v = accumulate ? reinterpret_cast<const double2*>(y)[e >> 1] : make_double2(0.0, 0.0);
                for (int j = 0; j < Z.size(); ++j)
                {
                    const double2 z = reinterpret_cast<const double2*>(Z.vec(j))[e >> 1];
                    v.x += c.value[j] * z.x;
                    v.y += c.value[j] * z.y;
                }
                if (!a.x) v.x = accumulate ? y[e] : 0.0;
                if (!a.y) v.y = accumulate ? y[e + 1] : 0.0;
                reinterpret_cast<double2*>(y)[e >> 1] = v;
            }
        }

        __global__ void __launch_bounds__(256) scale_by_inverse_norm_kernel(double* __restrict__ dst, const double* __restrict__ src,
            const double* __restrict__ norm2, const uint8_t* __restrict__ active, Sweep range)
        {
            const double a = 1.0 / sqrt(fmax(0.0, norm2[0]));
            for (int64_t item = blockIdx.x; item < range.items; item += gridDim.x)
            {
                const int64_t e = range.base(item) + 2 * threadIdx.x;
                if (e >= range.padded) continue;
                const uchar2 m = reinterpret_cast<const uchar2*>(active)[e >> 1];
                const double2 v = reinterpret_cast<const double2*>(src)[e >> 1];
                reinterpret_cast<double2*>(dst)[e >> 1] = make_double2(m.x ? a * v.x : 0.0, m.y ? a * v.y : 0.0);
            }
        }

        // ---- delayed CGS2 (one dot pass and one update pass per Krylov column) -------------------
        // Pass 1 for Q = [C | V_0..V_{j-1}] (final), v = V_j (projected once) and w = A z_j:
        // s = Q^T v, t = Q^T w, v.v, v.w, w.w -> partial[block][2 * kMaxSet + 3].
        constexpr int kDcgsStride = 2 * kMaxSet + 4;
        // Warp w of a CTA takes basis vectors [V w, V w + V), V = ceil(m / 8), and its 32 lanes walk
        // consecutive element pairs, so every load of a warp reads 512 contiguous bytes of one
        // vector.  Every warp reads v and w as well (mostly from L1); warp 0 also sums v.v, v.w and
        // w.w.  A lane loads kGroup sub-blocks of pairs before it sums, to keep enough bytes in
        // flight with few vectors per warp.  Each sum is per lane over the CTA's items, then a warp
        // reduction; partial[block][j] holds the owning warp's sum.
        template <int V>
        __host__ __device__ constexpr int dcgs_group() { return V <= 2 ? 2 : 1; }
        template <int V>
        __global__ void __launch_bounds__(kThreadsBlock) dcgs_dot_kernel(VecSet Q, const double* __restrict__ vv,
            const double* __restrict__ w, const uint8_t* __restrict__ active, Sweep range, double* __restrict__ partial)
        {
            __shared__ double shared[kDcgsStride];
            double as[V], at[V], vv2 = 0.0, vw = 0.0, ww = 0.0;
#pragma unroll
            for (int u = 0; u < V; ++u) { as[u] = 0.0; at[u] = 0.0; }
            const int count = Q.size();
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            const int first = V * warp;
            const bool norms = warp == 0;
            constexpr int kGroup = dcgs_group<V>();
            constexpr int kSubBlocks = 512 / 64;       // an item is 512 entries = 8 sub-blocks of 32 pairs
            if (first < count || norms)
                for (int64_t item = blockIdx.x; item < range.items; item += gridDim.x)
                {
                    const int64_t base = range.base(item);
#pragma unroll 1
                    for (int sub0 = 0; sub0 < kSubBlocks; sub0 += kGroup)
                    {
                        uchar2 a[kGroup];
                        double2 v0[kGroup], w0[kGroup], b[kGroup][V];
#pragma unroll
                        for (int g = 0; g < kGroup; ++g)
                        {
                            const int64_t e = base + 2 * (32 * (sub0 + g) + lane);
                            const bool valid = e < range.padded;
                            const int64_t q = valid ? e >> 1 : 0;
                            a[g] = valid ? reinterpret_cast<const uchar2*>(active)[q] : make_uchar2(0, 0);
                            v0[g] = valid ? reinterpret_cast<const double2*>(vv)[q] : make_double2(0.0, 0.0);
                            w0[g] = valid ? reinterpret_cast<const double2*>(w)[q] : make_double2(0.0, 0.0);
#pragma unroll
                            for (int u = 0; u < V; ++u)
                                b[g][u] = valid && first + u < count ? reinterpret_cast<const double2*>(Q.vec(first + u))[q]
                                                                     : make_double2(0.0, 0.0);
                        }
#pragma unroll
                        for (int g = 0; g < kGroup; ++g)
                        {
#pragma unroll
                            for (int u = 0; u < V; ++u)
                            {
                                as[u] += (a[g].x ? b[g][u].x * v0[g].x : 0.0) + (a[g].y ? b[g][u].y * v0[g].y : 0.0);
                                at[u] += (a[g].x ? b[g][u].x * w0[g].x : 0.0) + (a[g].y ? b[g][u].y * w0[g].y : 0.0);
                            }
                            if (norms)
                            {
                                vv2 += (a[g].x ? v0[g].x * v0[g].x : 0.0) + (a[g].y ? v0[g].y * v0[g].y : 0.0);
                                vw += (a[g].x ? v0[g].x * w0[g].x : 0.0) + (a[g].y ? v0[g].y * w0[g].y : 0.0);
                                ww += (a[g].x ? w0[g].x * w0[g].x : 0.0) + (a[g].y ? w0[g].y * w0[g].y : 0.0);
                            }
                        }
                    }
                }
            for (int j = threadIdx.x; j < kDcgsStride; j += blockDim.x) shared[j] = 0.0;
            __syncthreads();
#pragma unroll
            for (int u = 0; u < V; ++u)
            {
                const double x = warp_sum(as[u]), y = warp_sum(at[u]);
                if (lane == 0 && first + u < count)
                {
                    shared[first + u] = x;
                    shared[kMaxSet + first + u] = y;
                }
            }
            if (norms)
            {
                const double a1 = warp_sum(vv2), a2 = warp_sum(vw), a3 = warp_sum(ww);
                if (lane == 0)
                {
                    shared[2 * kMaxSet] = a1;
                    shared[2 * kMaxSet + 1] = a2;
                    shared[2 * kMaxSet + 2] = a3;
                }
            }
            __syncthreads();
            for (int j = threadIdx.x; j < kDcgsStride - 1; j += blockDim.x) partial[int64_t(blockIdx.x) * kDcgsStride + j] = shared[j];
        }

        // Sums the pass-1 partials (fixed order) and forms the update coefficients:
        //   r = |v - Q s| = sqrt(v.v - s.s), c = (v.w - s.t) / r, rho^2 = w.w - t.t - c^2,
        //   v_new = v / r - Q (s / r),  w_new = w - (c / r) v - Q (t - (c / r) s),  next = w_new / rho.
        // out: [0, 32) s, [32, 64) t, [64, 96) s / r, [96, 128) t - (c / r) s, then v.v, v.w, w.w,
        // r, c, rho, 1 / r, c / r, 1 / rho (rho and r are 0 when their squares are not positive).
        // One CTA per sum j (grid 2 kMaxSet + 3): thread partials over blocks b = t, t + 256, ...,
        // a warp tree, then the 8 warps in order, into total[j].  The CTA that finishes last (a
        // ticket taken after a memory fence, no waiting) forms the coefficients and resets the
        // ticket for the next launch.
        __global__ void __launch_bounds__(256) dcgs_final_kernel(const double* __restrict__ partial, int blocks, int count,
                                                                 double* total, unsigned* ticket, double* __restrict__ out)
        {
            __shared__ double shared[8];
            __shared__ bool last;
            const int j = blockIdx.x;
            const bool used = j < count || (j >= kMaxSet && j < kMaxSet + count) || j >= 2 * kMaxSet;
            double v = 0.0;
            if (used)
                for (int b = threadIdx.x; b < blocks; b += blockDim.x) v += partial[int64_t(b) * kDcgsStride + j];
            v = warp_sum(v);
            if ((threadIdx.x & 31) == 0) shared[threadIdx.x >> 5] = v;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                double t = 0.0;
                for (int w = 0; w < 8; ++w) t += shared[w];
                total[j] = t;
                __threadfence();
                last = atomicAdd(ticket, 1u) == gridDim.x - 1;
            }
            __syncthreads();
            if (!last) return;
            // the last CTA: every total is in L2 (each writer fenced before its ticket); read them
            // past L1
            __shared__ double sum[kDcgsStride];
            if (threadIdx.x < 2 * kMaxSet + 3) sum[threadIdx.x] = __ldcg(total + threadIdx.x);
            __syncthreads();
            if (threadIdx.x != 0) return;
            *ticket = 0u;
            double ss = 0.0, st = 0.0, tt = 0.0;
            for (int l = 0; l < count; ++l)
            {
                ss += sum[l] * sum[l];
                st += sum[l] * sum[kMaxSet + l];
                tt += sum[kMaxSet + l] * sum[kMaxSet + l];
            }
            const double vv = sum[2 * kMaxSet], vw = sum[2 * kMaxSet + 1], ww = sum[2 * kMaxSet + 2];
            const double r2 = vv - ss, r = r2 > 0.0 ? sqrt(r2) : 0.0;
            const double c = r > 0.0 ? (vw - st) / r : 0.0;
            const double rho2 = ww - tt - c * c, rho = rho2 > 0.0 ? sqrt(rho2) : 0.0;
            const double inv_r = r > 0.0 ? 1.0 / r : 0.0, c_r = c * inv_r;
            for (int l = 0; l < kMaxSet; ++l)
            {
                const bool in = l < count;
                out[l] = in ? sum[l] : 0.0;
                out[kMaxSet + l] = in ? sum[kMaxSet + l] : 0.0;
                out[2 * kMaxSet + l] = in ? sum[l] * inv_r : 0.0;
                out[3 * kMaxSet + l] = in ? sum[kMaxSet + l] - c_r * sum[l] : 0.0;
            }
            double* sc = out + 4 * kMaxSet;
            sc[0] = vv; sc[1] = vw; sc[2] = ww; sc[3] = r; sc[4] = c; sc[5] = rho; sc[6] = inv_r; sc[7] = c_r;
            sc[8] = rho > 0.0 ? 1.0 / rho : 0.0;
        }

        // Pass 2: v <- v / r - Q (s / r) in place, next = (w - (c / r) v_old - Q (t - (c / r) s)) / rho.
        // One element pair per thread; the thread walks the basis vectors in order (j = 0, 1, ...)
        // in chunks of eight loads in flight, so each warp reads 512 contiguous bytes of every
        // vector and no sum crosses lanes.  (The dot pass cannot do the same: 2m + 3 running sums
        // per thread would not fit its registers, so it splits the vectors across warps instead.)
        constexpr int kUpdateChunk = 8;
        __global__ void __launch_bounds__(kThreadsBlock) dcgs_update_kernel(VecSet Q, const double* __restrict__ coefficient,
            double* __restrict__ vv, const double* __restrict__ w, double* __restrict__ next, const uint8_t* __restrict__ active, Sweep range)
        {
            __shared__ double cv[kMaxSet], cw[kMaxSet];
            if (threadIdx.x < kMaxSet)
            {
                cv[threadIdx.x] = coefficient[2 * kMaxSet + threadIdx.x];
                cw[threadIdx.x] = coefficient[3 * kMaxSet + threadIdx.x];
            }
            __syncthreads();
            const double inv_r = coefficient[4 * kMaxSet + 6], c_r = coefficient[4 * kMaxSet + 7], inv_rho = coefficient[4 * kMaxSet + 8];
            const int count = Q.size();
            for (int64_t item = blockIdx.x; item < range.items; item += gridDim.x)
            {
                const int64_t e = range.base(item) + 2 * threadIdx.x;
                if (e >= range.padded) continue;
                const int64_t q = e >> 1;
                double vx = 0.0, vy = 0.0, wx = 0.0, wy = 0.0;
                for (int j0 = 0; j0 < count; j0 += kUpdateChunk)
                {
                    double2 b[kUpdateChunk];
#pragma unroll
                    for (int u = 0; u < kUpdateChunk; ++u)
                        b[u] = j0 + u < count ? reinterpret_cast<const double2*>(Q.vec(j0 + u))[q] : make_double2(0.0, 0.0);
#pragma unroll
                    for (int u = 0; u < kUpdateChunk; ++u)
                    {
                        if (j0 + u >= count) break;
                        const double sv = cv[j0 + u], sw = cw[j0 + u];
                        vx += sv * b[u].x; vy += sv * b[u].y;
                        wx += sw * b[u].x; wy += sw * b[u].y;
                    }
                }
                const uchar2 a = reinterpret_cast<const uchar2*>(active)[q];
                const double2 v0 = reinterpret_cast<const double2*>(vv)[q], w0 = reinterpret_cast<const double2*>(w)[q];
                const double2 vn = make_double2(a.x ? inv_r * v0.x - vx : 0.0, a.y ? inv_r * v0.y - vy : 0.0);
                const double2 nx = make_double2(a.x ? inv_rho * (w0.x - c_r * v0.x - wx) : 0.0,
                                                a.y ? inv_rho * (w0.y - c_r * v0.y - wy) : 0.0);
                reinterpret_cast<double2*>(vv)[q] = vn;
                reinterpret_cast<double2*>(next)[q] = nx;
            }
        }

        Sweep sweep_range(const System& s)
        {
            if (s.bs != 8) return Sweep{nullptr, 0, (int64_t(s.Sp) + 511) / 512, 0, s.Sp};   // contiguous chunks
            const int64_t tail = (int64_t(s.Sp) - s.structured + 511) / 512;
            return Sweep{s.active_brick_list, s.active_bricks, int64_t(s.active_bricks) + std::max<int64_t>(0, tail), s.structured,
                         s.Sp};
        }

        // Grid of a block kernel: the CTAs that are resident at once (SMs x CTAs per SM that the
        // kernel's registers allow), at most 592, the partial buffers' row count.  A grid of more
        // CTAs than fit leaves a second, partly empty wave behind the first, with every CTA
        // holding the same share of the sweep.  The grid depends only on the kernel and the
        // device, so the reduction order is fixed.
        template <typename Kernel>
        int block_grid(Kernel kernel)
        {
            static int sms = 0;
            static std::mutex lock;
            static std::unordered_map<const void*, int> grids;
            std::lock_guard<std::mutex> guard(lock);
            if (!sms)
            {
                int device = 0;
                cuda_check(cudaGetDevice(&device), "device");
                cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
            }
            const void* key = reinterpret_cast<const void*>(kernel);
            auto found = grids.find(key);
            if (found != grids.end()) return found->second;
            int resident = 0;
            cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, kThreadsBlock, 0), "block kernel occupancy");
            const int grid = std::max(1, std::min(592, std::max(1, resident) * sms));
            grids.emplace(key, grid);
            return grid;
        }

        template <int kMode>
        int launch_block(System& s, const VecSet& Q, const double* h, double* w, const VecSet& U, double sign, double* y)
        {
            const int m = std::max(Q.size(), U.size());
            int grid = 0;
            auto go = [&](auto kernel) {
                grid = block_grid(kernel);
                kernel<<<grid, kThreadsBlock, 0, launch_stream(s)>>>(Q, h, w, U, sign, y, s.active, sweep_range(s), s.block_partial);
            };
            if (m <= 4) go(block_kernel<1, kMode>);
            else if (m <= 8) go(block_kernel<2, kMode>);
            else if (m <= 16) go(block_kernel<4, kMode>);
            else go(block_kernel<8, kMode>);
            return grid;
        }

        void require_aligned(const VecSet& set, const char* what)
        {
            for (int g = 0; g < 2; ++g) require(!set.count[g] || aligned16(set.base[g]), what);
            require(set.size() <= 1 || (set.stride * int64_t(sizeof(double))) % 16 == 0, what);
        }
    }

    int64_t krylov_sweep_entries(const System& s)
    {
        const Sweep range = sweep_range(s);
        if (!range.bricks) return range.padded;
        return range.brick_count * 512 + std::max<int64_t>(0, range.padded - range.structured);
    }

    void prime_block_grids()
    {
        const auto modes = [](auto kernel1, auto kernel2, auto kernel4, auto kernel8) {
            block_grid(kernel1); block_grid(kernel2); block_grid(kernel4); block_grid(kernel8);
        };
        modes(block_kernel<1, -1>, block_kernel<2, -1>, block_kernel<4, -1>, block_kernel<8, -1>);
        modes(block_kernel<1, 0>, block_kernel<2, 0>, block_kernel<4, 0>, block_kernel<8, 0>);
        modes(block_kernel<1, 1>, block_kernel<2, 1>, block_kernel<4, 1>, block_kernel<8, 1>);
        modes(block_kernel<1, 2>, block_kernel<2, 2>, block_kernel<4, 2>, block_kernel<8, 2>);
        modes(dcgs_dot_kernel<1>, dcgs_dot_kernel<2>, dcgs_dot_kernel<3>, dcgs_dot_kernel<4>);
        block_grid(dcgs_update_kernel);
    }

    void block_dot(System& s, const VecSet& Q, const double* w, double* out)
    {
        require(Q.size() >= 0 && Q.size() <= kMaxSet, "block dot: too many vectors");
        require(aligned16(w), "block dot: vector not 16-byte aligned");
        require_aligned(Q, "block dot: vector not 16-byte aligned");
        const VecSet none(Q.stride);
        const int grid = launch_block<-1>(s, Q, nullptr, const_cast<double*>(w), none, 0.0, nullptr);
        block_final_kernel<<<1, 256, 0, launch_stream(s)>>>(s.block_partial, grid, Q.size(), out);
    }

    void block_update(System& s, const VecSet& Q, const double* h, double* w, const VecSet& U, double sign, double* y, int mode,
                      double* out)
    {
        require(Q.size() <= kMaxSet && U.size() <= Q.size(), "block update: invalid vector sets");
        require(aligned16(w) && (!U.size() || aligned16(y)), "block update: vector not 16-byte aligned");
        require_aligned(Q, "block update: vector not 16-byte aligned");
        require_aligned(U, "block update: vector not 16-byte aligned");
        int grid;
        if (mode == 0) grid = launch_block<0>(s, Q, h, w, U, sign, y);
        else if (mode == 1) grid = launch_block<1>(s, Q, h, w, U, sign, y);
        else grid = launch_block<2>(s, Q, h, w, U, sign, y);
        if (mode >= 1)
            block_final_kernel<<<1, 256, 0, launch_stream(s)>>>(s.block_partial, grid, mode == 2 ? Q.size() : 0, out);
    }

    void dcgs_pass(System& s, const VecSet& Q, double* v, const double* w, double* next, double* coefficient)
    {
        require(Q.size() <= kMaxSet, "delayed CGS2: too many vectors");
        require(aligned16(v) && aligned16(w) && aligned16(next), "delayed CGS2: vector not 16-byte aligned");
        require_aligned(Q, "delayed CGS2: vector not 16-byte aligned");
        const int m = Q.size();
        const Sweep range = sweep_range(s);
        int grid = 0;
        auto dot = [&](auto kernel) {
            grid = block_grid(kernel);
            kernel<<<grid, kThreadsBlock, 0, launch_stream(s)>>>(Q, v, w, s.active, range, s.dcgs_partial);
        };
        // V = ceil(m / 8) basis vectors per warp (kMaxSet = 32)
        if (m <= 8) dot(dcgs_dot_kernel<1>);
        else if (m <= 16) dot(dcgs_dot_kernel<2>);
        else if (m <= 24) dot(dcgs_dot_kernel<3>);
        else dot(dcgs_dot_kernel<4>);
        dcgs_final_kernel<<<2 * kMaxSet + 3, 256, 0, launch_stream(s)>>>(s.dcgs_partial, grid, m, s.dcgs_total, s.dcgs_ticket,
                                                                       coefficient);
        dcgs_update_kernel<<<block_grid(dcgs_update_kernel), kThreadsBlock, 0, launch_stream(s)>>>(Q, coefficient, v, w, next, s.active,
                                                                                                  range);
    }

    void block_combine(System& s, const VecSet& Z, const Coefficients& c, double* y, bool accumulate)
    {
        require(Z.size() <= kMaxSet, "block combine: too many vectors");
        require(aligned16(y), "block combine: vector not 16-byte aligned");
        require_aligned(Z, "block combine: vector not 16-byte aligned");
        combine_kernel<<<4 * 148, 256, 0, launch_stream(s)>>>(Z, c, y, accumulate ? 1 : 0, s.active, sweep_range(s));
    }

    void scale_by_inverse_norm(System& s, double* dst, const double* src, const double* norm2)
    {
        require(aligned16(dst) && aligned16(src), "scale: vector not 16-byte aligned");
        scale_by_inverse_norm_kernel<<<4 * 148, 256, 0, launch_stream(s)>>>(dst, src, norm2, s.active, sweep_range(s));
    }
}
