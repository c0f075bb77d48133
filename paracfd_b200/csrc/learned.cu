// learned.cu -- brick-local learned preconditioner (no reference counterpart).
//
// A 3-level U-Net per 8^3 brick (levels 8^3/4^3/2^3 with 16/32/64 channels, 3x3x3 convolutions
// with zero padding at the brick boundary, 2x2x2 average pooling, nearest upsampling, skip
// connections by concatenation, ReLU, no biases, a 1x1x1 head).  The input of a brick is
// D^-1 r / s and the active mask, s the RMS of D^-1 r over the brick's active cells; the output is
// z = s * net(...) on the active cells, so the map is positively homogeneous in r.  The
// definition, and the numbers every kernel here is checked against, are the numpy oracle in
// oracle/unet.py.
//
// Convolutions run on the 5th-generation tensor cores: tcgen05.mma kind::f16 (BF16 operands,
// FP32 accumulators in TMEM), M = 128 output voxels x N = Cout x K = 16 input channels per
// instruction.  A CTA stages a group of bricks into shared memory in a zero-padded K-major
// layout ([channel chunk of 8][padded voxel][8 x BF16]), so that the A operand of every tap
// (dz,dy,dx) is the same layout shifted by a constant number of 16-byte rows: each tap is one
// shared-memory descriptor, no im2col copy.  On the 8^3 level a tile is 16 padded (z,y) rows of
// 8 voxels (stride 10 rows); on the 4^3 and 2^3 levels a tile is 128 consecutive padded
// positions.  Rows that fall on padding are computed and discarded.
//
// Training (pcfd_learned_train): (residual, multigrid correction) brick pairs harvested from the
// solver's own preconditioner calls, masked mean-square loss on z/s, backward pass with the
// transposed convolutions on the same tensor-core kernel (flipped taps, transposed channels),
// weight gradients on CUDA cores in FP32, Adam on FP32 master weights.
#include "pcfd_internal.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

namespace pcfd
{
    namespace
    {
        using bf16 = __nv_bfloat16;

        // ---- network shape (must match oracle/unet.py) ----
        // parameter tensors in flat order: enc0.0 enc1.0 bott.0 dec1.0 dec1.1 dec0.0 dec0.1 ([27][cout][cin]
        // each), then the head [16]
        constexpr int kHead = 16;
        enum Tensor { ENC0, ENC1, BOTT, DEC1A, DEC1B, DEC0A, DEC0B };
        __host__ __device__ constexpr int tensor_cout(int k) { return k == 0 ? 16 : k == 1 ? 32 : k == 2 ? 64 : k <= 4 ? 32 : 16; }
        __host__ __device__ constexpr int tensor_cin(int k) { return k <= 1 ? 16 : k == 2 ? 32 : k == 3 ? 64 : k == 4 ? 32 : k == 5 ? 32 : 16; }
        __host__ __device__ constexpr int64_t tensor_size(int k) { return int64_t(27) * tensor_cout(k) * tensor_cin(k); }
        __host__ __device__ constexpr int64_t tensor_offset(int k) { return k == 0 ? 0 : tensor_offset(k - 1) + tensor_size(k - 1); }
        constexpr int64_t kWeights = tensor_offset(7);
        constexpr int64_t kParams = kWeights + kHead;
        static_assert(kParams == 179728, "parameter count must match oracle/unet.py");

        // A tensor-core wait gives up after the system's wait limit (pcfd_learned_set_wait, 2 s by
        // default); after a wait gave up, the kernel drains its last commit with this fixed limit
        // before freeing its tensor memory.
        constexpr uint64_t kMaxWaitNs = 2000000000ull;

        // ---- geometry of one level's staged group of bricks ----
        // N: brick edge; XP: padded edge; NB: bricks per CTA; G: positions between the 8-row
        // groups of a tile; T: tiles per group; NPOS: staged positions per channel chunk.
        template <int N> struct Geometry;
        template <> struct Geometry<8>
        {
            static constexpr int XP = 10, P = 1000, NB = 2, G = 10, T = 10, NPOS = 2024;
            // tile k of brick b starts at padded row 11 + 16 (k % 5), x = 0
            __host__ __device__ static constexpr int tile_start(int t) { return (t / 5) * P + (11 + 16 * (t % 5)) * XP + 1; }
        };
        template <> struct Geometry<4>
        {
            static constexpr int XP = 6, P = 216, NB = 4, G = 8, T = 7, NPOS = 984;
            __host__ __device__ static constexpr int tile_start(int t) { return 43 + 128 * t; }
        };
        template <> struct Geometry<2>
        {
            static constexpr int XP = 4, P = 64, NB = 16, G = 8, T = 8, NPOS = 1072;
            __host__ __device__ static constexpr int tile_start(int t) { return 21 + 128 * t; }
        };
        // padded position of voxel (x,y,z) of brick b
        template <int N> __host__ __device__ constexpr int padded(int b, int x, int y, int z)
        {
            using Gm = Geometry<N>;
            return b * Gm::P + ((z + 1) * Gm::XP + y + 1) * Gm::XP + x + 1;
        }
        // M row m of tile t -> padded position
        template <int N> __host__ __device__ constexpr int row_position(int t, int m)
        {
            using Gm = Geometry<N>;
            return Gm::tile_start(t) + (m >> 3) * Gm::G + (m & 7);
        }
        template <int N> __host__ __device__ constexpr int tap_shift(int tap)
        {
            using Gm = Geometry<N>;
            return ((tap / 9) - 1) * Gm::XP * Gm::XP + ((tap / 3) % 3 - 1) * Gm::XP + (tap % 3) - 1;
        }
        // compile-time proof that every descriptor stays inside the staged rows and that the
        // tiles cover every interior voxel of every brick of a group
        template <int N> constexpr bool geometry_in_bounds()
        {
            using Gm = Geometry<N>;
            bool seen[Gm::NB * Gm::P] = {};
            for (int t = 0; t < Gm::T; ++t)
                for (int m = 0; m < 128; ++m)
                {
                    const int p = row_position<N>(t, m);
                    if (p + tap_shift<N>(0) < 0 || p + tap_shift<N>(26) >= Gm::NPOS) return false;
                    if (p < Gm::NB * Gm::P) seen[p] = true;
                }
            for (int b = 0; b < Gm::NB; ++b)
                for (int z = 0; z < N; ++z)
                    for (int y = 0; y < N; ++y)
                        for (int x = 0; x < N; ++x)
                            if (!seen[padded<N>(b, x, y, z)]) return false;
            return Gm::NPOS % 8 == 0;
        }
        static_assert(geometry_in_bounds<2>(), "2^3 tiling out of bounds");
        static_assert(geometry_in_bounds<4>(), "4^3 tiling out of bounds");
        static_assert(geometry_in_bounds<8>(), "8^3 tiling out of bounds");

        // ---- tcgen05 / mbarrier primitives (inline PTX) ----
        __device__ inline uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

        // K-major, no-swizzle shared-memory matrix descriptor: 8-row core matrices of 16-byte rows,
        // lbo = bytes between the two 8-element K halves, sbo = bytes between 8-row groups.
        __device__ inline uint64_t smem_descriptor(uint32_t address, uint32_t lbo, uint32_t sbo)
        {
            uint64_t d = uint64_t((address >> 4) & 0x3FFFu);
            d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
            d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
            d |= uint64_t(1) << 46;   // descriptor version (sm_100)
            return d;                 // base offset 0, swizzle none
        }
        // kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 D, M = 128, N = cout
        __host__ __device__ constexpr uint32_t instruction_descriptor(int cout)
        {
            return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(cout >> 3) << 17) | (uint32_t(128 >> 4) << 24);
        }
        __device__ inline void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
        {
            const uint32_t mask = 0;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                :
                : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask));
        }
        __device__ inline void mma_commit(uint64_t* bar)
        {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
        }
        __device__ inline void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
        __device__ inline void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
        __device__ inline void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
        __device__ inline void barrier_init(uint64_t* bar)
        {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        }
        __device__ inline uint64_t global_ns()
        {
            uint64_t t;
            asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
            return t;
        }
        // polls the barrier phase with the given parity; false after limit_ns nanoseconds
        __device__ inline bool barrier_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns)
        {
            const uint32_t a = smem_u32(bar);
            const uint64_t start = global_ns();
            for (;;)
            {
                uint32_t done;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(a), "r"(parity)
                    : "memory");
                if (done) return true;
                if (global_ns() - start > limit_ns) return false;
            }
        }
        __device__ inline void tmem_alloc(uint32_t* slot, uint32_t cols)
        {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols) : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        __device__ inline void tmem_dealloc(uint32_t taddr, uint32_t cols)
        {
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
        }
        // 16 consecutive FP32 accumulator columns of this thread's TMEM lane
        __device__ inline void tmem_load16(uint32_t taddr, float* v)
        {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
                  "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
        }

        __device__ inline uint4 pack8(const float* f)
        {
            uint4 u;
            uint32_t* w = reinterpret_cast<uint32_t*>(&u);
            for (int i = 0; i < 4; ++i)
            {
                const __nv_bfloat162 h = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
                w[i] = *reinterpret_cast<const uint32_t*>(&h);
            }
            return u;
        }
        __device__ inline void unpack8(const uint4& u, float* f)
        {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(&u);
            for (int i = 0; i < 4; ++i)
            {
                const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
                const float2 v = __bfloat1622float2(h);
                f[2 * i] = v.x;
                f[2 * i + 1] = v.y;
            }
        }

        // ---- convolution ----
        enum SourceMode { SAME = 0, POOL = 1, UP = 2 };
        struct ConvSource
        {
            const bf16* x;     // [samples][level voxels][channels]
            const bf16* w;     // [27][cout][channels]
            int channels, mode;
        };
        struct ConvParams
        {
            ConvSource src[2];
            int sources, cout, samples, relu, out_fp32;
            void* y;           // [samples][N^3][cout], BF16 or FP32
            int* error;        // set to 1 when a barrier wait gave up
            uint64_t wait_ns;  // limit of each tensor-core wait
            int idle_wait;     // 1: the first wait polls a barrier that no commit completes (fault-path check)
        };

        __host__ __device__ constexpr int tmem_columns(int cols)
        {
            return cols <= 32 ? 32 : cols <= 64 ? 64 : cols <= 128 ? 128 : cols <= 256 ? 256 : 512;
        }

        // 8 channels [c0, c0 + 8) of voxel (x,y,z) of sample b from a source at level N (after
        // its pooling / upsampling), as 8 BF16
        template <int N> __device__ inline uint4 load_source(const ConvSource& s, int64_t b, int x, int y, int z, int c0)
        {
            const int C = s.channels;
            if (s.mode == SAME)
                return *reinterpret_cast<const uint4*>(s.x + ((b * N + z) * N + y) * int64_t(N) * C + int64_t(x) * C + c0);
            if (s.mode == UP)
            {
                constexpr int M = N / 2;
                return *reinterpret_cast<const uint4*>(s.x + ((b * M + z / 2) * M + y / 2) * int64_t(M) * C + int64_t(x / 2) * C + c0);
            }
            constexpr int F = 2 * N;
            float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, v[8];
            for (int k = 0; k < 8; ++k)
            {
                const int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
                unpack8(*reinterpret_cast<const uint4*>(s.x + ((b * F + fz) * F + fy) * int64_t(F) * C + int64_t(fx) * C + c0), v);
                for (int i = 0; i < 8; ++i) acc[i] += v[i];
            }
            for (int i = 0; i < 8; ++i) acc[i] *= 0.125f;
            return pack8(acc);
        }

        // address of the 8 channels [c0, c0 + 8) of voxel (x,y,z) of sample b for a SAME or UP source
        template <int N> __device__ inline const bf16* source_address(const ConvSource& s, int64_t b, int x, int y, int z, int c0)
        {
            const int C = s.channels;
            if (s.mode == SAME) return s.x + ((b * N + z) * N + y) * int64_t(N) * C + int64_t(x) * C + c0;
            constexpr int M = N / 2;
            return s.x + ((b * M + z / 2) * M + y / 2) * int64_t(M) * C + int64_t(x / 2) * C + c0;
        }
        __device__ inline void cp_async16(void* dst, const void* src)
        {
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
        }
        __device__ inline void cp_async_wait_all()
        {
            asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        }

        // One CTA of 128 threads per group of Geometry<N>::NB bricks (persistent over groups).
        // Shared memory: A [2][NPOS][16 B] | B [27][2][cout][16 B] | barrier | TMEM address.
        template <int N>
        __global__ void __launch_bounds__(128) conv_kernel(ConvParams p)
        {
            using Gm = Geometry<N>;
            extern __shared__ __align__(128) uint8_t smem[];
            uint4* A = reinterpret_cast<uint4*>(smem);
            const int cout = p.cout;
            uint4* Bw = A + 2 * Gm::NPOS;
            uint64_t* bar = reinterpret_cast<uint64_t*>(Bw + 27 * 2 * cout);
            uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
            uint64_t* idle = bar + 2;      // initialised, never arrived on
            __shared__ int failed;
            const int tid = threadIdx.x, warp = tid >> 5;
            const uint32_t cols = tmem_columns(Gm::T * cout);

            for (int i = tid; i < 2 * Gm::NPOS; i += 128) A[i] = make_uint4(0, 0, 0, 0);
            if (tid == 0) { barrier_init(bar); barrier_init(idle); failed = 0; }
            if (warp == 0) tmem_alloc(tslot, cols);
            fence_before_sync();
            __syncthreads();
            fence_after_sync();
            const uint32_t tmem = *tslot;
            const uint32_t a_base = smem_u32(A), b_base = smem_u32(Bw);
            const uint32_t idesc = instruction_descriptor(cout);
            uint32_t phase = 0;
            const int groups = (p.samples + Gm::NB - 1) / Gm::NB;
            constexpr int V = N * N * N;

            for (int group = blockIdx.x; group < groups; group += gridDim.x)
            {
                const int b0 = group * Gm::NB, nb = min(Gm::NB, p.samples - b0);
                bool first = true;
                for (int si = 0; si < p.sources; ++si)
                {
                    const ConvSource& s = p.src[si];
                    for (int c0 = 0; c0 < s.channels; c0 += 16)
                    {
                        // stage 16 channels of the group's bricks and the matching weights: copies
                        // straight to shared memory (cp.async) for plain and upsampled sources, a
                        // register average for pooled ones (two voxels in flight per thread)
                        const int items = nb * V * 2;
                        if (s.mode != POOL)
                        {
                            for (int i = tid; i < items; i += 128)
                            {
                                const int half = i & 1, v = (i >> 1) % V, b = (i >> 1) / V;
                                const int x = v % N, y = (v / N) % N, z = v / (N * N);
                                cp_async16(&A[half * Gm::NPOS + padded<N>(b, x, y, z)], source_address<N>(s, b0 + b, x, y, z, c0 + 8 * half));
                            }
                        }
                        else
                        {
                            for (int i = tid; i < items; i += 256)
                            {
                                const int j = i + 128;
                                uint4 u0, u1 = make_uint4(0, 0, 0, 0);
                                const int h0 = i & 1, v0 = (i >> 1) % V, bb0 = (i >> 1) / V;
                                u0 = load_source<N>(s, b0 + bb0, v0 % N, (v0 / N) % N, v0 / (N * N), c0 + 8 * h0);
                                const int h1 = j & 1, v1 = (j >> 1) % V, bb1 = (j >> 1) / V;
                                if (j < items) u1 = load_source<N>(s, b0 + bb1, v1 % N, (v1 / N) % N, v1 / (N * N), c0 + 8 * h1);
                                A[h0 * Gm::NPOS + padded<N>(bb0, v0 % N, (v0 / N) % N, v0 / (N * N))] = u0;
                                if (j < items) A[h1 * Gm::NPOS + padded<N>(bb1, v1 % N, (v1 / N) % N, v1 / (N * N))] = u1;
                            }
                        }
                        for (int i = tid; i < 27 * 2 * cout; i += 128)
                        {
                            const int co = i % cout, half = (i / cout) & 1, tap = i / (2 * cout);
                            cp_async16(&Bw[i], s.w + (int64_t(tap) * cout + co) * s.channels + c0 + 8 * half);
                        }
                        cp_async_wait_all();
                        fence_async_shared();
                        __syncthreads();
                        if (tid == 0)
                        {
                            fence_after_sync();
                            for (int t = 0; t < Gm::T; ++t)
                                for (int tap = 0; tap < 27; ++tap)
                                {
                                    const uint64_t a = smem_descriptor(a_base + uint32_t(Gm::tile_start(t) + tap_shift<N>(tap)) * 16u,
                                                                       uint32_t(Gm::NPOS) * 16u, uint32_t(Gm::G) * 16u);
                                    const uint64_t b = smem_descriptor(b_base + uint32_t(tap) * 2u * uint32_t(cout) * 16u, uint32_t(cout) * 16u, 128u);
                                    mma_bf16(tmem + uint32_t(t * cout), a, b, idesc, (first && tap == 0) ? 0u : 1u);
                                }
                            mma_commit(bar);
                        }
                        first = false;
                        const bool done = p.idle_wait ? barrier_wait(idle, 0, p.wait_ns) : barrier_wait(bar, phase, p.wait_ns);
                        if (!done) failed = 1;
                        phase ^= 1;
                        __syncthreads();
                        if (failed) break;
                    }
                    if (failed) break;
                }
                if (failed) break;
                // epilogue: TMEM lane = tile row; warp w reads lanes 32w..32w+31
                fence_after_sync();
                for (int t = 0; t < Gm::T; ++t)
                {
                    const int m = 32 * warp + (tid & 31);
                    const int pos = row_position<N>(t, m);
                    const int b = pos / Gm::P, rem = pos % Gm::P;
                    const int zp = rem / (Gm::XP * Gm::XP), yp = (rem / Gm::XP) % Gm::XP, xp = rem % Gm::XP;
                    const bool valid = b < nb && zp >= 1 && zp <= N && yp >= 1 && yp <= N && xp >= 1 && xp <= N;
                    const int64_t voxel = (int64_t(b0 + b) * V + ((zp - 1) * N + (yp - 1)) * N + (xp - 1));
                    for (int c = 0; c < cout; c += 16)
                    {
                        float v[16];
                        tmem_load16(tmem + (uint32_t(32 * warp) << 16) + uint32_t(t * cout + c), v);
                        if (!valid) continue;
                        if (p.relu)
                            for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.0f);
                        if (p.out_fp32)
                        {
                            float4* o = reinterpret_cast<float4*>(static_cast<float*>(p.y) + voxel * cout + c);
                            for (int i = 0; i < 4; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                        }
                        else
                        {
                            uint4* o = reinterpret_cast<uint4*>(static_cast<bf16*>(p.y) + voxel * cout + c);
                            o[0] = pack8(v);
                            o[1] = pack8(v + 8);
                        }
                    }
                }
                fence_before_sync();
                __syncthreads();
            }
            if (failed)
            {
                if (tid == 0) atomicExch(p.error, 1);
                // the last commit has not been seen: wait for it (fixed bound) before the tensor
                // memory its MMAs write is freed
                barrier_wait(bar, phase ^ 1, kMaxWaitNs);
            }
            fence_before_sync();
            __syncthreads();
            if (warp == 0) tmem_dealloc(tmem, cols);
        }

        template <int N> size_t conv_smem(int cout)
        {
            const size_t bytes = size_t(2) * Geometry<N>::NPOS * 16 + size_t(27) * 2 * cout * 16 + 32;
            // co-resident CTAs must fit their TMEM allocations into the SM's 512 columns
            const int cols = tmem_columns(Geometry<N>::T * cout);
            const size_t floor_bytes = cols == 512 ? 116 * 1024 : cols == 256 ? 80 * 1024 : cols == 128 ? 48 * 1024 : 0;
            return std::max(bytes, floor_bytes);
        }

        // ---- elementwise / small kernels ----
        // network input for system bricks: x0 [bricks][512][16], scale [bricks]
        __global__ void prepare_kernel(const int* slots, int bricks, const double* r, const double* diag, const uint8_t* active,
                                       bf16* x0, float* scale)
        {
            const int b = blockIdx.x;
            if (b >= bricks) return;
            const int64_t q0 = int64_t(slots[b]) * 512;
            __shared__ double red[2][8];
            double q[2], ss = 0, cnt = 0;
            for (int k = 0; k < 2; ++k)
            {
                const int v = threadIdx.x + 256 * k;
                const int64_t qq = q0 + v;
                q[k] = active[qq] && diag[qq] > 0 ? r[qq] / diag[qq] : 0.0;
                ss += q[k] * q[k];
                cnt += active[qq] ? 1.0 : 0.0;
            }
            for (int o = 16; o; o >>= 1) { ss += __shfl_xor_sync(0xffffffffu, ss, o); cnt += __shfl_xor_sync(0xffffffffu, cnt, o); }
            if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = ss; red[1][threadIdx.x >> 5] = cnt; }
            __syncthreads();
            double tss = 0, tcnt = 0;
            for (int w = 0; w < 8; ++w) { tss += red[0][w]; tcnt += red[1][w]; }
            double s = std::sqrt(tss / fmax(tcnt, 1.0));
            if (!(s > 0)) s = 1.0;
            if (threadIdx.x == 0) scale[b] = float(s);
            for (int k = 0; k < 2; ++k)
            {
                const int v = threadIdx.x + 256 * k;
                float f[8] = {float(q[k] / s), active[q0 + v] ? 1.0f : 0.0f, 0, 0, 0, 0, 0, 0}, zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                uint4* o = reinterpret_cast<uint4*>(x0 + (int64_t(b) * 512 + v) * 16);
                o[0] = pack8(f);
                o[1] = pack8(zero);
            }
        }

        // z = s * head(d0) on the active cells of the system bricks
        __global__ void head_apply_kernel(const int* slots, int bricks, const bf16* d0, const float* head, const float* scale,
                                          const uint8_t* active, double* z)
        {
            const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (i >= int64_t(bricks) * 512) return;
            const int b = int(i / 512), v = int(i % 512);
            const int64_t q = int64_t(slots[b]) * 512 + v;
            float f[16];
            const uint4* src = reinterpret_cast<const uint4*>(d0 + i * 16);
            unpack8(src[0], f);
            unpack8(src[1], f + 8);
            float acc = 0;
            for (int c = 0; c < 16; ++c) acc += f[c] * head[c];
            z[q] = active[q] ? double(scale[b]) * double(acc) : 0.0;
        }

        // EB fragments and other DOFs after the structured slots: one damped Jacobi step
        __global__ void jacobi_tail_kernel(int64_t begin, int64_t end, const double* r, const double* diag, const uint8_t* active, double* z)
        {
            const int64_t q = begin + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q < end) z[q] = active[q] && diag[q] > 0 ? (2.0 / 3.0) * r[q] / diag[q] : 0.0;
        }

        // 256-thread block sum
        __device__ inline double block_sum(double v, double* red)
        {
            for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            __syncthreads();
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
            __syncthreads();
            double t = 0;
            for (int w = 0; w < 8; ++w) t += red[w];
            return t;
        }

        // x = A_B^-1 b on one brick by conjugate gradients in shared memory: A_B is the operator's
        // diagonal block of the brick (the full diagonal D, minus h for every open face to a cell of
        // the same brick); 2 cells per thread, to 1e-8 relative or 400 iterations
        __device__ void brick_solve(const double* b, double* x, const uint8_t* code, const double* D, double h, double* ps, double* red)
        {
            double r[2], p[2], Ap[2];
            for (int k = 0; k < 2; ++k)
            {
                const int v = threadIdx.x + 256 * k;
                x[v] = 0;
                r[k] = b[v];
                p[k] = r[k];
                ps[v] = p[k];
            }
            double rr = block_sum(r[0] * r[0] + r[1] * r[1], red);
            const double stop = 1e-16 * rr;
            for (int it = 0; it < 400 && rr > stop; ++it)
            {
                __syncthreads();
                for (int k = 0; k < 2; ++k)
                {
                    const int v = threadIdx.x + 256 * k;
                    const int c[3] = {v & 7, (v >> 3) & 7, v >> 6};
                    double a = D[v] * ps[v];
                    for (int axis = 0; axis < 3; ++axis)
                        for (int pos = 0; pos < 2; ++pos)
                        {
                            const int q = c[axis] + (pos ? 1 : -1);
                            if (q < 0 || q > 7 || !(code[v] & (1u << (2 * axis + pos)))) continue;
                            a -= h * ps[v + (pos ? 1 : -1) * (axis == 0 ? 1 : axis == 1 ? 8 : 64)];
                        }
                    Ap[k] = D[v] > 0 ? a : 0.0;
                }
                const double pAp = block_sum(p[0] * Ap[0] + p[1] * Ap[1], red);
                if (!(pAp > 0)) break;
                const double alpha = rr / pAp;
                for (int k = 0; k < 2; ++k)
                {
                    x[threadIdx.x + 256 * k] += alpha * p[k];
                    r[k] -= alpha * Ap[k];
                }
                const double next = block_sum(r[0] * r[0] + r[1] * r[1], red);
                const double beta = next / rr;
                rr = next;
                __syncthreads();
                for (int k = 0; k < 2; ++k)
                {
                    p[k] = r[k] + beta * p[k];
                    ps[threadIdx.x + 256 * k] = p[k];
                }
            }
            __syncthreads();
        }

        // harvest: brick k of preconditioner call `pair` -> store slot; input D^-1 r / s, mask,
        // target z / s with z the multigrid output (local = 0) or the brick-local solve (local = 1)
        __global__ void harvest_kernel(const int* slots, int bricks, int64_t pair, int per_pair, uint64_t seed, int64_t capacity,
                                       const double* r, const double* z, const double* diag, const uint8_t* active, bf16* hx,
                                       uint8_t* hm, float* ht, int local, const uint8_t* code, const int* brick_level,
                                       const double* level_h)
        {
            const int k = blockIdx.x;
            const int64_t sample = pair * per_pair + k;
            if (sample >= capacity) return;
            uint64_t h = seed ^ (uint64_t(pair) * 0x9E3779B97F4A7C15ull) ^ (uint64_t(k) * 0xC2B2AE3D27D4EB4Full);
            h ^= h >> 33; h *= 0xff51afd7ed558ccdull; h ^= h >> 33; h *= 0xc4ceb9fe1a85ec53ull; h ^= h >> 33;
            const int b = int(h % uint64_t(bricks));
            const int64_t q0 = int64_t(slots[b]) * 512;
            __shared__ double red[2][8];
            double q[2], ss = 0, cnt = 0;
            for (int j = 0; j < 2; ++j)
            {
                const int64_t qq = q0 + threadIdx.x + 256 * j;
                q[j] = active[qq] && diag[qq] > 0 ? r[qq] / diag[qq] : 0.0;
                ss += q[j] * q[j];
                cnt += active[qq] ? 1.0 : 0.0;
            }
            for (int o = 16; o; o >>= 1) { ss += __shfl_xor_sync(0xffffffffu, ss, o); cnt += __shfl_xor_sync(0xffffffffu, cnt, o); }
            if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = ss; red[1][threadIdx.x >> 5] = cnt; }
            __syncthreads();
            double tss = 0, tcnt = 0;
            for (int w = 0; w < 8; ++w) { tss += red[0][w]; tcnt += red[1][w]; }
            double s = std::sqrt(tss / fmax(tcnt, 1.0));
            if (!(s > 0)) s = 1.0;
            __shared__ double bs[512], xs[512], ps[512], Ds[512], red2[8];
            __shared__ uint8_t cs[512];
            if (local)
            {
                for (int j = 0; j < 2; ++j)
                {
                    const int v = threadIdx.x + 256 * j;
                    const int64_t qq = q0 + v;
                    const bool on = active[qq] && diag[qq] > 0;
                    bs[v] = on ? r[qq] : 0.0;
                    Ds[v] = on ? diag[qq] : 0.0;
                    cs[v] = on ? code[qq] : 0;
                }
                __syncthreads();
                brick_solve(bs, xs, cs, Ds, level_h[brick_level[slots[b]]], ps, red2);
            }
            for (int j = 0; j < 2; ++j)
            {
                const int v = threadIdx.x + 256 * j;
                const int64_t qq = q0 + v;
                hx[sample * 512 + v] = __float2bfloat16_rn(float(q[j] / s));
                hm[sample * 512 + v] = active[qq] ? 1 : 0;
                const double target = local ? xs[v] : z[qq];
                ht[sample * 512 + v] = active[qq] ? float(target / s) : 0.0f;
            }
        }

        // sum of squared targets and active count over the harvest store
        __global__ void target_moment_kernel(int64_t n, const uint8_t* hm, const float* ht, double* out)
        {
            double ss = 0, cnt = 0;
            for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
                if (hm[i]) { ss += double(ht[i]) * ht[i]; cnt += 1; }
            for (int o = 16; o; o >>= 1) { ss += __shfl_xor_sync(0xffffffffu, ss, o); cnt += __shfl_xor_sync(0xffffffffu, cnt, o); }
            if ((threadIdx.x & 31) == 0) { atomicAdd(&out[0], ss); atomicAdd(&out[1], cnt); }
        }

        // training batch: x0 [batch][512][16], target * target_scale, mask; count += active cells
        __global__ void gather_batch_kernel(const int* index, int batch, const bf16* hx, const uint8_t* hm, const float* ht, float target_scale,
                                            bf16* x0, float* target, uint8_t* mask, float* count)
        {
            const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (i >= int64_t(batch) * 512) return;
            const int b = int(i / 512), v = int(i % 512);
            const int64_t src = int64_t(index[b]) * 512 + v;
            float f[8] = {__bfloat162float(hx[src]), float(hm[src]), 0, 0, 0, 0, 0, 0}, zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint4* o = reinterpret_cast<uint4*>(x0 + i * 16);
            o[0] = pack8(f);
            o[1] = pack8(zero);
            target[i] = ht[src] * target_scale;
            mask[i] = hm[src];
            if (hm[src]) atomicAdd(count, 1.0f);
        }

        // head forward + backward: zhat, loss, dhead, G4 = bf16(dz * head * [d0 > 0])
        __global__ void head_backward_kernel(int samples, const bf16* d0, const float* head, const float* target, const uint8_t* mask,
                                             const float* count, float* zhat, bf16* G4, float* dhead, float* loss)
        {
            const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            float f[16], part[16], l = 0;
            for (int c = 0; c < 16; ++c) part[c] = 0;
            if (i < int64_t(samples) * 512)
            {
                const uint4* src = reinterpret_cast<const uint4*>(d0 + i * 16);
                unpack8(src[0], f);
                unpack8(src[1], f + 8);
                float acc = 0;
                for (int c = 0; c < 16; ++c) acc += f[c] * head[c];
                zhat[i] = acc;
                const float inv = 1.0f / fmaxf(*count, 1.0f);
                const float diff = mask[i] ? acc - target[i] : 0.0f;
                l = diff * diff * inv;
                const float dz = 2.0f * diff * inv;
                float g[16];
                for (int c = 0; c < 16; ++c)
                {
                    part[c] = f[c] * dz;
                    g[c] = f[c] > 0 ? dz * head[c] : 0.0f;
                }
                uint4* o = reinterpret_cast<uint4*>(G4 + i * 16);
                o[0] = pack8(g);
                o[1] = pack8(g + 8);
            }
            for (int o = 16; o; o >>= 1)
            {
                l += __shfl_xor_sync(0xffffffffu, l, o);
                for (int c = 0; c < 16; ++c) part[c] += __shfl_xor_sync(0xffffffffu, part[c], o);
            }
            if ((threadIdx.x & 31) == 0)
            {
                atomicAdd(loss, l);
                for (int c = 0; c < 16; ++c) atomicAdd(&dhead[c], part[c]);
            }
        }

        // G = bf16(sum over the 8 children of U (fine level 2n) * [act > 0]) at level n
        __global__ void sum_children_relu_kernel(int samples, int n, int C, const float* U, const bf16* act, bf16* G)
        {
            const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            const int V = n * n * n;
            if (i >= int64_t(samples) * V * C) return;
            const int c = int(i % C);
            const int64_t vb = i / C;
            const int v = int(vb % V);
            const int64_t b = vb / V;
            const int x = v % n, y = (v / n) % n, z = v / (n * n), F = 2 * n;
            float sum = 0;
            for (int k = 0; k < 8; ++k)
            {
                const int fx = 2 * x + (k & 1), fy = 2 * y + ((k >> 1) & 1), fz = 2 * z + (k >> 2);
                sum += U[((b * F + fz) * F + fy) * int64_t(F) * C + int64_t(fx) * C + c];
            }
            G[i] = __float2bfloat16_rn(__bfloat162float(act[i]) > 0 ? sum : 0.0f);
        }

        // G = bf16((S + P[parent] / 8) * [act > 0]) at level n (P at level n/2)
        __global__ void combine_relu_kernel(int samples, int n, int C, const float* S, const float* P, const bf16* act, bf16* G)
        {
            const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            const int V = n * n * n;
            if (i >= int64_t(samples) * V * C) return;
            const int c = int(i % C);
            const int64_t vb = i / C;
            const int v = int(vb % V);
            const int64_t b = vb / V;
            const int x = v % n, y = (v / n) % n, z = v / (n * n), M = n / 2;
            const float parent = P[((b * M + z / 2) * M + y / 2) * int64_t(M) * C + int64_t(x / 2) * C + c];
            G[i] = __float2bfloat16_rn(__bfloat162float(act[i]) > 0 ? S[i] + 0.125f * parent : 0.0f);
        }

        // dW[t][co][ci] += sum_b sum_v G[b][v][co] * src[b][v + shift_t][ci] (FP32, CUDA cores).
        // Block: 256 threads, each owning a 4 (co) x 4 (ci) block of one tap; blockIdx.y walks a
        // chunk of samples, staging the padded source and G of one sample at a time.
        template <int N>
        __global__ void __launch_bounds__(256) weight_grad_kernel(ConvSource s, const bf16* G, int cout, int samples, int chunk, float* dW)
        {
            constexpr int XP = N + 2, P = XP * XP * XP, V = N * N * N;
            extern __shared__ __align__(16) uint8_t wsm[];
            const int C = s.channels;
            bf16* xs = reinterpret_cast<bf16*>(wsm);        // [P][C]
            bf16* gs = xs + P * C;                          // [V][cout]
            const int cb = cout / 4, ib = C / 4;
            const int e = blockIdx.x * 256 + threadIdx.x;
            const bool owner = e < 27 * cb * ib;
            const int tap = owner ? e / (cb * ib) : 0, co0 = owner ? 4 * ((e / ib) % cb) : 0, ci0 = owner ? 4 * (e % ib) : 0;
            const int shift = ((tap / 9) - 1) * XP * XP + ((tap / 3) % 3 - 1) * XP + (tap % 3) - 1;
            float acc[16];
            for (int k = 0; k < 16; ++k) acc[k] = 0;
            const int first = blockIdx.y * chunk, last = min(samples, first + chunk);
            for (int b = first; b < last; ++b)
            {
                __syncthreads();
                for (int i = threadIdx.x; i < P * C / 8; i += 256) reinterpret_cast<uint4*>(xs)[i] = make_uint4(0, 0, 0, 0);
                __syncthreads();
                for (int i = threadIdx.x; i < V * (C / 8); i += 256)
                {
                    const int v = i / (C / 8), c0 = 8 * (i % (C / 8));
                    const int x = v % N, y = (v / N) % N, z = v / (N * N);
                    reinterpret_cast<uint4*>(xs + (((z + 1) * XP + y + 1) * XP + x + 1) * C + c0)[0] = load_source<N>(s, b, x, y, z, c0);
                }
                for (int i = threadIdx.x; i < V * cout / 8; i += 256)
                    reinterpret_cast<uint4*>(gs)[i] = reinterpret_cast<const uint4*>(G + int64_t(b) * V * cout)[i];
                __syncthreads();
                if (!owner) continue;
                for (int v = 0; v < V; ++v)
                {
                    const int x = v % N, y = (v / N) % N, z = v / (N * N);
                    const int pos = ((z + 1) * XP + y + 1) * XP + x + 1 + shift;
                    float g[4], xv[4];
                    for (int k = 0; k < 4; ++k)
                    {
                        g[k] = __bfloat162float(gs[v * cout + co0 + k]);
                        xv[k] = __bfloat162float(xs[pos * C + ci0 + k]);
                    }
                    for (int a = 0; a < 4; ++a)
                        for (int c = 0; c < 4; ++c) acc[4 * a + c] += g[a] * xv[c];
                }
            }
            if (!owner) return;
            for (int a = 0; a < 4; ++a)
                for (int c = 0; c < 4; ++c)
                    atomicAdd(&dW[(int64_t(tap) * cout + co0 + a) * C + ci0 + c], acc[4 * a + c]);
        }

        // BF16 forward weights, BF16 transposed weights (taps flipped, channels swapped) and the
        // BF16-rounded head from the FP32 masters
        __global__ void convert_weights_kernel(const float* master, bf16* forward, bf16* transposed, float* head)
        {
            const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (i >= kParams) return;
            if (i >= kWeights)
            {
                head[i - kWeights] = __bfloat162float(__float2bfloat16_rn(master[i]));
                return;
            }
            int k = 0;
            while (k < 6 && i >= tensor_offset(k + 1)) ++k;
            const int64_t local = i - tensor_offset(k);
            const int cout = tensor_cout(k), cin = tensor_cin(k);
            const int tap = int(local / (int64_t(cout) * cin)), co = int((local / cin) % cout), ci = int(local % cin);
            const bf16 w = __float2bfloat16_rn(master[i]);
            forward[i] = w;
            transposed[tensor_offset(k) + (int64_t(26 - tap) * cin + ci) * cout + co] = w;
        }

        __global__ void adam_kernel(float* master, float* m, float* v, const float* grad, float lr, float b1, float b2, float c1, float c2)
        {
            const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (i >= kParams) return;
            const float g = grad[i];
            const float mi = b1 * m[i] + (1 - b1) * g, vi = b2 * v[i] + (1 - b2) * g * g;
            m[i] = mi;
            v[i] = vi;
            master[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
        }
    }

    // ==================================================================================
    // state
    // ==================================================================================
    struct Learned
    {
        DBuf<float> master, adam_m, adam_v, grad, head;
        DBuf<bf16> wf, wt;          // forward / transposed BF16 weights, flat parameter order
        bool has_weights = false;
        int64_t adam_step = 0;
        // activations for `capacity` samples
        int capacity = 0;
        DBuf<bf16> x0, e0, e1, bt, d1, d0, G4, G3, G2, G1, G0;
        DBuf<float> U0, S0, U1, S1, P1, P0, scale, zhat, target;
        DBuf<uint8_t> mask;
        DBuf<int> batch_index;
        DBuf<float> scalars;        // [0] count, [1] loss
        DBuf<int> error;
        bool harvesting = false;
        uint64_t wait_ns = kMaxWaitNs;   // limit of each tensor-core wait
        bool idle_wait_once = false;     // the next convolution's first wait runs out (fault-path check)
    };

    namespace
    {
        // Harvested training bricks.  One store per process (the device of the first system that
        // harvests), shared by every system, so pairs from several grids accumulate.
        struct Store
        {
            int device = -1, per_pair = 0, local = 1;
            int64_t capacity = 0, pairs = 0;
            uint64_t seed = 0;
            DBuf<bf16> hx;          // [capacity][512] D^-1 r / s
            DBuf<uint8_t> hm;       // [capacity][512] active mask
            DBuf<float> ht;         // [capacity][512] z / s
            int64_t samples() const { return std::min(pairs * per_pair, capacity); }
        };
        Store& store()
        {
            static Store* st = new Store();   // never destroyed: the CUDA context may be gone at exit
            return *st;
        }
    }

    namespace
    {
        bf16* wf(Learned& L, int k) { return L.wf.p + tensor_offset(k); }
        bf16* wt(Learned& L, int k) { return L.wt.p + tensor_offset(k); }

        void ensure_capacity(Learned& L, int samples)
        {
            if (samples <= L.capacity) return;
            const size_t n = size_t(samples);
            L.x0.alloc(n * 512 * 16); L.e0.alloc(n * 512 * 16); L.e1.alloc(n * 64 * 32); L.bt.alloc(n * 8 * 64);
            L.d1.alloc(n * 64 * 32); L.d0.alloc(n * 512 * 16);
            L.G4.alloc(n * 512 * 16); L.G3.alloc(n * 64 * 32); L.G2.alloc(n * 8 * 64); L.G1.alloc(n * 64 * 32); L.G0.alloc(n * 512 * 16);
            L.U0.alloc(n * 512 * 32); L.S0.alloc(n * 512 * 16); L.U1.alloc(n * 64 * 64); L.S1.alloc(n * 64 * 32);
            L.P1.alloc(n * 8 * 32); L.P0.alloc(n * 64 * 16);
            L.scale.alloc(n); L.zhat.alloc(n * 512); L.target.alloc(n * 512); L.mask.alloc(n * 512); L.batch_index.alloc(n);
            L.capacity = samples;
        }

        Learned& state(System& s)
        {
            if (!s.learned)
            {
                s.learned = new Learned();
                Learned& L = *s.learned;
                L.master.alloc(kParams); L.adam_m.alloc(kParams); L.adam_v.alloc(kParams); L.grad.alloc(kParams);
                L.head.alloc(kHead); L.wf.alloc(kWeights); L.wt.alloc(kWeights);
                L.scalars.alloc(4); L.error.alloc(1);
            }
            return *s.learned;
        }

        int sm_count(System& s)
        {
            static int count = 0;
            if (!count) cuda_check(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, s.device), "SM count");
            return count;
        }

        template <int N>
        void conv(System& s, Learned& L, int samples, int cout, ConvSource a, const ConvSource* b, void* y, bool relu, bool fp32)
        {
            if (!samples) return;
            ConvParams p{};
            p.src[0] = a;
            p.sources = 1;
            if (b) { p.src[1] = *b; p.sources = 2; }
            for (int k = 0; k < p.sources; ++k)
                require(p.src[k].channels % 16 == 0 && p.src[k].channels <= 64, "learned: channel count");
            require(cout % 16 == 0 && cout <= 64 && Geometry<N>::T * cout <= 512, "learned: output channels");
            p.cout = cout;
            p.samples = samples;
            p.relu = relu;
            p.out_fp32 = fp32;
            p.y = y;
            p.error = L.error;
            p.wait_ns = L.wait_ns;
            p.idle_wait = L.idle_wait_once ? 1 : 0;
            L.idle_wait_once = false;
            const size_t smem = conv_smem<N>(cout);
            static size_t configured[3] = {0, 0, 0};
            const int slot = N == 8 ? 0 : N == 4 ? 1 : 2;
            if (smem > configured[slot])
            {
                cuda_check(cudaFuncSetAttribute(conv_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "conv smem");
                configured[slot] = smem;
            }
            const int groups = (samples + Geometry<N>::NB - 1) / Geometry<N>::NB;
            const int per_sm = smem > 114 * 1024 ? 1 : smem > 76 * 1024 ? 2 : 3;
            const int grid = std::min(groups, sm_count(s) * per_sm);
            conv_kernel<N><<<grid, 128, smem, launch_stream(s)>>>(p);
            cuda_check(cudaGetLastError(), "conv launch");
        }

        template <int N> void weight_grad(System& s, ConvSource src, const bf16* G, int cout, int samples, float* dW)
        {
            constexpr int P = (N + 2) * (N + 2) * (N + 2), V = N * N * N;
            const size_t smem = size_t(P) * src.channels * 2 + size_t(V) * cout * 2;
            require(smem <= 200 * 1024, "learned: weight-gradient staging");
            static size_t configured[3] = {0, 0, 0};
            const int slot = N == 8 ? 0 : N == 4 ? 1 : 2;
            if (smem > configured[slot])
            {
                cuda_check(cudaFuncSetAttribute(weight_grad_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)), "wgrad smem");
                configured[slot] = smem;
            }
            const int entries = 27 * (cout / 4) * (src.channels / 4);
            const int chunk = 8;
            dim3 grid((entries + 255) / 256, (samples + chunk - 1) / chunk);
            weight_grad_kernel<N><<<grid, 256, smem, launch_stream(s)>>>(src, G, cout, samples, chunk, dW);
        }

        ConvSource source(const bf16* x, const bf16* w, int channels, int mode) { return ConvSource{x, w, channels, mode}; }

        // forward from L.x0 through d0 for `samples` samples
        void forward(System& s, Learned& L, int samples)
        {
            conv<8>(s, L, samples, 16, source(L.x0, wf(L, ENC0), 16, SAME), nullptr, L.e0, true, false);
            conv<4>(s, L, samples, 32, source(L.e0, wf(L, ENC1), 16, POOL), nullptr, L.e1, true, false);
            conv<2>(s, L, samples, 64, source(L.e1, wf(L, BOTT), 32, POOL), nullptr, L.bt, true, false);
            const ConvSource skip1 = source(L.e1, wf(L, DEC1B), 32, SAME);
            conv<4>(s, L, samples, 32, source(L.bt, wf(L, DEC1A), 64, UP), &skip1, L.d1, true, false);
            const ConvSource skip0 = source(L.e0, wf(L, DEC0B), 16, SAME);
            conv<8>(s, L, samples, 16, source(L.d1, wf(L, DEC0A), 32, UP), &skip0, L.d0, true, false);
        }

        // backward from the loss on L.target / L.mask; gradients accumulate into L.grad (zeroed here)
        void backward(System& s, Learned& L, int samples)
        {
            cuda_check(cudaMemsetAsync(L.grad, 0, kParams * sizeof(float), s.stream), "zero gradients");
            cuda_check(cudaMemsetAsync(L.scalars.p + 1, 0, sizeof(float), s.stream), "zero loss");
            float* g = L.grad;
            const int64_t V8 = int64_t(samples) * 512;
            head_backward_kernel<<<blocks_for(V8), kThreads, 0, launch_stream(s)>>>(samples, L.d0, L.head, L.target, L.mask, L.scalars.p,
                                                                                     L.zhat, L.G4, g + kWeights, L.scalars.p + 1);
            // dec0
            conv<8>(s, L, samples, 32, source(L.G4, wt(L, DEC0A), 16, SAME), nullptr, L.U0, false, true);
            conv<8>(s, L, samples, 16, source(L.G4, wt(L, DEC0B), 16, SAME), nullptr, L.S0, false, true);
            weight_grad<8>(s, source(L.d1, nullptr, 32, UP), L.G4, 16, samples, g + tensor_offset(DEC0A));
            weight_grad<8>(s, source(L.e0, nullptr, 16, SAME), L.G4, 16, samples, g + tensor_offset(DEC0B));
            sum_children_relu_kernel<<<blocks_for(int64_t(samples) * 64 * 32), kThreads, 0, launch_stream(s)>>>(samples, 4, 32, L.U0, L.d1, L.G3);
            // dec1
            conv<4>(s, L, samples, 64, source(L.G3, wt(L, DEC1A), 32, SAME), nullptr, L.U1, false, true);
            conv<4>(s, L, samples, 32, source(L.G3, wt(L, DEC1B), 32, SAME), nullptr, L.S1, false, true);
            weight_grad<4>(s, source(L.bt, nullptr, 64, UP), L.G3, 32, samples, g + tensor_offset(DEC1A));
            weight_grad<4>(s, source(L.e1, nullptr, 32, SAME), L.G3, 32, samples, g + tensor_offset(DEC1B));
            sum_children_relu_kernel<<<blocks_for(int64_t(samples) * 8 * 64), kThreads, 0, launch_stream(s)>>>(samples, 2, 64, L.U1, L.bt, L.G2);
            // bottleneck
            conv<2>(s, L, samples, 32, source(L.G2, wt(L, BOTT), 64, SAME), nullptr, L.P1, false, true);
            weight_grad<2>(s, source(L.e1, nullptr, 32, POOL), L.G2, 64, samples, g + tensor_offset(BOTT));
            combine_relu_kernel<<<blocks_for(int64_t(samples) * 64 * 32), kThreads, 0, launch_stream(s)>>>(samples, 4, 32, L.S1, L.P1, L.e1, L.G1);
            // enc1
            conv<4>(s, L, samples, 16, source(L.G1, wt(L, ENC1), 32, SAME), nullptr, L.P0, false, true);
            weight_grad<4>(s, source(L.e0, nullptr, 16, POOL), L.G1, 32, samples, g + tensor_offset(ENC1));
            combine_relu_kernel<<<blocks_for(int64_t(samples) * 512 * 16), kThreads, 0, launch_stream(s)>>>(samples, 8, 16, L.S0, L.P0, L.e0, L.G0);
            // enc0
            weight_grad<8>(s, source(L.x0, nullptr, 16, SAME), L.G0, 16, samples, g + tensor_offset(ENC0));
        }

        void convert(System& s, Learned& L)
        {
            convert_weights_kernel<<<blocks_for(kParams), kThreads, 0, launch_stream(s)>>>(L.master, L.wf, L.wt, L.head);
            L.has_weights = true;
        }

        void check_error(System& s, Learned& L)
        {
            int e = 0;
            cuda_check(cudaMemcpyAsync(&e, L.error, sizeof(int), cudaMemcpyDeviceToHost, s.stream), "learned error flag");
            cuda_check(cudaStreamSynchronize(s.stream), "learned sync");
            if (e)
            {
                cuda_check(cudaMemsetAsync(L.error, 0, sizeof(int), s.stream), "reset error flag");
                throw Error(PCFD_TIMEOUT, "learned preconditioner: a tensor-core wait timed out");
            }
        }

        void default_parameters(System& s, Learned& L)
        {
            // He-normal weights from a fixed seed, as oracle/unet.py init_params draws them in shape
            std::vector<float> p(static_cast<size_t>(kParams));
            std::mt19937_64 rng(20261203);
            std::normal_distribution<double> normal(0.0, 1.0);
            for (int k = 0; k < 7; ++k)
            {
                const double sd = std::sqrt(2.0 / (27.0 * tensor_cin(k)));
                for (int64_t i = 0; i < tensor_size(k); ++i) p[size_t(tensor_offset(k) + i)] = float(sd * normal(rng));
            }
            for (int c = 0; c < kHead; ++c) p[size_t(kWeights + c)] = float(0.25 * normal(rng));
            cuda_check(cudaMemcpyAsync(L.master, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice, s.stream), "upload parameters");
            convert(s, L);
        }
    }

    // ==================================================================================
    // entry points used by the solver and the C ABI
    // ==================================================================================
    int64_t learned_parameter_count() { return kParams; }

    void learned_destroy(System& s)
    {
        delete s.learned;
        s.learned = nullptr;
    }

    void learned_set_parameters(System& s, const float* host, int64_t count)
    {
        require(count == kParams, "learned: parameter count mismatch");
        Learned& L = state(s);
        cuda_check(cudaMemcpyAsync(L.master, host, size_t(kParams) * sizeof(float), cudaMemcpyHostToDevice, s.stream), "upload parameters");
        cuda_check(cudaMemsetAsync(L.adam_m, 0, size_t(kParams) * sizeof(float), s.stream), "reset adam");
        cuda_check(cudaMemsetAsync(L.adam_v, 0, size_t(kParams) * sizeof(float), s.stream), "reset adam");
        L.adam_step = 0;
        convert(s, L);
        cuda_check(cudaStreamSynchronize(s.stream), "set parameters");
    }

    void learned_get_parameters(System& s, float* host, int64_t count)
    {
        require(count == kParams, "learned: parameter count mismatch");
        Learned& L = state(s);
        if (!L.has_weights) default_parameters(s, L);
        cuda_check(cudaMemcpyAsync(host, L.master, size_t(kParams) * sizeof(float), cudaMemcpyDeviceToHost, s.stream), "download parameters");
        cuda_check(cudaStreamSynchronize(s.stream), "get parameters");
    }

    // z = net(r) on the structured bricks, one damped Jacobi step on the DOFs after them
    void learned_apply(System& s, const double* r, double* z)
    {
        Learned& L = state(s);
        if (!L.has_weights) default_parameters(s, L);
        const int bricks = s.active_bricks;
        ensure_capacity(L, bricks);
        cuda_check(cudaMemsetAsync(z, 0, size_t(s.structured) * sizeof(double), s.stream), "clear z");
        if (bricks)
        {
            prepare_kernel<<<bricks, 256, 0, launch_stream(s)>>>(s.active_brick_list, bricks, r, s.diagonal, s.active, L.x0, L.scale);
            forward(s, L, bricks);
            head_apply_kernel<<<blocks_for(int64_t(bricks) * 512), kThreads, 0, launch_stream(s)>>>(s.active_brick_list, bricks, L.d0, L.head,
                                                                                                   L.scale, s.active, z);
        }
        if (s.Sp > s.structured)
            jacobi_tail_kernel<<<blocks_for(int64_t(s.Sp) - s.structured), kThreads, 0, launch_stream(s)>>>(s.structured, s.S, r, s.diagonal,
                                                                                                          s.active, z);
    }

    void learned_check(System& s)
    {
        if (s.learned) check_error(s, *s.learned);
    }

    void learned_set_wait(System& s, double seconds, bool idle_barrier_once)
    {
        require(seconds > 0 && seconds <= 60, "learned: wait limit must be in (0, 60] s");
        Learned& L = state(s);
        L.wait_ns = uint64_t(seconds * 1e9);
        L.idle_wait_once = idle_barrier_once;
    }

    void learned_harvest_begin(System& s, int capacity_pairs, int per_pair, uint64_t seed, int target)
    {
        require(capacity_pairs > 0 && per_pair > 0 && per_pair <= 4096, "learned: harvest sizes");
        require(target == PCFD_LEARNED_TARGET_MULTIGRID || target == PCFD_LEARNED_TARGET_BRICK_SOLVE, "learned: harvest target");
        require(target == PCFD_LEARNED_TARGET_MULTIGRID || s.fine.enabled, "learned: the brick-solve target needs 8^3 bricks");
        Learned& L = state(s);
        Store& st = store();
        require(st.device < 0 || st.device == s.device, "learned: the harvest store lives on another device");
        const int64_t capacity = int64_t(capacity_pairs) * per_pair;
        if (capacity != st.capacity || per_pair != st.per_pair || target != st.local)
        {
            cuda_check(cudaStreamSynchronize(s.stream), "harvest store");
            st.hx.alloc(size_t(capacity) * 512);
            st.hm.alloc(size_t(capacity) * 512);
            st.ht.alloc(size_t(capacity) * 512);
            st.capacity = capacity;
            st.per_pair = per_pair;
            st.pairs = 0;
            st.device = s.device;
            st.local = target;
        }
        st.seed = seed;
        L.harvesting = true;
    }

    int64_t learned_harvest_stop(System& s)
    {
        if (s.learned) s.learned->harvesting = false;
        return store().samples();
    }

    bool learned_harvesting(const System& s) { return s.learned && s.learned->harvesting; }

    void learned_harvest(System& s, const double* r, const double* z)
    {
        Store& st = store();
        if (!s.active_bricks || st.pairs * st.per_pair >= st.capacity) return;
        harvest_kernel<<<st.per_pair, 256, 0, launch_stream(s)>>>(s.active_brick_list, s.active_bricks, st.pairs, st.per_pair,
                                                                  st.seed, st.capacity, r, z, s.diagonal, s.active, st.hx, st.hm, st.ht,
                                                                  st.local, s.fine.code, s.brick_level, s.d_level_h);
        ++st.pairs;
    }

    namespace
    {
        // head master weights *= factor (and the BF16 copies)
        void scale_head(System& s, Learned& L, double factor)
        {
            float h[kHead];
            cuda_check(cudaMemcpyAsync(h, L.master.p + kWeights, sizeof(h), cudaMemcpyDeviceToHost, s.stream), "head");
            cuda_check(cudaStreamSynchronize(s.stream), "head");
            for (float& v : h) v = float(v * factor);
            cuda_check(cudaMemcpyAsync(L.master.p + kWeights, h, sizeof(h), cudaMemcpyHostToDevice, s.stream), "head");
            cuda_check(cudaStreamSynchronize(s.stream), "head");
            convert(s, L);
        }

        // one optimiser step on L.x0 / target / mask for `batch` samples; returns nothing (loss on device)
        void train_step(System& s, Learned& L, int batch, float lr)
        {
            forward(s, L, batch);
            backward(s, L, batch);
            ++L.adam_step;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.0f - std::pow(b1, float(L.adam_step)), c2 = 1.0f - std::pow(b2, float(L.adam_step));
            adam_kernel<<<blocks_for(kParams), kThreads, 0, launch_stream(s)>>>(L.master, L.adam_m, L.adam_v, L.grad, lr, b1, b2, c1, c2);
            convert(s, L);
        }
    }

    // `steps` Adam steps on random batches of the harvested samples; returns the mean loss of the
    // last min(steps, 50) steps
    double learned_train(System& s, int steps, int batch, double lr, uint64_t seed)
    {
        require(steps >= 0 && batch > 0 && lr > 0, "learned: training arguments");
        Learned& L = state(s);
        if (!L.has_weights) default_parameters(s, L);
        Store& st = store();
        const int64_t samples = st.samples();
        require(samples > 0 && st.device == s.device, "learned: no harvested samples on this device to train on");
        ensure_capacity(L, batch);
        // Targets (multigrid corrections over D^-1 r / s) are 10^2..10^4 in size: train against
        // targets divided by their RMS tau over the store, with the head divided by tau, and fold
        // tau back into the head afterwards (the head is linear, so the trained map is unchanged).
        double tau = 1.0;
        {
            DBuf<double> moment;
            moment.alloc(2);
            target_moment_kernel<<<4 * sm_count(s), 256, 0, launch_stream(s)>>>(samples * 512, st.hm, st.ht, moment);
            double h[2] = {0, 0};
            cuda_check(cudaMemcpyAsync(h, moment.p, sizeof(h), cudaMemcpyDeviceToHost, s.stream), "target moment");
            cuda_check(cudaStreamSynchronize(s.stream), "target moment");
            if (h[1] > 0 && h[0] > 0) tau = std::sqrt(h[0] / h[1]);
        }
        scale_head(s, L, 1.0 / tau);
        cuda_check(cudaMemsetAsync(L.adam_m, 0, size_t(kParams) * sizeof(float), s.stream), "reset adam");
        cuda_check(cudaMemsetAsync(L.adam_v, 0, size_t(kParams) * sizeof(float), s.stream), "reset adam");
        L.adam_step = 0;
        std::mt19937_64 rng(seed);
        std::vector<int> index(static_cast<size_t>(batch));
        std::vector<float> losses;
        const int tail = std::min(steps, 50);
        float* pinned = nullptr;
        cuda_check(cudaMallocHost(&pinned, size_t(std::max(tail, 1)) * sizeof(float)), "pinned losses");
        try
        {
            for (int step = 0; step < steps; ++step)
            {
                for (int& i : index) i = int(rng() % uint64_t(samples));
                cuda_check(cudaMemcpyAsync(L.batch_index, index.data(), index.size() * sizeof(int), cudaMemcpyHostToDevice, s.stream),
                           "batch indices");
                cuda_check(cudaMemsetAsync(L.scalars, 0, sizeof(float), s.stream), "zero count");
                gather_batch_kernel<<<blocks_for(int64_t(batch) * 512), kThreads, 0, launch_stream(s)>>>(L.batch_index, batch, st.hx, st.hm,
                                                                                                        st.ht, float(1.0 / tau), L.x0, L.target,
                                                                                                        L.mask, L.scalars);
                // cosine decay to 10 % of the initial rate
                const double frac = steps > 1 ? double(step) / double(steps - 1) : 0.0;
                const float rate = float(lr * (0.1 + 0.45 * (1.0 + std::cos(M_PI * frac))));
                train_step(s, L, batch, rate);
                if (step >= steps - tail)
                    cuda_check(cudaMemcpyAsync(pinned + (step - (steps - tail)), L.scalars.p + 1, sizeof(float), cudaMemcpyDeviceToHost, s.stream),
                               "loss");
                // the host synchronises every 64 steps so that the batch indices stay in order
                if ((step & 63) == 63) cuda_check(cudaStreamSynchronize(s.stream), "train sync");
            }
            check_error(s, L);
            scale_head(s, L, tau);
        }
        catch (...)
        {
            cudaFreeHost(pinned);
            throw;
        }
        double mean = 0;
        for (int i = 0; i < tail; ++i) mean += pinned[i];
        cudaFreeHost(pinned);
        return tail ? mean / tail : 0.0;
    }

    // forward (and, with gradients != null, backward) on host samples: x [n][512][2] (input
    // channel 0 and mask), target [n][512]; returns the loss, zhat [n][512], gradients [params]
    double learned_evaluate(System& s, int n, const float* x, const float* target, float* zhat, float* gradients)
    {
        require(n > 0 && x && target && zhat, "learned: evaluate arguments");
        Learned& L = state(s);
        if (!L.has_weights) default_parameters(s, L);
        ensure_capacity(L, n);
        std::vector<uint16_t> hx(size_t(n) * 512);
        std::vector<uint8_t> hm(size_t(n) * 512);
        std::vector<float> ht(target, target + size_t(n) * 512);
        for (size_t i = 0; i < hx.size(); ++i)
        {
            const bf16 b = __float2bfloat16_rn(x[2 * i]);
            std::memcpy(&hx[i], &b, 2);
            hm[i] = x[2 * i + 1] != 0 ? 1 : 0;
        }
        DBuf<bf16> dx;
        DBuf<uint8_t> dm;
        DBuf<float> dt;
        dx.alloc(hx.size(), false);
        cuda_check(cudaMemcpy(dx.p, hx.data(), hx.size() * 2, cudaMemcpyHostToDevice), "upload inputs");
        dm.upload(hm);
        dt.upload(ht);
        std::vector<int> index(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i) index[size_t(i)] = i;
        cuda_check(cudaMemcpyAsync(L.batch_index, index.data(), index.size() * sizeof(int), cudaMemcpyHostToDevice, s.stream), "indices");
        cuda_check(cudaMemsetAsync(L.scalars, 0, sizeof(float), s.stream), "zero count");
        gather_batch_kernel<<<blocks_for(int64_t(n) * 512), kThreads, 0, launch_stream(s)>>>(L.batch_index, n, dx, dm, dt, 1.0f, L.x0,
                                                                                            L.target, L.mask, L.scalars);
        forward(s, L, n);
        backward(s, L, n);
        float loss = 0;
        cuda_check(cudaMemcpyAsync(&loss, L.scalars.p + 1, sizeof(float), cudaMemcpyDeviceToHost, s.stream), "loss");
        cuda_check(cudaMemcpyAsync(zhat, L.zhat, size_t(n) * 512 * sizeof(float), cudaMemcpyDeviceToHost, s.stream), "zhat");
        if (gradients)
            cuda_check(cudaMemcpyAsync(gradients, L.grad, size_t(kParams) * sizeof(float), cudaMemcpyDeviceToHost, s.stream), "gradients");
        check_error(s, L);
        return loss;
    }
}
