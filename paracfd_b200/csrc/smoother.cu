// smoother.cu -- fused fine-level work of the multigrid preconditioner for 8^3 bricks.
//
// The reference cycle (src/core/fluid/amr_pressure.cu:1103-1154) runs, per application,
// z = w D^-1 r, then three times "t = A_orth z; z += w D^-1 (r - t)", restricts r - A_orth z to
// the level-0 aggregates and prolongs the coarse correction back: ~10 full passes over the FP64
// vectors plus a serial per-aggregate gather.  Here every fine-level stage is one brick-tiled
// launch that reads z (tile + halo staged in shared memory), r and one code byte per DOF:
//   sweep      z_new = z + w (r - A_struct z) / D          (ping-pong buffers)
//   residual   per-brick partial sums of r - A_struct z for each level-0 cell the brick covers
//   prolong    the coarse correction is added while the tile is staged (z + e[aggregate])
// The code byte holds the six open-face bits (both cells active and the face not cut), the
// X-max outlet bit and a "deferred" bit.  Deferred DOFs are those whose operator row has more
// than the structured 7-point part -- compact coarse/fine, embedded or regular edges, gauges,
// EB fragments, a diagonal that the code bits do not reproduce bit for bit -- and a small
// per-DOF "finish" kernel completes them with the reference's irregular gather in the same
// summation order.  Non-deferred rows use D = sum of h over the open faces (+ 2h outlet), which
// equals the assembled diagonal bit for bit (checked at setup); their update is computed as
// z + (r - Az) * (w / D) with w / D from a per-level table instead of a division, and the
// restriction sums in a different (fixed) order -- the only departures from the unfused cycle.
#include "pcfd_internal.h"

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <unordered_map>

namespace pcfd
{
    namespace
    {
        constexpr uint8_t kDeferred = 0x80, kOutlet = 0x40, kOpenMask = 0x3f;
        constexpr int kBS = 8, kC3 = 512;

        // Per active brick (indexed by position in the active list, so that one round trip
        // fetches everything a CTA needs before its data loads): 64 bytes.
        struct BrickMeta
        {
            int slot, level, base, partial;
            int nbr[6];     // active same-level neighbour slot or -1
            int nbase[6];   // level-0 cell of each neighbour's first cell
        };


        struct BrickView
        {
            const BrickMeta* meta;
            const double* level_h;
            const uint8_t* code;
            double prolong;            // scale of the prolonged coarse correction
            // composite cycle: per brick (active-list order = brick rank) the rank of each face
            // neighbour or -1.  Stage 1 is numbered rank * 64 + (i >> 1) + 4 (j >> 1) + 16 (k >> 1),
            // so the prolongation computes a cell's stage-1 row instead of loading it.
            const int* stage_neighbour;
        };

        // Shared tile of one brick plus its face halos: rows of 12 doubles so that interior rows
        // start 16-byte aligned (x = -1 at offset 1, x = 0..7 at 2..9, x = 8 at 10).
        constexpr int kP1 = 12, kP2 = 120, kTileSize = 10 * kP2;
        __device__ inline int tix(int i, int j, int k) { return (k + 1) * kP2 + (j + 1) * kP1 + (i + 2); }
        // Staged right-hand sides and face codes keep each 64-entry z-plane 72 (rhs) or 80 (codes)
        // entries apart, so that the four z-planes a warp reads at once fall on disjoint
        // shared-memory banks; a 16-byte copy never crosses a plane.
        constexpr int kRPlane = 72, kCPlane = 80, kRSize = kBS * kRPlane, kCSize = kBS * kCPlane;
        __device__ inline int rix(int c) { return c + (kRPlane - 64) * (c >> 6); }
        __device__ inline int cix(int c) { return c + (kCPlane - 64) * (c >> 6); }

        // base cell of cell (i,j,k) of a brick at level l whose (0,0,0) cell lies in base cell `b0`
        __device__ inline int base_cell_of(int b0, int l, int i, int j, int k)
        {
            return b0 + ((k >> l) << 6) + ((j >> l) << 3) + (i >> l);
        }

        // Structured 7-point row of cell s of the tile (order -x,+x,-y,+y,-z,+z, then outlet);
        // identical arithmetic to the unfused operator kernel.
        template <class T>
        __device__ inline T structured_row(const T* tile, int s, uint8_t code, T h)
        {
            const T pa = tile[s];
            T Az = T(0);
            if (code & 1) Az += h * (pa - tile[s - 1]);
            if (code & 2) Az += h * (pa - tile[s + 1]);
            if (code & 4) Az += h * (pa - tile[s - kP1]);
            if (code & 8) Az += h * (pa - tile[s + kP1]);
            if (code & 16) Az += h * (pa - tile[s - kP2]);
            if (code & 32) Az += h * (pa - tile[s + kP2]);
            if (code & kOutlet) Az += T(2) * h * pa;
            return Az;
        }

        // Damping over the diagonal, w / D, of a non-deferred row: D is h per open face plus 2h
        // for the outlet, so it is looked up by (open-face count, outlet) per level.
        constexpr int kDiagonalKinds = 14;
        __device__ inline int diagonal_kind(uint8_t code) { return __popc(code & kOpenMask) + 7 * ((code >> 6) & 1); }

        // ---- persistent, double-buffered variant -------------------------------------------
        // Each CTA walks bricks b, b + G, ... and stages brick n+1 (tile + halos, r, codes) with
        // cp.async into the second shared buffer while it computes brick n, so every SM keeps two
        // bricks' loads in flight per CTA; the metadata of brick n+2 is fetched during brick n.
        __device__ inline unsigned smem_addr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
        __device__ inline void copy16(void* dst, const void* src, bool valid)
        {
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 16 : 0));
        }
        __device__ inline void copy8(void* dst, const void* src, bool valid)
        {
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 8 : 0));
        }
        __device__ inline void copy4(void* dst, const void* src, bool valid)
        {
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_addr(dst)), "l"(src), "r"(valid ? 4 : 0));
        }
        // two consecutive values / one value of the field type
        template <class T> __device__ inline void copy_pair(void* dst, const void* src, bool valid)
        {
            if (sizeof(T) == 8) copy16(dst, src, valid);
            else copy8(dst, src, valid);
        }
        template <class T> __device__ inline void copy_one(void* dst, const void* src, bool valid)
        {
            if (sizeof(T) == 8) copy8(dst, src, valid);
            else copy4(dst, src, valid);
        }
        __device__ inline void copy_commit() { asm volatile("cp.async.commit_group;\n" ::); }
        template <int N> __device__ inline void copy_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

        // What one thread needs of a brick: the head and the neighbour of the halo face it copies.
        struct Ticket
        {
            int slot, level, base, partial, nbr, nbase, rank, nrank;
        };
        __device__ inline int halo_face(int t) { return t < 128 ? 2 + (t >> 5) : ((t - 128) >> 6); }
        __device__ inline Ticket load_ticket(const BrickView& v, int64_t b)
        {
            const BrickMeta* m = v.meta + b;
            const int4 h = *reinterpret_cast<const int4*>(m);
            const int face = halo_face(threadIdx.x);
            return Ticket{h.x, h.y, h.z, h.w, m->nbr[face], m->nbase[face], int(b), v.stage_neighbour ? v.stage_neighbour[6 * b + face] : -1};
        }

        template <class T, bool kWithR>
        __device__ inline void issue_brick(const Ticket& k, const T* __restrict__ z, const T* __restrict__ r,
                                           const uint8_t* __restrict__ code, T* tile, T* rbuf, uint8_t* cbuf)
        {
            const int t = threadIdx.x;
            const int64_t base = int64_t(k.slot) * kC3;
            {
                const int c = 2 * t, i = c & 7, j = (c >> 3) & 7, kk = c >> 6;
                copy_pair<T>(tile + tix(i, j, kk), z + base + c, true);
                if (kWithR) copy_pair<T>(rbuf + rix(c), r + base + c, true);
            }
            if (t < 32) copy16(cbuf + cix(16 * t), code + base + 16 * t, true);
            const bool valid = k.nbr >= 0;
            const int64_t nb = int64_t(valid ? k.nbr : k.slot) * kC3;   // any valid address when zero-filling
            if (t < 128)
            {
                const int face = 2 + (t >> 5), w = t & 31;
                int i, j, kk, hj, hk;
                if (face < 4) { kk = w >> 2; i = (w & 3) * 2; j = face == 2 ? kBS - 1 : 0; hj = face == 2 ? -1 : kBS; hk = kk; }
                else { i = (w * 2) & 7; j = (w * 2) >> 3; kk = face == 4 ? kBS - 1 : 0; hj = j; hk = face == 4 ? -1 : kBS; }
                copy_pair<T>(tile + tix(i, hj, hk), z + nb + (kk * kBS + j) * kBS + i, valid);
            }
            else
            {
                const int u = t - 128, face = u >> 6, j = u & 7, kk = (u >> 3) & 7;
                const int i = face == 0 ? kBS - 1 : 0, hi = face == 0 ? -1 : kBS;
                copy_one<T>(tile + tix(hi, j, kk), z + nb + (kk * kBS + j) * kBS + i, valid);
            }
        }

        // Composite cycle: the two stage-1 correction values this thread's prolongation adds, staged
        // with the tile by the thread itself (its own copy wait then covers them): [0] the row of
        // its own two cells (they share a 2x2x2 block), [1] the row of its halo cells in the face
        // neighbour (zero-filled without one).
        template <class TC>
        __device__ inline void issue_stage_values(const Ticket& k, const TC* __restrict__ e, TC* ebuf)
        {
            const int t = threadIdx.x;
            const int c = 2 * t, i = c & 7, j = (c >> 3) & 7, kk = c >> 6;
            copy_one<TC>(ebuf + 2 * t, e + int64_t(k.rank) * 64 + (i >> 1) + 4 * (j >> 1) + 16 * (kk >> 1), true);
            const bool valid = k.nbr >= 0 && k.nrank >= 0;
            int hi, hj, hk;
            if (t < 128)
            {
                const int face = 2 + (t >> 5), w = t & 31;
                if (face < 4) { hk = w >> 2; hi = (w & 3) * 2; hj = face == 2 ? kBS - 1 : 0; }
                else { hi = (w * 2) & 7; hj = (w * 2) >> 3; hk = face == 4 ? kBS - 1 : 0; }
            }
            else
            {
                const int u = t - 128, face = u >> 6;
                hj = u & 7; hk = (u >> 3) & 7; hi = face == 0 ? kBS - 1 : 0;
            }
            copy_one<TC>(ebuf + 2 * t + 1, e + int64_t(valid ? k.nrank : k.rank) * 64 + (hi >> 1) + 4 * (hj >> 1) + 16 * (hk >> 1), valid);
        }

        // adds the coarse correction to the tile entries this thread copied; kMapped: the composite
        // cycle's stage-1 row of the cell (its brick's rank * 64 + the 2x2x2 block of the cell;
        // an inactive cell's tile entry takes a correction too, but no open face reads it), read
        // from the values this thread staged (ebuf), else the geometric level-0 cell
        template <class T, class TC, bool kMapped>
        __device__ inline void prolong_own(const Ticket& k, const TC* __restrict__ e, double scale, T* tile, const TC* ebuf)
        {
            const int t = threadIdx.x, l = k.level;
            auto add = [&](int s_tile, int64_t q, int b0, int i, int j, int kk) {
                if (kMapped) tile[s_tile] += T(scale * double(ebuf[2 * t + b0]));
                else tile[s_tile] += T(scale * double(e[base_cell_of(b0, l, i, j, kk)]));
            };
            {
                const int c = 2 * t, i = c & 7, j = (c >> 3) & 7, kk = c >> 6;
                const int64_t q = int64_t(k.slot) * kC3 + c;
                const int own = kMapped ? 0 : k.base;
                add(tix(i, j, kk), q, own, i, j, kk);
                add(tix(i + 1, j, kk), q + 1, own, i + 1, j, kk);
            }
            if (k.nbr < 0 || (kMapped && k.nrank < 0)) return;
            const int other = kMapped ? 1 : k.nbase;
            const int64_t nb = int64_t(k.nbr) * kC3;
            if (t < 128)
            {
                const int face = 2 + (t >> 5), w = t & 31;
                int i, j, kk, hj, hk;
                if (face < 4) { kk = w >> 2; i = (w & 3) * 2; j = face == 2 ? kBS - 1 : 0; hj = face == 2 ? -1 : kBS; hk = kk; }
                else { i = (w * 2) & 7; j = (w * 2) >> 3; kk = face == 4 ? kBS - 1 : 0; hj = j; hk = face == 4 ? -1 : kBS; }
                const int64_t q = nb + (kk * kBS + j) * kBS + i;
                add(tix(i, hj, hk), q, other, i, j, kk);
                add(tix(i + 1, hj, hk), q + 1, other, i + 1, j, kk);
            }
            else
            {
                const int u = t - 128, face = u >> 6, j = u & 7, kk = (u >> 3) & 7;
                const int i = face == 0 ? kBS - 1 : 0, hi = face == 0 ? -1 : kBS;
                add(tix(hi, j, kk), nb + (kk * kBS + j) * kBS + i, other, i, j, kk);
            }
        }

        // What the rows the structured 7-point part does not complete need: the packed rows and
        // compact edges (other endpoint with its map index, coefficient), gauges, the assembled
        // diagonal.
        struct DeferredView
        {
            const int4* row;
            const int2* edge;
            const double* edge_coefficient;
            const int* gauge_offset;
            const double* gauge_coefficient;
            const double* diag;
            const int* aggregate;          // level-0 aggregate per DOF (reference-cycle prolongation)
            int base_offset, base_cells;
            double omega;
        };

        // Completes deferred row d from its structured part t[a] (structured DOFs) and right-hand
        // side r[a]: the compact-edge gather and the gauges, in the order of the unfused operator.
        // kFinish 0: z_new into out[a], 1: residual into residual[d], 2: residual into out[a].
        // The packed row holds every index the row needs, so its gathers are two loads deep.
        template <int kFinish, class T, class TO, class TC, int kProlong>
        __device__ inline void finish_row(const DeferredView& dv, int d, int64_t structured, const T* __restrict__ z,
                                          const T* __restrict__ r, const T* __restrict__ t, const TC* __restrict__ e,
                                          double scale, TO* __restrict__ out, double* __restrict__ residual)
        {
            const int4 row = dv.row[d];
            const int a = row.x, edges = row.w >> 8, gauges = (row.w >> 2) & 63;
            const bool on = row.w & 1, incident = row.w & 2;
            // the prolonged iterate at DOF q with map index c (active DOFs only)
            auto value = [&](int q, int c) {
                double v = double(z[q]);
                if (kProlong == 2)
                {
                    if (c >= 0) v += scale * double(e[c]);
                }
                else if (kProlong == 1)
                {
                    const int base = dv.aggregate[q] - dv.base_offset;
                    if (base >= 0 && base < dv.base_cells) v += scale * double(e[base]);
                }
                return v;
            };
            // the row's independent loads first, so that they are in flight together
            double Az = a < structured ? double(t[a]) : 0.0;
            const double rc = double(r[a]);
            const double D = dv.diag[a];
            const double za = on ? value(a, row.z) : double(z[a]);
            if (incident)
            {
                // the compact edges' two-point terms, coefficient * (z_a - z_other): the reference's
                // sign * coefficient * (z_lower - z_upper) bit for bit (exact negations)
                double sum = 0.0;
#pragma unroll 2
                for (int q = row.y; q < row.y + edges; ++q)
                {
                    const int2 other = dv.edge[q];
                    sum += dv.edge_coefficient[q] * (za - value(other.x, other.y));
                }
                Az += sum;
            }
            if (gauges)
                for (int g = dv.gauge_offset[d], g1 = g + gauges; g < g1; ++g) Az += dv.gauge_coefficient[g] * za;
            if (kFinish == 0)
            {
                if (!on) out[a] = TO(0);
                else out[a] = TO(D > 0.0 ? za + dv.omega * (rc - Az) / D : za);
            }
            else if (kFinish == 1) residual[d] = on ? rc - Az : 0.0;
            else out[a] = TO(on ? rc - Az : 0.0);
        }

        // CTAs of 256 threads the launch bounds keep resident per SM: six for the float sweeps and
        // the FP64 operator (<= 40 registers, <= 27 KB shared memory), four for the FP64 sweeps.
        template <int kMode, class T> constexpr int pipe_resident() { return (sizeof(T) == 4 || kMode == 2) ? 6 : 4; }

        // kMode 0: Jacobi sweep, 1: residual restriction, 2: structured apply (out = A_struct z)
        // T: field type of z, r, t (double, or float for the FP32 multigrid); TO: output type.
        // kProlong: 0 none, 1 level-0 cell (reference cycle), 2 mapped (composite cycle);
        // kMode 3: write the residual r - A_struct z (composite cycle's first restriction)
        template <int kMode, class T, class TO, class TC, int kProlong>
        __global__ void __launch_bounds__(256, pipe_resident<kMode, T>()) brick_pipe_kernel(BrickView v, int64_t bricks, const T* __restrict__ z,
            const T* __restrict__ r, TO* __restrict__ out, T* __restrict__ t, const TC* __restrict__ e,
            double* __restrict__ partial, const T* __restrict__ damping)
        {
            constexpr bool kWithR = kMode != 2;
            __shared__ __align__(16) T tile[2][kTileSize];
            __shared__ __align__(16) T rbuf[kWithR ? 2 : 1][kRSize];
            __shared__ __align__(16) uint8_t cbuf[2][kCSize];
            __shared__ double residual[kMode == 1 ? kC3 : 1];
            __shared__ __align__(16) TC ebuf[kProlong == 2 ? 2 : 1][kProlong == 2 ? 512 : 1];   // per thread: own, halo
            int64_t b = blockIdx.x;
            if (b >= bricks) return;
            const int64_t G = gridDim.x;
            Ticket cur = load_ticket(v, b);
            issue_brick<T, kWithR>(cur, z, r, v.code, tile[0], rbuf[0], cbuf[0]);
            if (kProlong == 2) issue_stage_values<TC>(cur, e, ebuf[0]);
            copy_commit();
            Ticket next = b + G < bricks ? load_ticket(v, b + G) : cur;
            for (int it = 0;; ++it)
            {
                const int st = it & 1;
                const bool has_next = b + G < bricks;
                Ticket after = next;
                if (has_next)
                {
                    issue_brick<T, kWithR>(next, z, r, v.code, tile[st ^ 1], rbuf[kWithR ? (st ^ 1) : 0], cbuf[st ^ 1]);
                    if (kProlong == 2) issue_stage_values<TC>(next, e, ebuf[st ^ 1]);
                    copy_commit();
                    if (b + 2 * G < bricks) after = load_ticket(v, b + 2 * G);
                    copy_wait<1>();
                }
                else copy_wait<0>();
                if (kProlong) prolong_own<T, TC, kProlong == 2>(cur, e, v.prolong, tile[st], ebuf[kProlong == 2 ? st : 0]);
                __syncthreads();
                // ---- compute brick `cur` from buffer st.  Thread t owns cell (i, j, k) = (t & 7,
                // t >> 5, (t >> 3 & 3) + 4 q), q = 0, 1: a warp covers one x-row of 8 cells in each
                // of four consecutive z-planes.  With rows 12 and planes 120 tile entries apart the
                // four rows fall on disjoint shared-memory banks (float: 32 banks, offsets 0, 24, 16,
                // 8 words; double: each half-warp's two rows 240 words apart), so no stencil read
                // replays (the staged rhs and codes are padded per plane for the same reason);
                // consecutive cells of a row make 32- or 64-byte global segments.
                const T* F = tile[st];
                const int l = cur.level;
                const T h = T(v.level_h[l]);
                const int64_t base = int64_t(cur.slot) * kC3;
                const int n = l >= 3 ? 1 : (kBS >> l);
                const int size = l >= 3 ? kC3 : (1 << (3 * l));
                const int mask = (1 << l) - 1;
#pragma unroll
                for (int q = 0; q < 2; ++q)
                {
                    const int i = threadIdx.x & 7, j = threadIdx.x >> 5, k = ((threadIdx.x >> 3) & 3) + 4 * q;
                    const int c = (k * kBS + j) * kBS + i;
                    const int s = tix(i, j, k);
                    const uint8_t code = cbuf[st][cix(c)];
                    const T Az = structured_row<T>(F, s, code, h);
                    if (kMode == 2) out[base + c] = TO(Az);
                    else
                    {
                        const T rc = rbuf[st][rix(c)];
                        if (code & kDeferred) t[base + c] = Az;
                        if (kMode == 0)
                        {
                            if (!(code & kDeferred))
                                out[base + c] = code ? TO(F[s] + (rc - Az) * damping[l * kDiagonalKinds + diagonal_kind(code)]) : TO(0);
                        }
                        else if (kMode == 3)
                        {
                            if (!(code & kDeferred)) out[base + c] = code ? TO(rc - Az) : TO(0);
                        }
                        else
                        {
                            const int group = l >= 3 ? 0 : ((k >> l) * n + (j >> l)) * n + (i >> l);
                            const int within = l >= 3 ? c : ((((k & mask) << l) + (j & mask)) << l) + (i & mask);
                            residual[group * size + within] = (code && !(code & kDeferred)) ? double(rc - Az) : 0.0;
                        }
                    }
                }
                if (kMode == 1)
                {
                    // fixed-order reduction of each aggregate group (groups are contiguous runs of
                    // `size` entries): pair sums, then shuffles inside the group, then warps
                    __syncthreads();
                    const int tt = threadIdx.x;
                    if (size == 1)
                    {
                        partial[cur.partial + 2 * tt] = residual[2 * tt];
                        partial[cur.partial + 2 * tt + 1] = residual[2 * tt + 1];
                    }
                    else
                    {
                        double v = residual[2 * tt] + residual[2 * tt + 1];
                        const int pairs = size >> 1;                         // pairs per group: 4, 32 or 256
                        const int width = pairs < 32 ? pairs : 32;
                        for (int o = width >> 1; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, width);
                        if (pairs <= 32)
                        {
                            if ((tt & (width - 1)) == 0) partial[cur.partial + tt / pairs] = v;
                        }
                        else
                        {
                            __syncthreads();                              // every pair read first
                            if ((tt & 31) == 0) residual[tt >> 5] = v;
                            __syncthreads();
                            if (tt == 0)
                            {
                                double total = 0.0;
                                for (int w = 0; w < 8; ++w) total += residual[w];
                                partial[cur.partial] = total;
                            }
                        }
                    }
                }
                __syncthreads();   // buffer st and the residual scratch are refilled next
                if (!has_next) break;
                b += G;
                cur = next;
                next = after;
            }
        }

        // z = w r / D for every DOF (first sweep from zero); deferred rows read the assembled D.
        // (FP32 multigrid: also writes the float copy of r that the float sweeps read.)
        // Four consecutive DOFs per thread (one code word, two 16-byte r loads, one 16-byte z and
        // r-copy store each), so every thread keeps four entries' loads in flight; the last
        // partial group takes the scalar path.
        template <class T>
        __device__ inline T first_sweep_value(uint8_t c, double rq, int64_t q, int level, const T* __restrict__ damping,
                                              const double* __restrict__ diag, const uint8_t* __restrict__ active, int64_t structured,
                                              double omega)
        {
            if (q >= structured || (c & kDeferred))
            {
                const double D = active[q] ? diag[q] : 0.0;
                return D > 0.0 ? T(omega * rq / D) : T(0);
            }
            return c ? T(rq) * damping[level * kDiagonalKinds + diagonal_kind(c)] : T(0);
        }
        template <class T>
        __global__ void first_sweep_kernel(const uint8_t* __restrict__ code, const int* __restrict__ brick_level,
                                           const T* __restrict__ damping, const double* __restrict__ diag,
                                           const uint8_t* __restrict__ active, const double* __restrict__ r,
                                           T* __restrict__ z, T* __restrict__ r_copy, int64_t structured, int64_t n, double omega)
        {
            const int64_t q0 = 4 * (int64_t(blockIdx.x) * blockDim.x + threadIdx.x);
            if (q0 >= n) return;
            if (q0 + 4 > n)
            {
                for (int64_t q = q0; q < n; ++q)
                {
                    if (r_copy) r_copy[q] = T(r[q]);
                    z[q] = first_sweep_value<T>(code[q], r[q], q, q < structured ? brick_level[q >> 9] : 0, damping, diag, active,
                                                structured, omega);
                }
                return;
            }
            const uchar4 c = *reinterpret_cast<const uchar4*>(code + q0);
            const double2 ra = reinterpret_cast<const double2*>(r + q0)[0], rb = reinterpret_cast<const double2*>(r + q0)[1];
            const int level = q0 < structured ? brick_level[q0 >> 9] : 0;
            T out[4];
            const uint8_t cs[4] = {c.x, c.y, c.z, c.w};
            const double rs[4] = {ra.x, ra.y, rb.x, rb.y};
#pragma unroll
            for (int k = 0; k < 4; ++k) out[k] = first_sweep_value<T>(cs[k], rs[k], q0 + k, level, damping, diag, active, structured, omega);
            if (sizeof(T) == 4)
            {
                *reinterpret_cast<float4*>(z + q0) = make_float4(float(out[0]), float(out[1]), float(out[2]), float(out[3]));
                if (r_copy) *reinterpret_cast<float4*>(r_copy + q0) = make_float4(float(rs[0]), float(rs[1]), float(rs[2]), float(rs[3]));
            }
            else
            {
                reinterpret_cast<double2*>(z + q0)[0] = make_double2(double(out[0]), double(out[1]));
                reinterpret_cast<double2*>(z + q0)[1] = make_double2(double(out[2]), double(out[3]));
                if (r_copy)
                {
                    reinterpret_cast<double2*>(r_copy + q0)[0] = make_double2(rs[0], rs[1]);
                    reinterpret_cast<double2*>(r_copy + q0)[1] = make_double2(rs[2], rs[3]);
                }
            }
        }

        // Brick-local block smoother: z = x_k after k Chebyshev iterations for the brick's diagonal
        // block A_B x = r (x_0 = 0, D^-1 preconditioned), A_B = the full diagonal D minus h for every
        // open face between two cells of the brick.  D^-1 A_B is diagonally dominant, so its
        // spectrum lies in (0, 2); [lo, hi] = [0.06, 2] covers an interior 8^3 block of uniform
        // couplings (1 -+ cos(pi/9)).  One CTA per brick, two cells per thread, the search
        // direction in shared memory; the iteration is a fixed polynomial in D^-1 A_B, so the
        // smoother is linear.
        __global__ void __launch_bounds__(256) block_smooth_kernel(const int* __restrict__ slots, const uint8_t* __restrict__ code,
            const int* __restrict__ brick_level, const double* __restrict__ level_h, const double* __restrict__ diag,
            const uint8_t* __restrict__ active, const double* __restrict__ r, double* __restrict__ z, int iterations, double lo, double hi)
        {
            __shared__ double ds[kC3];
            const int slot = slots[blockIdx.x];
            const int64_t q0 = int64_t(slot) * kC3;
            const double h = level_h[brick_level[slot]];
            double res[2], dinv[2], D[2], x[2], d[2];
            uint8_t c[2];
            const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
            for (int k = 0; k < 2; ++k)
            {
                const int64_t q = q0 + threadIdx.x + 256 * k;
                const bool on = active[q] && diag[q] > 0.0;
                D[k] = on ? diag[q] : 0.0;
                dinv[k] = on ? 1.0 / D[k] : 0.0;
                res[k] = on ? r[q] : 0.0;
                c[k] = on ? uint8_t(code[q] & kOpenMask) : uint8_t(0);
                d[k] = dinv[k] * res[k] / theta;
                x[k] = d[k];
            }
            double rho = 1.0 / sigma;
            for (int it = 1; it < iterations; ++it)
            {
                for (int k = 0; k < 2; ++k) ds[threadIdx.x + 256 * k] = d[k];
                __syncthreads();
                double Ad[2];
                for (int k = 0; k < 2; ++k)
                {
                    const int v = threadIdx.x + 256 * k;
                    const int i = v & 7, j = (v >> 3) & 7, l = v >> 6;
                    double a = D[k] * d[k], nb = 0.0;
                    if ((c[k] & 1) && i > 0) nb += ds[v - 1];
                    if ((c[k] & 2) && i < 7) nb += ds[v + 1];
                    if ((c[k] & 4) && j > 0) nb += ds[v - 8];
                    if ((c[k] & 8) && j < 7) nb += ds[v + 8];
                    if ((c[k] & 16) && l > 0) nb += ds[v - 64];
                    if ((c[k] & 32) && l < 7) nb += ds[v + 64];
                    Ad[k] = a - h * nb;
                }
                __syncthreads();
                const double next = 1.0 / (2.0 * sigma - rho);
                for (int k = 0; k < 2; ++k)
                {
                    res[k] -= Ad[k];
                    d[k] = next * rho * d[k] + (2.0 * next / delta) * dinv[k] * res[k];
                    x[k] += d[k];
                }
                rho = next;
            }
            for (int k = 0; k < 2; ++k) z[q0 + threadIdx.x + 256 * k] = x[k];
        }

        // DOFs after the structured slots (EB fragments): z = w r / D
        __global__ void tail_jacobi_kernel(int64_t begin, int64_t end, const double* __restrict__ r, const double* __restrict__ diag,
                                           const uint8_t* __restrict__ active, double* __restrict__ z, double omega)
        {
            const int64_t q = begin + int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q < end) z[q] = active[q] && diag[q] > 0.0 ? omega * r[q] / diag[q] : 0.0;
        }

        // Completes deferred rows after the pipeline launch: A_orth z = t (structured part) +
        // compact-edge gather + gauges.  One thread per row: the rows are a sparse, irregular
        // subset (cut cells, coarse/fine interfaces), so a launch of their own keeps every SM busy
        // where finishing them inside the brick CTAs left most threads idle (measured slower).
        // kMode 0: z_new, 1: residual into the compact deferred list, 2: residual into out[a]
        template <int kMode, class T, class TO, class TC, int kProlong>
        __global__ void __launch_bounds__(256) finish_deferred_kernel(DeferredView dv, int count, int64_t structured,
                                                                      const TC* __restrict__ e, double scale, const T* __restrict__ z,
                                                                      const T* __restrict__ r, const T* __restrict__ t,
                                                                      TO* __restrict__ out, double* __restrict__ residual)
        {
            const int d = blockIdx.x * blockDim.x + threadIdx.x;
            if (d >= count) return;
            finish_row<kMode, T, TO, TC, kProlong>(dv, d, structured, z, r, t, e, scale, out, residual);
        }

        // map indices of the packed deferred rows and edges (composite cycle)
        __global__ void attach_deferred_map_kernel(int4* __restrict__ row, int rows, int2* __restrict__ edge, int edges,
                                                   const int* __restrict__ map)
        {
            const int i = blockIdx.x * blockDim.x + threadIdx.x;
            if (i < rows) row[i].z = row[i].w & 1 ? map[row[i].x] : -1;
            if (i < edges) edge[i].y = map[edge[i].x];
        }

        // base-level right-hand side: brick partials (levels in order) then deferred-row residuals
        template <class TC>
        __global__ void gather_base_kernel(int cells, const int* __restrict__ offset, const int* __restrict__ entry,
                                           const double* __restrict__ partial, const double* __restrict__ deferred, TC* __restrict__ rhs)
        {
            const int c = blockIdx.x * blockDim.x + threadIdx.x;
            if (c >= cells) return;
            double sum = 0.0;
            for (int q = offset[c]; q < offset[c + 1]; ++q)
            {
                const int x = entry[q];
                sum += x >= 0 ? partial[x] : deferred[-x - 1];
            }
            rhs[c] = TC(sum);
        }
    }

    // ==================================================================================
    // setup
    // ==================================================================================
    void build_fine_smoother(System& s, const pcfd_topology& t, const std::vector<double>& diag)
    {
        FineSmoother& f = s.fine;
        f.enabled = false;
        if (s.bs != kBS || s.mg64.empty()) return;
        const int S = s.S, structured = s.structured;
        std::vector<uint8_t> code(size_t(S), 0);
        std::vector<int> slot_level(size_t(s.B));
        std::vector<const pcfd_level*> slot_lev(size_t(s.B));
        std::vector<int> slot_brick(size_t(s.B));
        for (int l = 0, slot = 0; l < t.level_count; ++l)
            for (int b = 0; b < t.levels[l].brick_count; ++b, ++slot)
            {
                slot_level[slot] = l;
                slot_lev[slot] = &t.levels[l];
                slot_brick[slot] = b;
            }
        // deferred rows: compact-edge incidence, gauges, fragments
        std::vector<uint8_t> deferred(size_t(S), 0);
        const IrregularOperator& o = s.irr;
        std::vector<int> incident_dof(o.incident_dofs);
        if (o.incident_dofs)
            cuda_check(cudaMemcpy(incident_dof.data(), o.incident_dof.p, incident_dof.size() * sizeof(int), cudaMemcpyDeviceToHost),
                       "incidence download");
        for (int q : incident_dof) deferred[q] = 1;
        for (int g = 0; g < t.gauge_count; ++g) deferred[t.gauge_dof[g]] = 1;
        for (int q = structured; q < S; ++q) deferred[q] = t.active[q] ? 1 : 0;
        // open faces per structured DOF, same rules as the unfused operator kernel
        for (int slot = 0; slot < s.B; ++slot)
        {
            const pcfd_level& lev = *slot_lev[slot];
            const int b = slot_brick[slot];
            if (lev.flags[b] & PCFD_BRICK_COVERED) continue;
            const int slot0 = slot - b;
            const double h = lev.h;
            for (int c = 0; c < kC3; ++c)
            {
                const int64_t a = int64_t(slot) * kC3 + c;
                if (!t.active[a]) continue;
                const int ijk[3] = {c & 7, (c >> 3) & 7, c >> 6};
                uint8_t bits = 0;
                for (int axis = 0; axis < 3; ++axis)
                    for (int positive = 0; positive < 2; ++positive)
                    {
                        int q[3] = {ijk[0], ijk[1], ijk[2]};
                        q[axis] += positive ? 1 : -1;
                        int64_t nb = -1;
                        if (q[axis] >= 0 && q[axis] < kBS) nb = int64_t(slot) * kC3 + (q[2] * kBS + q[1]) * kBS + q[0];
                        else
                        {
                            const int n = lev.neighbors[b * 6 + 2 * axis + positive];
                            if (n >= 0 && !(lev.flags[n] & PCFD_BRICK_COVERED))
                            {
                                q[axis] = positive ? 0 : kBS - 1;
                                nb = int64_t(slot0 + n) * kC3 + (q[2] * kBS + q[1]) * kBS + q[0];
                            }
                        }
                        const int64_t lower = positive ? a : nb;
                        if (nb >= 0 && t.active[nb] && !(t.cut_face_mask[lower] & (1u << axis))) bits |= uint8_t(1u << (2 * axis + positive));
                    }
                if (s.outlet && (lev.flags[b] & PCFD_BRICK_XMAX) && ijk[0] == kBS - 1) bits |= kOutlet;
                double D = 0.0;
                for (int face = 0; face < 6; ++face)
                    if (bits & (1 << face)) D += h;
                if (bits & kOutlet) D += 2.0 * h;
                if (!(D > 0.0) || D != diag[a]) deferred[a] = 1;
                code[a] = bits;
            }
        }
        for (int q = 0; q < S; ++q)
            if (deferred[q] && t.active[q]) code[q] |= kDeferred;
        // deferred list with its incidence row and gauge entries (gauge order kept per DOF)
        std::unordered_map<int, int> incident_index;
        for (int n = 0; n < o.incident_dofs; ++n) incident_index[incident_dof[n]] = n;
        std::vector<int> ddof, dinc, goff(1, 0);
        std::vector<double> gcoef;
        std::vector<std::vector<double>> gauges_of;
        std::unordered_map<int, std::vector<double>> gauge_map;
        for (int g = 0; g < t.gauge_count; ++g) gauge_map[t.gauge_dof[g]].push_back(t.gauge_coefficient[g]);
        std::vector<int> deferred_index(size_t(S), -1);
        for (int q = 0; q < S; ++q)
        {
            if (!deferred[q]) continue;
            deferred_index[q] = int(ddof.size());
            ddof.push_back(q);
            const auto it = incident_index.find(q);
            dinc.push_back(it == incident_index.end() ? -1 : it->second);
            const auto g = gauge_map.find(q);
            if (g != gauge_map.end()) gcoef.insert(gcoef.end(), g->second.begin(), g->second.end());
            goff.push_back(int(gcoef.size()));
        }
        // geometric level-0 cell of every brick; must reproduce the aggregate of every active DOF
        const pcfd_level& base = t.levels[0];
        std::unordered_map<int64_t, int> base_slot;
        auto key = [](int64_t x, int64_t y, int64_t z) { return (x << 42) ^ (y << 21) ^ z; };
        for (int b = 0; b < base.brick_count; ++b)
            base_slot[key(base.coord[3 * b], base.coord[3 * b + 1], base.coord[3 * b + 2])] = b;
        std::vector<int> brick_base(size_t(s.B), -1);
        bool geometric = true;
        for (int slot = 0; slot < s.B && geometric; ++slot)
        {
            const pcfd_level& lev = *slot_lev[slot];
            const int b = slot_brick[slot], l = slot_level[slot];
            if (lev.flags[b] & PCFD_BRICK_COVERED) continue;
            int64_t g[3];
            for (int a = 0; a < 3; ++a) g[a] = (int64_t(lev.coord[3 * b + a]) * kBS) >> l;   // level-0 cell of (0,0,0)
            const auto it = base_slot.find(key(g[0] / kBS, g[1] / kBS, g[2] / kBS));
            if (it == base_slot.end() || g[0] < 0 || g[1] < 0 || g[2] < 0) { geometric = false; break; }
            brick_base[slot] = it->second * kC3 + int((g[2] % kBS) * 64 + (g[1] % kBS) * 8 + g[0] % kBS);
            for (int c = 0; c < kC3; ++c)
            {
                const int64_t a = int64_t(slot) * kC3 + c;
                if (!t.active[a]) continue;
                const int expect = brick_base[slot] + (((c >> 6) >> l) << 6) + ((((c >> 3) & 7) >> l) << 3) + ((c & 7) >> l);
                if (t.preconditioner_aggregate[a] - s.base_offset != expect) { geometric = false; break; }
            }
        }
        if (!geometric) return;
        // brick partial layout and the base-cell gather lists
        std::vector<int> poff(size_t(s.B), -1);
        std::vector<std::vector<int>> entries(size_t(s.base_cells));
        int partials = 0;
        for (int slot = 0; slot < s.B; ++slot)
        {
            const pcfd_level& lev = *slot_lev[slot];
            const int b = slot_brick[slot], l = slot_level[slot];
            if (lev.flags[b] & PCFD_BRICK_COVERED) continue;
            const int n = l >= 3 ? 1 : (kBS >> l);
            poff[slot] = partials;
            for (int z = 0; z < n; ++z)
                for (int y = 0; y < n; ++y)
                    for (int x = 0; x < n; ++x)
                        entries[size_t(brick_base[slot] + z * 64 + y * 8 + x)].push_back(partials + (z * n + y) * n + x);
            partials += n * n * n;
        }
        for (size_t d = 0; d < ddof.size(); ++d)
        {
            const int q = ddof[d];
            const int c = t.active[q] ? t.preconditioner_aggregate[q] - s.base_offset : -1;
            if (c >= 0 && c < s.base_cells) entries[size_t(c)].push_back(-int(d) - 1);
        }
        std::vector<int> eoff(size_t(s.base_cells) + 1, 0), elist;
        for (int c = 0; c < s.base_cells; ++c)
        {
            elist.insert(elist.end(), entries[c].begin(), entries[c].end());
            eoff[c + 1] = int(elist.size());
        }
        // w / D per level and (open faces, outlet), D summed exactly as in the code-bit check
        std::vector<double> damping(size_t(s.levels) * kDiagonalKinds, 0.0);
        for (int l = 0; l < s.levels; ++l)
            for (int outlet = 0; outlet < 2; ++outlet)
                for (int faces = 0; faces <= 6; ++faces)
                {
                    double D = 0.0;
                    for (int q = 0; q < faces; ++q) D += s.level_h[l];
                    if (outlet) D += 2.0 * s.level_h[l];
                    damping[size_t(l) * kDiagonalKinds + faces + 7 * outlet] = D > 0.0 ? (2.0 / 3.0) / D : 0.0;
                }
        f.damping.upload(damping);
        if (s.mg_precision == PCFD_MG_FP32 && !s.mg32.empty())
        {
            f.damping32.upload(std::vector<float>(damping.begin(), damping.end()));
            f.z32.alloc(size_t(S));
            f.z32b.alloc(size_t(S));
            f.r32.alloc(size_t(S));
            f.t32.alloc(size_t(S));
            f.res32.alloc(size_t(S));
        }
        if (s.mg_fine_chebyshev >= 2)
        {
            // Chebyshev-Richardson schedule for the two pre- and the two post-sweeps: the step sizes
            // are the inverse roots of the degree-2 Chebyshev polynomial on [2 / ratio, 2], smaller
            // step first; each step's w / D table is the w = 2/3 table rescaled
            const double hi = 2.0, lo = hi / s.mg_fine_chebyshev, theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
            const double steps[2] = {1.0 / (theta + delta * std::sqrt(0.5)), 1.0 / (theta - delta * std::sqrt(0.5))};
            f.cheb_stride = damping.size();
            std::vector<double> table(4 * damping.size());
            for (int slot = 0; slot < 4; ++slot)
            {
                f.cheb_omega[slot] = steps[slot & 1];
                for (size_t i = 0; i < damping.size(); ++i) table[slot * damping.size() + i] = damping[i] * (steps[slot & 1] / (2.0 / 3.0));
            }
            f.cheb_damping.upload(table);
            if (s.mg_precision == PCFD_MG_FP32 && !s.mg32.empty()) f.cheb_damping32.upload(std::vector<float>(table.begin(), table.end()));
        }
        f.code.upload(code);
        f.deferred_count = int(ddof.size());
        {
            // packed rows and their edges to active endpoints, in incidence order
            std::vector<int> ioff, iother;
            std::vector<double> icoef;
            if (o.incident_dofs)
            {
                ioff.resize(size_t(o.incident_dofs) + 1);
                cuda_check(cudaMemcpy(ioff.data(), o.incident_offset.p, ioff.size() * sizeof(int), cudaMemcpyDeviceToHost),
                           "incidence offsets download");
                iother.resize(size_t(ioff.back()));
                icoef.resize(size_t(ioff.back()));
                if (!iother.empty())
                {
                    cuda_check(cudaMemcpy(iother.data(), o.incident_other.p, iother.size() * sizeof(int), cudaMemcpyDeviceToHost),
                               "incidence download");
                    cuda_check(cudaMemcpy(icoef.data(), o.incident_coefficient.p, icoef.size() * sizeof(double),
                                          cudaMemcpyDeviceToHost), "incidence download");
                }
            }
            std::vector<int4> rows(ddof.size());
            std::vector<int2> edges;
            std::vector<double> ecoef;
            for (size_t d = 0; d < ddof.size(); ++d)
            {
                const int a = ddof[d], node = dinc[d], first = int(edges.size());
                const bool on = t.active[a] != 0, incident = node >= 0 && on;
                if (incident)
                    for (int q = ioff[size_t(node)]; q < ioff[size_t(node) + 1]; ++q)
                        if (t.active[iother[size_t(q)]])
                        {
                            edges.push_back(make_int2(iother[size_t(q)], -1));
                            ecoef.push_back(icoef[size_t(q)]);
                        }
                const int count = int(edges.size()) - first, gauges = goff[d + 1] - goff[d];
                if (gauges > 63 || count >= (1 << 23)) throw Error(PCFD_INTERNAL, "deferred row: too many gauges or edges");
                rows[d] = make_int4(a, first, -1, (count << 8) | (gauges << 2) | (incident ? 2 : 0) | (on ? 1 : 0));
            }
            if (edges.empty()) { edges.push_back(make_int2(0, -1)); ecoef.push_back(0.0); }
            f.deferred_row.upload(rows);
            f.deferred_edge.upload(edges);
            f.deferred_edge_coefficient.upload(ecoef);
            f.map_attached = false;
        }
        f.gauge_offset.upload(goff);
        f.gauge_coefficient.upload(gcoef.empty() ? std::vector<double>(1, 0.0) : gcoef);
        // per active brick, in active-list order: slot, level, base cell, partial offset,
        // neighbour slots, neighbour base cells (BrickMeta)
        std::vector<int> meta;
        meta.reserve(size_t(s.active_bricks) * 16);
        for (int slot = 0; slot < s.B; ++slot)
        {
            const pcfd_level& lev = *slot_lev[slot];
            const int b = slot_brick[slot];
            if (lev.flags[b] & PCFD_BRICK_COVERED) continue;
            const int slot0 = slot - b;
            int nbr[6];
            for (int face = 0; face < 6; ++face)
            {
                const int n = lev.neighbors[b * 6 + face];
                nbr[face] = n >= 0 && !(lev.flags[n] & PCFD_BRICK_COVERED) ? slot0 + n : -1;
            }
            meta.push_back(slot);
            meta.push_back(slot_level[slot]);
            meta.push_back(brick_base[slot]);
            meta.push_back(poff[slot]);
            for (int face = 0; face < 6; ++face) meta.push_back(nbr[face]);
            for (int face = 0; face < 6; ++face) meta.push_back(nbr[face] >= 0 ? brick_base[nbr[face]] : -1);
        }
        if (meta.size() != size_t(s.active_bricks) * 16) return;
        f.meta.upload(meta);
        f.partial.alloc(size_t(std::max(1, partials)));
        f.deferred_residual.alloc(size_t(std::max(1, f.deferred_count)));
        f.gather_offset.upload(eoff);
        f.gather_entry.upload(elist.empty() ? std::vector<int>(1, 0) : elist);
        f.t.alloc(size_t(S));
        f.z.alloc(size_t(S));
        f.enabled = true;
    }

    // Fills the packed deferred rows' and edges' map indices from the composite cycle's
    // fine -> stage-1 map (called once the map exists).
    void attach_deferred_map(System& s)
    {
        FineSmoother& f = s.fine;
        if (!f.enabled || !s.fine_map.p) return;
        const int rows = f.deferred_count, edges = int(f.deferred_edge.n);
        const int n = std::max(rows, edges);
        if (n > 0)
            attach_deferred_map_kernel<<<blocks_for(n), kThreads, 0, launch_stream(s)>>>(f.deferred_row, rows, f.deferred_edge, edges,
                                                                                          s.fine_map);
        cuda_check(cudaGetLastError(), "deferred map indices");
        cuda_check(cudaStreamSynchronize(launch_stream(s)), "deferred map indices");
        f.map_attached = true;
    }

    // ==================================================================================
    // launches
    // ==================================================================================
    namespace
    {
        BrickView view(System& s)
        {
            return BrickView{reinterpret_cast<const BrickMeta*>(s.fine.meta.p), s.d_level_h, s.fine.code, s.mg_prolong_scale,
                             s.fine.stage_neighbour.p};
        }

        // the deferred rows' arrays
        DeferredView deferred_view(System& s, double omega)
        {
            FineSmoother& f = s.fine;
            return DeferredView{f.deferred_row, f.deferred_edge, f.deferred_edge_coefficient, f.gauge_offset, f.gauge_coefficient,
                                s.diagonal, s.aggregate, s.base_offset, s.base_cells, omega};
        }

        template <int kMode, class T, class TO, class TC, int kProlong>
        void finish(System& s, const T* z, const T* r, TO* out, const TC* e, const T* t, double omega = 2.0 / 3.0)
        {
            FineSmoother& f = s.fine;
            if (!f.deferred_count) return;
            require(kProlong != 2 || f.map_attached, "deferred rows: composite map indices not attached");
            finish_deferred_kernel<kMode, T, TO, TC, kProlong><<<blocks_for(f.deferred_count), kThreads, 0, launch_stream(s)>>>(
                deferred_view(s, omega), f.deferred_count, s.structured, e, s.mg_prolong_scale, z, r, t, out, f.deferred_residual);
        }

        // Persistent grid of a pipeline kernel: the system's CTAs per SM (autotuned), capped by the
        // kernel's guaranteed residency (its launch bounds), so that no CTA waits for a second
        // wave while the others run.
        template <int kMode, class T>
        int pipe_grid(const System& s)
        {
            static int sms = 0;
            if (!sms)
            {
                int device = 0;
                cuda_check(cudaGetDevice(&device), "device");
                cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
            }
            return std::max(1, std::min(s.active_bricks, std::min(s.pipe_ctas_per_sm, pipe_resident<kMode, T>()) * sms));
        }

        // the working buffers of the fine level in field type T
        template <class T> struct FineBuffers;
        template <> struct FineBuffers<double>
        {
            double *a, *t;
            const double *damping, *chebyshev;
            explicit FineBuffers(FineSmoother& f) : a(f.z.p), t(f.t.p), damping(f.damping.p), chebyshev(f.cheb_damping.p) {}
        };
        template <> struct FineBuffers<float>
        {
            float *a, *t;
            const float *damping, *chebyshev;
            explicit FineBuffers(FineSmoother& f) : a(f.z32.p), t(f.t32.p), damping(f.damping32.p), chebyshev(f.cheb_damping32.p) {}
        };

        // one fine sweep z + w (r - A z) / D; slot >= 0 selects the w of that step of the
        // Chebyshev-Richardson schedule (mg_fine_chebyshev), otherwise w = 2/3
        template <class T, class TO, class TC, int kProlong>
        void sweep(System& s, const T* z, const T* r, TO* out, const TC* e, int slot = -1)
        {
            FineBuffers<T> w(s.fine);
            require(kProlong != 2 || s.fine.stage_neighbour.p, "mapped prolongation: stage-1 brick ranks not set");
            const bool cheb = slot >= 0 && w.chebyshev;
            const T* damping = cheb ? w.chebyshev + size_t(slot) * s.fine.cheb_stride : w.damping;
            const double omega = cheb ? s.fine.cheb_omega[slot] : 2.0 / 3.0;
            brick_pipe_kernel<0, T, TO, TC, kProlong><<<pipe_grid<0, T>(s), 256, 0, launch_stream(s)>>>(
                view(s), s.active_bricks, z, r, out, w.t, e, nullptr, damping);
            finish<0, T, TO, TC, kProlong>(s, z, r, out, e, w.t, omega);
        }
        // the first pre-sweep from z = 0 (slot 0 of the schedule when it is on)
        template <class T> void first_sweep(System& s, const double* r, T* z, T* r_copy)
        {
            FineSmoother& f = s.fine;
            FineBuffers<T> w(f);
            const bool cheb = w.chebyshev != nullptr;
            first_sweep_kernel<T><<<blocks_for((int64_t(s.S) + 3) / 4), kThreads, 0, launch_stream(s)>>>(
                f.code, s.brick_level, cheb ? w.chebyshev : w.damping, s.diagonal, s.active, r, z, r_copy, s.structured, s.S,
                cheb ? f.cheb_omega[0] : 2.0 / 3.0);
        }

        template <class T>
        void restrict_residual(System& s, const T* z, const T* r)
        {
            FineSmoother& f = s.fine;
            FineBuffers<T> w(f);
            brick_pipe_kernel<1, T, T, double, 0><<<pipe_grid<1, T>(s), 256, 0, launch_stream(s)>>>(
                view(s), s.active_bricks, z, r, nullptr, w.t, nullptr, f.partial, w.damping);
            finish<1, T, T, double, 0>(s, z, r, nullptr, nullptr, w.t);
        }
    }

    void brick_apply(System& s, const double* p, double* out)
    {
        brick_pipe_kernel<2, double, double, double, 0><<<pipe_grid<2, double>(s), 256, 0, launch_stream(s)>>>(
            view(s), s.active_bricks, p, nullptr, out, nullptr, nullptr, nullptr, nullptr);
    }

    // One application of the reference cycle with its fine level fused.  FP64: z_a, z and r are
    // the double vectors.  FP32 multigrid (the coarse levels in float): the fine sweeps run on
    // float copies -- r is converted once by the first sweep, the iterate ping-pongs between two
    // float buffers and only the last sweep writes the double result -- so the smoother moves
    // 4-byte values; the outer Krylov vectors, dots and the operator stay FP64.
    template <class TC>
    void fine_preconditioner(System& s, const double* r, double* z, std::vector<MgLevel<TC>>& levels)
    {
        FineSmoother& f = s.fine;
        MgLevel<TC>& base = levels.front();
        auto coarse = [&](auto* zz, auto* rr) {
            cuda_check(cudaMemsetAsync(base.x, 0, size_t(base.cells) * sizeof(TC), s.stream), "clear base correction");
            restrict_residual(s, zz, rr);
            gather_base_kernel<TC><<<blocks_for(base.cells), kThreads, 0, launch_stream(s)>>>(
                base.cells, f.gather_offset, f.gather_entry, f.partial, f.deferred_residual, base.rhs);
            multigrid_levels(s, levels);
        };
        if (std::is_same<TC, float>::value && f.z32.n)
        {
            float *a = f.z32.p, *b = f.z32b.p, *r32 = f.r32.p;
            first_sweep_kernel<float><<<blocks_for((int64_t(s.S) + 3) / 4), kThreads, 0, launch_stream(s)>>>(
                f.code, s.brick_level, f.damping32.p, s.diagonal, s.active, r, a, r32, s.structured, s.S, 2.0 / 3.0);
            sweep<float, float, TC, 0>(s, a, r32, b, nullptr);
            coarse(b, r32);
            sweep<float, float, TC, 1>(s, b, r32, a, base.x.p);
            sweep<float, double, TC, 0>(s, a, r32, z, nullptr);
        }
        else
        {
            double* a = f.z.p;
            first_sweep_kernel<double><<<blocks_for((int64_t(s.S) + 3) / 4), kThreads, 0, launch_stream(s)>>>(
                f.code, s.brick_level, f.damping.p, s.diagonal, s.active, r, a, nullptr, s.structured, s.S, 2.0 / 3.0);
            sweep<double, double, TC, 0>(s, a, r, z, nullptr);
            coarse(z, r);
            sweep<double, double, TC, 1>(s, z, r, a, base.x.p);
            sweep<double, double, TC, 0>(s, a, r, z, nullptr);
        }
        cuda_check(cudaGetLastError(), "fused preconditioner");
    }

    namespace
    {
        template <class TC, class TR>
        __global__ void gather_first_kernel(int cells, const int* __restrict__ offset, const int* __restrict__ dof,
                                            const TR* __restrict__ residual, TC* __restrict__ rhs)
        {
            const int c = blockIdx.x * blockDim.x + threadIdx.x;
            if (c >= cells) return;
            double sum = 0.0;
            for (int q = offset[c]; q < offset[c + 1]; ++q) sum += residual[dof[q]];
            rhs[c] = TC(sum);
        }

        // The same gather with stage 1 numbered by brick rank: row c's structured members are the
        // 2x2x2 block (c & 63) of brick slot[c >> 6], summed in ascending DOF order (inactive DOFs
        // hold a zero residual), then its EB fragments from the CSR.
        template <class TC, class TR>
        __global__ void __launch_bounds__(256) gather_first_brick_kernel(int cells, const int* __restrict__ slot,
            const int* __restrict__ offset, const int* __restrict__ dof, const TR* __restrict__ residual, TC* __restrict__ rhs)
        {
            const int c = blockIdx.x * blockDim.x + threadIdx.x;
            if (c >= cells) return;
            const int block = c & 63;
            const int64_t base = int64_t(slot[c >> 6]) * kC3 + 2 * (block & 3) + 16 * ((block >> 2) & 3) + 128 * (block >> 4);
            const int q0 = offset[c], q1 = offset[c + 1];
            TR v[8];
#pragma unroll
            for (int m = 0; m < 4; ++m)
            {
                v[2 * m] = residual[base + 64 * (m >> 1) + 8 * (m & 1)];
                v[2 * m + 1] = residual[base + 64 * (m >> 1) + 8 * (m & 1) + 1];
            }
            double sum = 0.0;
#pragma unroll
            for (int m = 0; m < 8; ++m) sum += v[m];
            for (int q = q0; q < q1; ++q) sum += residual[dof[q]];
            rhs[c] = TC(sum);
        }

        template <class TC, class TR>
        void gather_first(System& s, const TR* residual, MgLevel<TC>& first)
        {
            if (s.first_stage_bricks)
                gather_first_brick_kernel<TC, TR><<<blocks_for(first.cells), kThreads, 0, launch_stream(s)>>>(
                    first.cells, s.active_brick_list, s.fine_restrict_offset, s.fine_restrict_dof, residual, first.rhs);
            else
                gather_first_kernel<TC, TR><<<blocks_for(first.cells), kThreads, 0, launch_stream(s)>>>(
                    first.cells, s.fine_restrict_offset, s.fine_restrict_dof, residual, first.rhs);
        }

        // residual of the pre-smoothed z, its gather into stage 1, the stage V-cycle, the weighted
        // prolongation fused into the first post-sweep, one more post-sweep
        template <class TC> void composite_tail(System& s, const double* r, double* z, MgLevel<TC>& first, bool schedule = true);

        template <class TC>
        void composite_cycle(System& s, const double* r, double* z, MgLevel<TC>& first)
        {
            FineSmoother& f = s.fine;
            if (s.mg_block_iterations > 0)
            {
                // the brick-local block solve in place of the two Jacobi pre-sweeps
                cuda_check(cudaMemsetAsync(z, 0, size_t(s.structured) * sizeof(double), s.stream), "clear z");
                if (s.active_bricks)
                    block_smooth_kernel<<<s.active_bricks, 256, 0, launch_stream(s)>>>(s.active_brick_list, f.code, s.brick_level,
                                                                                      s.d_level_h, s.diagonal, s.active, r, z,
                                                                                      s.mg_block_iterations, 0.06, 2.0);
                if (s.S > s.structured)
                    tail_jacobi_kernel<<<blocks_for(int64_t(s.S) - s.structured), kThreads, 0, launch_stream(s)>>>(
                        s.structured, s.S, r, s.diagonal, s.active, z, 2.0 / 3.0);
                composite_tail<TC>(s, r, z, first);
                return;
            }
            double* a = f.z.p;
            first_sweep<double>(s, r, a, nullptr);
            sweep<double, double, TC, 0>(s, a, r, z, nullptr, 1);
            composite_tail<TC>(s, r, z, first);
        }
    }

    // The learned preconditioner around the fused fine level: a = net(r), then one damped Jacobi
    // sweep (PCFD_PRECONDITIONER_LEARNED), or the composite cycle's residual, stage correction and
    // post-sweeps with the network in place of the fine pre-sweeps
    // (PCFD_PRECONDITIONER_LEARNED_MULTIGRID).
    void learned_preconditioner(System& s, const double* r, double* z, bool coarse)
    {
        if (!coarse)
        {
            learned_apply(s, r, s.fine.z.p);
            sweep<double, double, double, 0>(s, s.fine.z.p, r, z, nullptr);
            return;
        }
        require(s.composite, "the learned multigrid preconditioner needs the composite cycle");
        learned_apply(s, r, z);
        if (s.composite_fp32) composite_tail<float>(s, r, z, s.inter32.front());
        else composite_tail<double>(s, r, z, s.inter64.front());
    }

    namespace
    {
        // schedule: the post-sweeps take the Chebyshev-Richardson steps of the fine schedule (the
        // second half of a pre/post pair), otherwise w = 2/3
        template <class TC> void composite_tail(System& s, const double* r, double* z, MgLevel<TC>& first, bool schedule)
        {
            FineSmoother& f = s.fine;
            double* a = f.z.p;
            double* res = s.fine_residual.p;
            brick_pipe_kernel<3, double, double, TC, 0><<<pipe_grid<3, double>(s), 256, 0, launch_stream(s)>>>(
                view(s), s.active_bricks, z, r, res, f.t.p, nullptr, nullptr, f.damping.p);
            finish<2, double, double, TC, 0>(s, z, r, res, static_cast<const TC*>(nullptr), f.t.p);
            gather_first<TC, double>(s, res, first);
            cuda_check(cudaMemsetAsync(first.x, 0, size_t(first.cells) * sizeof(TC), s.stream), "clear stage correction");
            composite_levels(s);
            sweep<double, double, TC, 2>(s, z, r, a, first.x.p, schedule ? 2 : -1);
            sweep<double, double, TC, 0>(s, a, r, z, nullptr, schedule ? 3 : -1);
            cuda_check(cudaGetLastError(), "composite preconditioner");
        }

        // the composite cycle with the FP32 multigrid: the fine sweeps on float copies as in the
        // reference cycle's FP32 path (r converted once by the first sweep, the iterate
        // ping-ponging between two float buffers, the residual gathered from floats, only the last
        // sweep writing the double result)
        void composite_cycle_fp32(System& s, const double* r, double* z, MgLevel<float>& first)
        {
            FineSmoother& f = s.fine;
            float *a = f.z32.p, *b = f.z32b.p, *r32 = f.r32.p, *res = f.res32.p;
            first_sweep<float>(s, r, a, r32);
            sweep<float, float, float, 0>(s, a, r32, b, nullptr, 1);
            brick_pipe_kernel<3, float, float, float, 0><<<pipe_grid<3, float>(s), 256, 0, launch_stream(s)>>>(
                view(s), s.active_bricks, b, r32, res, f.t32.p, nullptr, nullptr, f.damping32.p);
            finish<2, float, float, float, 0>(s, b, r32, res, static_cast<const float*>(nullptr), f.t32.p);
            gather_first<float, float>(s, res, first);
            cuda_check(cudaMemsetAsync(first.x, 0, size_t(first.cells) * sizeof(float), s.stream), "clear stage correction");
            composite_levels(s);
            sweep<float, float, float, 2>(s, b, r32, a, first.x.p, 2);
            sweep<float, double, float, 0>(s, a, r32, z, nullptr, 3);
            cuda_check(cudaGetLastError(), "composite preconditioner");
        }
    }

    // The composite cycle: the fused FP64 fine sweeps of the reference cycle around the stage
    // levels of the composite grid (solver.cu), in double or (FP32 multigrid) float.  Fine
    // pre-smoothing as in the reference cycle, the residual written once and gathered into stage
    // 1, the stage and lattice V-cycle, the weighted prolongation fused into the first post-sweep,
    // one more post-sweep.
    void composite_preconditioner(System& s, const double* r, double* z)
    {
        if (s.composite_fp32 && s.fine.res32.n && !s.mg_block_iterations) composite_cycle_fp32(s, r, z, s.inter32.front());
        else if (s.composite_fp32) composite_cycle<float>(s, r, z, s.inter32.empty() ? s.mg32.front() : s.inter32.front());
        else composite_cycle<double>(s, r, z, s.inter64.empty() ? s.mg64.front() : s.inter64.front());
    }

    // Stages of the fused FP64 cycle for component timing: 0 pre-smoothing, 1 residual restriction
    // to the level-0 aggregates, 2 the aggregation hierarchy, 3 prolongation + post-smoothing.
    void fine_preconditioner_stage(System& s, int stage, const double* r, double* z)
    {
        require(s.fine.enabled && !s.mg64.empty(), "fused preconditioner not enabled");
        FineSmoother& f = s.fine;
        std::vector<MgLevel<double>>& levels = s.mg64;
        MgLevel<double>& base = levels.front();
        double* a = f.z.p;
        if (stage == 0)
        {
            first_sweep_kernel<double><<<blocks_for((int64_t(s.S) + 3) / 4), kThreads, 0, launch_stream(s)>>>(
                f.code, s.brick_level, f.damping.p, s.diagonal, s.active, r, a, nullptr, s.structured, s.S, 2.0 / 3.0);
            sweep<double, double, double, 0>(s, a, r, z, nullptr);
        }
        else if (stage == 1)
        {
            restrict_residual<double>(s, z, r);
            gather_base_kernel<double><<<blocks_for(base.cells), kThreads, 0, launch_stream(s)>>>(
                base.cells, f.gather_offset, f.gather_entry, f.partial, f.deferred_residual, base.rhs);
        }
        else if (stage == 2)
        {
            cuda_check(cudaMemsetAsync(base.x, 0, size_t(base.cells) * sizeof(double), s.stream), "clear base correction");
            multigrid_levels(s, levels);
        }
        else
        {
            sweep<double, double, double, 1>(s, z, r, a, base.x.p);
            sweep<double, double, double, 0>(s, a, r, z, nullptr);
        }
    }

    // Autotuner of the brick pipeline's persistent grid: each candidate number of resident CTAs
    // per SM (1 up to what the kernel's registers and shared memory allow, at most 8) is timed on
    // this system's own bricks -- the structured FP64 operator and one fine-level sweep of the
    // multigrid in its precision, CUDA events over `iterations` launches on resident scratch
    // vectors -- and the fastest sum is kept.  Returns the number of candidates written.
    int autotune_pipe(System& s, int iterations, int* ctas, double* apply_ms, double* sweep_ms)
    {
        require(s.fine.enabled, "autotune: the brick pipeline needs 8^3 bricks");
        int fit = 0;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, brick_pipe_kernel<2, double, double, double, 0>, 256, 0),
                   "pipeline occupancy");
        int fit32 = fit;
        cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit32, brick_pipe_kernel<0, float, float, float, 0>, 256, 0),
                   "pipeline occupancy");
        const int top = std::max(1, std::min({8, fit, fit32}));
        const bool fp32 = s.composite_fp32 && s.fine.res32.n;
        cudaEvent_t e0, e1;
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        auto time = [&](auto&& body) {
            body();
            cuda_check(cudaEventRecord(e0, s.stream), "event");
            for (int q = 0; q < iterations; ++q) body();
            cuda_check(cudaEventRecord(e1, s.stream), "event");
            cuda_check(cudaEventSynchronize(e1), "event");
            float ms = 0;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event");
            return double(ms) / iterations;
        };
        int best = s.pipe_ctas_per_sm;
        double best_ms = 1e300;
        int n = 0;
        for (int c = 1; c <= top; ++c)
        {
            s.pipe_ctas_per_sm = c;
            apply_ms[n] = time([&] { brick_apply(s, s.scratch_p, s.scratch_out); });
            sweep_ms[n] = fp32 ? time([&] {
                FineSmoother& f = s.fine;
                sweep<float, float, float, 0>(s, f.z32.p, f.r32.p, f.z32b.p, nullptr);
            })
                               : time([&] { sweep<double, double, double, 0>(s, s.fine.z.p, s.scratch_p, s.scratch_out, nullptr); });
            ctas[n] = c;
            if (apply_ms[n] + sweep_ms[n] < best_ms) { best_ms = apply_ms[n] + sweep_ms[n]; best = c; }
            ++n;
        }
        s.pipe_ctas_per_sm = best;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return n;
    }

    template void fine_preconditioner<double>(System&, const double*, double*, std::vector<MgLevel<double>>&);
    template void fine_preconditioner<float>(System&, const double*, double*, std::vector<MgLevel<float>>&);
}
