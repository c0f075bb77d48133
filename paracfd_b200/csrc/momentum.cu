// momentum.cu -- collocated cell-momentum kernels of the time step (FP32 state, gather form).
//
// Operators (reference src/core/fluid/amr_advection.cu):
//   transport       MUSCL/minmod face value on regular faces (:58-93), bounded least-squares
//                   reconstruction on compact faces (:94-112), X inflow/outflow boundary fluxes
//   smagorinsky     nu = nu_mol + (Cs V^{1/3})^2 |S| (:198-222), explicit FV diffusion sub-cycled at
//                   diffusion CFL 0.7 (:223-252, 1339-1345)
//   wall            Spalding friction velocity, implicit 3x3 SPD solve per wall CV (:421-437)
//   impulse         face-centroid pressure traction on every open face, wall and boundary (:361-413)
//   reconstruction  cell -> face normal velocity (:262-293)
// Design: every cell gathers the fluxes of its own six faces (each face flux is evaluated with the
// reference's FP32 expression by both neighbours, so the two sides agree bit for bit and the update
// is conservative), DOFs touching compact edges finish in a second per-DOF pass, small-cell groups
// in a third.  No atomics: results are deterministic run to run.  The state is double-buffered.
#include "momentum.h"

#include <algorithm>
#include <cmath>

namespace pcfd
{
    namespace
    {
        struct CellCtx
        {
            int slot, i, j, k;
            int64_t dof;
            float h;
        };

        __device__ inline bool decode_cell(int64_t work, const int* brick_list, int bs, const int* brick_level,
                                           const double* level_h, CellCtx& c)
        {
            const int c3 = bs * bs * bs;
            // DOF counts fit in 32 bits (pcfd_topology indexes them with int): 32-bit division
            c.slot = brick_list[int(work) / c3];
            const int local = int(work) % c3;
            c.i = local % bs; c.j = (local / bs) % bs; c.k = local / (bs * bs);
            c.dof = int64_t(c.slot) * c3 + local;
            c.h = float(level_h[brick_level[c.slot]]);
            return true;
        }

        // Neighbour DOF along +-axis (same brick or same-level active brick), -1 when absent.
        __device__ inline int64_t step_dof(int bs, const int* nbr, int slot, int i, int j, int k, int axis, int sign, int* out_slot)
        {
            int c[3] = {i, j, k};
            int sl = slot;
            c[axis] += sign;
            if (c[axis] < 0 || c[axis] >= bs)
            {
                sl = nbr[slot * 6 + 2 * axis + (sign > 0)];
                if (sl < 0) return -1;
                c[axis] = sign > 0 ? 0 : bs - 1;
            }
            if (out_slot) *out_slot = sl;
            return int64_t(sl) * (bs * bs * bs) + (c[2] * bs + c[1]) * bs + c[0];
        }

        // The face between `lower` and the next cell along +axis is open for the structured stencil.
        __device__ inline bool face_open(uint8_t lower_code, int axis)
        {
            return !(lower_code & (1u << axis)) && !(lower_code & (1u << (CODE_COMPACT_SHIFT + axis)));
        }

        // structured_cell_neighbor (reference :192-197): neighbour across an open structured face.
        __device__ inline int64_t open_neighbor(int bs, const int* nbr, const uint8_t* code, int slot, int i, int j, int k,
                                                int64_t self, int axis, int sign)
        {
            const int64_t n = step_dof(bs, nbr, slot, i, j, k, axis, sign, nullptr);
            if (n < 0 || !(code[n] & CODE_ACTIVE)) return -1;
            const int64_t lower = sign > 0 ? self : n;
            return face_open(code[lower], axis) ? n : -1;
        }

        __device__ inline float comp3(const float* x, const float* y, const float* z, int64_t q, int c)
        {
            return c == 0 ? x[q] : (c == 1 ? y[q] : z[q]);
        }
        __device__ inline float minmod_cell(float a, float b)
        {
            if (a * b <= 0.0f) return 0.0f;
            return a >= 0.0f ? fminf(a, b) : fmaxf(a, b);
        }
        __device__ inline float muscl_value(float va, float vb, float vl, float vu, bool has_l, bool has_u, float swept, float courant)
        {
            if (swept >= 0.0f)
            {
                if (!has_l) return va;
                return va + 0.5f * (1.0f - fminf(1.0f, courant)) * minmod_cell(va - vl, vb - va);
            }
            if (!has_u) return vb;
            return vb - 0.5f * (1.0f - fminf(1.0f, courant)) * minmod_cell(vb - va, vu - vb);
        }

        // X-min inflow normal velocity of boundary face (j, k) of a brick: the per-face profile when one
        // was set (pcfd_core_set_inflow_host), otherwise the uniform freestream.
        __device__ inline float inflow_value(const int* slot_map, const float* inflow, int bs, int slot, int j, int k, float U)
        {
            if (!inflow) return U;
            const int pos = slot_map[slot];
            return pos >= 0 ? inflow[int64_t(pos) * bs * bs + k * bs + j] : U;
        }

        __device__ inline float face_at(const float* u,const float* v, const float* w, int bs, int axis, int slot, int i, int j, int k)
        {
            return axis == 0 ? u[u_face(bs, slot, i, j, k)] : (axis == 1 ? v[v_face(bs, slot, i, j, k)] : w[w_face(bs, slot, i, j, k)]);
        }

        // MUSCL momentum flux through the +axis face of cell `a` (a -> b).  Same arithmetic
        // whichever neighbour evaluates it.
        __device__ inline void regular_face_flux(int bs, const int* nbr, const uint8_t* code, const float* x, const float* y,
                                                 const float* z, int slot_a, int ia, int ja, int ka, int64_t a, int slot_b,
                                                 int64_t b, float normal, float dt, float h, int axis, float f[3])
        {
            int cb[3] = {ia, ja, ka};
            cb[axis] = (cb[axis] + 1) % bs;
            const int64_t lower = open_neighbor(bs, nbr, code, slot_a, ia, ja, ka, a, axis, -1);
            const int64_t upper = open_neighbor(bs, nbr, code, slot_b, cb[0], cb[1], cb[2], b, axis, 1);
            const float swept = dt * h * h * normal, courant = fabsf(normal) * dt / h;
            for (int c = 0; c < 3; ++c)
            {
                const float va = comp3(x, y, z, a, c), vb = comp3(x, y, z, b, c);
                const float vl = lower >= 0 ? comp3(x, y, z, lower, c) : 0.0f, vu = upper >= 0 ? comp3(x, y, z, upper, c) : 0.0f;
                f[c] = swept * muscl_value(va, vb, vl, vu, lower >= 0, upper >= 0, swept, courant);
            }
        }

        // ---------------------------------------------------------------- transport
        template <int kBS>
        __global__ void transport_struct_kernel(const int* __restrict__ brick_list, int nbricks, int bs_arg, const int* __restrict__ brick_level,
            const int* __restrict__ nbr, const uint32_t* __restrict__ flags, const double* __restrict__ level_h,
            const uint8_t* __restrict__ code, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float dt, int external, float U,
            const int* __restrict__ inflow_slot, const float* __restrict__ inflow, float* __restrict__ xn, float* __restrict__ yn, float* __restrict__ zn, float* __restrict__ dx, float* __restrict__ dy,
            float* __restrict__ dz)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(nbricks) * bs * bs * bs) return;
            CellCtx c;
            decode_cell(work, brick_list, bs, brick_level, level_h, c);
            const int64_t a = c.dof;
            const uint8_t ca = code[a];
            if (!(ca & CODE_ACTIVE)) { xn[a] = x[a]; yn[a] = y[a]; zn[a] = z[a]; return; }
            float D[3] = {0.0f, 0.0f, 0.0f};
            const int ijk[3] = {c.i, c.j, c.k};
            for (int axis = 0; axis < 3; ++axis)
            {
                // + face: a -> b
                int sb;
                const int64_t b = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, 1, &sb);
                if (b >= 0 && (code[b] & CODE_ACTIVE) && face_open(ca, axis))
                {
                    int f[3] = {c.i, c.j, c.k};
                    ++f[axis];
                    const float normal = face_at(u, v, w, bs, axis, c.slot, f[0], f[1], f[2]);
                    float flux[3];
                    regular_face_flux(bs, nbr, code, x, y, z, c.slot, c.i, c.j, c.k, a, sb, b, normal, dt, c.h, axis, flux);
                    D[0] -= flux[0]; D[1] -= flux[1]; D[2] -= flux[2];
                }
                // - face: p -> a
                int sp;
                const int64_t p = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, -1, &sp);
                if (p >= 0 && (code[p] & CODE_ACTIVE) && face_open(code[p], axis))
                {
                    int q[3] = {c.i, c.j, c.k};
                    q[axis] = ijk[axis] == 0 ? bs - 1 : ijk[axis] - 1;
                    int f[3] = {q[0], q[1], q[2]};
                    ++f[axis];
                    const float normal = face_at(u, v, w, bs, axis, sp, f[0], f[1], f[2]);
                    float flux[3];
                    regular_face_flux(bs, nbr, code, x, y, z, sp, q[0], q[1], q[2], p, c.slot, a, normal, dt, c.h, axis, flux);
                    D[0] += flux[0]; D[1] += flux[1]; D[2] += flux[2];
                }
            }
            if (external)
            {
                const float area = c.h * c.h;
                const uint32_t fl = flags[c.slot];
                if (c.i == 0 && (fl & PCFD_BRICK_XMIN))
                {
                    const float normal = u[u_face(bs, c.slot, 0, c.j, c.k)], swept = dt * area * normal;
                    const float in = inflow_value(inflow_slot, inflow, bs, c.slot, c.j, c.k, U);
                    if (swept >= 0.0f) { D[0] += swept * in; D[1] += swept * 0.0f; D[2] += swept * 0.0f; }
                    else { D[0] += swept * x[a]; D[1] += swept * y[a]; D[2] += swept * z[a]; }
                }
                if (c.i == bs - 1 && (fl & PCFD_BRICK_XMAX))
                {
                    const float normal = u[u_face(bs, c.slot, bs, c.j, c.k)], swept = dt * area * normal;
                    if (swept >= 0.0f) { D[0] += -swept * x[a]; D[1] += -swept * y[a]; D[2] += -swept * z[a]; }
                    else D[0] += -swept * U;
                }
            }
            if (ca & CODE_DEFERRED) { dx[a] = D[0]; dy[a] = D[1]; dz[a] = D[2]; return; }
            const double hd = level_h[brick_level[c.slot]];
            const float inverse = 1.0f / float(hd * hd * hd);
            xn[a] = x[a] + D[0] * inverse; yn[a] = y[a] + D[1] * inverse; zn[a] = z[a] + D[2] * inverse;
        }

        // ---------------------------------------------------------------- transport, 8^3 bricks
        // One CTA per active brick.  The brick's momentum and codes plus a two-cell halo along each
        // axis (from the same-level face neighbours; absent neighbours read as inactive) are staged
        // in shared memory as a 12^3 tile (cells -2..9).  Each of the brick's 3 x 9 x 64 faces then
        // evaluates its MUSCL flux once with the per-cell kernel's expression (regular_face_flux), so
        // a face shared with the neighbouring brick gets the bit-identical flux there; each cell sums
        // its six faces in the per-cell kernel's order.  The normal velocity of a face is read from the
        // brick of the face's lower cell, as the per-cell kernel reads it.
        constexpr int kTile = 12;
        __device__ inline int tile_index(int i, int j, int k) { return ((k + 2) * kTile + (j + 2)) * kTile + (i + 2); }

        __global__ void __launch_bounds__(256, 5) transport_brick_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const uint32_t* __restrict__ flags,
            const double* __restrict__ level_h, const uint8_t* __restrict__ code, const float* __restrict__ u,
            const float* __restrict__ v, const float* __restrict__ w, const float* __restrict__ x, const float* __restrict__ y,
            const float* __restrict__ z, float dt, int external, float U, const int* __restrict__ inflow_slot,
            const float* __restrict__ inflow, float* __restrict__ xn, float* __restrict__ yn, float* __restrict__ zn,
            float* __restrict__ dx, float* __restrict__ dy, float* __restrict__ dz)
        {
            constexpr int bs = 8, c3 = 512, T3 = kTile * kTile * kTile, F = 9 * 64;
            __shared__ float sv[3][T3];
            __shared__ uint8_t sc[T3];
            __shared__ float flux[3][F][3];            // [axis][face][component]
            __shared__ int neighbour[6];
            const int slot = brick_list[blockIdx.x], tid = threadIdx.x;
            if (tid < 6) neighbour[tid] = nbr[slot * 6 + tid];
            for (int q = tid; q < T3; q += 256) sc[q] = 0;
            __syncthreads();
            const int64_t base = int64_t(slot) * c3;
            for (int q = tid; q < c3; q += 256)
            {
                const int t = tile_index(q & 7, (q >> 3) & 7, q >> 6);
                sv[0][t] = x[base + q]; sv[1][t] = y[base + q]; sv[2][t] = z[base + q]; sc[t] = code[base + q];
            }
            // halos: direction d = 2 axis + (side > 0), two layers of 64 cells each
            for (int q = tid; q < 6 * 128; q += 256)
            {
                const int d = q >> 7, layer = (q >> 6) & 1, a = q & 7, b = (q >> 3) & 7, axis = d >> 1;
                const int ns = neighbour[d];
                if (ns < 0) continue;
                const int src = (d & 1) ? layer : bs - 1 - layer, dst = (d & 1) ? bs + layer : -1 - layer;
                int si[3], ti[3];
                // the two transverse coordinates of the halo cell, in axis order
                const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
                si[axis] = src; ti[axis] = dst;
                si[t0] = ti[t0] = a; si[t1] = ti[t1] = b;
                const int64_t g = int64_t(ns) * c3 + (si[2] * bs + si[1]) * bs + si[0];
                const int t = tile_index(ti[0], ti[1], ti[2]);
                sv[0][t] = x[g]; sv[1][t] = y[g]; sv[2][t] = z[g]; sc[t] = code[g];
            }
            __syncthreads();
            const float h = float(level_h[brick_level[slot]]);
            // face fluxes: face p (0..8) along `axis` lies between tile cells p - 1 (lower) and p.
            // The normal velocities of a thread's faces (stored in the brick of each face's lower
            // cell) are loaded first, all at once, so their latencies overlap.
            constexpr int kFacesPerThread = (3 * F + 255) / 256;
            float normals[kFacesPerThread];
#pragma unroll
            for (int n = 0; n < kFacesPerThread; ++n)
            {
                const int q = tid + 256 * n;
                normals[n] = 0.0f;
                if (q >= 3 * F) continue;
                const int axis = q / F, f = q % F, p = f % 9, a = (f / 9) & 7, b = f / 72;
                const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
                int fs = slot, fi[3];
                fi[axis] = p; fi[t0] = a; fi[t1] = b;
                if (p == 0)
                {
                    fs = neighbour[2 * axis];
                    fi[axis] = bs;
                    if (fs < 0) continue;   // no lower neighbour: the face is closed below
                }
                normals[n] = axis == 0 ? u[u_face(bs, fs, fi[0], fi[1], fi[2])]
                           : (axis == 1 ? v[v_face(bs, fs, fi[0], fi[1], fi[2])] : w[w_face(bs, fs, fi[0], fi[1], fi[2])]);
            }
#pragma unroll
            for (int n = 0; n < kFacesPerThread; ++n)
            {
                const int q = tid + 256 * n;
                if (q >= 3 * F) continue;
                const int axis = q / F, f = q % F, p = f % 9, a = (f / 9) & 7, b = f / 72;
                int lo[3];
                const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
                lo[axis] = p - 1; lo[t0] = a; lo[t1] = b;
                int step[3] = {0, 0, 0};
                step[axis] = 1;
                const int stride = step[0] + kTile * (step[1] + kTile * step[2]);
                const int ta = tile_index(lo[0], lo[1], lo[2]), tb = ta + stride;
                const uint8_t ca = sc[ta], cb = sc[tb];
                float* out = flux[axis][f];
                if (!(ca & CODE_ACTIVE) || !(cb & CODE_ACTIVE) || !face_open(ca, axis)) { out[0] = out[1] = out[2] = 0.0f; continue; }
                const float normal = normals[n];
                const int tl = ta - stride, tu = tb + stride;
                const bool has_l = (sc[tl] & CODE_ACTIVE) && face_open(sc[tl], axis);
                const bool has_u = (sc[tu] & CODE_ACTIVE) && face_open(cb, axis);
                const float swept = dt * h * h * normal, courant = fabsf(normal) * dt / h;
                for (int c = 0; c < 3; ++c)
                {
                    const float va = sv[c][ta], vb = sv[c][tb];
                    const float vl = has_l ? sv[c][tl] : 0.0f, vu = has_u ? sv[c][tu] : 0.0f;
                    out[c] = swept * muscl_value(va, vb, vl, vu, has_l, has_u, swept, courant);
                }
            }
            __syncthreads();
            const double hd = level_h[brick_level[slot]];
            const float inverse = 1.0f / float(hd * hd * hd);
            const uint32_t fl = flags[slot];
            for (int q = tid; q < c3; q += 256)
            {
                const int i = q & 7, j = (q >> 3) & 7, k = q >> 6, t = tile_index(i, j, k);
                const int64_t a = base + q;
                const uint8_t ca = sc[t];
                if (!(ca & CODE_ACTIVE)) { xn[a] = sv[0][t]; yn[a] = sv[1][t]; zn[a] = sv[2][t]; continue; }
                float D[3] = {0.0f, 0.0f, 0.0f};
                const int ijk[3] = {i, j, k};
                for (int axis = 0; axis < 3; ++axis)
                {
                    const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
                    int step[3] = {0, 0, 0};
                    step[axis] = 1;
                    const int stride = step[0] + kTile * (step[1] + kTile * step[2]);
                    const int fplus = (ijk[axis] + 1) + 9 * (ijk[t0] + 8 * ijk[t1]), fminus = fplus - 1;
                    const uint8_t cp = sc[t + stride], cm = sc[t - stride];
                    if ((cp & CODE_ACTIVE) && face_open(ca, axis))
                    {
                        const float* f = flux[axis][fplus];
                        D[0] -= f[0]; D[1] -= f[1]; D[2] -= f[2];
                    }
                    if ((cm & CODE_ACTIVE) && face_open(cm, axis))
                    {
                        const float* f = flux[axis][fminus];
                        D[0] += f[0]; D[1] += f[1]; D[2] += f[2];
                    }
                }
                if (external)
                {
                    const float area = h * h;
                    if (i == 0 && (fl & PCFD_BRICK_XMIN))
                    {
                        const float normal = u[u_face(bs, slot, 0, j, k)], swept = dt * area * normal;
                        const float in = inflow_value(inflow_slot, inflow, bs, slot, j, k, U);
                        if (swept >= 0.0f) { D[0] += swept * in; D[1] += swept * 0.0f; D[2] += swept * 0.0f; }
                        else { D[0] += swept * sv[0][t]; D[1] += swept * sv[1][t]; D[2] += swept * sv[2][t]; }
                    }
                    if (i == bs - 1 && (fl & PCFD_BRICK_XMAX))
                    {
                        const float normal = u[u_face(bs, slot, bs, j, k)], swept = dt * area * normal;
                        if (swept >= 0.0f) { D[0] += -swept * sv[0][t]; D[1] += -swept * sv[1][t]; D[2] += -swept * sv[2][t]; }
                        else D[0] += -swept * U;
                    }
                }
                if (ca & CODE_DEFERRED) { dx[a] = D[0]; dy[a] = D[1]; dz[a] = D[2]; continue; }
                xn[a] = sv[0][t] + D[0] * inverse; yn[a] = sv[1][t] + D[1] * inverse; zn[a] = sv[2][t] + D[2] * inverse;
            }
        }

        __device__ inline float edge_velocity(int e, const int* source, const int8_t* axis, const int64_t* face, const float* u,
                                              const float* v, const float* w, const float* special)
        {
            const int s = source[e];
            if (s >= 0) return special[s];
            const int ax = axis[e];
            return ax == 0 ? u[face[e]] : (ax == 1 ? v[face[e]] : w[face[e]]);
        }

        struct CompactArgs
        {
            const int *a, *b, *source, *sa, *sb, *pa, *pb;
            const int8_t* axis;
            const int64_t* face;
            const float *area, *conductance, *weight, *disp, *gradient, *volume;
        };

        __device__ inline void compact_transport_flux(const CompactArgs& k, int e, float dt, const float* u, const float* v, const float* w,
                                                      const float* special, const float* x, const float* y, const float* z, float f[3])
        {
            const int first = k.a[e], second = k.b[e];
            const float vel = edge_velocity(e, k.source, k.axis, k.face, u, v, w, special);
            const float swept = dt * k.area[e] * vel;
            const bool from_first = swept >= 0.0f;
            const int donor = from_first ? first : second;
            const int sp = from_first ? k.sa[e] : k.sb[e];
            const float* disp = k.disp + 6 * e + (from_first ? 0 : 3);
            const float courant = fminf(1.0f, fabsf(swept) / k.volume[donor]);
            for (int c = 0; c < 3; ++c)
            {
                const float va = comp3(x, y, z, first, c), vb = comp3(x, y, z, second, c), base = from_first ? va : vb;
                float value = base;
                if (sp >= 0)
                {
                    const float* g = k.gradient + 9 * sp + 3 * c;
                    const float rec = base + (1.0f - courant) * (g[0] * disp[0] + g[1] * disp[1] + g[2] * disp[2]);
                    value = fmaxf(fminf(va, vb), fminf(fmaxf(va, vb), rec));
                }
                f[c] = swept * value;
            }
        }

        // Finish deferred DOFs: structured part (from the brick pass) + compact edges; apply or
        // hand the increment to the group pass.  mode 0 transport, 1 diffusion.
        __global__ void deferred_finish_kernel(int nD, const int* __restrict__ d_dof, const int* __restrict__ d_offset,
            const int* __restrict__ d_edge, const int8_t* __restrict__ d_sign, const int* __restrict__ d_group, int64_t structured,
            CompactArgs k, int mode, float dt, const float* __restrict__ viscosity, const float* __restrict__ u,
            const float* __restrict__ v, const float* __restrict__ w, const float* __restrict__ special, const float* __restrict__ x,
            const float* __restrict__ y, const float* __restrict__ z, const float* __restrict__ dx, const float* __restrict__ dy,
            const float* __restrict__ dz, float* __restrict__ xn, float* __restrict__ yn, float* __restrict__ zn, float* __restrict__ d_delta)
        {
            const int d = blockIdx.x * blockDim.x + threadIdx.x;
            if (d >= nD) return;
            const int q = d_dof[d];
            float D[3] = {0.0f, 0.0f, 0.0f};
            if (q < structured) { D[0] = dx[q]; D[1] = dy[q]; D[2] = dz[q]; }
            for (int t = d_offset[d]; t < d_offset[d + 1]; ++t)
            {
                const int e = d_edge[t];
                const float sign = float(d_sign[t]);
                if (mode == 0)
                {
                    float f[3];
                    compact_transport_flux(k, e, dt, u, v, w, special, x, y, z, f);
                    D[0] += sign * f[0]; D[1] += sign * f[1]; D[2] += sign * f[2];
                }
                else
                {
                    const int a = k.a[e], b = k.b[e];
                    const float scale = dt * k.conductance[e] * 0.5f * (viscosity[a] + viscosity[b]);
                    // lower endpoint (sign -1) gains scale*(vb-va), upper loses it
                    D[0] += -sign * (scale * (x[b] - x[a]));
                    D[1] += -sign * (scale * (y[b] - y[a]));
                    D[2] += -sign * (scale * (z[b] - z[a]));
                }
            }
            if (d_group[d] >= 0) { d_delta[3 * d] = D[0]; d_delta[3 * d + 1] = D[1]; d_delta[3 * d + 2] = D[2]; return; }
            const float inverse = 1.0f / k.volume[q];
            xn[q] = x[q] + D[0] * inverse; yn[q] = y[q] + D[1] * inverse; zn[q] = z[q] + D[2] * inverse;
        }

        // Small-cell group: the summed increment of all members is spread over the group volume.
        __global__ void group_apply_kernel(int nG, const int* __restrict__ g_offset, const int* __restrict__ g_member,
            const float* __restrict__ g_volume, const int* __restrict__ d_dof, const float* __restrict__ d_delta,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float* __restrict__ xn,
            float* __restrict__ yn, float* __restrict__ zn)
        {
            const int g = blockIdx.x * blockDim.x + threadIdx.x;
            if (g >= nG) return;
            float S[3] = {0.0f, 0.0f, 0.0f};
            for (int t = g_offset[g]; t < g_offset[g + 1]; ++t)
            {
                const int d = g_member[t];
                S[0] += d_delta[3 * d]; S[1] += d_delta[3 * d + 1]; S[2] += d_delta[3 * d + 2];
            }
            const float inverse = 1.0f / g_volume[g];
            for (int t = g_offset[g]; t < g_offset[g + 1]; ++t)
            {
                const int q = d_dof[g_member[t]];
                xn[q] = x[q] + S[0] * inverse; yn[q] = y[q] + S[1] * inverse; zn[q] = z[q] + S[2] * inverse;
            }
        }

        // Increment redistribution after an in-place or buffered update (reference
        // accumulate_redistributed_increment / finalize_redistributed_state, :130-149).
        __global__ void group_increment_kernel(int nG, const int* __restrict__ g_offset, const int* __restrict__ g_member,
            const float* __restrict__ g_volume, const int* __restrict__ d_dof, const float* __restrict__ volume,
            const float* __restrict__ bx, const float* __restrict__ by, const float* __restrict__ bz, int base_by_deferred,
            float* __restrict__ x, float* __restrict__ y, float* __restrict__ z)
        {
            const int g = blockIdx.x * blockDim.x + threadIdx.x;
            if (g >= nG) return;
            float S[3] = {0.0f, 0.0f, 0.0f};
            for (int t = g_offset[g]; t < g_offset[g + 1]; ++t)
            {
                const int d = g_member[t], q = d_dof[d], b = base_by_deferred ? d : q;
                const float V = volume[q];
                S[0] += V * (x[q] - bx[b]); S[1] += V * (y[q] - by[b]); S[2] += V * (z[q] - bz[b]);
            }
            const float inverse = 1.0f / g_volume[g];
            for (int t = g_offset[g]; t < g_offset[g + 1]; ++t)
            {
                const int d = g_member[t], q = d_dof[d], b = base_by_deferred ? d : q;
                x[q] = bx[b] + S[0] * inverse; y[q] = by[b] + S[1] * inverse; z[q] = bz[b] + S[2] * inverse;
            }
        }

        // LS velocity gradients at special nodes: g = inverse * sum w (v_n - v_node)
        __global__ void special_gradient_kernel(int nS, const int* __restrict__ s_dof, const int* __restrict__ s_offset,
            const int* __restrict__ s_neighbor, const float* __restrict__ s_weight, const float* __restrict__ s_inverse,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float* __restrict__ gradient)
        {
            const int sp = blockIdx.x * blockDim.x + threadIdx.x;
            if (sp >= nS) return;
            const int node = s_dof[sp];
            float rhs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            const float vn[3] = {x[node], y[node], z[node]};
            for (int t = s_offset[sp]; t < s_offset[sp + 1]; ++t)
            {
                const int o = s_neighbor[t];
                const float d[3] = {x[o] - vn[0], y[o] - vn[1], z[o] - vn[2]};
                for (int c = 0; c < 3; ++c)
                    for (int a = 0; a < 3; ++a) rhs[c * 3 + a] += s_weight[3 * t + a] * d[c];
            }
            const float* m = s_inverse + 9 * sp;
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r)
                    gradient[9 * sp + 3 * c + r] = m[3 * r] * rhs[3 * c] + m[3 * r + 1] * rhs[3 * c + 1] + m[3 * r + 2] * rhs[3 * c + 2];
        }

        // ---------------------------------------------------------------- Smagorinsky
        __device__ inline float strain_rate(const float* g)
        {
            const float sxx = g[0], syy = g[4], szz = g[8];
            const float sxy = 0.5f * (g[1] + g[3]), sxz = 0.5f * (g[2] + g[6]), syz = 0.5f * (g[5] + g[7]);
            return 2.0f * (sxx * sxx + syy * syy + szz * szz + 2.0f * (sxy * sxy + sxz * sxz + syz * syz));
        }

        template <int kBS>
        __global__ void viscosity_struct_kernel(const int* __restrict__ brick_list, int nbricks, int bs_arg, const int* __restrict__ brick_level,
            const int* __restrict__ nbr, const double* __restrict__ level_h, const uint8_t* __restrict__ code,
            const uint8_t* __restrict__ special, const float* __restrict__ volume, const float* __restrict__ x,
            const float* __restrict__ y, const float* __restrict__ z, float nu, float cs, float* __restrict__ viscosity)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(nbricks) * bs * bs * bs) return;
            CellCtx c;
            decode_cell(work, brick_list, bs, brick_level, level_h, c);
            const int64_t a = c.dof;
            if (!(code[a] & CODE_ACTIVE)) return;
            viscosity[a] = nu;
            if (special[a] || cs == 0.0f) return;
            float g[9];
            for (int axis = 0; axis < 3; ++axis)
            {
                const int64_t lo = open_neighbor(bs, nbr, code, c.slot, c.i, c.j, c.k, a, axis, -1);
                const int64_t hi = open_neighbor(bs, nbr, code, c.slot, c.i, c.j, c.k, a, axis, 1);
                for (int comp = 0; comp < 3; ++comp)
                {
                    const float cur = comp3(x, y, z, a, comp);
                    float gv;
                    if (lo >= 0 && hi >= 0) gv = (comp3(x, y, z, hi, comp) - comp3(x, y, z, lo, comp)) / (2.0f * c.h);
                    else if (hi >= 0) gv = (comp3(x, y, z, hi, comp) - cur) / c.h;
                    else if (lo >= 0) gv = (cur - comp3(x, y, z, lo, comp)) / c.h;
                    else gv = 0.0f;
                    g[comp * 3 + axis] = gv;
                }
            }
            const float strain = sqrtf(fmaxf(0.0f, strain_rate(g))), length = cs * cbrtf(volume[a]);
            viscosity[a] += length * length * strain;
        }

        __global__ void viscosity_special_kernel(int nS, const int* __restrict__ s_dof, const float* __restrict__ gradient,
            const float* __restrict__ volume, float nu, float cs, float* __restrict__ viscosity)
        {
            const int sp = blockIdx.x * blockDim.x + threadIdx.x;
            if (sp >= nS) return;
            const int node = s_dof[sp];
            const float strain = sqrtf(fmaxf(0.0f, strain_rate(gradient + 9 * sp))), length = cs * cbrtf(volume[node]);
            viscosity[node] = nu + length * length * strain;
        }

        // Spectral diffusion rate sum(conductance * mean nu) / V per control volume; block maxima.
        __device__ inline float block_max(float v, float* shared)
        {
            for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            if (lane == 0) shared[warp] = v;
            __syncthreads();
            v = threadIdx.x < (blockDim.x >> 5) ? shared[threadIdx.x] : 0.0f;
            if (warp == 0)
                for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
            return v;
        }

        template <int kBS>
        __global__ void __launch_bounds__(256) rate_struct_kernel(const int* __restrict__ brick_list, int nbricks, int bs_arg,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const double* __restrict__ level_h,
            const uint8_t* __restrict__ code, const float* __restrict__ viscosity, float* __restrict__ partial_rate,
            float* __restrict__ block_partial)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            __shared__ float shared[8];
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            float local_max = 0.0f;
            if (work < int64_t(nbricks) * bs * bs * bs)
            {
                CellCtx c;
                decode_cell(work, brick_list, bs, brick_level, level_h, c);
                const int64_t a = c.dof;
                const uint8_t ca = code[a];
                if (ca & CODE_ACTIVE)
                {
                    float rate = 0.0f;
                    for (int axis = 0; axis < 3; ++axis)
                    {
                        const int64_t b = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, 1, nullptr);
                        if (b >= 0 && (code[b] & CODE_ACTIVE) && face_open(ca, axis)) rate += c.h * 0.5f * (viscosity[a] + viscosity[b]);
                        const int64_t p = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, -1, nullptr);
                        if (p >= 0 && (code[p] & CODE_ACTIVE) && face_open(code[p], axis)) rate += c.h * 0.5f * (viscosity[p] + viscosity[a]);
                    }
                    if (ca & CODE_DEFERRED) partial_rate[a] = rate;
                    else
                    {
                        const double hd = level_h[brick_level[c.slot]];
                        local_max = rate / float(hd * hd * hd);
                    }
                }
            }
            local_max = block_max(local_max, shared);
            if (threadIdx.x == 0) block_partial[blockIdx.x] = local_max;
        }

        __global__ void __launch_bounds__(256) rate_deferred_kernel(int nD, const int* __restrict__ d_dof, const int* __restrict__ d_offset,
            const int* __restrict__ d_edge, int64_t structured, CompactArgs k, const float* __restrict__ viscosity,
            const float* __restrict__ partial_rate, float* __restrict__ block_partial)
        {
            __shared__ float shared[8];
            const int d = blockIdx.x * blockDim.x + threadIdx.x;
            float local_max = 0.0f;
            if (d < nD)
            {
                const int q = d_dof[d];
                float rate = q < structured ? partial_rate[q] : 0.0f;
                for (int t = d_offset[d]; t < d_offset[d + 1]; ++t)
                {
                    const int e = d_edge[t];
                    if (k.conductance[e] > 0.0f) rate += k.conductance[e] * 0.5f * (viscosity[k.a[e]] + viscosity[k.b[e]]);
                }
                local_max = rate / k.volume[q];
            }
            local_max = block_max(local_max, shared);
            if (threadIdx.x == 0) block_partial[blockIdx.x] = local_max;
        }

        __global__ void __launch_bounds__(256) max_final_kernel(const float* __restrict__ partial, int count, float* __restrict__ out)
        {
            __shared__ float shared[8];
            float v = 0.0f;
            for (int q = threadIdx.x; q < count; q += blockDim.x) v = fmaxf(v, partial[q]);
            v = block_max(v, shared);
            if (threadIdx.x == 0) *out = v;
        }

        template <int kBS>
        __global__ void diffuse_struct_kernel(const int* __restrict__ brick_list, int nbricks, int bs_arg, const int* __restrict__ brick_level,
            const int* __restrict__ nbr, const double* __restrict__ level_h, const uint8_t* __restrict__ code,
            const float* __restrict__ viscosity, const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
            float dt, float* __restrict__ xn, float* __restrict__ yn, float* __restrict__ zn, float* __restrict__ dx,
            float* __restrict__ dy, float* __restrict__ dz)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(nbricks) * bs * bs * bs) return;
            CellCtx c;
            decode_cell(work, brick_list, bs, brick_level, level_h, c);
            const int64_t a = c.dof;
            const uint8_t ca = code[a];
            if (!(ca & CODE_ACTIVE)) { xn[a] = x[a]; yn[a] = y[a]; zn[a] = z[a]; return; }
            float D[3] = {0.0f, 0.0f, 0.0f};
            for (int axis = 0; axis < 3; ++axis)
            {
                const int64_t b = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, 1, nullptr);
                if (b >= 0 && (code[b] & CODE_ACTIVE) && face_open(ca, axis))
                {
                    const float scale = dt * c.h * 0.5f * (viscosity[a] + viscosity[b]);
                    D[0] += scale * (x[b] - x[a]); D[1] += scale * (y[b] - y[a]); D[2] += scale * (z[b] - z[a]);
                }
                const int64_t p = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, -1, nullptr);
                if (p >= 0 && (code[p] & CODE_ACTIVE) && face_open(code[p], axis))
                {
                    const float scale = dt * c.h * 0.5f * (viscosity[p] + viscosity[a]);
                    D[0] -= scale * (x[a] - x[p]); D[1] -= scale * (y[a] - y[p]); D[2] -= scale * (z[a] - z[p]);
                }
            }
            if (ca & CODE_DEFERRED) { dx[a] = D[0]; dy[a] = D[1]; dz[a] = D[2]; return; }
            const double hd = level_h[brick_level[c.slot]];
            const float inverse = 1.0f / float(hd * hd * hd);
            xn[a] = x[a] + D[0] * inverse; yn[a] = y[a] + D[1] * inverse; zn[a] = z[a] + D[2] * inverse;
        }

        // ---------------------------------------------------------------- smooth wall
        __device__ inline float friction_velocity(float speed, float distance, float nu)
        {
            // Spalding's law written as u+ y+(u+) = Re_y, solved by 36 bisections on u+ in [0, 80].
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

        __global__ void wall_coefficient_kernel(int nW, const int* __restrict__ w_dof, const float* __restrict__ w_normal,
            const float* __restrict__ w_area, const float* __restrict__ w_distance, const float* __restrict__ x,
            const float* __restrict__ y, const float* __restrict__ z, float nu, float* __restrict__ w_k)
        {
            const int s = blockIdx.x * blockDim.x + threadIdx.x;
            if (s >= nW) return;
            const int q = w_dof[s];
            const float* n = w_normal + 3 * s;
            const float vx = x[q], vy = y[q], vz = z[q], un = vx * n[0] + vy * n[1] + vz * n[2];
            const float tx = vx - un * n[0], ty = vy - un * n[1], tz = vz - un * n[2];
            const float speed = sqrtf(fmaxf(0.0f, tx * tx + ty * ty + tz * tz));
            float k = 0.0f;
            if (speed > 0.0f)
            {
                const float uf = friction_velocity(speed, w_distance[s], nu);
                k = w_area[s] * uf * uf / speed;
            }
            w_k[s] = k;
        }

        __global__ void wall_apply_kernel(int nWall, const int* __restrict__ wall_dof, const int* __restrict__ wall_offset,
            const int* __restrict__ wall_side, const float* __restrict__ w_normal, const float* __restrict__ w_k,
            const float* __restrict__ volume, float dt, float* __restrict__ x, float* __restrict__ y, float* __restrict__ z)
        {
            const int n = blockIdx.x * blockDim.x + threadIdx.x;
            if (n >= nWall) return;
            float m[6] = {0, 0, 0, 0, 0, 0};
            for (int t = wall_offset[n]; t < wall_offset[n + 1]; ++t)
            {
                const int s = wall_side[t];
                const float k = w_k[s];
                if (!(k > 0.0f)) continue;
                const float* nn = w_normal + 3 * s;
                m[0] += k * (1.0f - nn[0] * nn[0]); m[1] += -k * nn[0] * nn[1]; m[2] += -k * nn[0] * nn[2];
                m[3] += k * (1.0f - nn[1] * nn[1]); m[4] += -k * nn[1] * nn[2]; m[5] += k * (1.0f - nn[2] * nn[2]);
            }
            const int q = wall_dof[n];
            const float scale = dt / volume[q];
            const float a00 = 1.0f + scale * m[0], a01 = scale * m[1], a02 = scale * m[2], a11 = 1.0f + scale * m[3], a12 = scale * m[4],
                        a22 = 1.0f + scale * m[5];
            const float l00 = sqrtf(a00), l10 = a01 / l00, l20 = a02 / l00, l11 = sqrtf(a11 - l10 * l10), l21 = (a12 - l20 * l10) / l11,
                        l22 = sqrtf(a22 - l20 * l20 - l21 * l21);
            const float v0 = x[q] / l00, v1 = (y[q] - l10 * v0) / l11, v2 = (z[q] - l20 * v0 - l21 * v1) / l22;
            const float n2 = v2 / l22, n1 = (v1 - l21 * n2) / l11, n0 = (v0 - l10 * n1 - l20 * n2) / l00;
            x[q] = n0; y[q] = n1; z[q] = n2;
        }

        __global__ void wall_force_kernel(int nW, const int* __restrict__ w_dof, const float* __restrict__ w_normal,
            const float* __restrict__ w_k, const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
            float* __restrict__ force)
        {
            const int s = blockIdx.x * blockDim.x + threadIdx.x;
            if (s >= nW) return;
            const int q = w_dof[s];
            const float* n = w_normal + 3 * s;
            const float k = w_k[s], un = x[q] * n[0] + y[q] * n[1] + z[q] * n[2];
            force[3 * s] = k * (x[q] - un * n[0]);
            force[3 * s + 1] = k * (y[q] - un * n[1]);
            force[3 * s + 2] = k * (z[q] - un * n[2]);
        }

        __global__ void save_deferred_kernel(int nD, const int* __restrict__ d_dof, const int* __restrict__ d_group,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float* __restrict__ bx,
            float* __restrict__ by, float* __restrict__ bz)
        {
            const int d = blockIdx.x * blockDim.x + threadIdx.x;
            if (d >= nD || d_group[d] < 0) return;
            const int q = d_dof[d];
            bx[d] = x[q]; by[d] = y[q]; bz[d] = z[q];
        }

        // ---------------------------------------------------------------- pressure impulse
        __global__ void pressure_gradient32_kernel(int nodes, const int* __restrict__ dof, const int* __restrict__ offset,
            const int* __restrict__ neighbour, const float* __restrict__ weight, const float* __restrict__ p, float* __restrict__ gradient)
        {
            const int node = blockIdx.x * blockDim.x + threadIdx.x;
            if (node >= nodes) return;
            const float centre = p[dof[node]];
            float gx = 0, gy = 0, gz = 0;
            for (int q = offset[node]; q < offset[node + 1]; ++q)
            {
                const float d = p[neighbour[q]] - centre;
                gx += weight[3 * q] * d; gy += weight[3 * q + 1] * d; gz += weight[3 * q + 2] * d;
            }
            gradient[3 * node] = gx; gradient[3 * node + 1] = gy; gradient[3 * node + 2] = gz;
        }

        // ---------------------------------------------------------------- 8^3 brick forms
        // One CTA per active brick: the brick's codes and the per-cell values an operator reads,
        // with the facing layer of each same-level neighbour (absent neighbours: code 0, inactive),
        // are staged once into a 10^3 shared tile (cells -1..8); the per-cell expressions then read
        // neighbours from shared memory instead of chasing the neighbour table per access.  Same
        // arithmetic, same order as the per-cell kernels above.
        constexpr int kHalo = 10, kHalo3 = 1000;
        __device__ inline int halo_index(int i, int j, int k) { return ((k + 1) * kHalo + (j + 1)) * kHalo + (i + 1); }
        __device__ inline int halo_stride(int axis) { return axis == 0 ? 1 : (axis == 1 ? kHalo : kHalo * kHalo); }

        template <int NF> struct HaloSources { const float* p[NF > 0 ? NF : 1]; };

        template <int NF>
        __device__ inline void stage_halo(int slot, const int* __restrict__ nbr, const uint8_t* __restrict__ code,
                                          HaloSources<NF> src, float (*tile)[kHalo3], uint8_t* tcode, int* neighbour)
        {
            // the brick's own values are loaded into registers first (256 threads, two cells each),
            // so that their latency overlaps the neighbour-table load and the tile clearing
            const int tid = threadIdx.x;
            const int64_t base = int64_t(slot) * 512;
            uint8_t own_code[2];
            float own[2][NF > 0 ? NF : 1];
#pragma unroll
            for (int r = 0; r < 2; ++r)
            {
                const int q = tid + 256 * r;
                own_code[r] = code[base + q];
#pragma unroll
                for (int f = 0; f < NF; ++f) own[r][f] = src.p[f][base + q];
            }
            if (tid < 6) neighbour[tid] = nbr[slot * 6 + tid];
            for (int q = tid; q < kHalo3; q += blockDim.x) tcode[q] = 0;
            __syncthreads();
#pragma unroll
            for (int r = 0; r < 2; ++r)
            {
                const int q = tid + 256 * r, t = halo_index(q & 7, (q >> 3) & 7, q >> 6);
                tcode[t] = own_code[r];
#pragma unroll
                for (int f = 0; f < NF; ++f) tile[f][t] = own[r][f];
            }
            for (int q = tid; q < 6 * 64; q += blockDim.x)
            {
                const int d = q >> 6, a = q & 7, b = (q >> 3) & 7, axis = d >> 1;
                const int ns = neighbour[d];
                if (ns < 0) continue;
                const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
                int si[3], ti[3];
                si[axis] = (d & 1) ? 0 : 7;
                ti[axis] = (d & 1) ? 8 : -1;
                si[t0] = ti[t0] = a;
                si[t1] = ti[t1] = b;
                const int64_t g = int64_t(ns) * 512 + (si[2] * 8 + si[1]) * 8 + si[0];
                const int t = halo_index(ti[0], ti[1], ti[2]);
                tcode[t] = code[g];
                for (int f = 0; f < NF; ++f) tile[f][t] = src.p[f][g];
            }
            __syncthreads();
        }

        __global__ void __launch_bounds__(256) diffuse_brick_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const double* __restrict__ level_h,
            const uint8_t* __restrict__ code, const float* __restrict__ viscosity, const float* __restrict__ x,
            const float* __restrict__ y, const float* __restrict__ z, float dt, float* __restrict__ xn, float* __restrict__ yn,
            float* __restrict__ zn, float* __restrict__ dx, float* __restrict__ dy, float* __restrict__ dz)
        {
            __shared__ float tile[4][kHalo3];      // x, y, z, viscosity
            __shared__ uint8_t tcode[kHalo3];
            __shared__ int neighbour[6];
            const int slot = brick_list[blockIdx.x];
            stage_halo<4>(slot, nbr, code, HaloSources<4>{{x, y, z, viscosity}}, tile, tcode, neighbour);
            const double hd = level_h[brick_level[slot]];
            const float h = float(hd), inverse = 1.0f / float(hd * hd * hd);
            const int64_t base = int64_t(slot) * 512;
            for (int q = threadIdx.x; q < 512; q += blockDim.x)
            {
                const int t = halo_index(q & 7, (q >> 3) & 7, q >> 6);
                const int64_t a = base + q;
                const uint8_t ca = tcode[t];
                if (!(ca & CODE_ACTIVE)) { xn[a] = tile[0][t]; yn[a] = tile[1][t]; zn[a] = tile[2][t]; continue; }
                float D[3] = {0.0f, 0.0f, 0.0f};
                for (int axis = 0; axis < 3; ++axis)
                {
                    const int s = halo_stride(axis), b = t + s, p = t - s;
                    if ((tcode[b] & CODE_ACTIVE) && face_open(ca, axis))
                    {
                        const float scale = dt * h * 0.5f * (tile[3][t] + tile[3][b]);
                        D[0] += scale * (tile[0][b] - tile[0][t]); D[1] += scale * (tile[1][b] - tile[1][t]);
                        D[2] += scale * (tile[2][b] - tile[2][t]);
                    }
                    if ((tcode[p] & CODE_ACTIVE) && face_open(tcode[p], axis))
                    {
                        const float scale = dt * h * 0.5f * (tile[3][p] + tile[3][t]);
                        D[0] -= scale * (tile[0][t] - tile[0][p]); D[1] -= scale * (tile[1][t] - tile[1][p]);
                        D[2] -= scale * (tile[2][t] - tile[2][p]);
                    }
                }
                if (ca & CODE_DEFERRED) { dx[a] = D[0]; dy[a] = D[1]; dz[a] = D[2]; continue; }
                xn[a] = tile[0][t] + D[0] * inverse; yn[a] = tile[1][t] + D[1] * inverse; zn[a] = tile[2][t] + D[2] * inverse;
            }
        }

        __global__ void __launch_bounds__(256) viscosity_brick_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const double* __restrict__ level_h,
            const uint8_t* __restrict__ code, const uint8_t* __restrict__ special, const float* __restrict__ volume,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float nu, float cs,
            float* __restrict__ viscosity)
        {
            __shared__ float tile[3][kHalo3];
            __shared__ uint8_t tcode[kHalo3];
            __shared__ int neighbour[6];
            const int slot = brick_list[blockIdx.x];
            stage_halo<3>(slot, nbr, code, HaloSources<3>{{x, y, z}}, tile, tcode, neighbour);
            const float h = float(level_h[brick_level[slot]]);
            const int64_t base = int64_t(slot) * 512;
            for (int q = threadIdx.x; q < 512; q += blockDim.x)
            {
                const int t = halo_index(q & 7, (q >> 3) & 7, q >> 6);
                const int64_t a = base + q;
                const uint8_t ca = tcode[t];
                if (!(ca & CODE_ACTIVE)) continue;
                float value = nu;
                if (!special[a] && cs != 0.0f)
                {
                    float g[9];
                    for (int axis = 0; axis < 3; ++axis)
                    {
                        const int s = halo_stride(axis), lo = t - s, hi = t + s;
                        // open_neighbor: the neighbour is active and the face between them is open
                        const bool has_lo = (tcode[lo] & CODE_ACTIVE) && face_open(tcode[lo], axis);
                        const bool has_hi = (tcode[hi] & CODE_ACTIVE) && face_open(ca, axis);
                        for (int comp = 0; comp < 3; ++comp)
                        {
                            const float cur = tile[comp][t];
                            float gv;
                            if (has_lo && has_hi) gv = (tile[comp][hi] - tile[comp][lo]) / (2.0f * h);
                            else if (has_hi) gv = (tile[comp][hi] - cur) / h;
                            else if (has_lo) gv = (cur - tile[comp][lo]) / h;
                            else gv = 0.0f;
                            g[comp * 3 + axis] = gv;
                        }
                    }
                    const float strain = sqrtf(fmaxf(0.0f, strain_rate(g))), length = cs * cbrtf(volume[a]);
                    value += length * length * strain;
                }
                viscosity[a] = value;
            }
        }

        __global__ void __launch_bounds__(256) rate_brick_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const double* __restrict__ level_h,
            const uint8_t* __restrict__ code, const float* __restrict__ viscosity, float* __restrict__ partial_rate,
            float* __restrict__ block_partial)
        {
            __shared__ float tile[1][kHalo3];
            __shared__ uint8_t tcode[kHalo3];
            __shared__ int neighbour[6];
            __shared__ float shared[8];
            const int slot = brick_list[blockIdx.x];
            stage_halo<1>(slot, nbr, code, HaloSources<1>{{viscosity}}, tile, tcode, neighbour);
            const double hd = level_h[brick_level[slot]];
            const float h = float(hd);
            const int64_t base = int64_t(slot) * 512;
            float local_max = 0.0f;
            for (int q = threadIdx.x; q < 512; q += blockDim.x)
            {
                const int t = halo_index(q & 7, (q >> 3) & 7, q >> 6);
                const uint8_t ca = tcode[t];
                if (!(ca & CODE_ACTIVE)) continue;
                float rate = 0.0f;
                for (int axis = 0; axis < 3; ++axis)
                {
                    const int s = halo_stride(axis), b = t + s, p = t - s;
                    if ((tcode[b] & CODE_ACTIVE) && face_open(ca, axis)) rate += h * 0.5f * (tile[0][t] + tile[0][b]);
                    if ((tcode[p] & CODE_ACTIVE) && face_open(tcode[p], axis)) rate += h * 0.5f * (tile[0][p] + tile[0][t]);
                }
                if (ca & CODE_DEFERRED) partial_rate[base + q] = rate;
                else local_max = fmaxf(local_max, rate / float(hd * hd * hd));
            }
            local_max = block_max(local_max, shared);
            if (threadIdx.x == 0) block_partial[blockIdx.x] = local_max;
        }

        __global__ void __launch_bounds__(256) impulse_brick_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const uint32_t* __restrict__ flags,
            const double* __restrict__ level_h, const uint8_t* __restrict__ code, const float* __restrict__ p, float scale,
            int outlet, int physical, const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
            float* __restrict__ xn, float* __restrict__ yn, float* __restrict__ zn, float* __restrict__ dx, float* __restrict__ dy,
            float* __restrict__ dz)
        {
            __shared__ float tile[1][kHalo3];
            __shared__ uint8_t tcode[kHalo3];
            __shared__ int neighbour[6];
            const int slot = brick_list[blockIdx.x];
            stage_halo<1>(slot, nbr, code, HaloSources<1>{{p}}, tile, tcode, neighbour);
            const double hd = level_h[brick_level[slot]];
            const float h = float(hd), area = h * h, inverse = 1.0f / float(hd * hd * hd);
            const uint32_t fl = flags[slot];
            const int64_t base = int64_t(slot) * 512;
            for (int q = threadIdx.x; q < 512; q += blockDim.x)
            {
                const int i = q & 7, j = (q >> 3) & 7, k = q >> 6, t = halo_index(i, j, k);
                const int64_t a = base + q;
                const uint8_t ca = tcode[t];
                if (!(ca & CODE_ACTIVE)) { xn[a] = x[a]; yn[a] = y[a]; zn[a] = z[a]; continue; }
                float D[3] = {0.0f, 0.0f, 0.0f};
                for (int axis = 0; axis < 3; ++axis)
                {
                    const int s = halo_stride(axis), b = t + s, m = t - s;
                    if ((tcode[b] & CODE_ACTIVE) && face_open(ca, axis)) D[axis] -= scale * area * 0.5f * (tile[0][t] + tile[0][b]);
                    if ((tcode[m] & CODE_ACTIVE) && face_open(tcode[m], axis)) D[axis] += scale * area * 0.5f * (tile[0][m] + tile[0][t]);
                }
                if (physical)
                {
                    const float boundary = scale * area * tile[0][t];
                    if (i == 0 && (fl & PCFD_BRICK_XMIN)) D[0] += boundary;
                    if (i == 7 && (fl & PCFD_BRICK_XMAX) && !outlet) D[0] -= boundary;
                    if (j == 0 && (fl & PCFD_BRICK_YMIN)) D[1] += boundary;
                    if (j == 7 && (fl & PCFD_BRICK_YMAX)) D[1] -= boundary;
                    if (k == 0 && (fl & PCFD_BRICK_ZMIN)) D[2] += boundary;
                    if (k == 7 && (fl & PCFD_BRICK_ZMAX)) D[2] -= boundary;
                }
                if (ca & CODE_DEFERRED) { dx[a] = D[0]; dy[a] = D[1]; dz[a] = D[2]; continue; }
                xn[a] = x[a] + D[0] * inverse; yn[a] = y[a] + D[1] * inverse; zn[a] = z[a] + D[2] * inverse;
            }
        }

        __global__ void __launch_bounds__(256) reconstruct_brick_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ nbr, const uint8_t* __restrict__ code, const float* __restrict__ x, const float* __restrict__ y,
            const float* __restrict__ z, float* u, float* v, float* w)
        {
            __shared__ float tile[3][kHalo3];
            __shared__ uint8_t tcode[kHalo3];
            __shared__ int neighbour[6];
            const int slot = brick_list[blockIdx.x];
            stage_halo<3>(slot, nbr, code, HaloSources<3>{{x, y, z}}, tile, tcode, neighbour);
            for (int q = threadIdx.x; q < 512; q += blockDim.x)
            {
                const int ijk[3] = {q & 7, (q >> 3) & 7, q >> 6};
                const int t = halo_index(ijk[0], ijk[1], ijk[2]);
                const uint8_t ca = tcode[t];
                if (!(ca & CODE_ACTIVE)) continue;
                for (int axis = 0; axis < 3; ++axis)
                {
                    const int b = t + halo_stride(axis);
                    if (!(tcode[b] & CODE_ACTIVE) || !face_open(ca, axis)) continue;
                    const float value = 0.5f * (tile[axis][t] + tile[axis][b]);
                    int f[3] = {ijk[0], ijk[1], ijk[2]};
                    ++f[axis];
                    float* faces = axis == 0 ? u : (axis == 1 ? v : w);
                    faces[axis_face(8, axis, slot, f[0], f[1], f[2])] = value;
                    if (ijk[axis] == 7)
                    {
                        // the shared face is stored in the neighbour brick too (its face 0)
                        int m[3] = {ijk[0], ijk[1], ijk[2]};
                        m[axis] = 0;
                        faces[axis_face(8, axis, neighbour[2 * axis + 1], m[0], m[1], m[2])] = value;
                    }
                }
            }
        }

        __global__ void __launch_bounds__(256) cfl_brick_kernel(const int* __restrict__ brick_list,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const uint32_t* __restrict__ flags,
            const double* __restrict__ level_h, const uint8_t* __restrict__ code, const float* __restrict__ u,
            const float* __restrict__ v, const float* __restrict__ w, const float* __restrict__ x, const float* __restrict__ y,
            const float* __restrict__ z, int external, float* __restrict__ partial_outflow, float* __restrict__ block_partial)
        {
            __shared__ uint8_t tcode[kHalo3];
            __shared__ int neighbour[6];
            __shared__ float shared[8];
            const int slot = brick_list[blockIdx.x];
            stage_halo<0>(slot, nbr, code, HaloSources<0>{{nullptr}}, nullptr, tcode, neighbour);
            const double hd = level_h[brick_level[slot]];
            const float h = float(hd), area = h * h;
            const uint32_t fl = flags[slot];
            const int64_t base = int64_t(slot) * 512;
            float vmax = 0.0f, rmax = 0.0f;
            for (int q = threadIdx.x; q < 512; q += blockDim.x)
            {
                const int ijk[3] = {q & 7, (q >> 3) & 7, q >> 6};
                const int t = halo_index(ijk[0], ijk[1], ijk[2]);
                const int64_t a = base + q;
                const uint8_t ca = tcode[t];
                if (!(ca & CODE_ACTIVE)) continue;
                vmax = fmaxf(vmax, fmaxf(fabsf(x[a]), fmaxf(fabsf(y[a]), fabsf(z[a]))));
                float out = 0.0f;
                for (int axis = 0; axis < 3; ++axis)
                {
                    const int s = halo_stride(axis), b = t + s, p = t - s;
                    if ((tcode[b] & CODE_ACTIVE) && face_open(ca, axis))
                    {
                        int f[3] = {ijk[0], ijk[1], ijk[2]};
                        ++f[axis];
                        out += fmaxf(area * face_at(u, v, w, 8, axis, slot, f[0], f[1], f[2]), 0.0f);
                    }
                    if ((tcode[p] & CODE_ACTIVE) && face_open(tcode[p], axis))
                    {
                        // the lower neighbour's +axis face (in its own brick)
                        int f[3] = {ijk[0], ijk[1], ijk[2]};
                        const int sp = f[axis] == 0 ? neighbour[2 * axis] : slot;
                        f[axis] = f[axis] == 0 ? 8 : f[axis];
                        out += fmaxf(-(area * face_at(u, v, w, 8, axis, sp, f[0], f[1], f[2])), 0.0f);
                    }
                }
                if (external)
                {
                    if (ijk[0] == 0 && (fl & PCFD_BRICK_XMIN)) out += fmaxf(-area * u[u_face(8, slot, 0, ijk[1], ijk[2])], 0.0f);
                    if (ijk[0] == 7 && (fl & PCFD_BRICK_XMAX)) out += fmaxf(area * u[u_face(8, slot, 8, ijk[1], ijk[2])], 0.0f);
                }
                if (ca & CODE_DEFERRED) partial_outflow[a] = out;
                else rmax = fmaxf(rmax, out / float(hd * hd * hd));
            }
            vmax = block_max(vmax, shared);
            __syncthreads();
            rmax = block_max(rmax, shared);
            if (threadIdx.x == 0) { block_partial[2 * blockIdx.x] = vmax; block_partial[2 * blockIdx.x + 1] = rmax; }
        }

        template <int kBS>
        __global__ void impulse_struct_kernel(const int* __restrict__ brick_list, int nbricks, int bs_arg, const int* __restrict__ brick_level,
            const int* __restrict__ nbr, const uint32_t* __restrict__ flags, const double* __restrict__ level_h,
            const uint8_t* __restrict__ code, const float* __restrict__ p, float scale, int outlet, int physical,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float* __restrict__ xn,
            float* __restrict__ yn, float* __restrict__ zn, float* __restrict__ dx, float* __restrict__ dy, float* __restrict__ dz)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(nbricks) * bs * bs * bs) return;
            CellCtx c;
            decode_cell(work, brick_list, bs, brick_level, level_h, c);
            const int64_t a = c.dof;
            const uint8_t ca = code[a];
            if (!(ca & CODE_ACTIVE)) { xn[a] = x[a]; yn[a] = y[a]; zn[a] = z[a]; return; }
            const float area = c.h * c.h;
            float D[3] = {0.0f, 0.0f, 0.0f};
            for (int axis = 0; axis < 3; ++axis)
            {
                const int64_t b = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, 1, nullptr);
                if (b >= 0 && (code[b] & CODE_ACTIVE) && face_open(ca, axis)) D[axis] -= scale * area * 0.5f * (p[a] + p[b]);
                const int64_t q = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, -1, nullptr);
                if (q >= 0 && (code[q] & CODE_ACTIVE) && face_open(code[q], axis)) D[axis] += scale * area * 0.5f * (p[q] + p[a]);
            }
            if (physical)
            {
                const float boundary = scale * area * p[a];
                const uint32_t fl = flags[c.slot];
                if (c.i == 0 && (fl & PCFD_BRICK_XMIN)) D[0] += boundary;
                if (c.i == bs - 1 && (fl & PCFD_BRICK_XMAX) && !outlet) D[0] -= boundary;
                if (c.j == 0 && (fl & PCFD_BRICK_YMIN)) D[1] += boundary;
                if (c.j == bs - 1 && (fl & PCFD_BRICK_YMAX)) D[1] -= boundary;
                if (c.k == 0 && (fl & PCFD_BRICK_ZMIN)) D[2] += boundary;
                if (c.k == bs - 1 && (fl & PCFD_BRICK_ZMAX)) D[2] -= boundary;
            }
            if (ca & CODE_DEFERRED) { dx[a] = D[0]; dy[a] = D[1]; dz[a] = D[2]; return; }
            const double hd = level_h[brick_level[c.slot]];
            const float inverse = 1.0f / float(hd * hd * hd);
            xn[a] = x[a] + D[0] * inverse; yn[a] = y[a] + D[1] * inverse; zn[a] = z[a] + D[2] * inverse;
        }

        __global__ void impulse_deferred_kernel(int nD, const int* __restrict__ d_dof, const int* __restrict__ d_offset,
            const int* __restrict__ d_edge, const int8_t* __restrict__ d_sign, const int* __restrict__ d_side_offset,
            const int* __restrict__ d_side, const int* __restrict__ d_boundary_offset, const int* __restrict__ d_boundary,
            int64_t structured, CompactArgs k, const float* __restrict__ p, const float* __restrict__ pgrad,
            const int* __restrict__ w_pnode, const float* __restrict__ w_coefficient, const float* __restrict__ w_disp,
            const float* __restrict__ b_coefficient, float scale, int physical, const float* __restrict__ x,
            const float* __restrict__ y, const float* __restrict__ z, const float* __restrict__ dx, const float* __restrict__ dy,
            const float* __restrict__ dz, float* __restrict__ xn, float* __restrict__ yn, float* __restrict__ zn)
        {
            const int d = blockIdx.x * blockDim.x + threadIdx.x;
            if (d >= nD) return;
            const int q = d_dof[d];
            float D[3] = {0.0f, 0.0f, 0.0f};
            if (q < structured) { D[0] = dx[q]; D[1] = dy[q]; D[2] = dz[q]; }
            for (int t = d_offset[d]; t < d_offset[d + 1]; ++t)
            {
                const int e = d_edge[t];
                const int lo = k.a[e], up = k.b[e], ga = k.pa[e], gb = k.pb[e];
                const float wgt = k.weight[e];
                float fp = (1.0f - wgt) * p[lo] + wgt * p[up];
                if (ga >= 0 && gb >= 0)
                    for (int c = 0; c < 3; ++c)
                    {
                        const float skew = (1.0f - wgt) * k.disp[6 * e + c] + wgt * k.disp[6 * e + 3 + c];
                        fp += skew * ((1.0f - wgt) * pgrad[3 * ga + c] + wgt * pgrad[3 * gb + c]);
                    }
                const float impulse = scale * k.area[e] * fp;
                D[k.axis[e]] += float(d_sign[t]) * impulse;   // lower loses, upper gains
            }
            for (int t = d_side_offset[d]; t < d_side_offset[d + 1]; ++t)
            {
                const int s = d_side[t], g = w_pnode[s];
                float pw = p[q];
                if (g >= 0)
                    for (int c = 0; c < 3; ++c) pw += pgrad[3 * g + c] * w_disp[3 * s + c];
                const float impulse = scale * pw;
                D[0] += impulse * w_coefficient[3 * s]; D[1] += impulse * w_coefficient[3 * s + 1]; D[2] += impulse * w_coefficient[3 * s + 2];
            }
            if (physical)
                for (int t = d_boundary_offset[d]; t < d_boundary_offset[d + 1]; ++t)
                {
                    const int f = d_boundary[t];
                    const float impulse = scale * p[q];
                    D[0] += impulse * b_coefficient[3 * f]; D[1] += impulse * b_coefficient[3 * f + 1]; D[2] += impulse * b_coefficient[3 * f + 2];
                }
            const float inverse = 1.0f / k.volume[q];
            xn[q] = x[q] + D[0] * inverse; yn[q] = y[q] + D[1] * inverse; zn[q] = z[q] + D[2] * inverse;
        }

        // ---------------------------------------------------------------- reconstruction
        template <int kBS>
        __global__ void reconstruct_struct_kernel(const int* __restrict__ brick_list, int nbricks, int bs_arg, const int* __restrict__ brick_level,
            const int* __restrict__ nbr, const double* __restrict__ level_h, const uint8_t* __restrict__ code,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z, float* u, float* v, float* w)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(nbricks) * bs * bs * bs) return;
            CellCtx c;
            decode_cell(work, brick_list, bs, brick_level, level_h, c);
            const int64_t a = c.dof;
            const uint8_t ca = code[a];
            if (!(ca & CODE_ACTIVE)) return;
            for (int axis = 0; axis < 3; ++axis)
            {
                int sb = c.slot;
                const int64_t b = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, 1, &sb);
                if (b < 0 || !(code[b] & CODE_ACTIVE) || !face_open(ca, axis)) continue;
                const float value = 0.5f * (comp3(x, y, z, a, axis) + comp3(x, y, z, b, axis));
                int f[3] = {c.i, c.j, c.k};
                ++f[axis];
                float* faces = axis == 0 ? u : (axis == 1 ? v : w);
                faces[axis_face(bs, axis, c.slot, f[0], f[1], f[2])] = value;
                if (sb != c.slot)
                {
                    int m[3] = {c.i, c.j, c.k};
                    m[axis] = 0;
                    faces[axis_face(bs, axis, sb, m[0], m[1], m[2])] = value;
                }
            }
        }

        __global__ void reconstruct_compact_kernel(int nK, CompactArgs k, const float* __restrict__ x, const float* __restrict__ y,
            const float* __restrict__ z, float* u, float* v, float* w, float* special)
        {
            const int e = blockIdx.x * blockDim.x + threadIdx.x;
            if (e >= nK) return;
            const int comp = k.axis[e];
            const float wgt = k.weight[e];
            const int a = k.a[e], b = k.b[e];
            const float va = comp3(x, y, z, a, comp), vb = comp3(x, y, z, b, comp);
            const float* da = k.disp + 6 * e;
            const float* db = da + 3;
            const float skew[3] = {(1.0f - wgt) * da[0] + wgt * db[0], (1.0f - wgt) * da[1] + wgt * db[1], (1.0f - wgt) * da[2] + wgt * db[2]};
            float corr[2] = {0.0f, 0.0f};
            for (int side = 0; side < 2; ++side)
            {
                const int sp = side ? k.sb[e] : k.sa[e];
                if (sp < 0) continue;
                const float* g = k.gradient + 9 * sp + 3 * comp;
                corr[side] = g[0] * skew[0] + g[1] * skew[1] + g[2] * skew[2];
            }
            const float value = (1.0f - wgt) * va + wgt * vb + minmod_cell(corr[0], corr[1]);
            const int s = k.source[e];
            if (s >= 0) special[s] = value;
            else
            {
                float* faces = comp == 0 ? u : (comp == 1 ? v : w);
                faces[k.face[e]] = value;
            }
        }

        // ---------------------------------------------------------------- boundaries
        __global__ void external_boundary_kernel(const int* __restrict__ brick_list, int nbricks, int bs, const uint32_t* __restrict__ flags,
            float speed, const int* __restrict__ inflow_slot, const float* __restrict__ inflow, float* u, float* v, float* w)
        {
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            const int per = bs * bs;
            if (work >= int64_t(nbricks) * 6 * per) return;
            const int brick = int(work / (6 * per)), rem = int(work % (6 * per)), face = rem / per, a = rem % bs, b = (rem / bs) % bs;
            const int slot = brick_list[brick];
            const uint32_t fl = flags[slot];
            if (!(fl & (1u << face))) return;
            if (face == 0) u[u_face(bs, slot, 0, a, b)] = inflow_value(inflow_slot, inflow, bs, slot, a, b, speed);   // X-min inflow
            else if (face == 2 || face == 3) v[v_face(bs, slot, a, face == 3 ? bs : 0, b)] = 0.0f;   // Y free slip
            else if (face == 4 || face == 5) w[w_face(bs, slot, a, b, face == 5 ? bs : 0)] = 0.0f;   // Z free slip
        }

        // ---------------------------------------------------------------- CFL reductions
        template <int kBS>
        __global__ void __launch_bounds__(256) cfl_struct_kernel(const int* __restrict__ brick_list, int nbricks, int bs_arg,
            const int* __restrict__ brick_level, const int* __restrict__ nbr, const uint32_t* __restrict__ flags,
            const double* __restrict__ level_h, const uint8_t* __restrict__ code, const float* __restrict__ u,
            const float* __restrict__ v, const float* __restrict__ w, const float* __restrict__ x, const float* __restrict__ y,
            const float* __restrict__ z, int external, float* __restrict__ partial_outflow, float* __restrict__ block_partial)
        {
            const int bs = kBS ? kBS : bs_arg;   // 8^3 bricks: index math folded at compile time
            __shared__ float shared[8];
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            float vmax = 0.0f, rmax = 0.0f;
            if (work < int64_t(nbricks) * bs * bs * bs)
            {
                CellCtx c;
                decode_cell(work, brick_list, bs, brick_level, level_h, c);
                const int64_t a = c.dof;
                const uint8_t ca = code[a];
                if (ca & CODE_ACTIVE)
                {
                    vmax = fmaxf(fabsf(x[a]), fmaxf(fabsf(y[a]), fabsf(z[a])));
                    const float area = c.h * c.h;
                    float out = 0.0f;
                    for (int axis = 0; axis < 3; ++axis)
                    {
                        const int64_t b = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, 1, nullptr);
                        if (b >= 0 && (code[b] & CODE_ACTIVE) && face_open(ca, axis))
                        {
                            int f[3] = {c.i, c.j, c.k};
                            ++f[axis];
                            out += fmaxf(area * face_at(u, v, w, bs, axis, c.slot, f[0], f[1], f[2]), 0.0f);
                        }
                        int sp;
                        const int64_t p = step_dof(bs, nbr, c.slot, c.i, c.j, c.k, axis, -1, &sp);
                        if (p >= 0 && (code[p] & CODE_ACTIVE) && face_open(code[p], axis))
                        {
                            // the lower neighbour's +axis face (in its own brick)
                            int f[3] = {c.i, c.j, c.k};
                            f[axis] = f[axis] == 0 ? bs : f[axis];
                            out += fmaxf(-(area * face_at(u, v, w, bs, axis, sp, f[0], f[1], f[2])), 0.0f);
                        }
                    }
                    if (external)
                    {
                        const uint32_t fl = flags[c.slot];
                        if (c.i == 0 && (fl & PCFD_BRICK_XMIN)) out += fmaxf(-area * u[u_face(bs, c.slot, 0, c.j, c.k)], 0.0f);
                        if (c.i == bs - 1 && (fl & PCFD_BRICK_XMAX)) out += fmaxf(area * u[u_face(bs, c.slot, bs, c.j, c.k)], 0.0f);
                    }
                    if (ca & CODE_DEFERRED) partial_outflow[a] = out;
                    else
                    {
                        const double hd = level_h[brick_level[c.slot]];
                        rmax = out / float(hd * hd * hd);
                    }
                }
            }
            vmax = block_max(vmax, shared);
            __syncthreads();
            rmax = block_max(rmax, shared);
            if (threadIdx.x == 0) { block_partial[2 * blockIdx.x] = vmax; block_partial[2 * blockIdx.x + 1] = rmax; }
        }

        __global__ void __launch_bounds__(256) cfl_deferred_kernel(int nD, const int* __restrict__ d_dof, const int* __restrict__ d_offset,
            const int* __restrict__ d_edge, const int8_t* __restrict__ d_sign, int64_t structured, CompactArgs k,
            const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w, const float* __restrict__ special,
            const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
            const float* __restrict__ partial_outflow, float* __restrict__ block_partial)
        {
            __shared__ float shared[8];
            const int d = blockIdx.x * blockDim.x + threadIdx.x;
            float vmax = 0.0f, rmax = 0.0f;
            if (d < nD)
            {
                const int q = d_dof[d];
                vmax = fmaxf(fabsf(x[q]), fmaxf(fabsf(y[q]), fabsf(z[q])));
                float out = q < structured ? partial_outflow[q] : 0.0f;
                for (int t = d_offset[d]; t < d_offset[d + 1]; ++t)
                {
                    const int e = d_edge[t];
                    if (!(k.area[e] > 0.0f)) continue;
                    const float flux = k.area[e] * edge_velocity(e, k.source, k.axis, k.face, u, v, w, special);
                    out += d_sign[t] < 0 ? fmaxf(flux, 0.0f) : fmaxf(-flux, 0.0f);
                }
                rmax = out / k.volume[q];
            }
            vmax = block_max(vmax, shared);
            __syncthreads();
            rmax = block_max(rmax, shared);
            if (threadIdx.x == 0) { block_partial[2 * blockIdx.x] = vmax; block_partial[2 * blockIdx.x + 1] = rmax; }
        }

        // grid-wide maxima of the per-block partials and of |special|; out (zeroed before) holds the
        // non-negative maxima as float bit patterns, whose unsigned order is their float order
        __global__ void __launch_bounds__(256) cfl_final_kernel(const float* __restrict__ partial, int count, const float* __restrict__ special,
            int nspecial, unsigned int* __restrict__ out)
        {
            __shared__ float shared[8];
            float vm = 0.0f, rm = 0.0f, sm = 0.0f;
            const int stride = gridDim.x * blockDim.x;
            for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += stride)
            {
                vm = fmaxf(vm, partial[2 * q]);
                rm = fmaxf(rm, partial[2 * q + 1]);
            }
            for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nspecial; q += stride) sm = fmaxf(sm, fabsf(special[q]));
            vm = block_max(vm, shared);
            __syncthreads();
            rm = block_max(rm, shared);
            __syncthreads();
            sm = block_max(sm, shared);
            if (threadIdx.x == 0)
            {
                atomicMax(&out[0], __float_as_uint(vm));
                atomicMax(&out[1], __float_as_uint(rm));
                atomicMax(&out[2], __float_as_uint(sm));
            }
        }

        CompactArgs compact_args(System& s, Momentum& m)
        {
            CompactArgs k;
            k.a = m.k_a; k.b = m.k_b; k.source = m.k_source; k.sa = m.k_sa; k.sb = m.k_sb; k.pa = m.k_pnode_a; k.pb = m.k_pnode_b;
            k.axis = m.k_axis; k.face = m.k_face; k.area = m.k_area; k.conductance = m.k_conductance; k.weight = m.k_weight;
            k.disp = m.k_disp; k.gradient = m.s_gradient; k.volume = m.volume32;
            (void)s;
            return k;
        }

        int cell_blocks(System& s) { return blocks_for(int64_t(s.active_bricks) * s.bs3); }

        void swap_state(Momentum& m)
        {
            std::swap(m.x.p, m.xn.p);
            std::swap(m.y.p, m.yn.p);
            std::swap(m.z.p, m.zn.p);
        }

        void special_gradients(System& s, Momentum& m)
        {
            if (m.nS)
                special_gradient_kernel<<<blocks_for(m.nS), kThreads, 0, launch_stream(s)>>>(m.nS, m.s_dof, m.s_offset, m.s_neighbor, m.s_weight,
                                                                                   m.s_inverse, m.x, m.y, m.z, m.s_gradient);
        }

        void finish_buffered(System& s, Momentum& m, int mode, float dt)
        {
            const CompactArgs k = compact_args(s, m);
            if (m.nD)
                deferred_finish_kernel<<<blocks_for(m.nD), kThreads, 0, launch_stream(s)>>>(
                    m.nD, m.d_dof, m.d_offset, m.d_edge, m.d_sign, m.d_group, s.structured, k, mode, dt, m.viscosity, s.u, s.v, s.w,
                    s.special, m.x, m.y, m.z, m.dx, m.dy, m.dz, m.xn, m.yn, m.zn, m.d_delta);
            if (m.nG)
                group_apply_kernel<<<blocks_for(m.nG), kThreads, 0, launch_stream(s)>>>(m.nG, m.g_offset, m.g_member, m.g_volume, m.d_dof,
                                                                               m.d_delta, m.x, m.y, m.z, m.xn, m.yn, m.zn);
            swap_state(m);
        }
    }

    void momentum_transport(System& s, Momentum& m, float dt, float freestream, bool external_aero)
    {
        special_gradients(s, m);
        if (s.active_bricks && s.bs == 8)
            transport_brick_kernel<<<s.active_bricks, 256, 0, launch_stream(s)>>>(
                s.active_brick_list, s.brick_level, s.brick_nbr, s.brick_flags, s.d_level_h, m.code, s.u, s.v, s.w, m.x, m.y, m.z, dt,
                external_aero ? 1 : 0, freestream, s.inflow_slot_of_brick, s.inflow_set ? s.inflow.p : nullptr, m.xn, m.yn, m.zn, m.dx,
                m.dy, m.dz);
        else if (s.active_bricks)
            transport_struct_kernel<0><<<cell_blocks(s), kThreads, 0, launch_stream(s)>>>(
                s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr, s.brick_flags, s.d_level_h, m.code, s.u, s.v,
                s.w, m.x, m.y, m.z, dt, external_aero ? 1 : 0, freestream, s.inflow_slot_of_brick, s.inflow_set ? s.inflow.p : nullptr, m.xn, m.yn, m.zn, m.dx, m.dy, m.dz);
        finish_buffered(s, m, 0, dt);
        cuda_check(cudaGetLastError(), "momentum transport");
    }

    double momentum_smagorinsky(System& s, Momentum& m, float nu, float cs, float dt)
    {
        if (nu == 0.0f && cs == 0.0f) { m.last_rate = 0; m.last_substeps = 1; return 0; }
        special_gradients(s, m);
        const bool bricks8 = s.active_bricks && s.bs == 8;
        if (bricks8)
            viscosity_brick_kernel<<<s.active_bricks, 256, 0, launch_stream(s)>>>(
                s.active_brick_list, s.brick_level, s.brick_nbr, s.d_level_h, m.code, m.special, m.volume32, m.x, m.y, m.z, nu, cs,
                m.viscosity);
        else if (s.active_bricks)
            viscosity_struct_kernel<0><<<cell_blocks(s), kThreads, 0, launch_stream(s)>>>(
                s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr, s.d_level_h, m.code, m.special, m.volume32,
                m.x, m.y, m.z, nu, cs, m.viscosity);
        if (m.nS)
            viscosity_special_kernel<<<blocks_for(m.nS), kThreads, 0, launch_stream(s)>>>(m.nS, m.s_dof, m.s_gradient, m.volume32, nu, cs, m.viscosity);
        // spectral rate -> substeps (one scalar readback)
        const CompactArgs k = compact_args(s, m);
        const int cb = s.active_bricks ? (bricks8 ? s.active_bricks : cell_blocks(s)) : 0, db = m.nD ? blocks_for(m.nD) : 0;
        require(cb + db <= int(m.reduce_partial.n), "reduction scratch too small");
        if (bricks8)
            rate_brick_kernel<<<cb, 256, 0, launch_stream(s)>>>(s.active_brick_list, s.brick_level, s.brick_nbr, s.d_level_h, m.code,
                                                               m.viscosity, m.dx, m.reduce_partial);
        else if (cb)
            rate_struct_kernel<0><<<cb, 256, 0, launch_stream(s)>>>(s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr,
                                                        s.d_level_h, m.code, m.viscosity, m.dx, m.reduce_partial);
        if (db)
            rate_deferred_kernel<<<db, 256, 0, launch_stream(s)>>>(m.nD, m.d_dof, m.d_offset, m.d_edge, s.structured, k, m.viscosity, m.dx,
                                                          m.reduce_partial.p + cb);
        max_final_kernel<<<1, 256, 0, launch_stream(s)>>>(m.reduce_partial, cb + db, m.reduce_result);
        cuda_check(cudaMemcpyAsync(m.pinned, m.reduce_result, sizeof(float), cudaMemcpyDeviceToHost, s.stream), "rate readback");
        cuda_check(cudaStreamSynchronize(s.stream), "rate readback");
        m.last_rate = double(m.pinned[0]);
        m.last_substeps = std::max(1, int(std::ceil(double(dt) * m.last_rate / 0.7)));
        const float sub_dt = dt / float(m.last_substeps);
        for (int sub = 0; sub < m.last_substeps; ++sub)
        {
            if (bricks8)
                diffuse_brick_kernel<<<s.active_bricks, 256, 0, launch_stream(s)>>>(
                    s.active_brick_list, s.brick_level, s.brick_nbr, s.d_level_h, m.code, m.viscosity, m.x, m.y, m.z, sub_dt, m.xn,
                    m.yn, m.zn, m.dx, m.dy, m.dz);
            else if (s.active_bricks)
                diffuse_struct_kernel<0><<<cell_blocks(s), kThreads, 0, launch_stream(s)>>>(
                    s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr, s.d_level_h, m.code, m.viscosity, m.x, m.y,
                    m.z, sub_dt, m.xn, m.yn, m.zn, m.dx, m.dy, m.dz);
            finish_buffered(s, m, 1, sub_dt);
        }
        cuda_check(cudaGetLastError(), "smagorinsky diffusion");
        return m.last_rate;
    }

    void momentum_wall(System& s, Momentum& m, float dt, float nu)
    {
        if (!m.nW) return;
        if (m.nG)
            save_deferred_kernel<<<blocks_for(m.nD), kThreads, 0, launch_stream(s)>>>(m.nD, m.d_dof, m.d_group, m.x, m.y, m.z, m.baseline_x,
                                                                             m.baseline_y, m.baseline_z);
        wall_coefficient_kernel<<<blocks_for(m.nW), kThreads, 0, launch_stream(s)>>>(m.nW, m.w_dof, m.w_normal, m.w_area, m.w_distance, m.x,
                                                                           m.y, m.z, nu, m.w_k);
        wall_apply_kernel<<<blocks_for(m.nWall), kThreads, 0, launch_stream(s)>>>(m.nWall, m.wall_dof, m.wall_offset, m.wall_side, m.w_normal,
                                                                        m.w_k, m.volume32, dt, m.x, m.y, m.z);
        wall_force_kernel<<<blocks_for(m.nW), kThreads, 0, launch_stream(s)>>>(m.nW, m.w_dof, m.w_normal, m.w_k, m.x, m.y, m.z, m.w_force);
        if (m.nG)
            group_increment_kernel<<<blocks_for(m.nG), kThreads, 0, launch_stream(s)>>>(m.nG, m.g_offset, m.g_member, m.g_volume, m.d_dof,
                                                                              m.volume32, m.baseline_x, m.baseline_y, m.baseline_z, 1,
                                                                              m.x, m.y, m.z);
        cuda_check(cudaGetLastError(), "smooth wall");
    }

    void momentum_pressure_impulse(System& s, Momentum& m, float dt, float rho, bool physical)
    {
        const float scale = dt / rho;
        IrregularOperator& o = s.irr;
        if (o.gradient_nodes)
            pressure_gradient32_kernel<<<blocks_for(o.gradient_nodes), kThreads, 0, launch_stream(s)>>>(
                o.gradient_nodes, o.grad_dof, o.grad_offset, o.grad_neighbour, m.p_weight, s.pressure32, m.p_gradient);
        if (s.active_bricks && s.bs == 8)
            impulse_brick_kernel<<<s.active_bricks, 256, 0, launch_stream(s)>>>(
                s.active_brick_list, s.brick_level, s.brick_nbr, s.brick_flags, s.d_level_h, m.code, s.pressure32, scale,
                s.outlet ? 1 : 0, physical ? 1 : 0, m.x, m.y, m.z, m.xn, m.yn, m.zn, m.dx, m.dy, m.dz);
        else if (s.active_bricks)
            impulse_struct_kernel<0><<<cell_blocks(s), kThreads, 0, launch_stream(s)>>>(
                s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr, s.brick_flags, s.d_level_h, m.code, s.pressure32,
                scale, s.outlet ? 1 : 0, physical ? 1 : 0, m.x, m.y, m.z, m.xn, m.yn, m.zn, m.dx, m.dy, m.dz);
        const CompactArgs k = compact_args(s, m);
        if (m.nD)
            impulse_deferred_kernel<<<blocks_for(m.nD), kThreads, 0, launch_stream(s)>>>(
                m.nD, m.d_dof, m.d_offset, m.d_edge, m.d_sign, m.d_side_offset, m.d_side, m.d_boundary_offset, m.d_boundary,
                s.structured, k, s.pressure32, m.p_gradient, m.w_pnode, m.w_coefficient, m.w_disp, m.b_coefficient, scale,
                physical ? 1 : 0, m.x, m.y, m.z, m.dx, m.dy, m.dz, m.xn, m.yn, m.zn);
        swap_state(m);   // previous state (now xn) is the redistribution baseline
        if (m.nG)
            group_increment_kernel<<<blocks_for(m.nG), kThreads, 0, launch_stream(s)>>>(m.nG, m.g_offset, m.g_member, m.g_volume, m.d_dof,
                                                                              m.volume32, m.xn, m.yn, m.zn, 0, m.x, m.y, m.z);
        cuda_check(cudaGetLastError(), "pressure impulse");
    }

    void momentum_reconstruct_fluxes(System& s, Momentum& m)
    {
        special_gradients(s, m);
        if (s.active_bricks && s.bs == 8)
            reconstruct_brick_kernel<<<s.active_bricks, 256, 0, launch_stream(s)>>>(s.active_brick_list, s.brick_nbr, m.code, m.x, m.y,
                                                                                   m.z, s.u, s.v, s.w);
        else if (s.active_bricks)
            reconstruct_struct_kernel<0><<<cell_blocks(s), kThreads, 0, launch_stream(s)>>>(s.active_brick_list, s.active_bricks, s.bs, s.brick_level,
                                                                               s.brick_nbr, s.d_level_h, m.code, m.x, m.y, m.z, s.u, s.v, s.w);
        if (m.nK)
            reconstruct_compact_kernel<<<blocks_for(m.nK), kThreads, 0, launch_stream(s)>>>(m.nK, compact_args(s, m), m.x, m.y, m.z, s.u, s.v,
                                                                                  s.w, s.special);
        cuda_check(cudaGetLastError(), "flux reconstruction");
    }

    void momentum_external_boundaries(System& s, float speed)
    {
        if (!s.active_bricks) return;
        external_boundary_kernel<<<blocks_for(int64_t(s.active_bricks) * 6 * s.bs * s.bs), kThreads, 0, launch_stream(s)>>>(
            s.active_brick_list, s.active_bricks, s.bs, s.brick_flags, speed, s.inflow_slot_of_brick,
            s.inflow_set ? s.inflow.p : nullptr, s.u, s.v, s.w);
        cuda_check(cudaGetLastError(), "external boundaries");
    }

    void momentum_cfl(System& s, Momentum& m, bool external_aero, float out[4])
    {
        const CompactArgs k = compact_args(s, m);
        const bool bricks8 = s.active_bricks && s.bs == 8;
        const int cb = s.active_bricks ? (bricks8 ? s.active_bricks : cell_blocks(s)) : 0, db = m.nD ? blocks_for(m.nD) : 0;
        require(2 * (cb + db) <= int(m.reduce_partial.n), "reduction scratch too small");
        if (bricks8)
            cfl_brick_kernel<<<cb, 256, 0, launch_stream(s)>>>(s.active_brick_list, s.brick_level, s.brick_nbr, s.brick_flags,
                                                              s.d_level_h, m.code, s.u, s.v, s.w, m.x, m.y, m.z,
                                                              external_aero ? 1 : 0, m.dx, m.reduce_partial);
        else if (cb)
            cfl_struct_kernel<0><<<cb, 256, 0, launch_stream(s)>>>(s.active_brick_list, s.active_bricks, s.bs, s.brick_level, s.brick_nbr,
                                                       s.brick_flags, s.d_level_h, m.code, s.u, s.v, s.w, m.x, m.y, m.z,
                                                       external_aero ? 1 : 0, m.dx, m.reduce_partial);
        if (db)
            cfl_deferred_kernel<<<db, 256, 0, launch_stream(s)>>>(m.nD, m.d_dof, m.d_offset, m.d_edge, m.d_sign, s.structured, k, s.u, s.v, s.w,
                                                         s.special, m.x, m.y, m.z, m.dx, m.reduce_partial.p + 2 * cb);
        cuda_check(cudaMemsetAsync(m.reduce_result, 0, 4 * sizeof(float), s.stream), "cfl maxima");
        {
            const int work = std::max(cb + db, s.cf_count + s.eb_count);
            const int grid = std::max(1, std::min(592, blocks_for(work)));
            cfl_final_kernel<<<grid, 256, 0, launch_stream(s)>>>(m.reduce_partial, cb + db, s.special, s.cf_count + s.eb_count,
                                                                 reinterpret_cast<unsigned int*>(m.reduce_result.p));
        }
        cuda_check(cudaMemcpyAsync(m.pinned, m.reduce_result, 4 * sizeof(float), cudaMemcpyDeviceToHost, s.stream), "cfl readback");
        cuda_check(cudaStreamSynchronize(s.stream), "cfl readback");
        for (int q = 0; q < 4; ++q) out[q] = m.pinned[q];
    }
}
