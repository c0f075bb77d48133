// mac.cu -- the staggered MAC momentum mode: semi-Lagrangian MacCormack advection of the face
// velocities with a limited MUSCL update in the near-fabric band, Smagorinsky eddy viscosity and
// explicit face diffusion, on every AMR level at once.
//
// This is the reference's non-default momentum path (DeviceAmrAdvection::advect and
// diffuse_smagorinsky, src/core/fluid/amr_advection.cu:588-720 and 1663-1690), restated on the
// compact per-brick face layout (no ghost rings) in the reference's FP32 arithmetic:
//   forward   each face node is traced back with a two-stage (midpoint) characteristic and the
//             field is sampled trilinearly on the finest brick that owns the foot; faces in the
//             near-fabric band (link bit 6) take a limited MUSCL update along their open
//             same-side links instead (amr_advection.cu:633-647)
//   correct   MacCormack: the forward field is traced forward again and half the round-trip
//             error is added back, clamped to the backward foot's eight samples -- only when the
//             node and both feet lie on the face's own level (amr_advection.cu:653-666)
//   LES       nut = (cs h)^2 |S| from central differences of the sampled velocity (:705-708)
//   diffusion explicit 7-point face Laplacian with nu + mean nut of the two cells across the
//             face; band faces use only their open links and molecular nu (:709-713)
// Samples that leave a brick take the same-level neighbour across one face, else the finest brick
// that contains the lattice node (one-sided linear extension across 2:1 transitions).  One launch
// covers all brick slots of all levels; covered bricks are skipped (their output faces are 0, as
// the reference's scratch commit leaves them).  The link bytes are the caller's preprocessing
// (the fabric band and its open directions come from the caller's surface BVH).
#include "locator.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace pcfd
{
    namespace
    {
        struct MacView
        {
            LocatorView loc;
            const int* neighbour;       // [B][6] same-level neighbour slot or -1
            const uint32_t* flags;      // [B] brick flags by slot
            const int* slot_level;      // [B]
            int bs;
        };
        struct Faces
        {
            const float* c[3];
        };

        __device__ inline bool valid_face(int c, int bs, int i, int j, int k)
        {
            return i >= 0 && j >= 0 && k >= 0 && i < (c == 0 ? bs + 1 : bs) && j < (c == 1 ? bs + 1 : bs) && k < (c == 2 ? bs + 1 : bs);
        }
        __device__ inline float4 record_of(const MacView& m, int level, int64_t slot)
        {
            const LocatorLevel lev = m.loc.levels[level];
            return lev.record[slot - lev.slot0];
        }
        __device__ inline bool covered(const MacView& m, int64_t slot) { return (m.flags[slot] & PCFD_BRICK_COVERED) != 0; }

        // face value with indices clamped to the component's lattice of the brick
        __device__ inline float clamped(const Faces& f, int bs, int c, int64_t slot, int i, int j, int k)
        {
            i = max(0, min(c == 0 ? bs : bs - 1, i));
            j = max(0, min(c == 1 ? bs : bs - 1, j));
            k = max(0, min(c == 2 ? bs : bs - 1, k));
            return f.c[c][axis_face(bs, c, slot, i, j, k)];
        }
        // one-sided linear extension past the lattice ends (weights 2, -1 per axis)
        __device__ float extended(const Faces& f, int bs, int c, int64_t slot, int i, int j, int k)
        {
            const int n[3] = {c == 0 ? bs + 1 : bs, c == 1 ? bs + 1 : bs, c == 2 ? bs + 1 : bs}, want[3] = {i, j, k};
            int at[3][2], count[3];
            float w[3][2];
            for (int a = 0; a < 3; ++a)
            {
                if (want[a] < 0) { at[a][0] = 0; at[a][1] = 1; w[a][0] = 2.0f; w[a][1] = -1.0f; count[a] = 2; }
                else if (want[a] >= n[a]) { at[a][0] = n[a] - 1; at[a][1] = n[a] - 2; w[a][0] = 2.0f; w[a][1] = -1.0f; count[a] = 2; }
                else { at[a][0] = want[a]; w[a][0] = 1.0f; count[a] = 1; }
            }
            float result = 0;
            for (int az = 0; az < count[2]; ++az)
                for (int ay = 0; ay < count[1]; ++ay)
                    for (int ax = 0; ax < count[0]; ++ax)
                        result += w[0][ax] * w[1][ay] * w[2][az] * clamped(f, bs, c, slot, at[0][ax], at[1][ay], at[2][az]);
            return result;
        }
        // trilinear sample of component c at point p inside brick `slot`, with the extension
        __device__ float sample_extended(const Faces& f, int bs, const float4& rec, int c, int64_t slot, float px, float py, float pz)
        {
            float x = (px - rec.x) / rec.w - (c == 0 ? 0.0f : 0.5f);
            float y = (py - rec.y) / rec.w - (c == 1 ? 0.0f : 0.5f);
            float z = (pz - rec.z) / rec.w - (c == 2 ? 0.0f : 0.5f);
            const int i0 = int(floorf(x)), j0 = int(floorf(y)), k0 = int(floorf(z));
            x -= i0;
            y -= j0;
            z -= k0;
            float result = 0;
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx)
                    {
                        const float wx = dx ? x : 1.0f - x, wy = dy ? y : 1.0f - y, wz = dz ? z : 1.0f - z;
                        result += wx * wy * wz * extended(f, bs, c, slot, i0 + dx, j0 + dy, k0 + dz);
                    }
            return result;
        }
        __device__ inline void face_point(const float4& rec, int c, int i, int j, int k, float& x, float& y, float& z)
        {
            x = rec.x + (i + (c == 0 ? 0.0f : 0.5f)) * rec.w;
            y = rec.y + (j + (c == 1 ? 0.0f : 0.5f)) * rec.w;
            z = rec.z + (k + (c == 2 ? 0.0f : 0.5f)) * rec.w;
        }
        __device__ inline int nearest_index(float coordinate, float origin, float h, float offset)
        {
            return int(floorf((coordinate - origin) / h - offset + 0.5f));
        }
        // finest non-covered brick containing the point: level, slot (or -1)
        __device__ inline int locate(const MacView& m, float x, float y, float z, int& level)
        {
            int where[5];
            locate_one(m.loc, x, y, z, where);
            level = where[0];
            return where[0] < 0 ? -1 : m.loc.levels[where[0]].slot0 + where[1];
        }
        // the face on which a brick boundary lies: 0..5, or -1 when outside more than one face
        __device__ inline int outside_face(int nx, int ny, int nz, int i, int j, int k)
        {
            int face = -1, outside = 0;
            if (i < 0) { face = 0; ++outside; } else if (i >= nx) { face = 1; ++outside; }
            if (j < 0) { face = 2; ++outside; } else if (j >= ny) { face = 3; ++outside; }
            if (k < 0) { face = 4; ++outside; } else if (k >= nz) { face = 5; ++outside; }
            return outside == 1 ? face : -1;
        }
        __device__ inline void shift_into(int face, int bs, int& i, int& j, int& k)
        {
            if (face == 0) i += bs; else if (face == 1) i -= bs; else if (face == 2) j += bs;
            else if (face == 3) j -= bs; else if (face == 4) k += bs; else k -= bs;
        }

        // value of lattice node (i,j,k) of component c of brick `slot` (level `level`), which may
        // lie outside the brick
        __device__ __noinline__ float node_value(const MacView& m, const Faces& f, int level, int64_t slot, int c, int i, int j, int k)
        {
            const int bs = m.bs;
            if (valid_face(c, bs, i, j, k)) return clamped(f, bs, c, slot, i, j, k);
            const int face = outside_face(c == 0 ? bs + 1 : bs, c == 1 ? bs + 1 : bs, c == 2 ? bs + 1 : bs, i, j, k);
            if (face >= 0)
            {
                const int nb = m.neighbour[slot * 6 + face];
                if (nb >= 0 && !covered(m, nb))
                {
                    shift_into(face, bs, i, j, k);
                    return clamped(f, bs, c, nb, i, j, k);
                }
            }
            const float4 rec = record_of(m, level, slot);
            float nx, ny, nz;
            face_point(rec, c, i, j, k, nx, ny, nz);
            const float* lo = m.loc.lo;
            const float* hi = m.loc.hi;
            if (nx < lo[0] || ny < lo[1] || nz < lo[2] || nx > hi[0] || ny > hi[1] || nz > hi[2]) return clamped(f, bs, c, slot, i, j, k);
            const float eps = 1e-5f * rec.w;
            const float px = fminf(hi[0] - eps, fmaxf(lo[0] + eps, nx)), py = fminf(hi[1] - eps, fmaxf(lo[1] + eps, ny)),
                        pz = fminf(hi[2] - eps, fmaxf(lo[2] + eps, nz));
            int at_level;
            const int at = locate(m, px, py, pz, at_level);
            if (at < 0) return clamped(f, bs, c, slot, i, j, k);
            const float4 r = record_of(m, at_level, at);
            if (at_level != level) return sample_extended(f, bs, r, c, at, nx, ny, nz);
            return clamped(f, bs, c, at, nearest_index(nx, r.x, r.w, c == 0 ? 0.0f : 0.5f), nearest_index(ny, r.y, r.w, c == 1 ? 0.0f : 0.5f),
                           nearest_index(nz, r.z, r.w, c == 2 ? 0.0f : 0.5f));
        }
        // trilinear sample of component c at p from brick `slot`'s lattice, with the range of the
        // eight node values
        __device__ float sample_bounded(const MacView& m, const Faces& f, int level, int64_t slot, const float4& rec, int c, float px,
                                        float py, float pz, float* lower, float* upper)
        {
            const int bs = m.bs;
            float x = (px - rec.x) / rec.w - (c == 0 ? 0.0f : 0.5f);
            float y = (py - rec.y) / rec.w - (c == 1 ? 0.0f : 0.5f);
            float z = (pz - rec.z) / rec.w - (c == 2 ? 0.0f : 0.5f);
            const int i0 = int(floorf(x)), j0 = int(floorf(y)), k0 = int(floorf(z));
            x -= i0;
            y -= j0;
            z -= k0;
            float result = 0, mn = 0, mx = 0;
            bool first = true;
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx)
                    {
                        const int ni = i0 + dx, nj = j0 + dy, nk = k0 + dz;
                        const float wx = dx ? x : 1.0f - x, wy = dy ? y : 1.0f - y, wz = dz ? z : 1.0f - z;
                        const float value = valid_face(c, bs, ni, nj, nk) ? clamped(f, bs, c, slot, ni, nj, nk)
                                                                          : node_value(m, f, level, slot, c, ni, nj, nk);
                        result += wx * wy * wz * value;
                        if (first) { mn = mx = value; first = false; }
                        else { mn = fminf(mn, value); mx = fmaxf(mx, value); }
                    }
            if (lower) *lower = mn;
            if (upper) *upper = mx;
            return result;
        }
        __device__ inline float sample(const MacView& m, const Faces& f, int level, int64_t slot, const float4& rec, int c, float px,
                                       float py, float pz)
        {
            return sample_bounded(m, f, level, slot, rec, c, px, py, pz, nullptr, nullptr);
        }
        __device__ inline void clamp_point(const MacView& m, float& x, float& y, float& z)
        {
            x = fminf(m.loc.hi[0] - 1e-5f, fmaxf(m.loc.lo[0] + 1e-5f, x));
            y = fminf(m.loc.hi[1] - 1e-5f, fmaxf(m.loc.lo[1] + 1e-5f, y));
            z = fminf(m.loc.hi[2] - 1e-5f, fmaxf(m.loc.lo[2] + 1e-5f, z));
        }
        // sample on the finest brick owning p (clamped into the domain); `fallback` when none does
        __device__ float sample_finest(const MacView& m, const Faces& f, int c, float x, float y, float z, float fallback, float* lower,
                                       float* upper)
        {
            clamp_point(m, x, y, z);
            int level;
            const int at = locate(m, x, y, z, level);
            if (at < 0)
            {
                if (lower) *lower = fallback;
                if (upper) *upper = fallback;
                return fallback;
            }
            return sample_bounded(m, f, level, at, record_of(m, level, at), c, x, y, z, lower, upper);
        }
        // two-stage characteristic from p over dt (negative dt traces forward)
        __device__ void trace(const MacView& m, const Faces& f, int level, int64_t slot, const float4& rec, float& x, float& y, float& z,
                              float dt)
        {
            const float ux = sample(m, f, level, slot, rec, 0, x, y, z), uy = sample(m, f, level, slot, rec, 1, x, y, z),
                        uz = sample(m, f, level, slot, rec, 2, x, y, z);
            float mx = x - float(0.5f * dt * ux), my = y - float(0.5f * dt * uy), mz = z - float(0.5f * dt * uz);
            clamp_point(m, mx, my, mz);
            const float vx = sample_finest(m, f, 0, mx, my, mz, ux, nullptr, nullptr), vy = sample_finest(m, f, 1, mx, my, mz, uy, nullptr, nullptr),
                        vz = sample_finest(m, f, 2, mx, my, mz, uz, nullptr, nullptr);
            x = x - float(dt * vx);
            y = y - float(dt * vy);
            z = z - float(dt * vz);
            clamp_point(m, x, y, z);
        }
        __device__ inline void decode(int64_t q, int bs, int& c, int64_t& slot, int& i, int& j, int& k)
        {
            const int per = bs * bs * (bs + 1);
            int local = int(q % per);
            const int64_t r = q / per;
            c = int(r % 3);
            slot = r / 3;
            i = j = k = 0;
            if (c == 0) { i = local % (bs + 1); local /= bs + 1; j = local % bs; k = local / bs; }
            else if (c == 1) { i = local % bs; local /= bs; j = local % (bs + 1); k = local / (bs + 1); }
            else { i = local % bs; local /= bs; j = local % bs; k = local / bs; }
        }
        __device__ inline float minmod(float a, float b) { return a * b <= 0.0f ? 0.0f : (fabsf(a) < fabsf(b) ? a : b); }
        // one step along `axis` from face node (i,j,k) of brick `slot` inside the same level
        __device__ bool step_same_level(const MacView& m, int c, int axis, int direction, int64_t& slot, int& i, int& j, int& k)
        {
            const int bs = m.bs;
            if (axis == 0) i += direction; else if (axis == 1) j += direction; else k += direction;
            if (valid_face(c, bs, i, j, k)) return true;
            const int face = outside_face(c == 0 ? bs + 1 : bs, c == 1 ? bs + 1 : bs, c == 2 ? bs + 1 : bs, i, j, k);
            if (face < 0) return false;
            const int nb = m.neighbour[slot * 6 + face];
            if (nb < 0 || covered(m, nb)) return false;
            shift_into(face, bs, i, j, k);
            slot = nb;
            return valid_face(c, bs, i, j, k);
        }
        // limited MUSCL update of a near-fabric face along its open same-side links
        __device__ float band_update(const MacView& m, const Faces& f, const uint8_t* const* links, int level, int64_t slot,
                                     const float4& rec, int c, int i, int j, int k, float current, uint8_t link, float dt)
        {
            const int bs = m.bs;
            float px, py, pz;
            face_point(rec, c, i, j, k, px, py, pz);
            const float velocity[3] = {sample(m, f, level, slot, rec, 0, px, py, pz), sample(m, f, level, slot, rec, 1, px, py, pz),
                                       sample(m, f, level, slot, rec, 2, px, py, pz)};
            float weighted = 0, weights = 0, lower = current, upper = current;
            for (int axis = 0; axis < 3; ++axis)
            {
                const int up_dir = velocity[axis] >= 0.0f ? -1 : 1, up_bit = 2 * axis + (up_dir > 0), down_bit = 2 * axis + (up_dir < 0);
                if (!(link & (1u << up_bit))) continue;
                int64_t us = slot;
                int ui = i, uj = j, uk = k;
                if (!step_same_level(m, c, axis, up_dir, us, ui, uj, uk)) continue;
                const float upstream = clamped(f, bs, c, us, ui, uj, uk);
                lower = fminf(lower, upstream);
                upper = fmaxf(upper, upstream);
                const float weight = dt * fabsf(velocity[axis]) / rec.w;
                float delta = weight * (upstream - current);
                // the limited linear reconstruction needs all three further segments on same-side
                // links; otherwise the first-order donor update stays
                const uint8_t up_links = links[c][axis_face(bs, c, us, ui, uj, uk)];
                int64_t u2s = us, ds = slot;
                int u2i = ui, u2j = uj, u2k = uk, di = i, dj = j, dk = k;
                const bool second = (link & (1u << down_bit)) && (up_links & (1u << up_bit)) &&
                                    step_same_level(m, c, axis, up_dir, u2s, u2i, u2j, u2k) &&
                                    step_same_level(m, c, axis, -up_dir, ds, di, dj, dk);
                if (second)
                {
                    const float upstream2 = clamped(f, bs, c, u2s, u2i, u2j, u2k), downstream = clamped(f, bs, c, ds, di, dj, dk);
                    lower = fminf(lower, downstream);
                    upper = fmaxf(upper, downstream);
                    const float up_slope = minmod(upstream - upstream2, current - upstream),
                                slope = minmod(current - upstream, downstream - current);
                    const float incoming = upstream + 0.5f * up_slope, outgoing = current + 0.5f * slope;
                    delta = -weight * (outgoing - incoming);
                }
                weighted += delta;
                weights += weight;
            }
            const float scale = weights > 1.0f ? 1.0f / weights : 1.0f;
            return fmaxf(lower, fminf(upper, current + scale * weighted));
        }

        struct Links
        {
            const uint8_t* c[3];
        };
        struct Out
        {
            float* c[3];
        };

        __global__ void mac_forward_kernel(MacView m, Faces f, Links links, int64_t total, float dt, Out out)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= total) return;
            int c, i, j, k;
            int64_t slot;
            decode(q, m.bs, c, slot, i, j, k);
            if (covered(m, slot)) return;
            const int level = m.slot_level[slot];
            const float4 rec = record_of(m, level, slot);
            const int64_t at = axis_face(m.bs, c, slot, i, j, k);
            const float current = f.c[c][at];
            const uint8_t link = links.c[c][at];
            float result;
            if (link & 0x40) result = band_update(m, f, links.c, level, slot, rec, c, i, j, k, current, link, dt);
            else
            {
                float x, y, z;
                face_point(rec, c, i, j, k, x, y, z);
                trace(m, f, level, slot, rec, x, y, z, dt);
                result = sample_finest(m, f, c, x, y, z, current, nullptr, nullptr);
            }
            out.c[c][at] = result;
        }

        __global__ void mac_correct_kernel(MacView m, Faces f, Faces forward, Links links, int64_t total, float dt, Out out)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= total) return;
            int c, i, j, k;
            int64_t slot;
            decode(q, m.bs, c, slot, i, j, k);
            if (covered(m, slot)) return;
            const int level = m.slot_level[slot];
            const float4 rec = record_of(m, level, slot);
            const int64_t at = axis_face(m.bs, c, slot, i, j, k);
            const float current = f.c[c][at], phf = forward.c[c][at];
            float result = phf;
            if (!(links.c[c][at] & 0x40))
            {
                float px, py, pz;
                face_point(rec, c, i, j, k, px, py, pz);
                float bx = px, by = py, bz = pz;
                trace(m, f, level, slot, rec, bx, by, bz, dt);
                float mn, mx;
                sample_finest(m, f, c, bx, by, bz, current, &mn, &mx);
                float fx = px, fy = py, fz = pz;
                trace(m, f, level, slot, rec, fx, fy, fz, -dt);
                // the reverse correction only when the node and both feet are on this level: across a
                // 2:1 transition the forward field mixes independently evolved lattices
                float ox = px, oy = py, oz = pz;
                clamp_point(m, ox, oy, oz);
                int owner_level, back_level, forward_level;
                locate(m, ox, oy, oz, owner_level);
                locate(m, bx, by, bz, back_level);
                locate(m, fx, fy, fz, forward_level);
                if (owner_level == level && back_level == level && forward_level == level)
                {
                    const float phn = sample_finest(m, forward, c, fx, fy, fz, phf, nullptr, nullptr);
                    result = fmaxf(mn, fminf(mx, phf + 0.5f * (current - phn)));
                }
            }
            out.c[c][at] = result;
        }

        // ---- LES and diffusion ----
        __device__ inline float cell_clamped(const float* nut, int bs, int64_t slot, int i, int j, int k)
        {
            i = max(0, min(bs - 1, i));
            j = max(0, min(bs - 1, j));
            k = max(0, min(bs - 1, k));
            return nut[slot * bs * bs * bs + (int64_t(k) * bs + j) * bs + i];
        }
        __device__ float cell_extended(const float* nut, int bs, int64_t slot, int i, int j, int k)
        {
            const int want[3] = {i, j, k};
            int at[3][2], count[3];
            float w[3][2];
            for (int a = 0; a < 3; ++a)
            {
                if (want[a] < 0) { at[a][0] = 0; at[a][1] = 1; w[a][0] = 2.0f; w[a][1] = -1.0f; count[a] = 2; }
                else if (want[a] >= bs) { at[a][0] = bs - 1; at[a][1] = bs - 2; w[a][0] = 2.0f; w[a][1] = -1.0f; count[a] = 2; }
                else { at[a][0] = want[a]; w[a][0] = 1.0f; count[a] = 1; }
            }
            float result = 0;
            for (int az = 0; az < count[2]; ++az)
                for (int ay = 0; ay < count[1]; ++ay)
                    for (int ax = 0; ax < count[0]; ++ax)
                        result += w[0][ax] * w[1][ay] * w[2][az] * cell_clamped(nut, bs, slot, at[0][ax], at[1][ay], at[2][az]);
            return result;
        }
        __device__ float cell_sample_extended(const float* nut, int bs, const float4& rec, int64_t slot, float px, float py, float pz)
        {
            float x = (px - rec.x) / rec.w - 0.5f, y = (py - rec.y) / rec.w - 0.5f, z = (pz - rec.z) / rec.w - 0.5f;
            const int i0 = int(floorf(x)), j0 = int(floorf(y)), k0 = int(floorf(z));
            x -= i0;
            y -= j0;
            z -= k0;
            float result = 0;
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx)
                    {
                        const float wx = dx ? x : 1.0f - x, wy = dy ? y : 1.0f - y, wz = dz ? z : 1.0f - z;
                        result += wx * wy * wz * cell_extended(nut, bs, slot, i0 + dx, j0 + dy, k0 + dz);
                    }
            return result;
        }
        // cell value (i,j,k) of brick `slot`, which may lie outside the brick
        __device__ __noinline__ float cell_node_value(const MacView& m, const float* nut, int level, int64_t slot, int i, int j, int k)
        {
            const int bs = m.bs;
            if (i >= 0 && j >= 0 && k >= 0 && i < bs && j < bs && k < bs) return cell_clamped(nut, bs, slot, i, j, k);
            const int face = outside_face(bs, bs, bs, i, j, k);
            if (face >= 0)
            {
                const int nb = m.neighbour[slot * 6 + face];
                if (nb >= 0 && !covered(m, nb))
                {
                    shift_into(face, bs, i, j, k);
                    return cell_clamped(nut, bs, nb, i, j, k);
                }
            }
            const float4 rec = record_of(m, level, slot);
            const float nx = rec.x + (i + 0.5f) * rec.w, ny = rec.y + (j + 0.5f) * rec.w, nz = rec.z + (k + 0.5f) * rec.w;
            const float* lo = m.loc.lo;
            const float* hi = m.loc.hi;
            if (nx < lo[0] || ny < lo[1] || nz < lo[2] || nx >= hi[0] || ny >= hi[1] || nz >= hi[2]) return cell_clamped(nut, bs, slot, i, j, k);
            int at_level;
            const int at = locate(m, nx, ny, nz, at_level);
            if (at < 0) return cell_clamped(nut, bs, slot, i, j, k);
            const float4 r = record_of(m, at_level, at);
            if (at_level != level) return cell_sample_extended(nut, bs, r, at, nx, ny, nz);
            return cell_clamped(nut, bs, at, nearest_index(nx, r.x, r.w, 0.5f), nearest_index(ny, r.y, r.w, 0.5f),
                                nearest_index(nz, r.z, r.w, 0.5f));
        }

        __global__ void mac_smagorinsky_kernel(MacView m, Faces f, int64_t cells, float cs, float* nut)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= cells) return;
            const int bs = m.bs, c3 = bs * bs * bs;
            const int64_t slot = q / c3;
            const int local = int(q % c3);
            if (covered(m, slot)) return;
            const int i = local % bs, j = (local / bs) % bs, k = local / (bs * bs);
            const int level = m.slot_level[slot];
            const float4 rec = record_of(m, level, slot);
            const float h = rec.w;
            const float cx = rec.x + (i + 0.5f) * h, cy = rec.y + (j + 0.5f) * h, cz = rec.z + (k + 0.5f) * h;
            float g[3][3];
            for (int c = 0; c < 3; ++c)
                for (int axis = 0; axis < 3; ++axis)
                {
                    float lx = cx, ly = cy, lz = cz, ux = cx, uy = cy, uz = cz;
                    if (axis == 0) { lx -= h; ux += h; } else if (axis == 1) { ly -= h; uy += h; } else { lz -= h; uz += h; }
                    g[c][axis] = (sample(m, f, level, slot, rec, c, ux, uy, uz) - sample(m, f, level, slot, rec, c, lx, ly, lz)) / (2.0f * h);
                }
            const float sxx = g[0][0], syy = g[1][1], szz = g[2][2], sxy = 0.5f * (g[0][1] + g[1][0]), sxz = 0.5f * (g[0][2] + g[2][0]),
                        syz = 0.5f * (g[1][2] + g[2][1]);
            const float magnitude = sqrtf(2.0f * (sxx * sxx + syy * syy + szz * szz + 2.0f * (sxy * sxy + sxz * sxz + syz * syz)));
            const float length = cs * h;
            nut[q] = length * length * magnitude;
        }

        __global__ void mac_diffuse_kernel(MacView m, Faces f, Links links, const float* nut, int64_t total, float nu, float dt, Out out)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= total) return;
            int c, i, j, k;
            int64_t slot;
            decode(q, m.bs, c, slot, i, j, k);
            if (covered(m, slot)) return;
            const int bs = m.bs;
            const int level = m.slot_level[slot];
            const int64_t at = axis_face(bs, c, slot, i, j, k);
            const float current = f.c[c][at];
            const uint8_t link = links.c[c][at];
            auto face_value = [&](int a, int b, int d) {
                return valid_face(c, bs, a, b, d) ? clamped(f, bs, c, slot, a, b, d) : node_value(m, f, level, slot, c, a, b, d);
            };
            float laplacian = 0, viscosity = nu;
            if (!(link & 0x40))
            {
                laplacian = face_value(i - 1, j, k) + face_value(i + 1, j, k) + face_value(i, j - 1, k) + face_value(i, j + 1, k) +
                            face_value(i, j, k - 1) + face_value(i, j, k + 1) - 6.0f * current;
                int ci = i, cj = j, ck = k;
                if (c == 0) --ci; else if (c == 1) --cj; else --ck;
                const int ci2 = ci + (c == 0), cj2 = cj + (c == 1), ck2 = ck + (c == 2);
                auto cell_value = [&](int a, int b, int d) {
                    return a >= 0 && b >= 0 && d >= 0 && a < bs && b < bs && d < bs ? cell_clamped(nut, bs, slot, a, b, d)
                                                                                    : cell_node_value(m, nut, level, slot, a, b, d);
                };
                viscosity += 0.5f * (cell_value(ci, cj, ck) + cell_value(ci2, cj2, ck2));
            }
            else
                for (int axis = 0; axis < 3; ++axis)
                    for (int direction = -1; direction <= 1; direction += 2)
                    {
                        const int bit = 2 * axis + (direction > 0);
                        if (!(link & (1u << bit))) continue;
                        int p[3] = {i, j, k};
                        p[axis] += direction;
                        laplacian += face_value(p[0], p[1], p[2]) - current;
                    }
            const float h = m.loc.levels[level].h;
            out.c[c][at] = current + dt * viscosity * laplacian / (h * h);
        }
    }

    namespace
    {
        // max |face velocity| over the faces of non-covered bricks (DeviceAmrFields::
        // max_abs_velocity, amr_fields.cu:65-68, 195-198), as float bits in an unsigned int
        __global__ void mac_max_face_kernel(Faces f, const uint32_t* flags, int64_t per_slot, int64_t per_component, unsigned int* out)
        {
            __shared__ float shared[8];
            float m = 0.0f;
            for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < 3 * per_component; q += int64_t(gridDim.x) * blockDim.x)
            {
                const int c = int(q / per_component);
                const int64_t i = q % per_component;
                if (!(flags[i / per_slot] & PCFD_BRICK_COVERED)) m = fmaxf(m, fabsf(f.c[c][i]));
            }
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

    inline float uint_bits_to_float(unsigned int bits)
    {
        float f;
        std::memcpy(&f, &bits, sizeof(f));
        return f;
    }

    // ---- system state and launches ----
    struct MacState
    {
        DBuf<int> neighbour;
        DBuf<uint32_t> flags;
        DBuf<uint8_t> links[3];
        DBuf<float> forward[3], out[3], nut;
        DBuf<unsigned int> maximum;
        bool has_links = false;
    };

    namespace
    {
        MacState& mac_state(System& s)
        {
            require(s.mac != nullptr, "MAC momentum not set up");
            return *static_cast<MacState*>(s.mac);
        }
        MacView mac_view(System& s)
        {
            MacState& st = mac_state(s);
            return MacView{locator_view(s), st.neighbour.p, st.flags.p, s.brick_level, s.bs};
        }
    }

    void build_mac(System& s, const pcfd_topology& t)
    {
        auto* st = new MacState();
        s.mac = st;
        std::vector<int> neighbour(size_t(s.B) * 6, -1);
        std::vector<uint32_t> flags(size_t(s.B), 0);
        for (int l = 0, slot0 = 0; l < t.level_count; ++l)
        {
            const pcfd_level& lev = t.levels[l];
            for (int b = 0; b < lev.brick_count; ++b)
            {
                flags[size_t(slot0 + b)] = lev.flags[b];
                for (int face = 0; face < 6; ++face)
                {
                    const int n = lev.neighbors[b * 6 + face];
                    neighbour[size_t(slot0 + b) * 6 + face] = n >= 0 ? slot0 + n : -1;
                }
            }
            slot0 += lev.brick_count;
        }
        st->neighbour.upload(neighbour);
        st->flags.upload(flags);
        st->maximum.alloc(1);
    }

    void destroy_mac(System& s)
    {
        delete static_cast<MacState*>(s.mac);
        s.mac = nullptr;
    }

    void mac_set_links(System& s, const uint8_t* const host[3])
    {
        MacState& st = mac_state(s);
        for (int c = 0; c < 3; ++c)
        {
            st.links[c].upload(std::vector<uint8_t>(host[c], host[c] + s.faces));
            if (!st.forward[c].n) st.forward[c].alloc(size_t(s.faces));
            if (!st.out[c].n) st.out[c].alloc(size_t(s.faces));
        }
        if (!st.nut.n) st.nut.alloc(size_t(s.S));
        st.has_links = true;
    }

    void mac_advect(System& s, float dt)
    {
        MacState& st = mac_state(s);
        require(st.has_links, "MAC advection: links not set");
        const MacView m = mac_view(s);
        const Faces f{{s.u.p, s.v.p, s.w.p}};
        const Links links{{st.links[0].p, st.links[1].p, st.links[2].p}};
        const int64_t total = int64_t(s.B) * 3 * s.bs * s.bs * (s.bs + 1);
        const Out forward{{st.forward[0].p, st.forward[1].p, st.forward[2].p}};
        mac_forward_kernel<<<blocks_for(total), kThreads, 0, launch_stream(s)>>>(m, f, links, total, dt, forward);
        const Faces fw{{st.forward[0].p, st.forward[1].p, st.forward[2].p}};
        const Out out{{st.out[0].p, st.out[1].p, st.out[2].p}};
        mac_correct_kernel<<<blocks_for(total), kThreads, 0, launch_stream(s)>>>(m, f, fw, links, total, dt, out);
        float* target[3] = {s.u.p, s.v.p, s.w.p};
        for (int c = 0; c < 3; ++c)
            cuda_check(cudaMemcpyAsync(target[c], st.out[c].p, size_t(s.faces) * sizeof(float), cudaMemcpyDeviceToDevice, s.stream),
                       "commit MAC advection");
        cuda_check(cudaGetLastError(), "MAC advection");
    }

    void mac_diffuse_smagorinsky(System& s, float nu, float cs, float dt)
    {
        MacState& st = mac_state(s);
        require(st.has_links, "MAC diffusion: links not set");
        const MacView m = mac_view(s);
        const Faces f{{s.u.p, s.v.p, s.w.p}};
        const Links links{{st.links[0].p, st.links[1].p, st.links[2].p}};
        const int64_t cells = int64_t(s.B) * s.bs * s.bs * s.bs;
        mac_smagorinsky_kernel<<<blocks_for(cells), kThreads, 0, launch_stream(s)>>>(m, f, cells, cs, st.nut.p);
        const int64_t total = int64_t(s.B) * 3 * s.bs * s.bs * (s.bs + 1);
        const Out out{{st.out[0].p, st.out[1].p, st.out[2].p}};
        mac_diffuse_kernel<<<blocks_for(total), kThreads, 0, launch_stream(s)>>>(m, f, links, st.nut.p, total, nu, dt, out);
        float* target[3] = {s.u.p, s.v.p, s.w.p};
        for (int c = 0; c < 3; ++c)
            cuda_check(cudaMemcpyAsync(target[c], st.out[c].p, size_t(s.faces) * sizeof(float), cudaMemcpyDeviceToDevice, s.stream),
                       "commit MAC diffusion");
        cuda_check(cudaGetLastError(), "MAC diffusion");
    }

    void mac_eddy_viscosity(System& s, float* host_nut)
    {
        MacState& st = mac_state(s);
        require(st.nut.n == size_t(s.S), "MAC eddy viscosity: no diffusion step yet");
        cuda_check(cudaStreamSynchronize(s.stream), "synchronize");
        cuda_check(cudaMemcpy(host_nut, st.nut.p, size_t(s.S) * sizeof(float), cudaMemcpyDeviceToHost), "download eddy viscosity");
    }

    bool mac_ready(const System& s) { return s.mac && static_cast<const MacState*>(s.mac)->has_links; }

    float mac_max_face_speed(System& s)
    {
        MacState& st = mac_state(s);
        const Faces f{{s.u.p, s.v.p, s.w.p}};
        const int64_t per_slot = int64_t(s.bs + 1) * s.bs * s.bs, per_component = int64_t(s.B) * per_slot;
        cuda_check(cudaMemsetAsync(st.maximum.p, 0, sizeof(unsigned int), s.stream), "clear maximum");
        mac_max_face_kernel<<<int(std::min<int64_t>(592, (3 * per_component + kThreads - 1) / kThreads)), kThreads, 0, launch_stream(s)>>>(
            f, st.flags, per_slot, per_component, st.maximum);
        unsigned int bits = 0;
        cuda_check(cudaMemcpyAsync(&bits, st.maximum.p, sizeof(bits), cudaMemcpyDeviceToHost, s.stream), "read maximum");
        cuda_check(cudaStreamSynchronize(s.stream), "face maximum");
        return uint_bits_to_float(bits);
    }
}
