// locator.h -- finest-brick point location on the device (shared by the locator and the MAC
// momentum kernels).  Location follows the reference's DeviceAmrLocator::locate_points
// (src/core/fluid/amr_fields.cu:131-168, 200-249) in the same FP32 arithmetic; each level keeps a
// dense brick-index grid over the bounding box of its brick coordinates.
#pragma once

#include "pcfd_internal.h"

namespace pcfd
{
    struct LocatorLevel
    {
        const int* grid;         // [nz][ny][nx] brick index within the level, or -1
        const float4* record;    // per brick: origin x, y, z and h (FP32, as the reference's records)
        const uint32_t* flags;   // per brick
        int nx, ny, nz, min_x, min_y, min_z, brick_count, slot0;
        float h;
    };
    struct LocatorView
    {
        const LocatorLevel* levels;
        int level_count, brick_size;
        float lo[3], hi[3];
    };

    __device__ inline void locate_one(const LocatorView& v, float px, float py, float pz, int* out)
    {
        out[0] = out[1] = -1;
        out[2] = out[3] = out[4] = 0;
        if (px < v.lo[0] || py < v.lo[1] || pz < v.lo[2] || px >= v.hi[0] || py >= v.hi[1] || pz >= v.hi[2]) return;
        for (int level = v.level_count - 1; level >= 0; --level)
        {
            const LocatorLevel lev = v.levels[level];
            const float width = float(v.brick_size) * lev.h;
            const int bx = int(floorf((px - v.lo[0]) / width)) - lev.min_x;
            const int by = int(floorf((py - v.lo[1]) / width)) - lev.min_y;
            const int bz = int(floorf((pz - v.lo[2]) / width)) - lev.min_z;
            if (bx < 0 || by < 0 || bz < 0 || bx >= lev.nx || by >= lev.ny || bz >= lev.nz) continue;
            const int brick = lev.grid[(int64_t(bz) * lev.ny + by) * lev.nx + bx];
            if (brick < 0 || brick >= lev.brick_count || (lev.flags[brick] & PCFD_BRICK_COVERED)) continue;
            const float4 r = lev.record[brick];
            const int last = v.brick_size - 1;
            out[0] = level;
            out[1] = brick;
            out[2] = max(0, min(last, int(floorf((px - r.x) / r.w))));
            out[3] = max(0, min(last, int(floorf((py - r.y) / r.w))));
            out[4] = max(0, min(last, int(floorf((pz - r.z) / r.w))));
            return;
        }
    }

    // the system's locator (built at system creation)
    const LocatorView& locator_view(const System& s);
}
