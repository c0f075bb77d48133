// pseudoinverse3.h -- pseudoinverse of a symmetric 3x3 matrix by cyclic Jacobi rotations, shared by
// the topology builder (WLS pressure-gradient stencils) and the momentum setup (least-squares
// velocity-gradient nodes).  The rotations visit the pairs (0,1), (0,2), (1,2) in turn until no
// off-diagonal entry exceeds 1e-14 of its diagonal pair or `sweeps` sweeps are done; eigenvalues
// above `cutoff` times the largest |eigenvalue| are inverted, the others dropped.  Returns the rank.
// The host reproduces the FP64 WLS weights of the reference builder bit for bit with it, which fixes
// the operation order (reference amr_pressure.cpp:63-189).
#pragma once

#include <algorithm>
#include <cmath>

namespace pcfd
{
    inline int pseudoinverse3(const double* input, double* inverse, int sweeps, double cutoff)
    {
        double a[9], v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        std::copy(input, input + 9, a);
        for (int sweep = 0; sweep < sweeps; ++sweep)
        {
            bool rotated = false;
            for (int pair = 0; pair < 3; ++pair)
            {
                const int p = pair == 2 ? 1 : 0, q = pair == 0 ? 1 : 2;
                const double apq = a[p * 3 + q], scale = std::max({std::abs(a[p * 3 + p]), std::abs(a[q * 3 + q]), 1e-300});
                if (std::abs(apq) <= 1e-14 * scale) continue;
                rotated = true;
                const double phi = 0.5 * std::atan2(2 * apq, a[q * 3 + q] - a[p * 3 + p]);
                const double c = std::cos(phi), s = std::sin(phi), app = a[p * 3 + p], aqq = a[q * 3 + q];
                for (int k = 0; k < 3; ++k)
                    if (k != p && k != q)
                    {
                        const double akp = a[k * 3 + p], akq = a[k * 3 + q];
                        a[k * 3 + p] = a[p * 3 + k] = c * akp - s * akq;
                        a[k * 3 + q] = a[q * 3 + k] = s * akp + c * akq;
                    }
                a[p * 3 + p] = c * c * app - 2 * s * c * apq + s * s * aqq;
                a[q * 3 + q] = s * s * app + 2 * s * c * apq + c * c * aqq;
                a[p * 3 + q] = a[q * 3 + p] = 0;
                for (int k = 0; k < 3; ++k)
                {
                    const double vkp = v[k * 3 + p], vkq = v[k * 3 + q];
                    v[k * 3 + p] = c * vkp - s * vkq;
                    v[k * 3 + q] = s * vkp + c * vkq;
                }
            }
            if (!rotated) break;
        }
        std::fill(inverse, inverse + 9, 0.0);
        const double maximum = std::max({std::abs(a[0]), std::abs(a[4]), std::abs(a[8])}), threshold = maximum * cutoff;
        int rank = 0;
        for (int mode = 0; mode < 3; ++mode)
        {
            const double lambda = a[mode * 3 + mode];
            if (!(lambda > threshold)) continue;
            ++rank;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) inverse[r * 3 + c] += v[r * 3 + mode] * v[c * 3 + mode] / lambda;
        }
        return rank;
    }
}
