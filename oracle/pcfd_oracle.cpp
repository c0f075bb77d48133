// pcfd_oracle.cpp -- CPU restatement of the composite pressure operator, MG preconditioner,
// PCG/GCRO solvers and projection divergence/correction (see pcfd_oracle.h).
// TEST INFRASTRUCTURE ONLY (checker + CPU baseline).  OpenMP over bricks/rows/vectors.
#include "pcfd_oracle.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

namespace
{
    constexpr uint32_t COVERED = 128, XMIN = 1, XMAX = 2;

    struct Edge { int a, b; double c; };
    struct MgLevel
    {
        int cells = 0;
        std::vector<std::array<int, 3>> coord;
        std::vector<double> diag;
        std::vector<Edge> edges;
        std::vector<int> aggregate, roff, rdof, row, nbr;
        std::vector<double> coef, rhs, x, tmp, res;
    };
}

struct po_system
{
    pcfd_topology t;
    int bs = 0, c3 = 0, S = 0, B = 0, structured = 0;
    std::vector<int> slot0, active_slots, slot_level;
    std::vector<int> nbr;                 // [B][6] active neighbour slot or -1
    std::vector<uint32_t> flags;
    std::vector<double> h;
    // compact edges: connections (cf then eb) + regular corrections
    int nc = 0, nr = 0;
    std::vector<int> lo, up, lnode, unode;
    std::vector<double> coef, corr, uw, area;
    std::vector<int> inc_dof, inc_off, inc_edge;
    std::vector<int8_t> inc_sign;
    std::vector<double> gradient;         // [nodes][3]
    std::vector<double> diagonal;
    int base_offset = 0, base_cells = 0;
    std::vector<int> base_roff, base_rdof;
    std::vector<MgLevel> mg;
    std::vector<double> r, z, d, Ad, tv, corrv, defect;
    std::vector<double> V, Z, RU, RC;     // GCRO bases
    int recycle = 0;
    // composite cycle (po_set_composite): stages, fine -> stage-1 map, coarsest inverse
    bool composite = false;
    int stage_steps = 6, stage_ratio = 30, fine_ratio = 10;
    std::vector<MgLevel> stages;
    std::vector<int> fine_map, fine_roff, fine_rdof;
    std::vector<double> coarse_inverse, fine_res, stage_d;
};

namespace
{
    double factor_of(const pcfd_connections& c, int e)
    {
        const double f = c.orthogonal_gradient_factor[e];
        return f > 0 ? f : (c.normal_distance[e] > 0 ? 1.0 / c.normal_distance[e] : 0.0);
    }

    // ---- operator (apply_cpu semantics, gather form) ----------------------------------------
    void structured_apply(po_system& s, const double* p, double* out)
    {
        const pcfd_topology& t = s.t;
        const int bs = s.bs, c3 = s.c3;
#pragma omp parallel for schedule(static)
        for (int n = 0; n < int(s.active_slots.size()); ++n)
        {
            const int slot = s.active_slots[n];
            const double h = s.h[s.slot_level[slot]];
            for (int local = 0; local < c3; ++local)
            {
                const int a = slot * c3 + local;
                if (!t.active[a]) { out[a] = 0; continue; }
                const int ijk[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
                double v = 0;
                for (int axis = 0; axis < 3; ++axis)
                    for (int sign = -1; sign <= 1; sign += 2)
                    {
                        int c[3] = {ijk[0], ijk[1], ijk[2]}, sl = slot;
                        c[axis] += sign;
                        if (c[axis] < 0 || c[axis] >= bs)
                        {
                            sl = s.nbr[slot * 6 + 2 * axis + (sign > 0)];
                            if (sl < 0) continue;
                            c[axis] = sign > 0 ? 0 : bs - 1;
                        }
                        const int b = sl * c3 + (c[2] * bs + c[1]) * bs + c[0];
                        const int lower = sign > 0 ? a : b;
                        if (t.active[b] && !(t.cut_face_mask[lower] & (1u << axis))) v += h * (p[a] - p[b]);
                    }
                if (t.pressure_outlet_xmax && (s.flags[slot] & XMAX) && ijk[0] == bs - 1) v += 2.0 * h * p[a];
                out[a] = v;
            }
        }
#pragma omp parallel for schedule(static)
        for (int q = s.structured; q < s.S; ++q) out[q] = 0;
    }

    void apply(po_system& s, const double* p, double* out, bool orthogonal)
    {
        const pcfd_topology& t = s.t;
        structured_apply(s, p, out);
        const int nodes = t.gradient_node_count;
        if (!orthogonal && nodes)
        {
#pragma omp parallel for schedule(static)
            for (int n = 0; n < nodes; ++n)
            {
                const double centre = p[t.gradient_dof[n]];
                double g[3] = {0, 0, 0};
                for (int q = t.gradient_offset[n]; q < t.gradient_offset[n + 1]; ++q)
                    for (int c = 0; c < 3; ++c) g[c] += t.gradient_weight[3 * q + c] * (p[t.gradient_neighbour[q]] - centre);
                for (int c = 0; c < 3; ++c) s.gradient[3 * n + c] = g[c];
            }
        }
#pragma omp parallel for schedule(static)
        for (int node = 0; node < int(s.inc_dof.size()); ++node)
        {
            double sum = 0;
            for (int q = s.inc_off[node]; q < s.inc_off[node + 1]; ++q)
            {
                const int e = s.inc_edge[q], a = s.lo[e], b = s.up[e];
                if (!t.active[a] || !t.active[b]) continue;
                double flux = s.coef[e] * (p[a] - p[b]);
                if (!orthogonal && nodes && s.lnode[e] >= 0 && s.unode[e] >= 0)
                {
                    double der = 0;
                    const double w = s.uw[e];
                    for (int c = 0; c < 3; ++c)
                        der += s.corr[3 * e + c] * ((1 - w) * s.gradient[3 * s.lnode[e] + c] + w * s.gradient[3 * s.unode[e] + c]);
                    flux += -s.area[e] * der;
                }
                sum += double(s.inc_sign[q]) * flux;
            }
            out[s.inc_dof[node]] += sum;
        }
        for (int g = 0; g < t.gauge_count; ++g)
            if (t.active[t.gauge_dof[g]]) out[t.gauge_dof[g]] += t.gauge_coefficient[g] * p[t.gauge_dof[g]];
    }

    double dot(const po_system& s, const double* a, const double* b)
    {
        double v = 0;
#pragma omp parallel for reduction(+ : v) schedule(static)
        for (int q = 0; q < s.S; ++q) if (s.t.active[q]) v += a[q] * b[q];
        return v;
    }

    // ---- multigrid (reference setup amr_pressure.cu:857-1069) ---------------------------------
    void finalize(MgLevel& L)
    {
        L.row.assign(size_t(L.cells) + 1, 0);
        for (const Edge& e : L.edges) { ++L.row[e.a + 1]; ++L.row[e.b + 1]; }
        for (int q = 0; q < L.cells; ++q) L.row[q + 1] += L.row[q];
        L.nbr.resize(L.row.back());
        L.coef.resize(L.row.back());
        std::vector<int> cur = L.row;
        for (const Edge& e : L.edges)
        {
            int k = cur[e.a]++;
            L.nbr[k] = e.b; L.coef[k] = e.c;
            k = cur[e.b]++;
            L.nbr[k] = e.a; L.coef[k] = e.c;
        }
        L.rhs.assign(L.cells, 0); L.x.assign(L.cells, 0); L.tmp.assign(L.cells, 0); L.res.assign(L.cells, 0);
    }

    void build_mg(po_system& s)
    {
        const pcfd_topology& t = s.t;
        const int bs = s.bs, c3 = s.c3;
        const pcfd_level& base = t.levels[0];
        s.base_offset = base.level_offset;
        s.base_cells = base.brick_count * c3;
        const int BC = s.base_cells, BO = s.base_offset;
        const int32_t* agg = t.preconditioner_aggregate;
        s.base_roff.assign(size_t(BC) + 1, 0);
        for (int q = 0; q < s.S; ++q) if (t.active[q]) { const int c = agg[q] - BO; if (c >= 0 && c < BC) ++s.base_roff[c + 1]; }
        for (int c = 0; c < BC; ++c) s.base_roff[c + 1] += s.base_roff[c];
        s.base_rdof.resize(s.base_roff.back());
        {
            std::vector<int> cur = s.base_roff;
            for (int q = 0; q < s.S; ++q) if (t.active[q]) { const int c = agg[q] - BO; if (c >= 0 && c < BC) s.base_rdof[cur[c]++] = q; }
        }
        auto gc = [&](int c) {
            const int brick = c / c3, local = c % c3;
            return std::array<int, 3>{base.coord[3 * brick] * bs + local % bs, base.coord[3 * brick + 1] * bs + (local / bs) % bs,
                                      base.coord[3 * brick + 2] * bs + local / (bs * bs)};
        };
        std::vector<double> positive(size_t(BC) * 3, 0.0), cdiag(BC, 0.0);
        std::vector<Edge> extra;
        auto add = [&](int a, int b, double c) {
            if (a < 0 || b < 0 || a == b || !t.active[a] || !t.active[b] || !(c > 0)) return;
            const int ca = agg[a] - BO, cb = agg[b] - BO;
            if (ca < 0 || cb < 0 || ca >= BC || cb >= BC || ca == cb) return;
            const auto ga = gc(ca), gb = gc(cb);
            int axis = -1, man = 0;
            for (int d = 0; d < 3; ++d) { const int dd = gb[d] - ga[d]; man += std::abs(dd); if (dd) axis = d; }
            if (man == 1 && axis >= 0) positive[size_t(ga[axis] < gb[axis] ? ca : cb) * 3 + axis] += c;
            else extra.push_back({ca, cb, c});
            cdiag[ca] += c;
            cdiag[cb] += c;
        };
        for (int l = 0; l < t.level_count; ++l)
        {
            const pcfd_level& lev = t.levels[l];
            for (int brick = 0; brick < lev.brick_count; ++brick)
            {
                if (lev.flags[brick] & COVERED) continue;
                for (int k = 0; k < bs; ++k)
                    for (int j = 0; j < bs; ++j)
                        for (int i = 0; i < bs; ++i)
                        {
                            const int a = lev.level_offset + brick * c3 + (k * bs + j) * bs + i;
                            if (!t.active[a]) continue;
                            for (int axis = 0; axis < 3; ++axis)
                            {
                                if (t.cut_face_mask[a] & (1u << axis)) continue;
                                int c[3] = {i, j, k}, b = -1;
                                if (++c[axis] < bs) b = lev.level_offset + brick * c3 + (c[2] * bs + c[1]) * bs + c[0];
                                else
                                {
                                    const int nb = lev.neighbors[brick * 6 + 2 * axis + 1];
                                    if (nb >= 0 && !(lev.flags[nb] & COVERED)) { c[axis] = 0; b = lev.level_offset + nb * c3 + (c[2] * bs + c[1]) * bs + c[0]; }
                                }
                                add(a, b, lev.h);
                            }
                            if (t.pressure_outlet_xmax && (lev.flags[brick] & XMAX) && i == bs - 1)
                            {
                                const int cc = agg[a] - BO;
                                if (cc >= 0 && cc < BC) cdiag[cc] += 2.0 * lev.h;
                            }
                        }
            }
        }
        for (int e = 0; e < t.coarse_fine.count; ++e) add(t.coarse_fine.coarse_dof[e], t.coarse_fine.fine_dof[e], t.coarse_fine.open_area[e] * factor_of(t.coarse_fine, e));
        for (int e = 0; e < t.embedded.count; ++e) add(t.embedded.coarse_dof[e], t.embedded.fine_dof[e], t.embedded.open_area[e] * factor_of(t.embedded, e));
        for (int e = 0; e < t.regular.count; ++e) add(t.regular.lower_dof[e], t.regular.upper_dof[e], t.regular.open_area[e] * t.regular.two_point_delta[e]);
        for (int g = 0; g < t.gauge_count; ++g) { const int cc = agg[t.gauge_dof[g]] - BO; if (cc >= 0 && cc < BC) cdiag[cc] += t.gauge_coefficient[g]; }
        MgLevel cur;
        cur.cells = BC;
        cur.diag = std::move(cdiag);
        cur.coord.resize(BC);
        for (int q = 0; q < BC; ++q) cur.coord[q] = gc(q);
        for (int q = 0; q < BC; ++q)
        {
            const int brick = q / c3, local = q % c3, ijk[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
            for (int axis = 0; axis < 3; ++axis)
            {
                const double c = positive[size_t(q) * 3 + axis];
                if (!(c > 0)) continue;
                int cc[3] = {ijk[0], ijk[1], ijk[2]}, other = -1;
                if (++cc[axis] < bs) other = brick * c3 + (cc[2] * bs + cc[1]) * bs + cc[0];
                else
                {
                    const int nb = base.neighbors[brick * 6 + 2 * axis + 1];
                    if (nb >= 0) { cc[axis] = 0; other = nb * c3 + (cc[2] * bs + cc[1]) * bs + cc[0]; }
                }
                if (other >= 0) cur.edges.push_back({q, other, c});
            }
        }
        cur.edges.insert(cur.edges.end(), extra.begin(), extra.end());
        for (;;)
        {
            int act = 0;
            for (double v : cur.diag) if (v > 0) ++act;
            if (act <= 512 || s.mg.size() >= 8) { finalize(cur); s.mg.push_back(std::move(cur)); break; }
            std::vector<int> parent(cur.cells, -1);
            for (int q = 0; q < cur.cells; ++q) if (cur.diag[q] > 0) parent[q] = q;
            auto root = [&](int q) { int r = q; while (parent[r] != r) r = parent[r]; while (parent[q] != q) { const int nx = parent[q]; parent[q] = r; q = nx; } return r; };
            for (const Edge& e : cur.edges)
            {
                const auto& A = cur.coord[e.a];
                const auto& Bc = cur.coord[e.b];
                if (A[0] / 2 != Bc[0] / 2 || A[1] / 2 != Bc[1] / 2 || A[2] / 2 != Bc[2] / 2) continue;
                const int ra = root(e.a), rb = root(e.b);
                if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
            }
            cur.aggregate.assign(cur.cells, -1);
            std::vector<int> ridx(cur.cells, -1);
            MgLevel next;
            for (int q = 0; q < cur.cells; ++q)
                if (parent[q] >= 0)
                {
                    const int r = root(q);
                    if (ridx[r] < 0) { ridx[r] = next.cells++; next.coord.push_back({cur.coord[q][0] / 2, cur.coord[q][1] / 2, cur.coord[q][2] / 2}); }
                    cur.aggregate[q] = ridx[r];
                }
            if (next.cells <= 0 || next.cells >= act) { finalize(cur); s.mg.push_back(std::move(cur)); break; }
            cur.roff.assign(size_t(next.cells) + 1, 0);
            for (int q = 0; q < cur.cells; ++q) if (cur.aggregate[q] >= 0) ++cur.roff[cur.aggregate[q] + 1];
            for (int q = 0; q < next.cells; ++q) cur.roff[q + 1] += cur.roff[q];
            cur.rdof.resize(cur.roff.back());
            {
                std::vector<int> rc = cur.roff;
                for (int q = 0; q < cur.cells; ++q) if (cur.aggregate[q] >= 0) cur.rdof[rc[cur.aggregate[q]]++] = q;
            }
            std::vector<double> incident(cur.cells, 0), ground(next.cells, 0);
            for (const Edge& e : cur.edges) { incident[e.a] += e.c; incident[e.b] += e.c; }
            for (int q = 0; q < cur.cells; ++q)
                if (cur.diag[q] > 0) ground[cur.aggregate[q]] += std::max(0.0, cur.diag[q] - incident[q]);
            std::unordered_map<uint64_t, double> w;
            for (const Edge& e : cur.edges)
            {
                int a = cur.aggregate[e.a], b = cur.aggregate[e.b];
                if (a == b) continue;
                if (a > b) std::swap(a, b);
                w[(uint64_t(uint32_t(a)) << 32) | uint32_t(b)] += e.c;
            }
            for (const auto& it : w) next.edges.push_back({int(it.first >> 32), int(it.first & 0xffffffffu), it.second});
            std::sort(next.edges.begin(), next.edges.end(), [](const Edge& a, const Edge& b) { return a.a < b.a || (a.a == b.a && a.b < b.b); });
            next.diag = std::move(ground);
            for (const Edge& e : next.edges) { next.diag[e.a] += e.c; next.diag[e.b] += e.c; }
            finalize(cur);
            s.mg.push_back(std::move(cur));
            cur = std::move(next);
        }
    }

    void jacobi(MgLevel& L, int sweeps)
    {
        const double omega = 2.0 / 3.0;
        for (int sw = 0; sw < sweeps; ++sw)
        {
#pragma omp parallel for schedule(static)
            for (int q = 0; q < L.cells; ++q)
            {
                if (!(L.diag[q] > 0)) { L.tmp[q] = 0; continue; }
                double Ax = L.diag[q] * L.x[q];
                for (int e = L.row[q]; e < L.row[q + 1]; ++e) Ax -= L.coef[e] * L.x[L.nbr[e]];
                L.tmp[q] = L.x[q] + omega * ((L.rhs[q] - Ax) / L.diag[q]);
            }
            std::swap(L.x, L.tmp);
        }
    }

    void mg_level(po_system& s, int index)
    {
        MgLevel& L = s.mg[index];
        if (index + 1 == int(s.mg.size())) { jacobi(L, 96); return; }
        jacobi(L, 2);
#pragma omp parallel for schedule(static)
        for (int q = 0; q < L.cells; ++q)
        {
            if (!(L.diag[q] > 0)) { L.res[q] = 0; continue; }
            double Ax = L.diag[q] * L.x[q];
            for (int e = L.row[q]; e < L.row[q + 1]; ++e) Ax -= L.coef[e] * L.x[L.nbr[e]];
            L.res[q] = L.rhs[q] - Ax;
        }
        MgLevel& C = s.mg[index + 1];
#pragma omp parallel for schedule(static)
        for (int c = 0; c < C.cells; ++c)
        {
            double v = 0;
            for (int q = L.roff[c]; q < L.roff[c + 1]; ++q) v += L.res[L.rdof[q]];
            C.rhs[c] = v;
        }
        std::fill(C.x.begin(), C.x.end(), 0.0);
        mg_level(s, index + 1);
#pragma omp parallel for schedule(static)
        for (int q = 0; q < L.cells; ++q) if (L.aggregate[q] >= 0) L.x[q] += C.x[L.aggregate[q]];
        jacobi(L, 2);
    }

    // ---- composite cycle (paracfd_b200 solver.cu build_composite, smoother.cu composite_cycle) ----
    // Stage k merges the level-l structured cells at global cell coordinates g into (l, g >> k);
    // Galerkin operators of the fine orthogonal couplings (+ outlet and gauge diagonal terms);
    // stages down to 512 cells; the coarsest solved with its explicit inverse.
    void build_composite(po_system& s)
    {
        const pcfd_topology& t = s.t;
        const int bs = s.bs, c3 = s.c3, S = s.S;
        std::vector<int> dof_level(S, -1);
        std::vector<std::array<int64_t, 3>> g(S);
        for (int l = 0; l < t.level_count; ++l)
        {
            const pcfd_level& lev = t.levels[l];
            for (int b = 0; b < lev.brick_count; ++b)
            {
                if (lev.flags[b] & COVERED) continue;
                for (int c = 0; c < c3; ++c)
                {
                    const int q = lev.level_offset + b * c3 + c;
                    if (!t.active[q]) continue;
                    dof_level[q] = l;
                    g[q] = {int64_t(lev.coord[3 * b]) * bs + c % bs, int64_t(lev.coord[3 * b + 1]) * bs + (c / bs) % bs,
                            int64_t(lev.coord[3 * b + 2]) * bs + c / (bs * bs)};
                }
            }
        }
        {
            // EB fragments (DOFs after the structured slots) join the cell that contains their
            // centroid: the finest non-covered brick there, the cell index clamped to the brick
            std::vector<std::unordered_map<uint64_t, int>> lookup(t.level_count);
            auto ck = [](int64_t x, int64_t y, int64_t z) { return (uint64_t(x & 0xfffff) << 40) | (uint64_t(y & 0xfffff) << 20) | uint64_t(z & 0xfffff); };
            for (int l = 0; l < t.level_count; ++l)
                for (int b = 0; b < t.levels[l].brick_count; ++b)
                    lookup[l][ck(t.levels[l].coord[3 * b], t.levels[l].coord[3 * b + 1], t.levels[l].coord[3 * b + 2])] = b;
            int placed = 0, total = 0;
            for (int q = s.B * c3; q < S; ++q)
            {
                if (!t.active[q]) continue;
                ++total;
                const double* c = t.centroid + 3 * size_t(q);
                for (int l = t.level_count - 1; l >= 0; --l)
                {
                    const pcfd_level& lev = t.levels[l];
                    const double w = bs * lev.h;
                    int64_t bc[3];
                    for (int a = 0; a < 3; ++a) bc[a] = int64_t(std::floor((c[a] - t.domain_lo[a]) / w));
                    auto it = lookup[l].find(ck(bc[0], bc[1], bc[2]));
                    if (it == lookup[l].end() || (lev.flags[it->second] & COVERED)) continue;
                    const int b = it->second;
                    int64_t gc[3];
                    for (int a = 0; a < 3; ++a)
                        gc[a] = int64_t(lev.coord[3 * b + a]) * bs +
                                std::min<int64_t>(bs - 1, std::max<int64_t>(0, int64_t(std::floor((c[a] - lev.origin[3 * b + a]) / lev.h))));
                    dof_level[q] = l;
                    g[q] = {gc[0], gc[1], gc[2]};
                    ++placed;
                    break;
                }
            }
            (void)placed; (void)total;
        }
        auto key = [](int m, int64_t x, int64_t y, int64_t z) {
            return (uint64_t(m) << 60) | (uint64_t(x & 0xfffff) << 40) | (uint64_t(y & 0xfffff) << 20) | uint64_t(z & 0xfffff);
        };
        std::vector<std::vector<int>> maps;
        std::vector<int> cells;
        for (int k = 1; k <= 16; ++k)
        {
            std::vector<int> m(S, -1);
            std::unordered_map<uint64_t, int> index;
            for (int q = 0; q < S; ++q)
            {
                if (dof_level[q] < 0) continue;
                const uint64_t kq = key(dof_level[q], g[q][0] >> k, g[q][1] >> k, g[q][2] >> k);
                auto it = index.find(kq);
                if (it == index.end()) it = index.emplace(kq, int(index.size())).first;
                m[q] = it->second;
            }
            const int n = int(index.size());
            if (n == 0 || (!cells.empty() && n >= cells.back())) break;
            maps.push_back(std::move(m));
            cells.push_back(n);
            if (n <= 512) break;
        }
        s.stages.assign(maps.size(), MgLevel());
        for (size_t k = 0; k < maps.size(); ++k)
        {
            const std::vector<int>& m = maps[k];
            MgLevel& L = s.stages[k];
            L.cells = cells[k];
            L.diag.assign(L.cells, 0.0);
            std::unordered_map<uint64_t, double> w;
            auto add = [&](int a, int b, double c) {
                if (a < 0 || b < 0 || a == b || !t.active[a] || !t.active[b] || !(c > 0)) return;
                int ca = m[a], cb = m[b];
                if (ca < 0 || cb < 0 || ca == cb) return;
                L.diag[ca] += c;
                L.diag[cb] += c;
                if (ca > cb) std::swap(ca, cb);
                w[(uint64_t(uint32_t(ca)) << 32) | uint32_t(cb)] += c;
            };
            for (int l = 0; l < t.level_count; ++l)
            {
                const pcfd_level& lev = t.levels[l];
                for (int brick = 0; brick < lev.brick_count; ++brick)
                {
                    if (lev.flags[brick] & COVERED) continue;
                    for (int c = 0; c < c3; ++c)
                    {
                        const int a = lev.level_offset + brick * c3 + c;
                        if (!t.active[a]) continue;
                        const int ijk[3] = {c % bs, (c / bs) % bs, c / (bs * bs)};
                        for (int axis = 0; axis < 3; ++axis)
                        {
                            if (t.cut_face_mask[a] & (1u << axis)) continue;
                            int q[3] = {ijk[0], ijk[1], ijk[2]}, b = -1;
                            if (++q[axis] < bs) b = lev.level_offset + brick * c3 + (q[2] * bs + q[1]) * bs + q[0];
                            else
                            {
                                const int nb = lev.neighbors[brick * 6 + 2 * axis + 1];
                                if (nb >= 0 && !(lev.flags[nb] & COVERED)) { q[axis] = 0; b = lev.level_offset + nb * c3 + (q[2] * bs + q[1]) * bs + q[0]; }
                            }
                            add(a, b, lev.h);
                        }
                        if (t.pressure_outlet_xmax && (lev.flags[brick] & XMAX) && ijk[0] == bs - 1 && m[a] >= 0) L.diag[m[a]] += 2.0 * lev.h;
                    }
                }
            }
            for (int e = 0; e < t.coarse_fine.count; ++e) add(t.coarse_fine.coarse_dof[e], t.coarse_fine.fine_dof[e], t.coarse_fine.open_area[e] * factor_of(t.coarse_fine, e));
            for (int e = 0; e < t.embedded.count; ++e) add(t.embedded.coarse_dof[e], t.embedded.fine_dof[e], t.embedded.open_area[e] * factor_of(t.embedded, e));
            for (int e = 0; e < t.regular.count; ++e) add(t.regular.lower_dof[e], t.regular.upper_dof[e], t.regular.open_area[e] * t.regular.two_point_delta[e]);
            for (int gg = 0; gg < t.gauge_count; ++gg)
            {
                const int q = t.gauge_dof[gg];
                if (t.active[q] && m[q] >= 0) L.diag[m[q]] += t.gauge_coefficient[gg];
            }
            for (const auto& it : w) L.edges.push_back({int(it.first >> 32), int(it.first & 0xffffffffu), it.second});
            std::sort(L.edges.begin(), L.edges.end(), [](const Edge& x, const Edge& y) { return x.a < y.a || (x.a == y.a && x.b < y.b); });
        }
        for (size_t k = 0; k < s.stages.size(); ++k)
        {
            MgLevel& L = s.stages[k];
            if (k + 1 < s.stages.size())
            {
                L.aggregate.assign(L.cells, -1);
                for (int q = 0; q < S; ++q) if (maps[k][q] >= 0) L.aggregate[maps[k][q]] = maps[k + 1][q];
                const int next = cells[k + 1];
                L.roff.assign(size_t(next) + 1, 0);
                for (int c = 0; c < L.cells; ++c) if (L.aggregate[c] >= 0) ++L.roff[L.aggregate[c] + 1];
                for (int c = 0; c < next; ++c) L.roff[c + 1] += L.roff[c];
                L.rdof.resize(L.roff.back());
                std::vector<int> cur = L.roff;
                for (int c = 0; c < L.cells; ++c) if (L.aggregate[c] >= 0) L.rdof[cur[L.aggregate[c]]++] = c;
            }
            finalize(L);
        }
        s.fine_map = maps.front();
        const int n1 = cells.front();
        s.fine_roff.assign(size_t(n1) + 1, 0);
        for (int q = 0; q < S; ++q) if (s.fine_map[q] >= 0) ++s.fine_roff[s.fine_map[q] + 1];
        for (int c = 0; c < n1; ++c) s.fine_roff[c + 1] += s.fine_roff[c];
        s.fine_rdof.resize(s.fine_roff.back());
        {
            std::vector<int> cur = s.fine_roff;
            for (int q = 0; q < S; ++q) if (s.fine_map[q] >= 0) s.fine_rdof[cur[s.fine_map[q]]++] = q;
        }
        // explicit inverse of the coarsest stage over its cells with a positive diagonal
        s.coarse_inverse.clear();
        const MgLevel& C = s.stages.back();
        if (C.cells <= 512)
        {
            const int n = C.cells;
            std::vector<int> live, idx(n, -1);
            for (int q = 0; q < n; ++q) if (C.diag[q] > 0) { idx[q] = int(live.size()); live.push_back(q); }
            const int m = int(live.size());
            std::vector<double> a(size_t(m) * m, 0.0), inv(size_t(m) * m, 0.0);
            double scale = 0;
            for (int i = 0; i < m; ++i) { a[size_t(i) * m + i] = C.diag[live[i]]; inv[size_t(i) * m + i] = 1; scale = std::max(scale, C.diag[live[i]]); }
            for (const Edge& e : C.edges)
            {
                const int i = idx[e.a], j = idx[e.b];
                if (i < 0 || j < 0) continue;
                a[size_t(i) * m + j] -= e.c;
                a[size_t(j) * m + i] -= e.c;
            }
            bool ok = m > 0;
            for (int c = 0; c < m && ok; ++c)
            {
                int p = c;
                for (int r = c + 1; r < m; ++r) if (std::abs(a[size_t(r) * m + c]) > std::abs(a[size_t(p) * m + c])) p = r;
                if (!(std::abs(a[size_t(p) * m + c]) > 1e-12 * scale)) { ok = false; break; }
                if (p != c)
                    for (int j = 0; j < m; ++j) { std::swap(a[size_t(p) * m + j], a[size_t(c) * m + j]); std::swap(inv[size_t(p) * m + j], inv[size_t(c) * m + j]); }
                const double d = 1.0 / a[size_t(c) * m + c];
                for (int j = 0; j < m; ++j) { a[size_t(c) * m + j] *= d; inv[size_t(c) * m + j] *= d; }
                for (int r = 0; r < m; ++r)
                {
                    if (r == c) continue;
                    const double f = a[size_t(r) * m + c];
                    if (f == 0.0) continue;
                    for (int j = 0; j < m; ++j) { a[size_t(r) * m + j] -= f * a[size_t(c) * m + j]; inv[size_t(r) * m + j] -= f * inv[size_t(c) * m + j]; }
                }
            }
            if (ok)
            {
                s.coarse_inverse.assign(size_t(n) * n, 0.0);
                for (int i = 0; i < m; ++i)
                    for (int j = 0; j < m; ++j) s.coarse_inverse[size_t(live[i]) * n + live[j]] = inv[size_t(i) * m + j];
            }
        }
        s.fine_res.assign(S, 0.0);
        s.composite = true;
    }

    // stage smoothing: damped Jacobi (ratio < 2) or Chebyshev of D^-1 A on [2 / ratio, 2]
    void stage_smooth(po_system& s, MgLevel& L, int steps)
    {
        if (s.stage_ratio < 2) { jacobi(L, steps); return; }
        const double hi = 2.0, lo = hi / s.stage_ratio, theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
        double rho = 1.0 / sigma;
        s.stage_d.assign(L.cells, 0.0);
        for (int k = 0; k < steps; ++k)
        {
            double c1 = 0.0, c2 = 1.0 / theta;
            if (k)
            {
                const double next = 1.0 / (2.0 * sigma - rho);
                c1 = next * rho;
                c2 = 2.0 * next / delta;
                rho = next;
            }
#pragma omp parallel for schedule(static)
            for (int q = 0; q < L.cells; ++q)
            {
                if (!(L.diag[q] > 0)) { L.tmp[q] = 0; s.stage_d[q] = 0; continue; }
                double Ax = L.diag[q] * L.x[q];
                for (int e = L.row[q]; e < L.row[q + 1]; ++e) Ax -= L.coef[e] * L.x[L.nbr[e]];
                const double step = c2 * ((L.rhs[q] - Ax) / L.diag[q]);
                const double dn = k ? c1 * s.stage_d[q] + step : step;
                s.stage_d[q] = dn;
                L.tmp[q] = L.x[q] + dn;
            }
            std::swap(L.x, L.tmp);
        }
    }

    void stage_cycle(po_system& s, int index)
    {
        MgLevel& L = s.stages[index];
        if (index + 1 == int(s.stages.size()))
        {
            if (!s.coarse_inverse.empty())
            {
                const int n = L.cells;
#pragma omp parallel for schedule(static)
                for (int i = 0; i < n; ++i)
                {
                    double v = 0;
                    for (int j = 0; j < n; ++j) v += s.coarse_inverse[size_t(i) * n + j] * L.rhs[j];
                    L.x[i] = v;
                }
            }
            else jacobi(L, 96);
            return;
        }
        stage_smooth(s, L, s.stage_steps);
#pragma omp parallel for schedule(static)
        for (int q = 0; q < L.cells; ++q)
        {
            if (!(L.diag[q] > 0)) { L.res[q] = 0; continue; }
            double Ax = L.diag[q] * L.x[q];
            for (int e = L.row[q]; e < L.row[q + 1]; ++e) Ax -= L.coef[e] * L.x[L.nbr[e]];
            L.res[q] = L.rhs[q] - Ax;
        }
        MgLevel& C = s.stages[index + 1];
#pragma omp parallel for schedule(static)
        for (int c = 0; c < C.cells; ++c)
        {
            double v = 0;
            for (int q = L.roff[c]; q < L.roff[c + 1]; ++q) v += L.res[L.rdof[q]];
            C.rhs[c] = v;
        }
        std::fill(C.x.begin(), C.x.end(), 0.0);
        stage_cycle(s, index + 1);
#pragma omp parallel for schedule(static)
        for (int q = 0; q < L.cells; ++q) if (L.aggregate[q] >= 0) L.x[q] += 2.0 * C.x[L.aggregate[q]];
        stage_smooth(s, L, s.stage_steps);
    }

    // fine sweeps with the Chebyshev-Richardson step sizes of [2 / fine_ratio, 2] (or w = 2/3),
    // two before and two after the stage correction, which is prolonged with weight 2
    void precondition_composite(po_system& s, const double* r, double* z)
    {
        const uint8_t* act = s.t.active;
        double w[4] = {2.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0};
        if (s.fine_ratio >= 2)
        {
            const double hi = 2.0, lo = hi / s.fine_ratio, theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
            const double steps[2] = {1.0 / (theta + delta * std::sqrt(0.5)), 1.0 / (theta - delta * std::sqrt(0.5))};
            for (int k = 0; k < 4; ++k) w[k] = steps[k & 1];
        }
        auto sweep = [&](double omega) {
            apply(s, z, s.tv.data(), true);
#pragma omp parallel for schedule(static)
            for (int q = 0; q < s.S; ++q) if (act[q] && s.diagonal[q] > 0) z[q] += omega * (r[q] - s.tv[q]) / s.diagonal[q];
        };
#pragma omp parallel for schedule(static)
        for (int q = 0; q < s.S; ++q) z[q] = act[q] && s.diagonal[q] > 0 ? w[0] * r[q] / s.diagonal[q] : 0.0;
        sweep(w[1]);
        apply(s, z, s.tv.data(), true);
        MgLevel& first = s.stages.front();
#pragma omp parallel for schedule(static)
        for (int c = 0; c < first.cells; ++c)
        {
            double v = 0;
            for (int q = s.fine_roff[c]; q < s.fine_roff[c + 1]; ++q) v += r[s.fine_rdof[q]] - s.tv[s.fine_rdof[q]];
            first.rhs[c] = v;
        }
        std::fill(first.x.begin(), first.x.end(), 0.0);
        stage_cycle(s, 0);
#pragma omp parallel for schedule(static)
        for (int q = 0; q < s.S; ++q) if (act[q] && s.fine_map[q] >= 0) z[q] += 2.0 * first.x[s.fine_map[q]];
        sweep(w[2]);
        sweep(w[3]);
    }

    void precondition(po_system& s, const double* r, double* z)
    {
        if (s.composite) { precondition_composite(s, r, z); return; }
        const double omega = 2.0 / 3.0;
        const uint8_t* act = s.t.active;
        auto jcorr = [&]() {
            apply(s, z, s.tv.data(), true);
#pragma omp parallel for schedule(static)
            for (int q = 0; q < s.S; ++q) if (act[q] && s.diagonal[q] > 0) z[q] += omega * (r[q] - s.tv[q]) / s.diagonal[q];
        };
#pragma omp parallel for schedule(static)
        for (int q = 0; q < s.S; ++q) z[q] = act[q] && s.diagonal[q] > 0 ? omega * r[q] / s.diagonal[q] : 0.0;
        jcorr();
        if (s.mg.empty()) return;
        MgLevel& b = s.mg.front();
        std::fill(b.x.begin(), b.x.end(), 0.0);
        apply(s, z, s.tv.data(), true);
#pragma omp parallel for schedule(static)
        for (int c = 0; c < b.cells; ++c)
        {
            double v = 0;
            for (int q = s.base_roff[c]; q < s.base_roff[c + 1]; ++q) v += r[s.base_rdof[q]] - s.tv[s.base_rdof[q]];
            b.rhs[c] = v;
        }
        mg_level(s, 0);
#pragma omp parallel for schedule(static)
        for (int q = 0; q < s.S; ++q)
        {
            if (!act[q]) continue;
            const int c = s.t.preconditioner_aggregate[q] - s.base_offset;
            if (c >= 0 && c < s.base_cells) z[q] += b.x[c];
        }
        jcorr();
        jcorr();
    }

    void axpy(po_system& s, double* y, const double* x, double a)
    {
#pragma omp parallel for schedule(static)
        for (int q = 0; q < s.S; ++q) if (s.t.active[q]) y[q] += a * x[q];
    }
    void copy_active(po_system& s, const double* x, double* y)
    {
#pragma omp parallel for schedule(static)
        for (int q = 0; q < s.S; ++q) y[q] = s.t.active[q] ? x[q] : 0.0;
    }
    void residual(po_system& s, const double* x, const double* b, double* r, bool orth)
    {
        apply(s, x, s.Ad.data(), orth);
#pragma omp parallel for schedule(static)
        for (int q = 0; q < s.S; ++q) r[q] = s.t.active[q] ? b[q] - s.Ad[q] : 0.0;
    }

    int solve_pcg(po_system& s, double* x, const double* b, double tol, int maxit, bool warm, double* out)
    {
        const int n = s.S;
        if (!warm) std::fill(x, x + n, 0.0);
        const double rhs2 = dot(s, b, b);
        out[0] = 0; out[1] = 0; out[2] = 0;
        if (rhs2 == 0) { std::fill(x, x + n, 0.0); return 1; }
        double r2;
        if (warm) { residual(s, x, b, s.r.data(), true); r2 = dot(s, s.r.data(), s.r.data()); }
        else { std::copy(b, b + n, s.r.data()); r2 = rhs2; }
        out[0] = std::sqrt(r2 / rhs2);
        if (out[0] <= tol) return 1;
        auto restart = [&]() { precondition(s, s.r.data(), s.z.data()); out[2] += 1; copy_active(s, s.z.data(), s.d.data()); return dot(s, s.r.data(), s.z.data()); };
        double rz = restart();
        int converged = 0;
        for (int it = 0; it < maxit; ++it)
        {
            apply(s, s.d.data(), s.Ad.data(), true);
            const double pAp = dot(s, s.d.data(), s.Ad.data());
            if (!(pAp > 0)) break;
            const double alpha = rz / pAp;
#pragma omp parallel for schedule(static)
            for (int q = 0; q < n; ++q) if (s.t.active[q]) { x[q] += alpha * s.d[q]; s.r[q] -= alpha * s.Ad[q]; }
            r2 = dot(s, s.r.data(), s.r.data());
            out[1] = it + 1;
            out[0] = std::sqrt(r2 / rhs2);
            if (out[0] <= tol || (it + 1) % 128 == 0)
            {
                residual(s, x, b, s.r.data(), true);
                out[0] = std::sqrt(dot(s, s.r.data(), s.r.data()) / rhs2);
                if (out[0] <= tol) { converged = 1; break; }
                rz = restart();
                continue;
            }
            precondition(s, s.r.data(), s.z.data());
            out[2] += 1;
            const double nrz = dot(s, s.r.data(), s.z.data());
            if (!(nrz > 0)) break;
            const double beta = nrz / rz;
#pragma omp parallel for schedule(static)
            for (int q = 0; q < n; ++q) s.d[q] = s.t.active[q] ? s.z[q] + beta * s.d[q] : 0.0;
            rz = nrz;
        }
        residual(s, x, b, s.defect.data(), true);
        out[0] = std::sqrt(dot(s, s.defect.data(), s.defect.data()) / rhs2);
        return out[0] <= tol ? 1 : converged;
    }

    int solve_gcro(po_system& s, double* x, const double* b, double tol, int maxit, bool warm, double* out)
    {
        const int n = s.S, R = 24, cap = 3;
        if ((int)s.V.size() != (R + 1) * n) { s.V.assign(size_t(R + 1) * n, 0); s.Z.assign(size_t(R) * n, 0); s.RU.assign(size_t(cap) * n, 0); s.RC.assign(size_t(cap) * n, 0); }
        out[0] = out[1] = out[2] = 0;
        if (!warm) { s.recycle = 0; std::fill(x, x + n, 0.0); }
        const double rhs2 = dot(s, b, b);
        if (rhs2 == 0) { std::fill(x, x + n, 0.0); return 1; }
        auto vec = [&](std::vector<double>& base, int c) { return base.data() + size_t(c) * n; };
        residual(s, x, b, s.defect.data(), false);
        double r2 = dot(s, s.defect.data(), s.defect.data());
        out[0] = std::sqrt(r2 / rhs2);
        if (out[0] <= tol) return 1;
        int its = 0;
        while (its < maxit)
        {
            const double before = r2;
            const int attempted = s.recycle;
            if (attempted) { copy_active(s, x, s.corrv.data()); copy_active(s, s.defect.data(), s.tv.data()); }
            for (int pass = 0; pass < 2; ++pass)
                for (int c = 0; c < s.recycle; ++c)
                {
                    const double v = dot(s, vec(s.RC, c), s.defect.data());
                    axpy(s, s.corrv.data(), vec(s.RU, c), v);
                    axpy(s, s.defect.data(), vec(s.RC, c), -v);
                }
            double gap2 = 0, truer2 = before;
            if (attempted)
            {
                copy_active(s, s.defect.data(), s.r.data());
                residual(s, s.corrv.data(), b, s.defect.data(), false);
                truer2 = dot(s, s.defect.data(), s.defect.data());
                axpy(s, s.r.data(), s.defect.data(), -1.0);
                gap2 = dot(s, s.r.data(), s.r.data());
            }
            const bool ok = !attempted || (std::sqrt(gap2) <= 0.25 * tol * std::sqrt(rhs2) && truer2 < before);
            if (attempted && ok) { copy_active(s, s.corrv.data(), x); r2 = truer2; }
            else if (attempted) { s.recycle = 0; copy_active(s, s.tv.data(), s.defect.data()); r2 = before; }
            out[0] = std::sqrt(r2 / rhs2);
            if (out[0] <= tol)
            {
                residual(s, x, b, s.defect.data(), false);
                r2 = dot(s, s.defect.data(), s.defect.data());
                out[0] = std::sqrt(r2 / rhs2);
                if (out[0] <= tol) return 1;
            }
            const double beta = std::sqrt(r2);
            const int cycle = std::min(R, maxit - its);
            std::vector<double> H(size_t(cycle + 1) * cycle, 0), cs(cycle), sn(cycle), g(cycle + 1, 0), y(cycle);
            g[0] = beta;
#pragma omp parallel for schedule(static)
            for (int q = 0; q < n; ++q) s.V[q] = s.t.active[q] ? s.defect[q] / beta : 0.0;
            int used = 0;
            for (int col = 0; col < cycle; ++col)
            {
                double* v = vec(s.V, col);
                double* z = vec(s.Z, col);
                precondition(s, v, z);
                out[2] += 1;
                apply(s, z, s.Ad.data(), false);
                for (int pass = 0; pass < 2; ++pass)
                    for (int c = 0; c < s.recycle; ++c)
                    {
                        const double val = dot(s, vec(s.RC, c), s.Ad.data());
                        axpy(s, s.Ad.data(), vec(s.RC, c), -val);
                        axpy(s, z, vec(s.RU, c), -val);
                    }
                const double scale = std::sqrt(std::max(0.0, dot(s, s.Ad.data(), s.Ad.data())));
                if (!(scale > 0)) break;
                for (int pass = 0; pass < 2; ++pass)
                    for (int row = 0; row <= col; ++row)
                    {
                        const double val = dot(s, vec(s.V, row), s.Ad.data());
                        H[size_t(row) * cycle + col] += val;
                        axpy(s, s.Ad.data(), vec(s.V, row), -val);
                    }
                double nn = std::sqrt(std::max(0.0, dot(s, s.Ad.data(), s.Ad.data())));
                if (nn > 64 * std::numeric_limits<double>::epsilon() * scale)
                {
                    double* vn = vec(s.V, col + 1);
#pragma omp parallel for schedule(static)
                    for (int q = 0; q < n; ++q) vn[q] = s.t.active[q] ? s.Ad[q] / nn : 0.0;
                }
                else nn = 0;
                H[size_t(col + 1) * cycle + col] = nn;
                for (int row = 0; row < col; ++row)
                {
                    double& a = H[size_t(row) * cycle + col];
                    double& bb = H[size_t(row + 1) * cycle + col];
                    const double rot = cs[row] * a + sn[row] * bb;
                    bb = -sn[row] * a + cs[row] * bb;
                    a = rot;
                }
                double& dg = H[size_t(col) * cycle + col];
                double& bl = H[size_t(col + 1) * cycle + col];
                const double nrm = std::hypot(dg, bl);
                if (!(nrm > 0)) break;
                cs[col] = dg / nrm; sn[col] = bl / nrm; dg = nrm; bl = 0;
                const double old = g[col];
                g[col] = cs[col] * old;
                g[col + 1] = -sn[col] * old;
                used = col + 1;
                ++its;
                if (std::abs(g[col + 1]) / std::sqrt(rhs2) <= tol || nn == 0) break;
            }
            if (!used) break;
            for (int row = used - 1; row >= 0; --row)
            {
                double v = g[row];
                for (int c = row + 1; c < used; ++c) v -= H[size_t(row) * cycle + c] * y[c];
                y[row] = v / H[size_t(row) * cycle + row];
            }
            std::fill(s.corrv.begin(), s.corrv.end(), 0.0);
            for (int c = 0; c < used; ++c) axpy(s, s.corrv.data(), vec(s.Z, c), y[c]);
            axpy(s, x, s.corrv.data(), 1.0);
            residual(s, x, b, s.defect.data(), false);
            r2 = dot(s, s.defect.data(), s.defect.data());
            out[0] = std::sqrt(r2 / rhs2);
            apply(s, s.corrv.data(), s.Ad.data(), false);
            const double cb = std::sqrt(std::max(0.0, dot(s, s.Ad.data(), s.Ad.data())));
            bool valid = cb > 0;
            for (int pass = 0; pass < 2 && valid; ++pass)
                for (int c = 0; c < s.recycle; ++c)
                {
                    const double val = dot(s, vec(s.RC, c), s.Ad.data());
                    axpy(s, s.Ad.data(), vec(s.RC, c), -val);
                    axpy(s, s.corrv.data(), vec(s.RU, c), -val);
                }
            const double ca = valid ? std::sqrt(std::max(0.0, dot(s, s.Ad.data(), s.Ad.data()))) : 0;
            if (valid && ca > 1e-12 * cb)
            {
                if (s.recycle == cap)
                {
                    for (int c = 1; c < cap; ++c)
                    {
                        std::copy(vec(s.RU, c), vec(s.RU, c) + n, vec(s.RU, c - 1));
                        std::copy(vec(s.RC, c), vec(s.RC, c) + n, vec(s.RC, c - 1));
                    }
                    --s.recycle;
                }
                double* u = vec(s.RU, s.recycle);
                double* cc = vec(s.RC, s.recycle);
#pragma omp parallel for schedule(static)
                for (int q = 0; q < n; ++q) { u[q] = s.t.active[q] ? s.corrv[q] / ca : 0.0; cc[q] = s.t.active[q] ? s.Ad[q] / ca : 0.0; }
                ++s.recycle;
            }
            if (out[0] <= tol) { out[1] = its; return 1; }
        }
        out[1] = its;
        residual(s, x, b, s.defect.data(), false);
        out[0] = std::sqrt(dot(s, s.defect.data(), s.defect.data()) / rhs2);
        return out[0] <= tol;
    }

    inline size_t face_index(int bs, int axis, size_t slot, int i, int j, int k)
    {
        const size_t per = size_t(bs + 1) * bs * bs;
        if (axis == 0) return slot * per + size_t((k * bs + j) * (bs + 1) + i);
        if (axis == 1) return slot * per + size_t((k * (bs + 1) + j) * bs + i);
        return slot * per + size_t((k * bs + j) * bs + i);
    }
}

extern "C" {

int po_threads(void) { return omp_get_max_threads(); }

po_system* po_create(const pcfd_topology* topology)
{
    auto* s = new po_system();
    s->t = *topology;
    const pcfd_topology& t = s->t;
    s->bs = t.brick_size;
    s->c3 = s->bs * s->bs * s->bs;
    s->S = t.storage_size;
    int slot = 0;
    for (int l = 0; l < t.level_count; ++l)
    {
        const pcfd_level& lev = t.levels[l];
        s->slot0.push_back(slot);
        s->h.push_back(lev.h);
        for (int b = 0; b < lev.brick_count; ++b)
        {
            s->slot_level.push_back(l);
            s->flags.push_back(lev.flags[b]);
            for (int f = 0; f < 6; ++f)
            {
                const int n = lev.neighbors[b * 6 + f];
                s->nbr.push_back(n >= 0 && !(lev.flags[n] & COVERED) ? slot + n : -1);
            }
            if (!(lev.flags[b] & COVERED)) s->active_slots.push_back(slot + b);
        }
        slot += lev.brick_count;
    }
    s->B = slot;
    s->structured = s->B * s->c3;
    const int cf = t.coarse_fine.count, eb = t.embedded.count;
    s->nc = cf + eb;
    s->nr = t.regular.count;
    const int ne = s->nc + s->nr;
    s->lo.resize(ne); s->up.resize(ne); s->lnode.resize(ne); s->unode.resize(ne);
    s->coef.resize(ne); s->corr.resize(size_t(ne) * 3); s->uw.resize(ne); s->area.resize(ne);
    for (int e = 0; e < s->nc; ++e)
    {
        const pcfd_connections& c = e < cf ? t.coarse_fine : t.embedded;
        const int q = e < cf ? e : e - cf;
        const bool fwd = c.direction[q] > 0;
        s->lo[e] = fwd ? c.coarse_dof[q] : c.fine_dof[q];
        s->up[e] = fwd ? c.fine_dof[q] : c.coarse_dof[q];
        s->coef[e] = c.open_area[q] * factor_of(c, q);
        s->lnode[e] = c.lower_gradient_node[q]; s->unode[e] = c.upper_gradient_node[q];
        for (int a = 0; a < 3; ++a) s->corr[3 * e + a] = c.nonorthogonal_correction[3 * q + a];
        s->uw[e] = c.upper_gradient_weight[q];
        s->area[e] = c.open_area[q];
    }
    for (int r = 0; r < s->nr; ++r)
    {
        const int e = s->nc + r;
        s->lo[e] = t.regular.lower_dof[r]; s->up[e] = t.regular.upper_dof[r];
        s->coef[e] = t.regular.open_area[r] * t.regular.two_point_delta[r];
        s->lnode[e] = t.regular.lower_gradient_node[r]; s->unode[e] = t.regular.upper_gradient_node[r];
        for (int a = 0; a < 3; ++a) s->corr[3 * e + a] = t.regular.nonorthogonal_correction[3 * r + a];
        s->uw[e] = t.regular.upper_gradient_weight[r];
        s->area[e] = t.regular.open_area[r];
    }
    struct Inc { int dof, edge; int8_t sign; };
    std::vector<Inc> inc;
    for (int e = 0; e < ne; ++e)
    {
        const int a = s->lo[e], b = s->up[e];
        if (a < 0 || b < 0 || a == b || !t.active[a] || !t.active[b]) continue;
        inc.push_back({a, e, 1});
        inc.push_back({b, e, -1});
    }
    std::sort(inc.begin(), inc.end(), [](const Inc& a, const Inc& b) { return a.dof != b.dof ? a.dof < b.dof : (a.edge != b.edge ? a.edge < b.edge : a.sign < b.sign); });
    for (size_t q = 0; q < inc.size(); ++q)
    {
        if (q == 0 || inc[q].dof != inc[q - 1].dof) { s->inc_dof.push_back(inc[q].dof); s->inc_off.push_back(int(q)); }
        s->inc_edge.push_back(inc[q].edge);
        s->inc_sign.push_back(inc[q].sign);
    }
    s->inc_off.push_back(int(inc.size()));
    s->gradient.assign(size_t(t.gradient_node_count) * 3, 0.0);
    // diagonal (diagonal_cpu): sum of two-point coefficients of every open face + outlet + gauges
    s->diagonal.assign(s->S, 0.0);
    {
        std::vector<double> ones(s->S, 0.0);
        // diag = sum_faces coefficient: evaluate A e_a structurally without the p factor
        const int bs = s->bs, c3 = s->c3;
        for (int slot_i : s->active_slots)
        {
            const double h = s->h[s->slot_level[slot_i]];
            for (int local = 0; local < c3; ++local)
            {
                const int a = slot_i * c3 + local;
                if (!t.active[a]) continue;
                const int ijk[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
                for (int axis = 0; axis < 3; ++axis)
                    for (int sign = -1; sign <= 1; sign += 2)
                    {
                        int c[3] = {ijk[0], ijk[1], ijk[2]}, sl = slot_i;
                        c[axis] += sign;
                        if (c[axis] < 0 || c[axis] >= bs)
                        {
                            sl = s->nbr[slot_i * 6 + 2 * axis + (sign > 0)];
                            if (sl < 0) continue;
                            c[axis] = sign > 0 ? 0 : bs - 1;
                        }
                        const int b = sl * c3 + (c[2] * bs + c[1]) * bs + c[0];
                        const int lower = sign > 0 ? a : b;
                        if (t.active[b] && !(t.cut_face_mask[lower] & (1u << axis))) s->diagonal[a] += h;
                    }
                if (t.pressure_outlet_xmax && (s->flags[slot_i] & XMAX) && ijk[0] == bs - 1) s->diagonal[a] += 2.0 * h;
            }
        }
        for (int e = 0; e < ne; ++e)
        {
            const int a = s->lo[e], b = s->up[e];
            if (a < 0 || b < 0 || a == b || !t.active[a] || !t.active[b]) continue;
            s->diagonal[a] += s->coef[e];
            s->diagonal[b] += s->coef[e];
        }
        for (int g = 0; g < t.gauge_count; ++g) if (t.active[t.gauge_dof[g]]) s->diagonal[t.gauge_dof[g]] += t.gauge_coefficient[g];
    }
    build_mg(*s);
    for (std::vector<double>* v : {&s->r, &s->z, &s->d, &s->Ad, &s->tv, &s->corrv, &s->defect}) v->assign(s->S, 0.0);
    return s;
}

void po_destroy(po_system* s) { delete s; }

void po_apply(po_system* s, const double* p, double* out, int orthogonal) { apply(*s, p, out, orthogonal != 0); }
void po_diagonal(po_system* s, double* d) { std::copy(s->diagonal.begin(), s->diagonal.end(), d); }
void po_precondition(po_system* s, const double* r, double* z) { precondition(*s, r, z); }

void po_set_composite(po_system* s, int steps, int stage_ratio, int fine_ratio)
{
    s->stage_steps = steps > 0 ? steps : 6;
    s->stage_ratio = stage_ratio;
    s->fine_ratio = fine_ratio;
    build_composite(*s);
}

int po_solve(po_system* s, double* x, const double* b, double tol, int maxit, int warm, double* out)
{
    if (s->t.gradient_node_count == 0)
    {
        const int budget = maxit > std::numeric_limits<int>::max() / 5 ? maxit : 5 * maxit;
        return solve_pcg(*s, x, b, tol, budget, warm != 0, out);
    }
    return solve_gcro(*s, x, b, tol, maxit, warm != 0, out);
}

void po_divergence(po_system* s, const float* u, const float* v, const float* w, const float* special, double* integrated, double* div)
{
    const pcfd_topology& t = s->t;
    const int bs = s->bs, c3 = s->c3;
    std::vector<double> net(s->S, 0.0);
    const float* F[3] = {u, v, w};
#pragma omp parallel for schedule(static)
    for (int n = 0; n < int(s->active_slots.size()); ++n)
    {
        const int slot = s->active_slots[n];
        const double h = s->h[s->slot_level[slot]], area = h * h;
        for (int local = 0; local < c3; ++local)
        {
            const int a = slot * c3 + local;
            if (!t.active[a]) continue;
            const int ijk[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
            double sum = 0;
            for (int axis = 0; axis < 3; ++axis)
            {
                // + face
                int c[3] = {ijk[0], ijk[1], ijk[2]}, sl = slot;
                if (++c[axis] >= bs) { sl = s->nbr[slot * 6 + 2 * axis + 1]; c[axis] = 0; }
                if (sl >= 0)
                {
                    const int b = sl * c3 + (c[2] * bs + c[1]) * bs + c[0];
                    if (t.active[b] && !(t.cut_face_mask[a] & (1u << axis)))
                    {
                        int f[3] = {ijk[0], ijk[1], ijk[2]};
                        ++f[axis];
                        sum += double(F[axis][face_index(bs, axis, slot, f[0], f[1], f[2])]) * area;
                    }
                }
                // - face (owned by the lower cell's brick)
                int q[3] = {ijk[0], ijk[1], ijk[2]}, ls = slot;
                if (--q[axis] < 0) { ls = s->nbr[slot * 6 + 2 * axis]; q[axis] = bs - 1; }
                if (ls >= 0)
                {
                    const int lo = ls * c3 + (q[2] * bs + q[1]) * bs + q[0];
                    if (t.active[lo] && !(t.cut_face_mask[lo] & (1u << axis)))
                    {
                        int f[3] = {q[0], q[1], q[2]};
                        ++f[axis];
                        sum -= double(F[axis][face_index(bs, axis, ls, f[0], f[1], f[2])]) * area;
                    }
                }
            }
            if ((s->flags[slot] & XMIN) && ijk[0] == 0) sum -= double(u[face_index(bs, 0, slot, 0, ijk[1], ijk[2])]) * area;
            if ((s->flags[slot] & XMAX) && ijk[0] == bs - 1) sum += double(u[face_index(bs, 0, slot, bs, ijk[1], ijk[2])]) * area;
            net[a] = sum;
        }
    }
    for (int e = 0; e < s->nc; ++e)
    {
        const int a = s->lo[e], b = s->up[e];
        if (!t.active[a] || !t.active[b]) continue;
        const double flux = double(special[e]) * s->area[e];
        net[a] += flux;
        net[b] -= flux;
    }
    for (int q = 0; q < s->S; ++q)
    {
        if (integrated) integrated[q] = t.active[q] ? net[q] : 0.0;
        if (div) div[q] = t.active[q] && t.volume[q] > 0 ? net[q] / t.volume[q] : 0.0;
    }
}

void po_correct(po_system* s, const double* p, double rho, double dt, float* u, float* v, float* w, float* special)
{
    const pcfd_topology& t = s->t;
    const int bs = s->bs, c3 = s->c3;
    const double scale = dt / rho;
    float* F[3] = {u, v, w};
#pragma omp parallel for schedule(static)
    for (int n = 0; n < int(s->active_slots.size()); ++n)
    {
        const int slot = s->active_slots[n];
        const double h = s->h[s->slot_level[slot]];
        for (int local = 0; local < c3; ++local)
        {
            const int a = slot * c3 + local;
            if (!t.active[a]) continue;
            const int ijk[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
            for (int axis = 0; axis < 3; ++axis)
            {
                if (t.cut_face_mask[a] & (1u << axis)) continue;
                int c[3] = {ijk[0], ijk[1], ijk[2]}, sl = slot, nb = -1;
                if (++c[axis] >= bs) { nb = s->nbr[slot * 6 + 2 * axis + 1]; sl = nb; c[axis] = 0; }
                if (sl < 0) continue;
                const int b = sl * c3 + (c[2] * bs + c[1]) * bs + c[0];
                if (!t.active[b]) continue;
                int f[3] = {ijk[0], ijk[1], ijk[2]};
                ++f[axis];
                float& face = F[axis][face_index(bs, axis, slot, f[0], f[1], f[2])];
                face = float(double(face) - scale * (p[b] - p[a]) / h);
                if (nb >= 0)
                {
                    int m[3] = {ijk[0], ijk[1], ijk[2]};
                    m[axis] = 0;
                    F[axis][face_index(bs, axis, nb, m[0], m[1], m[2])] = face;
                }
            }
            if (t.pressure_outlet_xmax && (s->flags[slot] & XMAX) && ijk[0] == bs - 1)
            {
                float& face = u[face_index(bs, 0, slot, bs, ijk[1], ijk[2])];
                face = float(double(face) + scale * p[a] / (0.5 * h));
            }
        }
    }
    // WLS gradients, regular corrections, special faces (composite_amr_correct_fluxes_cpu order)
    const int nodes = t.gradient_node_count;
    std::vector<double> g(size_t(nodes) * 3, 0.0);
    for (int nd = 0; nd < nodes; ++nd)
    {
        const double centre = p[t.gradient_dof[nd]];
        for (int q = t.gradient_offset[nd]; q < t.gradient_offset[nd + 1]; ++q)
            for (int c = 0; c < 3; ++c) g[3 * nd + c] += t.gradient_weight[3 * q + c] * (p[t.gradient_neighbour[q]] - centre);
    }
    auto skew = [&](int e) {
        if (s->lnode[e] < 0 || s->unode[e] < 0) return 0.0;
        double d = 0;
        for (int c = 0; c < 3; ++c) d += s->corr[3 * e + c] * ((1 - s->uw[e]) * g[3 * s->lnode[e] + c] + s->uw[e] * g[3 * s->unode[e] + c]);
        return d;
    };
    for (int r = 0; r < s->nr; ++r)
    {
        const int e = s->nc + r;
        const int l = t.regular.level[r], brick = t.regular.brick[r], ax = t.regular.axis[r];
        const int i = t.regular.ijk[3 * r], j = t.regular.ijk[3 * r + 1], k = t.regular.ijk[3 * r + 2];
        const size_t slot = size_t(s->slot0[l] + brick);
        float& face = F[ax][face_index(bs, ax, slot, i, j, k)];
        face = float(double(face) - scale * (t.regular.two_point_delta[r] * (p[s->up[e]] - p[s->lo[e]]) + skew(e)));
        const int coord = ax == 0 ? i : (ax == 1 ? j : k);
        if (coord == bs)
        {
            const int nb = t.levels[l].neighbors[brick * 6 + 2 * ax + 1];
            if (nb >= 0)
            {
                int m[3] = {i, j, k};
                m[ax] = 0;
                F[ax][face_index(bs, ax, size_t(s->slot0[l] + nb), m[0], m[1], m[2])] = face;
            }
        }
    }
    for (int e = 0; e < s->nc; ++e)
    {
        const int a = s->lo[e], b = s->up[e];
        if (!t.active[a] || !t.active[b]) continue;
        const pcfd_connections& c = e < t.coarse_fine.count ? t.coarse_fine : t.embedded;
        const int q = e < t.coarse_fine.count ? e : e - t.coarse_fine.count;
        const double der = (p[b] - p[a]) * factor_of(c, q) + skew(e);
        special[e] = float(double(special[e]) - scale * der);
    }
    // 2:1 tiles: fine face <- tile, coarse face <- area mean of its tiles (device bridge semantics)
    std::unordered_map<uint64_t, std::pair<double, double>> group;
    std::vector<uint64_t> order;
    for (int e = 0; e < t.coarse_fine.count; ++e)
    {
        const int ax = t.coarse_fine.axis[e], dir = t.coarse_fine.direction[e];
        auto addr = [&](int dof, bool positive) {
            const int slot = dof / c3, local = dof % c3;
            int cc[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
            cc[ax] += positive ? 1 : 0;
            return face_index(bs, ax, size_t(slot), cc[0], cc[1], cc[2]);
        };
        F[ax][addr(t.coarse_fine.fine_dof[e], dir < 0)] = special[e];
        const uint64_t key = (uint64_t(addr(t.coarse_fine.coarse_dof[e], dir > 0)) << 2) | uint64_t(ax);
        auto it = group.find(key);
        if (it == group.end()) { order.push_back(key); it = group.emplace(key, std::make_pair(0.0, 0.0)).first; }
        it->second.first += t.coarse_fine.open_area[e] * double(special[e]);
        it->second.second += t.coarse_fine.open_area[e];
    }
    for (uint64_t key : order)
    {
        const auto& sum = group[key];
        if (sum.second > 0) F[key & 3][key >> 2] = float(sum.first / sum.second);
    }
}

}  // extern "C"
