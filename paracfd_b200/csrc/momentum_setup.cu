// momentum_setup.cu -- host derivation of the compact cell-momentum topology from the composite
// pressure system (done once per geometry, like the reference's
// DeviceCompositeCellMomentumTransport constructor, src/core/fluid/amr_advection.cu:1101-1226).
//
// Derived here:
//  * regular perimeter edges: same-level faces touching a DOF incident to an EB aperture
//    (reference build_composite_eb_momentum_regular_connections, amr_advection.cu:795-812); they are
//    removed from the structured brick stencil (compact_plus bits) and transported as compact edges;
//  * least-squares velocity-gradient nodes (reference build_composite_cell_gradient_topology,
//    amr_advection.cu:830-865): special DOFs, area/distance^2-weighted incidences, symmetric
//    pseudoinverse of the normal matrix, replaced by the pressure WLS stencil where one exists;
//  * per-edge conductance, face interpolation weight (composite_face_interpolation_weight,
//    amr_advection.cu:732-754) and face displacements;
//  * small-cell redistribution groups (amr_advection.cu:1108-1178);
//  * smooth-wall patch sides and boundary pressure faces (amr_advection.cu:1186-1208).
// Everything is indexed for deterministic per-DOF gathers on the device (no atomics).
#include "pseudoinverse3.h"
#include "momentum.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <numeric>
#include <set>
#include <unordered_map>
#include <unordered_set>

namespace pcfd
{
    namespace
    {
        struct V3 { double x = 0, y = 0, z = 0; };
        inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
        inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
        inline double comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

        double interpolation_weight(V3 lower, V3 upper, V3 face, int axis)
        {
            const V3 sep = sub(upper, lower);
            const double distance = std::sqrt(dot(sep, sep)), normal = comp(sep, axis);
            if (!(distance > 0) || !std::isfinite(distance)) throw Error(PCFD_INVALID_ARG, "face interpolation has coincident centroids");
            if (std::abs(normal) > 1e-12 * distance)
            {
                const double w = (comp(face, axis) - comp(lower, axis)) / normal;
                if (std::isfinite(w) && w >= -1e-8 && w <= 1 + 1e-8) return std::clamp(w, 0.0, 1.0);
            }
            const V3 dl = sub(face, lower), du = sub(face, upper);
            const double ld = std::sqrt(dot(dl, dl)), ud = std::sqrt(dot(du, du)), total = ld + ud;
            if (!(total > 1e-14 * std::max(1.0, distance)) || !std::isfinite(total)) return 0.5;
            return std::clamp(ld / total, 0.0, 1.0);
        }

        struct Edge
        {
            int a, b, axis, kind, source;   // kind 0 regular perimeter, 1 coarse/fine, 2 embedded
            double area, conductance, weight;
            V3 face;
            int64_t face_index;
        };
    }

    void build_momentum(System& s, Momentum& m, const pcfd_topology& t, double minimum_volume_fraction)
    {
        const int bs = s.bs, c3 = s.bs3, S = s.S;
        m.min_volume_fraction = minimum_volume_fraction;
        auto centroid = [&](int q) { return V3{t.centroid[3 * q], t.centroid[3 * q + 1], t.centroid[3 * q + 2]}; };
        auto active = [&](int q) { return q >= 0 && q < S && t.active[q] != 0; };
        std::vector<int> slot_level(s.B);
        for (int l = 0; l < s.levels; ++l)
            for (int b = 0; b < t.levels[l].brick_count; ++b) slot_level[s.level_slot0[l] + b] = l;
        auto brick_active = [&](int l, int b) { return b >= 0 && !(t.levels[l].flags[b] & PCFD_BRICK_COVERED); };

        // ---- regular perimeter edges --------------------------------------------------------
        std::unordered_set<int> embedded_nodes;
        for (int e = 0; e < t.embedded.count; ++e)
        {
            if (t.embedded.coarse_dof[e] >= 0) embedded_nodes.insert(t.embedded.coarse_dof[e]);
            if (t.embedded.fine_dof[e] >= 0) embedded_nodes.insert(t.embedded.fine_dof[e]);
        }
        std::vector<int> sorted_nodes(embedded_nodes.begin(), embedded_nodes.end());
        std::sort(sorted_nodes.begin(), sorted_nodes.end());
        std::vector<Edge> edges;
        std::vector<uint8_t> compact_plus(S, 0);
        {
            std::set<std::array<int, 3>> emitted;
            for (int dof : sorted_nodes)
            {
                if (dof >= s.structured || !active(dof)) continue;
                const int slot = dof / c3, local = dof % c3, l = slot_level[slot], brick = slot - s.level_slot0[l];
                if (!brick_active(l, brick)) continue;
                const pcfd_level& lev = t.levels[l];
                const int cell[3] = {local % bs, (local / bs) % bs, local / (bs * bs)};
                for (int axis = 0; axis < 3; ++axis)
                    for (int sign = -1; sign <= 1; sign += 2)
                    {
                        int c[3] = {cell[0], cell[1], cell[2]}, ob = brick;
                        c[axis] += sign;
                        if (c[axis] < 0 || c[axis] >= bs)
                        {
                            ob = lev.neighbors[brick * 6 + 2 * axis + (sign > 0)];
                            if (ob < 0 || !brick_active(l, ob)) continue;
                            c[axis] = sign > 0 ? 0 : bs - 1;
                        }
                        const int other = lev.level_offset + ob * c3 + (c[2] * bs + c[1]) * bs + c[0];
                        if (!active(other)) continue;
                        const int lower = sign > 0 ? dof : other, upper = sign > 0 ? other : dof;
                        if (t.cut_face_mask[lower] & (1u << axis)) continue;
                        if (!emitted.insert({lower, upper, axis}).second) continue;
                        // canonical face: the lower cell's positive face in the lower cell's brick
                        const int lslot = lower / c3, llocal = lower % c3, ll = slot_level[lslot], lbrick = lslot - s.level_slot0[ll];
                        int f[3] = {llocal % bs, (llocal / bs) % bs, llocal / (bs * bs)};
                        f[axis] += 1;
                        V3 face{lev.origin[3 * lbrick] + (f[0] + 0.5) * lev.h, lev.origin[3 * lbrick + 1] + (f[1] + 0.5) * lev.h,
                                lev.origin[3 * lbrick + 2] + (f[2] + 0.5) * lev.h};
                        if (axis == 0) face.x = lev.origin[3 * lbrick] + f[0] * lev.h;
                        else if (axis == 1) face.y = lev.origin[3 * lbrick + 1] + f[1] * lev.h;
                        else face.z = lev.origin[3 * lbrick + 2] + f[2] * lev.h;
                        const double area = lev.h * lev.h;
                        const V3 delta = sub(centroid(upper), centroid(lower));
                        const double d2 = dot(delta, delta), nd = std::abs(comp(delta, axis));
                        if (!(d2 > 0 && nd > 0)) throw Error(PCFD_INVALID_ARG, "invalid perimeter conductance");
                        Edge e{lower, upper, axis, 0, -1, area, area * nd / d2, 0.0, face, axis_face(bs, axis, lslot, f[0], f[1], f[2])};
                        edges.push_back(e);
                        compact_plus[lower] |= uint8_t(1u << axis);
                    }
            }
        }
        m.nR = int(edges.size());
        auto factor = [](const pcfd_connections& c, int e) {
            const double f = c.orthogonal_gradient_factor[e];
            return f > 0 ? f : (c.normal_distance[e] > 0 ? 1.0 / c.normal_distance[e] : 0.0);
        };
        auto add_special = [&](const pcfd_connections& c, int kind, int base) {
            for (int e = 0; e < c.count; ++e)
            {
                const bool fwd = c.direction[e] > 0;
                const int a = fwd ? c.coarse_dof[e] : c.fine_dof[e], b = fwd ? c.fine_dof[e] : c.coarse_dof[e];
                if (!active(a) || !active(b)) continue;   // inactive apertures carry no flux
                const double cond = c.open_area[e] * factor(c, e);
                if (!(cond > 0) || !std::isfinite(cond)) throw Error(PCFD_INVALID_ARG, "invalid compact conductance");
                const V3 face{c.face_centroid[3 * e], c.face_centroid[3 * e + 1], c.face_centroid[3 * e + 2]};
                edges.push_back(Edge{a, b, c.axis[e], kind, base + e, c.open_area[e], cond, 0.0, face, -1});
            }
        };
        add_special(t.coarse_fine, 1, 0);
        m.nC = int(edges.size()) - m.nR;
        add_special(t.embedded, 2, t.coarse_fine.count);
        m.nE = int(edges.size()) - m.nR - m.nC;
        m.nK = int(edges.size());
        for (Edge& e : edges) e.weight = interpolation_weight(centroid(e.a), centroid(e.b), e.face, e.axis);

        // ---- special (least-squares) nodes ---------------------------------------------------
        std::vector<uint8_t> special(S, 0);
        for (int q = 0; q < S; ++q) if (t.active[q] && t.cut_face_mask[q]) special[q] = 1;
        auto mark = [&](int q) { if (active(q)) special[q] = 1; };
        for (const Edge& e : edges) { mark(e.a); mark(e.b); }
        for (int e = 0; e < t.coarse_fine.count; ++e) { mark(t.coarse_fine.coarse_dof[e]); mark(t.coarse_fine.fine_dof[e]); }
        for (int e = 0; e < t.embedded.count; ++e) { mark(t.embedded.coarse_dof[e]); mark(t.embedded.fine_dof[e]); }
        for (int p = 0; p < t.patches.count; ++p) { mark(t.patches.plus_dof[p]); mark(t.patches.minus_dof[p]); }
        std::vector<int> special_index(S, -1), special_dof;
        for (int q = 0; q < S; ++q) if (special[q]) { special_index[q] = int(special_dof.size()); special_dof.push_back(q); }
        const int nS = int(special_dof.size());
        std::vector<double> normal(size_t(nS) * 9, 0.0);
        struct Inc { int special, neighbor; double w[3]; };
        std::vector<Inc> incs;
        auto add_inc = [&](int node, int nb, double area) {
            const int sp = special_index[node];
            if (sp < 0) return;
            const V3 d = sub(centroid(nb), centroid(node));
            const double d2 = dot(d, d);
            if (!(area > 0) || !(d2 > 1e-20)) throw Error(PCFD_INVALID_ARG, "invalid cell gradient incidence geometry");
            const double w = area / d2;
            incs.push_back({sp, nb, {w * d.x, w * d.y, w * d.z}});
            const double dv[3] = {d.x, d.y, d.z};
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) normal[size_t(sp) * 9 + r * 3 + c] += w * dv[r] * dv[c];
        };
        auto add_conn = [&](int a, int b, double area) { add_inc(a, b, area); add_inc(b, a, area); };
        for (int l = 0; l < s.levels; ++l)
        {
            const pcfd_level& lev = t.levels[l];
            const double area = lev.h * lev.h;
            for (int brick = 0; brick < lev.brick_count; ++brick)
            {
                if (!brick_active(l, brick)) continue;
                for (int k = 0; k < bs; ++k)
                    for (int j = 0; j < bs; ++j)
                        for (int i = 0; i < bs; ++i)
                        {
                            const int a = lev.level_offset + brick * c3 + (k * bs + j) * bs + i;
                            if (!t.active[a]) continue;
                            for (int axis = 0; axis < 3; ++axis)
                            {
                                if ((t.cut_face_mask[a] | compact_plus[a]) & (1u << axis)) continue;
                                int c[3] = {i, j, k}, ob = brick;
                                if (++c[axis] >= bs)
                                {
                                    ob = lev.neighbors[brick * 6 + 2 * axis + 1];
                                    if (ob < 0 || !brick_active(l, ob)) continue;
                                    c[axis] = 0;
                                }
                                const int b = lev.level_offset + ob * c3 + (c[2] * bs + c[1]) * bs + c[0];
                                if (t.active[b] && (special[a] || special[b])) add_conn(a, b, area);
                            }
                        }
            }
        }
        for (const Edge& e : edges) add_conn(e.a, e.b, e.area);
        std::vector<double> inverse(size_t(nS) * 9);
        for (int sp = 0; sp < nS; ++sp) pseudoinverse3(&normal[size_t(sp) * 9], &inverse[size_t(sp) * 9], 16, 1e-4);
        // Nodes with a checked pressure WLS stencil reuse it (identity inverse, WLS weights).
        std::vector<int> pnode(S, -1);
        for (int n = 0; n < t.gradient_node_count; ++n) pnode[t.gradient_dof[n]] = n;
        std::vector<Inc> checked;
        for (const Inc& c : incs) if (pnode[special_dof[c.special]] < 0) checked.push_back(c);
        for (int sp = 0; sp < nS; ++sp)
        {
            const int node = pnode[special_dof[sp]];
            if (node < 0) continue;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) inverse[size_t(sp) * 9 + r * 3 + c] = r == c ? 1.0 : 0.0;
            for (int q = t.gradient_offset[node]; q < t.gradient_offset[node + 1]; ++q)
                checked.push_back({sp, t.gradient_neighbour[q], {t.gradient_weight[3 * q], t.gradient_weight[3 * q + 1], t.gradient_weight[3 * q + 2]}});
        }
        std::stable_sort(checked.begin(), checked.end(), [](const Inc& a, const Inc& b) { return a.special < b.special; });
        m.nS = nS;
        {
            std::vector<int> off(size_t(nS) + 1, 0), nbr(checked.size());
            std::vector<float> w(checked.size() * 3), inv(size_t(nS) * 9);
            for (size_t q = 0; q < checked.size(); ++q)
            {
                ++off[checked[q].special + 1];
                nbr[q] = checked[q].neighbor;
                for (int a = 0; a < 3; ++a) w[3 * q + a] = float(checked[q].w[a]);
            }
            for (int sp = 0; sp < nS; ++sp) off[sp + 1] += off[sp];
            for (size_t q = 0; q < inverse.size(); ++q) inv[q] = float(inverse[q]);
            m.s_dof.upload(special_dof); m.s_offset.upload(off); m.s_neighbor.upload(nbr);
            m.s_weight.upload(w); m.s_inverse.upload(inv);
            m.s_gradient.alloc(size_t(nS) * 9);
        }

        // ---- compact edge arrays ---------------------------------------------------------------
        {
            const int nK = m.nK;
            std::vector<int> a(nK), b(nK), src(nK), sa(nK), sb(nK), pa(nK), pb(nK);
            std::vector<int8_t> ax(nK);
            std::vector<int64_t> face(nK);
            std::vector<float> area(nK), cond(nK), weight(nK), disp(size_t(nK) * 6);
            for (int e = 0; e < nK; ++e)
            {
                const Edge& d = edges[e];
                a[e] = d.a; b[e] = d.b; ax[e] = int8_t(d.axis); face[e] = d.face_index;
                src[e] = d.kind == 0 ? -1 : d.source;
                area[e] = float(d.area); cond[e] = float(d.conductance); weight[e] = float(d.weight);
                const V3 da = sub(d.face, centroid(d.a)), db = sub(d.face, centroid(d.b));
                disp[6 * e] = float(da.x); disp[6 * e + 1] = float(da.y); disp[6 * e + 2] = float(da.z);
                disp[6 * e + 3] = float(db.x); disp[6 * e + 4] = float(db.y); disp[6 * e + 5] = float(db.z);
                sa[e] = special_index[d.a]; sb[e] = special_index[d.b];
                pa[e] = pnode[d.a]; pb[e] = pnode[d.b];
            }
            m.k_a.upload(a); m.k_b.upload(b); m.k_source.upload(src); m.k_axis.upload(ax); m.k_face.upload(face);
            m.k_area.upload(area); m.k_conductance.upload(cond); m.k_weight.upload(weight); m.k_disp.upload(disp);
            m.k_sa.upload(sa); m.k_sb.upload(sb); m.k_pnode_a.upload(pa); m.k_pnode_b.upload(pb);
        }

        // ---- redistribution groups --------------------------------------------------------------
        std::vector<int> group_of(S, -1);
        std::vector<std::vector<int>> groups;
        if (t.retained_count > 0 || minimum_volume_fraction > 0)
        {
            std::vector<int> parent(S);
            std::iota(parent.begin(), parent.end(), 0);
            auto root = [&](int q) { while (parent[q] != q) { parent[q] = parent[parent[q]]; q = parent[q]; } return q; };
            auto unite = [&](int a, int b) { a = root(a); b = root(b); if (a != b) parent[b] = a; };
            std::vector<int> seeds(t.retained_dofs, t.retained_dofs + t.retained_count);
            for (int r = 0; r < t.retained_count; ++r)
            {
                const int q = t.retained_dofs[r];
                if (!active(q)) throw Error(PCFD_INVALID_ARG, "retained pressure root is not an active DOF");
                bool connected = false;
                for (int e = 0; e < t.embedded.count; ++e)
                {
                    if (t.embedded.coarse_dof[e] == q) { unite(q, t.embedded.fine_dof[e]); connected = true; }
                    else if (t.embedded.fine_dof[e] == q) { unite(q, t.embedded.coarse_dof[e]); connected = true; }
                }
                if (!connected) throw Error(PCFD_INVALID_ARG, "retained pressure root has no aperture-connected donor");
            }
            std::map<int, std::array<double, 3>> directional;
            std::map<int, std::pair<double, int>> donor;
            for (int e = 0; e < t.embedded.count; ++e)
            {
                const int ends[2][2] = {{t.embedded.coarse_dof[e], t.embedded.fine_dof[e]}, {t.embedded.fine_dof[e], t.embedded.coarse_dof[e]}};
                for (const auto& end : ends)
                {
                    const int q = end[0];
                    if (q < s.structured || !active(q)) continue;
                    auto& d = directional[q];
                    d[t.embedded.axis[e]] += t.embedded.open_area[e];
                    auto found = donor.find(q);
                    if (found == donor.end()) donor[q] = {0.0, -1};
                    auto& best = donor[q];
                    if (t.embedded.open_area[e] > best.first) best = {t.embedded.open_area[e], end[1]};
                }
            }
            // point location of a fragment centroid: finest active brick containing it
            std::vector<std::map<std::array<int, 3>, int>> lookup(s.levels);
            for (int l = 0; l < s.levels; ++l)
                for (int b = 0; b < t.levels[l].brick_count; ++b)
                    lookup[l][{t.levels[l].coord[3 * b], t.levels[l].coord[3 * b + 1], t.levels[l].coord[3 * b + 2]}] = b;
            auto level_h_at = [&](V3 p) -> double {
                for (int l = s.levels - 1; l >= 0; --l)
                {
                    const double bw = bs * t.levels[l].h;
                    const std::array<int, 3> key{int(std::floor((p.x - t.domain_lo[0]) / bw)), int(std::floor((p.y - t.domain_lo[1]) / bw)),
                                                 int(std::floor((p.z - t.domain_lo[2]) / bw))};
                    auto it = lookup[l].find(key);
                    if (it != lookup[l].end() && brick_active(l, it->second)) return t.levels[l].h;
                }
                throw Error(PCFD_INVALID_ARG, "irregular momentum centroid outside the hierarchy");
            };
            for (const auto& item : directional)
            {
                const int q = item.first;
                const double h = level_h_at(centroid(q)), minimum = minimum_volume_fraction * h * h;
                bool weak = false;
                for (double area : item.second) weak = weak || (area > 0 && area < minimum);
                if (!weak) continue;
                const auto d = donor.find(q);
                if (d == donor.end() || d->second.second < 0) throw Error(PCFD_INVALID_ARG, "directionally weak node has no donor");
                unite(q, d->second.second);
                seeds.push_back(q);
            }
            std::map<int, int> compact;
            for (int seed : seeds)
            {
                const int r = root(seed);
                if (!compact.count(r)) { const int id = int(compact.size()); compact[r] = id; }
            }
            groups.resize(compact.size());
            for (int q = 0; q < S; ++q)
                if (t.active[q])
                {
                    auto found = compact.find(root(q));
                    if (found == compact.end()) continue;
                    group_of[q] = found->second;
                    groups[found->second].push_back(q);
                }
        }

        // ---- wall sides, boundary faces ----------------------------------------------------------
        struct Side { int dof; double coef[3], unit[3], area, distance, disp[3]; };
        std::vector<Side> sides;
        for (int p = 0; p < t.patches.count; ++p)
        {
            const double* n = t.patches.normal + 3 * p;
            const double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            if (!(len > 0) || !(t.patches.area[p] >= 0)) throw Error(PCFD_INVALID_ARG, "invalid surface patch");
            const double unit[3] = {n[0] / len, n[1] / len, n[2] / len};
            const V3 pc{t.patches.centroid[3 * p], t.patches.centroid[3 * p + 1], t.patches.centroid[3 * p + 2]};
            for (int side = 0; side < 2; ++side)
            {
                const int dof = side == 0 ? t.patches.plus_dof[p] : t.patches.minus_dof[p];
                const double sign = side == 0 ? 1.0 : -1.0;
                if (dof < 0 || !active(dof)) continue;
                const V3 d = sub(centroid(dof), pc);
                const double distance = std::abs(d.x * unit[0] + d.y * unit[1] + d.z * unit[2]);
                if (!(distance > std::max(1e-14, std::cbrt(t.volume[dof]) * 1e-10))) throw Error(PCFD_INVALID_ARG, "wall side has zero distance");
                Side sd;
                sd.dof = dof;
                for (int a = 0; a < 3; ++a) { sd.coef[a] = n[a] * (sign * t.patches.area[p]); sd.unit[a] = unit[a]; }
                sd.area = t.patches.area[p];
                sd.distance = distance;
                sd.disp[0] = pc.x - comp(centroid(dof), 0); sd.disp[1] = pc.y - comp(centroid(dof), 1); sd.disp[2] = pc.z - comp(centroid(dof), 2);
                sides.push_back(sd);
            }
        }
        m.nW = int(sides.size());
        std::vector<int> wall_dof, side_node(sides.size());
        {
            std::unordered_map<int, int> node;
            for (size_t q = 0; q < sides.size(); ++q)
            {
                auto ins = node.emplace(sides[q].dof, int(wall_dof.size()));
                if (ins.second) wall_dof.push_back(sides[q].dof);
                side_node[q] = ins.first->second;
            }
        }
        m.nWall = int(wall_dof.size());
        {
            std::vector<int> wd(sides.size()), wp(sides.size()), woff(size_t(m.nWall) + 1, 0), wside(sides.size());
            std::vector<float> wn(sides.size() * 3), wa(sides.size()), wdist(sides.size()), wc(sides.size() * 3), wdisp(sides.size() * 3);
            for (size_t q = 0; q < sides.size(); ++q)
            {
                wd[q] = sides[q].dof; wp[q] = pnode[sides[q].dof];
                for (int a = 0; a < 3; ++a)
                {
                    wn[3 * q + a] = float(sides[q].unit[a]); wc[3 * q + a] = float(sides[q].coef[a]); wdisp[3 * q + a] = float(sides[q].disp[a]);
                }
                wa[q] = float(sides[q].area); wdist[q] = float(sides[q].distance);
                ++woff[side_node[q] + 1];
            }
            for (int n = 0; n < m.nWall; ++n) woff[n + 1] += woff[n];
            std::vector<int> cur = woff;
            for (size_t q = 0; q < sides.size(); ++q) wside[cur[side_node[q]]++] = int(q);
            m.w_dof.upload(wd); m.w_node.upload(side_node); m.w_pnode.upload(wp); m.w_normal.upload(wn); m.w_area.upload(wa);
            m.w_distance.upload(wdist); m.w_coefficient.upload(wc); m.w_disp.upload(wdisp);
            m.w_k.alloc(sides.size()); m.w_force.alloc(sides.size() * 3);
            m.wall_dof.upload(wall_dof); m.wall_offset.upload(woff); m.wall_side.upload(wside);
        }
        m.nB = t.boundary_faces.count;
        {
            std::vector<int> bd(m.nB);
            std::vector<float> bc(size_t(m.nB) * 3);
            for (int f = 0; f < m.nB; ++f)
            {
                bd[f] = t.boundary_faces.dof[f];
                for (int a = 0; a < 3; ++a) bc[3 * f + a] = float(-t.boundary_faces.outward_area[3 * f + a]);
            }
            m.b_dof.upload(bd); m.b_coefficient.upload(bc);
        }

        // ---- deferred DOFs: compact endpoints, specials, group members, wall sides, boundary faces --
        std::vector<uint8_t> deferred(S, 0);
        for (const Edge& e : edges) { deferred[e.a] = 1; deferred[e.b] = 1; }
        for (int q = 0; q < S; ++q) if (special[q] || group_of[q] >= 0 || q >= s.structured) deferred[q] = 1;
        // Structured slots whose control volume absorbed a merged fragment are not h^3: their
        // update must divide by the stored volume, which only the per-DOF pass reads.
        for (int q = 0; q < s.structured; ++q)
        {
            if (!t.active[q]) continue;
            const double h = t.levels[slot_level[q / c3]].h;
            if (float(t.volume[q]) != float(h * h * h)) deferred[q] = 1;
        }
        for (const Side& sd : sides) deferred[sd.dof] = 1;
        for (int f = 0; f < m.nB; ++f) if (active(t.boundary_faces.dof[f])) deferred[t.boundary_faces.dof[f]] = 1;
        std::vector<int> d_of(S, -1), d_dof;
        for (int q = 0; q < S; ++q) if (deferred[q] && t.active[q]) { d_of[q] = int(d_dof.size()); d_dof.push_back(q); }
        m.nD = int(d_dof.size());
        {
            std::vector<std::vector<std::pair<int, int8_t>>> inc(m.nD);
            for (int e = 0; e < m.nK; ++e)
            {
                inc[d_of[edges[e].a]].push_back({e, int8_t(-1)});   // lower endpoint loses the a->b flux
                inc[d_of[edges[e].b]].push_back({e, int8_t(1)});
            }
            std::vector<int> off(size_t(m.nD) + 1, 0), edge, group(m.nD);
            std::vector<int8_t> sign;
            for (int d = 0; d < m.nD; ++d)
            {
                for (auto& pr : inc[d]) { edge.push_back(pr.first); sign.push_back(pr.second); }
                off[d + 1] = int(edge.size());
                group[d] = group_of[d_dof[d]];
            }
            m.d_dof.upload(d_dof); m.d_offset.upload(off); m.d_edge.upload(edge); m.d_sign.upload(sign); m.d_group.upload(group);
            m.d_delta.alloc(size_t(m.nD) * 3);
            // surface sides and boundary faces per deferred DOF
            std::vector<std::vector<int>> ds(m.nD), dbf(m.nD);
            for (size_t q = 0; q < sides.size(); ++q) ds[d_of[sides[q].dof]].push_back(int(q));
            for (int f = 0; f < m.nB; ++f) if (d_of[t.boundary_faces.dof[f]] >= 0) dbf[d_of[t.boundary_faces.dof[f]]].push_back(f);
            std::vector<int> so(size_t(m.nD) + 1, 0), sl, bo(size_t(m.nD) + 1, 0), bl;
            for (int d = 0; d < m.nD; ++d)
            {
                sl.insert(sl.end(), ds[d].begin(), ds[d].end()); so[d + 1] = int(sl.size());
                bl.insert(bl.end(), dbf[d].begin(), dbf[d].end()); bo[d + 1] = int(bl.size());
            }
            m.d_side_offset.upload(so); m.d_side.upload(sl); m.d_boundary_offset.upload(bo); m.d_boundary.upload(bl);
        }
        m.nG = int(groups.size());
        {
            std::vector<int> goff(size_t(m.nG) + 1, 0), gmem;
            std::vector<float> gvol(m.nG, 0.0f);
            for (int g = 0; g < m.nG; ++g)
            {
                for (int q : groups[g]) { gmem.push_back(d_of[q]); gvol[g] += float(t.volume[q]); }
                goff[g + 1] = int(gmem.size());
            }
            m.g_offset.upload(goff); m.g_member.upload(gmem); m.g_volume.upload(gvol);
        }

        // ---- per-DOF arrays ----------------------------------------------------------------------
        std::vector<uint8_t> code(S, 0);
        std::vector<float> vol32(S, 0.0f);
        for (int q = 0; q < S; ++q)
        {
            uint8_t c = uint8_t(t.cut_face_mask[q] & 7u);
            c |= uint8_t((compact_plus[q] & 7u) << CODE_COMPACT_SHIFT);
            if (deferred[q]) c |= CODE_DEFERRED;
            if (t.active[q]) c |= CODE_ACTIVE;
            code[q] = c;
            vol32[q] = float(t.volume[q]);
        }
        m.code.upload(code);
        m.special.upload(special);
        m.volume32.upload(vol32);
        if (t.gradient_node_count)
        {
            const int nnz = t.gradient_offset[t.gradient_node_count];
            std::vector<float> pw(size_t(nnz) * 3);
            for (int q = 0; q < nnz * 3; ++q) pw[q] = float(t.gradient_weight[q]);
            m.p_weight.upload(pw);
            m.p_gradient.alloc(size_t(t.gradient_node_count) * 3);
        }
        // state
        for (DBuf<float>* b : {&m.x, &m.y, &m.z, &m.xn, &m.yn, &m.zn, &m.dx, &m.dy, &m.dz, &m.viscosity, &m.baseline_x, &m.baseline_y, &m.baseline_z})
            b->alloc(size_t(S));
        const int64_t reduce_blocks = (int64_t(s.active_bricks) * c3 + kThreads - 1) / kThreads + (m.nD + kThreads - 1) / kThreads;
        m.reduce_partial.alloc(size_t(2 * reduce_blocks + 16));
        m.reduce_result.alloc(8);
        cuda_check(cudaMallocHost(&m.pinned, 8 * sizeof(float)), "pinned momentum scalars");
        m.ready = true;
    }

    Momentum::~Momentum()
    {
        if (pinned) cudaFreeHost(pinned);
    }
}
