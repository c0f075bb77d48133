// builder.cpp -- host preprocessing that turns a closed wing surface into the static 2:1 brick
// hierarchy and the composite pressure system consumed by pcfd_system_create.
//
// Hierarchy (reference AmrHierarchy, src/core/fluid/amr_grid.cpp:60-361): brick-padded domain,
// per-level refinement of bricks near the wing box, within a surface distance of the triangles
// (exact triangle/box separating-axis test) and in the near wake; 2:1 balance by probing the
// finest owner just outside every brick face; 6 same-level neighbours and boundary/EB flags.
// Brick ids follow the reference's creation order (children in refinement order, slot order
// z,y,x), so brick, neighbour and flag arrays match the reference bit for bit.
//
// Composite system (reference build_composite_amr_pressure_base + finalize_component_gauges +
// finalize_nonorthogonal_pressure_topology, src/core/fluid/amr_pressure.cpp:24-189, 255-301):
// DOF numbering, 2:1 tiles (4 per covered coarse face), outlet-connected components and gauges,
// skew coarse/fine corrections with weighted-least-squares pressure-gradient stencils extended
// ring by ring until full rank.  The solid is represented on the Cartesian cells (a cell whose
// centre lies inside the closed surface is solid; every fluid/solid face becomes a wall patch),
// which stands in for the reference's exact polyhedral cut-cell builder.
#include "pseudoinverse3.h"
#include "../../include/paracfd_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace pcfd_builder
{
    struct V3
    {
        double x = 0, y = 0, z = 0;
        double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
        double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    };
    inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
    inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
    inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
    inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
    inline double length2(V3 a) { return dot(a, a); }

    struct Box
    {
        V3 lo{1e300, 1e300, 1e300}, hi{-1e300, -1e300, -1e300};
        void expand(V3 p)
        {
            lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
            hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
        }
        bool valid() const { return lo.x <= hi.x && lo.y <= hi.y && lo.z <= hi.z; }
        bool overlaps(const Box& b) const
        {
            return lo.x <= b.hi.x && hi.x >= b.lo.x && lo.y <= b.hi.y && hi.y >= b.lo.y && lo.z <= b.hi.z && hi.z >= b.lo.z;
        }
        Box expanded(double d) const { Box b = *this; b.lo = lo - V3{d, d, d}; b.hi = hi + V3{d, d, d}; return b; }
    };

    // ------------------------------------------------------------------ triangle set + BVH
    struct Triangle { V3 a, b, c; };

    // Separating-axis triangle/box overlap (Akenine-Moller): 3 box axes, the triangle normal and
    // the 9 edge x axis cross products.
    bool separated(V3 axis, V3 v0, V3 v1, V3 v2, V3 half)
    {
        const double p0 = dot(axis, v0), p1 = dot(axis, v1), p2 = dot(axis, v2);
        const double r = half.x * std::abs(axis.x) + half.y * std::abs(axis.y) + half.z * std::abs(axis.z);
        return std::min({p0, p1, p2}) > r || std::max({p0, p1, p2}) < -r;
    }
    bool triangle_box(const Triangle& t, const Box& box)
    {
        Box tb;
        tb.expand(t.a); tb.expand(t.b); tb.expand(t.c);
        if (!tb.overlaps(box)) return false;
        const V3 c = (box.lo + box.hi) * 0.5, half = (box.hi - box.lo) * 0.5;
        const V3 v0 = t.a - c, v1 = t.b - c, v2 = t.c - c;
        if (separated({1, 0, 0}, v0, v1, v2, half) || separated({0, 1, 0}, v0, v1, v2, half) || separated({0, 0, 1}, v0, v1, v2, half))
            return false;
        const V3 e[3] = {v1 - v0, v2 - v1, v0 - v2};
        if (separated(cross(e[0], e[1]), v0, v1, v2, half)) return false;
        for (V3 q : e)
            if (separated(cross(q, {1, 0, 0}), v0, v1, v2, half) || separated(cross(q, {0, 1, 0}), v0, v1, v2, half) ||
                separated(cross(q, {0, 0, 1}), v0, v1, v2, half))
                return false;
        return true;
    }

    class Bvh
    {
        struct Node { Box bounds; int left = -1, right = -1, first = 0, count = 0; };
        std::vector<Node> nodes_;
        std::vector<int> order_;
        std::vector<Box> tb_;
        std::vector<V3> centre_;
        const std::vector<Triangle>* tris_ = nullptr;

        int build(int first, int count)
        {
            Node n;
            Box cb;
            for (int q = first; q < first + count; ++q) { n.bounds.expand(tb_[order_[q]].lo); n.bounds.expand(tb_[order_[q]].hi); cb.expand(centre_[order_[q]]); }
            const int id = int(nodes_.size());
            nodes_.push_back(n);
            if (count <= 4) { nodes_[id].first = first; nodes_[id].count = count; return id; }
            const V3 ext = cb.hi - cb.lo;
            int axis = ext.y > ext.x ? 1 : 0;
            if (ext.z > ext[axis]) axis = 2;
            const int mid = first + count / 2;
            std::nth_element(order_.begin() + first, order_.begin() + mid, order_.begin() + first + count,
                             [&](int a, int b) { return centre_[a][axis] < centre_[b][axis]; });
            const int l = build(first, mid - first), r = build(mid, first + count - mid);
            nodes_[id].left = l;
            nodes_[id].right = r;
            return id;
        }

    public:
        explicit Bvh(const std::vector<Triangle>& tris) : tris_(&tris)
        {
            order_.resize(tris.size());
            std::iota(order_.begin(), order_.end(), 0);
            tb_.resize(tris.size());
            centre_.resize(tris.size());
            for (size_t q = 0; q < tris.size(); ++q)
            {
                tb_[q].expand(tris[q].a); tb_[q].expand(tris[q].b); tb_[q].expand(tris[q].c);
                centre_[q] = (tb_[q].lo + tb_[q].hi) * 0.5;
            }
            if (!tris.empty()) build(0, int(tris.size()));
        }
        bool any(const Box& box) const
        {
            if (nodes_.empty() || !box.valid()) return false;
            std::vector<int> stack{0};
            while (!stack.empty())
            {
                const Node& n = nodes_[stack.back()];
                stack.pop_back();
                if (!n.bounds.overlaps(box)) continue;
                if (n.left < 0)
                {
                    for (int q = n.first; q < n.first + n.count; ++q)
                        if (triangle_box((*tris_)[order_[q]], box)) return true;
                }
                else { stack.push_back(n.left); stack.push_back(n.right); }
            }
            return false;
        }
        // Parity of crossings of the +X ray from p (Moller-Trumbore), for inside/outside.
        bool inside(V3 p) const
        {
            if (nodes_.empty()) return false;
            int crossings = 0;
            std::vector<int> stack{0};
            while (!stack.empty())
            {
                const Node& n = nodes_[stack.back()];
                stack.pop_back();
                if (p.y < n.bounds.lo.y || p.y > n.bounds.hi.y || p.z < n.bounds.lo.z || p.z > n.bounds.hi.z || p.x > n.bounds.hi.x) continue;
                if (n.left < 0)
                {
                    for (int q = n.first; q < n.first + n.count; ++q)
                    {
                        const Triangle& t = (*tris_)[order_[q]];
                        const V3 e1 = t.b - t.a, e2 = t.c - t.a, d{1, 0, 0};
                        const V3 pv = cross(d, e2);
                        const double det = dot(e1, pv);
                        if (std::abs(det) < 1e-300) continue;
                        const double inv = 1.0 / det;
                        const V3 tv = p - t.a;
                        const double u = dot(tv, pv) * inv;
                        if (u < 0 || u >= 1) continue;
                        const V3 qv = cross(tv, e1);
                        const double v = dot(d, qv) * inv;
                        if (v < 0 || u + v >= 1) continue;
                        if (dot(e2, qv) * inv > 0) ++crossings;
                    }
                }
                else { stack.push_back(n.left); stack.push_back(n.right); }
            }
            return (crossings & 1) != 0;
        }
    };

    // ------------------------------------------------------------------ hierarchy
    constexpr uint32_t XMIN = 1, XMAX = 2, YMIN = 4, YMAX = 8, ZMIN = 16, ZMAX = 32, EBF = 64, COVERED = 128;

    struct Brick
    {
        int level = 0;
        std::array<int, 3> coord{};
        V3 origin{};
        double h = 0;
        std::array<int, 6> nbr{{-1, -1, -1, -1, -1, -1}};
        int parent = -1;
        std::array<int, 8> children{{-1, -1, -1, -1, -1, -1, -1, -1}};
        uint32_t flags = 0;
        bool active() const { return !(flags & COVERED); }
    };
    struct Level
    {
        double h = 0;
        std::vector<Brick> bricks;
        std::unordered_map<uint64_t, int> lookup;
    };

    inline uint64_t key_of(std::array<int, 3> c)
    {
        return (uint64_t(uint32_t(c[0])) << 42) ^ (uint64_t(uint32_t(c[1])) << 21) ^ uint64_t(uint32_t(c[2]));
    }

    struct Hierarchy
    {
        Box domain;
        int bs = 8, max_levels = 1;
        std::vector<Level> levels;

        int find(int l, std::array<int, 3> c) const
        {
            if (l < 0 || l >= int(levels.size())) return -1;
            auto it = levels[l].lookup.find(key_of(c));
            if (it == levels[l].lookup.end()) return -1;
            return levels[l].bricks[it->second].coord == c ? it->second : -1;
        }
        Box brick_box(const Brick& b) const
        {
            const double w = bs * b.h;
            Box r;
            r.lo = b.origin;
            r.hi = b.origin + V3{w, w, w};
            return r;
        }
        void initialize_base(const Box& req, double h, bool anchor_y_min)
        {
            if (!req.valid() || !(h > 0) || bs <= 0) throw std::invalid_argument("invalid AMR domain/cell/brick size");
            const double bw = h * bs;
            const V3 size = req.hi - req.lo;
            const std::array<int, 3> dims{std::max(1, int(std::ceil(size.x / bw))), std::max(1, int(std::ceil(size.y / bw))),
                                          std::max(1, int(std::ceil(size.z / bw)))};
            const V3 padded{dims[0] * bw, dims[1] * bw, dims[2] * bw};
            const V3 excess = padded - size;
            domain.lo = {req.lo.x, anchor_y_min ? req.lo.y : req.lo.y - 0.5 * excess.y, req.lo.z - 0.5 * excess.z};
            domain.hi = domain.lo + padded;
            levels.assign(max_levels, {});
            for (int l = 0; l < max_levels; ++l) levels[l].h = h / double(1 << l);
            for (int z = 0; z < dims[2]; ++z)
                for (int y = 0; y < dims[1]; ++y)
                    for (int x = 0; x < dims[0]; ++x)
                    {
                        Brick b;
                        b.level = 0;
                        b.coord = {x, y, z};
                        b.h = levels[0].h;
                        b.origin = domain.lo + V3{x * bw, y * bw, z * bw};
                        levels[0].bricks.push_back(b);
                    }
        }
        void rebuild(const Bvh* bvh)
        {
            for (Level& lev : levels)
            {
                lev.lookup.clear();
                lev.lookup.reserve(lev.bricks.size() * 2);
                for (int id = 0; id < int(lev.bricks.size()); ++id)
                {
                    lev.bricks[id].flags &= COVERED;
                    lev.lookup[key_of(lev.bricks[id].coord)] = id;
                }
            }
            for (int l = 0; l < int(levels.size()); ++l)
            {
                Level& lev = levels[l];
                for (Brick& b : lev.bricks)
                {
                    static const int d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
                    for (int q = 0; q < 6; ++q) b.nbr[q] = find(l, {b.coord[0] + d[q][0], b.coord[1] + d[q][1], b.coord[2] + d[q][2]});
                    const double bw = bs * b.h;
                    const V3 bh = b.origin + V3{bw, bw, bw};
                    const double eps = 1e-9 * std::max(1.0, bw);
                    if (std::abs(b.origin.x - domain.lo.x) <= eps) b.flags |= XMIN;
                    if (std::abs(bh.x - domain.hi.x) <= eps) b.flags |= XMAX;
                    if (std::abs(b.origin.y - domain.lo.y) <= eps) b.flags |= YMIN;
                    if (std::abs(bh.y - domain.hi.y) <= eps) b.flags |= YMAX;
                    if (std::abs(b.origin.z - domain.lo.z) <= eps) b.flags |= ZMIN;
                    if (std::abs(bh.z - domain.hi.z) <= eps) b.flags |= ZMAX;
                    if (bvh && bvh->any(brick_box(b))) b.flags |= EBF;
                }
            }
        }
        void refine(int l, int id)
        {
            if (l < 0 || l + 1 >= max_levels || id < 0 || id >= int(levels[l].bricks.size())) return;
            const Brick parent = levels[l].bricks[id];
            if (!parent.active()) return;
            levels[l].bricks[id].flags |= COVERED;
            Level& fine = levels[l + 1];
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx)
                    {
                        const int slot = (dz * 2 + dy) * 2 + dx;
                        const std::array<int, 3> cc{parent.coord[0] * 2 + dx, parent.coord[1] * 2 + dy, parent.coord[2] * 2 + dz};
                        int child = find(l + 1, cc);
                        if (child < 0)
                        {
                            Brick b;
                            b.level = l + 1;
                            b.coord = cc;
                            b.h = fine.h;
                            b.parent = id;
                            const double bw = bs * b.h;
                            b.origin = domain.lo + V3{cc[0] * bw, cc[1] * bw, cc[2] * bw};
                            child = int(fine.bricks.size());
                            fine.bricks.push_back(b);
                            fine.lookup[key_of(cc)] = child;
                        }
                        levels[l].bricks[id].children[slot] = child;
                    }
        }
        bool in_domain(V3 p) const
        {
            return p.x >= domain.lo.x && p.y >= domain.lo.y && p.z >= domain.lo.z && p.x < domain.hi.x && p.y < domain.hi.y && p.z < domain.hi.z;
        }
        // finest active brick containing p: (level, brick, cell i,j,k) or level -1
        std::array<int, 5> locate(V3 p) const
        {
            if (!in_domain(p)) return {-1, -1, 0, 0, 0};
            for (int l = int(levels.size()) - 1; l >= 0; --l)
            {
                const double h = levels[l].h, bw = bs * h;
                const V3 q = p - domain.lo;
                const int id = find(l, {int(std::floor(q.x / bw)), int(std::floor(q.y / bw)), int(std::floor(q.z / bw))});
                if (id < 0 || !levels[l].bricks[id].active()) continue;
                const V3 r = p - levels[l].bricks[id].origin;
                return {l, id, std::clamp(int(std::floor(r.x / h)), 0, bs - 1), std::clamp(int(std::floor(r.y / h)), 0, bs - 1),
                        std::clamp(int(std::floor(r.z / h)), 0, bs - 1)};
            }
            return {-1, -1, 0, 0, 0};
        }
        void balance()
        {
            for (int iteration = 0; iteration < max_levels * 4; ++iteration)
            {
                std::vector<std::pair<int, int>> todo;
                for (int l = 0; l < int(levels.size()); ++l)
                    for (int id = 0; id < int(levels[l].bricks.size()); ++id)
                    {
                        const Brick& b = levels[l].bricks[id];
                        if (!b.active()) continue;
                        const double w = bs * b.h, eps = 1e-7 * w;
                        for (int face = 0; face < 6; ++face)
                            for (double a : {0.25, 0.75})
                                for (double c : {0.25, 0.75})
                                {
                                    V3 p = b.origin + V3{0.5 * w, 0.5 * w, 0.5 * w};
                                    if (face < 2) { p.x = b.origin.x + (face ? w + eps : -eps); p.y = b.origin.y + a * w; p.z = b.origin.z + c * w; }
                                    else if (face < 4) { p.y = b.origin.y + ((face & 1) ? w + eps : -eps); p.x = b.origin.x + a * w; p.z = b.origin.z + c * w; }
                                    else { p.z = b.origin.z + ((face & 1) ? w + eps : -eps); p.x = b.origin.x + a * w; p.y = b.origin.y + c * w; }
                                    const auto n = locate(p);
                                    if (n[0] < 0 || std::abs(n[0] - l) <= 1) continue;
                                    if (n[0] < l) todo.push_back({n[0], n[1]});
                                    else todo.push_back({l, id});
                                }
                    }
                std::sort(todo.begin(), todo.end());
                todo.erase(std::unique(todo.begin(), todo.end()), todo.end());
                if (todo.empty()) break;
                for (auto [l, id] : todo) refine(l, id);
                rebuild(nullptr);
            }
        }
    };

    // ------------------------------------------------------------------ composite system
    struct Connection
    {
        int coarse = -1, fine = -1;
        double area = 0, centre_distance = 0, normal_distance = 0;
        int8_t axis = 0, direction = 1;
        V3 face{};
        double factor = 0;
        int lower_node = -1, upper_node = -1;
        V3 correction{};
        double upper_weight = 0.5;
    };
    struct Patch { double area; V3 centroid, normal; int plus, minus; };

    struct System
    {
        const Hierarchy* H = nullptr;
        int bs = 0, storage = 0;
        bool outlet = true;
        std::vector<int> level_offset;
        std::vector<uint8_t> active, connected, cut;
        std::vector<double> volume;
        std::vector<V3> centroid;
        std::vector<int> aggregate;
        std::vector<Connection> cf;
        std::vector<Patch> patches;
        std::vector<int> grad_dof, grad_offset, grad_neighbour;
        std::vector<V3> grad_weight;
        std::vector<int> gauge_dof;
        std::vector<double> gauge_coefficient;

        int dof(int l, int b, int i, int j, int k) const { return level_offset[l] + b * bs * bs * bs + (k * bs + j) * bs + i; }

        // visit every open same-level face (lower a, upper b) in the reference traversal order
        template <class F> void faces(F&& f) const
        {
            for (int l = 0; l < int(H->levels.size()); ++l)
            {
                const Level& lev = H->levels[l];
                for (int brick = 0; brick < int(lev.bricks.size()); ++brick)
                {
                    const Brick& m = lev.bricks[brick];
                    if (!m.active()) continue;
                    for (int k = 0; k < bs; ++k)
                        for (int j = 0; j < bs; ++j)
                            for (int i = 0; i < bs; ++i)
                            {
                                const int a = dof(l, brick, i, j, k);
                                if (!active[a]) continue;
                                for (int axis = 0; axis < 3; ++axis)
                                {
                                    if (cut[a] & (1u << axis)) continue;
                                    int c[3] = {i, j, k}, b = -1;
                                    if (++c[axis] < bs) b = dof(l, brick, c[0], c[1], c[2]);
                                    else
                                    {
                                        const int n = m.nbr[2 * axis + 1];
                                        if (n >= 0 && lev.bricks[n].active()) { c[axis] = 0; b = dof(l, n, c[0], c[1], c[2]); }
                                    }
                                    f(l, a, b, axis);
                                }
                            }
                }
            }
        }

        int base_aggregate(V3 p) const
        {
            const Level& base = H->levels.front();
            const double bw = bs * base.h;
            const std::array<int, 3> coord{int(std::floor((p.x - H->domain.lo.x) / bw)), int(std::floor((p.y - H->domain.lo.y) / bw)),
                                           int(std::floor((p.z - H->domain.lo.z) / bw))};
            const int brick = H->find(0, coord);
            if (brick < 0) return -1;
            const Brick& m = base.bricks[brick];
            const int local[3] = {std::clamp(int(std::floor((p.x - m.origin.x) / base.h)), 0, bs - 1),
                                  std::clamp(int(std::floor((p.y - m.origin.y) / base.h)), 0, bs - 1),
                                  std::clamp(int(std::floor((p.z - m.origin.z) / base.h)), 0, bs - 1)};
            return dof(0, brick, local[0], local[1], local[2]);
        }
    };

    void build_base(System& s, const Hierarchy& H, const Bvh* solid)
    {
        s.H = &H;
        s.bs = H.bs;
        const int bs = s.bs, c3 = bs * bs * bs;
        s.level_offset.resize(H.levels.size());
        for (int l = 0; l < int(H.levels.size()); ++l)
        {
            s.level_offset[l] = s.storage;
            s.storage += int(H.levels[l].bricks.size()) * c3;
        }
        const int n = s.storage;
        s.active.assign(n, 0);
        s.volume.assign(n, 0.0);
        s.centroid.assign(n, {});
        s.aggregate.assign(n, -1);
        s.cut.assign(n, 0);
        for (int l = 0; l < int(H.levels.size()); ++l)
        {
            const Level& lev = H.levels[l];
            const double cv = double(lev.h) * lev.h * lev.h;
            for (int brick = 0; brick < int(lev.bricks.size()); ++brick)
            {
                if (!lev.bricks[brick].active()) continue;
                const bool near_surface = solid && (lev.bricks[brick].flags & EBF);
                bool brick_inside = false;
                if (solid && !near_surface)
                {
                    const Box b = H.brick_box(lev.bricks[brick]);
                    brick_inside = solid->inside((b.lo + b.hi) * 0.5);
                }
                for (int k = 0; k < bs; ++k)
                    for (int j = 0; j < bs; ++j)
                        for (int i = 0; i < bs; ++i)
                        {
                            const int q = s.dof(l, brick, i, j, k);
                            const V3 point = lev.bricks[brick].origin + V3{(i + 0.5) * lev.h, (j + 0.5) * lev.h, (k + 0.5) * lev.h};
                            const bool inside = solid ? (near_surface ? solid->inside(point) : brick_inside) : false;
                            s.active[q] = inside ? 0 : 1;
                            s.volume[q] = inside ? 0.0 : cv;
                            s.centroid[q] = point;
                            s.aggregate[q] = inside ? -1 : s.base_aggregate(point);
                        }
            }
        }
        // 2:1 tiles, four per coarse face cell, owned by the active coarse brick
        for (int l = 0; l + 1 < int(H.levels.size()); ++l)
        {
            const Level& coarse = H.levels[l];
            const Level& fine = H.levels[l + 1];
            const double hc = coarse.h, hf = fine.h;
            for (int brick = 0; brick < int(coarse.bricks.size()); ++brick)
            {
                const Brick& owner = coarse.bricks[brick];
                if (!owner.active()) continue;
                for (int face = 0; face < 6; ++face)
                {
                    const int cid = owner.nbr[face];
                    if (cid < 0 || coarse.bricks[cid].active()) continue;
                    const Brick& covered = coarse.bricks[cid];
                    const int axis = face / 2;
                    const bool positive = (face & 1) != 0;
                    for (int t1 = 0; t1 < bs; ++t1)
                        for (int t0 = 0; t0 < bs; ++t0)
                            for (int s1 = 0; s1 < 2; ++s1)
                                for (int s0 = 0; s0 < 2; ++s0)
                                {
                                    int ci = t0, cj = t1, ck = 0;
                                    if (axis == 0) { ci = positive ? bs - 1 : 0; cj = t0; ck = t1; }
                                    else if (axis == 1) { ci = t0; cj = positive ? bs - 1 : 0; ck = t1; }
                                    else { ci = t0; cj = t1; ck = positive ? bs - 1 : 0; }
                                    int pfi, pfj, pfk;
                                    if (axis == 0) { pfi = positive ? 0 : 2 * bs - 1; pfj = 2 * t0 + s0; pfk = 2 * t1 + s1; }
                                    else if (axis == 1) { pfi = 2 * t0 + s0; pfj = positive ? 0 : 2 * bs - 1; pfk = 2 * t1 + s1; }
                                    else { pfi = 2 * t0 + s0; pfj = 2 * t1 + s1; pfk = positive ? 0 : 2 * bs - 1; }
                                    const int slot = ((pfk / bs) * 2 + pfj / bs) * 2 + pfi / bs;
                                    const int child = covered.children[slot];
                                    if (child < 0 || !fine.bricks[child].active()) throw std::runtime_error("2:1 interface has missing or covered fine child");
                                    const int fi = pfi % bs, fj = pfj % bs, fk = pfk % bs, fc = axis == 0 ? fi : (axis == 1 ? fj : fk);
                                    V3 face_centroid = fine.bricks[child].origin + V3{(fi + 0.5) * hf, (fj + 0.5) * hf, (fk + 0.5) * hf};
                                    face_centroid[axis] = fine.bricks[child].origin[axis] + (fc + (positive ? 0 : 1)) * hf;
                                    const double cd = 0.5 * hc + 0.5 * hf;
                                    Connection e;
                                    e.coarse = s.dof(l, brick, ci, cj, ck);
                                    e.fine = s.dof(l + 1, child, fi, fj, fk);
                                    e.area = hf * hf;
                                    e.centre_distance = cd;
                                    e.normal_distance = cd;
                                    e.axis = int8_t(axis);
                                    e.direction = int8_t(positive ? 1 : -1);
                                    e.face = face_centroid;
                                    if (!solid || (s.active[e.coarse] && s.active[e.fine])) s.cf.push_back(e);
                                    else if (s.active[e.coarse] != s.active[e.fine])
                                    {
                                        // a 2:1 tile between fluid and solid is a wall for the fluid side
                                        const int fluid = s.active[e.coarse] ? e.coarse : e.fine;
                                        V3 normal{};
                                        // +axis points from the lower to the upper side; the coarse cell is
                                        // the lower side when the covered brick is on its positive face
                                        const bool fluid_is_lower = (fluid == e.coarse) == positive;
                                        normal[axis] = fluid_is_lower ? -1.0 : 1.0;
                                        s.patches.push_back({hf * hf, face_centroid, normal, fluid, -1});
                                    }
                                }
                }
            }
        }
        // wall patches on every fluid/solid Cartesian face (normal from the solid into the fluid)
        if (solid)
            for (int l = 0; l < int(H.levels.size()); ++l)
            {
                const Level& lev = H.levels[l];
                for (int brick = 0; brick < int(lev.bricks.size()); ++brick)
                {
                    const Brick& m = lev.bricks[brick];
                    if (!m.active()) continue;
                    for (int k = 0; k < bs; ++k)
                        for (int j = 0; j < bs; ++j)
                            for (int i = 0; i < bs; ++i)
                            {
                                const int a = s.dof(l, brick, i, j, k);
                                for (int axis = 0; axis < 3; ++axis)
                                {
                                    int c[3] = {i, j, k}, b = -1;
                                    if (++c[axis] < bs) b = s.dof(l, brick, c[0], c[1], c[2]);
                                    else
                                    {
                                        const int nb = m.nbr[2 * axis + 1];
                                        if (nb >= 0 && lev.bricks[nb].active()) { c[axis] = 0; b = s.dof(l, nb, c[0], c[1], c[2]); }
                                    }
                                    if (b < 0 || s.active[a] == s.active[b]) continue;
                                    V3 centre = m.origin + V3{(i + 0.5) * lev.h, (j + 0.5) * lev.h, (k + 0.5) * lev.h};
                                    centre[axis] += 0.5 * lev.h;
                                    V3 normal{};
                                    normal[axis] = s.active[b] ? 1.0 : -1.0;   // into the fluid cell
                                    s.patches.push_back({lev.h * lev.h, centre, normal, s.active[b] ? b : a, -1});
                                }
                            }
                }
            }
    }

    void finalize_gauges(System& s)
    {
        const int n = s.storage, bs = s.bs;
        s.connected.assign(n, 0);
        s.gauge_dof.clear();
        s.gauge_coefficient.clear();
        if (!s.outlet) { for (int q = 0; q < n; ++q) s.connected[q] = s.active[q]; return; }
        std::vector<int> parent(n, -1);
        for (int q = 0; q < n; ++q) if (s.active[q]) parent[q] = q;
        auto root = [&](int q) { while (parent[q] != q) { parent[q] = parent[parent[q]]; q = parent[q]; } return q; };
        auto join = [&](int a, int b) {
            if (a < 0 || b < 0 || !s.active[a] || !s.active[b]) return;
            a = root(a); b = root(b);
            if (a != b) parent[std::max(a, b)] = std::min(a, b);
        };
        s.faces([&](int, int a, int b, int) { join(a, b); });
        for (const Connection& e : s.cf) join(e.coarse, e.fine);
        std::vector<uint8_t> outlet_root(n, 0), external_root(n, 0);
        for (int l = 0; l < int(s.H->levels.size()); ++l)
        {
            const Level& lev = s.H->levels[l];
            for (int brick = 0; brick < int(lev.bricks.size()); ++brick)
            {
                const Brick& m = lev.bricks[brick];
                if (!m.active()) continue;
                for (int k = 0; k < bs; ++k)
                    for (int j = 0; j < bs; ++j)
                    {
                        if (m.flags & XMIN) { const int q = s.dof(l, brick, 0, j, k); if (s.active[q]) external_root[root(q)] = 1; }
                        if (m.flags & XMAX) { const int q = s.dof(l, brick, bs - 1, j, k); if (s.active[q]) outlet_root[root(q)] = external_root[root(q)] = 1; }
                    }
            }
        }
        std::vector<uint8_t> emitted(n, 0);
        for (int q = 0; q < n; ++q)
            if (s.active[q])
            {
                const int r = root(q);
                s.connected[q] = external_root[r];
                if (!outlet_root[r] && !emitted[r])
                {
                    emitted[r] = 1;
                    s.gauge_dof.push_back(q);
                    s.gauge_coefficient.push_back(std::max(1e-12, std::cbrt(std::max(0.0, s.volume[q]))));
                }
            }
    }

    void finalize_nonorthogonal(System& s)
    {
        const double resolution = 16.0 * double(std::numeric_limits<float>::epsilon());
        for (Connection& e : s.cf)
        {
            if (e.coarse == e.fine || !(e.area > 0)) throw std::runtime_error("invalid compact pressure connection");
            const int lower = e.direction > 0 ? e.coarse : e.fine, upper = e.direction > 0 ? e.fine : e.coarse;
            const V3 d = s.centroid[upper] - s.centroid[lower];
            const double d2 = length2(d), signed_nd = d[e.axis];
            if (!(d2 > 0)) throw std::runtime_error("invalid compact pressure centroid displacement");
            const double distance = std::sqrt(d2), eps = 1e-10 * std::max(distance, 1e-12);
            const double lf = e.face[e.axis] - s.centroid[lower][e.axis], uf = s.centroid[upper][e.axis] - e.face[e.axis];
            if (!(signed_nd > 2 * eps && lf > eps && uf > eps)) throw std::runtime_error("compact pressure face is not bracketed by its centroids");
            e.centre_distance = distance;
            e.normal_distance = signed_nd;
            e.factor = 1.0 / signed_nd;
            V3 normal{};
            normal[e.axis] = 1;
            e.correction = normal - d * e.factor;
            const double m2 = length2(e.correction);
            if (m2 > 0 && m2 <= resolution * resolution) e.correction = {};
            e.upper_weight = lf / (lf + uf);
            e.lower_node = e.upper_node = -1;
        }
        // Cartesian cell centres are aligned across same-level faces: no regular corrections.
        std::unordered_map<int, int> node;
        s.grad_dof.clear();
        auto reg = [&](int dof) { if (node.emplace(dof, int(node.size())).second) s.grad_dof.push_back(dof); };
        for (const Connection& e : s.cf)
        {
            if (length2(e.correction) <= 1e-24) continue;
            const int lower = e.direction > 0 ? e.coarse : e.fine, upper = e.direction > 0 ? e.fine : e.coarse;
            reg(lower);
            reg(upper);
        }
        for (const Patch& p : s.patches)
            for (int dof : {p.plus, p.minus})
                if (dof >= 0 && s.active[dof]) reg(dof);
        struct Sample { int neighbour; double weight; };
        std::vector<std::vector<Sample>> samples(s.grad_dof.size());
        auto add_sample = [&](int endpoint, int nb, double area) {
            auto f = node.find(endpoint);
            if (f == node.end() || nb < 0 || nb >= s.storage || !s.active[nb] || endpoint == nb) return;
            const V3 d = s.centroid[nb] - s.centroid[endpoint];
            const double d2 = length2(d);
            if (d2 > 1e-24 && area > 0) samples[f->second].push_back({nb, area / d2});
        };
        s.faces([&](int l, int a, int b, int) {
            if (b >= 0 && s.active[b])
            {
                const double area = s.H->levels[l].h * s.H->levels[l].h;
                add_sample(a, b, area);
                add_sample(b, a, area);
            }
        });
        for (const Connection& e : s.cf) { add_sample(e.coarse, e.fine, e.area); add_sample(e.fine, e.coarse, e.area); }
        auto rank_of = [&](int n, double* inverse) {
            const int centre = s.grad_dof[n];
            double m[9] = {};
            for (const Sample& q : samples[n])
            {
                const V3 d = s.centroid[q.neighbour] - s.centroid[centre];
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) m[r * 3 + c] += q.weight * d[r] * d[c];
            }
            double local[9];
            return pcfd::pseudoinverse3(m, inverse ? inverse : local, 20, 1e-4);
        };
        auto extend = [&](const std::vector<int>& deficient) {
            struct Src { int node; double path_area; };
            std::unordered_map<int, std::vector<Src>> sources;
            for (int n : deficient)
            {
                const int centre = s.grad_dof[n];
                for (const Sample& q : samples[n])
                    sources[q.neighbour].push_back({n, q.weight * length2(s.centroid[q.neighbour] - s.centroid[centre])});
            }
            std::vector<std::vector<Sample>> add(samples.size());
            auto propose = [&](int middle, int other, double area) {
                const auto f = sources.find(middle);
                if (f == sources.end()) return;
                for (const Src& src : f->second)
                {
                    const int centre = s.grad_dof[src.node];
                    if (other == centre) continue;
                    bool present = false;
                    for (const Sample& q : samples[src.node]) if (q.neighbour == other) { present = true; break; }
                    if (present) continue;
                    const double d2 = length2(s.centroid[other] - s.centroid[centre]);
                    if (!(d2 > 1e-24)) continue;
                    const double w = std::min(src.path_area, area) / d2;
                    auto& cand = add[src.node];
                    auto dup = std::find_if(cand.begin(), cand.end(), [&](const Sample& v) { return v.neighbour == other; });
                    if (dup == cand.end()) cand.push_back({other, w});
                    else dup->weight = std::max(dup->weight, w);
                }
            };
            s.faces([&](int l, int a, int b, int) {
                if (b >= 0 && s.active[b])
                {
                    const double area = s.H->levels[l].h * s.H->levels[l].h;
                    propose(a, b, area);
                    propose(b, a, area);
                }
            });
            for (const Connection& e : s.cf) { propose(e.coarse, e.fine, e.area); propose(e.fine, e.coarse, e.area); }
            for (int n : deficient)
            {
                auto& cand = add[n];
                std::sort(cand.begin(), cand.end(), [](const Sample& a, const Sample& b) { return a.neighbour < b.neighbour; });
                samples[n].insert(samples[n].end(), cand.begin(), cand.end());
            }
        };
        std::vector<int> deficient;
        for (int n = 0; n < int(samples.size()); ++n) if (rank_of(n, nullptr) < 3) deficient.push_back(n);
        for (int ring = 2; ring <= 3 && !deficient.empty(); ++ring)
        {
            extend(deficient);
            if (ring < 3)
            {
                std::vector<int> remaining;
                for (int n : deficient) if (rank_of(n, nullptr) < 3) remaining.push_back(n);
                deficient = std::move(remaining);
            }
        }
        deficient.clear();
        for (int n = 0; n < int(samples.size()); ++n) if (rank_of(n, nullptr) == 2) deficient.push_back(n);
        extend(deficient);
        s.grad_offset.assign(1, 0);
        s.grad_neighbour.clear();
        s.grad_weight.clear();
        for (int n = 0; n < int(s.grad_dof.size()); ++n)
        {
            const int centre = s.grad_dof[n];
            double inverse[9];
            rank_of(n, inverse);
            for (const Sample& q : samples[n])
            {
                const V3 d = s.centroid[q.neighbour] - s.centroid[centre];
                V3 w{};
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) w[r] += inverse[r * 3 + c] * q.weight * d[c];
                s.grad_neighbour.push_back(q.neighbour);
                s.grad_weight.push_back(w);
            }
            s.grad_offset.push_back(int(s.grad_neighbour.size()));
        }
        for (Connection& e : s.cf)
        {
            if (length2(e.correction) <= 1e-24) continue;
            const int lower = e.direction > 0 ? e.coarse : e.fine, upper = e.direction > 0 ? e.fine : e.coarse;
            e.lower_node = node.at(lower);
            e.upper_node = node.at(upper);
        }
    }
}

// ------------------------------------------------------------------ C ABI
struct pcfd_built_topology
{
    pcfd_builder::Hierarchy H;
    pcfd_builder::System S;
    pcfd_topology view{};
    std::vector<pcfd_level> levels;
    std::vector<std::vector<int32_t>> coord, nbr, children;
    std::vector<std::vector<double>> origin;
    std::vector<std::vector<uint32_t>> flags;
    std::vector<double> centroid, cf_area, cf_centre, cf_normal, cf_face, cf_factor, cf_corr, cf_weight, grad_w, gauge_c;
    std::vector<int32_t> cf_coarse, cf_fine, cf_ln, cf_un;
    std::vector<int8_t> cf_axis, cf_dir;
    std::vector<double> p_area, p_centroid, p_normal;
    std::vector<int32_t> p_plus, p_minus;
    std::string error;
};

namespace
{
    thread_local std::string g_builder_error;
}

extern "C" const char* pcfd_builder_last_error(void) { return g_builder_error.c_str(); }

extern "C" pcfd_status pcfd_topology_build(const pcfd_mesh* mesh, const pcfd_amr_config* cfg, int32_t solid,
                                           pcfd_built_topology** out, pcfd_topology* view)
{
    using namespace pcfd_builder;
    try
    {
        if (!mesh || !cfg || !out || !view) throw std::invalid_argument("null argument");
        if (cfg->brick_size <= 0 || cfg->brick_size > 32 || cfg->max_levels <= 0 || !(cfg->base_cell_size > 0))
            throw std::invalid_argument("invalid AMR configuration");
        auto t = std::make_unique<pcfd_built_topology>();
        std::vector<Triangle> tris(size_t(mesh->triangle_count));
        Box wing;
        for (int64_t q = 0; q < mesh->triangle_count; ++q)
        {
            V3 p[3];
            for (int c = 0; c < 3; ++c)
            {
                const uint32_t v = mesh->indices[3 * q + c];
                if (int64_t(v) >= mesh->vertex_count) throw std::invalid_argument("triangle index out of range");
                p[c] = {mesh->positions[3 * v], mesh->positions[3 * v + 1], mesh->positions[3 * v + 2]};
            }
            tris[q] = {p[0], p[1], p[2]};
        }
        // wing bounding box in FP32 coordinates, as the reference's display mesh stores it
        for (int64_t v = 0; v < mesh->vertex_count; ++v)
            wing.expand({double(float(mesh->positions[3 * v])), double(float(mesh->positions[3 * v + 1])), double(float(mesh->positions[3 * v + 2]))});
        Bvh bvh(tris);
        Hierarchy& H = t->H;
        H.bs = cfg->brick_size;
        H.max_levels = cfg->max_levels;
        Box req;
        req.lo = {cfg->domain_lo[0], cfg->domain_lo[1], cfg->domain_lo[2]};
        req.hi = {cfg->domain_hi[0], cfg->domain_hi[1], cfg->domain_hi[2]};
        H.initialize_base(req, cfg->base_cell_size, cfg->anchor_y_min != 0);
        H.rebuild(&bvh);
        const V3 wc = (wing.lo + wing.hi) * 0.5;
        Box wake;
        wake.lo = {wing.hi.x, wc.y - cfg->wake_radius, wc.z - cfg->wake_radius};
        wake.hi = {wing.hi.x + cfg->wake_length, wc.y + cfg->wake_radius, wc.z + cfg->wake_radius};
        for (int l = 0; l + 1 < H.max_levels; ++l)
        {
            const size_t count = H.levels[l].bricks.size();
            std::vector<uint8_t> refine(count, 0);
            for (size_t id = 0; id < count; ++id)
            {
                const Brick& b = H.levels[l].bricks[id];
                if (!b.active()) continue;
                const Box bb = H.brick_box(b);
                const bool wing_region = l == 0 && bb.overlaps(wing.expanded(cfg->wing_refinement_distance));
                const bool surface_region = bvh.any(bb.expanded(cfg->surface_refinement_distance));
                const bool wake_region = l + 1 < H.max_levels - 1 && bb.overlaps(wake);
                refine[id] = uint8_t(wing_region || surface_region || wake_region);
            }
            for (size_t id = 0; id < count; ++id) if (refine[id]) H.refine(l, int(id));
            H.rebuild(&bvh);
        }
        H.balance();
        H.rebuild(&bvh);

        System& S = t->S;
        S.outlet = true;
        build_base(S, H, solid ? &bvh : nullptr);
        finalize_gauges(S);
        finalize_nonorthogonal(S);

        // ---- flat view -----------------------------------------------------------------
        const int L = int(H.levels.size());
        t->levels.resize(L);
        t->coord.resize(L); t->nbr.resize(L); t->children.resize(L); t->origin.resize(L); t->flags.resize(L);
        for (int l = 0; l < L; ++l)
        {
            for (const Brick& b : H.levels[l].bricks)
            {
                t->coord[l].insert(t->coord[l].end(), {b.coord[0], b.coord[1], b.coord[2]});
                t->origin[l].insert(t->origin[l].end(), {b.origin.x, b.origin.y, b.origin.z});
                t->nbr[l].insert(t->nbr[l].end(), b.nbr.begin(), b.nbr.end());
                t->children[l].insert(t->children[l].end(), b.children.begin(), b.children.end());
                t->flags[l].push_back(b.flags);
            }
            pcfd_level& v = t->levels[l];
            v.h = H.levels[l].h;
            v.brick_count = int32_t(H.levels[l].bricks.size());
            v.level_offset = S.level_offset[l];
            v.coord = t->coord[l].data(); v.origin = t->origin[l].data(); v.neighbors = t->nbr[l].data();
            v.flags = t->flags[l].data(); v.children = t->children[l].data();
        }
        for (const V3& c : S.centroid) t->centroid.insert(t->centroid.end(), {c.x, c.y, c.z});
        for (const Connection& e : S.cf)
        {
            t->cf_coarse.push_back(e.coarse); t->cf_fine.push_back(e.fine); t->cf_area.push_back(e.area);
            t->cf_centre.push_back(e.centre_distance); t->cf_normal.push_back(e.normal_distance);
            t->cf_axis.push_back(e.axis); t->cf_dir.push_back(e.direction);
            t->cf_face.insert(t->cf_face.end(), {e.face.x, e.face.y, e.face.z});
            t->cf_factor.push_back(e.factor); t->cf_ln.push_back(e.lower_node); t->cf_un.push_back(e.upper_node);
            t->cf_corr.insert(t->cf_corr.end(), {e.correction.x, e.correction.y, e.correction.z});
            t->cf_weight.push_back(e.upper_weight);
        }
        for (const V3& w : S.grad_weight) t->grad_w.insert(t->grad_w.end(), {w.x, w.y, w.z});
        for (const Patch& p : S.patches)
        {
            t->p_area.push_back(p.area);
            t->p_centroid.insert(t->p_centroid.end(), {p.centroid.x, p.centroid.y, p.centroid.z});
            t->p_normal.insert(t->p_normal.end(), {p.normal.x, p.normal.y, p.normal.z});
            t->p_plus.push_back(p.plus); t->p_minus.push_back(p.minus);
        }
        pcfd_topology& o = t->view;
        std::memset(&o, 0, sizeof(o));
        o.brick_size = H.bs;
        o.level_count = L;
        o.levels = t->levels.data();
        for (int a = 0; a < 3; ++a) { o.domain_lo[a] = H.domain.lo[a]; o.domain_hi[a] = H.domain.hi[a]; }
        o.storage_size = S.storage;
        o.pressure_outlet_xmax = 1;
        o.active = S.active.data();
        o.freestream_connected = S.connected.data();
        o.cut_face_mask = S.cut.data();
        o.volume = S.volume.data();
        o.centroid = t->centroid.data();
        o.preconditioner_aggregate = S.aggregate.data();
        pcfd_connections& c = o.coarse_fine;
        c.count = int32_t(S.cf.size());
        c.coarse_dof = t->cf_coarse.data(); c.fine_dof = t->cf_fine.data(); c.open_area = t->cf_area.data();
        c.centre_distance = t->cf_centre.data(); c.normal_distance = t->cf_normal.data(); c.axis = t->cf_axis.data();
        c.direction = t->cf_dir.data(); c.face_centroid = t->cf_face.data(); c.orthogonal_gradient_factor = t->cf_factor.data();
        c.lower_gradient_node = t->cf_ln.data(); c.upper_gradient_node = t->cf_un.data();
        c.nonorthogonal_correction = t->cf_corr.data(); c.upper_gradient_weight = t->cf_weight.data();
        o.gradient_node_count = int32_t(S.grad_dof.size());
        o.gradient_dof = S.grad_dof.data();
        o.gradient_offset = S.grad_offset.data();
        o.gradient_neighbour = S.grad_neighbour.data();
        o.gradient_weight = t->grad_w.data();
        o.gauge_count = int32_t(S.gauge_dof.size());
        o.gauge_dof = S.gauge_dof.data();
        o.gauge_coefficient = S.gauge_coefficient.data();
        o.patches.count = int32_t(S.patches.size());
        o.patches.area = t->p_area.data(); o.patches.centroid = t->p_centroid.data(); o.patches.normal = t->p_normal.data();
        o.patches.plus_dof = t->p_plus.data(); o.patches.minus_dof = t->p_minus.data();
        *view = o;
        *out = t.release();
        return PCFD_OK;
    }
    catch (const std::invalid_argument& e) { g_builder_error = e.what(); return PCFD_INVALID_ARG; }
    catch (const std::exception& e) { g_builder_error = e.what(); return PCFD_TOPOLOGY_UNRESOLVED; }
}

extern "C" void pcfd_topology_free(pcfd_built_topology* t) { delete t; }
