// capi.cu -- the extern "C" boundary (include/paracfd_b200.h): topology validation and upload,
// resident state transfer, and the projection entry points.  Every entry point converts C++
// exceptions into a status code plus a thread-local message; no exception crosses the ABI.
#include "momentum.h"

#include <cmath>
#include <cstring>
#include <limits>
#include <memory>

namespace pcfd
{
    namespace
    {
        thread_local std::string g_error;

        template <class F> pcfd_status guarded(F&& f)
        {
            try
            {
                f();
                return PCFD_OK;
            }
            catch (const Error& e) { g_error = e.what(); return e.status; }
            catch (const std::bad_alloc&) { g_error = "host allocation failed"; return PCFD_OUT_OF_MEMORY; }
            catch (const std::exception& e) { g_error = e.what(); return PCFD_INTERNAL; }
            catch (...) { g_error = "unknown failure"; return PCFD_INTERNAL; }
        }

        // diagonal_cpu semantics (reference amr_pressure.cpp:525-543), host FP64.
        std::vector<double> host_diagonal(const pcfd_topology& t)
        {
            const int bs = t.brick_size, c3 = bs * bs * bs;
            std::vector<double> d(size_t(t.storage_size), 0.0);
            auto add = [&](int a, int b, double c) {
                if (a < 0 || b < 0 || a == b || !t.active[a] || !t.active[b]) return;
                d[a] += c;
                d[b] += c;
            };
            for (int l = 0; l < t.level_count; ++l)
            {
                const pcfd_level& lev = t.levels[l];
                for (int brick = 0; brick < lev.brick_count; ++brick)
                {
                    if (lev.flags[brick] & PCFD_BRICK_COVERED) continue;
                    for (int k = 0; k < bs; ++k)
                        for (int j = 0; j < bs; ++j)
                            for (int i = 0; i < bs; ++i)
                            {
                                const int a = lev.level_offset + brick * c3 + (k * bs + j) * bs + i;
                                if (!t.active[a]) continue;
                                for (int axis = 0; axis < 3; ++axis)
                                {
                                    if (t.cut_face_mask[a] & (1u << axis)) continue;
                                    int c[3] = {i, j, k};
                                    ++c[axis];
                                    if (c[axis] < bs) add(a, lev.level_offset + brick * c3 + (c[2] * bs + c[1]) * bs + c[0], lev.h);
                                    else
                                    {
                                        const int nb = lev.neighbors[brick * 6 + 2 * axis + 1];
                                        if (nb >= 0 && !(lev.flags[nb] & PCFD_BRICK_COVERED))
                                        {
                                            c[axis] = 0;
                                            add(a, lev.level_offset + nb * c3 + (c[2] * bs + c[1]) * bs + c[0], lev.h);
                                        }
                                    }
                                }
                                if (t.pressure_outlet_xmax && (lev.flags[brick] & PCFD_BRICK_XMAX) && i == bs - 1) d[a] += 2.0 * lev.h;
                            }
                }
            }
            auto factor = [](const pcfd_connections& c, int e) {
                const double f = c.orthogonal_gradient_factor[e];
                return f > 0 ? f : (c.normal_distance[e] > 0 ? 1.0 / c.normal_distance[e] : 0.0);
            };
            for (int e = 0; e < t.coarse_fine.count; ++e)
                add(t.coarse_fine.coarse_dof[e], t.coarse_fine.fine_dof[e], t.coarse_fine.open_area[e] * factor(t.coarse_fine, e));
            for (int e = 0; e < t.embedded.count; ++e)
                add(t.embedded.coarse_dof[e], t.embedded.fine_dof[e], t.embedded.open_area[e] * factor(t.embedded, e));
            for (int e = 0; e < t.regular.count; ++e)
                add(t.regular.lower_dof[e], t.regular.upper_dof[e], t.regular.open_area[e] * t.regular.two_point_delta[e]);
            for (int g = 0; g < t.gauge_count; ++g)
                if (t.gauge_dof[g] >= 0 && t.active[t.gauge_dof[g]]) d[t.gauge_dof[g]] += t.gauge_coefficient[g];
            return d;
        }

        void validate(const pcfd_topology& t)
        {
            require(t.brick_size > 0 && t.brick_size <= 32, "brick_size must be in 1..32");
            require(t.level_count > 0 && t.levels, "topology needs at least one level");
            require(t.storage_size > 0 && t.active && t.cut_face_mask && t.volume && t.preconditioner_aggregate,
                    "topology per-DOF arrays missing");
            const int64_t c3 = int64_t(t.brick_size) * t.brick_size * t.brick_size;
            int64_t expected = 0;
            for (int l = 0; l < t.level_count; ++l)
            {
                const pcfd_level& lev = t.levels[l];
                require(lev.level_offset == expected, "level_offset does not follow brick order");
                require(lev.h > 0 && std::isfinite(lev.h), "level cell size must be positive");
                require(lev.brick_count >= 0 && (lev.brick_count == 0 || (lev.neighbors && lev.flags && lev.coord)),
                        "level brick arrays missing");
                for (int b = 0; b < lev.brick_count * 6; ++b)
                    require(lev.neighbors[b] >= -1 && lev.neighbors[b] < lev.brick_count, "brick neighbour out of range");
                expected += int64_t(lev.brick_count) * c3;
            }
            require(expected <= t.storage_size, "storage_size smaller than the brick slots");
            require(t.storage_size < (int64_t(1) << 31), "storage_size exceeds 32-bit DOF indexing");
            auto check_conn = [&](const pcfd_connections& c, const char* what) {
                for (int e = 0; e < c.count; ++e)
                    require(c.coarse_dof[e] >= 0 && c.coarse_dof[e] < t.storage_size && c.fine_dof[e] >= 0 &&
                                c.fine_dof[e] < t.storage_size && c.axis[e] >= 0 && c.axis[e] < 3,
                            std::string("invalid ") + what + " connection");
            };
            check_conn(t.coarse_fine, "coarse/fine");
            check_conn(t.embedded, "embedded");
            for (int e = 0; e < t.regular.count; ++e)
                require(t.regular.lower_dof[e] >= 0 && t.regular.lower_dof[e] < t.storage_size && t.regular.upper_dof[e] >= 0 &&
                            t.regular.upper_dof[e] < t.storage_size && t.regular.level[e] >= 0 && t.regular.level[e] < t.level_count,
                        "invalid regular correction");
            for (int q = 0; q < t.gradient_node_count; ++q)
                require(t.gradient_dof[q] >= 0 && t.gradient_dof[q] < t.storage_size, "invalid gradient node");
            if (t.gradient_node_count)
                for (int q = 0; q < t.gradient_offset[t.gradient_node_count]; ++q)
                    require(t.gradient_neighbour[q] >= 0 && t.gradient_neighbour[q] < t.storage_size, "invalid gradient neighbour");
            for (int g = 0; g < t.gauge_count; ++g)
                require(t.gauge_dof[g] >= 0 && t.gauge_dof[g] < t.storage_size, "invalid gauge");
        }

        void create(const pcfd_topology& t, const pcfd_options* options, System& s)
        {
            validate(t);
            s.device = options ? options->device : 0;
            s.mg_precision = options ? options->mg_precision : PCFD_MG_FP64;
            cuda_check(cudaSetDevice(s.device), "cudaSetDevice");
            if (options && options->stream) s.stream = static_cast<cudaStream_t>(options->stream);
            else
            {
                cuda_check(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "create stream");
                s.own_stream = true;
            }
            s.bs = t.brick_size;
            s.bs3 = s.bs * s.bs * s.bs;
            s.levels = t.level_count;
            s.S = t.storage_size;
            s.Sp = (s.S + 63) & ~63;
            s.outlet = t.pressure_outlet_xmax != 0;
            s.full_nonorthogonal = t.gradient_node_count > 0;
            // brick slots
            std::vector<int> brick_level, nbr, active_list;
            std::vector<uint32_t> flags;
            s.level_h.resize(s.levels);
            s.level_slot0.resize(s.levels);
            int slot0 = 0;
            for (int l = 0; l < s.levels; ++l)
            {
                const pcfd_level& lev = t.levels[l];
                s.level_h[l] = lev.h;
                s.level_slot0[l] = slot0;
                for (int b = 0; b < lev.brick_count; ++b)
                {
                    brick_level.push_back(l);
                    flags.push_back(lev.flags[b]);
                    for (int f = 0; f < 6; ++f)
                    {
                        const int n = lev.neighbors[b * 6 + f];
                        nbr.push_back(n >= 0 && !(lev.flags[n] & PCFD_BRICK_COVERED) ? slot0 + n : -1);
                    }
                    if (!(lev.flags[b] & PCFD_BRICK_COVERED)) active_list.push_back(slot0 + b);
                }
                slot0 += lev.brick_count;
            }
            s.B = slot0;
            s.structured = s.B * s.bs3;
            s.faces = int64_t(s.B) * (s.bs + 1) * s.bs * s.bs;
            s.active_bricks = int(active_list.size());
            s.brick_level.upload(brick_level);
            s.brick_nbr.upload(nbr);
            s.brick_flags.upload(flags);
            s.active_brick_list.upload(active_list);
            std::vector<int> inflow_slot(size_t(s.B), -1);
            int inflow_bricks = 0;
            for (const int slot : active_list)
                if (flags[slot] & PCFD_BRICK_XMIN) inflow_slot[slot] = inflow_bricks++;
            s.inflow_faces = inflow_bricks * s.bs * s.bs;
            s.inflow_slot_of_brick.upload(inflow_slot);
            s.inflow.alloc(size_t(s.inflow_faces));
            s.d_level_h.upload(s.level_h);
            // per DOF
            s.h_active.assign(t.active, t.active + s.S);
            s.h_volume.assign(t.volume, t.volume + s.S);
            {
                std::vector<uint8_t> padded(s.h_active);
                padded.resize(size_t(s.Sp), 0);
                s.active.upload(padded);
            }
            s.cut_face_mask.upload(std::vector<uint8_t>(t.cut_face_mask, t.cut_face_mask + s.S));
            s.volume.upload(s.h_volume);
            s.aggregate.upload(std::vector<int>(t.preconditioner_aggregate, t.preconditioner_aggregate + s.S));
            const std::vector<double> diag = host_diagonal(t);
            s.diagonal.upload(diag);
            build_operator(s, t);
            if (options && options->gmres_restart)
            {
                require(options->gmres_restart > 0 && options->gmres_restart <= System::gmres_restart, "gmres_restart must be 0..24");
                s.restart = options->gmres_restart;
            }
            if (options && options->mg_stage_sweeps)
            {
                require(options->mg_stage_sweeps > 0 && options->mg_stage_sweeps <= 16, "mg_stage_sweeps must be 0..16");
                s.mg_stage_sweeps = options->mg_stage_sweeps;
            }
            if (options && options->mg_stage_fp16)
            {
                require(options->mg_stage_fp16 == 1, "mg_stage_fp16 must be 0 or 1");
                s.mg_stage_fp16 = 1;
            }
            if (options && options->mg_stage_csr)
            {
                require(options->mg_stage_csr == 1, "mg_stage_csr must be 0 or 1");
                s.mg_stage_csr = 1;
            }
            if (options && options->gmres_recycle)
            {
                require(options->gmres_recycle >= -1 && options->gmres_recycle <= System::recycle_capacity, "gmres_recycle must be -1..3");
                s.recycle_limit = options->gmres_recycle < 0 ? 0 : options->gmres_recycle;
            }
            if (options && options->gmres_delayed)
            {
                require(options->gmres_delayed == 1, "gmres_delayed must be 0 or 1");
                s.delayed_orthogonalisation = true;
            }
            if (options && options->mg_stage_chebyshev)
            {
                require(options->mg_stage_chebyshev >= 1 && options->mg_stage_chebyshev <= 1000, "mg_stage_chebyshev must be 0..1000");
                s.mg_stage_chebyshev = options->mg_stage_chebyshev == 1 ? 0 : options->mg_stage_chebyshev;
            }
            if (options && options->mg_fine_chebyshev)
            {
                require(options->mg_fine_chebyshev >= 1 && options->mg_fine_chebyshev <= 1000, "mg_fine_chebyshev must be 0..1000");
                s.mg_fine_chebyshev = options->mg_fine_chebyshev == 1 ? 0 : options->mg_fine_chebyshev;
            }
            if (options && options->mg_block_iterations)
            {
                require(options->mg_block_iterations > 0 && options->mg_block_iterations <= 64, "mg_block_iterations must be 0..64");
                s.mg_block_iterations = options->mg_block_iterations;
            }
            const int cycle = options ? options->mg_cycle : PCFD_MG_CYCLE_REFERENCE;
            require(cycle >= PCFD_MG_CYCLE_REFERENCE && cycle <= PCFD_MG_CYCLE_COMPOSITE, "unknown multigrid cycle");
            if (cycle == PCFD_MG_CYCLE_CORRECTED) { s.mg_prolong_scale = 2.0; s.mg_lattice_scale = 1.5; }
            if (cycle == PCFD_MG_CYCLE_COMPOSITE) s.mg_prolong_scale = 2.0;
            build_multigrid(s, t, diag);
            for (MgLevel<double>& level : s.mg64) level.prolong = s.mg_lattice_scale;
            for (MgLevel<float>& level : s.mg32) level.prolong = s.mg_lattice_scale;
            if (!options || !options->disable_fused_smoother) build_fine_smoother(s, t, diag);
            if (cycle == PCFD_MG_CYCLE_COMPOSITE)
            {
                require(s.fine.enabled, "the composite cycle needs the fused fine level (8^3 bricks)");
                s.composite_fp32 = s.mg_precision == PCFD_MG_FP32 && !s.mg32.empty();
                build_composite(s, t);
                attach_deferred_map(s);
            }
            // Krylov storage
            for (DBuf<double>* v : {&s.r, &s.z, &s.dvec, &s.Ad, &s.t, &s.correction, &s.defect, &s.scratch_p, &s.scratch_out,
                                     &s.integrated, &s.rhs, &s.pressure})
                v->alloc(size_t(s.Sp));
            if (s.full_nonorthogonal) allocate_gcro(s);
            s.dot_partial.alloc(4096);
            s.dot_result.alloc(16);
            s.block_partial.alloc(size_t(592) * (kMaxSet + 1));
            s.block_result.alloc(size_t(4) * (kMaxSet + 1));
            cuda_check(cudaMallocHost(&s.pinned, 16 * sizeof(double)), "pinned scalars");
            cuda_check(cudaMallocHost(&s.pinned_block, size_t(4) * (kMaxSet + 1) * sizeof(double)), "pinned block scalars");
            s.dcgs_partial.alloc(size_t(592) * (2 * kMaxSet + 4));
            s.dcgs_result.alloc(size_t(kDcgsCoefficients));
            s.dcgs_total.alloc(size_t(2 * kMaxSet + 4));
            s.dcgs_ticket.alloc(1);
            cuda_check(cudaMallocHost(&s.pinned_dcgs, size_t(2) * kDcgsCoefficients * sizeof(double)), "pinned orthogonalisation scalars");
            for (cudaEvent_t& e : s.dcgs_ready) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "column event");
            prime_block_grids();
            // flow state
            s.u.alloc(size_t(s.faces)); s.v.alloc(size_t(s.faces)); s.w.alloc(size_t(s.faces));
            s.divergence.alloc(size_t(s.S));
            s.pressure32.alloc(size_t(s.S));
            build_projection(s, t);
            s.h_connected = t.freestream_connected ? std::vector<uint8_t>(t.freestream_connected, t.freestream_connected + s.S)
                                                   : s.h_active;
            s.h_finest = t.levels[t.level_count - 1].h;
            s.momentum = new Momentum();
            build_momentum(s, *s.momentum, t, options ? options->momentum_min_volume_fraction : 0.0);
            build_loads(s, t);
            build_locator(s, t);
            build_mac(s, t);
            build_apertures(s, t);
            cuda_check(cudaDeviceSynchronize(), "system setup");
        }

        System& sys(pcfd_system* p)
        {
            require(p != nullptr, "null system");
            return *reinterpret_cast<System*>(p);
        }

        template <class T> void h2d(System& s, T* dst, const T* src, size_t n)
        {
            require(src != nullptr || n == 0, "null host buffer");
            if (n) cuda_check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s.stream), "host to device");
        }
        // Host inputs of the state setters are rejected when any entry is NaN or infinite, before
        // anything reaches the device (the reference checks its velocities before each step,
        // external_aero_core.cpp:308).
        template <class T> void require_finite(const T* src, size_t n, const char* what)
        {
            if (!src) return;
            for (size_t q = 0; q < n; ++q)
                if (!std::isfinite(src[q])) throw Error(PCFD_INVALID_ARG, std::string("non-finite ") + what + " at entry " + std::to_string(q));
        }
        template <class T> void d2h(System& s, T* dst, const T* src, size_t n)
        {
            require(dst != nullptr || n == 0, "null host buffer");
            if (n) cuda_check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, s.stream), "device to host");
        }
        void sync(System& s) { cuda_check(cudaStreamSynchronize(s.stream), "synchronize"); }
    }

    // basis storage of the flexible GCRO/LGMRES solver
    void allocate_gcro(System& s)
    {
        if (s.gmres_v.p) return;
        s.gmres_v.alloc(size_t(System::gmres_restart + 1) * s.Sp);
        s.gmres_z.alloc(size_t(System::gmres_restart) * s.Sp);
        s.recycle_u.alloc(size_t(System::recycle_capacity) * s.Sp);
        s.recycle_c.alloc(size_t(System::recycle_capacity) * s.Sp);
    }

    System::~System()
    {
        learned_destroy(*this);
        if (mg_graph_composite) cudaGraphExecDestroy(mg_graph_composite);
        for (cudaEvent_t& e : markers)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : profile_events) cudaEventDestroy(e);
        if (mg_graph64) cudaGraphExecDestroy(mg_graph64);
        if (mg_graph32) cudaGraphExecDestroy(mg_graph32);
        destroy_loads(*this);
        destroy_locator(*this);
        destroy_mac(*this);
        destroy_apertures(*this);
        delete momentum;
        if (pinned) cudaFreeHost(pinned);
        if (pinned_block) cudaFreeHost(pinned_block);
        if (pinned_dcgs) cudaFreeHost(pinned_dcgs);
        for (cudaEvent_t e : dcgs_ready)
            if (e) cudaEventDestroy(e);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
}

using namespace pcfd;

extern "C" {

const char* pcfd_last_error_message(void) { return g_error.c_str(); }
const char* pcfd_version(void) { return "paracfd_b200 0.1 (sm_100a)"; }

pcfd_status pcfd_system_create(const pcfd_topology* topology, const pcfd_options* options, pcfd_system** out)
{
    return guarded([&] {
        require(topology && out, "null topology or output handle");
        *out = nullptr;
        auto s = std::make_unique<System>();
        create(*topology, options, *s);
        *out = reinterpret_cast<pcfd_system*>(s.release());
    });
}

void pcfd_system_destroy(pcfd_system* system)
{
    if (!system) return;
    System* s = reinterpret_cast<System*>(system);
    cudaStreamSynchronize(s->stream);
    delete s;
}

pcfd_status pcfd_system_sizes(const pcfd_system* system, int64_t* storage, int64_t* bricks, int64_t* faces, int64_t* cf, int64_t* eb)
{
    return guarded([&] {
        require(system != nullptr, "null system");
        const System& s = *reinterpret_cast<const System*>(system);
        if (storage) *storage = s.S;
        if (bricks) *bricks = s.B;
        if (faces) *faces = s.faces;
        if (cf) *cf = s.cf_count;
        if (eb) *eb = s.eb_count;
    });
}

pcfd_status pcfd_system_synchronize(pcfd_system* system)
{
    return guarded([&] { sync(sys(system)); });
}

pcfd_status pcfd_pressure_apply_host(pcfd_system* system, const double* p, double* out, int32_t orthogonal)
{
    return guarded([&] {
        System& s = sys(system);
        h2d(s, s.scratch_p.p, p, size_t(s.S));
        launch_apply(s, s.scratch_p, s.scratch_out, orthogonal != 0);
        d2h(s, out, s.scratch_out.p, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_pressure_apply_device(pcfd_system* system, const double* d_p, double* d_out, int32_t orthogonal)
{
    return guarded([&] {
        System& s = sys(system);
        require(d_p && d_out, "null device vector");
        launch_apply(s, d_p, d_out, orthogonal != 0);
    });
}

pcfd_status pcfd_pressure_apply_device_noalloc(pcfd_system* system, const double* d_p, double* d_out, int32_t orthogonal)
{
    return guarded([&] {
        System& s = sys(system);
        require(d_p && d_out, "null device vector");
        launch_apply_noalloc(s, d_p, d_out, orthogonal != 0);
    });
}

pcfd_status pcfd_pressure_diagonal_host(pcfd_system* system, double* diag)
{
    return guarded([&] {
        System& s = sys(system);
        d2h(s, diag, s.diagonal.p, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_pressure_precondition_host(pcfd_system* system, const double* r, double* z)
{
    return guarded([&] {
        System& s = sys(system);
        h2d(s, s.scratch_p.p, r, size_t(s.S));
        apply_preconditioner(s, s.scratch_p, s.scratch_out);
        d2h(s, z, s.scratch_out.p, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_pressure_solve_host(pcfd_system* system, double* x, const double* b, double tolerance, int32_t max_iterations,
                                     int32_t warm_start, pcfd_solve_result* result)
{
    return guarded([&] {
        System& s = sys(system);
        require(tolerance > 0 && max_iterations >= 0, "invalid solve tolerance or iteration budget");
        require_finite(b, size_t(s.S), "right-hand side");
        if (warm_start) require_finite(x, size_t(s.S), "initial guess");
        h2d(s, s.scratch_p.p, b, size_t(s.S));
        if (warm_start) h2d(s, s.scratch_out.p, x, size_t(s.S));
        const pcfd_solve_result r = solve(s, s.scratch_out, s.scratch_p, tolerance, max_iterations, warm_start != 0);
        d2h(s, x, s.scratch_out.p, size_t(s.S));
        sync(s);
        if (result) *result = r;
    });
}

pcfd_status pcfd_set_faces_host(pcfd_system* system, const float* u, const float* v, const float* w)
{
    return guarded([&] {
        System& s = sys(system);
        require_finite(u, size_t(s.faces), "face velocity u");
        require_finite(v, size_t(s.faces), "face velocity v");
        require_finite(w, size_t(s.faces), "face velocity w");
        h2d(s, s.u.p, u, size_t(s.faces)); h2d(s, s.v.p, v, size_t(s.faces)); h2d(s, s.w.p, w, size_t(s.faces));
        sync(s);
    });
}
pcfd_status pcfd_get_faces_host(pcfd_system* system, float* u, float* v, float* w)
{
    return guarded([&] {
        System& s = sys(system);
        d2h(s, u, s.u.p, size_t(s.faces)); d2h(s, v, s.v.p, size_t(s.faces)); d2h(s, w, s.w.p, size_t(s.faces));
        sync(s);
    });
}
pcfd_status pcfd_set_special_host(pcfd_system* system, const float* cf, const float* eb)
{
    return guarded([&] {
        System& s = sys(system);
        require_finite(cf, size_t(s.cf_count), "coarse/fine velocity");
        require_finite(eb, size_t(s.eb_count), "embedded velocity");
        h2d(s, s.special.p, cf, size_t(s.cf_count));
        h2d(s, s.special.p + s.cf_count, eb, size_t(s.eb_count));
        sync(s);
    });
}
pcfd_status pcfd_get_special_host(pcfd_system* system, float* cf, float* eb)
{
    return guarded([&] {
        System& s = sys(system);
        d2h(s, cf, s.special.p, size_t(s.cf_count));
        d2h(s, eb, s.special.p + s.cf_count, size_t(s.eb_count));
        sync(s);
    });
}
pcfd_status pcfd_set_pressure_host(pcfd_system* system, const double* p)
{
    return guarded([&] {
        System& s = sys(system);
        require_finite(p, size_t(s.S), "pressure state");
        h2d(s, s.pressure.p, p, size_t(s.S));
        s.previous_count = 0;
        launch_convert_pressure(s);
        sync(s);
    });
}
pcfd_status pcfd_get_pressure_host(pcfd_system* system, double* p)
{
    return guarded([&] {
        System& s = sys(system);
        d2h(s, p, s.pressure.p, size_t(s.S));
        sync(s);
    });
}
pcfd_status pcfd_get_pressure_shadow_host(pcfd_system* system, float* p32)
{
    return guarded([&] {
        System& s = sys(system);
        d2h(s, p32, s.pressure32.p, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_projection_divergence_host(pcfd_system* system, float* divergence)
{
    return guarded([&] {
        System& s = sys(system);
        launch_integrated_flux(s);
        launch_normalize(s, 0.0, false);
        if (divergence) d2h(s, divergence, s.divergence.p, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_projection_rhs_host(pcfd_system* system, double rho, double dt, double* rhs)
{
    return guarded([&] {
        System& s = sys(system);
        require(rho > 0 && dt > 0, "projection rho/dt must be positive");
        launch_integrated_flux(s);
        launch_normalize(s, rho / dt, true);
        if (rhs) d2h(s, rhs, s.rhs.p, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_projection_correct(pcfd_system* system, double rho, double dt)
{
    return guarded([&] {
        System& s = sys(system);
        require(rho > 0 && dt > 0, "projection correction rho/dt must be positive");
        launch_correct_fluxes(s, rho, dt);
        sync(s);
    });
}

pcfd_status pcfd_projection_project(pcfd_system* system, double rho, double dt, double tolerance, int32_t max_iterations,
                                    int32_t warm_start, pcfd_solve_result* result)
{
    return guarded([&] {
        System& s = sys(system);
        require(rho > 0 && dt > 0, "projection rho/dt must be positive");
        launch_integrated_flux(s);
        launch_normalize(s, rho / dt, true);
        const pcfd_solve_result r = solve(s, s.pressure, s.rhs, tolerance, max_iterations, warm_start != 0);
        if (r.converged)
        {
            launch_convert_pressure(s);
            launch_correct_fluxes(s, rho, dt);
            launch_integrated_flux(s);
            launch_normalize(s, 0.0, false);
        }
        sync(s);
        if (result) *result = r;
        if (!r.converged) throw Error(PCFD_NOT_CONVERGED, "pressure solve did not reach the tolerance");
    });
}

pcfd_status pcfd_momentum_set_state_host(pcfd_system* system, const float* x, const float* y, const float* z)
{
    return guarded([&] {
        System& s = sys(system);
        Momentum& m = momentum_of(s);
        require_finite(x, size_t(s.S), "cell momentum x");
        require_finite(y, size_t(s.S), "cell momentum y");
        require_finite(z, size_t(s.S), "cell momentum z");
        h2d(s, m.x.p, x, size_t(s.S)); h2d(s, m.y.p, y, size_t(s.S)); h2d(s, m.z.p, z, size_t(s.S));
        h2d(s, m.xn.p, x, size_t(s.S)); h2d(s, m.yn.p, y, size_t(s.S)); h2d(s, m.zn.p, z, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_momentum_get_state_host(pcfd_system* system, float* x, float* y, float* z)
{
    return guarded([&] {
        System& s = sys(system);
        Momentum& m = momentum_of(s);
        d2h(s, x, m.x.p, size_t(s.S)); d2h(s, y, m.y.p, size_t(s.S)); d2h(s, z, m.z.p, size_t(s.S));
        sync(s);
    });
}

pcfd_status pcfd_momentum_transport(pcfd_system* system, double dt, double freestream_speed, int32_t external_aero)
{
    return guarded([&] {
        System& s = sys(system);
        require(dt > 0 && freestream_speed >= 0, "invalid cell momentum timestep");
        momentum_transport(s, momentum_of(s), float(dt), float(freestream_speed), external_aero != 0);
        sync(s);
    });
}

pcfd_status pcfd_momentum_smagorinsky(pcfd_system* system, double nu, double cs, double dt, double* rate, int32_t* substeps)
{
    return guarded([&] {
        System& s = sys(system);
        require(nu >= 0 && cs >= 0 && dt > 0, "invalid Smagorinsky timestep");
        Momentum& m = momentum_of(s);
        const double r = momentum_smagorinsky(s, m, float(nu), float(cs), float(dt));
        sync(s);
        if (rate) *rate = r;
        if (substeps) *substeps = m.last_substeps;
    });
}

pcfd_status pcfd_momentum_smooth_wall(pcfd_system* system, double dt, double nu)
{
    return guarded([&] {
        System& s = sys(system);
        require(dt > 0 && nu > 0, "invalid smooth-wall timestep");
        momentum_wall(s, momentum_of(s), float(dt), float(nu));
        sync(s);
    });
}

pcfd_status pcfd_momentum_wall_forces_host(pcfd_system* system, float* force, int64_t* sides)
{
    return guarded([&] {
        System& s = sys(system);
        Momentum& m = momentum_of(s);
        if (sides) *sides = m.nW;
        if (force) d2h(s, force, m.w_force.p, size_t(m.nW) * 3);
        sync(s);
    });
}

pcfd_status pcfd_momentum_pressure_impulse(pcfd_system* system, double dt, double rho, int32_t physical_boundaries, int32_t redistribute)
{
    return guarded([&] {
        System& s = sys(system);
        require(dt > 0 && rho > 0, "invalid pressure impulse");
        Momentum& m = momentum_of(s);
        const int groups = m.nG;
        if (!redistribute) m.nG = 0;
        try { momentum_pressure_impulse(s, m, float(dt), float(rho), physical_boundaries != 0); }
        catch (...) { m.nG = groups; throw; }
        m.nG = groups;
        sync(s);
    });
}

pcfd_status pcfd_momentum_reconstruct_fluxes(pcfd_system* system)
{
    return guarded([&] {
        System& s = sys(system);
        momentum_reconstruct_fluxes(s, momentum_of(s));
        sync(s);
    });
}

pcfd_status pcfd_apply_external_boundaries(pcfd_system* system, double speed)
{
    return guarded([&] {
        System& s = sys(system);
        momentum_external_boundaries(s, float(speed));
        sync(s);
    });
}

pcfd_status pcfd_momentum_cfl(pcfd_system* system, int32_t external_aero, double out[3])
{
    return guarded([&] {
        System& s = sys(system);
        require(out != nullptr, "null output");
        float r[4];
        momentum_cfl(s, momentum_of(s), external_aero != 0, r);
        for (int q = 0; q < 3; ++q) out[q] = r[q];
    });
}

pcfd_status pcfd_core_configure(pcfd_system* system, const pcfd_case* config)
{
    return guarded([&] {
        System& s = sys(system);
        require(config != nullptr, "null case");
        const pcfd_case& c = *config;
        require(c.speed >= 0 && c.rho > 0 && c.nu >= 0 && c.cfl > 0 && c.smagorinsky_cs >= 0 && c.projection_tolerance > 0 &&
                    c.projection_max_iterations > 0,
                "invalid case configuration");
        // a new flow case needs a new initialization; changing only the projection tolerance or
        // iteration budget keeps the initialized state and the physical time
        const pcfd_case& o = s.config;
        const bool same_flow = s.configured && o.speed == c.speed && o.rho == c.rho && o.nu == c.nu && o.cfl == c.cfl &&
                               o.smagorinsky_cs == c.smagorinsky_cs && o.smooth_wall == c.smooth_wall &&
                               o.pressure_impulse == c.pressure_impulse;
        s.config = c;
        s.configured = true;
        if (!same_flow)
        {
            s.initialized = false;
            s.physical_time = 0.0;
        }
    });
}

pcfd_status pcfd_core_initialize(pcfd_system* system, pcfd_step_stats* stats)
{
    return guarded([&] {
        System& s = sys(system);
        pcfd_step_stats local;
        core_initialize(s, local);
        if (stats) *stats = local;
        if (!s.initialized) throw Error(PCFD_NOT_CONVERGED, "initial projection did not converge");
    });
}

pcfd_status pcfd_core_step(pcfd_system* system, pcfd_step_stats* stats)
{
    return guarded([&] {
        System& s = sys(system);
        pcfd_step_stats local;
        core_step(s, local);
        if (stats) *stats = local;
        if (!local.pressure.converged) throw Error(PCFD_NOT_CONVERGED, "pressure solve did not converge; time not advanced");
    });
}

pcfd_status pcfd_core_conservation_stats(pcfd_system* system, pcfd_conservation_stats* out)
{
    return guarded([&] {
        System& s = sys(system);
        require(out != nullptr, "null output");
        double v[6];
        conservation_stats(s, v);
        out->max_abs_divergence = v[0];
        out->volume_weighted_rms_divergence = v[1];
        out->worst_control_volume = v[2];
        out->max_integrated_flux_error = v[3];
        out->absolute_integrated_flux_error = v[4];
        out->net_integrated_flux_error = v[5];
    });
}

pcfd_status pcfd_autotune(pcfd_system* system, int32_t iterations, pcfd_autotune_report* report)
{
    return guarded([&] {
        System& s = sys(system);
        require(iterations > 0 && iterations <= 1000, "autotune: 1..1000 iterations");
        pcfd_autotune_report r{};
        r.candidates = autotune_pipe(s, iterations, r.ctas_per_sm, r.apply_ms, r.sweep_ms);
        r.chosen = s.pipe_ctas_per_sm;
        if (report) *report = r;
    });
}

pcfd_status pcfd_set_pipeline_ctas(pcfd_system* system, int32_t ctas_per_sm)
{
    return guarded([&] {
        System& s = sys(system);
        require(ctas_per_sm >= 1 && ctas_per_sm <= 8, "pipeline CTAs per SM: 1..8");
        s.pipe_ctas_per_sm = ctas_per_sm;
    });
}

pcfd_status pcfd_locate_points_device(pcfd_system* system, const float* d_points, int32_t count, int32_t* d_locations)
{
    return guarded([&] {
        System& s = sys(system);
        require(count >= 0 && (count == 0 || (d_points && d_locations)), "null points or locations");
        locate_points(s, d_points, count, d_locations);
    });
}

pcfd_status pcfd_sample_slice_host(pcfd_system* system, const double origin[3], const double edge_u[3], const double edge_v[3],
                                   int32_t nu, int32_t nv, int32_t field, float* out)
{
    return guarded([&] {
        System& s = sys(system);
        require(origin && edge_u && edge_v && out, "null slice argument");
        require(nu > 0 && nv > 0, "slice: nu, nv must be positive");
        const size_t n = size_t(nu) * size_t(nv);
        if (s.slice_buffer.n < n) s.slice_buffer.alloc(n);
        sample_slice(s, origin, edge_u, edge_v, nu, nv, field, s.slice_buffer.p);
        d2h(s, out, s.slice_buffer.p, n);
        sync(s);
    });
}

pcfd_status pcfd_core_set_momentum_mode(pcfd_system* system, int32_t mode)
{
    return guarded([&] {
        System& s = sys(system);
        require(mode == PCFD_MOMENTUM_CELL || mode == PCFD_MOMENTUM_MAC, "momentum mode must be 0 (cell) or 1 (MAC)");
        require(mode == PCFD_MOMENTUM_CELL || mac_ready(s), "the MAC momentum mode needs pcfd_mac_set_links first");
        s.momentum_mode = mode;
        s.initialized = false;
    });
}

pcfd_status pcfd_mac_set_links(pcfd_system* system, const uint8_t* links_u, const uint8_t* links_v, const uint8_t* links_w)
{
    return guarded([&] {
        System& s = sys(system);
        require(links_u && links_v && links_w, "null MAC link array");
        const uint8_t* host[3] = {links_u, links_v, links_w};
        mac_set_links(s, host);
    });
}

pcfd_status pcfd_mac_advect(pcfd_system* system, double dt)
{
    return guarded([&] {
        System& s = sys(system);
        require(std::isfinite(dt) && dt > 0.0, "MAC advection timestep must be positive");
        mac_advect(s, float(dt));
        sync(s);
    });
}

pcfd_status pcfd_mac_diffuse_smagorinsky(pcfd_system* system, double nu, double cs, double dt)
{
    return guarded([&] {
        System& s = sys(system);
        require(std::isfinite(nu) && std::isfinite(cs) && std::isfinite(dt) && nu >= 0.0 && cs >= 0.0 && dt > 0.0,
                "invalid MAC LES/diffusion parameters");
        mac_diffuse_smagorinsky(s, float(nu), float(cs), float(dt));
        sync(s);
    });
}

pcfd_status pcfd_mac_transport_apertures(pcfd_system* system, double dt, double nu, double cs)
{
    return guarded([&] {
        System& s = sys(system);
        require(std::isfinite(nu) && std::isfinite(cs) && std::isfinite(dt) && nu >= 0.0 && cs >= 0.0 && dt > 0.0,
                "invalid aperture transport parameters");
        mac_transport_apertures(s, float(dt), float(nu), float(cs));
        sync(s);
    });
}

pcfd_status pcfd_mac_eddy_viscosity_host(pcfd_system* system, float* nut)
{
    return guarded([&] {
        System& s = sys(system);
        require(nut != nullptr, "null eddy-viscosity buffer");
        mac_eddy_viscosity(s, nut);
    });
}

pcfd_status pcfd_core_inflow_layout(pcfd_system* system, int64_t* face_count, int32_t* brick_slots)
{
    return guarded([&] {
        System& s = sys(system);
        require(face_count != nullptr, "null face count");
        *face_count = s.inflow_faces;
        if (brick_slots && s.inflow_faces)
        {
            std::vector<int> map(size_t(s.B));
            cuda_check(cudaMemcpy(map.data(), s.inflow_slot_of_brick, map.size() * sizeof(int), cudaMemcpyDeviceToHost),
                       "inflow layout");
            for (int slot = 0; slot < s.B; ++slot)
                if (map[slot] >= 0) brick_slots[map[slot]] = slot;
        }
    });
}

pcfd_status pcfd_core_set_inflow_host(pcfd_system* system, const float* normal_velocity, int64_t count)
{
    return guarded([&] {
        System& s = sys(system);
        if (count == 0) { s.inflow_set = false; return; }
        require(count == s.inflow_faces, "inflow count must equal the X-min boundary face count");
        require_finite(normal_velocity, size_t(count), "inflow velocity");
        h2d(s, s.inflow.p, normal_velocity, size_t(count));
        s.inflow_set = true;
    });
}

pcfd_status pcfd_preconditioner_fused(pcfd_system* system, int32_t* fused)
{
    return guarded([&] {
        System& s = sys(system);
        require(fused != nullptr, "null output");
        *fused = s.fine.enabled ? 1 : 0;
    });
}

pcfd_status pcfd_core_set_initial_guess(pcfd_system* system, int32_t mode)
{
    return guarded([&] {
        System& s = sys(system);
        require(mode >= 0 && mode <= 2, "initial guess mode must be 0, 1 or 2");
        if (mode >= 1 && !s.pressure_previous.p) s.pressure_previous.alloc(size_t(s.Sp));
        if (mode == 2 && !s.pressure_previous2.p) s.pressure_previous2.alloc(size_t(s.Sp));
        s.initial_guess = mode;
        s.previous_count = 0;
    });
}

pcfd_status pcfd_projection_keep_start(pcfd_system* system, int32_t keep)
{
    return guarded([&] {
        System& s = sys(system);
        if (keep && !s.start_pressure.p)
        {
            s.start_pressure.alloc(size_t(s.Sp));
            s.start_recycle_u.alloc(size_t(System::recycle_capacity) * s.Sp);
            s.start_recycle_c.alloc(size_t(System::recycle_capacity) * s.Sp);
        }
        s.keep_projection_start = keep != 0;
        s.start_saved = false;
    });
}

pcfd_status pcfd_projection_resolve(pcfd_system* system, double tolerance, int32_t max_iterations, double* ms,
                                    pcfd_solve_result* result)
{
    return guarded([&] {
        System& s = sys(system);
        require(tolerance > 0 && max_iterations >= 0 && ms, "invalid resolve request");
        const pcfd_solve_result r = resolve_projection(s, tolerance, max_iterations, ms);
        if (result) *result = r;
    });
}

pcfd_status pcfd_set_preconditioner(pcfd_system* system, int32_t kind)
{
    return guarded([&] {
        System& s = sys(system);
        require(kind >= PCFD_PRECONDITIONER_MULTIGRID && kind <= PCFD_PRECONDITIONER_LEARNED_MULTIGRID, "unknown preconditioner");
        require(kind != PCFD_PRECONDITIONER_LEARNED_MULTIGRID || (s.composite && s.fine.enabled),
                "the learned multigrid preconditioner needs the composite cycle (PCFD_MG_CYCLE_COMPOSITE)");
        if (kind == PCFD_PRECONDITIONER_LEARNED || kind == PCFD_PRECONDITIONER_LEARNED_MULTIGRID) allocate_gcro(s);
        s.preconditioner = kind;
    });
}

pcfd_status pcfd_learned_parameter_count(int64_t* count)
{
    return guarded([&] {
        require(count != nullptr, "null output");
        *count = learned_parameter_count();
    });
}

pcfd_status pcfd_learned_set_parameters(pcfd_system* system, const float* parameters, int64_t count)
{
    return guarded([&] {
        System& s = sys(system);
        require(parameters != nullptr, "null parameters");
        learned_set_parameters(s, parameters, count);
    });
}

pcfd_status pcfd_learned_get_parameters(pcfd_system* system, float* parameters, int64_t count)
{
    return guarded([&] {
        System& s = sys(system);
        require(parameters != nullptr, "null parameters");
        learned_get_parameters(s, parameters, count);
    });
}

pcfd_status pcfd_learned_harvest_begin(pcfd_system* system, int32_t capacity_pairs, int32_t bricks_per_pair, uint64_t seed,
                                       int32_t target)
{
    return guarded([&] { learned_harvest_begin(sys(system), capacity_pairs, bricks_per_pair, seed, target); });
}

pcfd_status pcfd_learned_harvest_stop(pcfd_system* system, int64_t* samples)
{
    return guarded([&] {
        System& s = sys(system);
        require(samples != nullptr, "null output");
        *samples = learned_harvest_stop(s);
    });
}

pcfd_status pcfd_learned_train(pcfd_system* system, int32_t steps, int32_t batch, double learning_rate, uint64_t seed, double* final_loss)
{
    return guarded([&] {
        System& s = sys(system);
        const double loss = learned_train(s, steps, batch, learning_rate, seed);
        if (final_loss) *final_loss = loss;
    });
}

pcfd_status pcfd_learned_evaluate_host(pcfd_system* system, int32_t samples, const float* inputs, const float* targets, float* zhat,
                                       double* loss, float* gradients)
{
    return guarded([&] {
        System& s = sys(system);
        const double l = learned_evaluate(s, samples, inputs, targets, zhat, gradients);
        if (loss) *loss = l;
    });
}

pcfd_status pcfd_learned_set_wait(pcfd_system* system, double seconds, int32_t idle_barrier_once)
{
    return guarded([&] { learned_set_wait(sys(system), seconds, idle_barrier_once != 0); });
}

pcfd_status pcfd_learned_apply_device(pcfd_system* system, const double* d_r, double* d_z)
{
    return guarded([&] {
        System& s = sys(system);
        require(d_r && d_z, "null vector");
        learned_apply(s, d_r, d_z);
        learned_check(s);
    });
}

pcfd_status pcfd_launch_count(pcfd_system* system, int64_t* launches)
{
    return guarded([&] {
        System& s = sys(system);
        require(launches != nullptr, "null launch count");
        *launches = s.launches;
    });
}

pcfd_status pcfd_profile_begin(pcfd_system* system, int32_t region, int32_t capacity)
{
    return guarded([&] {
        System& s = sys(system);
        require(region >= PCFD_PROFILE_STRUCTURED_APPLY && region <= PCFD_PROFILE_STAGE_SMOOTH, "unknown profile region");
        require(capacity > 0 && capacity <= (1 << 16), "profile capacity must be 1..65536");
        while (int(s.profile_events.size()) < 2 * capacity)
        {
            cudaEvent_t e;
            cuda_check(cudaEventCreate(&e), "profile event");
            s.profile_events.push_back(e);
        }
        s.profile_used = 0;
        s.profile_region = region;
    });
}

pcfd_status pcfd_profile_end(pcfd_system* system, double* ms_per_launch, int32_t capacity, int32_t* launches)
{
    return guarded([&] {
        System& s = sys(system);
        require(launches != nullptr, "null launch count");
        s.profile_region = -1;
        const int used = s.profile_used;
        *launches = used;
        if (used) cuda_check(cudaEventSynchronize(s.profile_events[2 * used - 1]), "profile sync");
        for (int q = 0; q < used && q < capacity && ms_per_launch; ++q)
        {
            float ms = 0;
            cuda_check(cudaEventElapsedTime(&ms, s.profile_events[2 * q], s.profile_events[2 * q + 1]), "profile elapsed");
            ms_per_launch[q] = ms;
        }
        s.profile_used = 0;
    });
}

pcfd_status pcfd_profile_bytes(pcfd_system* system, int32_t region, double* bytes_per_launch)
{
    return guarded([&] {
        System& s = sys(system);
        require(bytes_per_launch != nullptr, "null output");
        require(region >= PCFD_PROFILE_STRUCTURED_APPLY && region <= PCFD_PROFILE_DCGS_COLUMN, "unknown profile region");
        if (region == PCFD_PROFILE_STRUCTURED_APPLY)
        {
            *bytes_per_launch = 17.0 * double(s.active_bricks) * double(s.bs3);   // active_bricks: the non-covered bricks
        }
        else if (region == PCFD_PROFILE_STAGE_SMOOTH) *bytes_per_launch = stage_smooth_bytes(s);
        else if (region == PCFD_PROFILE_DCGS_COLUMN) *bytes_per_launch = 258.0 * double(krylov_sweep_entries(s));
        else *bytes_per_launch = 0.0;
    });
}

pcfd_status pcfd_stage_brick_structured(pcfd_system* system, int32_t* structured)
{
    return guarded([&] {
        System& s = sys(system);
        require(structured != nullptr, "null output");
        *structured = s.composite && ((s.composite_fp32 && !s.inter32.empty() && s.inter32.front().brick_rows.p) ||
                                      (!s.composite_fp32 && !s.inter64.empty() && s.inter64.front().brick_rows.p))
                          ? 1 : 0;
    });
}

pcfd_status pcfd_event_record(pcfd_system* system, int32_t slot)
{
    return guarded([&] {
        System& s = sys(system);
        require(slot >= 0 && slot < 8, "event slot must be 0..7");
        if (!s.markers[slot]) cuda_check(cudaEventCreate(&s.markers[slot]), "create marker");
        cuda_check(cudaEventRecord(s.markers[slot], s.stream), "record marker");
    });
}

pcfd_status pcfd_event_elapsed(pcfd_system* system, int32_t a, int32_t b, double* ms)
{
    return guarded([&] {
        System& s = sys(system);
        require(a >= 0 && a < 8 && b >= 0 && b < 8 && s.markers[a] && s.markers[b] && ms, "invalid marker slots");
        cuda_check(cudaEventSynchronize(s.markers[b]), "marker sync");
        float v = 0;
        cuda_check(cudaEventElapsedTime(&v, s.markers[a], s.markers[b]), "marker elapsed");
        *ms = v;
    });
}

pcfd_status pcfd_core_loads(pcfd_system* system, double pressure_reference, const double moment_origin[3], double reference_area,
                            int32_t include_viscous, pcfd_loads* out)
{
    return guarded([&] {
        System& s = sys(system);
        require(out != nullptr, "null loads output");
        const double zero[3] = {0, 0, 0};
        const double rho = s.configured ? s.config.rho : 1.0;
        double r[12];
        compute_loads(s, pressure_reference, moment_origin ? moment_origin : zero, rho, include_viscous != 0, r);
        std::memset(out, 0, sizeof(*out));
        for (int a = 0; a < 3; ++a)
        {
            out->pressure_force[a] = r[a];
            out->pressure_moment[a] = r[3 + a];
            out->viscous_force[a] = r[6 + a];
            out->viscous_moment[a] = r[9 + a];
            out->total_force[a] = r[a] + r[6 + a];
            out->total_moment[a] = r[3 + a] + r[9 + a];
        }
        const double q = s.configured ? 0.5 * s.config.rho * s.config.speed * s.config.speed : 0.0;
        const double nan = std::numeric_limits<double>::quiet_NaN();
        const bool valid = q > 0 && reference_area > 0;
        out->cd = valid ? out->total_force[0] / (q * reference_area) : nan;
        out->cs = valid ? out->total_force[1] / (q * reference_area) : nan;
        out->cl = valid ? out->total_force[2] / (q * reference_area) : nan;
    });
}

pcfd_status pcfd_time_kernel(pcfd_system* system, int32_t which, int32_t iterations, double* ms_per_launch)
{
    return guarded([&] {
        System& s = sys(system);
        require(iterations > 0 && ms_per_launch, "invalid timing request");
        auto once = [&]() {
            switch (which)
            {
            case 0: launch_apply(s, s.scratch_p, s.scratch_out, false); break;
            case 1: launch_apply(s, s.scratch_p, s.scratch_out, true); break;
            case 2: apply_preconditioner(s, s.scratch_p, s.scratch_out); break;
            case 3: launch_integrated_flux(s); launch_normalize(s, 0.0, false); break;
            case 4: launch_correct_fluxes(s, 1.0, 1e-3); break;
            case 5: device_dot(s, s.scratch_p, s.scratch_out); break;
            case 6:
            case 7:
            case 8: preconditioner_stage(s, which - 6, s.scratch_p, s.scratch_out); break;
            case 10:
            case 11:
            case 12:
            case 13: fine_preconditioner_stage(s, which - 10, s.scratch_p, s.scratch_out); break;
            case 9:
            case 14:
            case 15:
            {
                // one GCRO column orthogonalisation (CGS2, three passes) against 3 recycled + V
                // basis vectors: 13 (m = 16), 5 (m = 8) or 24 (m = 27)
                require(s.full_nonorthogonal, "block orthogonalisation needs the GCRO storage");
                const int basis = which == 9 ? 13 : (which == 14 ? 5 : 24);
                VecSet Q(s.Sp);
                const VecSet none(s.Sp);
                for (int c = 0; c < System::recycle_capacity; ++c) Q.push(s.recycle_c.p + size_t(c) * s.Sp);
                for (int row = 0; row < basis; ++row) Q.push(s.gmres_v.p + size_t(row) * s.Sp);
                double* h = s.block_result.p;
                block_dot(s, Q, s.Ad, h);
                block_update(s, Q, h, s.Ad, none, -1.0, nullptr, 2, h + kMaxSet + 1);
                block_update(s, Q, h + kMaxSet + 1, s.Ad, none, -1.0, nullptr, 1, h + 2 * (kMaxSet + 1));
                break;
            }
            case 16: learned_apply(s, s.scratch_p, s.scratch_out); break;
            case 17: stage_smooth_once(s); break;
            case 18:
            {
                // one delayed-CGS2 column (dot pass, coefficients, update pass) against 13 basis vectors
                require(s.full_nonorthogonal, "delayed CGS2 needs the GCRO storage");
                VecSet Q(s.Sp);
                for (int row = 0; row < 13; ++row) Q.push(s.gmres_v.p + size_t(row) * s.Sp);
                dcgs_pass(s, Q, s.gmres_v.p + size_t(13) * s.Sp, s.Ad, s.gmres_v.p + size_t(14) * s.Sp, s.dcgs_result);
                break;
            }
            default: throw Error(PCFD_INVALID_ARG, "unknown kernel id");
            }
        };
        once();
        sync(s);
        cudaEvent_t start, stop;
        cuda_check(cudaEventCreate(&start), "event");
        cuda_check(cudaEventCreate(&stop), "event");
        cuda_check(cudaEventRecord(start, s.stream), "event record");
        for (int q = 0; q < iterations; ++q) once();
        cuda_check(cudaEventRecord(stop, s.stream), "event record");
        cuda_check(cudaEventSynchronize(stop), "event sync");
        float ms = 0;
        cuda_check(cudaEventElapsedTime(&ms, start, stop), "event time");
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        *ms_per_launch = double(ms) / iterations;
    });
}

}  // extern "C"
