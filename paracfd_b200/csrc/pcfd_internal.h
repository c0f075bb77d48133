// pcfd_internal.h -- device-resident system state behind the C ABI.
//
// Layout in HBM (one allocation per array, all levels concatenated in reference DOF order):
//   * pressure-DOF vectors: [S] with S = B*bs^3 + appended EB root fragments.  DOF numbering is
//     the reference's level_offset + brick*bs^3 + (k*bs+j)*bs+i (amr_pressure.cpp:213-216), so a
//     brick is a contiguous 4 KiB FP64 tile (bs = 8).  Covered-brick slots exist but no kernel
//     reads or writes them; they stay zero.
//   * faces: per brick slot the interior MAC faces only, (bs+1)*bs*bs per component (no ghost
//     ring: 576 floats per brick instead of the reference's 1100, amr_fields.h:20-30).  A face
//     shared by two same-level bricks is stored in both, as the reference does.
//   * active brick list: every kernel over bricks is launched over the compact list of
//     non-covered brick slots of all levels at once (one launch instead of one per level).
#pragma once

#include "../../include/paracfd_b200.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace pcfd
{
    struct Error : std::runtime_error
    {
        pcfd_status status;
        Error(pcfd_status s, const std::string& m) : std::runtime_error(m), status(s) {}
    };

    inline void cuda_check(cudaError_t e, const char* what)
    {
        if (e == cudaSuccess) return;
        const pcfd_status s = e == cudaErrorMemoryAllocation ? PCFD_OUT_OF_MEMORY : PCFD_CUDA_ERROR;
        throw Error(s, std::string(what) + ": " + cudaGetErrorString(e));
    }
    inline void require(bool ok, const std::string& what)
    {
        if (!ok) throw Error(PCFD_INVALID_ARG, what);
    }

    // Owning device buffer.
    template <class T> struct DBuf
    {
        T* p = nullptr;
        size_t n = 0;
        DBuf() = default;
        DBuf(const DBuf&) = delete;
        DBuf& operator=(const DBuf&) = delete;
        DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
        DBuf& operator=(DBuf&& o) noexcept
        {
            if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
            return *this;
        }
        ~DBuf() { release(); }
        void release()
        {
            if (p) cudaFree(p);
            p = nullptr;
            n = 0;
        }
        void alloc(size_t count, bool zero = true)
        {
            release();
            n = count;
            if (!count) return;
            cuda_check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
            if (zero) cuda_check(cudaMemset(p, 0, count * sizeof(T)), "cudaMemset");
        }
        void upload(const std::vector<T>& host)
        {
            alloc(host.size(), false);
            if (!host.empty()) cuda_check(cudaMemcpy(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
        }
        operator T*() const { return p; }
    };

    // Compact non-orthogonal / two-point edge set used by the irregular operator gather.
    struct IrregularOperator
    {
        int incident_dofs = 0, connection_count = 0, regular_count = 0;
        DBuf<int> incident_dof, incident_offset, incident_edge;
        DBuf<int8_t> incident_sign;
        // the same incidence entries packed for the two-point sums: the edge's other endpoint and
        // its coefficient, so coefficient * (p[dof] - p[other]) equals sign * coefficient *
        // (p[lower] - p[upper]) bit for bit with one load chain less
        DBuf<int> incident_other;
        DBuf<double> incident_coefficient;
        // connections (coarse/fine then embedded), geometrically ordered endpoints
        DBuf<int> conn_lower, conn_upper, conn_lower_node, conn_upper_node;
        DBuf<double> conn_coefficient, conn_correction, conn_upper_weight, conn_area;
        // regular corrections
        DBuf<int> reg_lower, reg_upper, reg_lower_node, reg_upper_node;
        DBuf<double> reg_coefficient, reg_correction, reg_upper_weight, reg_area, reg_delta;
        // WLS gradient nodes
        int gradient_nodes = 0;
        DBuf<int> grad_dof, grad_offset, grad_neighbour;
        DBuf<double> grad_weight;
        DBuf<double> gradient;   // [nodes][3] scratch
        // gauges
        int gauges = 0;
        DBuf<int> gauge_dof;
        DBuf<double> gauge_coefficient;
    };

    // One level of the aggregation multigrid (host-built CSR, reference amr_pressure.cu:915-1083).
    template <class T> struct MgLevel
    {
        using value_type = T;
        int cells = 0;
        DBuf<int> row_offset, neighbour, aggregate, restrict_offset, restrict_dof;
        DBuf<T> coefficient, diagonal, rhs, x, temporary, residual;
        DBuf<T> inverse;                        // coarsest composite stage: explicit inverse [cells][cells] or empty
        DBuf<uint16_t> coefficient16;           // FP16 copy of the coefficients the kernels read instead (or empty)
        // The same level in brick-structured form (first composite stage, or empty): rows are 4^3
        // blocks per fine brick; per row the six face-neighbour coefficients (-z, -y, -x, +x, +y,
        // +z, in the row's type or FP16) and a descriptor (first rest entry << 5 | rest count),
        // as 16-byte words; per block its six face-neighbour blocks (-x, +x, -y, +y, -z, +z, or
        // -1); the couplings no face slot holds as (column, coefficient) rest entries.
        DBuf<uint4> brick_rows;
        DBuf<int> brick_neighbour, rest_column;
        DBuf<T> rest_coefficient;
        DBuf<uint16_t> rest_coefficient16;
        double prolong = 1.0;                   // weight of the next level's correction added here
        int sweeps = 2;                         // smoothing steps before and after the coarse correction
        int chebyshev = 0;                      // 0: damped Jacobi; r >= 2: Chebyshev on [2 / r, 2]
    };

    struct Scalars;   // device scalar block for the Krylov recurrences

    // Fused fine-level multigrid work for 8^3 bricks (smoother.cu).
    struct FineSmoother
    {
        bool enabled = false;
        DBuf<uint8_t> code;                     // [S] open faces (bits 0-5), outlet (6), deferred (7)
        int deferred_count = 0;
        // Deferred rows packed so that one load gives all a row's indices: {DOF, first edge, map
        // index of the DOF (composite cycle, else -1), (edges << 8) | (gauges << 2) | (has an
        // incidence row << 1) | active}.  The edges are the row's compact-edge incidence entries
        // whose other endpoint is active, in incidence order: {other endpoint, its map index}
        // and the coefficient.
        DBuf<int4> deferred_row;
        DBuf<int2> deferred_edge;
        DBuf<double> deferred_edge_coefficient;
        DBuf<int> gauge_offset;
        DBuf<double> gauge_coefficient;
        bool map_attached = false;              // deferred map indices filled from the composite stage-1 map
        DBuf<int> stage_neighbour;              // composite cycle: [active bricks][6] face-neighbour brick ranks or -1
        DBuf<int> meta;                         // [active bricks][16] slot, level, level-0 cell, partial, neighbours
        DBuf<double> partial, deferred_residual;
        DBuf<int> gather_offset, gather_entry;  // base cell -> partials (>= 0) / deferred rows (< 0)
        DBuf<double> t, z;                      // [S] deferred structured rows, ping-pong iterate
        DBuf<double> damping;                   // [levels][14] w / D of non-deferred rows
        DBuf<float> damping32, z32, z32b, r32, t32, res32;   // FP32 multigrid: float fine-level buffers
        DBuf<double> cheb_damping;              // [4][damping] Chebyshev-Richardson w / D per sweep (or empty)
        DBuf<float> cheb_damping32;
        size_t cheb_stride = 0;
        double cheb_omega[4] = {};
    };

    // Up to kMaxSet vectors of one system, passed by value to the fused block kernels (krylov.cu):
    // at most two groups of consecutive slots of a multi-vector buffer (e.g. recycled C then the
    // Krylov basis), so a kernel addresses vector j as base + j * stride instead of holding a
    // pointer per vector in registers.
    constexpr int kMaxSet = 32;   // >= GCRO restart (24) + recycled pairs (3) + 1
    struct VecSet
    {
        const double* base[2] = {nullptr, nullptr};
        int count[2] = {0, 0};
        int64_t stride = 0;
        VecSet() = default;
        explicit VecSet(int64_t slot_stride) : stride(slot_stride) {}
        __host__ __device__ int size() const { return count[0] + count[1]; }
        __host__ __device__ const double* vec(int j) const
        {
            return j < count[0] ? base[0] + j * stride : base[1] + (j - count[0]) * stride;
        }
        void push(const double* p)
        {
            if (!count[0]) { base[0] = p; count[0] = 1; }
            else if (!count[1] && p == base[0] + count[0] * stride) ++count[0];
            else if (!count[1]) { base[1] = p; count[1] = 1; }
            else if (p == base[1] + count[1] * stride) ++count[1];
            else throw Error(PCFD_INTERNAL, "vector set is not two strided groups");
        }
    };
    struct Coefficients
    {
        double value[kMaxSet] = {};
    };

    struct System
    {
        // sizes
        int bs = 0, bs3 = 0, levels = 0, S = 0, B = 0, structured = 0, active_bricks = 0;
        int Sp = 0;   // S rounded up to 64: length/stride of internal DOF vectors (16-byte aligned slots)
        int64_t faces = 0;   // per component
        bool outlet = true, full_nonorthogonal = false;
        int mg_precision = PCFD_MG_FP64;
        double mg_prolong_scale = 1.0, mg_lattice_scale = 1.0;   // coarse-correction weights (pcfd_mg_cycle)
        int mg_stage_sweeps = 6;                                 // composite-stage sweeps (pcfd_options)
        int mg_block_iterations = 0;                             // composite cycle: brick block pre-smoother (pcfd_options)
        int mg_stage_chebyshev = 30;                             // composite stages: Chebyshev ratio, 0 = Jacobi (pcfd_options)
        int mg_stage_fp16 = 0;                                   // composite stages: FP16 coefficients (pcfd_options)
        int mg_stage_csr = 0;                                    // composite cycle: first stage kept as CSR (pcfd_options)
        int mg_fine_chebyshev = 10;                              // composite fine sweeps: Chebyshev-Richardson ratio, 0 = Jacobi
        cudaStream_t stream = nullptr;
        bool own_stream = false;
        int device = 0;
        int pipe_ctas_per_sm = 4;               // resident CTAs per SM of the brick pipeline (autotune_pipe)
        double* noalloc_gradient = nullptr;     // static scratch of the allocation-free apply (pressure.cu), once looked up

        // host copies of topology needed after setup
        std::vector<double> level_h;
        std::vector<int> level_slot0;           // first brick slot of each level
        std::vector<uint8_t> h_active;
        std::vector<double> h_volume;
        int cf_count = 0, eb_count = 0;

        // per brick slot
        DBuf<int> brick_level;                  // [B]
        DBuf<int> brick_nbr;                    // [B][6] active same-level neighbour slot or -1
        DBuf<uint32_t> brick_flags;             // [B]
        DBuf<int> active_brick_list;            // [active_bricks]
        DBuf<double> d_level_h;                 // [levels]

        // per DOF
        DBuf<uint8_t> active, cut_face_mask;
        DBuf<double> volume, diagonal;
        DBuf<int> aggregate;                    // preconditioner aggregate (level-0 DOF)

        IrregularOperator irr;

        // multigrid (FP64 parity mode and FP32 mode share structure)
        int base_offset = 0, base_cells = 0;
        DBuf<int> base_restrict_offset, base_restrict_dof;
        std::vector<MgLevel<double>> mg64;
        std::vector<MgLevel<float>> mg32;
        // composite cycle (PCFD_MG_CYCLE_COMPOSITE): Galerkin stages of the AMR composite grid, every
        // level coarsened 2x2x2 per stage; the last stage is the coarsest
        bool composite = false;
        std::vector<MgLevel<double>> inter64;
        std::vector<MgLevel<float>> inter32;    // the same stages in float (FP32 multigrid)
        DBuf<int> fine_map, fine_restrict_offset, fine_restrict_dof;   // fine DOF -> first coarse cell
        bool first_stage_bricks = false;        // stage 1 numbered by brick rank: the restriction CSR lists EB fragments only
        DBuf<double> fine_residual;             // [S] r - A_orth z before the first restriction
        FineSmoother fine;
        cudaGraphExec_t mg_graph64 = nullptr, mg_graph32 = nullptr, mg_graph_composite = nullptr;   // captured hierarchies
        int64_t mg_graph64_launches = 0, mg_graph32_launches = 0, mg_graph_composite_launches = 0;
        bool composite_fp32 = false;            // composite stages in float
        DBuf<float> diagonal32;

        // Krylov vectors
        DBuf<double> r, z, dvec, Ad, t, correction, defect, scratch_p, scratch_out;
        DBuf<double> gmres_v, gmres_z, recycle_u, recycle_c;
        int recycle_count = 0;
        static constexpr int gmres_restart = 24;   // the reference's LGMRES(24) (storage and default)
        int restart = gmres_restart;               // columns per cycle actually used (<= gmres_restart)
        static constexpr int recycle_capacity = 3;
        int recycle_limit = recycle_capacity;      // recycled pairs kept between solves (pcfd_options)
        DBuf<double> dot_partial;               // reduction scratch
        DBuf<double> block_partial;             // [592][kMaxSet + 1] block-kernel partial sums
        DBuf<double> block_result;              // [4][kMaxSet + 1] device coefficients / norms
        DBuf<double> dcgs_partial, dcgs_result; // delayed CGS2 partials [592][2 kMaxSet + 4] and coefficients
        DBuf<double> dcgs_total;                // [2 kMaxSet + 4] the partials' sums
        DBuf<unsigned> dcgs_ticket;             // CTAs of the sum kernel done (0 between launches)
        double* pinned_dcgs = nullptr;          // pinned host copies of dcgs_result, two columns
        cudaEvent_t dcgs_ready[2] = {};         // readback of column j lands in slot j & 1
        bool delayed_orthogonalisation = false; // pcfd_options.gmres_delayed
        double* pinned_block = nullptr;         // pinned host copy of block_result
        DBuf<double> dot_result;                // device scalars
        double* pinned = nullptr;               // pinned host scalars

        // projection state
        DBuf<float> u, v, w;                    // [faces] each
        DBuf<float> special;                    // [cf + eb]
        DBuf<double> special_area, special_factor, special_correction, special_upper_weight;
        DBuf<int> special_lower, special_upper, special_lower_node, special_upper_node;
        int special_incident_dofs = 0;
        DBuf<int> special_incident_dof, special_incident_offset, special_incident_edge;
        DBuf<int8_t> special_incident_sign;
        DBuf<double> integrated;                // [S]
        DBuf<float> divergence;                 // [S]
        DBuf<double> conservation_scratch;      // conservation statistics: block partials and result
        DBuf<int64_t> conservation_index;
        DBuf<double> rhs, pressure;             // [S]
        DBuf<float> pressure32;                 // [S]
        // regular correction face addresses (face array index, mirror or -1)
        DBuf<int64_t> reg_face, reg_mirror;
        DBuf<int8_t> reg_axis;
        // coarse/fine tile <-> face synchronisation
        int cf_groups = 0;
        DBuf<int64_t> cf_fine_face, cf_group_face;
        DBuf<int8_t> cf_axis, cf_group_axis;
        DBuf<int> cf_group_offset, cf_group_member;
        DBuf<double> cf_group_area;

        // saved solver start of the last projection (pcfd_projection_keep_start / resolve)
        bool keep_projection_start = false, start_saved = false, start_warm = false;
        int start_recycle_count = 0;
        DBuf<double> start_pressure, start_recycle_u, start_recycle_c;
        // initial guess of a warm projection: 0 = the last pressure (the reference's warm start),
        // 1 = 2 p_n - p_(n-1), 2 = 3 p_n - 3 p_(n-1) + p_(n-2) from the last converged pressures
        // (pressure_previous holds p_(n-1), pressure_previous2 p_(n-2); previous_count of them valid)
        int initial_guess = 0;
        DBuf<double> pressure_previous, pressure_previous2;
        int previous_count = 0;

        // preconditioner of the Krylov solvers (pcfd_preconditioner) and the learned network state
        int preconditioner = PCFD_PRECONDITIONER_MULTIGRID;
        struct Learned* learned = nullptr;

        // cell-momentum transport and time-step orchestration
        struct Momentum* momentum = nullptr;
        void* loads = nullptr;                  // surface-load integration state (loads.cu)
        void* locator = nullptr;                // point location / slice sampling state (locator.cu)
        void* mac = nullptr;                    // staggered MAC momentum state (mac.cu)
        void* apertures = nullptr;              // MAC-mode compact aperture transport state (mac_apertures.cu)
        int momentum_mode = PCFD_MOMENTUM_CELL; // pcfd_momentum_mode of pcfd_core_initialize / step
        DBuf<float> slice_buffer;               // device output of pcfd_sample_slice_host
        cudaEvent_t markers[8] = {};
        int64_t launches = 0;                   // kernels launched on the system stream so far
        // per-launch event pairs around one instrumented region (PCFD_PROFILE_*), for the roofline
        int profile_region = -1;
        std::vector<cudaEvent_t> profile_events;   // [2 * capacity]
        int profile_used = 0;
        // X-min inflow: one normal velocity per boundary face, or uniform freestream when empty
        int inflow_faces = 0;
        DBuf<int> inflow_slot_of_brick;           // [B] -> position among X-min bricks or -1
        DBuf<float> inflow;                       // [inflow_faces]
        bool inflow_set = false;
        std::vector<uint8_t> h_connected;       // freestream_connected
        std::vector<int> xface_dof;             // [bricks with XMIN/XMAX faces] helper for initialisation
        pcfd_case config{};
        bool configured = false, initialized = false;
        double physical_time = 0.0, h_finest = 0.0;

        ~System();
    };

    // Every kernel launch takes its stream from here, so the system counts its own launches.
    inline cudaStream_t launch_stream(System& s)
    {
        ++s.launches;
        return s.stream;
    }

    // Programmatic dependent launch for chains of short dependent kernels (the multigrid stages):
    // launch_chained lets the kernel be scheduled while the previous kernel on the stream drains.
    // Such a kernel starts with chain_wait() (it returns once the previous grid has completed and
    // its memory is visible), so nothing it reads or writes overlaps the previous kernel, and then
    // calls chain_release() so that the next kernel may be scheduled once all its CTAs run.
    // Without a programmatic predecessor both are no-ops.
    __device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
    __device__ __forceinline__ void chain_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
    template <typename T> struct Exactly { using type = T; };   // keeps Params deduced from the kernel only
    template <typename... Params>
    inline void launch_chained(System& s, void (*kernel)(Params...), unsigned grid, unsigned block,
                               typename Exactly<Params>::type... args)
    {
        cudaLaunchConfig_t config{};
        config.gridDim = dim3(grid);
        config.blockDim = dim3(block);
        config.dynamicSmemBytes = 0;
        config.stream = launch_stream(s);
        cudaLaunchAttribute attribute{};
        attribute.id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attribute.val.programmaticStreamSerializationAllowed = 1;
        config.attrs = &attribute;
        config.numAttrs = 1;
        cuda_check(cudaLaunchKernelEx(&config, kernel, args...), "chained launch");
    }

    // Records a start/stop event pair on the system stream around one launch of the region being
    // profiled; a no-op for every other region or once the event capacity is used up.
    struct ProfileScope
    {
        System& s;
        bool on;
        ProfileScope(System& sys, int region)
            : s(sys), on(region >= 0 && sys.profile_region == region && 2 * (sys.profile_used + 1) <= int(sys.profile_events.size()))
        {
            if (on) cuda_check(cudaEventRecord(s.profile_events[2 * s.profile_used], s.stream), "profile event");
        }
        ~ProfileScope()
        {
            if (on) cudaEventRecord(s.profile_events[2 * s.profile_used++ + 1], s.stream);
        }
    };

    // ---- kernels / launchers (pressure.cu) ----
    void launch_apply(System& s, const double* p, double* out, bool orthogonal_only);
    // same operator with the WLS gradient scratch in a static device array (pressure.cu)
    void launch_apply_noalloc(System& s, const double* p, double* out, bool orthogonal_only);
    void launch_apply32(System& s, const float* p, float* out);
    double device_dot(System& s, const double* a, const double* b);
    void build_operator(System& s, const pcfd_topology& t);
    void build_multigrid(System& s, const pcfd_topology& t, const std::vector<double>& diagonal);
    void apply_preconditioner(System& s, const double* r, double* z);
    // 0: pre-smoothing (first Jacobi sweep pair), 1: coarse-grid correction, 2: post-smoothing
    void preconditioner_stage(System& s, int stage, const double* r, double* z);
    // fused fine level (smoother.cu) around the coarse hierarchy below it (solver.cu)
    void build_fine_smoother(System& s, const pcfd_topology& t, const std::vector<double>& diagonal);
    void attach_deferred_map(System& s);
    void brick_apply(System& s, const double* p, double* out);   // code-byte structured operator
    void fine_preconditioner_stage(System& s, int stage, const double* r, double* z);
    template <class T> void fine_preconditioner(System& s, const double* r, double* z, std::vector<MgLevel<T>>& levels);
    template <class T> void multigrid_levels(System& s, std::vector<MgLevel<T>>& levels);
    void build_composite(System& s, const pcfd_topology& t);
    void composite_levels(System& s);                 // V-cycle below the fine level, composite chain
    int64_t krylov_sweep_entries(const System& s);    // vector entries the Krylov block kernels sweep
    void composite_preconditioner(System& s, const double* r, double* z);   // smoother.cu
    void learned_preconditioner(System& s, const double* r, double* z, bool coarse);   // smoother.cu
    pcfd_solve_result solve(System& s, double* x, const double* b, double tolerance, int max_iterations, bool warm);
    void allocate_gcro(System& s);   // GCRO/LGMRES basis storage (capi.cu), idempotent
    pcfd_solve_result resolve_projection(System& s, double tolerance, int max_iterations, double* ms);   // core.cu
    // ---- learned preconditioner (learned.cu) ----
    int64_t learned_parameter_count();
    void learned_destroy(System& s);
    void learned_set_parameters(System& s, const float* host, int64_t count);
    void learned_get_parameters(System& s, float* host, int64_t count);
    void learned_apply(System& s, const double* r, double* z);
    void learned_check(System& s);   // throws PCFD_TIMEOUT when a tensor-core wait gave up
    void learned_set_wait(System& s, double seconds, bool idle_barrier_once);
    void learned_harvest_begin(System& s, int capacity_pairs, int per_pair, uint64_t seed, int target);
    int64_t learned_harvest_stop(System& s);
    bool learned_harvesting(const System& s);
    void learned_harvest(System& s, const double* r, const double* z);
    double learned_train(System& s, int steps, int batch, double lr, uint64_t seed);
    double learned_evaluate(System& s, int n, const float* x, const float* target, float* zhat, float* gradients);
    // vector helpers
    void vec_copy_active(System& s, const double* src, double* dst);
    void vec_subtract(System& s, double* residual, const double* value);   // r = active ? r - v : 0
    void vec_axpy_active(System& s, double* y, const double* x, double a);
    void vec_scaled_copy_active(System& s, double* dst, const double* src, double a);
    void vec_zero(System& s, double* x);
    void vec_update_solution_residual(System& s, double* x, double* r, const double* d, const double* Ad, double alpha);
    void vec_update_direction(System& s, const double* z, double* d, double beta);

    // ---- fused block vector kernels (krylov.cu); all active-masked, deterministic ----
    void block_dot(System& s, const VecSet& Q, const double* w, double* out);   // out[0..|Q|) = Q^T w, out[|Q|] = w.w
    // w -= Q h; y += sign * U h[0..|U|); mode 1: out[0] = w'.w'; mode 2: out = Q^T w' then w'.w'
    void block_update(System& s, const VecSet& Q, const double* h, double* w, const VecSet& U, double sign, double* y, int mode,
                      double* out);
    void block_combine(System& s, const VecSet& Z, const Coefficients& c, double* y, bool accumulate);   // y (+)= Z c
    void scale_by_inverse_norm(System& s, double* dst, const double* src, const double* norm2);        // dst = src / sqrt(n2)
    // delayed CGS2 column step: reorthogonalise v against Q in place and write the next basis vector
    // from w; coefficient[0..4*kMaxSet+9) as dcgs_final_kernel documents (krylov.cu)
    void dcgs_pass(System& s, const VecSet& Q, double* v, const double* w, double* next, double* coefficient);
    // looks up the grid of every block kernel once (an occupancy query), before any stream capture
    void prime_block_grids();
    constexpr int kDcgsCoefficients = 4 * kMaxSet + 9;

    // ---- projection (projection.cu) ----
    void build_projection(System& s, const pcfd_topology& t);
    void launch_integrated_flux(System& s);
    void launch_normalize(System& s, double rho_over_dt, bool with_rhs);
    void launch_correct_fluxes(System& s, double rho, double dt);
    void launch_convert_pressure(System& s);
    void conservation_stats(System& s, double out[6]);
    int autotune_pipe(System& s, int iterations, int* ctas, double* apply_ms, double* sweep_ms);   // smoother.cu
    double stage_smooth_bytes(const System& s);   // solver.cu: algorithmic bytes of one first-stage smoothing step
    void stage_smooth_once(System& s);            // solver.cu: one first-stage Chebyshev step (kernel timing)
    // point location and slice sampling (locator.cu)
    void build_locator(System& s, const pcfd_topology& t);
    void destroy_locator(System& s);
    // staggered MAC momentum mode (mac.cu)
    void build_mac(System& s, const pcfd_topology& t);
    void destroy_mac(System& s);
    void mac_set_links(System& s, const uint8_t* const host[3]);
    void mac_advect(System& s, float dt);
    void mac_diffuse_smagorinsky(System& s, float nu, float cs, float dt);
    void mac_eddy_viscosity(System& s, float* host_nut);
    void build_apertures(System& s, const pcfd_topology& t);   // mac_apertures.cu
    void destroy_apertures(System& s);
    void mac_transport_apertures(System& s, float dt, float nu, float cs);
    void mac_sync_coarse_fine(System& s);
    void mac_smooth_wall(System& s, float dt, float nu);
    float mac_embedded_cfl_rate(System& s);
    float mac_max_special_speed(System& s);
    float mac_max_face_speed(System& s);       // mac.cu
    bool mac_ready(const System& s);
    void locate_points(System& s, const float* d_points, int count, int* d_out);
    void sample_slice(System& s, const double origin[3], const double edge_u[3], const double edge_v[3], int nu, int nv,
                      int field, float* d_out);   // [max |div|, rms, worst V, max |div V|, sum |div V|, sum div V]

    // face array index helpers (compact per-brick layout)
    __host__ __device__ inline int64_t u_face(int bs, int64_t slot, int i, int j, int k)
    {
        return slot * int64_t((bs + 1) * bs * bs) + int64_t((k * bs + j) * (bs + 1) + i);
    }
    __host__ __device__ inline int64_t v_face(int bs, int64_t slot, int i, int j, int k)
    {
        return slot * int64_t((bs + 1) * bs * bs) + int64_t((k * (bs + 1) + j) * bs + i);
    }
    __host__ __device__ inline int64_t w_face(int bs, int64_t slot, int i, int j, int k)
    {
        return slot * int64_t((bs + 1) * bs * bs) + int64_t((k * bs + j) * bs + i);
    }
    __host__ __device__ inline int64_t axis_face(int bs, int axis, int64_t slot, int i, int j, int k)
    {
        return axis == 0 ? u_face(bs, slot, i, j, k) : (axis == 1 ? v_face(bs, slot, i, j, k) : w_face(bs, slot, i, j, k));
    }

    inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

    constexpr int kThreads = 256;
    inline int blocks_for(int64_t n, int threads = kThreads) { return int((n + threads - 1) / threads); }
}
