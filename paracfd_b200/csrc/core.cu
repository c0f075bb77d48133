// core.cu -- time-step orchestration (ExternalAeroCore::initialize / step, reference
// src/core/fluid/external_aero_core.cpp:245-328) and the momentum entry points of the C ABI.
//
// Differences by design: every stage is enqueued on one stream with no device-wide syncs; the
// only host reads inside a step are the fused CFL reduction (4 floats), the diffusion spectral
// rate (1 float) and the Krylov scalars of the pressure solve.
#include "momentum.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace pcfd
{
    namespace
    {
        thread_local std::string* g_core_error = nullptr;

        __global__ void init_state_kernel(const uint8_t* active, const uint8_t* connected, int64_t n, float speed, float* x, float* y,
                                          float* z, float* xn, float* yn, float* zn)
        {
            const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (q >= n) return;
            const float vx = active[q] && connected[q] ? speed : 0.0f;
            x[q] = xn[q] = vx;
            y[q] = yn[q] = 0.0f;
            z[q] = zn[q] = 0.0f;
        }

        // X-boundary faces of the initial state: freestream where the adjacent CV is connected.
        __global__ void init_x_boundary_kernel(const int* brick_list, int nbricks, int bs, const uint32_t* flags, const uint8_t* active,
                                               const uint8_t* connected, float speed, float* u)
        {
            const int64_t work = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
            if (work >= int64_t(nbricks) * bs * bs) return;
            const int slot = brick_list[work / (bs * bs)], r = int(work % (bs * bs)), j = r % bs, k = r / bs;
            const uint32_t fl = flags[slot];
            const int64_t base = int64_t(slot) * bs * bs * bs + (k * bs + j) * bs;
            if (fl & PCFD_BRICK_XMIN) { const int64_t q = base; u[u_face(bs, slot, 0, j, k)] = active[q] && connected[q] ? speed : 0.0f; }
            if (fl & PCFD_BRICK_XMAX) { const int64_t q = base + bs - 1; u[u_face(bs, slot, bs, j, k)] = active[q] && connected[q] ? speed : 0.0f; }
        }
    }

    // the solver's starting state of a projection: warm-start pressure and recycled subspace
    void save_projection_start(System& s, bool warm)
    {
        const size_t n = size_t(s.Sp) * sizeof(double);
        s.start_saved = true;
        s.start_warm = warm;
        cuda_check(cudaMemcpyAsync(s.start_pressure, s.pressure, n, cudaMemcpyDeviceToDevice, s.stream), "save start");
        s.start_recycle_count = s.recycle_count;
        if (s.recycle_count)
        {
            cuda_check(cudaMemcpyAsync(s.start_recycle_u, s.recycle_u, n * s.recycle_count, cudaMemcpyDeviceToDevice, s.stream), "save U");
            cuda_check(cudaMemcpyAsync(s.start_recycle_c, s.recycle_c, n * s.recycle_count, cudaMemcpyDeviceToDevice, s.stream), "save C");
        }
    }

    // solves the last projection's system again from its saved start with the current
    // preconditioner; the pressure and recycled subspace end as that solve leaves them
    pcfd_solve_result resolve_projection(System& s, double tolerance, int max_iterations, double* ms)
    {
        require(s.keep_projection_start && s.start_saved, "no saved projection start");
        const size_t n = size_t(s.Sp) * sizeof(double);
        cuda_check(cudaMemcpyAsync(s.pressure, s.start_pressure, n, cudaMemcpyDeviceToDevice, s.stream), "restore start");
        s.recycle_count = s.start_recycle_count;
        if (s.recycle_count)
        {
            cuda_check(cudaMemcpyAsync(s.recycle_u, s.start_recycle_u, n * s.recycle_count, cudaMemcpyDeviceToDevice, s.stream), "restore U");
            cuda_check(cudaMemcpyAsync(s.recycle_c, s.start_recycle_c, n * s.recycle_count, cudaMemcpyDeviceToDevice, s.stream), "restore C");
        }
        cudaEvent_t start, stop;
        cuda_check(cudaEventCreate(&start), "event");
        cuda_check(cudaEventCreate(&stop), "event");
        cuda_check(cudaEventRecord(start, s.stream), "event");
        const pcfd_solve_result r = solve(s, s.pressure, s.rhs, tolerance, max_iterations, s.start_warm);
        cuda_check(cudaEventRecord(stop, s.stream), "event");
        cuda_check(cudaEventSynchronize(stop), "event");
        float t = 0;
        cuda_check(cudaEventElapsedTime(&t, start, stop), "event");
        cudaEventDestroy(start);
        cudaEventDestroy(stop);
        *ms = t;
        return r;
    }

    Momentum& momentum_of(System& s)
    {
        require(s.momentum && s.momentum->ready, "cell-momentum topology was not built");
        return *s.momentum;
    }

    // Extrapolation in time from the last converged pressures, elementwise: with order 1,
    // p <- 2 p - previous; with order 2, p <- 3 p - 3 previous + previous2 and previous2 <- previous;
    // then previous <- p (the old p).  previous2 may be null for order 1.
    __global__ void extrapolate_pressure_kernel(double* __restrict__ p, double* __restrict__ previous, double* __restrict__ previous2,
                                                int64_t n, int order)
    {
        const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
        if (q >= n) return;
        const double a = p[q], b = previous[q];
        if (order == 2)
        {
            const double c = previous2[q];
            previous2[q] = b;
            p[q] = 3.0 * (a - b) + c;
        }
        else
        {
            if (previous2) previous2[q] = b;
            p[q] = 2.0 * a - b;
        }
        previous[q] = a;
    }

    // the initial guess of a warm step projection (pcfd_core_set_initial_guess): the highest
    // extrapolation order the valid history allows, up to the chosen one
    void initial_guess(System& s, bool warm)
    {
        if (!warm) { s.previous_count = 0; return; }
        if (s.initial_guess == 0 || !s.pressure_previous.p) return;
        const int order = std::min(s.initial_guess, s.previous_count);
        if (order == 0)
            cuda_check(cudaMemcpyAsync(s.pressure_previous, s.pressure, size_t(s.S) * sizeof(double), cudaMemcpyDeviceToDevice, s.stream),
                       "keep pressure");
        else
            extrapolate_pressure_kernel<<<blocks_for(s.S), kThreads, 0, launch_stream(s)>>>(s.pressure, s.pressure_previous,
                                                                                           s.pressure_previous2.p, s.S, order);
        s.previous_count = std::min(s.previous_count + 1, s.initial_guess);
    }

    pcfd_solve_result project(System& s, double rho, double dt, double tolerance, int max_iterations, bool warm)
    {
        launch_integrated_flux(s);
        launch_normalize(s, rho / dt, true);
        initial_guess(s, warm);
        if (s.keep_projection_start) save_projection_start(s, warm);
        const pcfd_solve_result r = solve(s, s.pressure, s.rhs, tolerance, max_iterations, warm);
        if (!r.converged) s.previous_count = 0;
        if (r.converged)
        {
            launch_convert_pressure(s);
            launch_correct_fluxes(s, rho, dt);
            launch_integrated_flux(s);
            launch_normalize(s, 0.0, false);
        }
        return r;
    }

    void core_initialize(System& s, pcfd_step_stats& stats)
    {
        require(s.configured, "core is not configured");
        Momentum& m = momentum_of(s);
        const pcfd_case& c = s.config;
        const float speed = float(c.speed);
        DBuf<uint8_t> connected;
        connected.upload(s.h_connected);
        init_state_kernel<<<blocks_for(s.S), kThreads, 0, launch_stream(s)>>>(s.active, connected, s.S, speed, m.x, m.y, m.z, m.xn, m.yn, m.zn);
        cuda_check(cudaMemsetAsync(s.u, 0, size_t(s.faces) * sizeof(float), s.stream), "clear faces");
        cuda_check(cudaMemsetAsync(s.v, 0, size_t(s.faces) * sizeof(float), s.stream), "clear faces");
        cuda_check(cudaMemsetAsync(s.w, 0, size_t(s.faces) * sizeof(float), s.stream), "clear faces");
        cuda_check(cudaMemsetAsync(s.special, 0, size_t(s.cf_count + s.eb_count) * sizeof(float), s.stream), "clear special");
        momentum_reconstruct_fluxes(s, m);
        if (s.active_bricks)
            init_x_boundary_kernel<<<blocks_for(int64_t(s.active_bricks) * s.bs * s.bs), kThreads, 0, launch_stream(s)>>>(
                s.active_brick_list, s.active_bricks, s.bs, s.brick_flags, s.active, connected, speed, s.u);
        momentum_external_boundaries(s, speed);
        const double maximum = std::max(1e-9, std::abs(c.speed));
        const double dt = c.cfl * s.h_finest / maximum;
        vec_zero(s, s.pressure);
        std::memset(&stats, 0, sizeof(stats));
        if (s.momentum_mode == PCFD_MOMENTUM_MAC)
        {
            // the MAC mode carries no cell momentum: the projection syncs the coarse/fine slots
            // from the fine faces first and no impulse follows (external_aero_core.cpp:296-300)
            mac_sync_coarse_fine(s);
            stats.pressure = project(s, c.rho, dt, c.projection_tolerance, c.projection_max_iterations, false);
            stats.dt = dt;
            stats.max_abs_velocity = mac_max_face_speed(s);
            stats.max_abs_special_velocity = mac_max_special_speed(s);
            stats.cfl_velocity = maximum;
            stats.effective_cfl = maximum * dt / s.h_finest;
            s.initialized = stats.pressure.converged != 0;
            stats.physical_time = s.physical_time;
            cuda_check(cudaStreamSynchronize(s.stream), "initialize");
            return;
        }
        stats.pressure = project(s, c.rho, dt, c.projection_tolerance, c.projection_max_iterations, false);
        if (c.pressure_impulse && stats.pressure.converged) momentum_pressure_impulse(s, m, float(dt), float(c.rho), true);
        float cfl[4];
        momentum_cfl(s, m, true, cfl);
        stats.dt = dt;
        stats.max_abs_velocity = cfl[0];
        stats.max_abs_special_velocity = cfl[2];
        stats.cfl_velocity = maximum;
        stats.effective_cfl = maximum * dt / s.h_finest;
        s.initialized = stats.pressure.converged != 0;
        stats.physical_time = s.physical_time;
        cuda_check(cudaStreamSynchronize(s.stream), "initialize");
    }

    // ExternalAeroCore::step with the staggered MAC momentum (external_aero_core.cpp:304-311,
    // 321-325): CFL from the regular faces, the special velocities and the EB aperture rate;
    // MacCormack advection, LES + face diffusion, boundaries, compact aperture transport, the
    // smooth fabric wall, then the projection with the coarse/fine slots synced from the fine faces.
    void core_step_mac(System& s, pcfd_step_stats& stats)
    {
        const pcfd_case& c = s.config;
        cudaEvent_t e0, e1, p0, p1;
        cuda_check(cudaEventCreate(&e0), "event"); cuda_check(cudaEventCreate(&e1), "event");
        cuda_check(cudaEventCreate(&p0), "event"); cuda_check(cudaEventCreate(&p1), "event");
        cuda_check(cudaEventRecord(e0, s.stream), "event");
        std::memset(&stats, 0, sizeof(stats));
        const float face_max = mac_max_face_speed(s), special_max = mac_max_special_speed(s), eb_rate = mac_embedded_cfl_rate(s);
        if (!std::isfinite(face_max) || !std::isfinite(special_max) || !std::isfinite(eb_rate))
            throw Error(PCFD_INTERNAL, "non-finite regular or embedded-boundary velocity before the time step");
        const double cfl_rate = std::max({1e-9, std::abs(c.speed) / s.h_finest, double(face_max) / s.h_finest, double(eb_rate)});
        const double dt_value = c.cfl / cfl_rate;
        const float dt = float(dt_value), nu = float(c.nu), cs = float(c.smagorinsky_cs), speed = float(c.speed), rho = float(c.rho);
        mac_advect(s, dt);
        mac_diffuse_smagorinsky(s, nu, cs, dt);
        momentum_external_boundaries(s, speed);
        mac_transport_apertures(s, dt, nu, cs);
        if (c.smooth_wall) mac_smooth_wall(s, dt, nu);
        mac_sync_coarse_fine(s);
        cuda_check(cudaEventRecord(p0, s.stream), "event");
        stats.pressure = project(s, double(rho), dt_value, c.projection_tolerance, c.projection_max_iterations, true);
        cuda_check(cudaEventRecord(p1, s.stream), "event");
        cuda_check(cudaEventRecord(e1, s.stream), "event");
        cuda_check(cudaEventSynchronize(e1), "step");
        float ms = 0, pms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventElapsedTime(&pms, p0, p1);
        cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(p0); cudaEventDestroy(p1);
        stats.dt = dt_value;
        stats.max_abs_velocity = std::max(face_max, special_max);
        stats.max_abs_special_velocity = special_max;
        stats.max_outflow_rate = eb_rate;
        stats.cfl_velocity = cfl_rate * s.h_finest;
        stats.effective_cfl = cfl_rate * dt_value;
        stats.step_ms = ms;
        stats.projection_ms = pms;
        if (stats.pressure.converged) s.physical_time += dt_value;
        stats.physical_time = s.physical_time;
    }

    void core_step(System& s, pcfd_step_stats& stats)
    {
        require(s.initialized, "the core needs a converged initialization before stepping");
        if (s.momentum_mode == PCFD_MOMENTUM_MAC) { core_step_mac(s, stats); return; }
        Momentum& m = momentum_of(s);
        const pcfd_case& c = s.config;
        cudaEvent_t e0, e1, p0, p1;
        cuda_check(cudaEventCreate(&e0), "event"); cuda_check(cudaEventCreate(&e1), "event");
        cuda_check(cudaEventCreate(&p0), "event"); cuda_check(cudaEventCreate(&p1), "event");
        cuda_check(cudaEventRecord(e0, s.stream), "event");
        std::memset(&stats, 0, sizeof(stats));
        float cfl[4];
        momentum_cfl(s, m, true, cfl);
        if (!std::isfinite(cfl[0]) || !std::isfinite(cfl[1]) || !std::isfinite(cfl[2]))
            throw Error(PCFD_INTERNAL, "non-finite cell or special velocity before the time step");
        const double cfl_rate = std::max({1e-9, std::abs(c.speed) / s.h_finest, double(cfl[1])});
        const double dt_value = c.cfl / cfl_rate;
        const float dt = float(dt_value), nu = float(c.nu), cs = float(c.smagorinsky_cs), speed = float(c.speed), rho = float(c.rho);
        momentum_transport(s, m, dt, speed, true);
        stats.max_diffusion_rate = momentum_smagorinsky(s, m, nu, cs, dt);
        stats.diffusion_substeps = m.last_substeps;
        if (c.smooth_wall) momentum_wall(s, m, dt, nu);
        momentum_reconstruct_fluxes(s, m);
        momentum_external_boundaries(s, speed);
        cuda_check(cudaEventRecord(p0, s.stream), "event");
        stats.pressure = project(s, double(rho), dt_value, c.projection_tolerance, c.projection_max_iterations, true);
        cuda_check(cudaEventRecord(p1, s.stream), "event");
        if (c.pressure_impulse && stats.pressure.converged) momentum_pressure_impulse(s, m, dt, rho, true);
        cuda_check(cudaEventRecord(e1, s.stream), "event");
        cuda_check(cudaEventSynchronize(e1), "step");
        float ms = 0, pms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventElapsedTime(&pms, p0, p1);
        cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(p0); cudaEventDestroy(p1);
        stats.dt = dt_value;
        stats.max_abs_velocity = cfl[0];
        stats.max_abs_special_velocity = cfl[2];
        stats.max_outflow_rate = cfl[1];
        stats.cfl_velocity = cfl_rate * s.h_finest;
        stats.effective_cfl = cfl_rate * dt_value;
        stats.step_ms = ms;
        stats.projection_ms = pms;
        if (stats.pressure.converged) s.physical_time += dt_value;
        stats.physical_time = s.physical_time;
    }
}
