// adapter_probe.cpp -- runs the reference-side adapter (ExternalAeroCoreB200,
// external_aero_core_b200.h) beside the reference's own ExternalAeroCore on the same fixture and
// prints one JSON line: convergence, dt and the largest cell-momentum difference (relative to the
// freestream) after initialize and every step, and both pressure-load integrals at the end.
// TEST INFRASTRUCTURE (tests/test_adapter_gpu.py); needs a GPU.
//
//   adapter_probe [steps] [base_cell_size]
#include "../ref_shim.h"
#include "external_aero_core_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace paracfd_b200_adapter;

int main(int argc, char** argv)
{
    const int steps = argc > 1 ? std::atoi(argv[1]) : 3;
    const double h = argc > 2 ? std::atof(argv[2]) : 1.0 / 16.0;
    ref_case_params params;
    ref_default_params(REF_CASE_NACA_SLAB, &params);
    params.base_cell_size = h;
    void* rc = ref_case_create(&params);
    if (!rc) { std::fprintf(stderr, "reference case: %s\n", ref_last_error()); return 2; }
    const void *hp = nullptr, *sp = nullptr, *cp = nullptr;
    ref_case_objects(rc, &hp, &sp, &cp);
    const auto& hierarchy = *static_cast<const AmrHierarchy*>(hp);
    const auto& system = *static_cast<const CompositeAmrPressureSystem*>(sp);
    ParagliderConfig config = *static_cast<const ParagliderConfig*>(cp);
    config.freestream.speed = 10.0;
    config.freestream.rho = 1.225;
    config.freestream.nu = 1.5e-5;
    config.solver.cfl = 0.5;
    config.solver.smagorinsky_cs = 0.10;
    config.solver.projection_tolerance = 1e-8;
    config.solver.projection_max_iterations = 600;
    try
    {
        ExternalAeroCoreB200 ours(hierarchy, system, config);
        ref_core_case cc{config.freestream.speed, config.freestream.rho, config.freestream.nu, config.solver.cfl,
                         config.solver.smagorinsky_cs, config.solver.projection_tolerance,
                         config.solver.projection_max_iterations};
        void* theirs = ref_core_create(rc, &cc);
        if (!theirs) { std::fprintf(stderr, "reference core: %s\n", ref_last_error()); return 2; }
        const std::size_t n = std::size_t(system.storage_size);
        std::vector<float> rx(n), ry(n), rz(n);
        std::vector<double> rp(n);
        auto compare = [&](const char* what, const ExternalAeroStepStats& a, const double* b) {
            CompositeCellMomentumState st;
            ours.download_cell_momentum_state(st);
            ref_core_state(theirs, rx.data(), ry.data(), rz.data(), rp.data());
            double diff = 0, scale = 0;
            for (std::size_t q = 0; q < n; ++q)
            {
                if (!system.active[q]) continue;
                scale = std::max(scale, double(std::abs(rx[q])));
                diff = std::max({diff, double(std::abs(st.x[q] - rx[q])), double(std::abs(st.y[q] - ry[q])),
                                 double(std::abs(st.z[q] - rz[q]))});
            }
            std::printf("{\"%s\": {\"converged\": [%d, %d], \"dt\": [%.17g, %.17g], \"state_error\": %.6g}}, ", what,
                        int(a.pressure.converged), int(b[4] != 0), a.dt, b[0], diff / std::max(scale, 1e-30));
        };
        double stats[6];
        std::printf("{\"records\": [");
        const ExternalAeroStepStats init = ours.initialize();
        ref_core_initialize(theirs, stats);
        compare("initialize", init, stats);
        for (int k = 0; k < steps; ++k)
        {
            const ExternalAeroStepStats s = ours.step();
            ref_core_step(theirs, stats);
            compare("step", s, stats);
        }
        // pressure loads: the adapter's (device integration of its pressure) and the reference's
        // compute_pressure_loads of its own pressure
        const AerodynamicLoads mine = ours.pressure_loads();
        FreestreamConfig fs;
        AeroReferenceConfig ref_cfg;
        const AerodynamicLoads ref_loads = compute_pressure_loads(system, rp, std::size_t(1) << 30, fs, ref_cfg, 0.0);
        std::printf("{\"loads\": {\"adapter\": [%.17g, %.17g, %.17g], \"reference\": [%.17g, %.17g, %.17g]}}]}\n",
                    mine.pressure_force.x, mine.pressure_force.y, mine.pressure_force.z, ref_loads.pressure_force.x,
                    ref_loads.pressure_force.y, ref_loads.pressure_force.z);
        ref_core_destroy(theirs);
    }
    catch (const std::exception& e)
    {
        std::fprintf(stderr, "adapter probe: %s\n", e.what());
        ref_case_destroy(rc);
        return 1;
    }
    ref_case_destroy(rc);
    return 0;
}
