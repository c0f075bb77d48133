// momentum.h -- collocated cell-momentum transport state (FP32 control-volume velocity) and the
// compact topology it needs beyond the pressure system.
#pragma once

#include "pcfd_internal.h"

namespace pcfd
{
    // cell_code bits (one byte per pressure DOF, read by every brick kernel of the momentum path)
    enum : uint8_t
    {
        CODE_CUT_MASK = 0x07,       // +X/+Y/+Z regular face suppressed by the cut geometry
        CODE_COMPACT_SHIFT = 3,     // +X/+Y/+Z face owned by a compact perimeter edge (bits 3..5)
        CODE_DEFERRED = 0x40,       // finished by the compact per-DOF pass (compact edges/groups/walls)
        CODE_ACTIVE = 0x80
    };

    struct Momentum
    {
        bool ready = false;
        // compact edges: [0,nR) regular perimeter, [nR,nR+nC) coarse/fine, [nR+nC,nK) embedded
        int nR = 0, nC = 0, nE = 0, nK = 0;
        DBuf<int> k_a, k_b, k_source;          // source: face array index class (see kernels)
        DBuf<int8_t> k_axis;
        DBuf<int64_t> k_face;                  // canonical face (regular perimeter edges)
        DBuf<float> k_area, k_conductance, k_weight, k_disp;   // disp: [nK][6]
        DBuf<int> k_pnode_a, k_pnode_b;        // pressure WLS node of each endpoint or -1
        // least-squares velocity-gradient nodes
        int nS = 0;
        DBuf<int> s_dof, s_offset, s_neighbor;
        DBuf<float> s_weight, s_inverse, s_gradient;           // [inc][3], [nS][9], [nS][9]
        DBuf<int> k_sa, k_sb;                  // special index of each edge endpoint or -1
        // per DOF
        DBuf<uint8_t> code, special;
        DBuf<float> volume32;
        // deferred DOFs
        int nD = 0;
        DBuf<int> d_dof, d_offset, d_edge, d_group;            // CSR of incident compact edges
        DBuf<int8_t> d_sign;
        DBuf<float> d_delta;                   // [nD][3] total increment (group pass input)
        // redistribution groups
        int nG = 0;
        DBuf<int> g_offset, g_member;          // members as deferred indices
        DBuf<float> g_volume;
        // smooth wall: sides (one per patch side), wall nodes (unique DOFs)
        int nW = 0, nWall = 0;
        DBuf<int> w_dof, w_node, w_pnode;
        DBuf<float> w_normal, w_area, w_distance, w_coefficient, w_disp, w_k, w_force;
        DBuf<int> wall_dof, wall_offset, wall_side;
        // boundary pressure faces
        int nB = 0;
        DBuf<int> b_dof;
        DBuf<float> b_coefficient;
        DBuf<int> d_boundary_offset, d_boundary;               // per deferred DOF
        DBuf<int> d_side_offset, d_side;                       // surface sides per deferred DOF
        // pressure WLS gradient in FP32 (impulse reconstruction)
        DBuf<float> p_weight, p_gradient;
        // state (double-buffered) and scratch
        DBuf<float> x, y, z, xn, yn, zn, dx, dy, dz, viscosity, baseline_x, baseline_y, baseline_z;
        DBuf<float> reduce_partial;            // [blocks][4]
        DBuf<float> reduce_result;             // [4]
        float* pinned = nullptr;
        int last_substeps = 1;
        double last_rate = 0;
        double min_volume_fraction = 0;
        ~Momentum();
    };

    void build_momentum(System& s, Momentum& m, const pcfd_topology& t, double minimum_volume_fraction);
    // transport / diffusion / wall / impulse / reconstruction (momentum.cu)
    void momentum_transport(System& s, Momentum& m, float dt, float freestream, bool external_aero);
    double momentum_smagorinsky(System& s, Momentum& m, float nu, float cs, float dt);   // returns rate
    void momentum_wall(System& s, Momentum& m, float dt, float nu);
    void momentum_pressure_impulse(System& s, Momentum& m, float dt, float rho, bool physical_boundaries);
    void momentum_reconstruct_fluxes(System& s, Momentum& m);
    void momentum_external_boundaries(System& s, float speed);
    // [max |v| over cells, max outflow rate, max |special velocity|, max EB cfl rate]
    void momentum_cfl(System& s, Momentum& m, bool external_aero, float out[4]);

    // surface loads (loads.cu): out = [pressure F(3), pressure M(3), viscous F(3), viscous M(3)]
    void build_loads(System& s, const pcfd_topology& t);
    void destroy_loads(System& s);
    void compute_loads(System& s, double pref, const double origin[3], double rho, bool viscous, double out[12]);

    // time step (core.cu)
    Momentum& momentum_of(System& s);
    pcfd_solve_result project(System& s, double rho, double dt, double tolerance, int max_iterations, bool warm);
    void core_initialize(System& s, pcfd_step_stats& stats);
    void core_step(System& s, pcfd_step_stats& stats);
}
