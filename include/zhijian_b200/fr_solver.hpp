// fr_solver.hpp -- header-only C++ facade over the C-ABI (zj_fr.h) with the
// method names and argument meanings of the reference zhijian::FRSolver
// (include/solver/fr_solver.hpp:77-180 in the Zhijian project), so a caller of
// that class switches by changing its include and namespace.
//
// Differences from the reference, all at the boundary:
//  - errors throw zhijian_b200::Error (code + text) instead of std::exit;
//  - the mesh is passed as plain arrays (Mesh / zj_mesh_desc) instead of the
//    reference's Mesh class, and is not borrowed beyond initialize();
//  - advance() queues the step; solution()/copyToHost() synchronise.
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "zj_fr.h"

namespace zhijian_b200 {

struct Vec2 {
    double x = 0.0, y = 0.0;
};
using State = std::array<double, 4>;   // rho, rho*u, rho*v, rho*E

class Error : public std::runtime_error {
public:
    Error(zj_status code, const std::string& what) : std::runtime_error(what), code_(code) {}
    zj_status code() const { return code_; }

private:
    zj_status code_;
};

inline void check(zj_status st, const zj_solver* s) {
    if (st != ZJ_OK) throw Error(st, std::string("zj error ") + std::to_string(st) + ": " + zj_last_error(s));
}

// Quad mesh as arrays: nodes, CCW element connectivity (4, 9 or 25 nodes per
// element), boundary edges (v0, v1, tag).
struct Mesh {
    std::vector<double> xy;                  // [n_nodes][2]
    std::vector<int64_t> conn;               // [n_elem][nodes_per_elem]
    int nodes_per_elem = 4;
    std::vector<int64_t> boundary_edges;     // [n][3]
    int64_t numNodes() const { return (int64_t)xy.size() / 2; }
    int64_t numElements() const { return (int64_t)conn.size() / nodes_per_elem; }
};

class FRSolver {
public:
    FRSolver() = default;
    ~FRSolver() { zj_solver_destroy(s_); }
    FRSolver(const FRSolver&) = delete;
    FRSolver& operator=(const FRSolver&) = delete;

    // FRSolver::initialize(const Mesh&, const SimParams&) (fr_solver.cpp:30-73)
    void initialize(const Mesh& m, const zj_params& params) {
        const int64_t ne = m.numElements();
        std::vector<int32_t> type(ne, ZJ_ELEM_QUAD);
        const int order = m.nodes_per_elem == 4 ? 1 : m.nodes_per_elem == 9 ? 2 : 4;
        std::vector<int32_t> ord(ne, order);
        std::vector<int64_t> off(ne + 1);
        for (int64_t e = 0; e <= ne; ++e) off[e] = e * m.nodes_per_elem;
        zj_mesh_desc d{m.numNodes(), m.xy.data(), ne, type.data(), ord.data(), off.data(),
                       m.conn.data(), (int64_t)m.boundary_edges.size() / 3, m.boundary_edges.data()};
        zj_solver_destroy(s_);
        s_ = nullptr;
        check(zj_solver_create(&d, &params, &s_), nullptr);
        params_ = params;
        n_sp_ = zj_num_solution_points(s_);
        n_elem_ = zj_num_elements(s_);
    }

    // The mesh from a Gmsh file (GmshReader::read, gmsh_reader.cpp:161-760, as
    // main.cpp's -m option loads it), boundary types from its physical names.
    void initializeFromGmsh(const std::string& path, const zj_params& params) {
        zj_solver_destroy(s_);
        s_ = nullptr;
        check(zj_solver_create_from_gmsh(path.c_str(), &params, &s_), nullptr);
        params_ = params;
        n_sp_ = zj_num_solution_points(s_);
        n_elem_ = zj_num_elements(s_);
    }

    // FRSolver::setInitialCondition(std::function<State(Vec2)>) (fr_solver.cpp:268-299)
    void setInitialCondition(const std::function<State(Vec2)>& ic) {
        std::vector<double> xy((size_t)n_elem_ * n_sp_ * 2);
        check(zj_solution_point_coords(s_, xy.data()), s_);
        host_.resize((size_t)n_elem_ * n_sp_ * 4);
        for (size_t k = 0; k < (size_t)n_elem_ * n_sp_; ++k) {
            const State st = ic(Vec2{xy[2 * k], xy[2 * k + 1]});
            for (int v = 0; v < 4; ++v) host_[4 * k + v] = st[v];
        }
        check(zj_set_state(s_, host_.data()), s_);
    }

    // FRSolver::advance(Real dt) (fr_solver.cpp:305-333)
    void advance(double dt) { check(zj_step(s_, dt, 1), s_); }
    void advance(double dt, int nsteps) { check(zj_step(s_, dt, nsteps), s_); }

    // FRSolver::computeTimeStep() (fr_solver.cpp:784-816), on the device state
    double computeTimeStep() const {
        double dt = 0.0;
        check(zj_compute_dt(s_, &dt), s_);
        return dt;
    }

    // FRSolver::computeResidual() (fr_solver.cpp:818-833)
    double computeResidual() const {
        double r = 0.0;
        check(zj_residual_norm(s_, &r), s_);
        return r;
    }

    double currentTime() const { return zj_time(s_); }
    int currentIteration() const { return zj_iteration(s_); }

    // RestartIO::write / read (src/io/restart.cpp:8-144) in the library's
    // dependency-free restart format; reading resumes time and iteration.
    void writeRestart(const std::string& path) { check(zj_restart_write(s_, path.c_str()), s_); }
    void readRestart(const std::string& path) { check(zj_restart_read(s_, path.c_str()), s_); }
    int iteration() const { return zj_iteration(s_); }

    // FRSolver::copyToHost / copyToDevice (fr_solver.cpp:835-871): the flat
    // [element][solution point][variable] array stands in for ElementSolution.
    void copyToHost() {
        host_.resize((size_t)zj_state_size(s_));
        check(zj_get_state(s_, host_.data()), s_);
    }
    void copyToDevice() { check(zj_set_state(s_, host_.data()), s_); }
    const std::vector<double>& solution() const { return host_; }
    std::vector<double>& solution() { return host_; }
    // Queued copies of a caller's host buffer (zj_set_state_async /
    // zj_get_state_async): the buffer stays alive and unchanged until
    // synchronize(); page-locked buffers overlap the copy with other streams.
    void copyToDeviceAsync(const double* U) { check(zj_set_state_async(s_, U), s_); }
    void copyToHostAsync(double* U) { check(zj_get_state_async(s_, U), s_); }
    void synchronize() { check(zj_synchronize(s_), s_); }
    // Blocks of six steps replayed from captured CUDA graphs (default on).
    void setStepGraphs(bool enable) { check(zj_set_step_graphs(s_, enable ? 1 : 0), s_); }

    const zj_params& params() const { return params_; }
    zj_solver* handle() { return s_; }

private:
    zj_solver* s_ = nullptr;
    zj_params params_{};
    int n_sp_ = 0;
    int64_t n_elem_ = 0;
    std::vector<double> host_;
};

}  // namespace zhijian_b200
