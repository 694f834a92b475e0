// zj_run.cpp -- C++ driver over the FRSolver facade, the counterpart of the
// reference's time loop (src/main.cpp:395-476): config file with the
// reference grammar, a structured quad mesh, uniform-flow or isentropic-vortex
// initial state, then computeTimeStep -> advance -> computeResidual.
//
//   zj_run <config> (<nx> <ny> <x0> <x1> <y0> <y1> | -m <mesh.msh>) [steps] [vortex]
//          [-r <restart file>] [-w <restart file>]
// -m reads the mesh from a Gmsh file as the reference's -m does (boundary
// types from the physical names); otherwise a structured quad mesh.
// prints "iter time dt residual" every 10 iterations and the final state
// checksum (sum of |U|) on the last line.  -r resumes from a restart file
// (state, time, iteration; src/main.cpp:345-360), -w writes one every
// restart_freq iterations and at the end (src/main.cpp:455-466).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "zhijian_b200/fr_solver.hpp"

using zhijian_b200::FRSolver;
using zhijian_b200::Mesh;
using zhijian_b200::State;
using zhijian_b200::Vec2;

static Mesh structured(int nx, int ny, double x0, double x1, double y0, double y1) {
    Mesh m;
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            m.xy.push_back(x0 + (x1 - x0) * i / nx);
            m.xy.push_back(y0 + (y1 - y0) * j / ny);
        }
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            int64_t n0 = (int64_t)j * (nx + 1) + i;
            m.conn.insert(m.conn.end(), {n0, n0 + 1, n0 + nx + 2, n0 + nx + 1});
        }
    auto edge = [&](int64_t a, int64_t b) { m.boundary_edges.insert(m.boundary_edges.end(), {a, b, 1}); };
    for (int i = 0; i < nx; ++i) edge(i, i + 1);
    for (int j = 0; j < ny; ++j) edge((int64_t)j * (nx + 1) + nx, (int64_t)(j + 1) * (nx + 1) + nx);
    for (int i = nx; i > 0; --i) edge((int64_t)ny * (nx + 1) + i, (int64_t)ny * (nx + 1) + i - 1);
    for (int j = ny; j > 0; --j) edge((int64_t)j * (nx + 1), (int64_t)(j - 1) * (nx + 1));
    return m;
}

int main(int argc, char** argv) {
    const bool from_file = argc >= 4 && std::string(argv[2]) == "-m";
    if (!from_file && argc < 8) {
        std::fprintf(stderr, "usage: zj_run <config> (<nx> <ny> <x0> <x1> <y0> <y1> | -m <mesh.msh>) "
                             "[steps] [vortex] [-r <restart>] [-w <restart>]\n");
        return 1;
    }
    zj_params p;
    zj_params_default(&p);
    if (zj_params_parse_file(argv[1], &p) != ZJ_OK) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 1;
    }
    std::string restart_in, restart_out;
    std::vector<std::string> pos;
    for (int a = from_file ? 4 : 8; a < argc; ++a) {
        const std::string arg = argv[a];
        if ((arg == "-r" || arg == "-w") && a + 1 < argc) (arg == "-r" ? restart_in : restart_out) = argv[++a];
        else pos.push_back(arg);
    }
    const int steps = pos.size() > 0 ? std::atoi(pos[0].c_str()) : p.max_iter;
    const bool vortex = pos.size() > 1 && pos[1] == "vortex";
    try {
        FRSolver solver;
        if (from_file) {
            solver.initializeFromGmsh(argv[3], p);
        } else {
            Mesh mesh = structured(std::atoi(argv[2]), std::atoi(argv[3]), std::atof(argv[4]),
                                   std::atof(argv[5]), std::atof(argv[6]), std::atof(argv[7]));
            solver.initialize(mesh, p);
        }
        const double g = p.gamma;
        const double c = std::sqrt(g * p.p_inf / p.rho_inf);
        const double u_inf = p.Mach * c * std::cos(p.AoA * M_PI / 180.0);
        const double v_inf = p.Mach * c * std::sin(p.AoA * M_PI / 180.0);
        solver.setInitialCondition([&](Vec2 x) {
            double rho = p.rho_inf, u = u_inf, v = v_inf, pr = p.p_inf;
            if (vortex) {   // isentropic vortex of strength 5 at the origin, scaled to (rho_inf, p_inf)
                const double b = 5.0, r2 = x.x * x.x + x.y * x.y;
                const double f = b / (2.0 * M_PI) * std::exp(0.5 * (1.0 - r2)) * c;
                u -= f * x.y;
                v += f * x.x;
                const double T = 1.0 - (g - 1.0) * b * b / (8.0 * g * M_PI * M_PI) * std::exp(1.0 - r2);
                rho = p.rho_inf * std::pow(T, 1.0 / (g - 1.0));
                pr = p.p_inf * std::pow(T, g / (g - 1.0));
            }
            return State{rho, rho * u, rho * v, pr / (g - 1.0) + 0.5 * rho * (u * u + v * v)};
        });
        if (!restart_in.empty()) solver.readRestart(restart_in);
        const double dt = p.dt > 0 ? p.dt : solver.computeTimeStep();
        for (int it = solver.currentIteration(); it < steps; ++it) {
            solver.advance(dt);
            if (it % 10 == 0 || it == steps - 1)
                std::printf("%6d %.6e %.6e %.10e\n", it, solver.currentTime(), dt, solver.computeResidual());
            if (!restart_out.empty() && p.restart_freq > 0 && (it + 1) % p.restart_freq == 0)
                solver.writeRestart(restart_out);
        }
        if (!restart_out.empty()) solver.writeRestart(restart_out);
        solver.copyToHost();
        double sum = 0.0;
        for (double x : solver.solution()) sum += std::fabs(x);
        std::printf("checksum %.17g\n", sum);
    } catch (const zhijian_b200::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
    return 0;
}
