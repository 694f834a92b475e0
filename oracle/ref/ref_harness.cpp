// ref_harness.cpp -- TEST INFRASTRUCTURE: drives the reference's own code.
//
// Built by oracle/ref/Makefile from the reference sources where they lie
// (nothing is copied); output binaries go to oracle/_ref/.  Two builds:
//   ref_cpu : basis.cpp + mesh.cpp + gmsh_reader.cpp, runs on any host.
//             "ops P out"            -> FROperators (basis.cpp:464-613)
//             "tri P out"            -> FROperators on a triangle (basis.cpp:615-668)
//             "mesh mesh.bin P out"  -> faces, normals (mesh.cpp:18-194) and
//                                       J/Jinv exactly as fr_solver.cpp:85-129
//             "gmsh file.msh out"    -> GmshReader::read (gmsh_reader.cpp:161)
//             "visc in out gamma Re Pr" -> ViscousFlux::fluxX/fluxY and
//                                       BR2Scheme::commonFlux (navierstokes.hpp)
//   ref_gpu : + kernels.cu + fr_solver.cpp, needs a GPU.
//             "rhs mesh.bin params state out"           -> computeResidual_GPU
//             "step mesh.bin params state dt n out"     -> n x advance(dt)
//             "time mesh.bin params state dt nw n out"  -> wall ms of n advance(dt)
//             "traj mesh.bin params state n out"        -> dt = computeTimeStep(),
//                                                          then the state and the
//                                                          residual norm after each
//                                                          of n advance(dt)
//             "viscsp in out gamma Re Pr" -> gpu::computeViscousFluxSP
//                                            (kernels.cu:719-807) on the records
// Files are raw little-endian arrays; layouts are written by
// oracle/oracle.py (write_mesh_bin) and read back by it.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common/types.hpp"
#include "mesh/mesh.hpp"
#include "basis/basis.hpp"
#include "bc/boundary_condition.hpp"
#include "physics/euler.hpp"
#include "physics/navierstokes.hpp"

#ifdef ZJ_REF_GPU
#include <cuda_runtime.h>
#include "gpu/kernels.hpp"
#define private public
#define protected public
#include "solver/fr_solver.hpp"
#undef private
#undef protected
#endif

using namespace zhijian;

namespace {

struct Reader {
    std::ifstream f;
    explicit Reader(const char* p) : f(p, std::ios::binary) {
        if (!f) { std::fprintf(stderr, "cannot open %s\n", p); std::exit(2); }
    }
    template <class T> T get() { T v; f.read(reinterpret_cast<char*>(&v), sizeof(T)); return v; }
    template <class T> void arr(std::vector<T>& v, size_t n) {
        v.resize(n);
        f.read(reinterpret_cast<char*>(v.data()), n * sizeof(T));
    }
};

struct Writer {
    std::ofstream f;
    explicit Writer(const char* p) : f(p, std::ios::binary) {}
    template <class T> void put(T v) { f.write(reinterpret_cast<const char*>(&v), sizeof(T)); }
    template <class T> void arr(const std::vector<T>& v) {
        f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T));
    }
};

// Mesh file: int64 n_nodes, f64 xy[n][2], int64 n_elem, int32 nn, int32 order,
// int64 conn[E][nn], int64 n_bnd, int64 bnd[n][3], int32 n_tags,
// n_tags x (int32 id, int32 type, f64 p_static)
void load_mesh(const char* path, Mesh& mesh) {
    Reader r(path);
    int64_t nn_nodes = r.get<int64_t>();
    std::vector<double> xy; r.arr(xy, 2 * nn_nodes);
    for (int64_t i = 0; i < nn_nodes; ++i) mesh.nodes().push_back(Vec2(xy[2 * i], xy[2 * i + 1]));
    int64_t ne = r.get<int64_t>();
    int32_t nn = r.get<int32_t>(), order = r.get<int32_t>();
    std::vector<int64_t> conn; r.arr(conn, ne * nn);
    for (int64_t e = 0; e < ne; ++e) {
        Element el;
        el.type = ElementType::Quadrilateral;
        el.order = order;
        el.partition = 0;
        for (int k = 0; k < nn; ++k) el.node_ids.push_back(conn[e * nn + k]);
        mesh.elements().push_back(el);
    }
    int64_t nb = r.get<int64_t>();
    std::vector<int64_t> bnd; r.arr(bnd, 3 * nb);
    int32_t nt = r.get<int32_t>();
    for (int t = 0; t < nt; ++t) {
        int32_t id = r.get<int32_t>(), ty = r.get<int32_t>();
        double ps = r.get<double>();
        BCInfo info;
        info.tag = id; info.type = static_cast<BCType>(ty); info.name = "tag";
        info.p_total = 0; info.T_total = 0; info.flow_direction = Vec2(1, 0);
        info.p_static = ps; info.T_wall = 0;
        mesh.addBCInfo(id, info);
    }
    mesh.buildFaces();
    // gmsh_reader.cpp:720-758: vertex pair -> tag (last wins), then stamp.
    std::map<std::pair<Index, Index>, int> tags;
    for (int64_t i = 0; i < nb; ++i) {
        Index a = bnd[3 * i], b = bnd[3 * i + 1];
        int tag = static_cast<int>(bnd[3 * i + 2]);
        if (tag <= 0) continue;
        if (a > b) std::swap(a, b);
        tags[{a, b}] = tag;
    }
    for (Index f = 0; f < mesh.numFaces(); ++f) {
        Face& face = mesh.face(f);
        if (!face.is_boundary) continue;
        const Element& el = mesh.element(face.left_elem);
        Index a = el.node_ids[face.left_face % 4], b = el.node_ids[(face.left_face + 1) % 4];
        if (a > b) std::swap(a, b);
        auto it = tags.find({a, b});
        if (it != tags.end()) {
            face.bc_tag = it->second;
            if (mesh.hasBCInfo(it->second)) face.bc_type = mesh.getBCInfo(it->second).type;
        }
    }
    mesh.computeGeometry();
}

int cmd_ops(int P, const char* out) {
    FROperators ops;
    ops.init(ElementType::Quadrilateral, P, FluxType::HU);
    int nsp = ops.numSolutionPoints(), n1 = P + 1;
    std::vector<double> pts, w;
    GaussLegendre::getQuadrature(n1, pts, w);
    std::vector<std::vector<double>> D;
    Lagrange1D::buildDiffMatrix(pts, D);
    Writer wr(out);
    wr.arr(pts);
    for (auto& row : D) wr.arr(row);
    for (int i = 0; i < nsp; ++i) wr.arr(ops.diffXi()[i]);
    for (int i = 0; i < nsp; ++i) wr.arr(ops.diffEta()[i]);
    for (int e = 0; e < 4; ++e)
        for (int fp = 0; fp < n1; ++fp) wr.arr(ops.interpToFlux(e)[fp]);
    for (int e = 0; e < 4; ++e) wr.arr(ops.correctionDeriv()[e]);
    return 0;
}

// FROperators on a triangle (basis.cpp:615-668): solution points
// (SolutionPoints::getTriangle, basis.cpp:391-417), flux-point locations,
// interpolation, differentiation, correction derivatives, weights.
int cmd_tri(int P, const char* out) {
    FROperators ops;
    ops.init(ElementType::Triangle, P, FluxType::DG);
    const int nt = ops.numSolutionPoints(), n1 = ops.numFluxPointsPerEdge();
    Writer wr(out);
    wr.arr(ops.solutionXi());
    wr.arr(ops.solutionEta());
    for (int e = 0; e < 3; ++e) wr.arr(ops.fluxPointLoc()[e]);
    for (int e = 0; e < 3; ++e)
        for (int fp = 0; fp < n1; ++fp) wr.arr(ops.interpToFlux(e)[fp]);
    for (int i = 0; i < nt; ++i) wr.arr(ops.diffXi()[i]);
    for (int i = 0; i < nt; ++i) wr.arr(ops.diffEta()[i]);
    for (int e = 0; e < 3; ++e) wr.arr(ops.correctionDeriv()[e]);
    wr.arr(ops.quadWeights());
    return 0;
}

int cmd_mesh(const char* mpath, int P, const char* out) {
    Mesh mesh;
    load_mesh(mpath, mesh);
    FROperators ops;
    ops.init(ElementType::Quadrilateral, P, FluxType::HU);
    Writer wr(out);
    int64_t nf = mesh.numFaces();
    wr.put(nf);
    for (int64_t f = 0; f < nf; ++f) {
        const Face& fc = mesh.face(f);
        Vec2 n = mesh.faceNormal(f);
        wr.put<int32_t>(fc.left_elem); wr.put<int32_t>(fc.left_face);
        wr.put<int32_t>(fc.right_elem); wr.put<int32_t>(fc.right_face);
        wr.put<int32_t>(static_cast<int32_t>(fc.bc_type)); wr.put<int32_t>(fc.bc_tag);
        wr.put(n.x); wr.put(n.y);
    }
    // fr_solver.cpp:85-129, restated around ElementGeometry::jacobian
    std::vector<double> J, Jinv, sxy;
    for (Index i = 0; i < mesh.numElements(); ++i) {
        const Element& el = mesh.element(i);
        std::vector<Vec2> nodes;
        for (Index id : el.node_ids) nodes.push_back(mesh.node(id));
        for (int sp = 0; sp < ops.numSolutionPoints(); ++sp) {
            Real xi = ops.solutionXi()[sp], eta = ops.solutionEta()[sp];
            Real a, b, c, d;
            ElementGeometry::jacobian(nodes, el.type, el.order, xi, eta, a, b, c, d);
            Real Jd = a * d - b * c;
            J.push_back(Jd);
            Real invJ = 1.0 / Jd;
            Jinv.push_back(d * invJ); Jinv.push_back(-b * invJ);
            Jinv.push_back(-c * invJ); Jinv.push_back(a * invJ);
            Vec2 p = ElementGeometry::refToPhys(nodes, el.type, el.order, xi, eta);
            sxy.push_back(p.x); sxy.push_back(p.y);
        }
    }
    wr.arr(J); wr.arr(Jinv); wr.arr(sxy);
    std::vector<double> area;
    for (Index i = 0; i < mesh.numElements(); ++i) area.push_back(mesh.elementArea(i));
    wr.arr(area);
    return 0;
}

int cmd_gmsh(const char* path, const char* out) {
    Mesh mesh;
    GmshReader rd;
    if (!rd.read(path, mesh)) { std::fprintf(stderr, "%s\n", rd.errorMessage().c_str()); return 3; }
    Writer wr(out);
    wr.put<int64_t>(mesh.numNodes());
    for (auto& n : mesh.nodes()) { wr.put(n.x); wr.put(n.y); }
    wr.put<int64_t>(mesh.numElements());
    for (auto& e : mesh.elements()) {
        wr.put<int32_t>(static_cast<int32_t>(e.type)); wr.put<int32_t>(e.order);
        wr.put<int32_t>(static_cast<int32_t>(e.node_ids.size()));
        for (Index id : e.node_ids) wr.put<int64_t>(id);
    }
    wr.put<int64_t>(mesh.numFaces());
    for (Index f = 0; f < mesh.numFaces(); ++f) {
        const Face& fc = mesh.face(f);
        wr.put<int32_t>(fc.left_elem); wr.put<int32_t>(fc.left_face);
        wr.put<int32_t>(fc.right_elem); wr.put<int32_t>(fc.right_face);
        wr.put<int32_t>(static_cast<int32_t>(fc.bc_type)); wr.put<int32_t>(fc.bc_tag);
    }
    wr.put<int32_t>(static_cast<int32_t>(mesh.allBCInfo().size()));
    for (auto& kv : mesh.allBCInfo()) {
        wr.put<int32_t>(kv.first); wr.put<int32_t>(static_cast<int32_t>(kv.second.type));
    }
    return 0;
}

// "phys in.bin out.bin gamma Mach AoA rho_inf p_inf p_total T_total dx dy p_static T_wall"
// in: int64 N, then N x (UL[4], UR[4], nx, ny) f64.  out per record:
// Rusanov, Roe, HLLC fluxes (euler.hpp:184-375), then ghost states of
// NoSlipWall, IsothermalWall, SlipWall, Symmetry, FarField (fromMach), SubsonicInflow,
// SubsonicOutflow (boundary_condition.hpp:42-311) from UL.
int cmd_phys(char** a) {
    Reader r(a[0]);
    const int64_t n = r.get<int64_t>();
    std::vector<double> in; r.arr(in, n * 10);
    const double g = std::atof(a[2]), mach = std::atof(a[3]), aoa = std::atof(a[4]);
    const double rho_inf = std::atof(a[5]), p_inf = std::atof(a[6]);
    const double pt = std::atof(a[7]), Tt = std::atof(a[8]), dx = std::atof(a[9]), dy = std::atof(a[10]);
    const double ps = std::atof(a[11]), Tw = std::atof(a[12]);
    NoSlipWallBC wall(g);
    IsothermalWallBC iso(Tw, g);
    SlipWallBC slip(g);
    SymmetryBC sym(g);
    auto ff = FarFieldBC::fromMach(mach, aoa, rho_inf, p_inf, g);
    SubsonicInflowBC inflow(pt, Tt, dx, dy, g);
    SubsonicOutflowBC outflow(ps, g);
    const BoundaryCondition* bcs[7] = {&wall, &iso, &slip, &sym, ff.get(), &inflow, &outflow};
    Writer w(a[1]);
    for (int64_t k = 0; k < n; ++k) {
        const double* q = &in[k * 10];
        State UL, UR;
        for (int v = 0; v < 4; ++v) { UL[v] = q[v]; UR[v] = q[4 + v]; }
        const double nx = q[8], ny = q[9];
        State F[3] = {RiemannSolvers::rusanov(UL, UR, nx, ny, g), RiemannSolvers::roe(UL, UR, nx, ny, g),
                      RiemannSolvers::hllc(UL, UR, nx, ny, g)};
        for (auto& f : F) for (int v = 0; v < 4; ++v) w.put(f[v]);
        for (auto* bc : bcs) {
            State gs = bc->ghostState(UL, nx, ny);
            for (int v = 0; v < 4; ++v) w.put(gs[v]);
        }
    }
    return 0;
}

// Viscous pin records: in = int64 N, then N x (U[4], dUdx[4], dUdy[4],
// UR[4], dUdxR[4], dUdyR[4], nx, ny) f64.
int read_visc(const char* path, std::vector<double>& in) {
    Reader r(path);
    const int64_t n = r.get<int64_t>();
    r.arr(in, static_cast<size_t>(n) * 26);
    return static_cast<int>(n);
}

// "visc in out gamma Re Pr": per record the header's ViscousFlux::fluxX and
// fluxY at (U, dUdx, dUdy) with the header's own velocity and temperature
// gradients (navierstokes.hpp:52-96, 115-158), then
// BR2Scheme::commonFlux(UL=U, UR, ...) (navierstokes.hpp:166-201); 12 values.
int cmd_visc(char** a) {
    std::vector<double> in;
    const int n = read_visc(a[0], in);
    const double g = std::atof(a[2]), Re = std::atof(a[3]), Pr = std::atof(a[4]);
    ViscousFlux vf(g, Re, Pr);
    Writer w(a[1]);
    for (int k = 0; k < n; ++k) {
        const double* q = &in[static_cast<size_t>(k) * 26];
        State U, dx, dy, UR, dxR, dyR;
        for (int v = 0; v < 4; ++v) {
            U[v] = q[v]; dx[v] = q[4 + v]; dy[v] = q[8 + v];
            UR[v] = q[12 + v]; dxR[v] = q[16 + v]; dyR[v] = q[20 + v];
        }
        Real dudx, dudy, dvdx, dvdy, dTdx, dTdy;
        ViscousFlux::velocityGradients(U, dx, dy, dudx, dudy, dvdx, dvdy);
        vf.temperatureGradient(U, dx, dy, dTdx, dTdy);
        const State F = vf.fluxX(U, dudx, dudy, dvdx, dvdy, dTdx, dTdy);
        const State G = vf.fluxY(U, dudx, dudy, dvdx, dvdy, dTdx, dTdy);
        const State C = BR2Scheme::commonFlux(U, UR, dx, dy, dxR, dyR, q[24], q[25], g, Re, Pr);
        for (int v = 0; v < 4; ++v) w.put(F[v]);
        for (int v = 0; v < 4; ++v) w.put(G[v]);
        for (int v = 0; v < 4; ++v) w.put(C[v]);
    }
    return 0;
}

#ifdef ZJ_REF_GPU
// params: "P gamma rho_inf p_inf Mach AoA"
SimParams make_params(char** a) {
    SimParams p;
    p.poly_order = std::atoi(a[0]);
    p.gamma = std::atof(a[1]); p.rho_inf = std::atof(a[2]); p.p_inf = std::atof(a[3]);
    p.Mach_inf = std::atof(a[4]); p.AoA = std::atof(a[5]);
    p.riemann = RiemannSolver::Rusanov; p.flux_type = FluxType::HU; p.viscous = false;
    return p;
}

void put_state(FRSolver& s, const std::vector<double>& U) {
    size_t idx = 0;
    for (auto& es : s.solution_)
        for (auto& st : es.sol_pts)
            for (int v = 0; v < 4; ++v) st[v] = U[idx++];
    s.copyToDevice();
}

int cmd_gpu(int argc, char** argv) {
    std::string cmd = argv[1];
    Mesh mesh;
    load_mesh(argv[2], mesh);
    SimParams p = make_params(argv + 3);
    FRSolver s;
    s.initialize(mesh, p);
    size_t n = static_cast<size_t>(mesh.numElements()) * (p.poly_order + 1) * (p.poly_order + 1) * 4;
    Reader r(argv[9]);
    std::vector<double> U; r.arr(U, n);
    put_state(s, U);
    std::vector<double> out(n);
    if (cmd == "rhs") {
        s.computeResidual_GPU();
        cudaDeviceSynchronize();
        s.gpu_data_->dUdt.copyToHost(out.data(), n);
        Writer(argv[10]).arr(out);
    } else if (cmd == "traj") {
        // the reference's CFL step from the state just set (computeTimeStep
        // reads the host copy), then n steps, each one recorded
        const int ns = std::atoi(argv[10]);
        const double dt = s.computeTimeStep();
        Writer w(argv[11]);
        w.put(dt);
        for (int k = 0; k < ns; ++k) {
            s.advance(dt);
            s.gpu_data_->U.copyToHost(out.data(), n);
            w.arr(out);
            w.put(s.computeResidual());
        }
    } else if (cmd == "time") {
        // wall clock of nsteps advance() calls after nwarm, device idle at both
        // ends: the reference's step includes host work and copies
        double dt = std::atof(argv[10]);
        int nwarm = std::atoi(argv[11]), ns = std::atoi(argv[12]);
        for (int k = 0; k < nwarm; ++k) s.advance(dt);
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        for (int k = 0; k < ns; ++k) s.advance(dt);
        cudaDeviceSynchronize();
        auto t1 = std::chrono::steady_clock::now();
        double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        std::FILE* f = std::fopen(argv[13], "w");
        if (!f) return 2;
        std::fprintf(f, "%d %.6f\n", ns, ms);
        std::fclose(f);
    } else {
        double dt = std::atof(argv[10]);
        int ns = std::atoi(argv[11]);
        for (int k = 0; k < ns; ++k) s.advance(dt);
        s.gpu_data_->U.copyToHost(out.data(), n);
        Writer w(argv[12]);
        w.arr(out);
        s.gpu_data_->dUdt.copyToHost(out.data(), n);
        w.arr(out);
        double res = s.computeResidual();
        w.put(res);
    }
    return 0;
}

// "viscsp in out gamma Re Pr": the reference's computeViscousFluxSP kernel
// (kernels.cu:719-807) over the records' (U, dUdx, dUdy) as one element of N
// solution points; out = Fv_x[N][4], then Fv_y[N][4].
int cmd_viscsp(char** a) {
    std::vector<double> in;
    const int n = read_visc(a[0], in);
    const double g = std::atof(a[2]), Re = std::atof(a[3]), Pr = std::atof(a[4]);
    std::vector<double> U(4 * n), dx(4 * n), dy(4 * n);
    for (int k = 0; k < n; ++k)
        for (int v = 0; v < 4; ++v) {
            U[4 * k + v] = in[26 * k + v];
            dx[4 * k + v] = in[26 * k + 4 + v];
            dy[4 * k + v] = in[26 * k + 8 + v];
        }
    const size_t bytes = sizeof(double) * 4 * n;
    double *dU = nullptr, *ddx = nullptr, *ddy = nullptr, *fx = nullptr, *fy = nullptr;
    if (cudaMalloc(&dU, bytes) || cudaMalloc(&ddx, bytes) || cudaMalloc(&ddy, bytes) ||
        cudaMalloc(&fx, bytes) || cudaMalloc(&fy, bytes))
        return 4;
    cudaMemcpy(dU, U.data(), bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(ddx, dx.data(), bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(ddy, dy.data(), bytes, cudaMemcpyHostToDevice);
    gpu::computeViscousFluxSP(dU, ddx, ddy, fx, fy, g, Re, Pr, 1, n, 0);
    if (cudaDeviceSynchronize() != cudaSuccess) return 5;
    std::vector<double> ox(4 * n), oy(4 * n);
    cudaMemcpy(ox.data(), fx, bytes, cudaMemcpyDeviceToHost);
    cudaMemcpy(oy.data(), fy, bytes, cudaMemcpyDeviceToHost);
    Writer w(a[1]);
    w.arr(ox);
    w.arr(oy);
    cudaFree(dU); cudaFree(ddx); cudaFree(ddy); cudaFree(fx); cudaFree(fy);
    return 0;
}
#endif

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) { std::fprintf(stderr, "usage: see header\n"); return 1; }
    std::string cmd = argv[1];
    if (cmd == "ops" && argc == 4) return cmd_ops(std::atoi(argv[2]), argv[3]);
    if (cmd == "tri" && argc == 4) return cmd_tri(std::atoi(argv[2]), argv[3]);
    if (cmd == "mesh" && argc == 5) return cmd_mesh(argv[2], std::atoi(argv[3]), argv[4]);
    if (cmd == "gmsh" && argc == 4) return cmd_gmsh(argv[2], argv[3]);
    if (cmd == "phys" && argc == 15) return cmd_phys(argv + 2);
    if (cmd == "visc" && argc == 7) return cmd_visc(argv + 2);
#ifdef ZJ_REF_GPU
    if ((cmd == "rhs" && argc == 11) || (cmd == "step" && argc == 13) || (cmd == "time" && argc == 14) ||
        (cmd == "traj" && argc == 12))
        return cmd_gpu(argc, argv);
    if (cmd == "viscsp" && argc == 7) return cmd_viscsp(argv + 2);
#endif
    std::fprintf(stderr, "bad command\n");
    return 1;
}
