// zj_internal.h -- host-side structures shared by the setup code, the
// kernels' launchers and the C-ABI.  Not installed; the public boundary is
// include/zj_fr.h.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "zj_fr.h"

#ifdef __CUDACC__
#define ZJ_HD __host__ __device__
#else
#define ZJ_HD
#endif

namespace zj {

constexpr int kMaxP = 5;          // reference MAX_POLY_ORDER (types.hpp:27)

// Per-element, per-edge face record read by the stage kernels.  One record
// per (element, local edge) lets every element evaluate its own four edges
// without a face-indexed intermediate array.
struct EdgeRec {
    int32_t nbr;        // neighbour element, or -1 on a boundary / orphan edge
    int32_t nbr_edge;   // neighbour's local edge, or the boundary data slot
    int32_t flags;      // kEdge* bits, boundary type in bits 8..11
    int32_t pad;
};
constexpr int32_t kEdgeRight = 1;    // this element is the face's right side
constexpr int32_t kEdgeBoundary = 2; // boundary face (ghost state)
constexpr int32_t kEdgeOrphan = 4;   // edge on no face (non-manifold): no correction
// A face cut by a mesh partition (with kEdgeBoundary: its neighbour's trace
// and gradient trace sit in a ghost row, filled by the halo exchange instead
// of a boundary condition; kEdgeRight as on an interior face).
constexpr int32_t kEdgeInterface = 8;
ZJ_HD inline int32_t edge_bc_type(int32_t flags) { return (flags >> 8) & 0xF; }

// 1D operators of one polynomial order.  The 2D tensor-product operators of
// the reference (diff_xi, diff_eta, interp, corr_deriv) are exact Kronecker
// products of these with 0/1 factors, so the kernels apply them
// sum-factorised with the same terms in the same order.
struct Operators1D {
    int P = 0, n1 = 0;
    std::vector<double> pts, wts;   // Gauss-Legendre nodes / weights
    std::vector<double> D1;         // [n1][n1]  D1[i][k] = l_k'(x_i)
    std::vector<double> Lm, Lp;     // l_j(-1), l_j(+1)
    std::vector<double> gL, gR;     // correction derivatives g_L'(x_j), g_R'(x_j)
};

// Reference-compatible operator construction (basis.cpp:12-104,169-224,
// 314-379, 464-613): Radau (DG) correction for every flux type.
void build_operators_compat(int P, Operators1D& ops);
// Physics mode: VCJH correction with the c parameter of the flux type.
void build_operators_vcjh(int P, int flux_type, Operators1D& ops);
double lagrange_eval(const std::vector<double>& nodes, int j, double x);
double lagrange_deriv(const std::vector<double>& nodes, int j, double x);
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);

// FR operators of the straight-sided triangle (tri_setup.cpp), nt = (P+1)(P+2)/2
// solution points, 3 (P+1) flux points (edge-major, counter-clockwise).
struct TriOperators {
    int P = 0, n1 = 0, nt = 0;
    std::vector<double> r, s;       // solution points on the reference triangle
    std::vector<double> Dr, Ds;     // [nt][nt]
    std::vector<double> L;          // [3 n1][nt] interpolation to the flux points
    std::vector<double> Phi;        // [nt][3 n1] correction fields at the solution points
    std::vector<double> w;          // quadrature weights of the solution points
};
bool build_operators_tri(int P, int flux_type, TriOperators& t, std::string& msg);
double vcjh_c(int P, int flux_type);

// Topology and geometry of a quad (or quad/triangle) mesh, built on the host once.
struct HostMesh {
    int64_t n_nodes = 0, n_elem = 0, n_faces = 0;
    int nn = 4, order = 1;                 // node stride per element, geometric order
    std::vector<double> xy;                // [n_nodes][2]
    std::vector<int64_t> conn;             // [E][nn] (a triangle's 4th entry is -1)
    std::vector<int8_t> etype;             // [E] ZJ_ELEM_TRI / ZJ_ELEM_QUAD
    int64_t n_tri = 0;
    int nv(int64_t e) const { return etype[(size_t)e] == ZJ_ELEM_TRI ? 3 : 4; }
    // faces in the reference order (sorted vertex pair)
    std::vector<int32_t> fle, fll, fre, frl, fbct, ftag, fslot;
    std::vector<double> fnx, fny, flen;
    int64_t n_bnd_faces = 0;
    int64_t n_orphan_edges = 0;
};

// Builds faces exactly as Mesh::buildFaces + GmshReader::applyBoundaryTags
// (mesh.cpp:18-83, gmsh_reader.cpp:720-758) and normals as Mesh::faceNormal
// (mesh.cpp:159-183).  Returns false with msg on a bad mesh.
bool build_mesh(const zj_mesh_desc* d, const zj_params* p, HostMesh& m, std::string& msg);

// Metric terms at the solution points, [E][n_sp] J and [E][n_sp][4] Jinv =
// (xi_x, xi_y, eta_x, eta_y), as fr_solver.cpp:85-129.
// Triangles (tri != NULL) fill the first nt of their (P+1)^2 slots with the
// constant metric terms of the affine map x = -(r+s)/2 v0 + (1+r)/2 v1 + (1+s)/2 v2.
bool build_metrics(const HostMesh& m, const Operators1D& ops, std::vector<double>& J,
                   std::vector<double>& Jinv, std::string& msg, const TriOperators* tri = nullptr);
void sp_coords(const HostMesh& m, const Operators1D& ops, std::vector<double>& xy,
               const TriOperators* tri = nullptr);
void element_areas(const HostMesh& m, std::vector<double>& area);

// Boundary data, 8 doubles per boundary slot (fr_solver.cpp:432-482).
void build_bc_data(const HostMesh& m, const zj_params* p, std::vector<double>& bc);
void build_edge_records(const HostMesh& m, std::vector<EdgeRec>& rec, std::vector<double>& nrm);
// Curved meshes in physics mode: the face normal and edge Jacobian at every
// flux point, [E][4][n1][4] = (nx, ny, 2 |dx/dt|, 0).
void build_point_normals(const HostMesh& m, const Operators1D& ops, std::vector<double>& nrm);

// Mesh partitions (partition.cpp).  Recursive coordinate bisection of the
// element centroids into nparts balanced parts (deterministic).
void partition_rcb(const HostMesh& m, int nparts, std::vector<int32_t>& part);
// One part of a partitioned mesh: its elements (ascending global ids), its
// boundary slots, and its interface faces grouped by neighbouring part
// (ascending) and, within a group, in the global face order -- the order
// both sides of a cut agree on.  Interface k's ghost row is local boundary
// slot n_bnd + k.
struct PartSlice {
    int rank = 0, nparts = 1;
    std::vector<int64_t> elems;          // local -> global element
    std::vector<int64_t> g2l;            // global -> local element, -1 elsewhere
    std::vector<int32_t> bnd_slots;      // local boundary slot -> global slot
    std::vector<int32_t> nbr;            // neighbouring parts
    std::vector<int64_t> nbr_off;        // interfaces of nbr[i]: [nbr_off[i], nbr_off[i+1])
    std::vector<int64_t> face;           // global face id of interface k
    std::vector<int64_t> mine;           // global element*4 + edge of this part's side
    std::vector<int64_t> remote;         // global element*4 + edge of the other side
};
bool make_part_slice(const HostMesh& m, const int32_t* part, int nparts, int rank, PartSlice& ps,
                     std::string& msg);
// The global per-element arrays restricted to the part: edge records with
// local neighbours, local boundary slots and interface ghost slots; rows of
// width w of any [E][...] array; boundary data of the local slots followed by
// zero rows for the interfaces.
void slice_edge_records(const PartSlice& ps, const std::vector<EdgeRec>& rec, std::vector<EdgeRec>& out);
template <class T>
std::vector<T> slice_rows(const PartSlice& ps, const std::vector<T>& a, size_t w) {
    std::vector<T> out(ps.elems.size() * w);
    for (size_t l = 0; l < ps.elems.size(); ++l)
        for (size_t k = 0; k < w; ++k) out[l * w + k] = a[(size_t)ps.elems[l] * w + k];
    return out;
}
std::vector<double> slice_bc_data(const PartSlice& ps, const std::vector<double>& bc);

// Gmsh reader (gmsh.cpp).
struct GmshGroup {
    int tag = 0;
    int type = 0;          // zj_bc_type inferred from the name
    std::string name;
};
struct GmshMesh {
    std::vector<double> xy;        // [n][2]
    std::vector<int32_t> etype, eorder;
    std::vector<int64_t> offs;     // [n_elem + 1]
    std::vector<int64_t> conn;
    std::vector<int64_t> bnd;      // [n_bnd][3] (v0, v1, physical tag)
    std::vector<GmshGroup> groups; // boundary groups in tag order
};
bool read_gmsh(const std::string& path, GmshMesh& m, std::string& err);
int infer_bc_type(const std::string& name);

}  // namespace zj
