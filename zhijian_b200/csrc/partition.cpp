// partition.cpp -- element partitions of a mesh for the multi-part residual:
// recursive coordinate bisection and the per-part view (local elements,
// boundary slots, interfaces with their exchange order).
//
// The reference partitions the element dual graph with METIS k-way
// (src/mesh/partitioner.cpp:10-93) and exchanges element data between ranks
// (src/parallel/mpi_comm.cpp:68-171).  METIS is not in this image; recursive
// coordinate bisection gives balanced parts (sizes differ by at most one
// element) with short cuts on the meshes here, and what crosses a cut is the
// face traces, not element data: the FR residual couples elements only
// through the traces at their shared faces.
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "zj_internal.h"

namespace zj {

namespace {

void bisect(const std::vector<double>& cx, const std::vector<double>& cy, std::vector<int64_t>& ids, size_t lo,
            size_t hi, int first, int nparts, std::vector<int32_t>& part) {
    if (nparts == 1) {
        for (size_t i = lo; i < hi; ++i) part[(size_t)ids[i]] = first;
        return;
    }
    double x0 = cx[(size_t)ids[lo]], x1 = x0, y0 = cy[(size_t)ids[lo]], y1 = y0;
    for (size_t i = lo; i < hi; ++i) {
        const size_t e = (size_t)ids[i];
        x0 = std::min(x0, cx[e]); x1 = std::max(x1, cx[e]);
        y0 = std::min(y0, cy[e]); y1 = std::max(y1, cy[e]);
    }
    const std::vector<double>& c = (x1 - x0 >= y1 - y0) ? cx : cy;
    // the lower nl parts take their share of the elements, ties broken by id
    std::sort(ids.begin() + (long)lo, ids.begin() + (long)hi, [&](int64_t a, int64_t b) {
        const double ca = c[(size_t)a], cb = c[(size_t)b];
        return ca < cb || (ca == cb && a < b);
    });
    const int nl = nparts / 2;
    const size_t n = hi - lo;
    const size_t split = lo + (n * (size_t)nl) / (size_t)nparts;
    bisect(cx, cy, ids, lo, split, first, nl, part);
    bisect(cx, cy, ids, split, hi, first + nl, nparts - nl, part);
}

}  // namespace

void partition_rcb(const HostMesh& m, int nparts, std::vector<int32_t>& part) {
    const size_t ne = (size_t)m.n_elem;
    std::vector<double> cx(ne), cy(ne);
    for (size_t e = 0; e < ne; ++e) {
        const int nv = m.nv((int64_t)e);
        double sx = 0.0, sy = 0.0;
        for (int k = 0; k < nv; ++k) {
            const int64_t v = m.conn[e * m.nn + (size_t)k];
            sx += m.xy[2 * v];
            sy += m.xy[2 * v + 1];
        }
        cx[e] = sx / nv;
        cy[e] = sy / nv;
    }
    std::vector<int64_t> ids(ne);
    std::iota(ids.begin(), ids.end(), 0);
    part.assign(ne, 0);
    bisect(cx, cy, ids, 0, ne, 0, std::max(nparts, 1), part);
}

bool make_part_slice(const HostMesh& m, const int32_t* part, int nparts, int rank, PartSlice& ps,
                     std::string& msg) {
    if (nparts < 1 || rank < 0 || rank >= nparts) { msg = "rank must be in [0, nparts)"; return false; }
    ps = PartSlice();
    ps.rank = rank;
    ps.nparts = nparts;
    ps.g2l.assign((size_t)m.n_elem, -1);
    for (int64_t e = 0; e < m.n_elem; ++e) {
        const int32_t p = part[(size_t)e];
        if (p < 0 || p >= nparts) { msg = "element " + std::to_string(e) + " has a part outside [0, nparts)"; return false; }
        if (p == rank) {
            ps.g2l[(size_t)e] = (int64_t)ps.elems.size();
            ps.elems.push_back(e);
        }
    }
    if (ps.elems.empty()) { msg = "part " + std::to_string(rank) + " has no elements"; return false; }
    struct Cut { int32_t q; int64_t f, mine, remote; };
    std::vector<Cut> cuts;
    for (int64_t f = 0; f < m.n_faces; ++f) {
        const size_t fi = (size_t)f;
        if (m.fre[fi] < 0) {
            if (part[(size_t)m.fle[fi]] == rank) ps.bnd_slots.push_back(m.fslot[fi]);
            continue;
        }
        const int32_t pl = part[(size_t)m.fle[fi]], pr = part[(size_t)m.fre[fi]];
        if (pl == pr || (pl != rank && pr != rank)) continue;
        const int64_t sl = (int64_t)m.fle[fi] * 4 + m.fll[fi], sr = (int64_t)m.fre[fi] * 4 + m.frl[fi];
        if (pl == rank) cuts.push_back(Cut{pr, f, sl, sr});
        else cuts.push_back(Cut{pl, f, sr, sl});
    }
    std::stable_sort(cuts.begin(), cuts.end(), [](const Cut& a, const Cut& b) {
        return a.q < b.q || (a.q == b.q && a.f < b.f);
    });
    for (size_t k = 0; k < cuts.size(); ++k) {
        if (ps.nbr.empty() || ps.nbr.back() != cuts[k].q) {
            ps.nbr.push_back(cuts[k].q);
            ps.nbr_off.push_back((int64_t)k);
        }
        ps.face.push_back(cuts[k].f);
        ps.mine.push_back(cuts[k].mine);
        ps.remote.push_back(cuts[k].remote);
    }
    ps.nbr_off.push_back((int64_t)cuts.size());
    return true;
}

void slice_edge_records(const PartSlice& ps, const std::vector<EdgeRec>& rec, std::vector<EdgeRec>& out) {
    const int64_t nb = (int64_t)ps.bnd_slots.size();
    // global boundary slot -> local slot, and local edge slot -> interface
    std::vector<int32_t> bslot;
    int32_t maxg = -1;
    for (int32_t g : ps.bnd_slots) maxg = std::max(maxg, g);
    bslot.assign((size_t)(maxg + 1), -1);
    for (size_t l = 0; l < ps.bnd_slots.size(); ++l) bslot[(size_t)ps.bnd_slots[l]] = (int32_t)l;
    std::vector<int64_t> iface(ps.elems.size() * 4, -1);
    for (size_t k = 0; k < ps.mine.size(); ++k) {
        const int64_t e = ps.mine[k] / 4, edge = ps.mine[k] % 4;
        iface[(size_t)ps.g2l[(size_t)e] * 4 + (size_t)edge] = (int64_t)k;
    }
    out.resize(ps.elems.size() * 4);
    for (size_t l = 0; l < ps.elems.size(); ++l)
        for (int edge = 0; edge < 4; ++edge) {
            EdgeRec r = rec[(size_t)ps.elems[l] * 4 + (size_t)edge];
            const int64_t k = iface[l * 4 + (size_t)edge];
            if (k >= 0) {
                r = EdgeRec{-1, (int32_t)(nb + k), kEdgeBoundary | kEdgeInterface | (r.flags & kEdgeRight), 0};
            } else if (r.flags & kEdgeBoundary) {
                r.nbr_edge = bslot[(size_t)r.nbr_edge];
            } else if (!(r.flags & kEdgeOrphan)) {
                r.nbr = (int32_t)ps.g2l[(size_t)r.nbr];
            }
            out[l * 4 + (size_t)edge] = r;
        }
}

std::vector<double> slice_bc_data(const PartSlice& ps, const std::vector<double>& bc) {
    const size_t rows = std::max<size_t>(ps.bnd_slots.size() + ps.mine.size(), 1);
    std::vector<double> out(rows * 8, 0.0);
    for (size_t l = 0; l < ps.bnd_slots.size(); ++l)
        for (int k = 0; k < 8; ++k) out[l * 8 + (size_t)k] = bc[(size_t)ps.bnd_slots[l] * 8 + (size_t)k];
    return out;
}

}  // namespace zj
