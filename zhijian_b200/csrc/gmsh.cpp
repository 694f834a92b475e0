// gmsh.cpp -- ASCII Gmsh MSH v2.2 / v4.1 reader into the mesh descriptor
// (the behaviour of GmshReader::read, src/mesh/gmsh_reader.cpp:161-760):
//
//  * $MeshFormat decides the dialect (>= 4.0: entity blocks); binary files
//    (file type != 0) are refused;
//  * nodes are numbered in file order (v4: block order) and element node
//    tags are remapped through that numbering; an unknown tag is an error;
//  * line elements (types 1, 8, 26, 27, 28) are boundary edges carrying the
//    physical tag of the element (v2: its first tag; v4: the first physical
//    tag of its curve entity from $Entities);
//  * 2D elements: 3-node triangles (2), 6-node triangles (9), 4-node quads
//    (3), 9-node quads (10), 25-node quads (37), and 8-node serendipity
//    quads (16), which get a synthesised centre node
//    c = (n4+n5+n6+n7)/2 - (n0+n1+n2+n3)/4 appended to the node list (exact
//    for bilinear geometry); every other type is skipped;
//  * boundary groups: every positive physical tag of a boundary edge, named
//    from $PhysicalNames (dimension 1) or "BC_<tag>", typed by the name
//    (infer_bc_type); a boundary face takes the tag of the last edge with its
//    vertex pair.
// The reader allocates nothing on a device.
#include <algorithm>
#include <cctype>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "zj_internal.h"

namespace zj {

namespace {

// nodes of a Gmsh element type; -1 for types the format table does not list
// (gmsh_reader.cpp:15-42)
int gmsh_nodes(int t) {
    switch (t) {
        case 1: return 2;   case 2: return 3;   case 3: return 4;   case 4: return 4;
        case 5: return 8;   case 6: return 6;   case 7: return 5;   case 8: return 3;
        case 9: return 6;   case 10: return 9;  case 11: return 10; case 12: return 27;
        case 13: return 18; case 14: return 14; case 15: return 1;  case 16: return 8;
        case 20: return 9;  case 21: return 10; case 26: return 4;  case 27: return 5;
        case 28: return 6;  case 36: return 16; case 37: return 25;
        default: return -1;
    }
}

const char* gmsh_name(int t) {
    switch (t) {
        case 1: return "2-node line";               case 2: return "3-node triangle";
        case 3: return "4-node quadrilateral";      case 4: return "4-node tetrahedron";
        case 5: return "8-node hexahedron";         case 6: return "6-node prism";
        case 7: return "5-node pyramid";            case 8: return "3-node line (order 2)";
        case 9: return "6-node triangle (order 2)"; case 10: return "9-node quadrilateral (order 2)";
        case 11: return "10-node tetrahedron (order 2)";
        case 12: return "27-node hexahedron (order 2)";
        case 13: return "18-node prism (order 2)";  case 14: return "14-node pyramid (order 2)";
        case 15: return "1-node point";             case 16: return "8-node quadrilateral (serendipity)";
        case 20: return "9-node triangle (order 3)"; case 21: return "10-node triangle (order 3)";
        case 26: return "4-node line (order 3)";    case 27: return "5-node line (order 4)";
        case 28: return "6-node line (order 5)";    case 36: return "16-node quadrilateral (order 3)";
        case 37: return "25-node quadrilateral (order 4)";
        default: return "unknown";
    }
}

bool is_line(int t) { return t == 1 || t == 8 || t == 26 || t == 27 || t == 28; }
bool is_3d(int t) { return (t >= 4 && t <= 7) || (t >= 11 && t <= 14); }

bool contains(const std::string& s, const char* w) { return s.find(w) != std::string::npos; }

struct Reader {
    GmshMesh& m;
    std::string& err;
    std::map<long long, int64_t> node_index;          // file tag -> node
    std::map<int, int> curve_phys;                    // v4 curve entity -> physical tag
    std::map<std::pair<int, int>, std::string> names; // (dim, tag) -> name
    std::vector<std::vector<int64_t>> edges;          // boundary edges' nodes
    std::vector<int> edge_tags;
    std::map<int, long long> type_counts;

    bool node(long long tag, int64_t& out) {
        auto it = node_index.find(tag);
        if (it == node_index.end()) {
            err = "Element references unknown node tag " + std::to_string(tag);
            return false;
        }
        out = it->second;
        return true;
    }

    // One element with its remapped nodes: boundary edge, 2D element or skip.
    void element(int type, int phys, std::vector<int64_t>& nodes) {
        if (is_line(type)) {
            edges.push_back(nodes);
            edge_tags.push_back(phys);
            return;
        }
        int et = -1, order = 0;
        switch (type) {
            case 2: et = ZJ_ELEM_TRI; order = 1; break;
            case 9: et = ZJ_ELEM_TRI; order = 2; break;
            case 3: et = ZJ_ELEM_QUAD; order = 1; break;
            case 10: et = ZJ_ELEM_QUAD; order = 2; break;
            case 37: et = ZJ_ELEM_QUAD; order = 4; break;
            case 16: {
                double cx = 0.0, cy = 0.0;
                for (int k = 4; k < 8; ++k) { cx += 0.5 * m.xy[2 * nodes[k]]; cy += 0.5 * m.xy[2 * nodes[k] + 1]; }
                double sx = 0.0, sy = 0.0;
                for (int k = 0; k < 4; ++k) { sx += m.xy[2 * nodes[k]]; sy += m.xy[2 * nodes[k] + 1]; }
                m.xy.push_back(cx - 0.25 * sx);
                m.xy.push_back(cy - 0.25 * sy);
                nodes.push_back((int64_t)(m.xy.size() / 2 - 1));
                et = ZJ_ELEM_QUAD; order = 2;
                break;
            }
            default: return;
        }
        m.etype.push_back(et);
        m.eorder.push_back(order);
        m.conn.insert(m.conn.end(), nodes.begin(), nodes.end());
        m.offs.push_back((int64_t)m.conn.size());
    }

    bool nodes_v2(std::istream& f) {
        std::string line;
        std::getline(f, line);
        const long long n = std::stoll(line);
        m.xy.assign(2 * n, 0.0);
        for (long long i = 0; i < n; ++i) {
            std::getline(f, line);
            std::istringstream ss(line);
            long long tag; double x = 0, y = 0, z = 0;
            ss >> tag >> x >> y >> z;
            node_index[tag] = i;
            m.xy[2 * i] = x; m.xy[2 * i + 1] = y;
        }
        std::getline(f, line);   // $EndNodes
        return true;
    }

    bool nodes_v4(std::istream& f) {
        std::string line;
        std::getline(f, line);
        std::istringstream hs(line);
        long long nb = 0, n = 0, lo, hi;
        hs >> nb >> n >> lo >> hi;
        m.xy.assign(2 * n, 0.0);
        long long base = 0;
        for (long long b = 0; b < nb; ++b) {
            std::getline(f, line);
            std::istringstream bs(line);
            int dim, etag, param; long long cnt = 0;
            bs >> dim >> etag >> param >> cnt;
            for (long long i = 0; i < cnt; ++i) {
                std::getline(f, line);
                node_index[std::stoll(line)] = base + i;
            }
            for (long long i = 0; i < cnt; ++i) {
                std::getline(f, line);
                std::istringstream cs(line);
                double x = 0, y = 0, z = 0;
                cs >> x >> y >> z;
                m.xy[2 * (base + i)] = x; m.xy[2 * (base + i) + 1] = y;
            }
            base += cnt;
        }
        std::getline(f, line);   // $EndNodes
        return true;
    }

    bool elements_v2(std::istream& f) {
        std::string line;
        std::getline(f, line);
        const long long n = std::stoll(line);
        for (long long i = 0; i < n; ++i) {
            std::getline(f, line);
            std::istringstream ss(line);
            long long id; int type, ntags;
            ss >> id >> type >> ntags;
            type_counts[type]++;
            int phys = 0;
            for (int t = 0; t < ntags; ++t) {
                int v;
                ss >> v;
                if (t == 0) phys = v;
            }
            const int nn = gmsh_nodes(type);
            if (nn < 0) continue;
            std::vector<int64_t> nodes(nn);
            for (int k = 0; k < nn; ++k) {
                long long tag;
                ss >> tag;
                if (!node(tag, nodes[k])) return false;
            }
            element(type, phys, nodes);
        }
        std::getline(f, line);   // $EndElements
        return true;
    }

    bool elements_v4(std::istream& f) {
        std::string line;
        std::getline(f, line);
        std::istringstream hs(line);
        long long nb = 0, n, lo, hi;
        hs >> nb >> n >> lo >> hi;
        for (long long b = 0; b < nb; ++b) {
            std::getline(f, line);
            std::istringstream bs(line);
            int dim, etag, type; long long cnt = 0;
            bs >> dim >> etag >> type >> cnt;
            type_counts[type] += cnt;
            const int nn = gmsh_nodes(type);
            int phys = 0;
            if (dim == 1) {
                auto it = curve_phys.find(etag);
                if (it != curve_phys.end()) phys = it->second;
            }
            for (long long e = 0; e < cnt; ++e) {
                std::getline(f, line);
                if (nn < 0 || type == 15) continue;
                std::istringstream es(line);
                long long id;
                es >> id;
                std::vector<int64_t> nodes(nn);
                for (int k = 0; k < nn; ++k) {
                    long long tag;
                    es >> tag;
                    if (!node(tag, nodes[k])) return false;
                }
                element(type, phys, nodes);
            }
        }
        std::getline(f, line);   // $EndElements
        return true;
    }

    void physical_names(std::istream& f) {
        std::string line;
        std::getline(f, line);
        const int n = std::stoi(line);
        for (int i = 0; i < n; ++i) {
            std::getline(f, line);
            std::istringstream ss(line);
            int dim, tag;
            ss >> dim >> tag;
            std::string name;
            std::getline(ss, name);
            const size_t s = name.find_first_not_of(" \t");
            name = (s == std::string::npos) ? std::string() : name.substr(s);
            if (!name.empty() && name.front() == '"') name.erase(0, 1);
            if (!name.empty() && name.back() == '"') name.pop_back();
            names[{dim, tag}] = name;
        }
        skip_to(f, "$EndPhysicalNames");
    }

    void entities(std::istream& f) {
        std::string line;
        std::getline(f, line);
        std::istringstream hs(line);
        long long np = 0, nc = 0, ns = 0, nv = 0;
        hs >> np >> nc >> ns >> nv;
        for (long long i = 0; i < np; ++i) std::getline(f, line);
        for (long long i = 0; i < nc; ++i) {
            std::getline(f, line);
            std::istringstream ss(line);
            int tag; double b[6]; int nphys = 0;
            ss >> tag >> b[0] >> b[1] >> b[2] >> b[3] >> b[4] >> b[5] >> nphys;
            if (nphys > 0) {
                int p;
                ss >> p;
                curve_phys[tag] = p;
            }
        }
        for (long long i = 0; i < ns + nv; ++i) std::getline(f, line);
        skip_to(f, "$EndEntities");
    }

    static void skip_to(std::istream& f, const std::string& end) {
        std::string line;
        while (std::getline(f, line))
            if (line.find(end) != std::string::npos) break;
    }
};

}  // namespace

int infer_bc_type(const std::string& name) {
    std::string s = name;
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    if (contains(s, "wall")) return (contains(s, "slip") || contains(s, "inviscid")) ? ZJ_BC_SLIPWALL : ZJ_BC_WALL;
    if (contains(s, "airfoil") || contains(s, "wing") || contains(s, "body") || contains(s, "surface"))
        return ZJ_BC_WALL;
    if (contains(s, "farfield") || contains(s, "far_field") || contains(s, "far-field") ||
        contains(s, "freestream"))
        return ZJ_BC_FARFIELD;
    if (contains(s, "inflow") || contains(s, "inlet")) return ZJ_BC_INFLOW;
    if (contains(s, "outflow") || contains(s, "outlet") || contains(s, "exit") || s == "out")
        return ZJ_BC_OUTFLOW;
    if (contains(s, "symmetry") || contains(s, "sym")) return ZJ_BC_SYMMETRY;
    if (contains(s, "periodic")) return ZJ_BC_PERIODIC;
    return ZJ_BC_WALL;
}

bool read_gmsh(const std::string& path, GmshMesh& m, std::string& err) {
    m = GmshMesh();
    std::ifstream f(path);
    if (!f.is_open()) { err = "Failed to open Gmsh file: " + path; return false; }
    double version = 0.0;
    int file_type = 0, dsize = 0;
    std::string line;
    while (std::getline(f, line)) {
        if (line.find("$MeshFormat") != std::string::npos) {
            std::getline(f, line);
            std::istringstream ss(line);
            ss >> version >> file_type >> dsize;
            break;
        }
    }
    if (version == 0.0) { err = "No $MeshFormat section found in: " + path; return false; }
    if (file_type != 0) { err = "Only ASCII Gmsh files are supported (file_type must be 0)"; return false; }
    f.clear();
    f.seekg(0);

    Reader rd{m, err};
    m.offs.push_back(0);
    bool have_nodes = false, have_elems = false;
    while (std::getline(f, line)) {
        if (line.find("$MeshFormat") != std::string::npos) {
            Reader::skip_to(f, "$EndMeshFormat");
        } else if (line.find("$PhysicalNames") != std::string::npos) {
            rd.physical_names(f);
        } else if (line.find("$Entities") != std::string::npos) {
            rd.entities(f);
        } else if (line.find("$Nodes") != std::string::npos) {
            if (!(version >= 4.0 ? rd.nodes_v4(f) : rd.nodes_v2(f))) return false;
            have_nodes = true;
        } else if (line.find("$Elements") != std::string::npos) {
            if (!(version >= 4.0 ? rd.elements_v4(f) : rd.elements_v2(f))) return false;
            have_elems = true;
        } else if (!line.empty() && line[0] == '$' && line.find("$End") == std::string::npos) {
            Reader::skip_to(f, "$End" + line.substr(1));
        }
    }
    if (!have_nodes) { err = "No $Nodes section found"; return false; }
    if (!have_elems) { err = "No $Elements section found"; return false; }
    if (m.etype.empty()) {
        std::string d = "No 2D elements (triangles/quads) found in Gmsh file.";
        if (rd.type_counts.empty()) {
            d += " The $Elements section contained no elements at all.";
        } else {
            d += "\nElement types found in file:";
            bool has3d = false;
            for (const auto& kv : rd.type_counts) {
                d += "\n  Type " + std::to_string(kv.first) + " (" + gmsh_name(kv.first) + "): " +
                     std::to_string(kv.second);
                has3d = has3d || is_3d(kv.first);
            }
            d += has3d ? "\n\nThis appears to be a 3D mesh; a 2D mesh of triangles or quadrilaterals is needed."
                       : "\n\nNone of these are supported 2D elements (types 2, 3, 9, 10, 16, 37).";
        }
        err = d;
        return false;
    }
    // boundary groups and boundary edges (end vertices + physical tag)
    std::set<int> tags;
    for (size_t i = 0; i < rd.edges.size(); ++i) {
        if (rd.edge_tags[i] > 0) tags.insert(rd.edge_tags[i]);
        if (rd.edges[i].size() >= 2 && rd.edge_tags[i] > 0) {
            m.bnd.push_back(rd.edges[i][0]);
            m.bnd.push_back(rd.edges[i][1]);
            m.bnd.push_back(rd.edge_tags[i]);
        }
    }
    for (int t : tags) {
        auto it = rd.names.find({1, t});
        GmshGroup g;
        g.tag = t;
        g.name = (it != rd.names.end()) ? it->second : "BC_" + std::to_string(t);
        g.type = infer_bc_type(g.name);
        m.groups.push_back(g);
    }
    return true;
}

}  // namespace zj
