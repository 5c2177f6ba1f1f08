// Host mesh construction, compiled with -ffp-contract=off so every derived
// quantity is the plain IEEE sequence the reference spells out.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>

#include "svg_internal.h"

namespace svgb {

namespace {
constexpr double kPi = 3.141592653589793238;  // Geometry.cuh:18
}

// OBJ reader with the reference's accepted subset (Mesh.cu:40-59): a line
// starting "v " or "v\t" gives a vertex from its first three numbers, a line
// starting 'f' a triangle from its first three indices (1-based).  Other lines
// are ignored.  Beyond the reference: an index token may carry "/vt/vn"
// suffixes, and extra indices on an 'f' line are ignored instead of spilling
// into the next line's parse.
std::string parse_obj(const char* path, std::vector<double>& pos, std::vector<int32_t>& faces, bool& io_error) {
    io_error = false;
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        io_error = true;
        return std::string("cannot open file ") + path;
    }
    std::string line;
    char buf[1 << 16];
    long lineno = 0;
    std::string err;
    auto handle = [&](const std::string& s) {
        ++lineno;
        if (s.size() < 2) return;
        if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            const char* p = s.c_str() + 1;
            double xyz[3];
            for (int k = 0; k < 3; ++k) {
                char* end = nullptr;
                xyz[k] = std::strtod(p, &end);
                if (end == p) {
                    if (err.empty()) err = "bad vertex at line " + std::to_string(lineno);
                    return;
                }
                p = end;
            }
            pos.insert(pos.end(), xyz, xyz + 3);
        } else if (s[0] == 'f') {
            const char* p = s.c_str() + 1;
            long idx[3];
            for (int k = 0; k < 3; ++k) {
                while (*p == ' ' || *p == '\t') ++p;
                char* end = nullptr;
                idx[k] = std::strtol(p, &end, 10);
                if (end == p) {
                    if (err.empty()) err = "bad face at line " + std::to_string(lineno);
                    return;
                }
                p = end;
                while (*p && *p != ' ' && *p != '\t') ++p;  // skip "/vt/vn"
            }
            for (int k = 0; k < 3; ++k) faces.push_back((int32_t)(idx[k] - 1));
        }
    };
    while (std::fgets(buf, sizeof(buf), f)) {
        line.append(buf);
        if (!line.empty() && line.back() == '\n') {
            line.pop_back();
            if (!line.empty() && line.back() == '\r') line.pop_back();
            handle(line);
            line.clear();
        }
    }
    if (!line.empty()) handle(line);
    std::fclose(f);
    return err;
}

// Mesh::LoadFromFile (Mesh.cu:62-123) from arrays, plus the per-half-edge
// geometry the kernels read instead of recomputing it per window.
std::string build_host_mesh(int32_t nv, const double* pos, int32_t nf, const int32_t* faces, HostMesh& m) {
    if (nv <= 0 || nf <= 0) return "mesh needs at least one vertex and one face";
    if ((int64_t)nf * 3 >= (int64_t)1 << 31) return "too many faces for int32 half-edge ids";
    if (nf >= (1 << 24) - 2) return "too many faces: window levels are kept in 24 bits";
    m.nv = nv;
    m.nf = nf;
    m.ne = 3 * nf;
    m.pos.assign(pos, pos + 3 * (size_t)nv);
    m.faces.assign(faces, faces + 3 * (size_t)nf);
    for (size_t i = 0; i < m.faces.size(); ++i)
        if (m.faces[i] < 0 || m.faces[i] >= nv)
            return "face " + std::to_string(i / 3) + " references vertex " + std::to_string(m.faces[i]) +
                   " outside [0," + std::to_string(nv) + ")";
    const int32_t E = m.ne;
    m.he.assign(E, HeRec{});
    m.geo.assign(E, HeGeo{});
    m.vr.assign(nv, VertRec{-1, 0});
    m.angle.assign(nv, 0.0);

    std::unordered_map<uint64_t, int32_t> first;
    first.reserve((size_t)E);
    for (int32_t f = 0; f < nf; ++f) {
        for (int j = 0; j < 3; ++j) {
            int32_t e = 3 * f + j;
            int32_t a = faces[3 * f + j], b = faces[3 * f + (j + 1) % 3];
            HeRec& h = m.he[e];
            h.v0 = a;
            h.v1 = b;
            h.twin = -1;
            const double* pa = &pos[3 * (size_t)a];
            const double* pb = &pos[3 * (size_t)b];
            double dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
            h.len = std::sqrt(dx * dx + dy * dy + dz * dz);
            uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
            uint64_t key = ((uint64_t)lo << 32) | hi;
            auto it = first.find(key);
            if (it != first.end()) {  // pairs with the first half-edge of this vertex pair
                h.twin = it->second;
                m.he[it->second].twin = e;
            } else {
                first.emplace(key, e);
            }
        }
    }
    for (int32_t e = 0; e < E; ++e) {
        int32_t nx = e - e % 3 + (e % 3 + 1) % 3;
        int32_t pv = e - e % 3 + (e % 3 + 2) % 3;
        double l0 = m.he[e].len, l1 = m.he[nx].len, l2 = m.he[pv].len;
        double c = (l0 * l0 + l2 * l2 - l1 * l1) / (2.0 * l0 * l2);
        if (c > 1.0) c = 1.0;
        else if (c < -1.0) c = -1.0;
        c = std::acos(c);
        m.he[e].corner = c;
        m.angle[m.he[e].v0] += c;  // summed in half-edge order (Mesh.cu:106-122)
        m.vr[m.he[e].v0].first = e;

        HeGeo& g = m.geo[e];
        g.ax = (l1 * l1 + l0 * l0 - l2 * l2) / (2.0 * l0);
        g.ay = -std::sqrt(std::fabs(l1 * l1 - g.ax * g.ax));
        g.tx = (l2 * l2 + l0 * l0 - l1 * l1) / (2.0 * l0);
        g.ty = std::sqrt(std::fabs(l2 * l2 - g.tx * g.tx));
    }
    for (int32_t v = 0; v < nv; ++v) {
        int32_t fl = 0;
        if (!(m.angle[v] < 2.0 * kPi)) fl |= kVertSaddleGE;  // saddle test of Initialize / GenSubWins
        if (m.angle[v] > 2.0 * kPi) fl |= kVertSaddleGT;     // saddle test of PropagateWindow
        m.vr[v].flags = fl;
    }
    return std::string();
}

}  // namespace svgb
