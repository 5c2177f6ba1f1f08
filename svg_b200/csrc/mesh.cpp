// Host mesh construction, compiled with -ffp-contract=off so every derived
// quantity is the plain IEEE sequence the reference spells out.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <thread>
#include <vector>

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

namespace {
// Run fn(begin, end) over [0, n) on up to hardware_concurrency threads (one
// thread for small n).
template <class F>
void parallel_for(int64_t n, F fn) {
    const int64_t kMinPerThread = 1 << 16;
    int nt = (int)std::min<int64_t>(std::max(1u, std::thread::hardware_concurrency()), 32);
    nt = (int)std::min<int64_t>(nt, std::max<int64_t>(1, n / kMinPerThread));
    if (nt <= 1) {
        fn((int64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) th.emplace_back(fn, n * t / nt, n * (t + 1) / nt);
    for (auto& x : th) x.join();
}
}  // namespace

// Mesh::LoadFromFile (Mesh.cu:62-123) from arrays, plus the per-half-edge
// geometry the kernels read instead of recomputing it per window.
//
// Twins follow the reference's std::map pairing (Mesh.cu:66-84): half-edges
// are grouped by their unordered vertex pair; within a group (in half-edge
// order) every later half-edge pairs with the first, and the first keeps the
// last of them.  Groups are formed by a counting sort on the smaller vertex
// and a stable sort by the larger one inside each (small) bucket, in parallel.
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
    m.he.resize(E);   // every field is written below
    m.geo.resize(E);
    m.vr.assign(nv, VertRec{-1, 0});
    m.angle.assign(nv, 0.0);

    // half-edge endpoints and lengths
    parallel_for(E, [&](int64_t b, int64_t e_end) {
        for (int64_t e = b; e < e_end; ++e) {
            const int64_t f = e / 3;
            const int j = (int)(e % 3);
            const int32_t a = faces[3 * f + j], c = faces[3 * f + (j + 1) % 3];
            HeRec& h = m.he[e];
            h.v0 = a;
            h.v1 = c;
            h.twin = -1;
            h.pad = 0;
            h.corner = 0.0;
            const double* pa = &pos[3 * (size_t)a];
            const double* pb = &pos[3 * (size_t)c];
            double dx = pa[0] - pb[0], dy = pa[1] - pb[1], dz = pa[2] - pb[2];
            h.len = std::sqrt(dx * dx + dy * dy + dz * dz);
        }
    });

    // twins: bucket half-edges by their smaller vertex (counting sort keeps
    // half-edge order), then order each bucket by the larger vertex (stable)
    std::vector<int32_t> start((size_t)nv + 1, 0), order((size_t)E);
    for (int32_t e = 0; e < E; ++e) {
        const HeRec& h = m.he[e];
        ++start[(size_t)std::min(h.v0, h.v1) + 1];
    }
    for (int32_t v = 0; v < nv; ++v) start[v + 1] += start[v];
    {
        std::vector<int32_t> fill(start.begin(), start.end() - 1);
        for (int32_t e = 0; e < E; ++e) {
            const HeRec& h = m.he[e];
            order[(size_t)fill[(size_t)std::min(h.v0, h.v1)]++] = e;
        }
    }
    parallel_for(nv, [&](int64_t b, int64_t v_end) {
        for (int64_t v = b; v < v_end; ++v) {
            int32_t* o = order.data() + start[v];
            const int32_t n = start[v + 1] - start[v];
            auto hi = [&](int32_t e) { return std::max(m.he[e].v0, m.he[e].v1); };
            for (int32_t i = 1; i < n; ++i) {  // insertion sort by larger vertex, stable
                const int32_t x = o[i];
                const int32_t kx = hi(x);
                int32_t j = i - 1;
                while (j >= 0 && hi(o[j]) > kx) {
                    o[j + 1] = o[j];
                    --j;
                }
                o[j + 1] = x;
            }
            for (int32_t i = 0; i < n;) {
                int32_t k = i + 1;
                while (k < n && hi(o[k]) == hi(o[i])) ++k;
                if (k - i >= 2) {
                    const int32_t first = o[i];
                    for (int32_t q = i + 1; q < k; ++q) m.he[o[q]].twin = first;
                    m.he[first].twin = o[k - 1];
                }
                i = k;
            }
        }
    });

    // corner angles and unfolded positions per half-edge
    parallel_for(E, [&](int64_t b, int64_t e_end) {
        for (int64_t e = b; e < e_end; ++e) {
            const int64_t nx = e - e % 3 + (e % 3 + 1) % 3;
            const int64_t pv = e - e % 3 + (e % 3 + 2) % 3;
            const double l0 = m.he[e].len, l1 = m.he[nx].len, l2 = m.he[pv].len;
            double c = (l0 * l0 + l2 * l2 - l1 * l1) / (2.0 * l0 * l2);
            if (c > 1.0) c = 1.0;
            else if (c < -1.0) c = -1.0;
            m.he[e].corner = std::acos(c);
            HeGeo& g = m.geo[e];
            g.ax = (l1 * l1 + l0 * l0 - l2 * l2) / (2.0 * l0);
            g.ay = -std::sqrt(std::fabs(l1 * l1 - g.ax * g.ax));
            g.tx = (l2 * l2 + l0 * l0 - l1 * l1) / (2.0 * l0);
            g.ty = std::sqrt(std::fabs(l2 * l2 - g.tx * g.tx));
        }
    });
    // vertex angle sums in half-edge order (Mesh.cu:106-122); firstEdge = the last leaving half-edge
    for (int32_t e = 0; e < E; ++e) {
        m.angle[m.he[e].v0] += m.he[e].corner;
        m.vr[m.he[e].v0].first = e;
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
