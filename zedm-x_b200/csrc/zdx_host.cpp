// zdx_host.cpp -- host-side set-up of the contact path: STL loading and mesh build.
//
// Both run once per mesh on the host, like the reference's.  Results are bit-identical to
// load_stl (src/main.cpp:308-371) and build_mesh (src/main.cpp:445-497); unique_vertices (:287-306) is
// answered with a hash grid instead of the reference's O(V^2) scan, which keeps exactly the same
// vertices in the same order (a corner is dropped iff an earlier kept vertex is within squared
// distance 1e-10, and every such vertex lies in one of the 27 cells checked).
#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/zdemx.h"
#include "zdx_host.h"
#include "zdx_math.cuh"

using zdx::V3;

namespace zdx {

bool stl_read(const std::string& path, std::vector<double>& tris) {
    tris.clear();
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    in.seekg(0, std::ios::end);
    std::streampos size = in.tellg();
    in.seekg(0, std::ios::beg);
    if (size < 84) return false;
    char header[80];
    in.read(header, 80);
    uint32_t n_tri = 0;
    in.read(reinterpret_cast<char*>(&n_tri), 4);
    std::streampos expected = 84 + static_cast<std::streampos>(n_tri) * 50;
    if (expected == size) {
        tris.reserve(static_cast<size_t>(n_tri) * 9);
        for (uint32_t i = 0; i < n_tri; ++i) {
            float data[12];
            uint16_t attr = 0;
            in.read(reinterpret_cast<char*>(data), sizeof(data));
            in.read(reinterpret_cast<char*>(&attr), sizeof(attr));
            for (int k = 3; k < 12; ++k) tris.push_back(static_cast<double>(data[k]));
        }
        return true;
    }
    in.close();
    std::ifstream ia(path);
    if (!ia) return false;
    std::string line;
    std::vector<double> vbuf;
    while (std::getline(ia, line)) {
        std::string s = line;
        for (auto& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
        if (s.find("vertex") != std::string::npos) {
            std::istringstream iss(s);
            std::string tag;
            double x, y, z;
            if (iss >> tag >> x >> y >> z) {
                vbuf.push_back(x);
                vbuf.push_back(y);
                vbuf.push_back(z);
            }
        }
        if (s.find("endloop") != std::string::npos && vbuf.size() >= 9) {
            tris.insert(tris.end(), vbuf.end() - 9, vbuf.end());
        }
    }
    return !tris.empty();
}

namespace {

struct CellKey {
    int64_t x, y, z;
    bool operator==(const CellKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct CellHash {
    size_t operator()(const CellKey& k) const {
        uint64_t h = static_cast<uint64_t>(k.x) * 0x9E3779B97F4A7C15ull;
        h ^= static_cast<uint64_t>(k.y) + 0x7F4A7C159E3779B9ull + (h << 6) + (h >> 2);
        h ^= static_cast<uint64_t>(k.z) + 0x94D049BB133111EBull + (h << 6) + (h >> 2);
        return static_cast<size_t>(h);
    }
};

// unique_vertices, src/main.cpp:287-306, with a grid of cell 1.0001e-5 (> sqrt(1e-10)).
std::vector<V3> unique_vertices(const double* tris, int64_t ntri) {
    const double cell = 1.0001e-5;
    std::vector<V3> kept;
    std::unordered_map<CellKey, std::vector<int>, CellHash> grid;
    for (int64_t i = 0; i < 3 * ntri; ++i) {
        V3 v{tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
        CellKey c{static_cast<int64_t>(std::floor(v.x / cell)), static_cast<int64_t>(std::floor(v.y / cell)),
                  static_cast<int64_t>(std::floor(v.z / cell))};
        bool found = false;
        for (int dx = -1; dx <= 1 && !found; ++dx)
            for (int dy = -1; dy <= 1 && !found; ++dy)
                for (int dz = -1; dz <= 1 && !found; ++dz) {
                    auto it = grid.find(CellKey{c.x + dx, c.y + dy, c.z + dz});
                    if (it == grid.end()) continue;
                    for (int k : it->second) {
                        V3 d = v - kept[k];
                        if (dot(d, d) <= 1e-10) {
                            found = true;
                            break;
                        }
                    }
                }
        if (!found) {
            grid[c].push_back(static_cast<int>(kept.size()));
            kept.push_back(v);
        }
    }
    return kept;
}

}  // namespace

void mesh_build(const double* tris, int64_t ntri, bool center_mesh, double* tris_out, double* props) {
    std::vector<V3> verts = unique_vertices(tris, ntri);
    // compute_mass_properties, src/main.cpp:373-443
    double det_sum = 0.0;
    V3 csum{0.0, 0.0, 0.0};
    double Ixx = 0.0, Iyy = 0.0, Izz = 0.0, Ixy = 0.0, Ixz = 0.0, Iyz = 0.0;
    for (int64_t t = 0; t < ntri; ++t) {
        const double* p = tris + 9 * t;
        V3 a{p[0], p[1], p[2]}, b{p[3], p[4], p[5]}, c{p[6], p[7], p[8]};
        double det = dot(a, cross(b, c));
        det_sum += det;
        csum = csum + ((a + b) + c) * det;
        double x1 = a.x, x2 = b.x, x3 = c.x, y1 = a.y, y2 = b.y, y3 = c.y, z1 = a.z, z2 = b.z, z3 = c.z;
        double f2x = x1 * x1 + x2 * x2 + x3 * x3 + x1 * x2 + x1 * x3 + x2 * x3;
        double f2y = y1 * y1 + y2 * y2 + y3 * y3 + y1 * y2 + y1 * y3 + y2 * y3;
        double f2z = z1 * z1 + z2 * z2 + z3 * z3 + z1 * z2 + z1 * z3 + z2 * z3;
        Ixx += det * (f2y + f2z);
        Iyy += det * (f2x + f2z);
        Izz += det * (f2x + f2y);
        double gxy = 2.0 * x1 * y1 + 2.0 * x2 * y2 + 2.0 * x3 * y3 + x1 * y2 + x2 * y1 + x1 * y3 + x3 * y1 + x2 * y3 + x3 * y2;
        double gxz = 2.0 * x1 * z1 + 2.0 * x2 * z2 + 2.0 * x3 * z3 + x1 * z2 + x2 * z1 + x1 * z3 + x3 * z1 + x2 * z3 + x3 * z2;
        double gyz = 2.0 * y1 * z1 + 2.0 * y2 * z2 + 2.0 * y3 * z3 + y1 * z2 + y2 * z1 + y1 * z3 + y3 * z1 + y2 * z3 + y3 * z2;
        Ixy += det * gxy;
        Ixz += det * gxz;
        Iyz += det * gyz;
    }
    double volume = 0.0;
    V3 centroid{0.0, 0.0, 0.0};
    double I[9] = {0.0};
    if (!(std::abs(det_sum) < 1e-18)) {
        if (det_sum < 0.0) {
            det_sum = -det_sum;
            csum = csum * -1.0;
            Ixx *= -1.0; Iyy *= -1.0; Izz *= -1.0; Ixy *= -1.0; Ixz *= -1.0; Iyz *= -1.0;
        }
        volume = det_sum / 6.0;
        centroid = csum / (4.0 * det_sum);
        Ixx /= 60.0; Iyy /= 60.0; Izz /= 60.0;
        Ixy /= -120.0; Ixz /= -120.0; Iyz /= -120.0;
        I[0] = Ixx; I[4] = Iyy; I[8] = Izz;
        I[1] = Ixy; I[3] = Ixy; I[2] = Ixz; I[6] = Ixz; I[5] = Iyz; I[7] = Iyz;
    }
    // build_mesh, src/main.cpp:445-497
    double Icm[9];
    std::memcpy(Icm, I, sizeof(I));
    if (volume > 0.0) {
        double cc = dot(centroid, centroid);
        double cv[3] = {centroid.x, centroid.y, centroid.z};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double shift = (r == c ? 1.0 : 0.0) * cc - cv[r] * cv[c];
                Icm[3 * r + c] = I[3 * r + c] - shift * volume;
            }
    }
    V3 center = centroid;
    if (tris_out != tris) std::memcpy(tris_out, tris, sizeof(double) * 9 * static_cast<size_t>(ntri));
    if (center_mesh) {
        for (auto& v : verts) v = v - centroid;
        for (int64_t i = 0; i < 3 * ntri; ++i) {
            V3 v{tris_out[3 * i], tris_out[3 * i + 1], tris_out[3 * i + 2]};
            v = v - centroid;
            tris_out[3 * i] = v.x;
            tris_out[3 * i + 1] = v.y;
            tris_out[3 * i + 2] = v.z;
        }
        center = V3{0.0, 0.0, 0.0};
    }
    double r2 = 0.0;
    const double inf = std::numeric_limits<double>::infinity();
    V3 mn{inf, inf, inf}, mx{-inf, -inf, -inf};
    for (const auto& v : verts) {
        r2 = smax(r2, dot(v, v));
        mn.x = smin(mn.x, v.x); mn.y = smin(mn.y, v.y); mn.z = smin(mn.z, v.z);
        mx.x = smax(mx.x, v.x); mx.y = smax(mx.y, v.y); mx.z = smax(mx.z, v.z);
    }
    double edge_sum = 0.0;
    for (int64_t t = 0; t < ntri; ++t) {
        const double* p = tris_out + 9 * t;
        V3 a{p[0], p[1], p[2]}, b{p[3], p[4], p[5]}, c{p[6], p[7], p[8]};
        edge_sum += norm(b - a);
        edge_sum += norm(c - b);
        edge_sum += norm(a - c);
    }
    props[0] = volume;
    props[1] = center.x; props[2] = center.y; props[3] = center.z;
    props[4] = std::sqrt(r2);
    props[5] = ntri > 0 ? edge_sum / static_cast<double>(3 * ntri) : 0.0;
    props[6] = norm(mx - mn);
    for (int i = 0; i < 9; ++i) props[7 + i] = Icm[i];
    props[16] = static_cast<double>(verts.size());
}

}  // namespace zdx

extern "C" int64_t zdx_stl_load(const char* path, double* tris, int64_t cap) {
    if (!path) return -ZDX_ERR_INVALID;
    std::vector<double> t;
    if (!zdx::stl_read(path, t)) return -ZDX_ERR_IO;
    int64_t n = static_cast<int64_t>(t.size() / 9);
    if (tris && cap > 0) std::memcpy(tris, t.data(), sizeof(double) * 9 * static_cast<size_t>(std::min(n, cap)));
    return n;
}

extern "C" int zdx_mesh_build(const double* tris, int64_t ntri, int center_mesh, double* tris_out, double* props17) {
    if (ntri < 0 || (ntri > 0 && (!tris || !tris_out)) || !props17) return ZDX_ERR_INVALID;
    zdx::mesh_build(tris, ntri, center_mesh != 0, tris_out, props17);
    return ZDX_OK;
}
