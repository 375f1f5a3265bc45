// zdx_config.cpp -- host side of the DEM scene: the config grammar, particle/wall set-up and the outputs.
//
// Same grammar, defaults, messages and file formats as zdem_cpu:
//   parse_config_file      src/main.cpp:1531-1689
//   load_mesh_for + particle and wall set-up   src/main.cpp:1883-2022
//   write_vtk_particles    src/main.cpp:1710-1840
//   write_particle_state_txt  src/main.cpp:1842-1870
// Arithmetic keeps the reference's operand order (inertia, L0, wall normals are bit-identical).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <thread>
#include <unordered_map>

#include "../../include/zdemx.h"
#include "zdx_format.h"
#include "zdx_host.h"
#include "zdx_math.cuh"
#include "zdx_scene.h"

namespace zdx {

namespace {

struct M3 {
    double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};
M3 m3_identity() {
    M3 r;
    r.m[0][0] = r.m[1][1] = r.m[2][2] = 1.0;
    return r;
}
M3 m3_from(const double* p) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = p[3 * i + j];
    return r;
}
M3 m3_scale(const M3& a, double s) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] * s;
    return r;
}
M3 m3_mul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            r.m[i][j] = 0.0;
            for (int k = 0; k < 3; ++k) r.m[i][j] += a.m[i][k] * b.m[k][j];
        }
    return r;
}
M3 m3_transpose(const M3& a) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
    return r;
}
// mat3_inverse, src/main.cpp:203-220
M3 m3_inverse(const M3& a) {
    double det = a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
                 a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
                 a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
    if (std::abs(det) < 1e-18) return m3_identity();
    double invdet = 1.0 / det;
    M3 r;
    r.m[0][0] = (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) * invdet;
    r.m[0][1] = -(a.m[0][1] * a.m[2][2] - a.m[0][2] * a.m[2][1]) * invdet;
    r.m[0][2] = (a.m[0][1] * a.m[1][2] - a.m[0][2] * a.m[1][1]) * invdet;
    r.m[1][0] = -(a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) * invdet;
    r.m[1][1] = (a.m[0][0] * a.m[2][2] - a.m[0][2] * a.m[2][0]) * invdet;
    r.m[1][2] = -(a.m[0][0] * a.m[1][2] - a.m[0][2] * a.m[1][0]) * invdet;
    r.m[2][0] = (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]) * invdet;
    r.m[2][1] = -(a.m[0][0] * a.m[2][1] - a.m[0][1] * a.m[2][0]) * invdet;
    r.m[2][2] = (a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0]) * invdet;
    return r;
}
// quat_to_mat3, src/main.cpp:150-164
M3 q_to_m3(Q4 q) {
    Q4 n = qnormalize(q);
    double w = n.w, x = n.x, y = n.y, z = n.z;
    M3 R;
    R.m[0][0] = 1.0 - 2.0 * (y * y + z * z);
    R.m[0][1] = 2.0 * (x * y - z * w);
    R.m[0][2] = 2.0 * (x * z + y * w);
    R.m[1][0] = 2.0 * (x * y + z * w);
    R.m[1][1] = 1.0 - 2.0 * (x * x + z * z);
    R.m[1][2] = 2.0 * (y * z - x * w);
    R.m[2][0] = 2.0 * (x * z - y * w);
    R.m[2][1] = 2.0 * (y * z + x * w);
    R.m[2][2] = 1.0 - 2.0 * (x * x + y * y);
    return R;
}
V3 m3_mul_v(const M3& m, V3 v) {
    return V3{m.m[0][0] * v.x + m.m[0][1] * v.y + m.m[0][2] * v.z, m.m[1][0] * v.x + m.m[1][1] * v.y + m.m[1][2] * v.z,
              m.m[2][0] * v.x + m.m[2][1] * v.y + m.m[2][2] * v.z};
}

}  // namespace

bool parse_config(const std::string& path, SimConfig& cfg, std::string& err) {
    std::ifstream in(path);
    if (!in) {
        err = "Failed to open config: " + path;
        return false;
    }
    std::string line;
    bool in_particle = false, in_wall = false;
    ParticleInit cp;
    WallInit cw;
    while (std::getline(in, line)) {
        if (line.empty()) continue;
        std::string cleaned;
        cleaned.reserve(line.size());
        for (char c : line) {
            if (c == '#') break;
            cleaned.push_back(c == '=' ? ' ' : c);
        }
        std::istringstream iss(cleaned);
        std::string key;
        if (!(iss >> key)) continue;
        if (key == "particle") {
            if (in_particle) cfg.particles.push_back(cp);
            if (in_wall) {
                cfg.walls.push_back(cw);
                in_wall = false;
            }
            cp = ParticleInit{};
            in_particle = true;
            continue;
        }
        if (key == "end_particle" || key == "particle_end") {
            if (in_particle) {
                cfg.particles.push_back(cp);
                in_particle = false;
            }
            continue;
        }
        if (key == "wall") {
            if (in_particle) {
                cfg.particles.push_back(cp);
                in_particle = false;
            }
            if (in_wall) cfg.walls.push_back(cw);
            cw = WallInit{};
            in_wall = true;
            continue;
        }
        if (key == "end_wall" || key == "wall_end") {
            if (in_wall) {
                cfg.walls.push_back(cw);
                in_wall = false;
            }
            continue;
        }
        if (in_particle) {
            if (key == "stl") iss >> cp.stl;
            else if (key == "pos") iss >> cp.pos[0] >> cp.pos[1] >> cp.pos[2];
            else if (key == "vel") iss >> cp.vel[0] >> cp.vel[1] >> cp.vel[2];
            else if (key == "omega") iss >> cp.omega[0] >> cp.omega[1] >> cp.omega[2];
            else if (key == "quat") iss >> cp.quat[0] >> cp.quat[1] >> cp.quat[2] >> cp.quat[3];
            else if (key == "scale") iss >> cp.scale;
            else if (key == "density") iss >> cp.density;
            else if (key == "young") iss >> cp.young;
            else if (key == "poisson") iss >> cp.poisson;
            else if (key == "mu") iss >> cp.mu;
            else if (key == "restitution") iss >> cp.restitution;
        } else if (in_wall) {
            if (key == "stl") iss >> cw.stl;
            else if (key == "pos") iss >> cw.pos[0] >> cw.pos[1] >> cw.pos[2];
            else if (key == "quat") iss >> cw.quat[0] >> cw.quat[1] >> cw.quat[2] >> cw.quat[3];
            else if (key == "scale") iss >> cw.scale;
            else if (key == "mu") iss >> cw.mu;
            else if (key == "restitution") iss >> cw.restitution;
        } else if (key == "stl") {
            iss >> cfg.stl;
        } else if (key == "n") {
            iss >> cfg.n;
        } else if (key == "steps") {
            iss >> cfg.steps;
        } else if (key == "dt") {
            iss >> cfg.dt;
        } else if (key == "spacing") {
            iss >> cfg.spacing;
        } else if (key == "split_contacts") {
            int v = 1;
            iss >> v;
            cfg.split_contacts = (v != 0);
        } else if (key == "contact_debug") {
            int v = 0;
            iss >> v;
            cfg.contact_debug = (v != 0);
        } else if (key == "gravity") {
            iss >> cfg.gravity[0] >> cfg.gravity[1] >> cfg.gravity[2];
        } else if (key == "center_mesh") {
            int v = 1;
            iss >> v;
            cfg.center_mesh = (v != 0);
        } else if (key == "vtk_prefix") {
            iss >> cfg.vtk_prefix;
        } else if (key == "output_interval") {
            iss >> cfg.output_interval;
        } else if (key == "output_dir") {
            iss >> cfg.output_dir;
        } else if (key == "v0") {
            iss >> cfg.v0[0] >> cfg.v0[1] >> cfg.v0[2];
        } else if (key == "v1") {
            iss >> cfg.v1[0] >> cfg.v1[1] >> cfg.v1[2];
        } else if (key == "force_law") {
            std::string law;
            iss >> law;
            if (law == "zdem") cfg.force_law = 0;
            else if (law == "feng_min") cfg.force_law = 1;
            else {
                err = "Unknown force_law: " + law + " (zdem or feng_min)";
                return false;
            }
        } else if (key == "feng_k") {
            iss >> cfg.feng_k;
        } else if (key == "contact_cache") {
            iss >> cfg.contact_cache;
        } else if (key == "contact_cache_tau") {
            iss >> cfg.contact_cache_tau;
        }
        // unknown keys are ignored, as in the reference
    }
    if (in_particle) cfg.particles.push_back(cp);
    if (in_wall) cfg.walls.push_back(cw);
    if (cfg.output_interval < 1) cfg.output_interval = 1;
    if (!cfg.stl.empty()) return true;
    if (cfg.particles.empty()) {
        err.clear();  // zdem_cpu fails here without a message (src/main.cpp:1685-1688)
        return false;
    }
    return true;
}

// Particle and wall set-up, src/main.cpp:1883-2022.
int scene_from_config(zdx_ctx* ctx, const SimConfig& cfg, Scene& s, std::string& err) {
    (void)ctx;
    s = Scene{};
    s.cfg = cfg;
    std::unordered_map<std::string, std::vector<double>> tri_cache;
    std::unordered_map<std::string, int> mesh_cache;
    auto add_mesh = [&](const std::vector<double>& tris, bool center) -> int {
        int64_t n = static_cast<int64_t>(tris.size() / 9);
        std::vector<double> out(tris.size());
        double props[17];
        mesh_build(tris.data(), n, center, out.data(), props);
        s.mesh_tris.insert(s.mesh_tris.end(), out.begin(), out.end());
        s.mesh_off.push_back(s.mesh_off.back() + n);
        s.mesh_props.insert(s.mesh_props.end(), props, props + 17);
        return static_cast<int>(s.mesh_off.size() - 2);
    };
    auto load_mesh_for = [&](const std::string& path, double scale) -> int {
        std::string key = path + "|" + std::to_string(scale);
        auto itc = mesh_cache.find(key);
        if (itc != mesh_cache.end()) return itc->second;
        auto it = tri_cache.find(path);
        if (it == tri_cache.end()) {
            std::vector<double> t;
            if (!stl_read(path, t)) return -1;
            tri_cache[path] = t;
            it = tri_cache.find(path);
        }
        std::vector<double> t = it->second;
        for (auto& x : t) x *= scale;
        int idx = add_mesh(t, cfg.center_mesh);
        mesh_cache[key] = idx;
        return idx;
    };

    std::vector<ParticleInit> inits;
    if (!cfg.particles.empty()) {
        inits = cfg.particles;
    } else {
        inits.resize(cfg.n > 0 ? cfg.n : 0);
        for (int i = 0; i < cfg.n; ++i) {
            inits[i].stl = cfg.stl;
            inits[i].pos[0] = cfg.spacing * i;
            const double* v = (i == 0) ? cfg.v0 : (i == 1 ? cfg.v1 : nullptr);
            for (int k = 0; k < 3; ++k) inits[i].vel[k] = v ? v[k] : 0.0;
            inits[i].scale = 1.0;
            inits[i].density = 1.0;
        }
    }
    s.inits = inits;
    s.np = static_cast<int>(inits.size());
    s.state.assign(16 * (size_t)s.np, 0.0);
    s.mat.assign(17 * (size_t)s.np, 0.0);
    s.pmesh.assign(s.np, 0);
    for (int i = 0; i < s.np; ++i) {
        const ParticleInit& init = inits[i];
        std::string stl = init.stl.empty() ? cfg.stl : init.stl;
        if (stl.empty()) {
            err = "Missing stl for particle " + std::to_string(i);
            return ZDX_ERR_CONFIG;
        }
        double scale = init.scale > 0.0 ? init.scale : 1.0;
        int mi = load_mesh_for(stl, scale);
        if (mi < 0) {
            err = "Failed to load STL: " + stl;
            return ZDX_ERR_CONFIG;
        }
        const double* props = &s.mesh_props[17 * (size_t)mi];
        if (props[16] <= 0.0) {
            err = "Mesh has no vertices.";
            return ZDX_ERR_CONFIG;
        }
        double volume = props[0], radius = props[4];
        double mass, inv_mass;
        M3 Ibody, Iinv;
        double density = init.density > 0.0 ? init.density : 1.0;
        if (volume > 0.0) {
            mass = density * volume;
            inv_mass = 1.0 / mass;
            Ibody = m3_scale(m3_from(props + 7), density);
            Iinv = m3_inverse(Ibody);
        } else {
            mass = density;
            inv_mass = 1.0 / mass;
            double I = 0.4 * mass * radius * radius;
            Ibody = m3_identity();
            Ibody.m[0][0] = I;
            Ibody.m[1][1] = I;
            Ibody.m[2][2] = I;
            Iinv = m3_inverse(Ibody);
        }
        double equiv = volume > 0.0 ? std::cbrt(3.0 * volume / (4.0 * 3.141592653589793)) : radius;
        Q4 rot{init.quat[0], init.quat[1], init.quat[2], init.quat[3]};
        M3 R = q_to_m3(rot);
        V3 L = m3_mul_v(m3_mul(m3_mul(R, Ibody), m3_transpose(R)), V3{init.omega[0], init.omega[1], init.omega[2]});
        double* st = &s.state[16 * (size_t)i];
        double stv[16] = {init.pos[0], init.pos[1], init.pos[2], rot.w, rot.x, rot.y, rot.z, init.vel[0], init.vel[1],
                          init.vel[2], init.omega[0], init.omega[1], init.omega[2], L.x, L.y, L.z};
        std::memcpy(st, stv, sizeof(stv));
        double* mt = &s.mat[17 * (size_t)i];
        double mtv[8] = {mass, inv_mass, radius, equiv, init.young, init.poisson, init.mu, init.restitution};
        std::memcpy(mt, mtv, sizeof(mtv));
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) mt[8 + 3 * r + c] = Iinv.m[r][c];
        s.pmesh[i] = mi;
    }
    // walls, src/main.cpp:1989-2022
    for (const auto& wi : cfg.walls) {
        if (wi.stl.empty()) {
            std::cerr << "Wall missing stl path.\n";
            continue;
        }
        std::vector<double> t;
        if (!stl_read(wi.stl, t)) {
            std::cerr << "Failed to load wall STL: " << wi.stl << "\n";
            continue;
        }
        double scale = wi.scale > 0.0 ? wi.scale : 1.0;
        for (auto& x : t) x = x * scale;
        int mi = add_mesh(t, cfg.center_mesh);
        Q4 q{wi.quat[0], wi.quat[1], wi.quat[2], wi.quat[3]};
        Q4 qn = qnormalize(q);
        V3 tp{wi.pos[0], wi.pos[1], wi.pos[2]};
        const double* mt = &s.mesh_tris[9 * (size_t)s.mesh_off[mi]];
        int64_t nt = s.mesh_off[mi + 1] - s.mesh_off[mi];
        for (int64_t k = 0; k < nt; ++k) {
            V3 w[3];
            for (int c = 0; c < 3; ++c) w[c] = qrotate_n(qn, V3{mt[9 * k + 3 * c], mt[9 * k + 3 * c + 1], mt[9 * k + 3 * c + 2]}) + tp;
            for (int c = 0; c < 3; ++c) {
                s.wtris.push_back(w[c].x);
                s.wtris.push_back(w[c].y);
                s.wtris.push_back(w[c].z);
            }
            V3 n = normalize(cross(w[1] - w[0], w[2] - w[0]));
            s.wnormals.push_back(n.x);
            s.wnormals.push_back(n.y);
            s.wnormals.push_back(n.z);
        }
        s.wtri_off.push_back(s.wtri_off.back() + nt);
        s.wmesh.push_back(mi);
        double pose[7] = {wi.pos[0], wi.pos[1], wi.pos[2], wi.quat[0], wi.quat[1], wi.quat[2], wi.quat[3]};
        s.wpose.insert(s.wpose.end(), pose, pose + 7);
        s.wmat.push_back(wi.mu);
        s.wmat.push_back(wi.restitution);
        std::cout << "Loaded wall: " << wi.stl << " (tris=" << nt << ")\n";
    }
    s.nw = static_cast<int>(s.wmesh.size());
    s.force.assign(3 * (size_t)s.np, 0.0);
    s.torque.assign(3 * (size_t)s.np, 0.0);
    s.contact_count.assign(s.np, 0);
    s.host_dirty = false;
    return ZDX_OK;
}

namespace {
struct FileCloser {
    std::FILE* f;
    ~FileCloser() {
        if (f) std::fclose(f);
    }
};
}  // namespace

int output_threads() {
    unsigned h = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(h > 1 ? h - 1 : 1u, 16u));
}

ParticleFrame host_frame(const Scene& s) {
    return ParticleFrame{s.np, s.state.data(), s.force.data(), s.torque.data(), s.contact_count.data()};
}

// write_vtk_particles (src/main.cpp:1710-1840): the same sections, lines and number formats.
bool write_vtk_particles(const std::string& path, const Scene& s, const ParticleFrame& fr, int threads) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::cerr << "Failed to write VTK: " << path << "\n";
        return false;
    }
    FileCloser closer{f};
    const int np = fr.np;
    auto ntri = [&](int i) { return static_cast<std::size_t>(s.mesh_off[s.pmesh[i] + 1] - s.mesh_off[s.pmesh[i]]); };
    std::size_t total_tris = 0;
    for (int i = 0; i < np; ++i) total_tris += ntri(i);
    TextBuf h;
    h.lit("# vtk DataFile Version 3.0\nzdem particles\nASCII\nDATASET POLYDATA\nPOINTS ");
    h.integer(total_tris * 3);
    h.lit(" float\n");
    bool ok = std::fwrite(h.s.data(), 1, h.s.size(), f) == h.s.size();
    ok = write_sliced(f, np, threads, [&](int64_t b, int64_t e, TextBuf& o) {
        for (int64_t i = b; i < e; ++i) {
            const double* st = fr.state + 16 * i;
            Q4 qn = qnormalize(Q4{st[3], st[4], st[5], st[6]});
            V3 pos{st[0], st[1], st[2]};
            const double* mt = &s.mesh_tris[9 * (size_t)s.mesh_off[s.pmesh[i]]];
            for (std::size_t k = 0; k < ntri((int)i); ++k)
                for (int c = 0; c < 3; ++c) {
                    V3 v = qrotate_n(qn, V3{mt[9 * k + 3 * c], mt[9 * k + 3 * c + 1], mt[9 * k + 3 * c + 2]}) + pos;
                    o.f6(v.x);
                    o.ch(' ');
                    o.f6(v.y);
                    o.ch(' ');
                    o.f6(v.z);
                    o.ch('\n');
                }
        }
    }) && ok;
    h.s.clear();
    h.lit("POLYGONS ");
    h.integer(total_tris);
    h.ch(' ');
    h.integer(total_tris * 4);
    h.ch('\n');
    ok = std::fwrite(h.s.data(), 1, h.s.size(), f) == h.s.size() && ok;
    ok = write_sliced(f, (int64_t)total_tris, threads, [&](int64_t b, int64_t e, TextBuf& o) {
        for (int64_t i = b; i < e; ++i) {
            const std::size_t v = (std::size_t)i * 3;
            o.lit("3 ");
            o.integer(v);
            o.ch(' ');
            o.integer(v + 1);
            o.ch(' ');
            o.integer(v + 2);
            o.ch('\n');
        }
    }) && ok;
    h.s.clear();
    h.lit("CELL_DATA ");
    h.integer(total_tris);
    h.lit("\n");
    // one value per triangle of each particle
    auto per_tri = [&](const char* head, auto&& put) {
        h.lit(head);
        ok = std::fwrite(h.s.data(), 1, h.s.size(), f) == h.s.size() && ok;
        h.s.clear();
        ok = write_sliced(f, np, threads, [&](int64_t b, int64_t e, TextBuf& o) {
            for (int64_t i = b; i < e; ++i)
                for (std::size_t t = 0, n = ntri((int)i); t < n; ++t) put((int)i, o);
        }) && ok;
    };
    per_tri("SCALARS id int 1\nLOOKUP_TABLE default\n", [&](int i, TextBuf& o) {
        o.integer(i);
        o.ch('\n');
    });
    per_tri("SCALARS mass float 1\nLOOKUP_TABLE default\n", [&](int i, TextBuf& o) {
        o.f6(s.mat[17 * (size_t)i]);
        o.ch('\n');
    });
    per_tri("SCALARS radius float 1\nLOOKUP_TABLE default\n", [&](int i, TextBuf& o) {
        o.f6(s.mat[17 * (size_t)i + 2]);
        o.ch('\n');
    });
    per_tri("SCALARS contact_count int 1\nLOOKUP_TABLE default\n", [&](int i, TextBuf& o) {
        o.integer(fr.count[i]);
        o.ch('\n');
    });
    auto vec = [&](const char* head, const double* base, std::size_t stride) {
        per_tri(head, [&, base, stride](int i, TextBuf& o) {
            const double* v = base + stride * (size_t)i;
            o.f6(v[0]);
            o.ch(' ');
            o.f6(v[1]);
            o.ch(' ');
            o.f6(v[2]);
            o.ch('\n');
        });
    };
    vec("VECTORS velocity float\n", fr.state + 7, 16);
    vec("VECTORS omega float\n", fr.state + 10, 16);
    vec("VECTORS force float\n", fr.force, 3);
    vec("VECTORS torque float\n", fr.torque, 3);
    h.lit("FIELD FieldData 1\norientation 4 ");
    h.integer(total_tris);
    h.lit(" float\n");
    per_tri("", [&](int i, TextBuf& o) {
        const double* st = fr.state + 16 * (size_t)i;
        o.f6(st[3]);
        o.ch(' ');
        o.f6(st[4]);
        o.ch(' ');
        o.f6(st[5]);
        o.ch(' ');
        o.f6(st[6]);
        o.ch('\n');
    });
    return ok;
}

// write_particle_state_txt (src/main.cpp:1842-1870): fixed, 9 decimals.
bool write_state_txt(const std::string& path, const Scene& s, const ParticleFrame& fr, int threads) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::cerr << "Failed to write particle state: " << path << "\n";
        return false;
    }
    FileCloser closer{f};
    return write_sliced(f, fr.np, threads, [&](int64_t b, int64_t e, TextBuf& o) {
        auto line3 = [&o](const char* key, const double* v, int n) {
            o.lit(key);
            for (int k = 0; k < n; ++k) {
                if (k) o.ch(' ');
                o.fixed9(v[k]);
            }
            o.ch('\n');
        };
        auto line1 = [&o](const char* key, double v) {
            o.lit(key);
            o.fixed9(v);
            o.ch('\n');
        };
        for (int64_t i = b; i < e; ++i) {
            const double* st = fr.state + 16 * i;
            const ParticleInit& init = s.inits[i];
            o.lit("particle\nstl = ");
            o.lit(init.stl.c_str());
            o.ch('\n');
            line3("pos = ", st, 3);
            line3("vel = ", st + 7, 3);
            line3("quat = ", st + 3, 4);
            line3("omega = ", st + 10, 3);
            line1("scale = ", init.scale);
            line1("density = ", init.density);
            line1("young = ", init.young);
            line1("poisson = ", init.poisson);
            line1("mu = ", init.mu);
            line1("restitution = ", init.restitution);
            o.lit("end_particle\n\n");
        }
    });
}

}  // namespace zdx
