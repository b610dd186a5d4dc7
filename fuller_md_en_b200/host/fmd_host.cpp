// fmd_host.cpp -- see fmd_host.hpp.
#include "fmd_host.hpp"

#include <dirent.h>
#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <thread>

namespace fmdh {

Opts parse_args(int argc, char** argv) {
    Opts o;
    for (int i = 1; i < argc; i++) {
        const std::string a = argv[i];
        if (a.compare(0, 2, "--") != 0) continue;
        const size_t eq = a.find('=');
        std::string k = eq == std::string::npos ? a.substr(2) : a.substr(2, eq - 2);
        const std::string v = eq == std::string::npos ? std::string() : a.substr(eq + 1);
        for (char& c : k) c = (char)std::tolower((unsigned char)c);
        o[k] = v;
    }
    return o;
}

std::string gopt(const Opts& o, const std::string& k, const std::string& d) {
    auto it = o.find(k);
    return it == o.end() ? d : it->second;
}

bool file_exists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

bool dir_exists(const char* p) {
    struct stat st;
    return stat(p, &st) == 0 && S_ISDIR(st.st_mode);
}

std::string unique_file(const std::string& base, const std::string& ext) {
    if (!file_exists(base + ext)) return base + ext;
    for (int n = 1; n <= 9999; n++) {
        std::string c = base + "_" + std::to_string(n) + ext;
        if (!file_exists(c)) return c;
    }
    return base + "_9999" + ext;
}

std::string restart_filename(const std::string& oname, int istep, int nsteps) {
    std::string b = oname;
    const size_t dot = b.rfind('.');
    if (dot != std::string::npos) b = b.substr(0, dot);
    const size_t p = b.find("ovito_traj");
    if (p != std::string::npos) b.replace(p, 10, "restart");
    if (istep == nsteps) return b + ".rst";
    int digits = 1;
    for (int x = nsteps; x >= 10; x /= 10) digits++;
    char buf[64];
    snprintf(buf, sizeof(buf), "_%0*d", digits, istep);
    return b + buf + ".rst";
}

std::string build_suffix(const Opts& o) {
    static const char* keys[] = {"fullerene", "crystal", "cell", "temp", "pres", "step", "dt", "init_scale", "seed"};
    std::string s;
    for (const char* k : keys) {
        auto it = o.find(k);
        if (it == o.end()) continue;
        std::string v = it->second;
        for (char& c : v)
            if (c == ':') c = '_';
        if (v.size() >= 2 && v.compare(v.size() - 2, 2, ".0") == 0) v = v.substr(0, v.size() - 2);
        s += "_" + std::string(k) + "_" + v;
    }
    return s;
}

std::pair<std::string, std::string> resolve_fullerene(const std::string& spec, const std::string& lib, Dialect d) {
    std::string sl = spec;
    for (char& c : sl) c = (char)std::tolower((unsigned char)c);
    if (sl == "buckyball" || sl == "c60" || sl == "c60:ih") return {lib + "/C60-76/C60-Ih.cc1", "C60(Ih)"};
    if (sl == "c70" || sl == "c70:d5h") return {lib + "/C60-76/C70-D5h.cc1", "C70(D5h)"};
    if (sl == "c72" || sl == "c72:d6d") return {lib + "/C60-76/C72-D6d.cc1", "C72(D6d)"};
    if (sl == "c74" || sl == "c74:d3h") return {lib + "/C60-76/C74-D3h.cc1", "C74(D3h)"};
    if (sl.compare(0, 4, "c76:") == 0 && sl.size() > 4) {
        const std::string sym = spec.substr(4);
        return {lib + "/C60-76/C76-" + sym + ".cc1", "C76(" + sym + ")"};
    }
    if (sl.compare(0, 4, "c84:") == 0) {
        const std::string rest = spec.substr(4);
        const size_t c = rest.find(':');
        if (c != std::string::npos) {
            const int n = std::atoi(rest.substr(0, c).c_str());
            char buf[64];
            snprintf(buf, sizeof(buf), "C84-No.%02d-%s.cc1", n, rest.substr(c + 1).c_str());
            return {lib + "/C84/" + buf, "C84 No." + std::to_string(n)};
        }
        const int n = std::atoi(rest.c_str());
        char pfx[32];
        snprintf(pfx, sizeof(pfx), "C84-No.%02d-", n);
        const std::string dpath = lib + "/C84";
        if (DIR* dp = opendir(dpath.c_str())) {
            while (struct dirent* ep = readdir(dp)) {
                const std::string fn = ep->d_name;
                if (fn.find(pfx) == 0 && fn.size() > 4 && fn.compare(fn.size() - 4, 4, ".cc1") == 0) {
                    closedir(dp);
                    return {dpath + "/" + fn, "C84 No." + std::to_string(n)};
                }
            }
            closedir(dp);
        }
    }
    fprintf(stderr, d == Dialect::LJ ? "Unknown fullerene: %s\n" : "Unknown: %s\n", spec.c_str());
    exit(1);
}

Molecule load_cc1(const std::string& path, Dialect d) {
    Molecule m;
    std::ifstream f(path);
    if (!f) {
        fprintf(stderr, d == Dialect::AI ? "Cannot open %s\n" : "Error: cannot open %s\n", path.c_str());
        exit(1);
    }
    f >> m.natom;
    if (d == Dialect::LJ && m.natom > 84) {
        fprintf(stderr, "Error: natom=%d > MAX_NATOM=%d\n", m.natom, 84);
        exit(1);
    }
    m.coords.assign(3 * (size_t)std::max(m.natom, 0), 0.0);
    std::vector<std::vector<int>> adj(std::max(m.natom, 0));
    for (int i = 0; i < m.natom; i++) {
        std::string line;
        std::getline(f, line);
        while (line.empty() && f.good()) std::getline(f, line);
        std::istringstream ss(line);
        std::string el;
        int idx, fl;
        double x, y, z;
        ss >> el >> idx >> x >> y >> z >> fl;
        m.coords[3 * i] = x; m.coords[3 * i + 1] = y; m.coords[3 * i + 2] = z;
        int b;
        while (ss >> b) adj[i].push_back(b - 1);
    }
    double cm[3] = {0, 0, 0};
    for (int i = 0; i < m.natom; i++)
        for (int a = 0; a < 3; a++) cm[a] += m.coords[3 * i + a];
    for (int a = 0; a < 3; a++) cm[a] /= m.natom;
    for (int i = 0; i < m.natom; i++)
        for (int a = 0; a < 3; a++) m.coords[3 * i + a] -= cm[a];
    const double* c = m.coords.data();
    for (int i = 0; i < m.natom; i++) {
        const double r = std::sqrt(c[3 * i] * c[3 * i] + c[3 * i + 1] * c[3 * i + 1] + c[3 * i + 2] * c[3 * i + 2]);
        if (r > m.Rmol) m.Rmol = r;
        for (int j = i + 1; j < m.natom; j++) {
            const double dx = c[3 * i] - c[3 * j], dy = c[3 * i + 1] - c[3 * j + 1], dz = c[3 * i + 2] - c[3 * j + 2];
            const double dd = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (dd > m.Dmol) m.Dmol = dd;
        }
    }
    double Ixx = 0, Iyy = 0, Izz = 0;   // LJ:201-205
    for (int i = 0; i < m.natom; i++) {
        const double r2 = c[3 * i] * c[3 * i] + c[3 * i + 1] * c[3 * i + 1] + c[3 * i + 2] * c[3 * i + 2];
        Ixx += MC * (r2 - c[3 * i] * c[3 * i]);
        Iyy += MC * (r2 - c[3 * i + 1] * c[3 * i + 1]);
        Izz += MC * (r2 - c[3 * i + 2] * c[3 * i + 2]);
    }
    m.I0 = (Ixx + Iyy + Izz) / 3.0;
    m.Mmol = m.natom * MC;
    std::set<std::pair<int, int>> bset;
    for (int i = 0; i < m.natom; i++)
        for (int j : adj[i]) bset.insert({std::min(i, j), std::max(i, j)});
    m.bonds.assign(bset.begin(), bset.end());
    return m;
}

int make_crystal(const std::string& st, double a, int nc, double* pos, double* h) {
    int n = 0;
    for (int k = 0; k < 9; k++) h[k] = 0;
    if (st == "FCC") {
        const double bas[4][3] = {{0, 0, 0}, {.5 * a, .5 * a, 0}, {.5 * a, 0, .5 * a}, {0, .5 * a, .5 * a}};
        for (int x = 0; x < nc; x++)
            for (int y = 0; y < nc; y++)
                for (int z = 0; z < nc; z++)
                    for (int b = 0; b < 4; b++) {
                        pos[3 * n] = a * x + bas[b][0];
                        pos[3 * n + 1] = a * y + bas[b][1];
                        pos[3 * n + 2] = a * z + bas[b][2];
                        n++;
                    }
        h[0] = h[4] = h[8] = nc * a;
    } else if (st == "HCP") {
        const double c = a * std::sqrt(8.0 / 3.0);
        const double a1[3] = {a, 0, 0}, a2[3] = {a / 2, a * std::sqrt(3.0) / 2, 0}, a3[3] = {0, 0, c};
        const double bas[2][3] = {{0, 0, 0}, {1.0 / 3, 2.0 / 3, 0.5}};
        for (int x = 0; x < nc; x++)
            for (int y = 0; y < nc; y++)
                for (int z = 0; z < nc; z++)
                    for (int b = 0; b < 2; b++) {
                        const double fx = x + bas[b][0], fy = y + bas[b][1], fz = z + bas[b][2];
                        pos[3 * n] = fx * a1[0] + fy * a2[0] + fz * a3[0];
                        pos[3 * n + 1] = fx * a1[1] + fy * a2[1] + fz * a3[1];
                        pos[3 * n + 2] = fx * a1[2] + fy * a2[2] + fz * a3[2];
                        n++;
                    }
        h[0] = nc * a1[0]; h[3] = nc * a1[1]; h[1] = nc * a2[0]; h[4] = nc * a2[1]; h[8] = nc * a3[2];
    } else {
        const double bas[2][3] = {{0, 0, 0}, {.5 * a, .5 * a, .5 * a}};
        for (int x = 0; x < nc; x++)
            for (int y = 0; y < nc; y++)
                for (int z = 0; z < nc; z++)
                    for (int b = 0; b < 2; b++) {
                        pos[3 * n] = a * x + bas[b][0];
                        pos[3 * n + 1] = a * y + bas[b][1];
                        pos[3 * n + 2] = a * z + bas[b][2];
                        n++;
                    }
        h[0] = h[4] = h[8] = nc * a;
    }
    return n;
}

double default_a0(double dmax, const std::string& st, double s) {
    const double m = 1.4;
    double a0;
    if (st == "FCC") a0 = dmax * std::sqrt(2.0) * m;
    else if (st == "HCP") a0 = dmax * m;
    else a0 = dmax * 2.0 / std::sqrt(3.0) * m;
    return a0 * s;
}

void generate_c60(double* coords, double* I0, double* Mmol, double* Rmol) {
    // Cyclic permutations of (0, +-1, +-3phi), (+-2, +-(1+2phi), +-phi),
    // (+-1, +-(2+phi), +-2phi), centred and scaled by 0.72 (CORE:228-252).
    const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
    const int cyc[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
    double t[60][3] = {};
    int n = 0;
    const int sg[2] = {-1, 1};
    for (int p = 0; p < 3; p++)
        for (int s2 : sg)
            for (int s3 : sg) {
                t[n][cyc[p][1]] = s2;
                t[n][cyc[p][2]] = s3 * 3 * phi;
                n++;
            }
    for (int p = 0; p < 3; p++)
        for (int s1 : sg)
            for (int s2 : sg)
                for (int s3 : sg) {
                    t[n][cyc[p][0]] = s1 * 2;
                    t[n][cyc[p][1]] = s2 * (1 + 2 * phi);
                    t[n][cyc[p][2]] = s3 * phi;
                    n++;
                }
    for (int p = 0; p < 3; p++)
        for (int s1 : sg)
            for (int s2 : sg)
                for (int s3 : sg) {
                    t[n][cyc[p][0]] = s1;
                    t[n][cyc[p][1]] = s2 * (2 + phi);
                    t[n][cyc[p][2]] = s3 * 2 * phi;
                    n++;
                }
    double cm[3] = {0, 0, 0};
    for (int i = 0; i < 60; i++)
        for (int a = 0; a < 3; a++) cm[a] += t[i][a];
    for (int a = 0; a < 3; a++) cm[a] /= 60.0;
    for (int i = 0; i < 60; i++)
        for (int a = 0; a < 3; a++) t[i][a] = (t[i][a] - cm[a]) * 0.72;
    double rmax = 0, isum = 0;
    for (int i = 0; i < 60; i++) {
        const double r2 = t[i][0] * t[i][0] + t[i][1] * t[i][1] + t[i][2] * t[i][2];
        const double r = std::sqrt(r2);
        if (r > rmax) rmax = r;
        isum += MC * r2;
    }
    *I0 = isum * 2.0 / 3.0;
    *Mmol = 60 * MC;
    *Rmol = rmax;
    for (int i = 0; i < 60; i++)
        for (int a = 0; a < 3; a++) coords[3 * i + a] = t[i][a];
}

double mat_det9(const double* h) {
    return h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
           h[2] * (h[3] * h[7] - h[4] * h[6]);
}

void mat_inv9(const double* h, double* hi) {
    const double id = 1.0 / mat_det9(h);
    hi[0] = id * (h[4] * h[8] - h[5] * h[7]); hi[1] = id * (h[2] * h[7] - h[1] * h[8]);
    hi[2] = id * (h[1] * h[5] - h[2] * h[4]); hi[3] = id * (h[5] * h[6] - h[3] * h[8]);
    hi[4] = id * (h[0] * h[8] - h[2] * h[6]); hi[5] = id * (h[2] * h[3] - h[0] * h[5]);
    hi[6] = id * (h[3] * h[7] - h[4] * h[6]); hi[7] = id * (h[1] * h[6] - h[0] * h[7]);
    hi[8] = id * (h[0] * h[4] - h[1] * h[3]);
}

// ----------------------------------------------------------------- topology
namespace {
double dihedral0(const double* c, int i, int j, int k, int l) {   // MM:240-252
    const double b1x = c[3 * j] - c[3 * i], b1y = c[3 * j + 1] - c[3 * i + 1], b1z = c[3 * j + 2] - c[3 * i + 2];
    const double b2x = c[3 * k] - c[3 * j], b2y = c[3 * k + 1] - c[3 * j + 1], b2z = c[3 * k + 2] - c[3 * j + 2];
    const double b3x = c[3 * l] - c[3 * k], b3y = c[3 * l + 1] - c[3 * k + 1], b3z = c[3 * l + 2] - c[3 * k + 2];
    const double mx = b1y * b2z - b1z * b2y, my = b1z * b2x - b1x * b2z, mz = b1x * b2y - b1y * b2x;
    const double nx = b2y * b3z - b2z * b3y, ny = b2z * b3x - b2x * b3z, nz = b2x * b3y - b2y * b3x;
    const double mm = mx * mx + my * my + mz * mz, nn = nx * nx + ny * ny + nz * nz;
    if (mm < 1e-20 || nn < 1e-20) return 0;
    const double b2len = std::sqrt(b2x * b2x + b2y * b2y + b2z * b2z);
    double cp = (mx * nx + my * ny + mz * nz) / std::sqrt(mm * nn);
    cp = std::clamp(cp, -1.0, 1.0);
    const double sp = (mx * b3x + my * b3y + mz * b3z) * b2len / std::sqrt(mm * nn);
    return std::atan2(sp, cp);
}
}  // namespace

Topology build_flat_topology(const Molecule& mol, int nmol, double kb, double kth, double v2, double kimp) {
    const int na = mol.natom;
    const double* c = mol.coords.data();
    std::vector<std::vector<int>> adj(na);
    for (auto& b : mol.bonds) {
        adj[b.first].push_back(b.second);
        adj[b.second].push_back(b.first);
    }
    std::vector<std::array<int, 2>> bd;
    std::vector<double> br0;
    for (auto& b : mol.bonds) {
        const double dx = c[3 * b.first] - c[3 * b.second], dy = c[3 * b.first + 1] - c[3 * b.second + 1],
                     dz = c[3 * b.first + 2] - c[3 * b.second + 2];
        bd.push_back({b.first, b.second});
        br0.push_back(std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    std::vector<std::array<int, 3>> an;
    std::vector<double> ath;
    for (int j = 0; j < na; j++)
        for (size_t ii = 0; ii < adj[j].size(); ii++)
            for (size_t kk = ii + 1; kk < adj[j].size(); kk++) {
                const int i = adj[j][ii], k = adj[j][kk];
                double u[3], v[3];
                for (int a = 0; a < 3; a++) {
                    u[a] = c[3 * i + a] - c[3 * j + a];
                    v[a] = c[3 * k + a] - c[3 * j + a];
                }
                const double du = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
                const double dv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                const double ct = std::clamp((u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) / (du * dv), -1.0, 1.0);
                an.push_back({i, j, k});
                ath.push_back(std::acos(ct));
            }
    std::vector<std::array<int, 4>> dh;
    std::vector<double> dg;
    for (auto& b : mol.bonds) {
        const int bj = b.first, bk = b.second;
        for (int i : adj[bj]) {
            if (i == bk) continue;
            for (int l : adj[bk]) {
                if (l == bj || l == i) continue;
                dh.push_back({i, bj, bk, l});
                dg.push_back(2 * dihedral0(c, i, bj, bk, l) + PI);
            }
        }
    }
    std::vector<std::array<int, 4>> im;
    std::vector<double> ig;
    for (int i = 0; i < na; i++)
        if ((int)adj[i].size() == 3) {
            const int j = adj[i][0], k = adj[i][1], l = adj[i][2];
            im.push_back({i, j, k, l});
            ig.push_back(2 * dihedral0(c, j, i, k, l) + PI);
        }
    Topology t;
    t.nb_mol = (int)bd.size(); t.nang_mol = (int)an.size(); t.ndih_mol = (int)dh.size(); t.nimp_mol = (int)im.size();
    for (int m = 0; m < nmol; m++) {
        const int off = m * na;
        for (int a = 0; a < na; a++) t.mol_id.push_back(m);
        for (size_t q = 0; q < bd.size(); q++) {
            t.b_i0.push_back(bd[q][0] + off); t.b_i1.push_back(bd[q][1] + off);
            t.b_kb.push_back(kb); t.b_r0.push_back(br0[q]);
        }
        for (size_t q = 0; q < an.size(); q++) {
            t.a_i0.push_back(an[q][0] + off); t.a_i1.push_back(an[q][1] + off); t.a_i2.push_back(an[q][2] + off);
            t.a_kth.push_back(kth); t.a_th0.push_back(ath[q]);
        }
        for (size_t q = 0; q < dh.size(); q++) {
            t.d_i0.push_back(dh[q][0] + off); t.d_i1.push_back(dh[q][1] + off);
            t.d_i2.push_back(dh[q][2] + off); t.d_i3.push_back(dh[q][3] + off);
            t.d_vn.push_back(v2); t.d_mult.push_back(2); t.d_gamma.push_back(dg[q]);
        }
        for (size_t q = 0; q < im.size(); q++) {
            t.m_i0.push_back(im[q][0] + off); t.m_i1.push_back(im[q][1] + off);
            t.m_i2.push_back(im[q][2] + off); t.m_i3.push_back(im[q][3] + off);
            t.m_ki.push_back(kimp); t.m_gamma.push_back(ig[q]);
        }
    }
    printf("  Topology/mol: %d bonds, %d angles, %d dihedrals, %d impropers\n", t.nb_mol, t.nang_mol, t.ndih_mol,
           t.nimp_mol);
    printf("  Total:        %d bonds, %d angles, %d dihedrals, %d impropers\n", (int)t.b_i0.size(),
           (int)t.a_i0.size(), (int)t.d_i0.size(), (int)t.m_i0.size());
    return t;
}

fmd_mm_topology Topology::view() const {
    fmd_mm_topology v;
    v.nb = (int)b_i0.size(); v.b_i0 = b_i0.data(); v.b_i1 = b_i1.data(); v.b_kb = b_kb.data(); v.b_r0 = b_r0.data();
    v.nang = (int)a_i0.size(); v.ang_i0 = a_i0.data(); v.ang_i1 = a_i1.data(); v.ang_i2 = a_i2.data();
    v.ang_kth = a_kth.data(); v.ang_th0 = a_th0.data();
    v.ndih = (int)d_i0.size(); v.dih_i0 = d_i0.data(); v.dih_i1 = d_i1.data(); v.dih_i2 = d_i2.data();
    v.dih_i3 = d_i3.data(); v.dih_vn = d_vn.data(); v.dih_mult = d_mult.data(); v.dih_gamma = d_gamma.data();
    v.nimp = (int)m_i0.size(); v.imp_i0 = m_i0.data(); v.imp_i1 = m_i1.data(); v.imp_i2 = m_i2.data();
    v.imp_i3 = m_i3.data(); v.imp_ki = m_ki.data(); v.imp_gamma = m_gamma.data();
    return v;
}

// --------------------------------------------------------------------- OVITO

namespace {
// Lines of molecules [i0, i1) (rigid: natom sites each, lab frame R(q) body +
// centre) or atoms [i0, i1), in the reference's formats, appended to out.
void rigid_lines(std::string& out, const double* pos, const double* vel, const double* qv, const double* body,
                 int i0, int i1, int natom) {
    char ln[192];
    for (int i = i0; i < i1; i++) {
        const double* q = qv + 4 * i;
        const double w = q[0], x = q[1], y = q[2], z = q[3];
        const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                             2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                             2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)};
        for (int a = 0; a < natom; a++) {
            const double bx = body[3 * a], by = body[3 * a + 1], bz = body[3 * a + 2];
            const int k = snprintf(ln, sizeof(ln), "C %14.8f %14.8f %14.8f %5d %14.8e %14.8e %14.8e\n",
                                   pos[3 * i] + R[0] * bx + R[1] * by + R[2] * bz,
                                   pos[3 * i + 1] + R[3] * bx + R[4] * by + R[5] * bz,
                                   pos[3 * i + 2] + R[6] * bx + R[7] * by + R[8] * bz, i + 1, vel[3 * i],
                                   vel[3 * i + 1], vel[3 * i + 2]);
            out.append(ln, (size_t)std::min(k, (int)sizeof(ln) - 1));
        }
    }
}

void atom_lines(std::string& out, const double* pos, const double* vel, const int* mol_id, int mol_offset, int i0,
                int i1) {
    char ln[192];
    for (int i = i0; i < i1; i++) {
        const int k = snprintf(ln, sizeof(ln), "C %14.8f %14.8f %14.8f %5d %14.8e %14.8e %14.8e\n", pos[3 * i],
                               pos[3 * i + 1], pos[3 * i + 2], mol_id[i] + mol_offset, vel[3 * i], vel[3 * i + 1],
                               vel[3 * i + 2]);
        out.append(ln, (size_t)std::min(k, (int)sizeof(ln) - 1));
    }
}

std::string frame_head(int lines, const double* h, int istep, double dt) {
    char buf[512];
    std::string s = std::to_string(lines) + "\n";
    snprintf(buf, sizeof(buf),
             "Lattice=\"%.8f %.8f %.8f %.8f %.8f %.8f %.8f %.8f %.8f\" "
             "Properties=species:S:1:pos:R:3:c_mol:I:1:vx:R:1:vy:R:1:vz:R:1 Time=%.4f Step=%d pbc=\"T T T\"\n",
             h[0], h[3], h[6], h[1], h[4], h[7], h[2], h[5], h[8], istep * dt, istep);
    return s + buf;
}
}  // namespace

void write_ovito_rigid(FILE* fp, int istep, double dt, const double* pos, const double* vel, const double* qv,
                       const double* body, const double* h, int n, int natom) {
    std::string out = frame_head(n * natom, h, istep, dt);
    rigid_lines(out, pos, vel, qv, body, 0, n, natom);
    fwrite(out.data(), 1, out.size(), fp);
}

void write_ovito_atoms(FILE* fp, int istep, double dt, const double* pos, const double* vel, const int* mol_id,
                       int mol_offset, const double* h, int na) {
    std::string out = frame_head(na, h, istep, dt);
    atom_lines(out, pos, vel, mol_id, mol_offset, 0, na);
    fwrite(out.data(), 1, out.size(), fp);
}

struct OvitoWriter::Frame {
    bool rigid = false;
    int istep = 0, n = 0, natom = 1, mol_offset = 0;
    double dt = 0.0, h[9] = {};
    std::vector<double> pos, vel, qv, body;
    std::vector<int> mol_id;
};

OvitoWriter::OvitoWriter(FILE* fp, int threads) : fp_(fp) {
    const int hw = (int)std::thread::hardware_concurrency();
    threads_ = threads > 0 ? threads : std::max(1, std::min(hw, 16));
    th_ = std::thread([this] { loop(); });
}

OvitoWriter::~OvitoWriter() {
    finish();
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    th_.join();
}

void OvitoWriter::submit(std::unique_ptr<Frame> f) {
    std::unique_lock<std::mutex> g(mu_);
    cv_.wait(g, [this] { return inflight_ < kSlots; });
    queue_.push_back(std::move(f));
    inflight_++;
    cv_.notify_all();
}

void OvitoWriter::rigid(int istep, double dt, const double* pos, const double* vel, const double* qv,
                        const double* body, const double* h, int n, int natom) {
    auto f = std::make_unique<Frame>();
    f->rigid = true;
    f->istep = istep; f->dt = dt; f->n = n; f->natom = natom;
    std::copy(h, h + 9, f->h);
    f->pos.assign(pos, pos + 3 * (size_t)n);
    f->vel.assign(vel, vel + 3 * (size_t)n);
    f->qv.assign(qv, qv + 4 * (size_t)n);
    f->body.assign(body, body + 3 * (size_t)natom);
    submit(std::move(f));
}

void OvitoWriter::atoms(int istep, double dt, const double* pos, const double* vel, const int* mol_id,
                        int mol_offset, const double* h, int na) {
    auto f = std::make_unique<Frame>();
    f->istep = istep; f->dt = dt; f->n = na; f->mol_offset = mol_offset;
    std::copy(h, h + 9, f->h);
    f->pos.assign(pos, pos + 3 * (size_t)na);
    f->vel.assign(vel, vel + 3 * (size_t)na);
    f->mol_id.assign(mol_id, mol_id + na);
    submit(std::move(f));
}

void OvitoWriter::finish() {
    std::unique_lock<std::mutex> g(mu_);
    cv_.wait(g, [this] { return inflight_ == 0; });
}

void OvitoWriter::loop() {
    for (;;) {
        std::unique_ptr<Frame> f;
        {
            std::unique_lock<std::mutex> g(mu_);
            cv_.wait(g, [this] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;
            f = std::move(queue_.front());
            queue_.pop_front();
        }
        write(*f);
        {
            std::lock_guard<std::mutex> g(mu_);
            inflight_--;
        }
        cv_.notify_all();
    }
}

// Formats the frame in up to threads_ contiguous chunks (at least kChunk
// lines each) on worker threads, then writes them in order and flushes, so
// the file only ever grows by whole frames.
void OvitoWriter::write(const Frame& f) {
    constexpr int kChunk = 4096;
    const int per = f.rigid ? f.natom : 1;                       // lines per unit
    const int units = f.n;
    int parts = std::min(threads_, std::max(1, (units * per) / kChunk));
    parts = std::max(1, std::min(parts, units));
    std::vector<std::string> out((size_t)parts);
    auto work = [&](int p) {
        const int i0 = (int)((long long)units * p / parts), i1 = (int)((long long)units * (p + 1) / parts);
        out[p].reserve((size_t)(i1 - i0) * per * 100);
        if (f.rigid) rigid_lines(out[p], f.pos.data(), f.vel.data(), f.qv.data(), f.body.data(), i0, i1, f.natom);
        else atom_lines(out[p], f.pos.data(), f.vel.data(), f.mol_id.data(), f.mol_offset, i0, i1);
    };
    std::vector<std::thread> pool;
    for (int p = 1; p < parts; p++) pool.emplace_back(work, p);
    work(0);
    for (auto& t : pool) t.join();
    const std::string head = frame_head(units * per, f.h, f.istep, f.dt);
    fwrite(head.data(), 1, head.size(), fp_);
    for (auto& o : out) fwrite(o.data(), 1, o.size(), fp_);
    fflush(fp_);
}

// ------------------------------------------------------------------ restart
RestartWriter::RestartWriter() { th_ = std::thread([this] { loop(); }); }

RestartWriter::~RestartWriter() {
    finish();
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    th_.join();
}

void RestartWriter::submit(std::function<void()> job) {
    std::unique_lock<std::mutex> g(mu_);
    cv_.wait(g, [this] { return inflight_ < kSlots; });
    queue_.push_back(std::move(job));
    inflight_++;
    cv_.notify_all();
}

void RestartWriter::finish() {
    std::unique_lock<std::mutex> g(mu_);
    cv_.wait(g, [this] { return inflight_ == 0; });
}

void RestartWriter::loop() {
    for (;;) {
        std::function<void()> job;
        {
            std::unique_lock<std::mutex> g(mu_);
            cv_.wait(g, [this] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;
            job = std::move(queue_.front());
            queue_.pop_front();
        }
        job();
        {
            std::lock_guard<std::mutex> g(mu_);
            inflight_--;
        }
        cv_.notify_all();
    }
}

namespace {
void header(FILE* f, const char* prog, const Opts& o, const RunInfo& r, int istep) {
    fprintf(f, "# RESTART %s\n# OPTIONS:", prog);
    for (auto& kv : o) fprintf(f, " --%s=%s", kv.first.c_str(), kv.second.c_str());
    fprintf(f, "\nSTEP %d\nNSTEPS %d\nDT %.15e\nTEMP %.15e\nPRES %.15e\n", istep, r.nsteps, r.dt, r.T, r.Pe);
    fprintf(f, "CRYSTAL %s\nNC %d\nFULLERENE %s\nINIT_SCALE %.15e\nSEED %d\n", r.st.c_str(), r.nc, r.fspec.c_str(),
            r.init_scale, r.seed);
}
void cell_npt(FILE* f, const double* h, const fmd_npt& npt) {
    fprintf(f, "H");
    for (int k = 0; k < 9; k++) fprintf(f, " %.15e", h[k]);
    fprintf(f, "\nNPT %.15e %.15e %.15e %.15e %.15e %d\n", npt.xi, npt.Q, npt.W, npt.Pe, npt.Tt, npt.Nf);
    fprintf(f, "VG");
    for (int k = 0; k < 9; k++) fprintf(f, " %.15e", npt.Vg[k]);
    fprintf(f, "\n");
}
}  // namespace

void write_restart_lj(const std::string& fn, int istep, const Opts& o, const RunInfo& r, const double* h,
                      const fmd_npt& npt, const double* pos, const double* qv, const double* vel, const double* omg,
                      int n, int natom) {
    FILE* f = fopen(fn.c_str(), "w");
    if (!f) return;                                      // LJ:595: silent
    header(f, "fuller_LJ_npt_md_serial_omp_acc", o, r, istep);
    fprintf(f, "NMOL %d\nNATOM_MOL %d\n", n, natom);
    cell_npt(f, h, npt);
    for (int i = 0; i < n; i++)
        fprintf(f, "MOL %d %.15e %.15e %.15e %.15e %.15e %.15e %.15e %.15e %.15e %.15e %.15e %.15e %.15e\n", i + 1,
                pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], qv[4 * i], qv[4 * i + 1], qv[4 * i + 2], qv[4 * i + 3],
                vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], omg[3 * i], omg[3 * i + 1], omg[3 * i + 2]);
    fprintf(f, "END\n");
    fclose(f);
}

void write_restart_airebo(const std::string& fn, int istep, const Opts& o, const RunInfo& r, const double* h,
                          const fmd_npt& npt, const double* pos, const double* vel, const int* mol_id,
                          const double* mass, int na, int nmol, int natom_mol) {
    FILE* f = fopen(fn.c_str(), "w");
    if (!f) {
        fprintf(stderr, "Cannot write restart: %s\n", fn.c_str());
        return;
    }
    header(f, "fuller_airebo_npt_md_serial_omp_acc", o, r, istep);
    fprintf(f, "NMOL %d\nNATOM_MOL %d\nNATOM %d\n", nmol, natom_mol, na);
    cell_npt(f, h, npt);
    for (int i = 0; i < na; i++) {
        fprintf(f, "ATOM %d %d %.15e", i + 1, mol_id[i], mass[i]);
        fprintf(f, " %.15e %.15e %.15e", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        fprintf(f, " %.15e %.15e %.15e\n", vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    fprintf(f, "END\n");
    fclose(f);
}

void write_restart_mmmd(const std::string& fn, int istep, const Opts& o, const RunInfo& r, const double* h,
                        const fmd_npt& npt, const double* pos, const double* vel, int na, int nmol, int natom) {
    FILE* f = fopen(fn.c_str(), "w");
    if (!f) {
        fprintf(stderr, "Cannot write restart: %s\n", fn.c_str());
        return;
    }
    header(f, "fuller_LJ_npt_mmmd_serial_omp_acc", o, r, istep);
    fprintf(f, "NMOL %d\nNATOM_MOL %d\nNATOM %d\n", nmol, natom, na);
    cell_npt(f, h, npt);
    for (int i = 0; i < na; i++)
        fprintf(f, "ATOM %d %.15e %.15e %.15e %.15e %.15e %.15e\n", i + 1, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2],
                vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    fprintf(f, "END\n");
    fclose(f);
}

namespace {
// Shared tag parser; `row` handles the per-particle tag.
template <class RowFn>
bool read_tags(const std::string& fn, Restart& rd, const char* row_tag, RowFn row) {
    std::ifstream f(fn);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream ss(line);
        std::string tag;
        ss >> tag;
        if (tag == "STEP") ss >> rd.istep;
        else if (tag == "H") for (int k = 0; k < 9; k++) ss >> rd.h[k];
        else if (tag == "NPT") ss >> rd.npt.xi >> rd.npt.Q >> rd.npt.W >> rd.npt.Pe >> rd.npt.Tt >> rd.npt.Nf;
        else if (tag == "VG") for (int k = 0; k < 9; k++) ss >> rd.npt.Vg[k];
        else if (tag == row_tag) row(ss);
        else if (tag == "END") break;
    }
    return true;
}
}  // namespace

Restart read_restart_lj(const std::string& fn) {
    Restart rd;
    if (!read_tags(fn, rd, "MOL", [&](std::istringstream& ss) {
            int idx;
            double v[13];
            ss >> idx;
            for (double& x : v) ss >> x;
            for (int k = 0; k < 3; k++) rd.pos.push_back(v[k]);
            for (int k = 3; k < 7; k++) rd.qv.push_back(v[k]);
            for (int k = 7; k < 10; k++) rd.vel.push_back(v[k]);
            for (int k = 10; k < 13; k++) rd.omg.push_back(v[k]);
        }))
        return rd;                                       // LJ:614: silent
    rd.n = (int)rd.pos.size() / 3;
    rd.ok = rd.n > 0;
    if (rd.ok) printf("  Restart loaded: %s (step %d, %d mols)\n", fn.c_str(), rd.istep, rd.n);
    return rd;
}

Restart read_restart_airebo(const std::string& fn) {
    Restart rd;
    if (!read_tags(fn, rd, "ATOM", [&](std::istringstream& ss) {
            int idx, mid;
            double m, p[3], v[3];
            ss >> idx >> mid >> m >> p[0] >> p[1] >> p[2] >> v[0] >> v[1] >> v[2];
            for (int k = 0; k < 3; k++) { rd.pos.push_back(p[k]); rd.vel.push_back(v[k]); }
            rd.mol_id.push_back(mid);
            rd.mass.push_back(m);
        })) {
        fprintf(stderr, "Cannot read: %s\n", fn.c_str());
        return rd;
    }
    rd.n = (int)rd.pos.size() / 3;
    rd.ok = rd.n > 0;
    if (rd.ok) printf("  Restart loaded: %s (step %d, %d atoms)\n", fn.c_str(), rd.istep, rd.n);
    return rd;
}

Restart read_restart_mmmd(const std::string& fn) {
    Restart rd;
    if (!read_tags(fn, rd, "ATOM", [&](std::istringstream& ss) {
            int idx;
            double p[3], v[3];
            ss >> idx >> p[0] >> p[1] >> p[2] >> v[0] >> v[1] >> v[2];
            for (int k = 0; k < 3; k++) { rd.pos.push_back(p[k]); rd.vel.push_back(v[k]); }
        })) {
        fprintf(stderr, "Cannot read: %s\n", fn.c_str());
        return rd;
    }
    rd.n = (int)rd.pos.size() / 3;
    rd.ok = rd.n > 0;
    if (rd.ok) printf("  Restart loaded: %s (step %d, %d atoms)\n", fn.c_str(), rd.istep, rd.n);
    return rd;
}

fmd_npt make_npt(double T, double Pe, int nf) {
    fmd_npt s;
    s.xi = 0;
    s.Q = std::max(nf * KB * T * 100.0 * 100.0, 1e-20);
    for (int k = 0; k < 9; k++) s.Vg[k] = 0;
    s.W = std::max((nf + 9) * KB * T * 1000.0 * 1000.0, 1e-20);
    s.Pe = Pe;
    s.Tt = T;
    s.Nf = nf;
    return s;
}

fmd_npt make_npt_mm(double T, double Pe, int nf) {
    fmd_npt s = make_npt(T, Pe, nf);
    s.Q = std::max(nf * KB * T * 1e4, 1e-20);
    s.W = std::max((nf + 9) * KB * T * 1e6, 1e-20);
    return s;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
double elapsed_since(double t0) { return now_s() - t0; }

}  // namespace fmdh
