// The reference's input readers, for hosts that do not bring their own:
// .composition + .mol (composition.f90:84-142, Molecule.f90:142-209), the
// binary moltab (MoleculeTable.f90:240-319) and MoleculeTable_fillAtomicData
// (MoleculeTable.f90:584-705).  Molecule files are resolved relative to the
// composition file's directory.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "yamc_internal.h"

using namespace yamc;

struct yamc_inputs {
    yamc_params p{};
    std::vector<double> x, y, z, q, sigma, eps, hc, mass;
    std::vector<int32_t> first, last, mol_numbers;
};

namespace {

struct MolType {
    std::vector<double> x, y, z, sigma, eps, q, mass, hc;
};

// Molecule_read_from_file (Molecule.f90:142-188) and Molecule_centrate (:190-209)
int read_mol(const std::string &path, MolType *m) {
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) { set_error("cannot open " + path); return YAMC_EIO; }
    char line[2048];
    while (std::fgets(line, sizeof line, f)) {
        char name[64];
        double v[8];
        int k = std::sscanf(line, "%63s %lf %lf %lf %lf %lf %lf %lf %lf", name, v, v + 1, v + 2, v + 3, v + 4, v + 5, v + 6, v + 7);
        if (k <= 0) continue;
        if (k < 9) { std::fclose(f); set_error("malformed .mol line in " + path); return YAMC_EIO; }
        m->x.push_back(v[0]); m->y.push_back(v[1]); m->z.push_back(v[2]);
        m->sigma.push_back(v[3]); m->eps.push_back(v[4]); m->q.push_back(v[5]); m->mass.push_back(v[6]);
        double hc = v[7];
        if (hc < (double)1e-9f) hc = v[3] * (double)std::sqrt(0.4f);  // single-precision sqrt(0.4)
        m->hc.push_back(hc);
    }
    std::fclose(f);
    const size_t n = m->x.size();
    if (n == 0) { set_error("empty .mol file " + path); return YAMC_EIO; }
    double sx = 0, sy = 0, sz = 0, tm = 0;  // center_of_mass (geometry.f90:170-201)
    for (size_t i = 0; i < n; ++i) { sx = sx + m->mass[i] * m->x[i]; sy = sy + m->mass[i] * m->y[i]; sz = sz + m->mass[i] * m->z[i]; tm = tm + m->mass[i]; }
    const double xc = sx / tm, yc = sy / tm, zc = sz / tm;
    for (size_t i = 0; i < n; ++i) { m->x[i] = m->x[i] - xc; m->y[i] = m->y[i] - yc; m->z[i] = m->z[i] - zc; }
    return YAMC_OK;
}

// rot_vect about axis 3 (z) or 2 (y) (geometry.f90:28-63)
inline void rot_z(double &x, double &y, double c, double s) { const double x2 = x; x = c * x2 - s * y; y = s * x2 + c * y; }
inline void rot_y(double &x, double &z, double c, double s) { const double x2 = x; x = c * x2 + s * z; z = -s * x2 + c * z; }

}  // namespace

extern "C" int yamc_inputs_load(const char *prm, const char *comp, const char *moltab, const char *extra, yamc_inputs **out) {
    if (!out || !comp || !moltab) return YAMC_EPARAMETER;
    *out = nullptr;
    auto *in = new yamc_inputs();
    int r = yamc_params_read(prm, extra, &in->p);
    if (r) { delete in; return r; }
    std::string dir(comp);
    size_t sl = dir.rfind('/');
    dir = sl == std::string::npos ? std::string() : dir.substr(0, sl + 1);
    FILE *f = std::fopen(comp, "r");
    if (!f) { set_error(std::string("cannot open ") + comp); delete in; return YAMC_EIO; }
    int ntypes = 0;
    std::vector<MolType> types;
    if (std::fscanf(f, "%d", &ntypes) != 1 || ntypes < 1) { std::fclose(f); set_error("bad composition header"); delete in; return YAMC_EIO; }
    for (int t = 0; t < ntypes; ++t) {
        char name[1024];
        int cnt = 0;
        if (std::fscanf(f, "%1023s %d", name, &cnt) != 2 || cnt < 0) { std::fclose(f); set_error("bad composition line"); delete in; return YAMC_EIO; }
        MolType m;
        std::string path = name[0] == '/' ? std::string(name) : dir + name;
        if ((r = read_mol(path, &m))) { std::fclose(f); delete in; return r; }
        types.push_back(std::move(m));
        in->mol_numbers.push_back(cnt);
    }
    std::fclose(f);
    int nmol = 0;
    for (int c : in->mol_numbers) nmol += c;
    if ((r = yamc_params_init(&in->p, nmol))) { delete in; return r; }
    const yamc_params &p = in->p;

    // MoleculeTable_load_binary (MoleculeTable.f90:240-319)
    FILE *g = std::fopen(moltab, "rb");
    if (!g) { set_error(std::string("cannot open ") + moltab); delete in; return YAMC_EIO; }
    double pxyz = 1, pang = 1;
    for (int i = 0; i < p.input_nbytes_xyz; ++i) pxyz = pxyz * 256;
    for (int i = 0; i < p.input_nbytes_ang; ++i) pang = pang * 256;
    auto rd = [&](int nb, int *v) -> bool {
        int val = 0, pw = 1;
        for (int b = 0; b < nb; ++b) {
            int c = std::fgetc(g);
            if (c == EOF) return false;
            val = val + c * pw;
            pw = pw * 256;
        }
        *v = val;
        return true;
    };
    std::vector<int> mtype;
    for (int t = 0; t < ntypes; ++t) for (int i = 0; i < in->mol_numbers[t]; ++i) mtype.push_back(t);
    int natom = 0;
    for (int m = 0; m < nmol; ++m) {
        int xi, yi, zi, it, ip, is;
        if (!rd(p.input_nbytes_xyz, &xi) || !rd(p.input_nbytes_xyz, &yi) || !rd(p.input_nbytes_xyz, &zi) ||
            !rd(p.input_nbytes_ang, &it) || !rd(p.input_nbytes_ang, &ip) || !rd(p.input_nbytes_ang, &is)) {
            std::fclose(g); set_error("moltab shorter than the composition"); delete in; return YAMC_EIO;
        }
        const double cx = xi / pxyz - 0.5, cy = yi / pxyz - 0.5, cz = zi / pxyz - 0.5;
        const double th = it / pang * kTwoPi, ph = ip / pang * kTwoPi, ps = is / pang * kTwoPi;
        // MoleculeTable_fillAtomicData: rotate by psi about z, theta about y, phi about z
        const double ct = std::cos(th), st = std::sin(th), cp = std::cos(ph), sp = std::sin(ph);
        const double cs = std::cos(ps), ss = std::sin(ps);
        const MolType &M = types[mtype[m]];
        in->first.push_back(natom + 1);
        for (size_t a = 0; a < M.x.size(); ++a) {
            double x = M.x[a], y = M.y[a], z = M.z[a];
            rot_z(x, y, cs, ss);
            rot_y(x, z, ct, st);
            rot_z(x, y, cp, sp);
            in->x.push_back(x / p.BoxLength + cx);
            in->y.push_back(y / p.BoxLength + cy);
            in->z.push_back(z / p.BoxLength + cz);
            in->q.push_back(M.q[a]);
            in->sigma.push_back(M.sigma[a] / p.BoxLength);
            in->hc.push_back(M.hc[a]);
            in->eps.push_back(M.eps[a] / p.kT_kcal_mol);
            in->mass.push_back(M.mass[a]);
            ++natom;
        }
        in->last.push_back(natom);
    }
    std::fclose(g);
    *out = in;
    return YAMC_OK;
}

extern "C" int yamc_inputs_get(const yamc_inputs *in, yamc_system *sys, yamc_params *p) {
    if (!in || !sys) return YAMC_EPARAMETER;
    std::memset(sys, 0, sizeof(*sys));
    sys->natom = (int32_t)in->x.size();
    sys->nmol = (int32_t)in->first.size();
    sys->x = in->x.data(); sys->y = in->y.data(); sys->z = in->z.data();
    sys->charge = in->q.data(); sys->sigma = in->sigma.data(); sys->epsilon = in->eps.data();
    sys->hard_core_angstr = in->hc.data(); sys->mass = in->mass.data();
    sys->first_atom = in->first.data(); sys->last_atom = in->last.data();
    sys->n_species = (int32_t)in->mol_numbers.size();
    sys->mol_numbers = in->mol_numbers.data();
    sys->move_weights = nullptr;
    if (p) *p = in->p;
    return YAMC_OK;
}

extern "C" int yamc_inputs_free(yamc_inputs *in) {
    delete in;
    return YAMC_OK;
}
