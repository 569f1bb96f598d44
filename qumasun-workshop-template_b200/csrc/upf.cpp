// UPF (v2, ONCV norm-conserving) pseudopotentials: the nonlocal and local
// radial data the reference reads with LoadUPF_ONCV
// (source/upf_oncv_loader.h:353-520), and grid projector tables built from them
// for qsb_ham (host code).
//
// Radial data, as the reference holds it (PseudoPot_MBK, source/pp_struct.h):
//   * a log grid r_i = exp(xi_min + i xi_delta), i < 1000, xi_min = -9,
//     xi_delta = (ln r_last - xi_min) / 1000, r_last the UPF mesh's last point;
//   * per radial projector k: l_k, E_k = D_kk / 2 (Ry -> Ha), and
//     beta_k(r) = (r beta_k)(r) / r from the UPF's uniform mesh (its first
//     point replaced by the second for l = 0 and by 0 otherwise), resampled on
//     the log grid; cutoff_r[l] = the largest cutoff_radius of channel l;
//   * V_local(r): the UPF's local potential with its tail blended into
//     -2 Z_v / r beyond the local cutoff (the reference's correction of it),
//     resampled the same way, / 2 (Ry -> Ha); the cutoff it reports is the
//     corrected one.
// Resampling is the reference's uniform-grid interpolant (UniformGrid::GetValue,
// source/UniformGrid.h:38-89): on each mesh interval a quintic Hermite
// polynomial matching values, first and second derivatives at both ends, the
// derivatives from 4th-order central differences, the mesh continued to
// negative indices by parity (even for l even, odd for l odd) and by zero past
// its end.
//
// Grid tables (this library's own construction; the reference's SvF2 builder,
// source/PseudoPotNonlocal_SvF2_kpoint.h:911-1180, filters the projectors
// through FFTW on a supersampled subgrid, which its CPU build here cannot
// compile): every grid point within max_l cutoff_r[l] of the atom (periodic
// images unfolded) gets beta_k(|r - R|) Y_lm(r - R) with real spherical
// harmonics, m = -l..l, and the analytic gradient tables d/dx_d for forces.
// beta_k between log-grid points uses the same quintic in xi = ln r.
// An atom with more than 16 projectors (s2 p2 d2 = 18) is split into table
// entries of at most 16 at the same position -- V_NL is a sum over entries,
// so H psi is unchanged; entry_atom maps entries back to atoms (per-entry
// nonlocal forces add up to the atom's).
#include "../../include/qumasun_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace qsb {
qsb_status fail(qsb_status st, const std::string& msg);
}

struct qsb_upf {
    double z_valence = 0.0;
    int n_proj = 0;
    std::vector<int> l;
    std::vector<double> energy;      // Ha
    double cutoff_l[4] = {0, 0, 0, 0};
    double cutoff_vlocal = 0.0;
    double xi_min = -9.0, xi_delta = 0.0;
    int n_grid = 1000;
    std::vector<double> radius, v_local, proj;   // proj: n_proj x n_grid
};

namespace qsb {
namespace {

// ---- minimal UPF v2 (XML) access ------------------------------------------------
struct Span {
    size_t open = std::string::npos;   // '<' of the start tag
    size_t attr_end = 0;               // '>' of the start tag
    size_t end = 0;                    // one past the element (or its start tag when self-closing)
    bool ok() const { return open != std::string::npos; }
};

// first element named `name` inside [from, to)
Span find_element(const std::string& s, const std::string& name, size_t from, size_t to) {
    Span sp;
    size_t at = from;
    while (true) {
        at = s.find("<" + name, at);
        if (at == std::string::npos || at >= to) return sp;
        const char c = s[at + 1 + name.size()];
        if (c == ' ' || c == '>' || c == '\n' || c == '\r' || c == '\t' || c == '/') break;
        at += 1;
    }
    const size_t gt = s.find('>', at);
    if (gt == std::string::npos) return sp;
    sp.open = at;
    sp.attr_end = gt;
    if (s[gt - 1] == '/') {
        sp.end = gt + 1;
        return sp;
    }
    const size_t close = s.find("</" + name + ">", gt);
    sp.end = close == std::string::npos ? to : close;
    return sp;
}

Span find_path(const std::string& s, std::initializer_list<const char*> path) {
    size_t from = 0, to = s.size();
    Span sp;
    for (const char* n : path) {
        sp = find_element(s, n, from, to);
        if (!sp.ok()) return sp;
        from = sp.attr_end + 1;
        to = sp.end;
    }
    return sp;
}

bool attribute(const std::string& s, const Span& sp, const std::string& key, std::string& out) {
    size_t at = sp.open;
    while (true) {
        at = s.find(key, at);
        if (at == std::string::npos || at > sp.attr_end) return false;
        const char before = s[at - 1];
        size_t p = at + key.size();
        while (p < sp.attr_end && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\r')) ++p;
        if ((before == ' ' || before == '\n' || before == '\t' || before == '\r') && s[p] == '=') {
            const size_t q0 = s.find('"', p);
            const size_t q1 = q0 == std::string::npos ? q0 : s.find('"', q0 + 1);
            if (q1 == std::string::npos || q1 > sp.attr_end) return false;
            out = s.substr(q0 + 1, q1 - q0 - 1);
            return true;
        }
        at += key.size();
    }
}

// `count` numbers from the element's text; missing ones are 0 (as ReadDoubleList)
std::vector<double> numbers(const std::string& s, const Span& sp, int count) {
    std::vector<double> v(count > 0 ? count : 0, 0.0);
    const std::string text = s.substr(sp.attr_end + 1, sp.end - sp.attr_end - 1);
    const char* p = text.c_str();
    for (int i = 0; i < count; ++i) {
        char* e = nullptr;
        v[i] = std::strtod(p, &e);
        if (e == p) break;
        p = e;
    }
    return v;
}

// ---- the reference's uniform-grid interpolant, restated ------------------------
// value (and d/dxi) at xi of samples f on xi_0 + i h; parity continues f to i < 0
struct Quintic {
    const double* f;
    int n;
    double x0, h;
    int parity;   // +1 even, -1 odd, 0 zero
    double at(int i) const { return i < 0 ? f[-i] * (double)parity : (i >= n ? 0.0 : f[i]); }
    void eval(double xi, double& v, double* dv) const {
        const double t = (xi - x0) / h;
        const int i = (int)std::floor(t);
        const double x = t - (double)i;
        const double fm2 = at(i - 2), fm1 = at(i - 1), f0 = at(i), f1 = at(i + 1), f2 = at(i + 2), f3 = at(i + 3);
        // 4th-order central first and second differences at both ends (per unit step)
        const double a1 = (2.0 / 3.0) * (f1 - fm1) - (1.0 / 12.0) * (f2 - fm2);
        const double b1 = (2.0 / 3.0) * (f2 - f0) - (1.0 / 12.0) * (f3 - fm1);
        const double a2 = (4.0 / 3.0) * (f1 + fm1) - (1.0 / 12.0) * (f2 + fm2) - 2.5 * f0;
        const double b2 = (4.0 / 3.0) * (f2 + f0) - (1.0 / 12.0) * (f3 + fm1) - 2.5 * f1;
        // p(x) = f0 + a1 x + a2/2 x^2 + c3 x^3 + c4 x^4 + c5 x^5 with p, p', p'' matching at x = 1
        const double r0 = f1 - (f0 + a1 + 0.5 * a2);
        const double r1 = b1 - (a1 + a2);
        const double r2 = b2 - a2;
        const double c3 = 10.0 * r0 - 4.0 * r1 + 0.5 * r2;
        const double c4 = -15.0 * r0 + 7.0 * r1 - r2;
        const double c5 = f1 - f0 - a1 - 0.5 * a2 - c3 - c4;   // summed in the reference's order
        v = f0 + x * (a1 + x * (0.5 * a2 + x * (c3 + x * (c4 + x * c5))));
        if (dv) *dv = (a1 + x * (a2 + x * (3.0 * c3 + x * (4.0 * c4 + x * 5.0 * c5)))) / h;
    }
};

// ---- real spherical harmonics, l <= 3, with gradients (dual numbers) ------------
struct D {   // value and d/dx, d/dy, d/dz
    double v, d[3];
};
D mul(const D& a, const D& b) {
    return D{a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
D add(const D& a, const D& b) { return D{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}}; }
D scale(const D& a, double s) { return D{a.v * s, {a.d[0] * s, a.d[1] * s, a.d[2] * s}}; }

// homogeneous polynomial P_lm(x, y, z) with Y_lm = P_lm / r^l, m = -l..l
D poly(int l, int m, double x, double y, double z) {
    const double pi = 3.14159265358979323846;
    const D X{x, {1, 0, 0}}, Y{y, {0, 1, 0}}, Z{z, {0, 0, 1}};
    const D R2 = add(add(mul(X, X), mul(Y, Y)), mul(Z, Z));
    switch (l) {
    case 0: return D{0.5 / std::sqrt(pi), {0, 0, 0}};
    case 1: {
        const double c = std::sqrt(3.0 / (4.0 * pi));
        return scale(m == -1 ? Y : (m == 0 ? Z : X), c);
    }
    case 2: {
        const double c = 0.5 * std::sqrt(15.0 / pi);
        if (m == -2) return scale(mul(X, Y), c);
        if (m == -1) return scale(mul(Y, Z), c);
        if (m == 0) return scale(add(scale(mul(Z, Z), 3.0), scale(R2, -1.0)), 0.25 * std::sqrt(5.0 / pi));
        if (m == 1) return scale(mul(X, Z), c);
        return scale(add(mul(X, X), scale(mul(Y, Y), -1.0)), 0.25 * std::sqrt(15.0 / pi));
    }
    default: {
        const D X2 = mul(X, X), Y2 = mul(Y, Y), Z2 = mul(Z, Z);
        const D five_z2_r2 = add(scale(Z2, 5.0), scale(R2, -1.0));
        if (m == -3) return scale(mul(Y, add(scale(X2, 3.0), scale(Y2, -1.0))), 0.25 * std::sqrt(35.0 / (2.0 * pi)));
        if (m == -2) return scale(mul(mul(X, Y), Z), 0.5 * std::sqrt(105.0 / pi));
        if (m == -1) return scale(mul(Y, five_z2_r2), 0.25 * std::sqrt(21.0 / (2.0 * pi)));
        if (m == 0) return scale(mul(Z, add(scale(Z2, 5.0), scale(R2, -3.0))), 0.25 * std::sqrt(7.0 / pi));
        if (m == 1) return scale(mul(X, five_z2_r2), 0.25 * std::sqrt(21.0 / (2.0 * pi)));
        if (m == 2) return scale(mul(Z, add(X2, scale(Y2, -1.0))), 0.25 * std::sqrt(105.0 / pi));
        return scale(mul(X, add(X2, scale(Y2, -3.0))), 0.25 * std::sqrt(35.0 / (2.0 * pi)));
    }
    }
}

}  // namespace
}  // namespace qsb

using namespace qsb;

extern "C" {

qsb_status qsb_upf_load(qsb_upf** out, const char* path) {
    if (!out || !path) return fail(QSB_ERR_INVALID, "upf_load: bad argument");
    *out = nullptr;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(QSB_ERR_INVALID, std::string("upf_load: cannot open ") + path);
    std::string s;
    char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, fp)) > 0) s.append(buf, n);
    std::fclose(fp);
    auto* u = new qsb_upf;
    auto bad = [&](const std::string& what) {
        delete u;
        return fail(QSB_ERR_INVALID, "upf_load: " + what + " in " + path);
    };
    std::string a;
    const Span hdr = find_path(s, {"UPF", "PP_HEADER"});
    if (!hdr.ok() || !attribute(s, hdr, "number_of_proj", a)) return bad("no PP_HEADER number_of_proj");
    u->n_proj = std::atoi(a.c_str());
    if (!attribute(s, hdr, "z_valence", a)) return bad("no z_valence");
    u->z_valence = std::strtod(a.c_str(), nullptr);
    const std::string a_zval = a;
    const Span r = find_path(s, {"UPF", "PP_MESH", "PP_R"});
    if (!r.ok() || !attribute(s, r, "size", a)) return bad("no PP_MESH/PP_R size");
    const int nu = std::atoi(a.c_str());
    if (nu < 8 || u->n_proj < 0) return bad("mesh too small or bad projector count");
    const std::vector<double> mesh = numbers(s, r, nu);
    const double h = mesh[1] - mesh[0];
    if (!(h > 0)) return bad("PP_R is not an increasing uniform mesh");
    // log grid
    const double xi_max = std::log(mesh[nu - 1]);
    u->xi_delta = (xi_max - u->xi_min) / (double)u->n_grid;
    u->radius.resize(u->n_grid);
    for (int i = 0; i < u->n_grid; ++i) u->radius[i] = std::exp((double)i * u->xi_delta + u->xi_min);
    // channels and cutoffs
    u->l.resize(u->n_proj);
    for (int k = 0; k < u->n_proj; ++k) {
        const std::string name = "PP_BETA." + std::to_string(k + 1);
        const Span b = find_path(s, {"UPF", "PP_NONLOCAL", name.c_str()});
        if (!b.ok() || !attribute(s, b, "angular_momentum", a)) return bad("no " + name + " angular_momentum");
        u->l[k] = std::atoi(a.c_str());
        if (u->l[k] < 0 || u->l[k] > 3) return bad(name + ": l > 3 is not supported");
        if (!attribute(s, b, "cutoff_radius", a)) return bad("no " + name + " cutoff_radius");
        const double rc = std::strtod(a.c_str(), nullptr);
        if (u->cutoff_l[u->l[k]] < rc) u->cutoff_l[u->l[k]] = rc;
        u->cutoff_vlocal = std::max(u->cutoff_vlocal, rc);
    }
    // KB energies: the diagonal of D_ij (Ry -> Ha)
    u->energy.resize(u->n_proj);
    if (u->n_proj > 0) {
        const Span dij = find_path(s, {"UPF", "PP_NONLOCAL", "PP_DIJ"});
        if (!dij.ok()) return bad("no PP_DIJ");
        const std::vector<double> d = numbers(s, dij, u->n_proj * u->n_proj);
        for (int k = 0; k < u->n_proj; ++k) u->energy[k] = d[k + u->n_proj * k] / 2.0;
    }
    // local potential (Ry), tail-corrected to -2 Z_v / r as the reference does
    // (ONCV_CORRECT_VLOCAL 11, source/upf_oncv_loader.h:803-921), then Ry -> Ha
    const Span loc = find_path(s, {"UPF", "PP_LOCAL"});
    if (!loc.ok()) return bad("no PP_LOCAL");
    const std::vector<double> vl = numbers(s, loc, nu);
    {
        // the reference keeps the valence as an integer (std::stol of the attribute)
        const double zv = (double)std::strtol(a_zval.c_str(), nullptr, 10);
        // nuclear-charge density of the UPF's V_local: -(1 / 8 pi) (v'' + 2 v' / r),
        // 4th-order differences on the uniform mesh
        std::vector<double> rho(nu, 0.0);
        for (int i = 2; i < nu - 2; ++i) {
            const double d1 = (8.0 * (vl[i + 1] - vl[i - 1]) - (vl[i + 2] - vl[i - 2])) / (12.0 * h);
            const double d2 =
                (-30.0 * vl[i] + 16.0 * (vl[i + 1] + vl[i - 1]) - (vl[i + 2] + vl[i - 2])) / (12.0 * h * h);
            rho[i] = -(1.0 / (8.0 * M_PI)) * (d2 + (2.0 / mesh[i]) * d1);
        }
        rho[0] = rho[1] = rho[2];
        rho[nu - 2] = rho[nu - 1] = 0.0;
        int i_cut = (int)std::floor(u->cutoff_vlocal / h);
        // sign changes of rho and the most negative r^2 rho
        int nodes = 0, node2 = 0, i_peak = 0;
        double r2rho_min = 0.0;
        for (int i = 1; i < nu - 1; ++i) {
            if (rho[i] * rho[i + 1] < 0.0 && ++nodes == 2) node2 = i;
            const double r2rho = mesh[i] * mesh[i] * rho[i];
            if (r2rho_min > r2rho) {
                r2rho_min = r2rho;
                i_peak = i;
            }
        }
        if (node2 > i_cut) {   // the density's second node lies outside: extend the cutoff
            i_cut = std::min(node2, (int)(i_cut * 1.5));
            u->cutoff_vlocal = mesh[i_cut];
        }
        // blend start: where r^2 rho climbs back above half its minimum
        int i_in = 0;
        for (int i = i_peak + 1; i < i_cut - 1; ++i)
            if (r2rho_min * 0.5 < mesh[i] * mesh[i] * rho[i]) {
                i_in = i;
                break;
            }
        std::vector<double> vc(nu);
        for (int i = i_cut; i < nu; ++i) vc[i] = -2.0 * zv / mesh[i];
        for (int i = 0; i < i_in; ++i) vc[i] = vl[i];
        const double width = mesh[i_cut] - mesh[i_in];
        for (int i = i_in; i < i_cut; ++i) {
            const double x = (mesh[i] - mesh[i_in]) / width;
            const double f = x * x * x * x * (-20.0 * x * x * x + 70.0 * x * x - 84.0 * x + 35.0);
            vc[i] = f * (-2.0 * zv / mesh[i]) + (1.0 - f) * vl[i];
        }
        u->v_local.resize(u->n_grid);
        const Quintic qv{vc.data(), nu, mesh[0], h, 1};
        for (int i = 0; i < u->n_grid; ++i) {
            double v;
            qv.eval(u->radius[i], v, nullptr);
            u->v_local[i] = v / 2.0;
        }
    }
    // projectors: (r beta)(r) / r, resampled
    u->proj.resize((size_t)u->n_proj * u->n_grid);
    for (int k = 0; k < u->n_proj; ++k) {
        const std::string name = "PP_BETA." + std::to_string(k + 1);
        const Span b = find_path(s, {"UPF", "PP_NONLOCAL", name.c_str()});
        std::vector<double> p = numbers(s, b, nu);
        for (int i = 1; i < nu; ++i) p[i] /= mesh[i];
        p[0] = u->l[k] == 0 ? p[1] : 0.0;
        const Quintic q{p.data(), nu, mesh[0], h, (u->l[k] & 1) ? -1 : 1};
        for (int i = 0; i < u->n_grid; ++i) q.eval(u->radius[i], u->proj[(size_t)k * u->n_grid + i], nullptr);
    }
    *out = u;
    return QSB_OK;
}

qsb_status qsb_upf_destroy(qsb_upf* u) {
    delete u;
    return QSB_OK;
}

qsb_status qsb_upf_info(const qsb_upf* u, int* n_projectors, double* z_valence, int* n_grid, double* cutoff_l,
                        double* xi_min_delta) {
    if (!u) return fail(QSB_ERR_INVALID, "upf_info: null handle");
    if (n_projectors) *n_projectors = u->n_proj;
    if (z_valence) *z_valence = u->z_valence;
    if (n_grid) *n_grid = u->n_grid;
    if (cutoff_l) std::memcpy(cutoff_l, u->cutoff_l, sizeof(u->cutoff_l));
    if (xi_min_delta) {
        xi_min_delta[0] = u->xi_min;
        xi_min_delta[1] = u->xi_delta;
    }
    return QSB_OK;
}

qsb_status qsb_upf_radial(const qsb_upf* u, double* radius, double* v_local, int* l, double* energy,
                          double* projectors) {
    if (!u) return fail(QSB_ERR_INVALID, "upf_radial: null handle");
    if (radius) std::copy(u->radius.begin(), u->radius.end(), radius);
    if (v_local) std::copy(u->v_local.begin(), u->v_local.end(), v_local);
    if (l) std::copy(u->l.begin(), u->l.end(), l);
    if (energy) std::copy(u->energy.begin(), u->energy.end(), energy);
    if (projectors) std::copy(u->proj.begin(), u->proj.end(), projectors);
    return QSB_OK;
}

qsb_status qsb_radial_local_table(int n_r, const double* radius, const double* v, double z, double sigma,
                                 int n_g, double dg, double* table) {
    if (n_r < 5 || !radius || !v || !table || n_g <= 0 || !(dg > 0) || !(sigma > 0))
        return fail(QSB_ERR_INVALID, "radial_local_table: bad argument");
    if (!(radius[0] > 0.0) || !(radius[1] > radius[0]))
        return fail(QSB_ERR_INVALID, "radial_local_table: radius must start above 0 and increase");
    // log grid: r_i = r_0 exp(i dxi); integrals in xi with dr = r dxi (Simpson,
    // trapezoid on a last odd interval)
    const double dxi = std::log(radius[1] / radius[0]);
    for (int i = 2; i < n_r; ++i)
        if (std::fabs(std::log(radius[i] / radius[i - 1]) - dxi) > 1e-9 * std::fabs(dxi) + 1e-12)
            return fail(QSB_ERR_INVALID, "radial_local_table: radius is not a logarithmic grid");
    const double s2 = std::sqrt(2.0) * sigma;
    std::vector<double> sr(n_r);   // r^3 (V + z erf(r / (sqrt2 sigma)) / r), the short-range part times r^3
    for (int i = 0; i < n_r; ++i) {
        const double r = radius[i];
        sr[i] = r * r * r * (v[i] + z * std::erf(r / s2) / r);
    }
    auto simpson = [&](auto f) {
        const int m = (n_r - 1) % 2 ? n_r - 1 : n_r;   // odd point count for Simpson
        double acc = f(0) + f(m - 1);
        for (int i = 1; i < m - 1; ++i) acc += (i % 2 ? 4.0 : 2.0) * f(i);
        acc *= dxi / 3.0;
        if (m < n_r) acc += 0.5 * dxi * (f(n_r - 2) + f(n_r - 1));
        return acc;
    };
    for (int j = 0; j < n_g; ++j) {
        const double G = j * dg;
        // 4 pi int r^2 V_sr j0(G r) dr = 4 pi int r^3 V_sr j0(G r) dxi
        const double vs = 4.0 * M_PI * simpson([&](int i) {
            const double x = G * radius[i];
            return sr[i] * (x > 1e-8 ? std::sin(x) / x : 1.0 - x * x / 6.0);
        });
        const double coul = j == 0 ? 2.0 * M_PI * z * sigma * sigma
                                   : -4.0 * M_PI * z * std::exp(-0.5 * G * G * sigma * sigma) / (G * G);
        table[j] = vs + coul;
    }
    return QSB_OK;
}

qsb_status qsb_upf_grid_tables(const qsb_upf* const* upf, int n_species, int n_atoms, const double* pos,
                               const int* species, double dx, double dy, double dz, int* n_entries,
                               int64_t* n_points, int64_t* n_values, int* entry_atom, int* npts, int* widths,
                               int* coords, double* beta, double* energy, double* dbeta) {
    if (!upf || n_species <= 0 || n_atoms < 0 || (n_atoms > 0 && (!pos || !species)) || !n_entries || !n_points ||
        !n_values || !(dx > 0 && dy > 0 && dz > 0))
        return fail(QSB_ERR_INVALID, "upf_grid_tables: bad argument");
    struct Entry {
        int atom, k0, k1, width;
    };
    std::vector<Entry> entries;
    for (int a = 0; a < n_atoms; ++a) {
        const int s = species[a];
        if (s < 0 || s >= n_species || !upf[s]) return fail(QSB_ERR_INVALID, "upf_grid_tables: bad species");
        const qsb_upf& u = *upf[s];
        for (int k = 0; k < u.n_proj;) {   // whole radial projectors, at most 16 columns per entry
            Entry e{a, k, k, 0};
            while (e.k1 < u.n_proj && e.width + 2 * u.l[e.k1] + 1 <= 16) e.width += 2 * u.l[e.k1++] + 1;
            entries.push_back(e);
            k = e.k1;
        }
    }
    const bool fill = entry_atom && npts && widths && coords && beta && energy;
    int64_t tp = 0, tv = 0, te = 0;   // points, values (points x width), energies so far
    for (size_t ei = 0; ei < entries.size(); ++ei) {
        const Entry& e = entries[ei];
        const qsb_upf& u = *upf[species[e.atom]];
        double rmax = 0.0;
        for (int k = e.k0; k < e.k1; ++k) rmax = std::max(rmax, u.cutoff_l[u.l[k]]);
        const double Rx = pos[3 * e.atom], Ry = pos[3 * e.atom + 1], Rz = pos[3 * e.atom + 2];
        const int ix0 = (int)std::floor((Rx - rmax) / dx), ix1 = (int)std::ceil((Rx + rmax) / dx);
        const int iy0 = (int)std::floor((Ry - rmax) / dy), iy1 = (int)std::ceil((Ry + rmax) / dy);
        const int iz0 = (int)std::floor((Rz - rmax) / dz), iz1 = (int)std::ceil((Rz + rmax) / dz);
        std::vector<int> c;
        for (int iz = iz0; iz <= iz1; ++iz)
            for (int iy = iy0; iy <= iy1; ++iy)
                for (int ix = ix0; ix <= ix1; ++ix) {
                    const double x = ix * dx - Rx, y = iy * dy - Ry, z = iz * dz - Rz;
                    if (x * x + y * y + z * z > rmax * rmax) continue;
                    c.push_back(ix), c.push_back(iy), c.push_back(iz);
                }
        const int np = (int)(c.size() / 3);
        if (fill) {
            entry_atom[ei] = e.atom;
            npts[ei] = np;
            widths[ei] = e.width;
            std::copy(c.begin(), c.end(), coords + 3 * tp);
            double* bcol = beta + tv;                        // np x width, column-major
            double* gcol = dbeta ? dbeta + 3 * tv : nullptr;  // d/dx, d/dy, d/dz blocks of np x width
            int w = 0;
            for (int k = e.k0; k < e.k1; ++k) {
                const int l = u.l[k];
                const double* radial = u.proj.data() + (size_t)k * u.n_grid;
                const Quintic q{radial, u.n_grid, u.xi_min, u.xi_delta, 0};
                for (int m = -l; m <= l; ++m, ++w) {
                    energy[te + w] = u.energy[k];
                    for (int p = 0; p < np; ++p) {
                        const double x = c[3 * p] * dx - Rx, y = c[3 * p + 1] * dy - Ry, z = c[3 * p + 2] * dz - Rz;
                        const double r = std::sqrt(x * x + y * y + z * z);
                        double val = 0.0, g[3] = {0, 0, 0};
                        if (r <= u.cutoff_l[l]) {
                            if (r < u.radius[0]) {
                                // inside the log grid's first point: the l = 0 value, 0 otherwise
                                if (l == 0) val = radial[0] * poly(0, 0, 0, 0, 0).v;
                            } else {
                                double R, dR_dxi;
                                q.eval(std::log(r), R, &dR_dxi);
                                // beta = f P_lm with f = R / r^l; grad = f'(r) (x / r) P + f grad P
                                const double rl = std::pow(r, l);
                                const double f = R / rl;
                                const double df = dR_dxi / r / rl - (double)l * f / r;
                                const D P = poly(l, m, x, y, z);
                                val = f * P.v;
                                const double v[3] = {x, y, z};
                                for (int d = 0; d < 3; ++d) g[d] = df * v[d] / r * P.v + f * P.d[d];
                            }
                        }
                        bcol[(size_t)w * np + p] = val;
                        if (gcol)
                            for (int d = 0; d < 3; ++d) gcol[((size_t)d * e.width + w) * np + p] = g[d];
                    }
                }
            }
        }
        tp += np;
        tv += (int64_t)np * e.width;
        te += e.width;
    }
    *n_entries = (int)entries.size();
    *n_points = tp;
    *n_values = tv;
    return QSB_OK;
}

}  // extern "C"
