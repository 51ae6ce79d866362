// oracle.cpp -- FP64 CPU restatement of SurfMol's multi-system relaxation path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// library in surfmol_b200/: only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py load it.  The product never links or calls it.
//
// Parity is pinned against the reference's own known answers (H2 bond test
// crates/libs/oclff/tests/test_uff_cl.rs:8-56; pentacene energies and
// restoring force doc/topical_audit/uff.md:91-93, userguide/uff_spff.md:229)
// and, for the grid path that the reference never tests, against brute-force
// FP64 sums (Morse image sums, Ewald-2D vs a direct image sum, B-spline fit
// reproducing node values).
//
// What each part restates (reference file:line):
//   parameter tables ........ data/ElementTypes.dat, data/AtomTypes.dat (rows used here)
//   typing .................. crates/libs/moltopo/src/assign_uff.rs:8-125, topology.rs:7-35
//   topology ................ topology.rs:101-182, molecular.rs:34-79
//   UFF parameters .......... crates/libs/molff/src/uff.rs:699-887, moltopo/src/params.rs:595-657
//   term neighbour slots .... uff.rs:250-315
//   bonded forces ........... opencl/UFF.cl:141-322 (bonds), 326-501 (angles),
//                             505-670 (dihedrals), 674-795 (inversions), 801-880 (assembly)
//   non-bonded + grid ....... opencl/UFF.cl:57-95 (mixing, LJQH), 1384-1511 (B-spline sampler),
//                             1524-1718 (getNonBond_GridFF_Bspline)
//   grid build .............. opencl/gridff_build.cl:8-61 (B-spline forward operator),
//                             217-347 (make_MorseFF), opencl/Surface.cl:834-906 (Ewald-2D full),
//                             911-954 (brute image sum)
//   FIRE .................... crates/apps/molengine/src/main.rs:237-277 (relax_fire),
//                             crates/libs/molff/src/raff.rs:1040-1062 (FireState defaults)
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <string>
#include <vector>
#include <algorithm>
#include <tuple>
#include <array>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double COULOMB_K = 14.3996448915;          // eV*A/e^2, opencl/UFF.cl:51
const double KCAL_TO_EV = 4.1840 / 60.2214076 / 1.602176634;  // params.rs:601
const double UFF_K = 28.7989689090648;           // uff.rs:738, params.rs:638
const double DEG2RAD = M_PI / 180.0;

// ------------------------------------------------------------------ tables
struct Elem { const char* name; int Z; double r_vdw, e_vdw, q_uff, u_uff, v_uff, e_aff; };
// Rows of data/ElementTypes.dat (columns RvdW, EvdW, Quff, Uuff, Vuff, Eaff).
const Elem ELEMS[] = {
    {"H", 1, 1.4430, 0.00190802059, 0.712, 0.0, 0.0, -4.528},
    {"C", 6, 1.9255, 0.00455323095, 1.912, 0.08672820848, 0.09188853689, -5.343},
    {"N", 7, 1.8300, 0.00299212319, 2.544, 0.08672820848, 0.01951384691, -6.899},
    {"O", 8, 1.7500, 0.00260184625, 2.300, 0.08672820848, 0.00078055388, -8.741},
    {"Na", 11, 1.4915, 0.00130092313, 1.081, 0.05420513030, 0.0, -2.843},
    {"Cl", 17, 1.9735, 0.00984365166, 2.348, 0.05420513030, 0.0, -8.564},
};
struct AType { const char* name; const char* elem; double r_uff, r_vdw, e_vdw, q_base, h_b, a_ss; };
// Rows of data/AtomTypes.dat (columns Ruff, RvdW, EvdW, Qbase, Hb, Ass).  a_ss is
// 0 for rows shorter than 19 columns, as params.rs:178-187 parses them (H_).
const AType ATYPES[] = {
    {"H_", "H", 0.354, 1.4430, 0.00190802059, 0.0, 0.0, 0.0},
    {"C_3", "C", 0.757, 1.9255, 0.00455323095, 0.0, 0.0, 109.47},
    {"C_R", "C", 0.729, 1.9255, 0.00455323095, 0.0, 0.0, 120.0},
    {"C_2", "C", 0.732, 1.9255, 0.00455323095, 0.0, 0.0, 120.0},
    {"C_1", "C", 0.706, 1.9255, 0.00455323095, 0.0, 0.0, 180.0},
    {"N_3", "N", 0.700, 1.8300, 0.00299212319, 0.0, -0.9, 106.7},
    {"N_R", "N", 0.699, 1.8300, 0.00299212319, 0.0, 0.9, 120.0},
    {"N_2", "N", 0.685, 1.8300, 0.00299212319, 0.0, -0.9, 111.2},
    {"N_1", "N", 0.656, 1.8300, 0.00299212319, 0.0, 0.0, 180.0},
    {"O_3", "O", 0.658, 1.7500, 0.00260184625, 0.0, -0.95, 104.51},
    {"O_R", "O", 0.680, 1.7500, 0.00260184625, 0.0, -0.95, 110.0},
    {"O_2", "O", 0.634, 1.7500, 0.00260184625, 0.0, -0.95, 120.0},
    {"O_1", "O", 0.639, 1.7500, 0.00260184625, 0.0, 0.0, 180.0},
    {"Na", "Na", 1.539, 1.4915, 0.00130092313, 0.0, 0.0, 0.0},
    {"Cl", "Cl", 1.044, 1.9735, 0.00984365166, 0.0, 0.0, 0.0},
};
const int N_ATYPES = sizeof(ATYPES) / sizeof(ATYPES[0]);

const Elem* elem_by_name(const std::string& s) {
    for (const Elem& e : ELEMS) if (s == e.name) return &e;
    return nullptr;
}
const Elem* elem_by_Z(int Z) {
    for (const Elem& e : ELEMS) if (e.Z == Z) return &e;
    return nullptr;
}
int atype_index(const std::string& s) {
    for (int i = 0; i < N_ATYPES; i++) if (s == ATYPES[i].name) return i;
    return -1;
}
const AType* atype(const std::string& s) { int i = atype_index(s); return i < 0 ? nullptr : &ATYPES[i]; }
const Elem* elem_of_atype(const std::string& s) { const AType* t = atype(s); return t ? elem_by_name(t->elem) : nullptr; }

// ------------------------------------------------------------------ typing (assign_uff.rs, topology.rs)
int ne_pairs(const std::string& e) {   // topology.rs:7-20
    if (e == "N" || e == "P") return 1;
    if (e == "O" || e == "S") return 2;
    if (e == "F" || e == "Cl") return 3;
    return 0;
}
int hybridization(const std::string& e, int nn) {   // topology.rs:28-35
    if (e == "H") return 1;
    int npi = 4 - ne_pairs(e) - nn;
    if (npi < 0) return 1;
    return npi == 0 ? 3 : (npi == 1 ? 2 : 1);
}
bool type_exists(const std::string& s) {   // assign_uff.rs:119-122
    static const char* known[] = {"H_", "C_3", "C_R", "C_2", "C_1", "N_3", "N_R", "N_2", "N_1",
                                  "O_3", "O_R", "O_2", "O_1", "F", "Cl", "Si3", "P", "S"};
    for (const char* k : known) if (s == k) return true;
    return false;
}
std::vector<std::string> assign_types(const std::vector<std::string>& el, const std::vector<std::array<int,4>>& ng) {
    // assign_uff.rs:8-117
    int n = (int)el.size();
    std::vector<std::string> t(el);
    std::vector<char> set(n, 0);
    for (int ia = 0; ia < n; ia++) {
        if (set[ia]) continue;
        const std::string& e = el[ia];
        int nb = 0; while (nb < 4 && ng[ia][nb] >= 0) nb++;
        int h = hybridization(e, nb);
        if (e == "H") { t[ia] = "H_"; set[ia] = 1; continue; }
        if (e == "N" && nb == 3) {
            int no = 0;
            for (int s = 0; s < 3; s++) { int ja = ng[ia][s]; if (ja >= 0 && el[ja] == "O") no++; }
            if (no == 2) {
                t[ia] = "N_R"; set[ia] = 1;
                for (int s = 0; s < 3; s++) { int ja = ng[ia][s]; if (ja >= 0 && el[ja] == "O") { t[ja] = "O_R"; set[ja] = 1; } }
                continue;
            }
        }
        if (e == "O" && nb == 1) { t[ia] = "O_2"; set[ia] = 1; continue; }
        if (e == "C" && nb == 2) { t[ia] = "C_1"; set[ia] = 1; continue; }
        std::string suf = h == 3 ? "3" : (h == 2 ? ((e == "C" || e == "N" || e == "O") ? "R" : "2") : (h == 1 ? "1" : "3"));
        std::string tn = e + "_" + suf;
        if (type_exists(tn)) { t[ia] = tn; set[ia] = 1; }
        else if (type_exists(e)) { t[ia] = e; set[ia] = 1; }
    }
    return t;
}

char hyb_suffix(const std::string& t) {   // uff.rs:674-679
    size_t i = t.rfind('_');
    if (i != std::string::npos && i + 1 < t.size()) return t[i + 1];
    return '3';
}
std::string elem_sym(const std::string& t) { size_t i = t.find('_'); return i == std::string::npos ? t : t.substr(0, i); }

double bond_order_from_types(const std::string& a, const std::string& b) {   // params.rs:617-623
    auto ends = [](const std::string& s, const char* suf) { size_t n = strlen(suf); return s.size() >= n && s.compare(s.size() - n, n, suf) == 0; };
    if (ends(a, "_1") || ends(b, "_1")) return 3.0;
    if (ends(a, "_2") && ends(b, "_2")) return 2.0;
    return 1.0;
}
double calc_rij(const std::string& ta, const std::string& tb, double bo) {   // uff.rs:685-694, params.rs:627-635
    const AType* ti = atype(ta); const AType* tj = atype(tb);
    const Elem* ei = elem_of_atype(ta); const Elem* ej = elem_of_atype(tb);
    if (!ti || !tj || !ei || !ej) return 1.5;
    double r_bo = -0.1332 * (ti->r_uff + tj->r_uff) * std::log(bo);
    double r_en = 0.0;
    if (ei->e_aff < 0.0 && ej->e_aff < 0.0) {
        double s = std::sqrt(-ei->e_aff) - std::sqrt(-ej->e_aff);
        r_en = ti->r_uff * tj->r_uff * s * s / (-ei->e_aff * ti->r_uff - ej->e_aff * tj->r_uff);
    }
    return ti->r_uff + tj->r_uff + r_bo - r_en;
}

struct V3 { double x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(double s, V3 a) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
struct Q4 { V3 f; double w; };

}  // namespace

// ------------------------------------------------------------------ system
struct orc_sys {
    int n = 0;
    std::vector<std::array<int,4>> neighs, neighBs;
    std::vector<std::array<int,2>> bonds;
    std::vector<std::array<double,2>> bparams;          // (k, l0)
    std::vector<std::array<int,3>> angs; std::vector<std::array<int,2>> ang_ngs; std::vector<std::array<double,5>> angp; // (K,c0,c1,c2,c3)
    std::vector<std::array<int,4>> dihs; std::vector<std::array<int,3>> dih_ngs; std::vector<std::array<double,3>> dihp; // (V,d,n)
    std::vector<std::array<int,4>> invs; std::vector<std::array<int,3>> inv_ngs; std::vector<std::array<double,4>> invp; // (K,c0,c1,c2)
    std::vector<std::array<double,4>> req;               // (R, sqrt(E), Q, H)
    std::vector<int> type_id;
    // periodic molecules: per neighbour slot the lattice offset of the bonded image (neighCell,
    // opencl/UFF.cl:152, 229-236), as a cell code; empty for molecules without periodic bonds
    std::vector<std::array<int,4>> ngc;
    std::vector<std::array<int,3>> bond_off;             // per bond: offset of atom 1's image seen from atom 0
};

// Cell code of a lattice offset (ox, oy, oz), each in [-8, 7]: one 4-bit two's-complement field per axis.
inline int cell_code(int ox, int oy, int oz) { return (ox & 15) | ((oy & 15) << 4) | ((oz & 15) << 8); }
inline int cell_field(int c, int k) { int v = (c >> (4 * k)) & 15; return v >= 8 ? v - 16 : v; }

// Folded surface (crates/libs/surfff/src/lib.rs:126-351, SurfaceFolded): separable basis of
// lattice harmonics cos(2 pi k u), cos(2 pi k v) and z decays exp(-kz (z - z0)), one coefficient
// per basis function and channel (charge, Pauli, London), basis index ix + nx (iy + ny iz).
struct orc_folded {
    double inv[4];          // inv_ax, inv_bx, inv_ay, inv_by (inverse of the 2D lattice)
    int nx, ny, nz;
    const double *kx, *ky, *kz, *z0;
    const double *cq, *cp, *cl;
    double alpha;           // make_plqs exponent (molengine uses 2.0)
    double fmax;            // per-atom force clamp of eval_all_clamped (mol_world.rs:82: 100 eV/A)
};

struct orc_grid {
    int nx, ny, nz;
    double p0[3], step[3];
    const float* cf32;      // z-fastest (nx*ny*nz*4) float B-spline coefficients, or
    const double* cf64;     // the same in double (exactly one is non-null)
    double scale[4];        // per-channel scale folded into the atom prefactor (1 for fp32/f64 data)
    const orc_folded* folded;   // non-null: the substrate is this folded surface, not the grid
};

namespace {

void fill_neighs(orc_sys& S) {   // molecular.rs:34-79
    S.neighs.assign(S.n, {-1, -1, -1, -1});
    S.neighBs.assign(S.n, {-1, -1, -1, -1});
    for (size_t ib = 0; ib < S.bonds.size(); ib++) {
        int a = S.bonds[ib][0], b = S.bonds[ib][1];
        for (int s = 0; s < 4; s++) if (S.neighs[a][s] < 0) { S.neighs[a][s] = b; S.neighBs[a][s] = (int)ib; break; }
        for (int s = 0; s < 4; s++) if (S.neighs[b][s] < 0) { S.neighs[b][s] = a; S.neighBs[b][s] = (int)ib; break; }
    }
}

void build_terms(orc_sys& S) {
    int n = S.n;
    std::vector<std::vector<int>> adj(n);
    for (auto& b : S.bonds) { adj[b[0]].push_back(b[1]); adj[b[1]].push_back(b[0]); }
    // angles, topology.rs:113-129
    S.angs.clear();
    for (int j = 0; j < n; j++)
        for (size_t a = 0; a < adj[j].size(); a++)
            for (size_t b = a + 1; b < adj[j].size(); b++) S.angs.push_back({adj[j][a], j, adj[j][b]});
    // dihedrals, topology.rs:131-159; the reference collects through a HashSet, so the
    // order here is canonical (lexicographic) rather than hash order.
    S.dihs.clear();
    for (int j = 0; j < n; j++)
        for (int k : adj[j])
            for (int i : adj[j]) {
                if (i == k) continue;
                for (int l : adj[k]) { if (l == j) continue; if (l > i) S.dihs.push_back({i, j, k, l}); }
            }
    std::sort(S.dihs.begin(), S.dihs.end());
    S.dihs.erase(std::unique(S.dihs.begin(), S.dihs.end()), S.dihs.end());
    // inversions, topology.rs:161-182
    S.invs.clear();
    for (int i = 0; i < n; i++)
        if (adj[i].size() == 3) {
            const auto& s = adj[i];
            S.invs.push_back({i, s[0], s[1], s[2]});
            S.invs.push_back({i, s[2], s[0], s[1]});
            S.invs.push_back({i, s[1], s[2], s[0]});
        }
}

void bake_slots(orc_sys& S) {   // uff.rs:250-315
    S.ang_ngs.resize(S.angs.size());
    for (size_t a = 0; a < S.angs.size(); a++) {
        int i = S.angs[a][0], j = S.angs[a][1], k = S.angs[a][2], ji = -1, jk = -1;
        for (int s = 0; s < 4; s++) { int g = S.neighs[j][s]; if (g < 0) break; if (g == i) ji = j * 4 + s; else if (g == k) jk = j * 4 + s; }
        S.ang_ngs[a] = {ji, jk};
    }
    S.dih_ngs.resize(S.dihs.size());
    for (size_t d = 0; d < S.dihs.size(); d++) {
        int i = S.dihs[d][0], j = S.dihs[d][1], k = S.dihs[d][2], l = S.dihs[d][3], ji = -1, jk = -1, kl = -1;
        for (int s = 0; s < 4; s++) { int g = S.neighs[j][s]; if (g < 0) break; if (g == i) ji = j * 4 + s; else if (g == k) jk = j * 4 + s; }
        for (int s = 0; s < 4; s++) { int g = S.neighs[k][s]; if (g < 0) break; if (g == l) kl = k * 4 + s; }
        S.dih_ngs[d] = {ji, jk, kl};
    }
    S.inv_ngs.resize(S.invs.size());
    for (size_t v = 0; v < S.invs.size(); v++) {
        int i = S.invs[v][0], j = S.invs[v][1], k = S.invs[v][2], l = S.invs[v][3], ij = -1, ik = -1, il = -1;
        for (int s = 0; s < 3; s++) { int g = S.neighs[i][s]; if (g == j) ij = i * 4 + s; else if (g == k) ik = i * 4 + s; else if (g == l) il = i * 4 + s; }
        S.inv_ngs[v] = {ij, ik, il};
    }
}

void setup_params(orc_sys& S, const std::vector<std::string>& T) {   // uff.rs:699-887
    const auto& ng = S.neighs;
    auto nbonds_of = [&](int a) { int c = 0; while (c < 4 && ng[a][c] >= 0) c++; return (double)c; };
    S.bparams.resize(S.bonds.size());
    for (size_t ib = 0; ib < S.bonds.size(); ib++) {
        const std::string& ta = T[S.bonds[ib][0]]; const std::string& tb = T[S.bonds[ib][1]];
        double bo = bond_order_from_types(ta, tb);
        double l0 = calc_rij(ta, tb, bo);
        const Elem* ei = elem_of_atype(ta); const Elem* ej = elem_of_atype(tb);
        if (!ei || !ej) { S.bparams[ib] = {100.0, l0}; continue; }
        S.bparams[ib] = {0.5 * UFF_K * ei->q_uff * ej->q_uff / (l0 * l0 * l0), l0};
    }
    S.angp.resize(S.angs.size());
    for (size_t a = 0; a < S.angs.size(); a++) {
        int i = S.angs[a][0], j = S.angs[a][1], k = S.angs[a][2];
        const std::string &tj = T[j], &ti = T[i], &tk = T[k];
        S.angp[a] = {0, 0, 0, 0, 0};
        if (elem_sym(tj) == "H") continue;
        const AType* at = atype(tj); const Elem* ei = elem_of_atype(ti); const Elem* ek = elem_of_atype(tk);
        if (!at || !ei || !ek) continue;
        double ct = std::cos(at->a_ss * DEG2RAD), st = std::sin(at->a_ss * DEG2RAD), st2 = st * st;
        double rij = calc_rij(ti, tj, bond_order_from_types(ti, tj));
        double rjk = calc_rij(tj, tk, bond_order_from_types(tj, tk));
        double rik = std::sqrt(rij * rij + rjk * rjk - 2.0 * rij * rjk * ct);
        double kappa = UFF_K * ei->q_uff * ek->q_uff / std::pow(rik, 5) * (3.0 * rij * rjk * st2 - rik * rik * ct);
        char h = hyb_suffix(tj);
        if (h == '1') S.angp[a] = {kappa, 1.0, 1.0, 0.0, 0.0};
        else if (h == '2' || h == 'R') S.angp[a] = {kappa / 9.0, 1.0, 0.0, 0.0, -1.0};
        else if (h == '3') {
            double c2 = 1.0 / (4.0 * st2), c1 = -4.0 * c2 * ct, c0 = c2 * (2.0 * ct * ct + 1.0);
            S.angp[a] = {kappa, c0, c1, c2, 0.0};
        } else S.angp[a] = {kappa, 1.0, 0.0, 0.0, -1.0};
    }
    S.dihp.resize(S.dihs.size());
    for (size_t d = 0; d < S.dihs.size(); d++) {
        int i2 = S.dihs[d][1], i3 = S.dihs[d][2];
        const std::string &t2 = T[i2], &t3 = T[i3];
        S.dihp[d] = {0.0, 1.0, 3.0};
        if (elem_sym(t2) == "H" || elem_sym(t3) == "H") continue;
        char h2 = hyb_suffix(t2), h3 = hyb_suffix(t3);
        if (h2 == '1' || h3 == '1') continue;
        bool s2 = h2 == '3', s3 = h3 == '3';
        bool p2 = h2 == '2' || h2 == 'R', p3 = h3 == '2' || h3 == 'R';
        const Elem* e2 = elem_of_atype(t2); const Elem* e3 = elem_of_atype(t3);
        double u2 = e2 ? e2->u_uff : 0.0, u3 = e3 ? e3->u_uff : 0.0, v2 = e2 ? e2->v_uff : 0.0, v3 = e3 ? e3->v_uff : 0.0;
        double bo = bond_order_from_types(t2, t3);
        double V, dsg, nn;
        if (s2 && s3) {
            std::string el2 = elem_sym(t2), el3 = elem_sym(t3);
            if ((el2 == "O" || el2 == "S") && (el3 == "O" || el3 == "S")) {
                double k = KCAL_TO_EV; k *= (el2 == "O") ? 2.0 : 6.8; k *= (el3 == "O") ? 2.0 : 6.8;
                V = std::sqrt(k); dsg = 1.0; nn = 2.0;
            } else { V = std::sqrt(v2 * v3); dsg = 1.0; nn = 3.0; }
        } else if ((s2 && p3) || (p2 && s3)) {
            V = KCAL_TO_EV; dsg = -1.0; nn = 6.0;
            std::string el_sp3 = s2 ? elem_sym(t2) : elem_sym(t3);
            if (el_sp3 == "O" || el_sp3 == "S") { V = 5.0 * std::sqrt(u2 * u3) * (1.0 + 4.18 * std::log(bo)); dsg = 1.0; nn = 2.0; }
            int sp3i = s2 ? i2 : i3, sp2i = s2 ? i3 : i2;
            bool has = false;
            for (int s = 0; s < 4; s++) {
                int g = ng[sp2i][s]; if (g < 0) break;
                if (g == sp3i) continue;
                char hn = hyb_suffix(T[g]); if (hn == '2' || hn == 'R') { has = true; break; }
            }
            if (has) { V = 2.0 * KCAL_TO_EV; dsg = 1.0; nn = 3.0; }
        } else if (p2 && p3) {
            V = 5.0 * std::sqrt(u2 * u3) * (1.0 + 4.18 * std::log(bo)); dsg = -1.0; nn = 2.0;
        } else { V = 0.0; dsg = 1.0; nn = 3.0; }
        double den = 0.5 * (nbonds_of(i2) - 1.0) * (nbonds_of(i3) - 1.0);
        S.dihp[d] = {den > 0.0 ? V / den : V, dsg, nn};
    }
    S.invp.resize(S.invs.size());
    for (size_t v = 0; v < S.invs.size(); v++) {
        int i1 = S.invs[v][0];
        const std::string& t1 = T[i1];
        std::string el1 = elem_sym(t1); char h1 = hyb_suffix(t1);
        double K = 0, c0 = 0, c1 = 0, c2 = 0;
        if (el1 == "C" && (h1 == '2' || h1 == 'R')) {
            bool carbonyl = false;
            for (int s = 0; s < 4; s++) { int g = ng[i1][s]; if (g < 0) break; if (elem_sym(T[g]) == "O" && hyb_suffix(T[g]) == '2') carbonyl = true; }
            K = (carbonyl ? 50.0 : 6.0) * KCAL_TO_EV; c0 = 1.0; c1 = -1.0; c2 = 0.0;
        } else if (el1 == "N" && (h1 == '2' || h1 == 'R')) {
            K = 6.0 * KCAL_TO_EV; c0 = 1.0; c1 = -1.0; c2 = 0.0;
        } else if (el1 == "P") {
            double w0 = 84.4339 * DEG2RAD;
            c0 = 4.0 * std::cos(w0) * std::cos(w0) - std::cos(2.0 * w0); c1 = -4.0 * std::cos(w0); c2 = 1.0;
            K = 22.0 * KCAL_TO_EV / (c0 + c1 + c2);
        }
        S.invp[v] = {K / 3.0, c0, c1, c2};
    }
    S.req.resize(S.n);
    S.type_id.resize(S.n);
    for (int a = 0; a < S.n; a++) {   // params.rs:595-605 (get_reqh)
        const AType* t = atype(T[a]);
        S.type_id[a] = atype_index(T[a]);
        if (t) S.req[a] = {t->r_vdw, std::sqrt(t->e_vdw), t->q_base, t->h_b};
        else { const Elem* e = elem_by_name(T[a]); S.req[a] = e ? std::array<double,4>{e->r_vdw, std::sqrt(e->e_vdw), e->q_uff, 0.0} : std::array<double,4>{1.5, 0, 0, 0}; }
    }
}

// ------------------------------------------------------------------ force field
inline double getLJQH(V3 dp, double R0, double E0, double Q, double R2damp, V3& f) {   // UFF.cl:82-95
    double r2 = dot(dp, dp);
    double ir2_ = 1.0 / (r2 + R2damp);
    double Ec = COULOMB_K * Q * std::sqrt(ir2_);
    double ir2 = 1.0 / r2;
    double u2 = R0 * R0 * ir2;
    double u6 = u2 * u2 * u2;
    double vdW = u6 * E0;
    double E = (u6 - 2.0) * vdW + Ec;
    double fr = -12.0 * (u6 - 1.0) * vdW * ir2 - Ec * ir2_;
    f = dp * fr;
    return E;
}

inline void bbasis(double u, double b[4]) {   // UFF.cl:1410-1421
    const double i6 = 1.0 / 6.0, u2 = u * u, t = 1.0 - u;
    b[0] = i6 * t * t * t; b[1] = i6 * (3.0 * u2 * (u - 2.0) + 4.0);
    b[2] = i6 * (3.0 * u * (1.0 + u - u2) + 1.0); b[3] = i6 * u2 * u;
}
inline void dbasis(double u, double d[4]) {   // UFF.cl:1422-1432
    const double u2 = u * u, t = 1.0 - u;
    d[0] = -0.5 * t * t; d[1] = 0.5 * (3.0 * u2 - 4.0 * u);
    d[2] = 0.5 * (-3.0 * u2 + 2.0 * u + 1.0); d[3] = 0.5 * u2;
}
inline int modulo(int i, int m) { int r = i % m; if (r < 0) r += m; return r; }

// fe3d_pbc_comb (UFF.cl:1459-1511): returns (dE/du_x, dE/du_y, dE/du_z, E) in grid units.
// One atom on the folded surface: energy and force (surfff/src/lib.rs:277-320), force clamped to
// fmax as eval_all_clamped does (lib.rs:245-253, 340-351).  plq as NonBondedFF::make_plqs
// (molff/src/nonbonded.rs:98-108): e = exp(-alpha R), L = e sqrt(req[1]), P = e L, with req[1]
// holding sqrt(E_vdW) (moltopo/src/params.rs:595-597), so L carries E_vdW^(1/4) as the code does.
double folded_atom(const orc_folded& f, const double req[4], V3 p, V3& force) {
    const double e = std::exp(-f.alpha * req[0]);
    const double L = e * std::sqrt(req[1]), P = e * L, Q = req[2];
    double u = f.inv[0] * p.x + f.inv[2] * p.y, v = f.inv[1] * p.x + f.inv[3] * p.y;
    u -= std::floor(u); v -= std::floor(v);
    const double tau = 2.0 * 3.14159265358979323846;
    double E = 0, dEdu = 0, dEdv = 0, dEdz = 0;
    int ic = 0;
    for (int iz = 0; iz < f.nz; iz++) {
        const double bz = std::exp(-f.kz[iz] * (p.z - f.z0[iz])), dbz = -f.kz[iz] * bz;
        for (int iy = 0; iy < f.ny; iy++) {
            const double by = std::cos(tau * f.ky[iy] * v), dby = -tau * f.ky[iy] * std::sin(tau * f.ky[iy] * v);
            for (int ix = 0; ix < f.nx; ix++, ic++) {
                const double bx = std::cos(tau * f.kx[ix] * u), dbx = -tau * f.kx[ix] * std::sin(tau * f.kx[ix] * u);
                const double c = f.cq[ic] * Q + f.cp[ic] * P + f.cl[ic] * L;
                E += c * bx * by * bz;
                dEdu += c * dbx * by * bz;
                dEdv += c * bx * dby * bz;
                dEdz += c * bx * by * dbz;
            }
        }
    }
    force = {-(dEdu * f.inv[0] + dEdv * f.inv[1]), -(dEdu * f.inv[2] + dEdv * f.inv[3]), -dEdz};
    const double f2 = dot(force, force);
    if (f2 > f.fmax * f.fmax) force = force * (f.fmax / std::sqrt(f2));
    return E;
}

void sample_grid(const orc_grid& g, const double PLQH[4], V3 u, double out[4]) {
    int ix = (int)u.x, iy = (int)u.y, iz = (int)u.z;
    if (u.x < 0) ix--;
    if (u.y < 0) iy--;
    double tx = u.x - ix, ty = u.y - iy, tz = u.z - iz;
    out[0] = out[1] = out[2] = out[3] = 0.0;
    if (iz < 1 || iz >= g.nz - 2) return;
    ix = modulo(ix - 1, g.nx);
    iy = modulo(iy - 1, g.ny);
    double bx[4], dx[4], by[4], dy[4], bz[4], dz[4];
    bbasis(tx, bx); dbasis(tx, dx); bbasis(ty, by); dbasis(ty, dy); bbasis(tz, bz); dbasis(tz, dz);
    double C[4]; for (int c = 0; c < 4; c++) C[c] = PLQH[c] * g.scale[c];
    double Ex[4], Ey[4], Ez[4];   // per x-slice: dE/dy, dE/dz, E
    for (int a = 0; a < 4; a++) {
        int xa = (ix + a) % g.nx;
        double sdy = 0, sdz = 0, se = 0;
        for (int b = 0; b < 4; b++) {
            int yb = (iy + b) % g.ny;
            double p = 0, d = 0;
            for (int k = 0; k < 4; k++) {
                size_t i = (size_t)(iz - 1 + k) + (size_t)g.nz * ((size_t)yb + (size_t)g.ny * xa);
                double cs = 0;
                for (int c = 0; c < 4; c++) cs += C[c] * (g.cf32 ? (double)g.cf32[4 * i + c] : g.cf64[4 * i + c]);
                p += bz[k] * cs; d += dz[k] * cs;
            }
            sdy += p * dy[b]; sdz += d * by[b]; se += p * by[b];
        }
        Ex[a] = sdy; Ey[a] = sdz; Ez[a] = se;
    }
    out[0] = dx[0] * Ez[0] + dx[1] * Ez[1] + dx[2] * Ez[2] + dx[3] * Ez[3];
    out[1] = bx[0] * Ex[0] + bx[1] * Ex[1] + bx[2] * Ex[2] + bx[3] * Ex[3];
    out[2] = bx[0] * Ey[0] + bx[1] * Ey[1] + bx[2] * Ey[2] + bx[3] * Ey[3];
    out[3] = bx[0] * Ez[0] + bx[1] * Ez[1] + bx[2] * Ez[2] + bx[3] * Ez[3];
}

// lvec: lattice vectors a, b, c of the system (lvecs[iS], opencl/UFF.cl:1532-1574); npbc: image
// counts per axis (nPBC); with all npbc 0 the NB sum has no images, as for an isolated molecule.
struct NBParams { double rdamp, alpha, rcut; int excl13; double lvec[9]; int npbc[3]; };
inline V3 lattice_shift(const NBParams& nb, int ox, int oy, int oz) {
    return V3{ox * nb.lvec[0] + oy * nb.lvec[3] + oz * nb.lvec[6], ox * nb.lvec[1] + oy * nb.lvec[4] + oz * nb.lvec[7],
              ox * nb.lvec[2] + oy * nb.lvec[5] + oz * nb.lvec[8]};
}
enum { E_TOT = 0, E_BOND, E_ANG, E_DIH, E_INV, E_NB, E_GRID, E_NCOMP = 8 };

// One force evaluation; forces F (n), per-atom energy Ea (n, the reference's fapos.w),
// energy components (physical totals: each bond and each NB pair counted once).
void eval_forces(const orc_sys& S, const V3* P, const orc_grid* g, const NBParams& nb, V3* F, double* Ea, double* Ec) {
    int n = S.n;
    std::vector<Q4> hn(4 * (size_t)n);
    double eb = 0, ea = 0, ed = 0, ei = 0, enb = 0, eg = 0;
    // bonds + hneigh (UFF.cl:141-322), bSubtractBondNonBond = 0
    for (int a = 0; a < n; a++) {
        V3 f{0, 0, 0}; double E = 0;
        for (int s = 0; s < 4; s++) {
            int g2 = S.neighs[a][s];
            if (g2 < 0) { hn[4 * a + s] = {{0, 0, 0}, 1e6}; continue; }
            V3 dp = P[g2] - P[a];
            // a bond to a neighbour's image in another cell (UFF.cl:229-236: dp += pbc_shifts[ngC])
            if (!S.ngc.empty() && S.ngc[a][s]) {
                const int c = S.ngc[a][s];
                dp = dp + lattice_shift(nb, cell_field(c, 0), cell_field(c, 1), cell_field(c, 2));
            }
            double l2 = dot(dp, dp); if (l2 < 1e-16) l2 = 1e-16;
            double l = std::sqrt(l2), il = 1.0 / l;
            V3 h = dp * il;
            hn[4 * a + s] = {h, il};
            int ib = S.neighBs[a][s];
            if (ib < 0) continue;
            double k = S.bparams[ib][0], l0 = S.bparams[ib][1], dl = l - l0;
            f = f + h * (2.0 * k * dl);
            E += k * dl * dl;
        }
        F[a] = f; Ea[a] = E; eb += 0.5 * E;
    }
    // angles (UFF.cl:326-501), bSubtractAngleNonBond = 0
    for (size_t t = 0; t < S.angs.size(); t++) {
        const Q4 &qij = hn[S.ang_ngs[t][0]], &qkj = hn[S.ang_ngs[t][1]];
        const auto& p = S.angp[t];
        V3 h = qij.f + qkj.f;
        double c = 0.5 * (dot(h, h) - 2.0);
        c = std::min(1.0, std::max(-1.0, c));
        double s = std::sqrt(std::max(0.0, 1.0 - c * c) + 1e-14);
        double is = s > 1e-12 ? 1.0 / s : 0.0;
        double c2x = c * c - s * s, c2y = 2.0 * c * s;            // cos 2t, sin 2t
        double c3x = c2x * c - c2y * s, c3y = c2x * s + c2y * c;   // cos 3t, sin 3t
        double E = p[0] * (p[1] + p[3] * c2x + p[4] * c3x);
        double fm = p[0] * (p[2] + p[3] * c2y * is * 2.0 + p[4] * c3y * is * 3.0);
        double fi = fm * qij.w, fk = fm * qkj.w, fic = fi * c, fkc = fk * c;
        V3 fpi = qij.f * fic - qkj.f * fi;
        V3 fpk = qij.f * (-fk) + qkj.f * fkc;
        V3 fpj = qij.f * (fk - fic) + qkj.f * (fi - fkc);
        int ia = S.angs[t][0], ja = S.angs[t][1], ka = S.angs[t][2];
        F[ia] = F[ia] + fpi; F[ja] = F[ja] + fpj; F[ka] = F[ka] + fpk;
        Ea[ia] += E / 3.0; Ea[ja] += E / 3.0; Ea[ka] += E / 3.0;
        ea += E;
    }
    // dihedrals (UFF.cl:505-670), SubNBTorsionFactor = 0
    for (size_t t = 0; t < S.dihs.size(); t++) {
        const Q4 &q12 = hn[S.dih_ngs[t][0]], &q32 = hn[S.dih_ngs[t][1]], &q43 = hn[S.dih_ngs[t][2]];
        const auto& p = S.dihp[t];
        V3 n123 = cross(q12.f, q32.f), n234 = cross(q43.f, q32.f);
        double a2 = dot(n123, n123), b2 = dot(n234, n234);
        V3 f1{0, 0, 0}, f2{0, 0, 0}, f3{0, 0, 0}, f4{0, 0, 0}; double E = 0;
        if (!(a2 < 1e-30 || b2 < 1e-30)) {
            double il2a = 1.0 / a2, il2b = 1.0 / b2, inv = std::sqrt(il2a * il2b);
            double cx = dot(n123, n234) * inv, cy = -dot(n123, q43.f) * inv;
            double nx = cx, ny = cy;
            int ni = (int)p[2];
            for (int r = 1; r < ni; r++) { double tx = nx * cx - ny * cy; ny = nx * cy + ny * cx; nx = tx; }
            E = p[0] * (1.0 + p[1] * nx);
            double f = -p[0] * p[1] * p[2] * ny;
            f1 = n123 * (-f * il2a * q12.w);
            f4 = n234 * (f * il2b * q43.w);
            double c123 = dot(q32.f, q12.f) * (q32.w / q12.w);
            double c432 = dot(q32.f, q43.f) * (q32.w / q43.w);
            f3 = f1 * (-c123) + f4 * (-c432 - 1.0);
            f2 = f1 * (c123 - 1.0) + f4 * c432;
        }
        const auto& d = S.dihs[t];
        F[d[0]] = F[d[0]] + f1; F[d[1]] = F[d[1]] + f2; F[d[2]] = F[d[2]] + f3; F[d[3]] = F[d[3]] + f4;
        for (int r = 0; r < 4; r++) Ea[d[r]] += 0.25 * E;
        ed += E;
    }
    // inversions (UFF.cl:674-795)
    for (size_t t = 0; t < S.invs.size(); t++) {
        const Q4 &q21 = hn[S.inv_ngs[t][0]], &q31 = hn[S.inv_ngs[t][1]], &q41 = hn[S.inv_ngs[t][2]];
        const auto& p = S.invp[t];
        V3 n = cross(-q21.f, -q31.f);
        double nn = dot(n, n), il = 0.0;
        if (nn > 1e-16) { il = 1.0 / std::sqrt(nn); n = n * il; } else n = {0, 0, 0};
        double sw = -dot(n, q41.f);
        sw = std::min(1.0, std::max(-1.0, sw));
        double cw = std::sqrt(1.0 - sw * sw);
        double c2w = 2.0 * cw * cw - 1.0;
        double E = p[0] * (p[1] + p[2] * cw + p[3] * c2w);
        double s2w = 2.0 * sw * cw;
        double dEdw = -p[0] * (p[2] * sw + 2.0 * p[3] * s2w);
        double ft = cw > 1e-7 ? dEdw / cw : 0.0;
        double fq41 = ft * q41.w, fi123 = ft * il;
        V3 tq = n * (sw * fi123) + q41.f * fi123;
        V3 f4 = n * fq41 + q41.f * (sw * fq41);
        V3 f2 = cross(q31.f, tq) * q21.w;
        V3 f3 = cross(tq, q21.f) * q31.w;
        V3 f1 = -(f2 + f3 + f4);
        const auto& v = S.invs[t];
        F[v[0]] = F[v[0]] + f1; F[v[1]] = F[v[1]] + f2; F[v[2]] = F[v[2]] + f3; F[v[3]] = F[v[3]] + f4;
        for (int r = 0; r < 4; r++) Ea[v[r]] += 0.25 * E;
        ei += E;
    }
    // non-bonded + grid (UFF.cl:1524-1718)
    const double R2damp = nb.rdamp * nb.rdamp;
    const double rc2 = nb.rcut > 0 ? nb.rcut * nb.rcut : 1e300;
    const bool pbc = nb.npbc[0] > 0 || nb.npbc[1] > 0 || nb.npbc[2] > 0;
    for (int a = 0; a < n; a++) {
        V3 fe{0, 0, 0}; double E = 0;
        const auto& ri = S.req[a];
        const auto& ng = S.neighs[a];
        // PBC images (UFF.cl:1592-1650): every partner j != a in every image of the (2 npbc + 1)^3
        // block, iz outer and ix inner; a bonded pair is excluded only in the image of its bond
        // (neighbour index and cell both match); an atom never meets its own images
        for (int j = 0; pbc && j < n; j++) {
            if (j == a) continue;
            const auto& rj = S.req[j];
            for (int iz = -nb.npbc[2]; iz <= nb.npbc[2]; iz++)
                for (int iy = -nb.npbc[1]; iy <= nb.npbc[1]; iy++)
                    for (int ix = -nb.npbc[0]; ix <= nb.npbc[0]; ix++) {
                        const int code = cell_code(ix, iy, iz);
                        bool bonded = false;
                        for (int s = 0; s < 4; s++)
                            if (ng[s] == j && (S.ngc.empty() ? 0 : S.ngc[a][s]) == code) bonded = true;
                        if (bonded) continue;
                        V3 dp = P[j] - P[a] + lattice_shift(nb, ix, iy, iz);
                        if (dot(dp, dp) > rc2) continue;
                        V3 f;
                        E += getLJQH(dp, ri[0] + rj[0], ri[1] * rj[1], ri[2] * rj[2], R2damp, f);
                        fe = fe + f;
                    }
        }
        for (int j = 0; !pbc && j < n; j++) {
            if (j == a) continue;
            if (j == ng[0] || j == ng[1] || j == ng[2] || j == ng[3]) continue;
            if (nb.excl13) {   // 1-3 exclusion: j bonded to a neighbour of a (getNonBond_ex2 semantics)
                bool ex = false;
                for (int s = 0; s < 4 && !ex; s++) { int g2 = ng[s]; if (g2 < 0) continue;
                    for (int r = 0; r < 4; r++) if (S.neighs[g2][r] == j) { ex = true; break; } }
                if (ex) continue;
            }
            V3 dp = P[j] - P[a];
            if (dot(dp, dp) > rc2) continue;
            const auto& rj = S.req[j];
            double H = ri[3] * rj[3]; (void)H;   // mixREQ_arithmetic computes H; getLJQH ignores it
            V3 f;
            E += getLJQH(dp, ri[0] + rj[0], ri[1] * rj[1], ri[2] * rj[2], R2damp, f);
            fe = fe + f;
        }
        enb += 0.5 * E;
        if (g && g->folded) {
            V3 fs;
            const double E1 = folded_atom(*g->folded, ri.data(), P[a], fs);
            fe = fe + fs;
            E += E1;
            eg += E1;
        } else if (g) {
            double ej = std::exp(nb.alpha * ri[0]);
            double PLQH[4] = {ej * ej * ri[1], ej * ri[1], ri[2], 0.0};
            V3 u = {(P[a].x - g->p0[0]) / g->step[0], (P[a].y - g->p0[1]) / g->step[1], (P[a].z - g->p0[2]) / g->step[2]};
            double fg[4];
            sample_grid(*g, PLQH, u, fg);
            fe = fe + V3{-fg[0] / g->step[0], -fg[1] / g->step[1], -fg[2] / g->step[2]};
            E += fg[3];
            eg += fg[3];
        }
        F[a] = F[a] + fe;
        Ea[a] += E;
    }
    if (Ec) {
        for (int c = 0; c < E_NCOMP; c++) Ec[c] = 0;
        Ec[E_BOND] = eb; Ec[E_ANG] = ea; Ec[E_DIH] = ed; Ec[E_INV] = ei; Ec[E_NB] = enb; Ec[E_GRID] = eg;
        Ec[E_TOT] = eb + ea + ed + ei + enb + eg;
    }
}

struct FireParams { double dt0, dt_max, alpha0, f_inc, f_dec, f_alpha; int n_min; double fconv, flimit; };

const double KB_EV = 8.617333262145e-5;            // eV/K, opencl/UFF.cl:52

// The pseudo-random vector of the thermal drive of updateAtomsMMFFf4 (opencl/UFF.cl:982-991):
// per component k a byte of (ia + c_k + (int)(m_k seed)) * 2654435761 (64-bit product, shifted
// right by 16) scaled to [0, 1), then sin((r_k + seed) * 124.4565) with the sum and product in
// FP32, as the kernel forms them, and the sine in FP64.
V3 langevin_noise(int ia, float seed) {
    static const int c[3] = {136, 778, 4578};
    static const float m[3] = {1000.f, 1013.f, 998.f};
    double out[3];
    for (int k = 0; k < 3; k++) {
        const float ms = m[k] * seed;
        const long long x = (long long)(ia + c[k] + (int)ms);
        const float r = (float)((x * 2654435761LL) >> 16 & 0xFF) * 0.00390625f;
        const float s = r + seed;
        const float arg = s * 124.4565f;
        out[k] = std::sin((double)arg);
    }
    return {out[0], out[1], out[2]};
}

// Driving terms of updateAtomsMMFFf4 that act on FIRE but are not stored with the forces:
// constraint springs (UFF.cl:974-982; per atom target xyz + on flag, stiffness xyz) and the
// Langevin drive (UFF.cl:982-991; td = T [K], gamma, seed increment per step, seed).
struct Drive {
    const double* cons = nullptr;    // n x 7: target x, y, z, on (> 0), kx, ky, kz
    const double* td = nullptr;      // 4 values, or null
};

// relax_fire, crates/apps/molengine/src/main.rs:237-277 (unit masses).  The step
// uses the dt read at the top of the iteration (main.rs:242), positions advance
// even on the converging step (main.rs:270-275), then the loop breaks.  With a drive, the
// force FIRE uses at step s is the limited force plus the springs at the current positions
// plus -gamma v + noise(seed + s * seed_step) sqrt(2 kB T gamma / dt), v the velocity before
// the step.
int relax_fire(const orc_sys& S, V3* P, const orc_grid* g, const NBParams& nb, const FireParams& fp, int max_steps,
               V3* F, double* Ea, double* Ec, double* fmax_out, int* conv_out, const Drive& dr = Drive{}) {
    int n = S.n;
    std::vector<V3> V(n, V3{0, 0, 0}), Fd(n);
    double dt = fp.dt0, alpha = fp.alpha0; int npos = 0;
    int steps = 0; double fmax = 0; int conv = 0;
    const bool therm = dr.td && dr.td[1] > 0.0;
    for (int itr = 0; itr < max_steps; itr++) {
        const double dt_old = dt;
        eval_forces(S, P, g, nb, F, Ea, Ec);
        double vf = 0, vv = 0, ff = 0, f2max = 0;
        const float seed = therm ? std::fma((float)dr.td[2], (float)itr, (float)dr.td[3]) : 0.f;
        const double amp = therm ? std::sqrt(2.0 * KB_EV * (double)(float)dr.td[0] * (double)(float)dr.td[1] / dt_old) : 0.0;
        for (int a = 0; a < n; a++) {
            V3 f = F[a];
            double f2 = dot(f, f);
            if (fp.flimit > 0 && f2 > fp.flimit * fp.flimit) { f = f * (fp.flimit / std::sqrt(f2)); F[a] = f; f2 = dot(f, f); }
            if (dr.cons && dr.cons[7 * a + 3] > 0.0) {
                const double* c = dr.cons + 7 * a;
                f = f + V3{(c[0] - P[a].x) * std::max(c[4], 0.0), (c[1] - P[a].y) * std::max(c[5], 0.0),
                           (c[2] - P[a].z) * std::max(c[6], 0.0)};
            }
            if (therm) f = f + V[a] * -(double)(float)dr.td[1] + langevin_noise(a, seed) * amp;
            f2 = dot(f, f);
            Fd[a] = f;
            if (f2 > f2max) f2max = f2;
            ff += f2;
            V[a] = V[a] + f * dt_old;
            vf += dot(V[a], f);
            vv += dot(V[a], V[a]);
        }
        if (vf > 0.0 && ff > 1e-30 && vv > 1e-30) {
            double vm = std::sqrt(vv), fm = std::sqrt(ff);
            for (int a = 0; a < n; a++) V[a] = V[a] * (1.0 - alpha) + (Fd[a] * (1.0 / fm)) * (alpha * vm);
            npos++;
            if (npos > fp.n_min) { dt = std::min(dt * fp.f_inc, fp.dt_max); alpha *= fp.f_alpha; }
        } else {
            npos = 0; dt *= fp.f_dec; alpha = fp.alpha0;
            for (int a = 0; a < n; a++) V[a] = {0, 0, 0};
        }
        for (int a = 0; a < n; a++) P[a] = P[a] + V[a] * dt_old;
        steps = itr + 1;
        fmax = std::sqrt(f2max);
        if (fmax < fp.fconv) { conv = 1; break; }
    }
    if (fmax_out) *fmax_out = fmax;
    if (conv_out) *conv_out = conv;
    return steps;
}

}  // namespace

// ------------------------------------------------------------------ grid build (FP64)
namespace {

// Morse (Pauli, London) at one point: make_MorseFF, gridff_build.cl:217-347, with
// (2n_a+1)(2n_b+1) lateral images of the slab cell (n_c = 0 for a slab).
void morse_point(V3 p, int nions, const double* ions, const double* re, double ax, double ay, double bx, double by,
                 int na, int nb, double alpha, double& paul, double& lond) {
    paul = 0; lond = 0;
    for (int j = 0; j < nions; j++) {
        double R = re[4 * j + 0], E = re[4 * j + 1];
        for (int iy = -nb; iy <= nb; iy++)
            for (int ix = -na; ix <= na; ix++) {
                double dx = p.x - ions[4 * j + 0] + ix * ax + iy * bx;
                double dy = p.y - ions[4 * j + 1] + ix * ay + iy * by;
                double dz = p.z - ions[4 * j + 2];
                double r = std::sqrt(dx * dx + dy * dy + dz * dz + 1e-32);
                double e = std::exp(-alpha * (r - R));
                double eM = E * e;
                paul += eM * e;
                lond += -2.0 * eM;
            }
    }
}

// Ewald-2D potential at one point: eval_potential_full, Surface.cl:834-906,
// orthogonal cell (b1 = 2pi/Lx x, b2 = 2pi/Ly y), all G != 0 with |G| <= gcut.
double ewald_point(V3 p, int nions, const double* ions, double Lx, double Ly, double gcut) {
    const double A = Lx * Ly;
    double phi0 = 0;
    for (int i = 0; i < nions; i++) phi0 -= ions[4 * i + 3] * std::fabs(p.z - ions[4 * i + 2]);
    phi0 *= 2.0 * M_PI / A;
    const double g1 = 2.0 * M_PI / Lx, g2 = 2.0 * M_PI / Ly;
    int H = (int)std::floor(gcut / g1), K = (int)std::floor(gcut / g2);
    double phig = 0;
    for (int h = -H; h <= H; h++)
        for (int k = -K; k <= K; k++) {
            if (h == 0 && k == 0) continue;
            double Gx = h * g1, Gy = k * g2, Gn = std::sqrt(Gx * Gx + Gy * Gy);
            if (Gn > gcut) continue;
            double pref = 2.0 * M_PI / (A * Gn);
            for (int i = 0; i < nions; i++) {
                double ph = Gx * (p.x - ions[4 * i + 0]) + Gy * (p.y - ions[4 * i + 1]);
                phig += pref * ions[4 * i + 3] * std::cos(ph) * std::exp(-Gn * std::fabs(p.z - ions[4 * i + 2]));
            }
        }
    return (phi0 + phig) * COULOMB_K;
}

// Direct image sum with a circular cutoff: eval_potential_brute, Surface.cl:911-954.
double brute_coulomb_point(V3 p, int nions, const double* ions, double Lx, double Ly, int nrep) {
    double phi = 0;
    for (int nn = -nrep; nn <= nrep; nn++)
        for (int m = -nrep; m <= nrep; m++) {
            if (nn * nn + m * m > nrep * nrep) continue;
            for (int i = 0; i < nions; i++) {
                double dx = p.x - (ions[4 * i + 0] + nn * Lx), dy = p.y - (ions[4 * i + 1] + m * Ly), dz = p.z - ions[4 * i + 2];
                double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (r > 1e-12) phi += ions[4 * i + 3] / r;
            }
        }
    return phi * COULOMB_K;
}

// Solve the 1-D cubic B-spline interpolation system tridiag(1/6, 2/3, 1/6) c = v
// on a line of n samples with stride st; periodic (cyclic, Sherman-Morrison) or
// open with zero padding (the boundary rule of BsplineConv3D in z,
// gridff_build.cl:36-38).
void solve_line(double* x, int n, size_t st, bool periodic, std::vector<double>& w) {
    const double a = 1.0 / 6.0, b = 2.0 / 3.0;
    if (n == 1) { x[0] /= periodic ? (b + 2 * a) : b; return; }
    w.resize(3 * (size_t)n);
    double* cp = w.data(); double* d = cp + n; double* u = d + n;
    auto thomas = [&](double* rhs, double b0, double bn) {
        // tridiagonal with sub=super=a, diag=b except first (b0) and last (bn)
        double m = b0;
        cp[0] = a / m; rhs[0] /= m;
        for (int i = 1; i < n; i++) {
            double di = (i == n - 1) ? bn : b;
            m = di - a * cp[i - 1];
            cp[i] = a / m;
            rhs[i] = (rhs[i] - a * rhs[i - 1]) / m;
        }
        for (int i = n - 2; i >= 0; i--) rhs[i] -= cp[i] * rhs[i + 1];
    };
    for (int i = 0; i < n; i++) d[i] = x[i * st];
    if (!periodic) {
        thomas(d, b, b);
    } else {
        // A = T' + u v^T with corner terms; gamma = -b (Numerical Recipes cyclic form)
        double gamma = -b;
        for (int i = 0; i < n; i++) u[i] = 0;
        u[0] = gamma; u[n - 1] = a;
        thomas(d, b - gamma, b - a * a / gamma);
        thomas(u, b - gamma, b - a * a / gamma);
        double fact = (d[0] + a * d[n - 1] / gamma) / (1.0 + u[0] + a * u[n - 1] / gamma);
        for (int i = 0; i < n; i++) d[i] -= fact * u[i];
    }
    for (int i = 0; i < n; i++) x[i * st] = d[i];
}

}  // namespace

// ================================================================== C API
extern "C" {

static orc_sys* finish_sys(orc_sys* S, const std::vector<std::string>* types) {
    fill_neighs(*S);
    build_terms(*S);
    bake_slots(*S);
    if (types) setup_params(*S, *types);
    return S;
}

// Molecule -> bonds by cutoff (topology.rs:101-111), neighbours, typing, terms, parameters.
orc_sys* orc_sys_from_molecule(int n, const int* Z, const double* pos, const double* q, double bond_cut) {
    orc_sys* S = new orc_sys();
    S->n = n;
    double rc2 = bond_cut * bond_cut;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1], dz = pos[3 * j + 2] - pos[3 * i + 2];
            if (dx * dx + dy * dy + dz * dz < rc2) S->bonds.push_back({i, j});
        }
    fill_neighs(*S);
    std::vector<std::string> el(n);
    for (int i = 0; i < n; i++) { const Elem* e = elem_by_Z(Z[i]); el[i] = e ? e->name : "X"; }
    std::vector<std::string> T = assign_types(el, S->neighs);
    finish_sys(S, &T);
    if (q) for (int i = 0; i < n; i++) S->req[i][2] = q[i];
    return S;
}

// Periodic molecule: bonds by cutoff to every image within one cell along each nonzero lattice
// vector (lvec = a, b, c; a zero vector is a non-periodic axis), each bond remembering the cell of
// its partner (neighCell).  Terms are enumerated over atom indices, so a cell in which a pair bonds
// in two images, an atom bonds to its own image, or a 3-bond path returns to its first atom
// through the images is too small and is refused (null, message in err).
orc_sys* orc_sys_from_molecule_pbc(int n, const int* Z, const double* pos, const double* q, double bond_cut,
                                   const double* lvec, char* err, int errlen) {
    int range[3];
    for (int k = 0; k < 3; k++) range[k] = (lvec[3 * k] != 0 || lvec[3 * k + 1] != 0 || lvec[3 * k + 2] != 0) ? 1 : 0;
    NBParams L{}; for (int k = 0; k < 9; k++) L.lvec[k] = lvec[k];
    orc_sys* S = new orc_sys();
    S->n = n;
    const double rc2 = bond_cut * bond_cut;
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) {
            int found = 0;
            for (int oz = -range[2]; oz <= range[2]; oz++)
                for (int oy = -range[1]; oy <= range[1]; oy++)
                    for (int ox = -range[0]; ox <= range[0]; ox++) {
                        if (i == j && ox == 0 && oy == 0 && oz == 0) continue;
                        V3 d = V3{pos[3 * j] - pos[3 * i], pos[3 * j + 1] - pos[3 * i + 1], pos[3 * j + 2] - pos[3 * i + 2]} +
                               lattice_shift(L, ox, oy, oz);
                        if (dot(d, d) >= rc2) continue;
                        if (i == j) { std::snprintf(err, errlen, "atom %d bonds to its own image: cell too small", i); delete S; return nullptr; }
                        if (found++) { std::snprintf(err, errlen, "atoms %d and %d bond in two images: cell too small", i, j); delete S; return nullptr; }
                        S->bonds.push_back({i, j});
                        S->bond_off.push_back({ox, oy, oz});
                    }
        }
    fill_neighs(*S);
    S->ngc.assign(n, {0, 0, 0, 0});
    for (int a = 0; a < n; a++)
        for (int s = 0; s < 4; s++) {
            const int ib = S->neighBs[a][s];
            if (ib < 0) continue;
            const auto& o = S->bond_off[ib];
            const int sg = S->bonds[ib][0] == a ? 1 : -1;   // offsets are seen from the bond's first atom
            S->ngc[a][s] = cell_code(sg * o[0], sg * o[1], sg * o[2]);
        }
    // 3-bond paths i-j-k-l with l == i through the images
    for (int j = 0; j < n; j++)
        for (int sj = 0; sj < 4; sj++) {
            const int k = S->neighs[j][sj]; if (k < 0) continue;
            for (int si = 0; si < 4; si++) {
                const int i = S->neighs[j][si]; if (i < 0 || si == sj) continue;
                for (int sk = 0; sk < 4; sk++) {
                    const int l = S->neighs[k][sk]; if (l != i) continue;
                    int c[3];
                    for (int ax = 0; ax < 3; ax++)
                        c[ax] = -cell_field(S->ngc[j][si], ax) + cell_field(S->ngc[j][sj], ax) + cell_field(S->ngc[k][sk], ax);
                    if (c[0] || c[1] || c[2]) { std::snprintf(err, errlen, "bond path %d-%d-%d-%d closes through the images: cell too small", i, j, k, l); delete S; return nullptr; }
                }
            }
        }
    std::vector<std::string> el(n);
    for (int i = 0; i < n; i++) { const Elem* e = elem_by_Z(Z[i]); el[i] = e ? e->name : "X"; }
    std::vector<std::string> T = assign_types(el, S->neighs);
    finish_sys(S, &T);
    if (q) for (int i = 0; i < n; i++) S->req[i][2] = q[i];
    return S;
}

void orc_sys_cells(const orc_sys* S, int* ngc) {
    for (int a = 0; a < S->n; a++) for (int s = 0; s < 4; s++) ngc[4 * a + s] = S->ngc.empty() ? 0 : S->ngc[a][s];
}

// Explicit bonds and parameters (angles/dihedrals/inversions enumerated from the
// bonds with zero parameters unless set later).
orc_sys* orc_sys_from_bonds(int n, int nbonds, const int* bonds, const double* bparams, const double* req) {
    orc_sys* S = new orc_sys();
    S->n = n;
    for (int b = 0; b < nbonds; b++) { S->bonds.push_back({bonds[2 * b], bonds[2 * b + 1]}); S->bparams.push_back({bparams[2 * b], bparams[2 * b + 1]}); }
    finish_sys(S, nullptr);
    S->angp.assign(S->angs.size(), {0, 0, 0, 0, 0});
    S->dihp.assign(S->dihs.size(), {0, 1, 3});
    S->invp.assign(S->invs.size(), {0, 0, 0, 0});
    S->req.resize(n); S->type_id.assign(n, -1);
    for (int i = 0; i < n; i++) for (int c = 0; c < 4; c++) S->req[i][c] = req ? req[4 * i + c] : 0.0;
    return S;
}

void orc_sys_free(orc_sys* S) { delete S; }

void orc_sys_counts(const orc_sys* S, int* c) {
    c[0] = S->n; c[1] = (int)S->bonds.size(); c[2] = (int)S->angs.size(); c[3] = (int)S->dihs.size(); c[4] = (int)S->invs.size();
}

void orc_sys_export(const orc_sys* S, int* neighs, int* neighBs, int* bonds, double* bparams,
                    int* angs, int* ang_ngs, double* angp, int* dihs, int* dih_ngs, double* dihp,
                    int* invs, int* inv_ngs, double* invp, double* req, int* type_id) {
    for (int a = 0; a < S->n; a++) for (int s = 0; s < 4; s++) { neighs[4 * a + s] = S->neighs[a][s]; neighBs[4 * a + s] = S->neighBs[a][s]; }
    for (size_t b = 0; b < S->bonds.size(); b++) { bonds[2 * b] = S->bonds[b][0]; bonds[2 * b + 1] = S->bonds[b][1]; bparams[2 * b] = S->bparams[b][0]; bparams[2 * b + 1] = S->bparams[b][1]; }
    for (size_t t = 0; t < S->angs.size(); t++) { for (int r = 0; r < 3; r++) angs[3 * t + r] = S->angs[t][r]; for (int r = 0; r < 2; r++) ang_ngs[2 * t + r] = S->ang_ngs[t][r]; for (int r = 0; r < 5; r++) angp[5 * t + r] = S->angp[t][r]; }
    for (size_t t = 0; t < S->dihs.size(); t++) { for (int r = 0; r < 4; r++) dihs[4 * t + r] = S->dihs[t][r]; for (int r = 0; r < 3; r++) { dih_ngs[3 * t + r] = S->dih_ngs[t][r]; dihp[3 * t + r] = S->dihp[t][r]; } }
    for (size_t t = 0; t < S->invs.size(); t++) { for (int r = 0; r < 4; r++) { invs[4 * t + r] = S->invs[t][r]; invp[4 * t + r] = S->invp[t][r]; } for (int r = 0; r < 3; r++) inv_ngs[3 * t + r] = S->inv_ngs[t][r]; }
    for (int a = 0; a < S->n; a++) { for (int c = 0; c < 4; c++) req[4 * a + c] = S->req[a][c]; if (type_id) type_id[a] = S->type_id[a]; }
}

// Override term parameters (any pointer may be null).
void orc_sys_set_params(orc_sys* S, const double* angp, const double* dihp, const double* invp) {
    if (angp) for (size_t t = 0; t < S->angs.size(); t++) for (int r = 0; r < 5; r++) S->angp[t][r] = angp[5 * t + r];
    if (dihp) for (size_t t = 0; t < S->dihs.size(); t++) for (int r = 0; r < 3; r++) S->dihp[t][r] = dihp[3 * t + r];
    if (invp) for (size_t t = 0; t < S->invs.size(); t++) for (int r = 0; r < 4; r++) S->invp[t][r] = invp[4 * t + r];
}

const char* orc_type_name(int id) { return (id >= 0 && id < N_ATYPES) ? ATYPES[id].name : "?"; }

// nbp = (rdamp, alpha_morse, rcut (<=0: none), excl13 (0/1), lvec (9: a, b, c), npbc (3))
static NBParams nbp_of(const double* p) {
    NBParams nb{p[0], p[1], p[2], (int)p[3], {}, {}};
    for (int k = 0; k < 9; k++) nb.lvec[k] = p[4 + k];
    for (int k = 0; k < 3; k++) nb.npbc[k] = (int)p[13 + k];
    return nb;
}
// fp = (dt0, dt_max, alpha0, f_inc, f_dec, f_alpha, n_min, fconv, flimit)
static FireParams fp_of(const double* p) { return FireParams{p[0], p[1], p[2], p[3], p[4], p[5], (int)p[6], p[7], p[8]}; }

// Folded-surface energy and (clamped) force of isolated atoms: n x (x, y, z), n x req -> E[n], F[n x 3]
int orc_folded_points(const orc_folded* f, int n, const double* pos, const double* req, double* E, double* F) {
    for (int a = 0; a < n; a++) {
        V3 fo;
        E[a] = folded_atom(*f, req + 4 * a, V3{pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]}, fo);
        F[3 * a] = fo.x; F[3 * a + 1] = fo.y; F[3 * a + 2] = fo.z;
    }
    return 0;
}

// ------------------------------------------------------------------ RAFF multi-replica step (FP64)
// One step per replica as compute_collision_multi, compute_ports_current_multi and
// apply_corrections_multi (opencl/RRsp3.cl:1774-2048, massless_rot = 0), each pass over the
// positions of the step's start.  cfg = (dt, relaxation, momentum_beta, rot_mass_scale).
// Per replica and atom: pos (x, y, z, inverse mass), quat (x, y, z, w), momenta dmom / dqmom (4
// each); coll_out (3 per atom) and dnode_out (3 per node) receive the last step's corrections.
namespace {
struct Q4d { double x, y, z, w; };
inline Q4d qmul(Q4d a, Q4d b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
inline Q4d qnorm(Q4d q) {
    const double n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (n2 < 1e-16) return {0, 0, 0, 1};
    const double s = 1.0 / std::sqrt(n2);
    return {q.x * s, q.y * s, q.z * s, q.w * s};
}
inline V3 qrot(Q4d q, V3 v) {   // v + w t + u x t, t = 2 u x v
    const V3 u{q.x, q.y, q.z};
    const V3 t = cross(u, v) * 2.0;
    return v + t * q.w + cross(u, t);
}
}  // namespace

int orc_raff_step(int n, int nn, int nsys, int nsteps, const double* cfg, int collide, const double* radius, const int* neighs,
                  const int* excl1, const int* excl2, const int* fixmask, const double* port_local, const double* kport,
                  const int* bk, double* pos, double* quat, double* dmom, double* dqmom, double* coll_out, double* dnode_out) {
    const double dt = cfg[0], relax = cfg[1], beta = cfg[2], rms = cfg[3];
    // replicas are independent: one per thread
#pragma omp parallel for schedule(dynamic)
    for (int r = 0; r < nsys; r++) {
        std::vector<V3> C(n), DN(nn), DR(nn), DG(4 * (size_t)nn);
        double* P = pos + 4 * (size_t)r * n; double* Q = quat + 4 * (size_t)r * n;
        double* M = dmom + 4 * (size_t)r * n; double* MQ = dqmom + 4 * (size_t)r * n;
        auto p3 = [&](int i) { return V3{P[4 * i], P[4 * i + 1], P[4 * i + 2]}; };
        for (int it = 0; it < nsteps; it++) {
            for (int i = 0; i < n; i++) {                  // collisions (RRsp3.cl:1776-1832)
                C[i] = {0, 0, 0};
                if (!collide) continue;
                const double invMi = P[4 * i + 3], ri = radius[i];
                if (!(invMi > 1e-12) || !(ri > 0)) continue;
                for (int j = 0; j < n; j++) {
                    if (j == i) continue;
                    bool ex = false;
                    for (int k = 0; k < 4; k++) ex = ex || excl1[4 * i + k] == j || excl2[4 * i + k] == j;
                    if (ex) continue;
                    const double invMj = P[4 * j + 3], rj = radius[j];
                    if (!(invMj > 1e-12) || !(rj > 0)) continue;
                    const V3 d = p3(i) - p3(j);
                    const double d2 = dot(d, d), rs = ri + rj;
                    if (d2 < rs * rs && d2 > 1e-16) {
                        const double dist = std::sqrt(d2);
                        const double dl = 0.5 * (rs - dist) / (invMi + invMj + 1e-12);
                        C[i] = C[i] + d * (dl * invMi / dist);
                    }
                }
            }
            for (int i = 0; i < nn && i < n; i++) {        // ports (RRsp3.cl:1837-1934)
                const double invMi = P[4 * i + 3];
                DN[i] = DR[i] = {0, 0, 0};
                for (int k = 0; k < 4; k++) DG[4 * i + k] = {0, 0, 0};
                if (!(invMi > 1e-12)) continue;
                const Q4d qi{Q[4 * i], Q[4 * i + 1], Q[4 * i + 2], Q[4 * i + 3]};
                const double invI = rms / (0.4 / invMi + 1e-12), dt2 = dt * dt + 1e-16;
                for (int k = 0; k < 4; k++) {
                    const int j = neighs[4 * i + k];
                    if (j < 0 || j >= n) continue;
                    const double K = kport[4 * i + k];
                    if (!(K > 0)) continue;
                    const double invMj = P[4 * j + 3];
                    if (!(invMj > 1e-12)) continue;
                    const double* pl = port_local + 4 * (4 * i + k);
                    const V3 r_arm = qrot(qi, V3{pl[0], pl[1], pl[2]});
                    const V3 diff = p3(j) - (p3(i) + r_arm);
                    const double dist2 = dot(diff, diff);
                    if (dist2 < 1e-16) continue;
                    const double dist = std::sqrt(dist2);
                    const V3 nv = diff * (1.0 / dist);
                    const V3 rxn = cross(r_arm, nv);
                    const double w_ang = dot(rxn, rxn) * invI;
                    const bool jnode = j < nn;
                    double w_total = invMi + invMj + w_ang + 1.0 / (K * dt2) + 1e-12;
                    if (jnode) w_total += w_ang;
                    double imp = dist / w_total;
                    if (jnode) imp *= 0.5;
                    const V3 Pv = nv * imp;
                    DN[i] = DN[i] + Pv * invMi;
                    DR[i] = DR[i] + cross(r_arm, Pv) * invI;
                    DG[4 * i + k] = Pv * (-invMj);
                }
            }
            for (int i = 0; i < n; i++) {                  // corrections (RRsp3.cl:1939-2046)
                if (!(P[4 * i + 3] > 1e-12)) continue;
                const bool isnode = i < nn;
                V3 dx_port{0, 0, 0};
                if (isnode) dx_port = dx_port + DN[i];
                for (int k = 0; k < 4; k++) { const int sl = bk[4 * i + k]; if (sl >= 0) dx_port = dx_port + DG[sl]; }
                V3 dx = C[i] + dx_port;
                const int msk = fixmask ? fixmask[i] : 0;
                if (msk & 1) dx.x = 0;
                if (msk & 2) dx.y = 0;
                if (msk & 4) dx.z = 0;
                V3 move = dx * relax;
                if (beta != 0) move = move + V3{M[4 * i], M[4 * i + 1], M[4 * i + 2]} * beta;
                if (msk & 8) { if (std::fabs(P[4 * i + 2]) > 1e-6) move.z -= P[4 * i + 2]; else move.z = 0; }
                P[4 * i] += move.x; P[4 * i + 1] += move.y; P[4 * i + 2] += move.z;
                M[4 * i] = move.x; M[4 * i + 1] = move.y; M[4 * i + 2] = move.z; M[4 * i + 3] = 0;
                if (!isnode || (msk & 7)) continue;
                const V3 dth = DR[i] * relax;
                const double angle = std::sqrt(dot(dth, dth));
                const Q4d qo{Q[4 * i], Q[4 * i + 1], Q[4 * i + 2], Q[4 * i + 3]};
                Q4d q = qo;
                if (angle > 1e-8) {
                    const double s = std::sin(0.5 * angle), c = std::cos(0.5 * angle);
                    q = qnorm(qmul(Q4d{dth.x / angle * s, dth.y / angle * s, dth.z / angle * s, c}, qo));
                }
                if (beta != 0) q = {q.x + MQ[4 * i] * beta, q.y + MQ[4 * i + 1] * beta, q.z + MQ[4 * i + 2] * beta, q.w + MQ[4 * i + 3] * beta};
                q = qnorm(q);
                if (q.x * qo.x + q.y * qo.y + q.z * qo.z + q.w * qo.w < 0) q = {-q.x, -q.y, -q.z, -q.w};
                Q[4 * i] = q.x; Q[4 * i + 1] = q.y; Q[4 * i + 2] = q.z; Q[4 * i + 3] = q.w;
                MQ[4 * i] = q.x - qo.x; MQ[4 * i + 1] = q.y - qo.y; MQ[4 * i + 2] = q.z - qo.z; MQ[4 * i + 3] = q.w - qo.w;
            }
        }
        if (nsteps > 0) {
            if (coll_out) for (int i = 0; i < n; i++) { coll_out[3 * ((size_t)r * n + i)] = C[i].x; coll_out[3 * ((size_t)r * n + i) + 1] = C[i].y; coll_out[3 * ((size_t)r * n + i) + 2] = C[i].z; }
            if (dnode_out) for (int i = 0; i < nn; i++) { dnode_out[3 * ((size_t)r * nn + i)] = DN[i].x; dnode_out[3 * ((size_t)r * nn + i) + 1] = DN[i].y; dnode_out[3 * ((size_t)r * nn + i) + 2] = DN[i].z; }
        }
    }
    return 0;
}

int orc_eval(const orc_sys* S, const double* pos, const orc_grid* g, const double* nbp, double* F, double* Ea, double* Ec) {
    std::vector<V3> P(S->n), FF(S->n);
    for (int a = 0; a < S->n; a++) P[a] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    eval_forces(*S, P.data(), g, nbp_of(nbp), FF.data(), Ea, Ec);
    for (int a = 0; a < S->n; a++) { F[3 * a] = FF[a].x; F[3 * a + 1] = FF[a].y; F[3 * a + 2] = FF[a].z; }
    return 0;
}

int orc_relax(const orc_sys* S, double* pos, const orc_grid* g, const double* nbp, const double* fp, int max_steps,
              double* F, double* Ea, double* Ec, double* fmax, int* conv) {
    std::vector<V3> P(S->n), FF(S->n);
    for (int a = 0; a < S->n; a++) P[a] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    int steps = relax_fire(*S, P.data(), g, nbp_of(nbp), fp_of(fp), max_steps, FF.data(), Ea, Ec, fmax, conv);
    for (int a = 0; a < S->n; a++) { pos[3 * a] = P[a].x; pos[3 * a + 1] = P[a].y; pos[3 * a + 2] = P[a].z; if (F) { F[3 * a] = FF[a].x; F[3 * a + 1] = FF[a].y; F[3 * a + 2] = FF[a].z; } }
    return steps;
}

// orc_relax with the driving terms of updateAtomsMMFFf4: cons (n x 7, or null) and td (4, or null)
int orc_relax_drive(const orc_sys* S, double* pos, const orc_grid* g, const double* nbp, const double* fp, int max_steps,
                    const double* cons, const double* td, double* F, double* Ea, double* Ec, double* fmax, int* conv) {
    std::vector<V3> P(S->n), FF(S->n);
    for (int a = 0; a < S->n; a++) P[a] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    Drive dr; dr.cons = cons; dr.td = td;
    int steps = relax_fire(*S, P.data(), g, nbp_of(nbp), fp_of(fp), max_steps, FF.data(), Ea, Ec, fmax, conv, dr);
    for (int a = 0; a < S->n; a++) { pos[3 * a] = P[a].x; pos[3 * a + 1] = P[a].y; pos[3 * a + 2] = P[a].z; if (F) { F[3 * a] = FF[a].x; F[3 * a + 1] = FF[a].y; F[3 * a + 2] = FF[a].z; } }
    return steps;
}

// the thermal drive's pseudo-random vectors of atoms 0..n-1 at one seed (n x 3)
int orc_langevin_noise(int n, float seed, double* out) {
    for (int a = 0; a < n; a++) { V3 r = langevin_noise(a, seed); out[3 * a] = r.x; out[3 * a + 1] = r.y; out[3 * a + 2] = r.z; }
    return 0;
}

// CPU baseline: independent systems relaxed in parallel, one system per thread.
int orc_relax_batch(int nsys, const orc_sys* const* S, double* const* pos, const orc_grid* g, const double* nbp,
                    const double* fp, int max_steps, int* steps, double* fmax, int* conv, double* Etot, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int s = 0; s < nsys; s++) {
        int n = S[s]->n;
        std::vector<double> F(3 * (size_t)n), Ea(n), Ec(E_NCOMP);
        steps[s] = orc_relax(S[s], pos[s], g, nbp, fp, max_steps, F.data(), Ea.data(), Ec.data(), &fmax[s], &conv[s]);
        Etot[s] = Ec[E_TOT];
    }
    return 0;
}

// getLJQH (UFF.cl:82-95) on n pairs: dp (n x 3), mixed REQij (n x 4: R0, E0, Q, H) -> (fx, fy, fz, E)
void orc_ljqh_pairs(int n, const double* dp, const double* reqij, double R2damp, double* out) {
    for (int i = 0; i < n; i++) {
        V3 f;
        const double E = getLJQH(V3{dp[3 * i], dp[3 * i + 1], dp[3 * i + 2]}, reqij[4 * i], reqij[4 * i + 1], reqij[4 * i + 2],
                                 R2damp, f);
        out[4 * i] = f.x; out[4 * i + 1] = f.y; out[4 * i + 2] = f.z; out[4 * i + 3] = E;
    }
}

// fe3d_pbc_comb (UFF.cl:1459-1511) at np points u (grid units, np x 3) with prefactors PLQH (np x 4):
// (dE/du_x, dE/du_y, dE/du_z, E) per point
void orc_sample_points(const orc_grid* g, int np, const double* u, const double* plqh, double* out) {
    for (int i = 0; i < np; i++) sample_grid(*g, plqh + 4 * i, V3{u[3 * i], u[3 * i + 1], u[3 * i + 2]}, out + 4 * i);
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_morse_points(int np, const double* pts, int nions, const double* ions, const double* re,
                      const double* cell /*ax,ay,bx,by*/, int na, int nb, double alpha, double* out) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 0; i < np; i++) {
        double P_, L_;
        morse_point(V3{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}, nions, ions, re, cell[0], cell[1], cell[2], cell[3], na, nb, alpha, P_, L_);
        out[2 * i] = P_; out[2 * i + 1] = L_;
    }
}

void orc_ewald_points(int np, const double* pts, int nions, const double* ions, double Lx, double Ly, double gcut, double* out) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 0; i < np; i++) out[i] = ewald_point(V3{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}, nions, ions, Lx, Ly, gcut);
}

void orc_brute_coulomb_points(int np, const double* pts, int nions, const double* ions, double Lx, double Ly, int nrep, double* out) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 0; i < np; i++) out[i] = brute_coulomb_point(V3{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}, nions, ions, Lx, Ly, nrep);
}

// Exact cubic B-spline coefficients of one scalar channel, z-fastest layout
// i = iz + nz*(iy + ny*ix): periodic in x,y, zero-padded in z.
void orc_bspline_fit(int nx, int ny, int nz, const double* v, double* c) {
    size_t N = (size_t)nx * ny * nz;
    std::memcpy(c, v, N * sizeof(double));
    std::vector<double> w;
    for (int ix = 0; ix < nx; ix++) for (int iy = 0; iy < ny; iy++) solve_line(c + (size_t)nz * (iy + (size_t)ny * ix), nz, 1, false, w);
    for (int ix = 0; ix < nx; ix++) for (int iz = 0; iz < nz; iz++) solve_line(c + iz + (size_t)nz * ny * ix, ny, nz, true, w);
    for (int iy = 0; iy < ny; iy++) for (int iz = 0; iz < nz; iz++) solve_line(c + iz + (size_t)nz * iy, nx, (size_t)nz * ny, true, w);
}

// Forward operator: BsplineConv3D (gridff_build.cl:8-61), z-fastest layout.
void orc_bspline_conv(int nx, int ny, int nz, const double* c, double* v) {
    const double B0 = 2.0 / 3.0, B1 = 1.0 / 6.0;
    const double w[3] = {B1, B0, B1};
    for (int ix = 0; ix < nx; ix++) for (int iy = 0; iy < ny; iy++) for (int iz = 0; iz < nz; iz++) {
        double s = 0;
        for (int a = -1; a <= 1; a++) for (int b = -1; b <= 1; b++) for (int k = -1; k <= 1; k++) {
            int z = iz + k; if (z < 0 || z >= nz) continue;
            int x = modulo(ix + a, nx), y = modulo(iy + b, ny);
            s += w[a + 1] * w[b + 1] * w[k + 1] * c[z + (size_t)nz * (y + (size_t)ny * x)];
        }
        v[iz + (size_t)nz * (iy + (size_t)ny * ix)] = s;
    }
}

// Whole substrate grid in FP64: node values (Pauli, London from Morse image sums,
// Coulomb from Ewald-2D), exact B-spline fit per channel, packed (P, L, Q, 0)
// z-fastest.  values (optional) receives the node values in the same layout.
int orc_build_grid(int nions, const double* ions, const double* re, double Lx, double Ly,
                   int nx, int ny, int nz, const double* p0, const double* step, double alpha, int npbc, double gcut,
                   double* coef, double* values) {
    size_t N = (size_t)nx * ny * nz;
    std::vector<double> ch(3 * N);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int ix = 0; ix < nx; ix++)
        for (int iy = 0; iy < ny; iy++)
            for (int iz = 0; iz < nz; iz++) {
                V3 p{p0[0] + ix * step[0], p0[1] + iy * step[1], p0[2] + iz * step[2]};
                size_t i = iz + (size_t)nz * (iy + (size_t)ny * ix);
                double P_, L_;
                morse_point(p, nions, ions, re, Lx, 0.0, 0.0, Ly, npbc, npbc, alpha, P_, L_);
                ch[i] = P_; ch[N + i] = L_;
                ch[2 * N + i] = ewald_point(p, nions, ions, Lx, Ly, gcut);
            }
    std::vector<double> cf(N);
    for (int c = 0; c < 3; c++) {
        orc_bspline_fit(nx, ny, nz, ch.data() + c * N, cf.data());
        for (size_t i = 0; i < N; i++) { coef[4 * i + c] = cf[i]; if (values) values[4 * i + c] = ch[c * N + i]; }
    }
    for (size_t i = 0; i < N; i++) { coef[4 * i + 3] = 0.0; if (values) values[4 * i + 3] = 0.0; }
    return 0;
}

// Direct substrate energy/force on one probe atom (no grid): Morse image sum with the
// atom's PLQH prefactors plus Q*phi from Ewald-2D; force by central differences.
void orc_substrate_direct(int np, const double* pts, const double* req_atom /*np*4*/, int nions, const double* ions,
                          const double* re, double Lx, double Ly, int npbc, double alpha, double gcut, double h, double* out /*np*4*/) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 0; i < np; i++) {
        const double* r = req_atom + 4 * i;
        double ej = std::exp(alpha * r[0]);
        double pl[3] = {ej * ej * r[1], ej * r[1], r[2]};
        auto E = [&](V3 p) {
            double P_, L_;
            morse_point(p, nions, ions, re, Lx, 0.0, 0.0, Ly, npbc, npbc, alpha, P_, L_);
            return pl[0] * P_ + pl[1] * L_ + pl[2] * ewald_point(p, nions, ions, Lx, Ly, gcut);
        };
        V3 p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
        out[4 * i + 3] = E(p);
        V3 d[3] = {{h, 0, 0}, {0, h, 0}, {0, 0, h}};
        for (int k = 0; k < 3; k++) out[4 * i + k] = -(E(p + d[k]) - E(p - d[k])) / (2 * h);
    }
}

// Same grid as orc_build_grid for a slab entirely below the grid, with the Ewald-2D
// reciprocal sum evaluated plane by plane as a separable partial DFT (structure factors
// S_G = sum_i q_i exp(-iG.rho_i) exp(-|G|(z0 - z_i)), pruned below gtol of the largest
// amplitude).  Same formula as ewald_point, evaluated faster; used to build full-size
// grids for the CPU baseline.
int orc_build_grid_fast(int nions, const double* ions, const double* re, double Lx, double Ly,
                        int nx, int ny, int nz, const double* p0, const double* step, double alpha, int npbc, double gtol,
                        double* coef, double morse_rcut) {
    // Same values as orc_build_grid (make_MorseFF image sums, Ewald-2D, exact fit), evaluated
    // faster: Morse over per-column lists of the ion images (with morse_rcut > 0 only those
    // within morse_rcut of the column's points; 0 keeps every image, as make_MorseFF does), and
    // the reciprocal sum from separable x / y phase tables, G terms below gtol of the largest
    // amplitude at a plane skipped (their sum is below gtol relative).
    const size_t N = (size_t)nx * ny * nz;
    double ztop = -1e300, zlow = 1e300, qsum = 0, qz = 0;
    for (int i = 0; i < nions; i++) {
        ztop = std::max(ztop, ions[4 * i + 2]); zlow = std::min(zlow, ions[4 * i + 2]);
        qsum += ions[4 * i + 3]; qz += ions[4 * i + 3] * ions[4 * i + 2];
    }
    const double dmin = p0[2] - ztop;
    if (!(dmin > 0)) return -1;
    std::vector<double> ch(3 * N);
    // ion images (position, R, E) in the make_MorseFF image order
    struct Img { double x, y, z, R, E; };
    std::vector<Img> imgs;
    for (int j = 0; j < nions; j++)
        for (int iy = -npbc; iy <= npbc; iy++)
            for (int ix = -npbc; ix <= npbc; ix++)
                imgs.push_back({ions[4 * j] - ix * Lx, ions[4 * j + 1] - iy * Ly, ions[4 * j + 2], re[4 * j], re[4 * j + 1]});
    const double zmax = p0[2] + (nz - 1) * step[2];
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int ix = 0; ix < nx; ix++) {
        std::vector<const Img*> col;
        for (int iy = 0; iy < ny; iy++) {
            const double x = p0[0] + ix * step[0], y = p0[1] + iy * step[1];
            col.clear();
            for (const Img& m : imgs) {
                if (morse_rcut > 0) {
                    const double dx = x - m.x, dy = y - m.y;
                    // nearest z of the column to this ion (the column spans [p0z, zmax], ions lie below)
                    const double dz = std::max(0.0, std::min(std::fabs(p0[2] - m.z), std::fabs(zmax - m.z)));
                    if (dx * dx + dy * dy + dz * dz > morse_rcut * morse_rcut) continue;
                }
                col.push_back(&m);
            }
            for (int iz = 0; iz < nz; iz++) {
                const double z = p0[2] + iz * step[2];
                double P_ = 0, L_ = 0;
                for (const Img* m : col) {
                    const double dx = x - m->x, dy = y - m->y, dz = z - m->z;
                    const double r = std::sqrt(dx * dx + dy * dy + dz * dz + 1e-32);
                    const double e = std::exp(-alpha * (r - m->R)), eM = m->E * e;
                    P_ += eM * e;
                    L_ += -2.0 * eM;
                }
                const size_t i = iz + (size_t)nz * (iy + (size_t)ny * ix);
                ch[i] = P_; ch[N + i] = L_;
            }
        }
    }
    (void)zlow;
    const double g1 = 2 * M_PI / Lx, g2 = 2 * M_PI / Ly, A = Lx * Ly;
    const double gmax = -std::log(gtol) / dmin;
    const int H = (int)std::floor(gmax / g1), K = (int)std::floor(gmax / g2);
    struct GT { int h, k; double G, ar, ai; };
    std::vector<GT> gs;
    double amax = 0;
    for (int h = -H; h <= H; h++)
        for (int k = -K; k <= K; k++) {
            if (!h && !k) continue;
            double Gx = h * g1, Gy = k * g2, G = std::sqrt(Gx * Gx + Gy * Gy);
            if (G > gmax) continue;
            double sr = 0, si = 0;
            for (int i = 0; i < nions; i++) {
                double ph = -(Gx * ions[4 * i] + Gy * ions[4 * i + 1]);
                double w = ions[4 * i + 3] * std::exp(-G * (p0[2] - ions[4 * i + 2]));
                sr += w * std::cos(ph); si += w * std::sin(ph);
            }
            double pref = 2 * M_PI / (A * G);
            gs.push_back({h, k, G, sr * pref, si * pref});
            amax = std::max(amax, (std::fabs(sr) + std::fabs(si)) * pref);
        }
    std::vector<GT> act;
    for (auto& g : gs) if ((std::fabs(g.ar) + std::fabs(g.ai)) >= gtol * amax) act.push_back(g);
    // phase tables: e^{i h g1 x_ix} and e^{i k g2 y_iy}
    std::vector<double> cxh((size_t)(2 * H + 1) * nx), sxh(cxh.size()), cyk((size_t)(2 * K + 1) * ny), syk(cyk.size());
    for (int h = -H; h <= H; h++)
        for (int ix = 0; ix < nx; ix++) {
            const double ph = h * g1 * (p0[0] + ix * step[0]);
            cxh[(size_t)(h + H) * nx + ix] = std::cos(ph); sxh[(size_t)(h + H) * nx + ix] = std::sin(ph);
        }
    for (int k = -K; k <= K; k++)
        for (int iy = 0; iy < ny; iy++) {
            const double ph = k * g2 * (p0[1] + iy * step[1]);
            cyk[(size_t)(k + K) * ny + iy] = std::cos(ph); syk[(size_t)(k + K) * ny + iy] = std::sin(ph);
        }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int iz = 0; iz < nz; iz++) {
        const double z = p0[2] + iz * step[2], dz = iz * step[2];
        const double phi0 = -(2 * M_PI / A) * (qsum * z - qz);
        struct PG { const double *cx, *sx, *cy, *sy; double br, bi; };
        std::vector<PG> pl;
        for (auto& g : act) {
            const double d = std::exp(-g.G * dz);
            if ((std::fabs(g.ar) + std::fabs(g.ai)) * d < gtol * amax) continue;
            pl.push_back({&cxh[(size_t)(g.h + H) * nx], &sxh[(size_t)(g.h + H) * nx], &cyk[(size_t)(g.k + K) * ny],
                          &syk[(size_t)(g.k + K) * ny], d * g.ar, d * g.ai});
        }
        for (int ix = 0; ix < nx; ix++)
            for (int iy = 0; iy < ny; iy++) {
                double acc = 0;
                for (const PG& q : pl) {
                    // Re[(br + i bi) e^{i(phx + phy)}]
                    const double c = q.cx[ix] * q.cy[iy] - q.sx[ix] * q.sy[iy];
                    const double s = q.sx[ix] * q.cy[iy] + q.cx[ix] * q.sy[iy];
                    acc += q.br * c - q.bi * s;
                }
                ch[2 * N + iz + (size_t)nz * (iy + (size_t)ny * ix)] = COULOMB_K * (phi0 + acc);
            }
    }
    std::vector<double> cf(N);
    for (int c = 0; c < 3; c++) {
        orc_bspline_fit(nx, ny, nz, ch.data() + c * N, cf.data());
        for (size_t i = 0; i < N; i++) coef[4 * i + c] = cf[i];
    }
    for (size_t i = 0; i < N; i++) coef[4 * i + 3] = 0.0;
    return 0;
}

}  // extern "C"
