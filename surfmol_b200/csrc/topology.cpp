// topology.cpp -- host-side molecule preparation: bonds by cutoff, neighbour slots,
// UFF typing, bonded terms and their parameters, and the packing of terms into
// conflict-free rounds for the device.
//
// Semantics follow the reference's CPU input pipeline:
//   bonds by cutoff ............. crates/libs/moltopo/src/topology.rs:101-111
//   neighbour / bond slots ...... crates/libs/moltopo/src/molecular.rs:34-79
//   angles / dihedrals / invs ... topology.rs:113-182 (dihedrals sorted: the reference
//                                 collects them through a HashSet, i.e. in no fixed order)
//   hybridisation + typing ...... topology.rs:7-35, crates/libs/moltopo/src/assign_uff.rs:8-125
//   UFF parameters .............. crates/libs/molff/src/uff.rs:699-887, moltopo/src/params.rs:595-657
//   term neighbour slots ........ uff.rs:250-315
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "smr_internal.h"

namespace smr {
namespace {

constexpr double kUFF = 28.7989689090648;                       // kcal/mol bond/angle prefactor in eV units
constexpr double kKcal = 4.1840 / 60.2214076 / 1.602176634;     // 1 kcal/mol in eV
constexpr double kDeg = 3.14159265358979323846 / 180.0;

// Element and UFF atom-type parameters: the rows of the reference's
// data/ElementTypes.dat and data/AtomTypes.dat that the typing rules can produce.
enum El { EL_H, EL_C, EL_N, EL_O, EL_F, EL_SI, EL_P, EL_S, EL_CL, EL_NA, EL_X };
struct ElemRow { int Z; const char* sym; int lone_pairs; double rvdw, evdw, quff, uuff, vuff, eaff; bool known; };
const ElemRow kElem[] = {
    {1, "H", 0, 1.4430, 0.00190802059, 0.712, 0.0, 0.0, -4.528, true},
    {6, "C", 0, 1.9255, 0.00455323095, 1.912, 0.08672820848, 0.09188853689, -5.343, true},
    {7, "N", 1, 1.8300, 0.00299212319, 2.544, 0.08672820848, 0.01951384691, -6.899, true},
    {8, "O", 2, 1.7500, 0.00260184625, 2.300, 0.08672820848, 0.00078055388, -8.741, true},
    {9, "F", 3, 0, 0, 0, 0, 0, 0, false},
    {14, "Si", 0, 0, 0, 0, 0, 0, 0, false},
    {15, "P", 1, 0, 0, 0, 0, 0, 0, false},
    {16, "S", 2, 0, 0, 0, 0, 0, 0, false},
    {17, "Cl", 3, 1.9735, 0.00984365166, 2.348, 0.05420513030, 0.0, -8.564, true},
    {11, "Na", 0, 1.4915, 0.00130092313, 1.081, 0.05420513030, 0.0, -2.843, true},
};
struct TypeRow { const char* name; El el; char hyb; double ruff, rvdw, evdw, qbase, hb, ass; };
// ass is 0 for H_ (its row has fewer than 19 columns and the reference parser leaves it unset)
const TypeRow kType[] = {
    {"H_", EL_H, '3', 0.354, 1.4430, 0.00190802059, 0.0, 0.0, 0.0},
    {"C_3", EL_C, '3', 0.757, 1.9255, 0.00455323095, 0.0, 0.0, 109.47},
    {"C_R", EL_C, 'R', 0.729, 1.9255, 0.00455323095, 0.0, 0.0, 120.0},
    {"C_2", EL_C, '2', 0.732, 1.9255, 0.00455323095, 0.0, 0.0, 120.0},
    {"C_1", EL_C, '1', 0.706, 1.9255, 0.00455323095, 0.0, 0.0, 180.0},
    {"N_3", EL_N, '3', 0.700, 1.8300, 0.00299212319, 0.0, -0.9, 106.7},
    {"N_R", EL_N, 'R', 0.699, 1.8300, 0.00299212319, 0.0, 0.9, 120.0},
    {"N_2", EL_N, '2', 0.685, 1.8300, 0.00299212319, 0.0, -0.9, 111.2},
    {"N_1", EL_N, '1', 0.656, 1.8300, 0.00299212319, 0.0, 0.0, 180.0},
    {"O_3", EL_O, '3', 0.658, 1.7500, 0.00260184625, 0.0, -0.95, 104.51},
    {"O_R", EL_O, 'R', 0.680, 1.7500, 0.00260184625, 0.0, -0.95, 110.0},
    {"O_2", EL_O, '2', 0.634, 1.7500, 0.00260184625, 0.0, -0.95, 120.0},
    {"O_1", EL_O, '1', 0.639, 1.7500, 0.00260184625, 0.0, 0.0, 180.0},
    {"Na", EL_NA, '3', 1.539, 1.4915, 0.00130092313, 0.0, 0.0, 0.0},
    {"Cl", EL_CL, '3', 1.044, 1.9735, 0.00984365166, 0.0, 0.0, 0.0},
};
constexpr int kNType = sizeof(kType) / sizeof(kType[0]);
enum { T_H = 0, T_C3, T_CR, T_C2, T_C1, T_N3, T_NR, T_N2, T_N1, T_O3, T_OR, T_O2, T_O1, T_NA, T_CL };

El el_of_Z(int Z) {
    for (int e = 0; e < EL_X; e++) if (kElem[e].Z == Z) return (El)e;
    return EL_X;
}

// hybridisation from the octet rule: npi = 4 - lone_pairs - n_sigma (3 = sp3, 2 = sp2, 1 = sp)
int hybrid(El e, int nn) {
    if (e == EL_H) return 1;
    int npi = 4 - kElem[e].lone_pairs - nn;
    if (npi < 0) return 1;
    return npi == 0 ? 3 : (npi == 1 ? 2 : 1);
}

// type by element and hybridisation suffix; -1 when the reference has no such type
int type_of(El e, char suf) {
    for (int t = 0; t < kNType; t++)
        if (kType[t].el == e && kType[t].hyb == suf && kType[t].name[0] != 0 && std::strchr(kType[t].name, '_')) return t;
    return -1;
}

double bond_order(int ta, int tb) {
    char a = kType[ta].hyb, b = kType[tb].hyb;
    bool sp1a = std::strchr(kType[ta].name, '_') && a == '1', sp1b = std::strchr(kType[tb].name, '_') && b == '1';
    if (sp1a || sp1b) return 3.0;
    if (a == '2' && b == '2') return 2.0;
    return 1.0;
}

double rest_length(int ta, int tb, double bo) {
    const TypeRow &A = kType[ta], &B = kType[tb];
    const ElemRow &ea = kElem[A.el], &eb = kElem[B.el];
    double r = A.ruff + B.ruff - 0.1332 * (A.ruff + B.ruff) * std::log(bo);
    if (ea.eaff < 0.0 && eb.eaff < 0.0) {
        double d = std::sqrt(-ea.eaff) - std::sqrt(-eb.eaff);
        r -= A.ruff * B.ruff * d * d / (-ea.eaff * A.ruff - eb.eaff * B.ruff);
    }
    return r;
}

// "hybridisation suffix" of a type name as the reference reads it: the character after
// the last '_' if any, else '3' (so "Na", "Cl" and "H_" all read as '3').
char suffix_of(int t) {
    const char* s = std::strrchr(kType[t].name, '_');
    return (s && s[1]) ? s[1] : '3';
}

void assign_types(int n, const std::vector<El>& el, const std::vector<int>& ng, std::vector<int>& type) {
    type.assign(n, -1);
    for (int a = 0; a < n; a++) {
        if (type[a] >= 0) continue;
        int nb = 0;
        while (nb < 4 && ng[4 * a + nb] >= 0) nb++;
        El e = el[a];
        if (e == EL_H) { type[a] = T_H; continue; }
        if (e == EL_N && nb == 3) {
            int no = 0;
            for (int s = 0; s < 3; s++) if (ng[4 * a + s] >= 0 && el[ng[4 * a + s]] == EL_O) no++;
            if (no == 2) {
                type[a] = T_NR;
                for (int s = 0; s < 3; s++) if (ng[4 * a + s] >= 0 && el[ng[4 * a + s]] == EL_O) type[ng[4 * a + s]] = T_OR;
                continue;
            }
        }
        if (e == EL_O && nb == 1) { type[a] = T_O2; continue; }
        if (e == EL_C && nb == 2) { type[a] = T_C1; continue; }
        int h = hybrid(e, nb);
        char suf = h == 3 ? '3' : (h == 2 ? ((e == EL_C || e == EL_N || e == EL_O) ? 'R' : '2') : '1');
        int t = type_of(e, suf);
        if (t < 0)   // no "<El>_<suffix>" type: the atom keeps its element symbol as type name (Na, Cl)
            for (int k = 0; k < kNType; k++) if (std::strcmp(kType[k].name, kElem[e].sym) == 0) { t = k; break; }
        type[a] = t;
    }
}

void neighbour_slots(HostTopo& T) {
    int n = T.n;
    T.neighs.assign(4 * n, -1);
    T.neighBs.assign(4 * n, -1);
    for (size_t b = 0; b < T.bonds.size() / 2; b++) {
        int i = T.bonds[2 * b], j = T.bonds[2 * b + 1];
        for (int s = 0; s < 4; s++) if (T.neighs[4 * i + s] < 0) { T.neighs[4 * i + s] = j; T.neighBs[4 * i + s] = (int)b; break; }
        for (int s = 0; s < 4; s++) if (T.neighs[4 * j + s] < 0) { T.neighs[4 * j + s] = i; T.neighBs[4 * j + s] = (int)b; break; }
    }
}

int slot_of(const HostTopo& T, int a, int target, int nslots) {
    for (int s = 0; s < nslots; s++) {
        int g = T.neighs[4 * a + s];
        if (g < 0 && nslots == 4) break;
        if (g == target) return 4 * a + s;
    }
    return -1;
}

void enumerate_terms(HostTopo& T) {
    int n = T.n;
    std::vector<std::vector<int>> adj(n);
    for (size_t b = 0; b < T.bonds.size() / 2; b++) { adj[T.bonds[2 * b]].push_back(T.bonds[2 * b + 1]); adj[T.bonds[2 * b + 1]].push_back(T.bonds[2 * b]); }
    T.angs.clear(); T.ang_ngs.clear();
    for (int j = 0; j < n; j++)
        for (size_t p = 0; p < adj[j].size(); p++)
            for (size_t q = p + 1; q < adj[j].size(); q++) {
                int i = adj[j][p], k = adj[j][q];
                T.angs.insert(T.angs.end(), {i, j, k});
                T.ang_ngs.insert(T.ang_ngs.end(), {slot_of(T, j, i, 4), slot_of(T, j, k, 4)});
            }
    std::vector<std::array<int, 4>> d;
    for (int j = 0; j < n; j++)
        for (int k : adj[j])
            for (int i : adj[j]) {
                if (i == k) continue;
                for (int l : adj[k]) if (l != j && l > i) d.push_back({i, j, k, l});
            }
    std::sort(d.begin(), d.end());
    d.erase(std::unique(d.begin(), d.end()), d.end());
    T.dihs.clear(); T.dih_ngs.clear(); T.dih_kj.clear();
    for (auto& q : d) {
        T.dihs.insert(T.dihs.end(), q.begin(), q.end());
        T.dih_ngs.insert(T.dih_ngs.end(), {slot_of(T, q[1], q[0], 4), slot_of(T, q[1], q[2], 4), slot_of(T, q[2], q[3], 4)});
        T.dih_kj.push_back(slot_of(T, q[2], q[1], 4));
    }
    T.invs.clear(); T.inv_ngs.clear();
    for (int i = 0; i < n; i++) {
        if (adj[i].size() != 3) continue;
        const auto& s = adj[i];
        const int perm[3][3] = {{0, 1, 2}, {2, 0, 1}, {1, 2, 0}};
        for (auto& p : perm) {
            int j = s[p[0]], k = s[p[1]], l = s[p[2]];
            T.invs.insert(T.invs.end(), {i, j, k, l});
            T.inv_ngs.insert(T.inv_ngs.end(), {slot_of(T, i, j, 3), slot_of(T, i, k, 3), slot_of(T, i, l, 3)});
        }
    }
}

void uff_parameters(HostTopo& T) {
    const std::vector<int>& ty = T.type_id;
    auto nnb = [&](int a) { int c = 0; while (c < 4 && T.neighs[4 * a + c] >= 0) c++; return (double)c; };
    auto is_h = [&](int t) { return t < 0 || kType[t].el == EL_H; };
    size_t nb = T.bonds.size() / 2;
    T.bparams.assign(2 * nb, 0.0);
    for (size_t b = 0; b < nb; b++) {
        int ta = ty[T.bonds[2 * b]], tb = ty[T.bonds[2 * b + 1]];
        if (ta < 0 || tb < 0) { T.bparams[2 * b] = 100.0; T.bparams[2 * b + 1] = 1.5; continue; }
        double l0 = rest_length(ta, tb, bond_order(ta, tb));
        T.bparams[2 * b] = 0.5 * kUFF * kElem[kType[ta].el].quff * kElem[kType[tb].el].quff / (l0 * l0 * l0);
        T.bparams[2 * b + 1] = l0;
    }
    size_t na = T.angs.size() / 3;
    T.angp.assign(5 * na, 0.0);
    for (size_t a = 0; a < na; a++) {
        int ti = ty[T.angs[3 * a]], tj = ty[T.angs[3 * a + 1]], tk = ty[T.angs[3 * a + 2]];
        if (is_h(tj) || ti < 0 || tk < 0) continue;
        double th = kType[tj].ass * kDeg, ct = std::cos(th), st = std::sin(th), st2 = st * st;
        double rij = rest_length(ti, tj, bond_order(ti, tj)), rjk = rest_length(tj, tk, bond_order(tj, tk));
        double rik = std::sqrt(rij * rij + rjk * rjk - 2.0 * rij * rjk * ct);
        double kap = kUFF * kElem[kType[ti].el].quff * kElem[kType[tk].el].quff / std::pow(rik, 5) * (3.0 * rij * rjk * st2 - rik * rik * ct);
        double* p = &T.angp[5 * a];
        switch (suffix_of(tj)) {
            case '1': p[0] = kap; p[1] = 1; p[2] = 1; p[3] = 0; p[4] = 0; break;
            case '2': case 'R': p[0] = kap / 9.0; p[1] = 1; p[2] = 0; p[3] = 0; p[4] = -1; break;
            case '3': { double c2 = 1.0 / (4.0 * st2); p[0] = kap; p[1] = c2 * (2.0 * ct * ct + 1.0); p[2] = -4.0 * c2 * ct; p[3] = c2; p[4] = 0; break; }
            default: p[0] = kap; p[1] = 1; p[2] = 0; p[3] = 0; p[4] = -1;
        }
    }
    size_t nd = T.dihs.size() / 4;
    T.dihp.assign(3 * nd, 0.0);
    for (size_t d = 0; d < nd; d++) {
        int j = T.dihs[4 * d + 1], k = T.dihs[4 * d + 2];
        int tj = ty[j], tk = ty[k];
        double* p = &T.dihp[3 * d];
        p[0] = 0; p[1] = 1; p[2] = 3;
        if (is_h(tj) || is_h(tk)) continue;
        char hj = suffix_of(tj), hk = suffix_of(tk);
        if (hj == '1' || hk == '1') continue;
        bool s3j = hj == '3', s3k = hk == '3';
        bool s2j = hj == '2' || hj == 'R', s2k = hk == '2' || hk == 'R';
        const ElemRow &ej = kElem[kType[tj].el], &ek = kElem[kType[tk].el];
        double lnbo = std::log(bond_order(tj, tk));
        double V = 0, dd = 1, nn = 3;
        auto group16 = [&](int t) { return kType[t].el == EL_O || kType[t].el == EL_S; };
        if (s3j && s3k) {
            if (group16(tj) && group16(tk)) {
                double kk = kKcal * (kType[tj].el == EL_O ? 2.0 : 6.8) * (kType[tk].el == EL_O ? 2.0 : 6.8);
                V = std::sqrt(kk); dd = 1; nn = 2;
            } else { V = std::sqrt(ej.vuff * ek.vuff); dd = 1; nn = 3; }
        } else if ((s3j && s2k) || (s2j && s3k)) {
            V = kKcal; dd = -1; nn = 6;
            int sp3 = s3j ? j : k, sp2 = s3j ? k : j;
            if (group16(ty[sp3])) { V = 5.0 * std::sqrt(ej.uuff * ek.uuff) * (1.0 + 4.18 * lnbo); dd = 1; nn = 2; }
            for (int s = 0; s < 4; s++) {
                int g = T.neighs[4 * sp2 + s];
                if (g < 0) break;
                if (g == sp3) continue;
                char hg = suffix_of(ty[g]);
                if (hg == '2' || hg == 'R') { V = 2.0 * kKcal; dd = 1; nn = 3; break; }
            }
        } else if (s2j && s2k) {
            V = 5.0 * std::sqrt(ej.uuff * ek.uuff) * (1.0 + 4.18 * lnbo); dd = -1; nn = 2;
        }
        double den = 0.5 * (nnb(j) - 1.0) * (nnb(k) - 1.0);
        p[0] = den > 0 ? V / den : V; p[1] = dd; p[2] = nn;
    }
    size_t ni = T.invs.size() / 4;
    T.invp.assign(4 * ni, 0.0);
    for (size_t v = 0; v < ni; v++) {
        int c = T.invs[4 * v], tc = ty[c];
        double* p = &T.invp[4 * v];
        if (tc < 0) continue;
        char h = suffix_of(tc);
        El e = kType[tc].el;
        double K = 0, c0 = 0, c1 = 0, c2 = 0;
        if (e == EL_C && (h == '2' || h == 'R')) {
            bool carbonyl = false;
            for (int s = 0; s < 4; s++) { int g = T.neighs[4 * c + s]; if (g < 0) break; if (ty[g] >= 0 && kType[ty[g]].el == EL_O && suffix_of(ty[g]) == '2') carbonyl = true; }
            K = (carbonyl ? 50.0 : 6.0) * kKcal; c0 = 1; c1 = -1; c2 = 0;
        } else if (e == EL_N && (h == '2' || h == 'R')) {
            K = 6.0 * kKcal; c0 = 1; c1 = -1; c2 = 0;
        } else if (e == EL_P) {
            double w0 = 84.4339 * kDeg;
            c0 = 4.0 * std::cos(w0) * std::cos(w0) - std::cos(2.0 * w0); c1 = -4.0 * std::cos(w0); c2 = 1.0;
            K = 22.0 * kKcal / (c0 + c1 + c2);
        }
        p[0] = K / 3.0; p[1] = c0; p[2] = c1; p[3] = c2;
    }
    T.req.assign(4 * T.n, 0.0);
    for (int a = 0; a < T.n; a++) {
        int t = ty[a];
        if (t >= 0) { T.req[4 * a] = kType[t].rvdw; T.req[4 * a + 1] = std::sqrt(kType[t].evdw); T.req[4 * a + 2] = kType[t].qbase; T.req[4 * a + 3] = kType[t].hb; }
        else { T.req[4 * a] = 1.5; }
    }
}

void fill_bond_kl(HostTopo& T) {
    T.bond_kl.assign(8 * T.n, 0.0);
    for (int a = 0; a < T.n; a++)
        for (int s = 0; s < 4; s++) {
            int b = T.neighBs[4 * a + s];
            if (b < 0) continue;
            T.bond_kl[8 * a + 2 * s] = T.bparams[2 * b];
            T.bond_kl[8 * a + 2 * s + 1] = T.bparams[2 * b + 1];
        }
}

bool check_slots(const HostTopo& T, char* err, int errlen) {
    for (size_t i = 0; i < T.ang_ngs.size(); i++) if (T.ang_ngs[i] < 0) { std::snprintf(err, errlen, "angle %zu: neighbour slot not found", i / 2); return false; }
    for (size_t i = 0; i < T.dih_ngs.size(); i++) if (T.dih_ngs[i] < 0) { std::snprintf(err, errlen, "dihedral %zu: neighbour slot not found", i / 3); return false; }
    for (size_t i = 0; i < T.inv_ngs.size(); i++) if (T.inv_ngs[i] < 0) { std::snprintf(err, errlen, "inversion %zu: neighbour slot not found", i / 3); return false; }
    return true;
}

}  // namespace

const char* type_name(int id) { return (id >= 0 && id < kNType) ? kType[id].name : "?"; }

int build_molecule_topology(int n, const int* Z, const double* pos, const double* q, double bond_cut, HostTopo& T,
                            char* err, int errlen) {
    if (n <= 0 || n > 8191) { std::snprintf(err, errlen, "natoms=%d outside [1, 8191]", n); return -1; }
    std::vector<El> el(n);
    for (int a = 0; a < n; a++) {
        el[a] = el_of_Z(Z[a]);
        if (el[a] == EL_X || !kElem[el[a]].known) { std::snprintf(err, errlen, "atom %d: element Z=%d has no UFF parameters here", a, Z[a]); return -1; }
    }
    T = HostTopo();
    T.n = n;
    const double rc2 = bond_cut * bond_cut;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1], dz = pos[3 * j + 2] - pos[3 * i + 2];
            if (dx * dx + dy * dy + dz * dz < rc2) { T.bonds.push_back(i); T.bonds.push_back(j); }
        }
    std::vector<int> deg(n, 0);
    for (size_t k = 0; k < T.bonds.size(); k++) deg[T.bonds[k]]++;
    for (int a = 0; a < n; a++) if (deg[a] > 4) { std::snprintf(err, errlen, "atom %d has %d bonds within the cutoff (max 4)", a, deg[a]); return -1; }
    neighbour_slots(T);
    assign_types(n, el, T.neighs, T.type_id);
    enumerate_terms(T);
    if (!check_slots(T, err, errlen)) return -1;
    uff_parameters(T);
    if (q) for (int a = 0; a < n; a++) T.req[4 * a + 2] = q[a];
    fill_bond_kl(T);
    return 0;
}

// A periodic molecule: bonds by cutoff to every image of a partner within one cell along each
// nonzero lattice vector (lvec = a, b, c), each bond slot recording the cell of its partner's image
// (the neighCell of opencl/UFF.cl:152, 229-236).  Typing and terms follow the bond graph as for an
// isolated molecule; since terms are enumerated over atom indices, a cell in which an atom bonds
// to its own image, a pair bonds in two images, or a 3-bond path returns to its first atom through
// the images is too small and is refused.  The molecule's default images are one cell each side
// along its periodic axes.
int build_molecule_topology_pbc(int n, const int* Z, const double* pos, const double* q, double bond_cut,
                                const double lvec[9], HostTopo& T, char* err, int errlen) {
    if (n <= 0 || n > 8191) { std::snprintf(err, errlen, "natoms=%d outside [1, 8191]", n); return -1; }
    std::vector<El> el(n);
    for (int a = 0; a < n; a++) {
        el[a] = el_of_Z(Z[a]);
        if (el[a] == EL_X || !kElem[el[a]].known) { std::snprintf(err, errlen, "atom %d: element Z=%d has no UFF parameters here", a, Z[a]); return -1; }
    }
    int range[3];
    for (int k = 0; k < 3; k++) range[k] = (lvec[3 * k] != 0 || lvec[3 * k + 1] != 0 || lvec[3 * k + 2] != 0) ? 1 : 0;
    if (!range[0] && !range[1] && !range[2]) { std::snprintf(err, errlen, "all three lattice vectors are zero"); return -1; }
    T = HostTopo();
    T.n = n;
    for (int k = 0; k < 9; k++) T.lattice[k] = lvec[k];
    for (int k = 0; k < 3; k++) T.npbc[k] = range[k];
    const double rc2 = bond_cut * bond_cut;
    std::vector<int> off;                              // per bond: cell code of atom 1's image seen from atom 0
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) {
            int found = 0;
            for (int oz = -range[2]; oz <= range[2]; oz++)
                for (int oy = -range[1]; oy <= range[1]; oy++)
                    for (int ox = -range[0]; ox <= range[0]; ox++) {
                        if (i == j && !ox && !oy && !oz) continue;
                        double d[3];
                        for (int c = 0; c < 3; c++) d[c] = pos[3 * j + c] - pos[3 * i + c] + ox * lvec[c] + oy * lvec[3 + c] + oz * lvec[6 + c];
                        if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] >= rc2) continue;
                        if (i == j) { std::snprintf(err, errlen, "atom %d bonds to its own image: cell too small", i); return -1; }
                        if (found++) { std::snprintf(err, errlen, "atoms %d and %d bond in two images: cell too small", i, j); return -1; }
                        T.bonds.push_back(i); T.bonds.push_back(j);
                        off.push_back(cell_code(ox, oy, oz));
                    }
        }
    std::vector<int> deg(n, 0);
    for (size_t k = 0; k < T.bonds.size(); k++) deg[T.bonds[k]]++;
    for (int a = 0; a < n; a++) if (deg[a] > 4) { std::snprintf(err, errlen, "atom %d has %d bonds within the cutoff (max 4)", a, deg[a]); return -1; }
    neighbour_slots(T);
    T.neighc.assign(4 * (size_t)n, 0);
    for (int a = 0; a < n; a++)
        for (int s = 0; s < 4; s++) {
            const int b = T.neighBs[4 * a + s];
            if (b < 0) continue;
            const int c = off[b], sg = T.bonds[2 * b] == a ? 1 : -1;   // offsets are seen from the bond's first atom
            T.neighc[4 * a + s] = cell_code(sg * cell_field(c, 0), sg * cell_field(c, 1), sg * cell_field(c, 2));
        }
    for (int j = 0; j < n; j++)                        // 3-bond paths i-j-k-i through the images
        for (int sj = 0; sj < 4; sj++) {
            const int k = T.neighs[4 * j + sj];
            if (k < 0) continue;
            for (int si = 0; si < 4; si++) {
                const int i = T.neighs[4 * j + si];
                if (i < 0 || si == sj) continue;
                for (int sk = 0; sk < 4; sk++) {
                    if (T.neighs[4 * k + sk] != i) continue;
                    for (int ax = 0; ax < 3; ax++)
                        if (cell_field(T.neighc[4 * j + sj], ax) - cell_field(T.neighc[4 * j + si], ax) + cell_field(T.neighc[4 * k + sk], ax)) {
                            std::snprintf(err, errlen, "bond path %d-%d-%d-%d closes through the images: cell too small", i, j, k, i);
                            return -1;
                        }
                }
            }
        }
    assign_types(n, el, T.neighs, T.type_id);
    enumerate_terms(T);
    if (!check_slots(T, err, errlen)) return -1;
    uff_parameters(T);
    if (q) for (int a = 0; a < n; a++) T.req[4 * a + 2] = q[a];
    fill_bond_kl(T);
    return 0;
}

// A molecule whose bonds and angle / dihedral / inversion lists come from a file (the reference's
// TopologyData JSON or UFFTOPO binary, crates/libs/moltopo/src/export.rs:12-74,
// crates/apps/buildff/src/main.rs:10-28): the lists are taken as they are, as Uff::from_topology
// does (crates/libs/molff/src/uff.rs:238-240); atoms are typed from Z and the bond graph unless
// type ids are given; parameters follow the same UFF rules as build_molecule_topology.
int build_listed_topology(int n, const int* Z, const int* type_ids, const double* q, int nb, const int* bonds, int na,
                          const int* angs, int nd, const int* dihs, int ni, const int* invs, HostTopo& T, char* err, int errlen) {
    if (n <= 0 || n > 8191) { std::snprintf(err, errlen, "natoms=%d outside [1, 8191]", n); return -1; }
    std::vector<El> el(n);
    for (int a = 0; a < n; a++) {
        el[a] = el_of_Z(Z[a]);
        if (el[a] == EL_X || !kElem[el[a]].known) { std::snprintf(err, errlen, "atom %d: element Z=%d has no UFF parameters here", a, Z[a]); return -1; }
    }
    auto in_range = [&](const int* p, int m) { for (int r = 0; r < m; r++) if (p[r] < 0 || p[r] >= n) return false; return true; };
    T = HostTopo();
    T.n = n;
    std::vector<int> deg(n, 0);
    for (int b = 0; b < nb; b++) {
        if (!in_range(bonds + 2 * b, 2) || bonds[2 * b] == bonds[2 * b + 1]) { std::snprintf(err, errlen, "bond %d: invalid atoms", b); return -1; }
        T.bonds.push_back(bonds[2 * b]); T.bonds.push_back(bonds[2 * b + 1]);
        deg[bonds[2 * b]]++; deg[bonds[2 * b + 1]]++;
    }
    for (int a = 0; a < n; a++) if (deg[a] > 4) { std::snprintf(err, errlen, "atom %d has %d bonds (max 4)", a, deg[a]); return -1; }
    neighbour_slots(T);
    if (type_ids) {
        T.type_id.assign(type_ids, type_ids + n);
        for (int a = 0; a < n; a++)
            if (T.type_id[a] < 0 || T.type_id[a] >= kNType) { std::snprintf(err, errlen, "atom %d: unknown type id %d", a, T.type_id[a]); return -1; }
    } else {
        assign_types(n, el, T.neighs, T.type_id);
    }
    for (int t = 0; t < na; t++) {
        const int* a = angs + 3 * t;
        if (!in_range(a, 3)) { std::snprintf(err, errlen, "angle %d: atom index out of range", t); return -1; }
        T.angs.insert(T.angs.end(), {a[0], a[1], a[2]});
        T.ang_ngs.insert(T.ang_ngs.end(), {slot_of(T, a[1], a[0], 4), slot_of(T, a[1], a[2], 4)});
    }
    for (int t = 0; t < nd; t++) {
        const int* q4 = dihs + 4 * t;
        if (!in_range(q4, 4)) { std::snprintf(err, errlen, "dihedral %d: atom index out of range", t); return -1; }
        T.dihs.insert(T.dihs.end(), {q4[0], q4[1], q4[2], q4[3]});
        T.dih_ngs.insert(T.dih_ngs.end(), {slot_of(T, q4[1], q4[0], 4), slot_of(T, q4[1], q4[2], 4), slot_of(T, q4[2], q4[3], 4)});
        T.dih_kj.push_back(slot_of(T, q4[2], q4[1], 4));
    }
    for (int t = 0; t < ni; t++) {
        const int* q4 = invs + 4 * t;
        if (!in_range(q4, 4)) { std::snprintf(err, errlen, "inversion %d: atom index out of range", t); return -1; }
        T.invs.insert(T.invs.end(), {q4[0], q4[1], q4[2], q4[3]});
        T.inv_ngs.insert(T.inv_ngs.end(), {slot_of(T, q4[0], q4[1], 3), slot_of(T, q4[0], q4[2], 3), slot_of(T, q4[0], q4[3], 3)});
    }
    if (!check_slots(T, err, errlen)) return -1;
    uff_parameters(T);
    if (q) for (int a = 0; a < n; a++) T.req[4 * a + 2] = q[a];
    fill_bond_kl(T);
    return 0;
}

int type_id_of(const char* name) {
    for (int t = 0; t < kNType; t++) if (std::strcmp(kType[t].name, name) == 0) return t;
    return -1;
}

int build_desc_topology(int natoms, const double* req, const int* neighs, const double* bond_kl,
                        int nang, const int* angs, const double* angp, int ndih, const int* dihs, const double* dihp,
                        int ninv, const int* invs, const double* invp, HostTopo& T, char* err, int errlen) {
    if (natoms <= 0 || natoms > 8191) { std::snprintf(err, errlen, "natoms=%d outside [1, 8191]", natoms); return -1; }
    T = HostTopo();
    T.n = natoms;
    T.req.assign(req, req + 4 * natoms);
    T.neighs.assign(neighs, neighs + 4 * natoms);
    T.bond_kl.assign(bond_kl, bond_kl + 8 * natoms);
    T.neighBs.assign(4 * natoms, -1);
    T.type_id.assign(natoms, -1);
    for (int a = 0; a < natoms; a++)
        for (int s = 0; s < 4; s++) {
            int g = T.neighs[4 * a + s];
            if (g < -1 || g >= natoms || g == a) { std::snprintf(err, errlen, "atom %d slot %d: neighbour %d invalid", a, s, g); return -1; }
            if (g > a) {   // one bond record per pair, numbered in order of the lower index
                T.bonds.push_back(a); T.bonds.push_back(g);
                T.bparams.push_back(bond_kl[8 * a + 2 * s]); T.bparams.push_back(bond_kl[8 * a + 2 * s + 1]);
            }
        }
    for (size_t b = 0; b < T.bonds.size() / 2; b++) {
        int i = T.bonds[2 * b], j = T.bonds[2 * b + 1];
        for (int s = 0; s < 4; s++) { if (T.neighs[4 * i + s] == j) T.neighBs[4 * i + s] = (int)b; if (T.neighs[4 * j + s] == i) T.neighBs[4 * j + s] = (int)b; }
    }
    auto in_range = [&](const int* p, int m) { for (int r = 0; r < m; r++) if (p[r] < 0 || p[r] >= natoms) return false; return true; };
    for (int t = 0; t < nang; t++) {
        if (!in_range(angs + 3 * t, 3)) { std::snprintf(err, errlen, "angle %d: atom index out of range", t); return -1; }
        int i = angs[3 * t], j = angs[3 * t + 1], k = angs[3 * t + 2];
        T.angs.insert(T.angs.end(), {i, j, k});
        T.ang_ngs.insert(T.ang_ngs.end(), {slot_of(T, j, i, 4), slot_of(T, j, k, 4)});
        T.angp.insert(T.angp.end(), angp + 5 * t, angp + 5 * t + 5);
    }
    for (int t = 0; t < ndih; t++) {
        if (!in_range(dihs + 4 * t, 4)) { std::snprintf(err, errlen, "dihedral %d: atom index out of range", t); return -1; }
        const int* q = dihs + 4 * t;
        T.dihs.insert(T.dihs.end(), q, q + 4);
        T.dih_ngs.insert(T.dih_ngs.end(), {slot_of(T, q[1], q[0], 4), slot_of(T, q[1], q[2], 4), slot_of(T, q[2], q[3], 4)});
        T.dih_kj.push_back(slot_of(T, q[2], q[1], 4));
        T.dihp.insert(T.dihp.end(), dihp + 3 * t, dihp + 3 * t + 3);
    }
    for (int t = 0; t < ninv; t++) {
        if (!in_range(invs + 4 * t, 4)) { std::snprintf(err, errlen, "inversion %d: atom index out of range", t); return -1; }
        const int* q = invs + 4 * t;
        T.invs.insert(T.invs.end(), q, q + 4);
        T.inv_ngs.insert(T.inv_ngs.end(), {slot_of(T, q[0], q[1], 3), slot_of(T, q[0], q[2], 3), slot_of(T, q[0], q[3], 3)});
        T.invp.insert(T.invp.end(), invp + 4 * t, invp + 4 * t + 4);
    }
    if (!check_slots(T, err, errlen)) return -1;
    return 0;
}

// Packing of terms into rounds of `team` records such that within a round the atoms in
// each role are pairwise distinct (empty records have at.x = -1).  Greedy first-fit over a
// term order, where each term may be placed in either of its two equivalent orientations
// (an angle i-j-k as k-j-i, a dihedral i-j-k-l as l-k-j-i); the best of several seeded
// random orders is kept, so the result is deterministic.
namespace {
struct Xorshift {
    unsigned long long s;
    unsigned long long next() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }
};

// Lower bound on the rounds: capacity, and per atom the terms in which it holds a role (a role
// and its mirror under reversal share one count that may split over two orientations).
template <int R>
int rounds_lower_bound(int n, int nterms, const std::vector<int>& atoms, int team) {
    int lb = (nterms + team - 1) / team;
    std::vector<int> c((size_t)R * n, 0);
    bool rev = false;
    for (int t = 0; t < nterms; t++) {
        const int* a0 = &atoms[(size_t)t * 2 * R];
        const int* a1 = a0 + R;
        if (!std::equal(a0, a0 + R, a1)) rev = true;
        for (int k = 0; k < R; k++) c[(size_t)k * n + a0[k]]++;
    }
    for (int a = 0; a < n; a++)
        for (int k = 0; k < R; k++) {
            const int m = R - 1 - k;
            if (!rev || m == k) lb = std::max(lb, c[(size_t)k * n + a]);
            else if (k < m) lb = std::max(lb, (c[(size_t)k * n + a] + c[(size_t)m * n + a] + 1) / 2);
        }
    return lb;
}

// Min-conflicts search for an assignment in `rounds` rounds: each term's round and orientation
// are moved, one conflicted term at a time, to the choice that clashes least (atoms sharing a
// role in a round, rounds over capacity).  Conflicted terms are drawn from a candidate list: a
// term joining a clash is listed together with the round members it clashes with, so an empty
// list means no clash is left (checked once more by a full scan).  Deterministic (seeded); gives
// up after `budget` moves.  Returns true with round_of / orient_of set when it found no clash.
template <int R>
bool pack_min_conflicts(int n, int nterms, const std::vector<int>& atoms, int team, int rounds, std::vector<int>& round_of,
                        std::vector<int>& orient_of, unsigned long long seed, long long budget) {
    Xorshift rng{seed};
    std::vector<int> occ((size_t)rounds * R * n, 0), cnt(rounds, 0);
    auto at = [&](int t, int o) { return &atoms[((size_t)t * 2 + o) * R]; };
    auto slot = [&](int r, int k, int a) -> int& { return occ[((size_t)r * R + k) * n + a]; };
    std::vector<int> ro(nterms), oo(nterms), cand, where(nterms);
    std::vector<std::vector<int>> members(rounds);
    std::vector<char> listed(nterms, 0);
    auto add = [&](int t) { if (!listed[t]) { listed[t] = 1; cand.push_back(t); } };
    auto join = [&](int t, int r) { where[t] = (int)members[r].size(); members[r].push_back(t); };
    auto leave = [&](int t, int r) {
        const int w = where[t], last = members[r].back();
        members[r][w] = last; where[last] = w; members[r].pop_back();
    };
    for (int t = 0; t < nterms; t++) {            // start from the greedy assignment folded into `rounds`
        ro[t] = round_of[t] < rounds ? round_of[t] : (int)(rng.next() % (unsigned long long)rounds);
        oo[t] = orient_of[t];
        const int* a = at(t, oo[t]);
        for (int k = 0; k < R; k++) slot(ro[t], k, a[k])++;
        cnt[ro[t]]++;
        join(t, ro[t]);
    }
    auto clash = [&](int t, int r, int o, bool self) {
        const int* a = at(t, o);
        int c = 0;
        for (int k = 0; k < R; k++) c += slot(r, k, a[k]) - (self ? 1 : 0);
        const int load = cnt[r] - (self ? 1 : 0);
        if (load >= team) c += 1 + load - team;
        return c;
    };
    for (int t = 0; t < nterms; t++) if (clash(t, ro[t], oo[t], true) > 0) add(t);
    for (long long it = 0; it < budget; it++) {
        if (cand.empty()) {
            for (int t = 0; t < nterms; t++) if (clash(t, ro[t], oo[t], true) > 0) add(t);
            if (cand.empty()) { round_of = ro; orient_of = oo; return true; }
        }
        const size_t ci = (size_t)(rng.next() % (unsigned long long)cand.size());
        const int t = cand[ci];
        if (clash(t, ro[t], oo[t], true) == 0) {   // no longer in a clash: drop it from the list
            cand[ci] = cand.back(); cand.pop_back(); listed[t] = 0;
            continue;
        }
        const int* a = at(t, oo[t]);
        for (int k = 0; k < R; k++) slot(ro[t], k, a[k])--;
        cnt[ro[t]]--;
        leave(t, ro[t]);
        int best = 1 << 30, br = ro[t], bo = oo[t], ties = 0;
        const int no = std::equal(at(t, 0), at(t, 0) + R, at(t, 1)) ? 1 : 2;
        for (int r = 0; r < rounds; r++)
            for (int o = 0; o < no; o++) {
                int c = clash(t, r, o, false);
                if (r == ro[t] && o == oo[t]) c += 1;   // prefer moving
                if (c < best) { best = c; br = r; bo = o; ties = 1; }
                else if (c == best && rng.next() % (unsigned long long)(++ties) == 0) { br = r; bo = o; }
            }
        if (rng.next() % 16 == 0) { br = (int)(rng.next() % (unsigned long long)rounds); bo = no == 2 ? (int)(rng.next() & 1) : 0; }
        ro[t] = br; oo[t] = bo;
        a = at(t, bo);
        bool joined_clash = cnt[br] >= team;
        for (int k = 0; k < R; k++) joined_clash = joined_clash || slot(br, k, a[k]) > 0;
        if (joined_clash)                          // list the members it now clashes with
            for (int u : members[br]) {
                const int* b = at(u, oo[u]);
                bool hit = cnt[br] >= team;
                for (int k = 0; k < R && !hit; k++) hit = b[k] == a[k];
                if (hit) add(u);
            }
        for (int k = 0; k < R; k++) slot(br, k, a[k])++;
        cnt[br]++;
        join(t, br);
        if (clash(t, br, bo, true) == 0) { cand[ci] = cand.back(); cand.pop_back(); listed[t] = 0; }
    }
    return false;
}

// atoms[t*R*2 + o*R + k]: atom of role k in orientation o (o = 1 may equal o = 0)
template <int R>
int pack_assign(int n, int nterms, const std::vector<int>& atoms, int team, std::vector<int>& round_of,
                std::vector<int>& pos_of, std::vector<int>& orient_of) {
    if (nterms == 0) { round_of.clear(); pos_of.clear(); orient_of.clear(); return 0; }
    const int tries = std::max(1, std::min(8, 400000 / (nterms * R + 1)));
    Xorshift rng{0x9E3779B97F4A7C15ull ^ (unsigned long long)nterms};
    std::vector<int> order(nterms), r_of(nterms), p_of(nterms), o_of(nterms);
    int best = 1 << 30;
    for (int tr = 0; tr < tries; tr++) {
        for (int t = 0; t < nterms; t++) order[t] = t;
        if (tr > 0) for (int t = nterms - 1; t > 0; t--) std::swap(order[t], order[rng.next() % (unsigned long long)(t + 1)]);
        std::vector<std::vector<unsigned char>> used;
        std::vector<int> count;
        for (int t : order) {
            int br = -1, bo = 0;
            for (int o = 0; o < 2; o++) {
                const int* at = &atoms[((size_t)t * 2 + o) * R];
                if (o == 1 && std::equal(at, at + R, &atoms[(size_t)t * 2 * R])) break;
                for (int r = 0; r < (br < 0 ? (int)used.size() : br); r++) {
                    if (count[r] >= team) continue;
                    bool ok = true;
                    for (int k = 0; k < R && ok; k++) if (used[r][(size_t)k * n + at[k]]) ok = false;
                    if (ok) { br = r; bo = o; break; }
                }
            }
            if (br < 0) { br = (int)used.size(); bo = 0; used.emplace_back((size_t)R * n, 0); count.push_back(0); }
            const int* at = &atoms[((size_t)t * 2 + bo) * R];
            for (int k = 0; k < R; k++) used[br][(size_t)k * n + at[k]] = 1;
            r_of[t] = br; p_of[t] = count[br]++; o_of[t] = bo;
            if ((int)used.size() >= best) break;
        }
        if ((int)used.size() < best) { best = (int)used.size(); round_of = r_of; pos_of = p_of; orient_of = o_of; }
    }
    // fewer rounds than the greedy found, one at a time down to the lower bound, by min-conflicts
    // search; the first target it cannot reach within its budget ends the descent
    const int lb = rounds_lower_bound<R>(n, nterms, atoms, team);
    const long long budget = std::min<long long>(30000, 300LL * nterms + 20000);
    while (best > lb) {
        const int rr = best - 1;
        std::vector<int> ro = round_of, oo = orient_of;
        if (!pack_min_conflicts<R>(n, nterms, atoms, team, rr, ro, oo, 0xD1B54A32D192ED03ull ^ ((unsigned long long)nterms << 8) ^ rr, budget))
            break;
        std::vector<int> fill(rr, 0);
        for (int t = 0; t < nterms; t++) pos_of[t] = fill[ro[t]]++;
        round_of = ro; orient_of = oo;
        best = rr;
    }
    return best;
}

template <class Rec, class Fill>
void emit(int rounds, int team, int nterms, const std::vector<int>& round_of, const std::vector<int>& pos_of,
          const std::vector<int>& orient_of, std::vector<Rec>& out, Fill fill) {
    Rec empty;
    std::memset(&empty, 0, sizeof(Rec));
    empty.at = make_short4(-1, -1, -1, -1);
    out.assign((size_t)rounds * team, empty);
    for (int t = 0; t < nterms; t++) fill(out[(size_t)round_of[t] * team + pos_of[t]], t, orient_of[t]);
}
}  // namespace

// Gather form: every term once in canonical orientation, pieces laid out as angles (3 each),
// dihedrals (4), inversions (4), and for each atom the list of its pieces in that order.
void flat_terms(const HostTopo& T, FlatTerms& F) {
    const int na = (int)T.angs.size() / 3, nd = (int)T.dihs.size() / 4, ni = (int)T.invs.size() / 4;
    F.ang.resize(na); F.dih.resize(nd); F.inv.resize(ni);
    std::vector<std::vector<int>> per(T.n);
    for (int t = 0; t < na; t++) {
        const int* a = &T.angs[3 * t]; const int* s = &T.ang_ngs[2 * t]; const double* p = &T.angp[5 * t];
        AngRec& r = F.ang[t];
        r.at = make_short4((short)a[0], (short)a[1], (short)a[2], 0);
        r.sl = make_short4((short)s[0], (short)s[1], 0, 0);
        r.p = make_float4((float)(p[0] * p[1]), (float)(p[0] * p[2]), (float)(p[0] * p[3]), (float)(p[0] * p[4]));
        for (int k = 0; k < 3; k++) per[a[k]].push_back(3 * t + k);
    }
    for (int t = 0; t < nd; t++) {
        const int* a = &T.dihs[4 * t]; const int* s = &T.dih_ngs[3 * t]; const double* p = &T.dihp[3 * t];
        DihRec& r = F.dih[t];
        r.at = make_short4((short)a[0], (short)a[1], (short)a[2], (short)a[3]);
        r.sl = make_short4((short)s[0], (short)s[1], (short)s[2], 0);
        r.p = make_float4((float)p[0], (float)p[1], (float)p[2], 0.f);
        for (int k = 0; k < 4; k++) per[a[k]].push_back(3 * na + 4 * t + k);
    }
    for (int t = 0; t < ni; t++) {
        const int* a = &T.invs[4 * t]; const int* s = &T.inv_ngs[3 * t]; const double* p = &T.invp[4 * t];
        InvRec& r = F.inv[t];
        r.at = make_short4((short)a[0], (short)a[1], (short)a[2], (short)a[3]);
        r.sl = make_short4((short)s[0], (short)s[1], (short)s[2], 0);
        r.p = make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
        for (int k = 0; k < 4; k++) per[a[k]].push_back(3 * na + 4 * nd + 4 * t + k);
    }
    F.npieces = 3 * na + 4 * nd + 4 * ni;
    F.a2f.resize(T.n);
    F.idx.clear();
    for (int a = 0; a < T.n; a++) {
        F.a2f[a] = make_int2((int)F.idx.size(), (int)per[a].size());
        F.idx.insert(F.idx.end(), per[a].begin(), per[a].end());
    }
}

// Owner form: each term goes to an atom whose neighbour slots hold all its other atoms, so the
// owner keeps its own piece and the pieces of its neighbours in registers and a per-atom gather
// over the bond back-slots assembles them (the reference's a2f assembly, opencl/UFF.cl:801-880,
// with the piece buffer indexed by bond slot).  Angles go to the apex j, inversions to the centre
// i, and each dihedral i-j-k-l twice: to j (keeping the pieces of j and i) and to k (k and l).
// Needs symmetric neighbour lists (the back slot of every bond) and at most 255 terms of a kind
// per owner; otherwise ok = false and the caller uses another form.
bool owner_terms(const HostTopo& T, OwnerTerms& O) {
    const int n = T.n;
    const int na = (int)T.angs.size() / 3, nd = (int)T.dihs.size() / 4, ni = (int)T.invs.size() / 4;
    O = OwnerTerms{};
    O.meta.assign(n, 0);
    std::vector<int> back(4 * (size_t)n, 0);
    for (int i = 0; i < n; i++)
        for (int s = 0; s < 4; s++) {
            const int g = T.neighs[4 * i + s];
            if (g < 0) continue;
            int b = -1;
            for (int t = 0; t < 4; t++) if (T.neighs[4 * g + t] == i) b = t;
            if (b < 0) return false;
            back[4 * i + s] = b;
        }
    std::vector<std::vector<std::pair<short4, float4>>> A(n), I(n), D(n);
    for (int t = 0; t < na; t++) {
        const int* a = &T.angs[3 * t]; const int* s = &T.ang_ngs[2 * t]; const double* p = &T.angp[5 * t];
        if (s[0] >> 2 != a[1] || s[1] >> 2 != a[1]) return false;
        A[a[1]].push_back({make_short4((short)s[0], (short)s[1], 0, 0),
                           make_float4((float)(p[0] * p[1]), (float)(p[0] * p[2]), (float)(p[0] * p[3]), (float)(p[0] * p[4]))});
    }
    for (int t = 0; t < ni; t++) {
        const int* a = &T.invs[4 * t]; const int* s = &T.inv_ngs[3 * t]; const double* p = &T.invp[4 * t];
        if (s[0] >> 2 != a[0] || s[1] >> 2 != a[0] || s[2] >> 2 != a[0]) return false;
        I[a[0]].push_back({make_short4((short)s[0], (short)s[1], (short)s[2], 0),
                           make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3])});
    }
    for (int t = 0; t < nd; t++) {
        const int* a = &T.dihs[4 * t]; const int* s = &T.dih_ngs[3 * t]; const double* p = &T.dihp[3 * t];
        if (s[0] >> 2 != a[1] || s[1] >> 2 != a[1] || s[2] >> 2 != a[2]) return false;
        const float4 pp = make_float4((float)p[0], (float)p[1], (float)p[2], 0.f);
        D[a[1]].push_back({make_short4((short)s[0], (short)s[1], (short)s[2], 0), pp});
        D[a[2]].push_back({make_short4((short)s[0], (short)s[1], (short)s[2], 1), pp});
    }
    for (int i = 0; i < n; i++) {
        if (A[i].size() > 255 || I[i].size() > 255 || D[i].size() > 255) return false;
        O.rows_a = std::max(O.rows_a, (int)A[i].size());
        O.rows_i = std::max(O.rows_i, (int)I[i].size());
        O.rows_d = std::max(O.rows_d, (int)D[i].size());
        int m = (int)A[i].size() | ((int)I[i].size() << 8) | ((int)D[i].size() << 16);
        for (int s = 0; s < 4; s++) m |= back[4 * i + s] << (24 + 2 * s);
        O.meta[i] = m;
    }
    const size_t rows = (size_t)O.rows_a + O.rows_i + O.rows_d;
    O.geo.assign(rows * n, make_short4(0, 0, 0, 0));
    O.par.assign(rows * n, make_float4(0.f, 0.f, 0.f, 0.f));
    auto put = [&](const std::vector<std::vector<std::pair<short4, float4>>>& L, size_t row0) {
        for (int i = 0; i < n; i++)
            for (size_t r = 0; r < L[i].size(); r++) {
                O.geo[(row0 + r) * n + i] = L[i][r].first;
                O.par[(row0 + r) * n + i] = L[i][r].second;
            }
    };
    put(A, 0);
    put(I, O.rows_a);
    put(D, (size_t)O.rows_a + O.rows_i);
    O.ok = true;
    return true;
}

void pack_rounds(const HostTopo& T, int team, PackedTerms& P) {
    const int na = (int)T.angs.size() / 3, nd = (int)T.dihs.size() / 4, ni = (int)T.invs.size() / 4;
    std::vector<int> ro, po, oo;
    {   // angles: (i, j, k) or (k, j, i)
        std::vector<int> at(6 * (size_t)na);
        for (int t = 0; t < na; t++) {
            const int* a = &T.angs[3 * t];
            int* d = &at[6 * (size_t)t];
            d[0] = a[0]; d[1] = a[1]; d[2] = a[2]; d[3] = a[2]; d[4] = a[1]; d[5] = a[0];
        }
        P.ang_rounds = pack_assign<3>(T.n, na, at, team, ro, po, oo);
        emit(P.ang_rounds, team, na, ro, po, oo, P.ang, [&](AngRec& r, int t, int o) {
            const int* a = &T.angs[3 * t]; const int* s = &T.ang_ngs[2 * t]; const double* p = &T.angp[5 * t];
            if (o == 0) { r.at = make_short4((short)a[0], (short)a[1], (short)a[2], 0); r.sl = make_short4((short)s[0], (short)s[1], 0, 0); }
            else { r.at = make_short4((short)a[2], (short)a[1], (short)a[0], 0); r.sl = make_short4((short)s[1], (short)s[0], 0, 0); }
            r.p = make_float4((float)(p[0] * p[1]), (float)(p[0] * p[2]), (float)(p[0] * p[3]), (float)(p[0] * p[4]));
        });
    }
    {   // dihedrals: (i, j, k, l) or (l, k, j, i); the reversed form needs the slot of j in k's list
        std::vector<int> at(8 * (size_t)nd);
        for (int t = 0; t < nd; t++) {
            const int* a = &T.dihs[4 * t];
            int* d = &at[8 * (size_t)t];
            for (int k = 0; k < 4; k++) { d[k] = a[k]; d[4 + k] = a[3 - k]; }
            if (T.dih_kj.empty() || T.dih_kj[t] < 0) for (int k = 0; k < 4; k++) d[4 + k] = a[k];   // no reversed form
        }
        P.dih_rounds = pack_assign<4>(T.n, nd, at, team, ro, po, oo);
        emit(P.dih_rounds, team, nd, ro, po, oo, P.dih, [&](DihRec& r, int t, int o) {
            const int* a = &T.dihs[4 * t]; const int* s = &T.dih_ngs[3 * t]; const double* p = &T.dihp[3 * t];
            if (o == 0) { r.at = make_short4((short)a[0], (short)a[1], (short)a[2], (short)a[3]); r.sl = make_short4((short)s[0], (short)s[1], (short)s[2], 0); }
            else { r.at = make_short4((short)a[3], (short)a[2], (short)a[1], (short)a[0]); r.sl = make_short4((short)s[2], (short)T.dih_kj[t], (short)s[0], 0); }
            r.p = make_float4((float)p[0], (float)p[1], (float)p[2], 0.f);
        });
    }
    {   // inversions: the centre must stay first; one orientation
        std::vector<int> at(8 * (size_t)ni);
        for (int t = 0; t < ni; t++) for (int k = 0; k < 4; k++) at[8 * (size_t)t + k] = at[8 * (size_t)t + 4 + k] = T.invs[4 * t + k];
        P.inv_rounds = pack_assign<4>(T.n, ni, at, team, ro, po, oo);
        emit(P.inv_rounds, team, ni, ro, po, oo, P.inv, [&](InvRec& r, int t, int) {
            const int* a = &T.invs[4 * t]; const int* s = &T.inv_ngs[3 * t]; const double* p = &T.invp[4 * t];
            r.at = make_short4((short)a[0], (short)a[1], (short)a[2], (short)a[3]);
            r.sl = make_short4((short)s[0], (short)s[1], (short)s[2], 0);
            r.p = make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
        });
    }
}

}  // namespace smr
