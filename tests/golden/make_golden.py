"""Generate tests/golden/*.json from the reference's own files and documented answers.

Run where the reference tree is present, naming it by SURFMOL_REFERENCE or as the first
argument:  python tests/golden/make_golden.py <reference root>.  The outputs are committed,
so the tests need no reference at run time.

* pentacene.json  -- data/xyz/pentacene.xyz (36 atoms) plus the known answers of
  the reference's pentacene UFF test and docs:
    planar:        E_bond=3.834 E_angle=0.010 E_dih=0.000 E_inv=0.000 eV
                   (userguide/uff_spff.md:219-222, doc/topical_audit/uff.md:91)
    atom 0 z=+0.5: E_bond=3.979 E_angle=0.398 E_dih=2.634 E_inv=0.158, Fz=-11.72 eV/A
                   (userguide/uff_spff.md:224-228, doc/topical_audit/uff.md:92)
    term counts:   40 bonds, 66 angles, 104 dihedrals, 66 inversions (userguide/uff_spff.md:215)
  E_bond follows the reference CPU convention (uff.rs:611-637): summed over atoms,
  so every bond is counted from both ends.
* h2.json -- the GPU bond parity test, crates/libs/oclff/tests/test_uff_cl.rs:8-56.
* uff_rows.json -- the parameter rows of data/ElementTypes.dat and data/AtomTypes.dat
  used by the typing rules, parsed column by column as params.rs:145-205 does.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("SURFMOL_REFERENCE", "")


def read_xyz(path):
    lines = open(path).read().splitlines()
    n = int(lines[0].split()[0])
    el, pos = [], []
    for ln in lines[2:2 + n]:
        p = ln.split()
        el.append(p[0])
        pos.append([float(p[1]), float(p[2]), float(p[3])])
    return el, pos


def parse_dat(path, min_cols):
    rows = {}
    for ln in open(path).read().splitlines():
        ln = ln.strip()
        if not ln or ln.startswith("#"):
            continue
        p = ln.split()
        if len(p) < min_cols:
            continue
        rows[p[0]] = p          # later rows overwrite earlier ones, like the HashMap insert
    return rows


def main():
    global REF
    if len(sys.argv) > 1:
        REF = sys.argv[1]
    if not REF or not os.path.isdir(REF):
        sys.exit("give the reference root as the first argument or in SURFMOL_REFERENCE")
    el, pos = read_xyz(os.path.join(REF, "data/xyz/pentacene.xyz"))
    Zmap = {"H": 1, "C": 6, "N": 7, "O": 8}
    json.dump({
        "source": "data/xyz/pentacene.xyz",
        "Z": [Zmap[e] for e in el], "pos": pos,
        "counts": {"bonds": 40, "angles": 66, "dihedrals": 104, "inversions": 66},
        "planar": {"E_bond": 3.834, "E_angle": 0.010, "E_dih": 0.000, "E_inv": 0.000},
        "displaced": {"atom": 0, "z": 0.5, "E_bond": 3.979, "E_angle": 0.398, "E_dih": 2.634, "E_inv": 0.158,
                      "Fz": -11.72},
    }, open(os.path.join(HERE, "pentacene.json"), "w"), indent=1)
    json.dump({"source": "crates/libs/oclff/tests/test_uff_cl.rs:8-56", "k": 100.0, "l0": 0.9,
               "pos": [[0, 0, 0], [1, 0, 0]], "fx": [20.0, -20.0], "E_atom": [1.0, 1.0], "tol": 1e-4},
              open(os.path.join(HERE, "h2.json"), "w"), indent=1)
    et = parse_dat(os.path.join(REF, "data/ElementTypes.dat"), 10)
    at = parse_dat(os.path.join(REF, "data/AtomTypes.dat"), 13)
    elems = {}
    for name in ["H", "C", "N", "O", "Na", "Cl"]:
        p = et[name]
        elems[name] = {"r_vdw": float(p[7]), "e_vdw": float(p[8]), "q_uff": float(p[9]),
                       "u_uff": float(p[10]) if len(p) >= 11 else 0.0, "v_uff": float(p[11]) if len(p) >= 12 else 0.0,
                       "e_aff": float(p[12]) if len(p) >= 16 else 0.0}
    types = {}
    for name in ["H_", "C_3", "C_R", "C_2", "C_1", "N_3", "N_R", "N_2", "N_1", "O_3", "O_R", "O_2", "O_1", "Na", "Cl"]:
        p = at[name]
        types[name] = {"element": p[2], "r_uff": float(p[8]), "r_vdw": float(p[9]), "e_vdw": float(p[10]),
                       "q_base": float(p[11]), "h_b": float(p[12]), "a_ss": float(p[13]) if len(p) >= 19 else 0.0}
    json.dump({"source": ["data/ElementTypes.dat", "data/AtomTypes.dat"], "elements": elems, "atom_types": types},
              open(os.path.join(HERE, "uff_rows.json"), "w"), indent=1)


if __name__ == "__main__":
    main()
