"""ctypes binding of libsurfmol_b200.so (the C ABI of include/surfmol_relax.h).

The CUDA library is required: there is no CPU fallback.  If the shared library is
missing, importing this module raises ImportError telling how to build it.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsurfmol_b200.so")

DP = C.POINTER(C.c_double)
FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int)
SP = C.POINTER(C.c_short)
LLP = C.POINTER(C.c_longlong)
VP = C.c_void_p


class SmrConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("max_systems", C.c_int), ("max_atoms", C.c_longlong),
                ("reserved", C.c_int * 6)]


class SmrFireParams(C.Structure):
    _fields_ = [("dt0", C.c_double), ("dt_max", C.c_double), ("alpha0", C.c_double), ("f_inc", C.c_double),
                ("f_dec", C.c_double), ("f_alpha", C.c_double), ("n_min", C.c_int), ("fconv", C.c_double),
                ("flimit", C.c_double)]


class SmrNbParams(C.Structure):
    _fields_ = [("rdamp", C.c_float), ("alpha_morse", C.c_float), ("rcut", C.c_float), ("excl13", C.c_int)]


class SmrFoldedSurface(C.Structure):
    _fields_ = [("ax", C.c_double), ("bx", C.c_double), ("ay", C.c_double), ("by", C.c_double),
                ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("kx", DP), ("ky", DP), ("kz", DP), ("z0", DP), ("cq", DP), ("cp", DP), ("cl", DP),
                ("alpha", C.c_double), ("fmax", C.c_double)]


class SmrGridBuildParams(C.Structure):
    _fields_ = [("alpha_morse", C.c_double), ("npbc", C.c_int), ("ewald_tol", C.c_double), ("dtype", C.c_int),
                ("morse_rcut", C.c_double), ("reserved", C.c_int * 4)]


class SmrGridBuildParamsStatic(C.Structure):
    _fields_ = [("alpha_morse", C.c_double), ("npbc", C.c_int), ("ewald_tol", C.c_double), ("dtype", C.c_int),
                ("morse_rcut", C.c_double)]


class SmrTopologyDesc(C.Structure):
    _fields_ = [("natoms", C.c_int), ("req", DP), ("neighs", IP), ("bond_kl", DP),
                ("nang", C.c_int), ("angs", IP), ("angp", DP),
                ("ndih", C.c_int), ("dihs", IP), ("dihp", DP),
                ("ninv", C.c_int), ("invs", IP), ("invp", DP)]


# name -> (restype, argtypes); every function declared in include/surfmol_relax.h

class SmrRaffConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("natoms", C.c_int), ("nsys", C.c_int), ("reserved", C.c_int * 5)]


class SmrRaffStepConfig(C.Structure):
    _fields_ = [("dt", C.c_float), ("k_coll", C.c_float), ("relaxation", C.c_float), ("momentum_beta", C.c_float),
                ("rot_mass_scale", C.c_float), ("reserved", C.c_int * 3)]

SIGNATURES = {
    "smr_create": (C.c_int, [C.POINTER(SmrConfig), C.POINTER(VP)]),
    "smr_destroy": (C.c_int, [VP]),
    "smr_last_error": (C.c_char_p, [VP]),
    "smr_version": (C.c_char_p, []),
    "smr_set_nb_params": (C.c_int, [VP, C.POINTER(SmrNbParams)]),
    "smr_set_grid": (C.c_int, [VP, VP, C.c_int, FP, C.c_int, C.c_int, C.c_int, DP, DP]),
    "smr_get_grid": (C.c_int, [VP, VP, IP, FP, IP, DP, DP]),
    "smr_set_grid_planes": (C.c_int, [VP, VP, C.c_int, FP, C.c_int, C.c_int, C.c_int, DP, DP]),
    "smr_get_grid_planes": (C.c_int, [VP, FP]),
    "smr_set_grid_device": (C.c_int, [VP, VP, C.c_int, FP, C.c_int, C.c_int, C.c_int, DP, DP]),
    "smr_set_surface_folded": (C.c_int, [VP, VP]),
    "smr_grid_raw_slab": (C.c_int, [VP, C.c_int, DP, DP, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, DP, DP,
                                    C.POINTER(SmrGridBuildParams), C.c_int, C.c_int, VP]),
    "smr_grid_from_raw": (C.c_int, [VP, VP, C.c_int, C.c_int, C.c_int, DP, DP, C.c_int]),
    "smr_build_grid": (C.c_int, [VP, C.c_int, DP, DP, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, DP, DP,
                                 C.POINTER(SmrGridBuildParams)]),
    "smr_convert_grid": (C.c_int, [VP, C.c_int]),
    "smr_convert_grid_split": (C.c_int, [VP, C.c_int, C.c_int]),
    "smr_get_grid_split": (C.c_int, [VP, IP, FP]),
    "smr_build_grid_static": (C.c_int, [C.c_int, DP, DP, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, DP, DP,
                                        C.POINTER(SmrGridBuildParamsStatic), VP, VP, C.c_char_p, C.c_int]),
    "smr_add_molecule": (C.c_int, [VP, C.c_int, IP, DP, DP, C.c_double, IP]),
    "smr_add_molecule_pbc": (C.c_int, [VP, C.c_int, IP, DP, DP, C.c_double, DP, IP, IP]),
    "smr_set_pbc": (C.c_int, [VP, C.c_int, IP, DP, IP]),
    "smr_get_pbc": (C.c_int, [VP, C.c_int, DP, IP]),
    "smr_topology_cells": (C.c_int, [VP, C.c_int, IP]),
    "smr_set_constraints": (C.c_int, [VP, C.c_int, C.c_int, IP, DP, DP]),
    "smr_set_thermal_drive": (C.c_int, [VP, C.c_int, IP, DP]),
    "smr_add_molecules": (C.c_int, [VP, C.c_int, IP, IP, DP, DP, C.c_double, IP]),
    "smr_add_topology": (C.c_int, [VP, C.POINTER(SmrTopologyDesc), IP]),
    "smr_topology_counts": (C.c_int, [VP, C.c_int, IP]),
    "smr_topology_export": (C.c_int, [VP, C.c_int, IP, IP, IP, DP, IP, IP, DP, IP, IP, DP, IP, IP, DP, DP, IP]),
    "smr_type_name": (C.c_char_p, [C.c_int]),
    "smr_topo_build": (C.c_int, [C.c_int, IP, DP, DP, C.c_double, C.POINTER(VP), C.c_char_p, C.c_int]),
    "smr_topo_free": (None, [VP]),
    "smr_topo_counts": (C.c_int, [VP, IP]),
    "smr_topo_export": (C.c_int, [VP, IP, IP, IP, DP, IP, IP, DP, IP, IP, DP, IP, IP, DP, DP, IP]),
    "smr_topo_rounds": (C.c_int, [VP, C.c_int, IP, SP, SP, SP]),
    "smr_add_topo": (C.c_int, [VP, VP, IP]),
    "smr_topo_build_listed": (C.c_int, [C.c_int, IP, IP, DP, C.c_int, IP, C.c_int, IP, C.c_int, IP, C.c_int, IP,
                                        C.POINTER(VP), C.c_char_p, C.c_int]),
    "smr_add_listed_molecule": (C.c_int, [VP, C.c_int, IP, IP, DP, C.c_int, IP, C.c_int, IP, C.c_int, IP, C.c_int, IP, IP]),
    "smr_type_id": (C.c_int, [C.c_char_p]),
    "smr_topo_prepare": (C.c_int, [VP, C.c_int]),
    "smr_remove_topology": (C.c_int, [VP, C.c_int]),
    "smr_add_topos": (C.c_int, [VP, C.c_int, C.POINTER(VP), IP]),
    "smr_remove_topologies": (C.c_int, [VP, C.c_int, IP]),
    "smr_add_systems": (C.c_int, [VP, C.c_int, IP, FP, IP]),
    "smr_remove_systems": (C.c_int, [VP, C.c_int, IP]),
    "smr_set_positions": (C.c_int, [VP, C.c_int, IP, FP]),
    "smr_active_slots": (C.c_int, [VP, IP, IP]),
    "smr_eval_forces": (C.c_int, [VP, C.c_int, IP, FP, DP]),
    "smr_run_fire": (C.c_int, [VP, C.c_int, C.c_int, C.POINTER(SmrFireParams), C.c_int, IP]),
    "smr_reset_fire": (C.c_int, [VP, C.c_int, IP]),
    "smr_download": (C.c_int, [VP, C.c_int, IP, FP, FP, DP, IP, IP]),
    "smr_download_pos64": (C.c_int, [VP, C.c_int, IP, DP]),
    "smr_last_timing": (C.c_int, [VP, DP, LLP]),
    "smr_set_team_size": (C.c_int, [VP, C.c_int, C.c_int]),
    "smr_set_tuning": (C.c_int, [VP, C.c_int, C.c_int]),
    "smr_get_tuning": (C.c_int, [VP, C.c_int, IP]),
    "smr_set_graph": (C.c_int, [VP, C.c_int]),
    "smr_graph_stats": (C.c_int, [VP, LLP]),
    "smr_set_schedule": (C.c_int, [VP, C.c_int, C.c_int, C.c_int]),
    "smr_get_schedule": (C.c_int, [VP, IP, IP, IP]),
    "smr_set_stages": (C.c_int, [VP, C.c_int, IP, IP, IP, C.c_int]),
    "smr_get_stages": (C.c_int, [VP, IP, IP, IP, IP]),
    # multi-replica rigid-atom relaxation (include/surfmol_raff.h)
    "smr_raff_create": (C.c_int, [C.POINTER(SmrRaffConfig), C.POINTER(VP)]),
    "smr_raff_destroy": (C.c_int, [VP]),
    "smr_raff_last_error": (C.c_char_p, [VP]),
    "smr_raff_upload_radius": (C.c_int, [VP, FP]),
    "smr_raff_upload_neighs_and_exclusions": (C.c_int, [VP, IP, IP, IP]),
    "smr_raff_upload_fixmask": (C.c_int, [VP, IP]),
    "smr_raff_upload_cluster_ports": (C.c_int, [VP, FP, FP, C.c_int]),
    "smr_raff_upload_bk_slots": (C.c_int, [VP, IP]),
    "smr_raff_upload_state": (C.c_int, [VP, FP, FP, FP]),
    "smr_raff_step": (C.c_int, [VP, C.c_int, C.POINTER(SmrRaffStepConfig)]),
    "smr_raff_last_ms": (C.c_int, [VP, FP]),
    "smr_raff_download_pos": (C.c_int, [VP, C.c_int, FP]),
    "smr_raff_download_quat": (C.c_int, [VP, C.c_int, FP]),
    "smr_raff_download_dpos_coll": (C.c_int, [VP, C.c_int, FP]),
    "smr_raff_download_dpos_node": (C.c_int, [VP, C.c_int, FP]),
    "smr_raff_node_order": (C.c_int, [C.c_int, C.c_int, IP, IP]),
    "smr_raff_build_neighs": (C.c_int, [C.c_int, C.c_int, IP, IP]),
    "smr_raff_exclusions": (C.c_int, [C.c_int, IP, IP, IP]),
    "smr_raff_bk_slots": (C.c_int, [C.c_int, C.c_int, IP, IP]),
    "smr_raff_ports": (C.c_int, [C.c_int, FP, IP, C.c_float, FP, FP]),
    "smr_raff_element_mass": (C.c_float, [C.c_int]),
}

_lib = None


def lib():
    """Load the CUDA library (raises ImportError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not found: build it with `python -m surfmol_b200.build_ext` "
                              "(the CUDA library is required; there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
