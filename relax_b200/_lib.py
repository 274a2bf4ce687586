"""ctypes binding of librelax_b200.so (the C ABI of include/relax_b200.h).

The library is built in-tree by ``relax_b200/csrc/Makefile`` (nvcc, sm_100a).
There is no fallback: if the library is missing, ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

from .config import (relax_config, relax_input_info, relax_layer, relax_obsplane, relax_segment, relax_slippatch,
                     relax_source, relax_step_log, relax_tensor, relax_tensor_layer, relax_weakzone)

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "librelax_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "relax_b200.h")

_lib = None


class RelaxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"relax error {code}: {msg}")
        self.code = code


def build(verbose: bool = False):
    """Compiles the CUDA library for sm_100a (cross-compiles without a GPU)."""
    out = subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc")], capture_output=not verbose,
                         text=True)
    if out.returncode != 0:
        raise RuntimeError("building librelax_b200.so failed:\n" + (out.stderr or "") + (out.stdout or ""))


def header_functions():
    """Names of the functions include/relax_b200.h declares."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\**\s*([A-Za-z_][A-Za-z_0-9]*)\s*\(",
                       text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "for")))


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"{LIBPATH} is missing: build it with relax_b200._lib.build() "
                           "(the CUDA path has no fallback)")
    lib = C.CDLL(LIBPATH)
    P, I, D, S = C.c_void_p, C.c_int, C.c_double, C.c_size_t
    FP = C.POINTER(C.c_float)
    sig = {
        "relax_version": (C.c_char_p, []),
        "relax_last_error": (C.c_char_p, []),
        "relax_viscoelastic_structure": (I, [P, I, D, I, P]),
        "relax_tensor_structure": (I, [P, I, D, I, P]),
        "relax_create": (I, [C.POINTER(relax_config), I, C.POINTER(P)]),
        "relax_destroy": (I, [P]),
        "relax_release_cached_memory": (I, [I]),
        "relax_set_precision": (I, [P, I]),
        "relax_op_green_mixed": (I, [P, P, P, P, P, P, I, I, I, D, D, D, D, D, D, P]),
        "relax_op_dft64_tc": (I, [P, P, I, P]),
        "relax_get_stream": (I, [P, C.POINTER(P)]),
        "relax_coseismic": (I, [P, I, C.POINTER(relax_step_log)]),
        "relax_step": (I, [P, C.POINTER(D), C.POINTER(relax_step_log)]),
        "relax_run": (I, [P, I, C.POINTER(D), C.POINTER(relax_step_log), C.POINTER(I)]),
        "relax_get_field": (I, [P, I, P, S]),
        "relax_set_field": (I, [P, I, P, S]),
        "relax_get_patches": (I, [P, I, C.POINTER(relax_slippatch), S]),
        "relax_num_planes": (I, [P, C.POINTER(I)]),
        "relax_get_plane_shape": (I, [P, I, C.POINTER(I), C.POINTER(I)]),
        "relax_get_time": (I, [P, C.POINTER(D), C.POINTER(I), C.POINTER(I)]),
        "relax_synchronize": (I, [P]),
        "relax_profile": (I, [P, I]),
        "relax_profile_stages": (I, []),
        "relax_profile_read": (I, [P, I, C.POINTER(D), C.POINTER(I), C.POINTER(C.c_char_p)]),
        "relax_launch_count": (I, [P, C.POINTER(C.c_longlong)]),
        "relax_batch_create": (I, [C.POINTER(relax_config), I, I, C.POINTER(P)]),
        "relax_batch_destroy": (I, [P]),
        "relax_batch_size": (I, [P, C.POINTER(I)]),
        "relax_batch_member": (I, [P, I, C.POINTER(P)]),
        "relax_batch_coseismic": (I, [P, C.POINTER(relax_step_log)]),
        "relax_batch_step": (I, [P, C.POINTER(relax_step_log)]),
        "relax_batch_launch_count": (I, [P, C.POINTER(C.c_longlong)]),
        "relax_batch_get_stream": (I, [P, C.POINTER(P)]),
        "relax_batch_tuning": (I, [P, C.POINTER(I), C.POINTER(D), C.POINTER(D)]),
        "relax_ensemble_create": (I, [C.POINTER(relax_config), I, I, C.POINTER(P)]),
        "relax_ensemble_destroy": (I, [P]),
        "relax_ensemble_size": (I, [P, C.POINTER(I), C.POINTER(I)]),
        "relax_ensemble_member": (I, [P, I, C.POINTER(P)]),
        "relax_ensemble_coseismic": (I, [P, C.POINTER(relax_step_log)]),
        "relax_ensemble_step": (I, [P, C.POINTER(relax_step_log)]),
        "relax_ensemble_launch_count": (I, [P, C.POINTER(C.c_longlong)]),
        "relax_ensemble_tuning": (I, [P, I, C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(D),
                                      C.POINTER(D)]),
        "relax_op_stressupdate": (I, [P, P, P, D, D, D, D, D, I, I, I, P, P]),
        "relax_op_bodyforce": (I, [P, D, D, D, I, I, I, P, P, P, P, P, P, P]),
        "relax_op_viscouseigenstress": (I, [D, P, P, P, I, I, I, P, C.POINTER(D), P, P, P]),
        "relax_op_transienteigenstress": (I, [D, P, P, P, I, I, I, P, P, C.POINTER(D), P, P]),
        "relax_op_dgammadot0": (I, [P, I, I, I, I, D, D, D, D, P, P]),
        "relax_op_frictioneigenstress": (I, [D, D, D, D, D, D, D, D, D, P, D, P, I, I, I, D, D, D, P,
                                             C.POINTER(D), P]),
        "relax_op_green": (I, [P, P, P, P, P, P, I, I, I, D, D, D, D, D, D, P]),
        "relax_op_green_noalloc": (I, [P, P, P, P, P, P, I, I, I, D, D, D, D, D, D, P]),
        "relax_op_fft3": (I, [P, I, I, I, D, D, D, I, P]),
        "relax_op_tensoramplitude": (I, [P, I, I, I, D, D, D, C.POINTER(D), P]),
        "relax_get_grid": (I, [P, C.POINTER(I), C.POINTER(D)]),
        "relax_checkpoint_save": (I, [P, C.c_char_p]),
        "relax_checkpoint_load": (I, [P, C.c_char_p]),
        "relax_op_okada": (I, [P, I, D, D, I, I, I, D, D, D, P, P, P, P]),
        "relax_okada_point": (I, [C.POINTER(relax_source), D, D, D, D, D, C.POINTER(D)]),
        "relax_track_relaxation": (I, [P, I, I, I]),
        "relax_input_parse": (I, [C.c_char_p, I, C.POINTER(P)]),
        "relax_input_read": (I, [C.c_char_p, I, C.POINTER(P)]),
        "relax_input_free": (None, [P]),
        "relax_input_config": (C.POINTER(relax_config), [P]),
        "relax_input_get_info": (I, [P, C.POINTER(relax_input_info)]),
        "relax_input_weakzones": (I, [P, I, C.POINTER(C.POINTER(relax_weakzone)), C.POINTER(I)]),
        "relax_input_export_geometry": (I, [P, I]),
        "relax_write_vtk_grid": (I, [I, I, I, D, D, D, C.c_char_p]),
        "relax_write_vtk_rectangle": (I, [D, D, D, D, D, D, D, C.c_char_p]),
        "relax_write_xy_brick": (I, [C.POINTER(relax_weakzone), C.c_char_p]),
        "relax_write_vtk_bricks": (I, [I, C.POINTER(relax_weakzone), C.c_char_p]),
        "relax_write_faults": (I, [I, I, C.POINTER(relax_source), D, D, C.c_char_p]),
        "relax_input_obsplanes": (I, [P, C.POINTER(C.POINTER(relax_obsplane)), C.POINTER(I)]),
        "relax_input_segments": (I, [P, C.POINTER(C.POINTER(relax_segment)), C.POINTER(I)]),
        "relax_monitor_plane": (I, [P, I, C.POINTER(relax_obsplane), D, C.POINTER(relax_slippatch), S,
                                    C.POINTER(I), C.POINTER(I)]),
        "relax_segment_stress": (I, [P, I, C.POINTER(relax_segment), C.POINTER(relax_tensor)]),
        "relax_export_plane_stress": (I, [P, I, I, C.POINTER(relax_obsplane), D, D, C.c_char_p, I]),
        "relax_write_segments": (I, [I, I, C.POINTER(relax_segment), C.POINTER(relax_tensor),
                                     C.POINTER(relax_tensor), C.c_char_p]),
        "relax_write_coulomb": (I, [I, C.POINTER(relax_segment), C.POINTER(relax_tensor), D, C.c_char_p, I]),
        "relax_input_build_weakzones": (I, [P, I]),
        "relax_get_plane": (I, [P, I, I, P, S]),
        "relax_get_points": (I, [P, I, C.POINTER(I), C.POINTER(D), C.POINTER(relax_tensor)]),
        "relax_write_grd": (I, [FP, I, I, D, D, D, D, C.c_char_p, C.c_char_p]),
        "relax_write_grd3": (I, [FP, FP, FP, I, I, D, D, D, D, C.c_char_p, I, I]),
        "relax_export_grd": (I, [P, I, D, D, D, C.c_char_p, I]),
        "relax_write_vtk": (I, [C.POINTER(FP), I, I, I, I, D, D, D, I, I, I, C.c_char_p, C.c_char_p,
                                C.c_char_p]),
        "relax_export_vtk": (I, [P, I, I, I, I, I, C.c_char_p, C.c_char_p, C.c_char_p]),
        "relax_export_creep": (I, [P, C.c_char_p, I, I]),
        "relax_shifted_index": (I, [D, D, D, I, I, I, D, D, D, C.POINTER(I), C.POINTER(I), C.POINTER(I)]),
        "relax_export_points": (I, [P, I, C.POINTER(D), C.POINTER(C.c_char_p), D, D, C.c_char_p, I]),
        "relax_format_log": (I, [C.POINTER(relax_step_log), D, I, C.c_char_p, S]),
        "relax_log_header": (C.c_char_p, [I]),
        "relax_format_ned": (I, [D, C.POINTER(D), C.POINTER(relax_tensor), C.c_char_p, S]),
        "relax_ned_header": (C.c_char_p, []),
        "relax_es_format": (I, [D, I, I, I, C.c_char_p, S]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc: int):
    if rc != 0:
        msg = load().relax_last_error().decode(errors="replace")
        raise RelaxError(rc, msg)


def structure_fn(layers, dx3: float, nz: int):
    """viscoelasticstructure through the library (host-side helper)."""
    lib = load()
    arr_in = (relax_layer * len(layers))(*layers)
    out = (relax_layer * nz)()
    check(lib.relax_viscoelastic_structure(C.cast(arr_in, C.c_void_p), len(layers), dx3, nz,
                                           C.cast(out, C.c_void_p)))
    return out
