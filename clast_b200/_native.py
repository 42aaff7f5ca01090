"""ctypes binding of libclast_b200.so (declarations: include/clast_gpu.h).

The library is built in-tree (``clast_b200/libclast_b200.so``).  Loading it
fails loudly when it is missing: there is no CPU fallback for the device path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libclast_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "clast")


class clast_params(C.Structure):
    _fields_ = [("lmer", C.c_int32), ("stride", C.c_int32), ("cut_repeat", C.c_int32),
                ("width", C.c_int32), ("gap", C.c_int32), ("local", C.c_int32),
                ("cutoff", C.c_double), ("total_db", C.c_double), ("K", C.c_double),
                ("lambda_", C.c_double)]


class clast_hits(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(f, C.POINTER(C.c_int32)) for f in
                                     ("t_id", "t_idx", "q_id", "q_idx", "t_len", "q_len", "match", "score")] + \
               [("evalue", C.POINTER(C.c_double))]


class clast_seqs(C.Structure):
    _fields_ = [("n_seqs", C.c_int64), ("bases", C.c_void_p), ("offsets", C.POINTER(C.c_int64)),
                ("bases_on_device", C.c_int32)]


class clast_map_result(C.Structure):
    _fields_ = [("n", C.c_int64), ("load_offsets", C.POINTER(C.c_int64))] + \
               [(f, C.POINTER(C.c_int32)) for f in ("read", "strand", "t_load", "t_seq", "t_idx", "q_idx",
                                                   "t_len", "q_len", "match", "score")] + \
               [("evalue", C.POINTER(C.c_double)), ("owner", C.c_void_p)]


class clast_labels(C.Structure):
    _fields_ = [("n", C.c_int64), ("chars", C.c_void_p), ("offsets", C.POINTER(C.c_int64))]


class clast_tsv(C.Structure):
    _fields_ = [("n_bytes", C.c_int64), ("text", C.c_void_p), ("load_offsets", C.POINTER(C.c_int64)),
                ("owner", C.c_void_p)]


class clast_server_config(C.Structure):
    _fields_ = [("lanes", C.c_int32), ("q_vram", C.c_int32), ("q_ram", C.c_int32), ("reserved0", C.c_int32),
                ("max_batch_bases", C.c_int64), ("hbm_budget", C.c_int64), ("hbm_reserve", C.c_int64)]


class clast_server_stats(C.Structure):
    _fields_ = [(f, C.c_int64) for f in ("batches", "requests", "bases", "max_batch_requests", "queued", "running",
                                         "hbm_budget", "hbm_in_flight_max")]


class clast_stats(C.Structure):
    _fields_ = [("index_ms", C.c_double), ("index_upload_ms", C.c_double), ("map_ms", C.c_double),
                ("map_upload_ms", C.c_double), ("index_launches", C.c_int64), ("map_launches", C.c_int64),
                ("query_bases", C.c_int64), ("query_kmers", C.c_int64), ("seeds", C.c_int64), ("hits", C.c_int64),
                ("results", C.c_int64), ("dp_cells", C.c_int64), ("seed_ms", C.c_double),
                ("seed_launches", C.c_int64), ("dp_ms", C.c_double), ("dp_launches", C.c_int64),
                ("sort_ms", C.c_double), ("final_ms", C.c_double), ("index_wall_ms", C.c_double),
                ("map_wall_ms", C.c_double), ("map_prep_ms", C.c_double), ("map_call_ms", C.c_double),
                ("index_bases", C.c_int64), ("index_keys", C.c_int64), ("dp_order_ms", C.c_double),
                ("dp_order_kind", C.c_int32), ("dp_queue_chunk", C.c_int32),
                ("dp_warp_hits", C.c_int64)]


# symbol name -> (restype, argtypes); the full export list of include/clast_gpu.h
# plus the command-line entry of clast_host.h
SIGNATURES = {
    "clast_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "clast_ctx_destroy": (None, [C.c_void_p]),
    "clast_last_error": (C.c_char_p, [C.c_void_p]),
    "clast_index_build": (C.c_int, [C.c_void_p, C.POINTER(clast_params), C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "clast_index_free": (None, [C.c_void_p]),
    "clast_search": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(clast_params), C.c_void_p, C.c_int64,
                               C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(clast_hits)]),
    "clast_hits_free": (None, [C.POINTER(clast_hits)]),
    "clast_search_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(clast_params), C.c_void_p, C.c_int64,
                                       C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int64,
                                       C.POINTER(clast_hits)]),
    "clast_targets_create": (C.c_int, [C.c_void_p, C.POINTER(clast_params), C.c_int32, C.POINTER(clast_seqs),
                                       C.c_int32, C.c_void_p, C.POINTER(C.c_void_p)]),
    "clast_targets_free": (None, [C.c_void_p]),
    "clast_targets_save": (C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p]),
    "clast_targets_load": (C.c_int, [C.c_void_p, C.POINTER(clast_params), C.c_char_p, C.POINTER(C.c_void_p)]),
    "clast_targets_verify": (C.c_int, [C.POINTER(clast_params), C.c_char_p, C.c_char_p, C.c_int]),
    "clast_map": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(clast_params), C.c_int32, C.POINTER(clast_seqs),
                            C.c_int32, C.c_void_p, C.POINTER(clast_map_result)]),
    "clast_map_result_free": (None, [C.POINTER(clast_map_result)]),
    "clast_format_tsv": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(clast_map_result), C.c_int32,
                                   C.POINTER(clast_labels), C.POINTER(clast_labels), C.c_void_p, C.c_int32,
                                   C.POINTER(clast_tsv)]),
    "clast_tsv_free": (None, [C.POINTER(clast_tsv)]),
    "clast_write_file": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int64, C.c_int32]),
    "clast_last_map_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "clast_get_stats": (C.c_int, [C.c_void_p, C.POINTER(clast_stats)]),
    "clast_int32_peak": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "clast_ctx_trim": (C.c_int, [C.c_void_p]),
    "clast_server_create": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(clast_params),
                                      C.POINTER(clast_server_config), C.POINTER(C.c_void_p)]),
    "clast_server_submit": (C.c_int, [C.c_void_p, C.POINTER(clast_seqs), C.POINTER(C.c_int64)]),
    "clast_server_poll": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(clast_map_result)]),
    "clast_server_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
    "clast_server_release": (C.c_int, [C.c_void_p, C.c_int64]),
    "clast_server_times": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64)]),
    "clast_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(clast_server_stats)]),
    "clast_server_last_error": (C.c_char_p, [C.c_void_p]),
    "clast_server_destroy": (None, [C.c_void_p]),
    "clast_cli_main": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), C.c_char_p, C.c_int]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the in-tree library once; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libclast_b200.so is not built (run __graft_entry__.build() or "
                               "make -C clast_b200/csrc); the device path has no fallback")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
