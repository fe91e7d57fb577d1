"""ctypes binding of libexciting_b200.so (declarations in include/exciting_b200.h).

Loading fails loudly if the library was not built: there is no Python or CPU
stand-in for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libexciting_b200.so")

c_int, c_double, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
P = c_void_p


class exs_config(ctypes.Structure):
    _fields_ = [
        ("natmtot", c_int), ("nspecies", c_int), ("atom_species", P),
        ("lmaxapw", c_int), ("lmaxmat", c_int), ("apwordmax", c_int), ("apword", P),
        ("nlomax", c_int), ("nlorb", P), ("lorbl", P), ("rmt", P), ("omega", c_double),
        ("atposc", P), ("bvec", P), ("ngkmax", c_int), ("ngrtot", c_int), ("ngvec", c_int),
        ("intgv", P), ("ivg", P), ("ivgig", P), ("relativity", c_int), ("np_tail", c_int),
        ("max_batch", c_int),
    ]


class exs_scf_inputs(ctypes.Structure):
    _fields_ = [
        ("mt_aa", P), ("mt_loa", P), ("mt_lolo", P), ("oalo", P), ("ololo", P),
        ("h1aa", P), ("h1loa", P), ("h1lolo", P), ("veffig", P), ("meffig", P),
        ("cfunig", P), ("m2effig", P), ("spr_tail", P), ("apwfr_tail", P),
    ]


class exs_mt_radial(ctypes.Structure):
    _fields_ = [
        ("lmaxvr", c_int), ("nrmtmax", c_int), ("nrmt", P), ("spr", P), ("apwfr", P),
        ("lofr", P), ("veffmt", P),
    ]


# entry point -> (argtypes, restype); the list mirrors include/exciting_b200.h
SIGNATURES = {
    "exs_ctx_create": ([P, P], c_int),
    "exs_ctx_destroy": ([P], c_int),
    "exs_last_error": ([P], ctypes.c_char_p),
    "exs_ctx_sizes": ([P, P, P, P], c_int),
    "exs_set_scf_inputs": ([P, P], c_int),
    "exs_set_precision": ([P, c_int, c_int], c_int),
    "exs_set_wait_limit": ([P, ctypes.c_longlong], c_int),
    "exs_sort_index_1d": ([c_int, P, c_int, P], c_int),
    "exs_match": ([P, c_int, P, P, P, P], c_int),
    "exs_wavefmt": ([P, c_int, P, c_int, P, c_int, c_int, c_int, P, c_int, P], c_int),
    "exs_hamiltonandoverlapsetup": ([P, c_int, P, P, P, P, P], c_int),
    "exs_setup_batched": ([P, c_int, P, P, P, P, P], c_int),
    "exs_setup_batched_device": ([P, c_int, P, P, P, P, P], c_int),
    "exs_synchronize": ([P], c_int),
    "exs_set_host_copy_mode": ([P, c_int], c_int),
    "exs_solve_batched_device": ([P, c_int, P, P, P, c_int, P, P, c_int], c_int),
    "exs_setup_and_solve_batched": ([P, c_int, P, P, P, c_int, P, P, c_int], c_int),
    "exs_autotune": ([P, c_int, P, P, P, P, P, P], c_int),
    "exs_hmlistln": ([P, c_int, P, P, P, c_int], c_int),
    "exs_olpistln": ([P, c_int, P, P, P, c_int], c_int),
    "exs_interstitial_device": ([P, c_int, c_int, P, P, P, P, c_int], c_int),
    "exs_interstitial_batched_device": ([P, c_int, c_int, P, P, P, P, P, P], c_int),
    "exs_set_kernel_config": ([P, c_int], c_int),
    "exs_graph_create": ([P, c_int, P, P, P, P, P, P], c_int),
    "exs_graph_launch": ([P], c_int),
    "exs_graph_destroy": ([P], None),
    "exs_graph_create_multi": ([c_int, P, P, P, P, P, P, P, P], c_int),
    "exs_graph_synchronize": ([P], c_int),
    "exs_forcek": ([P, c_int, P, P, c_int, P, c_int, P, P, c_double, P, P, P], c_int),
    "exs_adjoint": ([P, c_int, P, P, c_int, P, c_int, P, P, P, P, P, P, P], c_int),
    "exs_set_stream": ([P, P], c_int),
    "exs_last_timings": ([P, P, c_int], c_int),
    "exs_mt_contract_noalloc": ([c_int, c_int, P, c_int, P, P, P, P, c_int, P], c_int),
    "exs_hmlint": ([P, P, P, P, P], c_int),
    "exs_hmlint_device": ([P, P], c_int),
    "exs_olprad": ([P, P, P, P, P, P, P], c_int),
    "exs_olprad_device": ([P, P], c_int),
    "exs_rttddft_set_pmat": ([P, c_int, P, P, c_int], c_int),
    "exs_rttddft_updateham": ([P, c_int, P, P, P, P, c_int, P, P, c_int], c_int),
    "exs_rttddft_updateham_device": ([P, c_int, P, P, P, P, c_int, P, P, P], c_int),
    "exs_rttddft_genpmat": ([P, c_int, P, P, P, P, P, P, c_int], c_int),
    "exs_clebgor_unit": ([c_int] * 5 + [P], c_int),
    "exs_gauntyry": ([c_int] * 6 + [P], c_int),
    "exs_ozaki_moduli": ([c_int, c_int, c_int, P, P, P, P, P, P], c_int),
    "exs_fderiv_int": ([c_int, P, P, P], c_int),
}

_LIB = None


def load(path: str = LIB_PATH):
    """Load the library and attach the signatures.  Raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"libexciting_b200.so not built ({path}); run exciting_b200/build.py")
    lib = ctypes.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


class ExsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"exciting_b200 error {code}: {msg}")
        self.code = code


def check(lib, ctx, rc):
    if rc < 0:
        msg = lib.exs_last_error(ctx)
        raise ExsError(rc, msg.decode() if msg else "")
    return rc
