"""ctypes view of include/mcmax_gpu.h (the C-ABI of libmcmax_gpu.so).

The shared library is built in-tree by mcmax_b200.build; loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MCMAX_GPU_LIB") or os.path.join(HERE, "libmcmax_gpu.so")

TMAX = 10000
TT = TMAX + 1
NANG = 180
NANGLE_SED = 30
NCOUNTERS = 16
STATIC_ARENA_BYTES = 64 * 1024 * 1024

MCG_OK, MCG_ERR_ARG, MCG_ERR_CUDA, MCG_ERR_STATE, MCG_ERR_NOMEM, MCG_ERR_LIMIT, MCG_ERR_RUN = range(7)
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_STATE", 4: "ERR_NOMEM", 5: "ERR_LIMIT", 6: "ERR_RUN"}
PREC_FP64, PREC_MIXED, PREC_EXACT = 0, 1, 2

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)


class PartIn(C.Structure):
    _fields_ = [
        ("nlam", C.c_int), ("lam", dp), ("nm", C.c_int), ("e1", dp), ("e2", dp),
        ("frac", dp), ("rho", dp), ("amin", C.c_double), ("amax", C.c_double),
        ("apow", C.c_double), ("fmax", C.c_double), ("porosity", C.c_double),
        ("normalize_abun", C.c_double), ("blend", C.c_int), ("ns", C.c_int), ("nf", C.c_int),
    ]


class PartOut(C.Structure):
    _fields_ = [
        ("kabs", dp), ("ksca", dp), ("kext", dp), ("F", dp),
        ("rho_av", C.c_double), ("mscale", C.c_double), ("rscale", C.c_double),
        ("n_dhs", C.c_int64), ("n_mie", C.c_int64), ("n_dhs_fail", C.c_int64),
    ]


class Zone(C.Structure):
    _fields_ = [("rin", C.c_double), ("rout", C.c_double), ("sh", C.c_double), ("rsh", C.c_double),
                ("shpow", C.c_double), ("denspow", C.c_double), ("fix_struct", C.c_int32)]


class Structure(C.Structure):
    _fields_ = [("nr", C.c_int32), ("nt", C.c_int32), ("ngrains", C.c_int32), ("R", C.POINTER(C.c_double)),
                ("Theta", C.POINTER(C.c_double)), ("V", C.POINTER(C.c_double)), ("Mstar", C.c_double),
                ("nzones", C.c_int32), ("zones", C.POINTER(Zone)), ("shscale", C.POINTER(C.c_double)),
                ("grain_scale", C.POINTER(C.c_double)), ("shtype", C.POINTER(C.c_int32))]


# scale-height types (MCG_SH_*), by the reference's keyword values
SHTYPES = ("DISK", "ZODI", "HALO", "LOBE", "JET", "SHELL", "CYLI", "CAVITY", "WEDGE", "KEEP")


class TraceOpts(C.Structure):
    _fields_ = [("angle", C.c_double), ("nphi", C.c_int32), ("nr", C.c_int32), ("nRfix", C.c_int32),
                ("Rfix", C.POINTER(C.c_double)), ("lam_path", C.c_double), ("tracestar", C.c_int32),
                ("dimstar", C.c_double), ("nphot_scatter", C.c_int64), ("nphot_star", C.c_int64),
                ("seed_scatter", C.c_uint64), ("nexits", C.c_int32)]


class ImageOpts(C.Structure):
    _fields_ = [("npixel", C.c_int32), ("nint", C.c_int32), ("Rmax", C.c_double), ("pa", C.c_double),
                ("seed", C.c_uint64), ("linear", C.c_int32), ("cap", C.c_int32), ("Rimg", C.POINTER(C.c_double)),
                ("rphi", C.POINTER(C.c_double))]


class Grid(C.Structure):
    _fields_ = [
        ("nr", C.c_int), ("nt", C.c_int), ("R", dp), ("Theta", dp), ("SinTheta", dp),
        ("dens", dp), ("V", dp), ("ncomp", C.c_int), ("comp_w", dp),
    ]


class Opacity(C.Structure):
    _fields_ = [
        ("nlam", C.c_int), ("lam", dp), ("nu", dp), ("ncomp", C.c_int),
        ("Kabs", dp), ("Ksca", dp), ("F", dp), ("BB", dp), ("Fstar", dp),
        ("Lstar", C.c_double), ("Tstar", C.c_double), ("Rstar_cm", C.c_double),
        ("scat_how", C.c_int),
    ]


class Run(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("randomwalk", C.c_int), ("factRW", C.c_double),
        ("maxinteract", C.c_int64), ("nruns", C.c_int), ("precision", C.c_int),
        ("threads", C.c_int), ("block", C.c_int), ("maxruntime", C.c_double), ("t4_single", C.c_int32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("EJv", dp), ("EJv2", dp), ("Eabs", dp), ("T", dp), ("Ni", ip),
        ("spec", dp), ("scatspec", dp), ("ispec", ip),
        ("counters", C.c_int64 * NCOUNTERS), ("tautot", C.c_double), ("device_ms", C.c_float),
        ("progress_ms", C.c_float * 5), ("Nabs", ip),
    ]


MLP_NIN, MLP_NOUT, MLP_NPARAMS, MLP_MAX_EPOCH_LOG = 6, 64, 215616, 256
fp = C.POINTER(C.c_float)


class MlpTrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float), ("lr_min", C.c_float),
                ("seed", C.c_uint64)]


class MlpTrainReport(C.Structure):
    _fields_ = [("final_loss", C.c_double), ("steps", C.c_int64), ("device_ms", C.c_float),
                ("epoch_loss", C.c_double * MLP_MAX_EPOCH_LOG)]


class BatchOpts(C.Structure):
    _fields_ = [("block", C.c_int), ("blocks_per_sm", C.c_int), ("chunk", C.c_int), ("autotune", C.c_int),
                ("use_graph", C.c_int), ("device_ms", C.c_float)]


# name -> (restype, argtypes): every symbol the header declares
SIGNATURES = {
    "mcg_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "mcg_destroy": (None, [C.c_void_p]),
    "mcg_last_error": (C.c_char_p, [C.c_void_p]),
    "mcg_version": (C.c_int, []),
    "mcg_compute_part": (C.c_int, [C.c_void_p, C.POINTER(PartIn), C.POINTER(PartOut)]),
    "mcg_compute_part_batch": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(PartIn), C.POINTER(PartOut)]),
    "mcg_compute_part_static": (C.c_int, [C.c_void_p, C.POINTER(PartIn), C.POINTER(PartOut)]),
    "mcg_bb_table": (C.c_int, [C.c_int, dp, dp]),
    "mcg_planck": (C.c_double, [C.c_double, C.c_double]),
    "mcg_set_model": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Opacity)]),
    "mcg_mcradiation": (C.c_int, [C.c_void_p, C.POINTER(Run), C.POINTER(C.c_int64), C.POINTER(Result)]),
    "mcg_finalize_t": (C.c_int, [C.c_void_p, dp, dp, dp]),
    "mcg_trace_spectrum": (C.c_int, [C.c_void_p, C.POINTER(TraceOpts), dp, C.c_int32, dp, dp,
                                     C.POINTER(C.c_int32)]),
    "mcg_scatter_field": (C.c_int, [C.c_void_p, C.POINTER(TraceOpts), dp, C.c_double, dp, C.c_int64,
                                    C.POINTER(C.c_int64)]),
    "mcg_trace_image": (C.c_int, [C.c_void_p, C.POINTER(TraceOpts), dp, C.c_double, C.POINTER(ImageOpts), dp, dp,
                                  C.POINTER(C.c_int32)]),
    "mcg_disk_structure": (C.c_int, [C.c_void_p, C.POINTER(Structure), dp, dp, dp, dp, dp, dp]),
    "mcg_diffuse": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.POINTER(C.c_int32), dp, dp, dp,
                              C.POINTER(C.c_int32)]),
    "mcg_add_model": (C.c_int, [C.c_void_p, C.POINTER(Grid), C.POINTER(Opacity), C.POINTER(C.c_int)]),
    "mcg_mcradiation_batch": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(Run),
                                        C.POINTER(C.c_int64), C.POINTER(Result), C.POINTER(BatchOpts)]),
    "mcg_mlp_set_params": (C.c_int, [C.c_void_p, fp, C.c_int64]),
    "mcg_mlp_get_params": (C.c_int, [C.c_void_p, fp, C.c_int64]),
    "mcg_mlp_forward": (C.c_int, [C.c_void_p, C.c_int64, fp, fp]),
    "mcg_mlp_gradient": (C.c_int, [C.c_void_p, C.c_int64, fp, fp, fp, fp, C.POINTER(C.c_double)]),
    "mcg_mlp_train": (C.c_int, [C.c_void_p, C.c_int64, fp, fp, fp, C.POINTER(MlpTrainOpts),
                                C.POINTER(MlpTrainReport)]),
    "mcg_surrogate_targets": (C.c_int, [C.c_void_p, C.c_int64, dp, C.c_double, C.c_int, fp]),
    "mcg_compute_part_surrogate": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(PartIn), C.POINTER(PartOut), C.c_double,
                                             C.c_int, ip]),
    "mcg_mlp_time": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.c_int, fp, fp]),
    "mcg_mlp_gemm_check": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), fp]),
}

_lib = None


def load(path=LIB_PATH):
    """Load libmcmax_gpu.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            "libmcmax_gpu.so is not built (%s); run `python -m mcmax_b200.build` "
            "or __graft_entry__.build()" % path)
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    """double* / int32* of a contiguous numpy array (None stays NULL)."""
    if a is None:
        return None
    import numpy as np
    if a.dtype == np.float64:
        return a.ctypes.data_as(dp)
    if a.dtype == np.int32:
        return a.ctypes.data_as(ip)
    if a.dtype == np.float32:
        return a.ctypes.data_as(fp)
    if a.dtype == np.uint16:
        return a.ctypes.data_as(C.POINTER(C.c_uint16))
    raise TypeError("unsupported dtype %s" % a.dtype)
