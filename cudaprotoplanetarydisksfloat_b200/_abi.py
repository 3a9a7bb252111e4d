"""ctypes binding of include/fargo_b200.h (the C ABI of libfargo_b200.so).

The structures mirror the header field by field.  The library is loaded from
this package directory; if it is missing, import fails loudly (there is no
CPU fallback of the hot path).
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfargo_b200.so")

FARGO_MAXPLANETS = 100
FARGO_DIMFXY = 11
FARGO_NOALLOC_MAXRAD = 4096
FARGO_STRLEN = 512
FARGO_MAX_SUBSTEPS = 100000
FARGO_PRECISION_REFERENCE = 0
FARGO_PRECISION_ACCURATE = 1
FARGO_STRIPE_GHOST = 8
FARGO_STRIPE_MAX_GHOST = 64
FARGO_STRIPE_HEAD = 3
FARGO_CFL_TILE = 4096

STATUS = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ECUFFT", 4: "ENONFINITE", 5: "ETIMEOUT", 6: "EOOM",
          7: "EIO", 8: "ENODEV"}

_NUM_F1 = ["DT", "SIGMA0"]
_NUM_I1 = ["NINTERM", "NTOT"]
_NUM_F2 = ["MASSTAPER"]
_NUM_I2 = ["NRAD", "NSEC"]
_NUM_F3 = ["RMIN", "RMAX", "THICKNESSSMOOTHING", "ROCHESMOOTHING", "ASPECTRATIO",
           "VISCOSITY", "ALPHAVISCOSITY", "SIGMASLOPE", "RELEASERADIUS", "RELEASEDATE",
           "OMEGAFRAME", "IMPOSEDDISKDRIFT", "FLARINGINDEX", "ECCENTRICITY",
           "CAVITYRADIUS", "CAVITYRATIO", "CAVITYWIDTH",
           "TRANSITIONRADIUS", "TRANSITIONRATIO", "TRANSITIONWIDTH", "LAMBDADOUBLING",
           "ADIABATICINDEX", "COOLINGTIME0"]
_STR_LONG = ["OUTPUTDIR", "PLANETCONFIG"]
_STR_SHORT = ["INNERBOUNDARY", "LABELADVECTION", "TRANSPORT", "RADIALSPACING",
              "DISK", "FRAME", "OUTERSOURCEMASS", "WRITEDENSITY", "WRITEVELOCITY",
              "WRITEENERGY", "WRITETEMPERATURE", "WRITEQPLUS", "INDIRECTTERM",
              "EXCLUDEHILL", "SELFGRAVITY", "CICPLANET", "FORCEDCIRCULAR",
              "ZMPLUS", "ADIABATIC", "COOLING"]
_SWITCHES = ["AdvecteLabel", "OuterSourceMass", "FastTransport", "OpenInner", "NonReflecting",
             "Evanescent", "LogGrid", "IsDisk", "Corotating", "GuidingCenter",
             "Write_Density", "Write_Velocity", "Write_Energy", "Write_Temperature", "Write_DivV",
             "Write_Qplus", "Indirect_Term", "SelfGravity", "SGZeroMode", "ZMPluss",
             "Adiabatic", "Cooling", "ExcludeHill", "CICPlanet", "ForcedCircular",
             "ViscosityAlpha", "RocheSmoothing"]


class FargoParams(C.Structure):
    _fields_ = ([(n, C.c_float) for n in _NUM_F1] + [(n, C.c_int) for n in _NUM_I1] +
                [(n, C.c_float) for n in _NUM_F2] + [(n, C.c_int) for n in _NUM_I2] +
                [(n, C.c_float) for n in _NUM_F3] +
                [(n, C.c_char * FARGO_STRLEN) for n in _STR_LONG] +
                [(n, C.c_char * 64) for n in _STR_SHORT] +
                [(n, C.c_int) for n in _SWITCHES] +
                [("SloppyCFL", C.c_int), ("ScalingFactor", C.c_float)])

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = v.decode() if isinstance(v, bytes) else v
        return d


class FargoPlanets(C.Structure):
    _fields_ = [("nb", C.c_int),
                ("mass", C.c_double * FARGO_MAXPLANETS), ("x", C.c_double * FARGO_MAXPLANETS),
                ("y", C.c_double * FARGO_MAXPLANETS), ("vx", C.c_double * FARGO_MAXPLANETS),
                ("vy", C.c_double * FARGO_MAXPLANETS), ("acc", C.c_double * FARGO_MAXPLANETS),
                ("feeldisk", C.c_int * FARGO_MAXPLANETS), ("feelothers", C.c_int * FARGO_MAXPLANETS),
                ("name", (C.c_char * 64) * FARGO_MAXPLANETS)]


class FargoStripeLayout(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("base", "nrad", "nsec", "own_lo", "own_hi", "ghost_lo", "ghost_hi",
                                        "nfields", "halo_floats_lo", "halo_floats_hi", "block_doubles")]


class FargoScalars(C.Structure):
    _fields_ = [("physical_time", C.c_float), ("omega_frame", C.c_float), ("mdcp1", C.c_float),
                ("lost_mass", C.c_float), ("nsub_last_dt", C.c_int), ("nsub_total", C.c_int),
                ("mass", C.c_double), ("angular_momentum", C.c_double), ("last_dt", C.c_double)]


# every symbol the header declares (tests check that each one is exported)
EXPORTS = [
    "fargo_params_default", "fargo_params_read", "fargo_params_derive", "fargo_planets_read",
    "fargo_grid_radii", "fargo_create", "fargo_destroy", "fargo_last_error", "fargo_init_state",
    "fargo_upload", "fargo_download", "fargo_get_planets", "fargo_set_planets", "fargo_advance_dt",
    "fargo_advance", "fargo_advance_async", "fargo_sync", "fargo_disk_force", "fargo_disk_force_noalloc",
    "fargo_sg_accelerations", "fargo_get_scalars",
    "fargo_get_substep_log", "fargo_batch_create", "fargo_batch_destroy", "fargo_batch_last_error",
    "fargo_batch_init_state", "fargo_batch_upload", "fargo_batch_download", "fargo_batch_advance",
    "fargo_batch_advance_async", "fargo_batch_sync", "fargo_batch_get_scalars",
    "fargo_batch_get_planets", "fargo_batch_count_launches", "fargo_batch_kernel_launches", "fargo_abi_version",
    "fargo_kernel_launches", "fargo_set_graph_mode", "fargo_batch_set_graph_mode",
    "fargo_set_max_substeps", "fargo_batch_set_max_substeps", "fargo_set_precision", "fargo_batch_set_precision", "fargo_batch_autotune", "fargo_autotune", "fargo_checkpoint_bytes", "fargo_checkpoint_save",
    "fargo_checkpoint_load", "fargo_stream", "fargo_batch_stream",
    "fargo_ctx_batch", "fargo_batch_upload_async", "fargo_batch_download_async", "fargo_batch_profile",
    "fargo_profile_kernel_name", "fargo_profile_kernel_count",
    "fargo_stripe_create", "fargo_stripe_info", "fargo_stripe_dt_begin", "fargo_stripe_forces",
    "fargo_stripe_substep", "fargo_stripe_halo_pack", "fargo_stripe_halo_unpack", "fargo_stripe_more",
    "fargo_stripe_init_state", "fargo_stripe_sg_rows", "fargo_stripe_sg_apply", "fargo_batch_segments",
]


class FargoError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libfargo_b200.so is not built (run `python cudaprotoplanetarydisksfloat_b200/build.py`); "
            "there is no CPU fallback of the CUDA hot path")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp = C.c_void_p
    fp = P(C.c_float)
    dp = P(C.c_double)
    sig = {
        "fargo_params_default": (C.c_int, [P(FargoParams)]),
        "fargo_params_read": (C.c_int, [C.c_char_p, P(FargoParams)]),
        "fargo_params_derive": (C.c_int, [P(FargoParams)]),
        "fargo_planets_read": (C.c_int, [C.c_char_p, P(FargoParams), P(FargoPlanets)]),
        "fargo_grid_radii": (C.c_int, [P(FargoParams), dp]),
        "fargo_create": (C.c_int, [P(FargoParams), P(FargoPlanets), dp, C.c_int, P(vp)]),
        "fargo_destroy": (None, [vp]),
        "fargo_last_error": (C.c_char_p, [vp]),
        "fargo_init_state": (C.c_int, [vp, fp, fp]),
        "fargo_upload": (C.c_int, [vp, fp, fp, fp, fp]),
        "fargo_download": (C.c_int, [vp, fp, fp, fp, fp, fp, fp]),
        "fargo_get_planets": (C.c_int, [vp, P(FargoPlanets)]),
        "fargo_set_planets": (C.c_int, [vp, P(FargoPlanets)]),
        "fargo_advance_dt": (C.c_int, [vp, P(C.c_int)]),
        "fargo_advance": (C.c_int, [vp, C.c_int]),
        "fargo_advance_async": (C.c_int, [vp, C.c_int]),
        "fargo_sync": (C.c_int, [vp]),
        "fargo_disk_force": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, dp]),
        "fargo_disk_force_noalloc": (C.c_int, [vp, vp, vp, vp, vp, C.c_int, C.c_int, C.c_double, C.c_double,
                                               C.c_double, C.c_double, C.c_int, dp, vp, C.c_char_p, C.c_int]),
        "fargo_sg_accelerations": (C.c_int, [vp, fp, fp]),
        "fargo_get_scalars": (C.c_int, [vp, P(FargoScalars)]),
        "fargo_get_substep_log": (C.c_int, [vp, C.c_int, P(C.c_int), dp, P(C.c_int)]),
        "fargo_batch_create": (C.c_int, [C.c_int, P(FargoParams), P(FargoPlanets), C.c_int, P(vp)]),
        "fargo_batch_destroy": (None, [vp]),
        "fargo_batch_last_error": (C.c_char_p, [vp]),
        "fargo_batch_init_state": (C.c_int, [vp, C.c_int, fp, fp]),
        "fargo_batch_upload": (C.c_int, [vp, C.c_int, fp, fp, fp, fp]),
        "fargo_batch_download": (C.c_int, [vp, C.c_int, fp, fp, fp, fp]),
        "fargo_batch_advance": (C.c_int, [vp, C.c_int]),
        "fargo_batch_advance_async": (C.c_int, [vp, C.c_int]),
        "fargo_batch_sync": (C.c_int, [vp]),
        "fargo_batch_get_scalars": (C.c_int, [vp, C.c_int, P(FargoScalars)]),
        "fargo_batch_get_planets": (C.c_int, [vp, C.c_int, P(FargoPlanets)]),
        "fargo_batch_count_launches": (C.c_longlong, [vp]),
        "fargo_batch_kernel_launches": (C.c_longlong, [vp]),
        "fargo_abi_version": (C.c_int, []),
        "fargo_kernel_launches": (C.c_longlong, [vp]),
        "fargo_set_graph_mode": (C.c_int, [vp, C.c_int]),
        "fargo_batch_set_graph_mode": (C.c_int, [vp, C.c_int]),
        "fargo_set_max_substeps": (C.c_int, [vp, C.c_int]),
        "fargo_batch_set_max_substeps": (C.c_int, [vp, C.c_int]),
        "fargo_set_precision": (C.c_int, [vp, C.c_int]),
        "fargo_batch_set_precision": (C.c_int, [vp, C.c_int]),
        "fargo_batch_autotune": (C.c_int, [vp, C.c_int, P(C.c_int)]),
        "fargo_autotune": (C.c_int, [vp, C.c_int, P(C.c_int)]),
        "fargo_checkpoint_bytes": (C.c_size_t, [vp]),
        "fargo_checkpoint_save": (C.c_int, [vp, vp, C.c_size_t]),
        "fargo_checkpoint_load": (C.c_int, [vp, vp, C.c_size_t]),
        "fargo_stream": (vp, [vp]),
        "fargo_batch_stream": (vp, [vp]),
        "fargo_ctx_batch": (vp, [vp]),
        "fargo_batch_upload_async": (C.c_int, [vp, C.c_int, fp, fp, fp, fp]),
        "fargo_batch_download_async": (C.c_int, [vp, C.c_int, fp, fp, fp, fp]),
        "fargo_batch_profile": (C.c_int, [vp, C.c_int, dp, P(C.c_int)]),
        "fargo_profile_kernel_name": (C.c_char_p, [C.c_int]),
        "fargo_profile_kernel_count": (C.c_int, []),
        "fargo_stripe_create": (C.c_int, [P(FargoParams), P(FargoPlanets), dp, C.c_int, C.c_int, C.c_int,
                                          C.c_int, P(vp)]),
        "fargo_stripe_info": (C.c_int, [vp, P(FargoStripeLayout)]),
        "fargo_stripe_dt_begin": (C.c_int, [vp]),
        "fargo_stripe_forces": (C.c_int, [vp, vp]),
        "fargo_stripe_substep": (C.c_int, [vp, vp, C.c_int, C.c_int]),
        "fargo_stripe_halo_pack": (C.c_int, [vp, vp, vp]),
        "fargo_stripe_halo_unpack": (C.c_int, [vp, vp, vp]),
        "fargo_stripe_more": (C.c_int, [vp, P(C.c_int)]),
        "fargo_stripe_init_state": (C.c_int, [vp, fp, fp]),
        "fargo_batch_segments": (C.c_int, [vp, C.c_int, P(C.c_int)]),
        "fargo_stripe_sg_rows": (C.c_int, [vp, vp]),
        "fargo_stripe_sg_apply": (C.c_int, [vp, vp, C.c_int, C.c_int, P(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(st, what="", ctx=None, batch=None):
    if st != 0:
        msg = ""
        if ctx:
            msg = lib.fargo_last_error(ctx).decode(errors="replace")
        elif batch:
            msg = lib.fargo_batch_last_error(batch).decode(errors="replace")
        raise FargoError("%s failed: %s %s" % (what, STATUS.get(st, st), msg))
