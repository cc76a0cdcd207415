"""ctypes binding of libeuvl_b200.so (the C ABI declared in include/euvl_b200.h).

The library is built in-tree by ``euvlitho_b200.build``.  There is no fallback:
if the shared library is missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeuvl_b200.so")

EUV_OK = 0
EUV_ERR_BAD_ARG = 1
EUV_ERR_CUDA = 2
EUV_ERR_WORKSPACE = 3
EUV_ERR_SINGULAR = 4
EUV_ERR_TIMEOUT = 5
# bits of a device status word (euv_amp_desc.d_status and friends)
EUV_STATUS_TIMEOUT = 1
EUV_STATUS_STEPS_CLAMPED = 2
EUV_STATUS_SINGULAR = 4
EUV_STATUS_NOT_CONVERGED = 8
EUV_MAX_SLICES = 32
EUV_PREC_FP64 = 0
EUV_PREC_MIXED = 1
EUV_NOALLOC_SCRATCH_BYTES = 16 * 1024 * 1024

# Every symbol include/euvl_b200.h declares.
EXPORTS = (
    "euv_version", "euv_last_error", "euv_kernel_launches",
    "euv_mask_spectrum_workspace_bytes", "euv_mask_spectrum",
    "euv_amp_workspace_bytes", "euv_amp", "euv_amp_euler_factors",
    "euv_abbe", "euv_m3d_fit",
    "euv_zgemm", "euv_zgemm_mixed_workspace_bytes", "euv_zgemm_mixed", "euv_lu_workspace_bytes", "euv_lu_factor", "euv_lu_solve",
    "euv_matfun_workspace_bytes", "euv_matfun_cs", "euv_matfun_cs_noalloc",
    "euv_wait_probe", "euv_linear_amp", "euv_mask_raster_workspace_bytes", "euv_mask_raster",
    "euv_heev_workspace_bytes", "euv_heev", "euv_socs_workspace_bytes", "euv_socs_image",
    "euv_cnn_blob_bytes", "euv_cnn_pack", "euv_cnn_workspace_bytes", "euv_cnn_predict",
    "euv_cnn_downsample",
    "euv_config_reference", "euv_plan_create", "euv_plan_destroy", "euv_plan_get_info",
    "euv_plan_get_orders", "euv_plan_get_pupil", "euv_plan_get_sources",
    "euv_plan_get_na_sources", "euv_plan_get_abbe_table", "euv_plan_device_bytes",
    "euv_plan_upload", "euv_plan_check", "euv_plan_intensity_workspace_bytes",
    "euv_plan_intensity", "euv_plan_amp_workspace_bytes", "euv_plan_amp",
    "euv_plan_m3d_workspace_bytes", "euv_plan_m3d",
    "euv_tune_set", "euv_tune_get", "euv_tune_clear",
)
EUV_KNOB_ABBE_SPLIT = 1
EUV_KNOB_LU_CLUSTER = 2
EUV_KNOB_ZGEMM_ROWS = 3
EUV_KNOB_LU_SUBST_COLS = 4
EUV_ORDERS_DIAMOND = 0
EUV_ORDERS_ELLIPSE = 1
EUV_ORDERS_BOX = 2


class EuvError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__("%s failed (status %d): %s" % (fn, code, msg))
        self.code = code


class c64(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]

    @classmethod
    def of(cls, z) -> "c64":
        z = complex(z)
        return cls(z.real, z.imag)


class Stack(C.Structure):
    _fields_ = [
        ("eps_mo", c64), ("eps_si", c64), ("eps_ru", c64), ("eps_mosi2", c64),
        ("eps_rusi", c64), ("eps_sio2", c64),
        ("d_mo", C.c_double), ("d_mosi", C.c_double), ("d_si", C.c_double),
        ("d_simo", C.c_double), ("d_siru", C.c_double), ("d_ru", C.c_double),
        ("nml", C.c_int),
    ]


P = C.c_void_p


class AmpDesc(C.Structure):
    _fields_ = [
        ("n_orders", C.c_int), ("lmax", C.c_int), ("mmax", C.c_int),
        ("d_lindex", P), ("d_mindex", P),
        ("dx", C.c_double), ("dy", C.c_double), ("k", C.c_double),
        ("n_slices", C.c_int),
        ("eabs", c64 * EUV_MAX_SLICES), ("dabs", C.c_double * EUV_MAX_SLICES),
        ("refresh_sigma", C.c_int),
        ("stack", Stack),
        ("n_units", C.c_int),
        ("d_kx0", P), ("d_ky0", P), ("d_polar", P), ("d_spec", P),
        ("n_src", C.c_int), ("d_src_order", P), ("d_src_2kz", P),
        ("precision", C.c_int), ("m_max", C.c_int), ("k0_max", C.c_double),
        ("d_status", P), ("d_dx", P), ("d_dy", P), ("euler_f", C.c_int),
    ]


class AbbeDesc(C.Structure):
    _fields_ = [
        ("xdiv", C.c_int), ("ydiv", C.c_int), ("lpx", C.c_int), ("lpy", C.c_int),
        ("ncut", C.c_int), ("n_units", C.c_int), ("n_src", C.c_int), ("n_order", C.c_int),
        ("d_coef", P), ("d_nidx", P), ("d_px", P), ("d_py", P), ("d_row_start", P),
        ("d_tab_of_unit", P), ("d_img_of_unit", P), ("d_nsrc_of_unit", P),
        ("n_images", C.c_int), ("d_inv_weight", P), ("precision", C.c_int),
    ]


class M3dDesc(C.Structure):
    _fields_ = [
        ("n_clips", C.c_int), ("n_src", C.c_int), ("ninput", C.c_int), ("n_order", C.c_int),
        ("n_order_narrow", C.c_int), ("lpx", C.c_int), ("lpy", C.c_int),
        ("k", C.c_double), ("dx", C.c_double), ("dy", C.c_double), ("z0", C.c_double),
        ("kx0", C.c_double), ("ky0", C.c_double),
        ("s_center", C.c_int),
        ("d_src_l", P), ("d_src_m", P), ("d_src_nidx_narrow", P),
        ("d_ax_vc", P), ("d_ax_ab", P),
        ("d_lin", P), ("d_min", P), ("d_xin", P), ("d_pair_order", P),
    ]


class LinearDesc(C.Structure):
    _fields_ = [
        ("n_clips", C.c_int), ("n_src", C.c_int), ("ncut", C.c_int), ("lpx", C.c_int),
        ("lpy", C.c_int), ("d_lp", P), ("d_mp", P), ("d_ls", P), ("d_ms", P),
        ("k", C.c_double), ("dx", C.c_double), ("dy", C.c_double), ("kx0", C.c_double),
        ("ky0", C.c_double), ("z0", C.c_double), ("amp_vc", c64), ("amp_ab", c64),
    ]


class SocsDesc(C.Structure):
    _fields_ = [
        ("n_clips", C.c_int), ("ncut", C.c_int), ("lpx", C.c_int), ("lpy", C.c_int),
        ("nsocs", C.c_int), ("nsocsxy", C.c_int), ("nout", C.c_int), ("xdiv", C.c_int),
        ("ydiv", C.c_int), ("d_lp", P), ("d_mp", P),
        ("k", C.c_double), ("dx", C.c_double), ("dy", C.c_double), ("kx0", C.c_double),
        ("ky0", C.c_double), ("z0", C.c_double), ("amp_vc", c64), ("amp_ab", c64),
        ("d_phi_s0", P), ("d_phi_sx", P), ("d_phi_sy", P),
        ("d_alpha_s0", P), ("d_alpha_sx", P), ("d_alpha_sy", P),
        ("d_e", P), ("d_kxT", P), ("d_ky", P),
    ]


EUV_CNN_MAX_MODELS = 6
EUV_CNN_MAX_OUT = 8192


class CnnModelWeights(C.Structure):
    _fields_ = [
        ("conv_w", P * 5), ("conv_b", P * 5), ("bn_w", P * 5), ("bn_b", P * 5),
        ("bn_mean", P * 5), ("bn_var", P * 5),
        ("fc1_w", P), ("fc1_b", P), ("fc2_w", P), ("fc2_b", P), ("n_out", C.c_int),
    ]


class CnnDesc(C.Structure):
    _fields_ = [
        ("n_models", C.c_int), ("n_masks", C.c_int), ("max_out", C.c_int),
        ("n_out", C.c_int * EUV_CNN_MAX_MODELS), ("d_factors", P), ("d_status", P),
    ]


class Config(C.Structure):
    """euv_config: the driver constants of intensity.cpp / m3d.cpp as parameters."""
    _fields_ = [
        ("ndivx", C.c_int), ("ndivy", C.c_int), ("delta", C.c_double),
        ("wavelength", C.c_double), ("theta0", C.c_double), ("azimuth", C.c_double),
        ("na", C.c_double), ("mx", C.c_int), ("my", C.c_int), ("illum_type", C.c_int),
        ("sigma1", C.c_double), ("sigma2", C.c_double), ("openangle", C.c_double),
        ("sigmadiv", C.c_double), ("ndivs", C.c_int), ("max_sources", C.c_int),
        ("n_slices", C.c_int), ("eabs", c64 * EUV_MAX_SLICES),
        ("dabs", C.c_double * EUV_MAX_SLICES), ("z0_offset", C.c_double), ("stack", Stack),
        ("refresh_sigma", C.c_int), ("order_kind", C.c_int), ("cut", C.c_double),
        ("lbox", C.c_int), ("mbox", C.c_int), ("z", C.c_double), ("yflip_offset", C.c_int),
        ("n_pols", C.c_int), ("pols", C.c_int * 2), ("precision", C.c_int),
    ]


class PlanInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "n_orders", "lmax", "mmax", "ncut", "lpx", "lpy", "lsx", "lsy", "n_na_sources", "ndivs",
        "n_families", "n_src_max", "sdivsum", "n_pols", "units_per_clip", "xdiv", "ydiv",
        "fdivx", "fdivy", "n_orders_narrow")] + [
        ("k", C.c_double), ("kx0", C.c_double), ("ky0", C.c_double), ("z0", C.c_double)]


_lib: Optional[C.CDLL] = None


def _declare(lib: C.CDLL) -> None:
    i, d, sz, ll = C.c_int, C.c_double, C.c_size_t, C.c_longlong
    lib.euv_version.restype = C.c_char_p
    lib.euv_last_error.restype = C.c_char_p
    lib.euv_kernel_launches.restype = C.c_ulonglong
    lib.euv_mask_spectrum_workspace_bytes.restype = sz
    lib.euv_mask_spectrum_workspace_bytes.argtypes = [i] * 7
    lib.euv_mask_spectrum.restype = i
    lib.euv_mask_spectrum.argtypes = [P, i, i, i, i, i, i, i, i, i, P, P, sz, P]
    lib.euv_amp_workspace_bytes.restype = sz
    lib.euv_amp_workspace_bytes.argtypes = [C.POINTER(AmpDesc)]
    lib.euv_amp_euler_factors.restype = i
    lib.euv_amp_euler_factors.argtypes = [C.POINTER(AmpDesc)]
    lib.euv_amp.restype = i
    lib.euv_amp.argtypes = [C.POINTER(AmpDesc), P, P, P, sz, P]
    lib.euv_abbe.restype = i
    lib.euv_abbe.argtypes = [C.POINTER(AbbeDesc), P, P, P]
    lib.euv_m3d_fit.restype = i
    lib.euv_m3d_fit.argtypes = [C.POINTER(M3dDesc), P, P, P, P, P, P]
    lib.euv_zgemm.restype = i
    lib.euv_zgemm.argtypes = [i, i, i, c64, P, P, i, ll, P, i, ll, c64, P, i, ll, c64, i, P, i, P]
    lib.euv_zgemm_mixed_workspace_bytes.restype = sz
    lib.euv_zgemm_mixed_workspace_bytes.argtypes = [i, i, i, i]
    lib.euv_zgemm_mixed.restype = i
    lib.euv_zgemm_mixed.argtypes = [i, i, i, c64, P, P, i, ll, P, i, ll, c64, P, i, ll, c64, i, P, i, P, sz,
                                     P, P]
    lib.euv_lu_workspace_bytes.restype = sz
    lib.euv_lu_workspace_bytes.argtypes = [i, i]
    lib.euv_lu_factor.restype = i
    lib.euv_lu_factor.argtypes = [i, P, i, ll, P, P, i, P]
    lib.euv_lu_solve.restype = i
    lib.euv_lu_solve.argtypes = [i, i, P, i, ll, P, P, i, ll, i, P]
    lib.euv_matfun_workspace_bytes.restype = sz
    lib.euv_matfun_workspace_bytes.argtypes = [i, i]
    lib.euv_matfun_cs.restype = i
    lib.euv_matfun_cs.argtypes = [i, P, P, P, P, i, i, i, P, sz, P]
    lib.euv_matfun_cs_noalloc.restype = i
    lib.euv_matfun_cs_noalloc.argtypes = [i, P, P, P, P, i, i, P]
    lib.euv_wait_probe.restype = i
    lib.euv_linear_amp.restype = i
    lib.euv_mask_raster_workspace_bytes.restype = sz
    lib.euv_mask_raster_workspace_bytes.argtypes = [i, i, i]
    lib.euv_mask_raster.restype = i
    lib.euv_heev_workspace_bytes.restype = sz
    lib.euv_heev_workspace_bytes.argtypes = [i]
    lib.euv_heev.restype = i
    lib.euv_socs_workspace_bytes.restype = sz
    lib.euv_socs_workspace_bytes.argtypes = [C.POINTER(SocsDesc)]
    lib.euv_socs_image.restype = i
    lib.euv_socs_image.argtypes = [C.POINTER(SocsDesc), P, P, P, P, P, P, sz, P]
    lib.euv_heev.argtypes = [i, P, i, P, P, i, i, d, P, sz, P, P]
    lib.euv_mask_raster.argtypes = [i, i, i, i, P, i, P, P, P, sz, P]
    lib.euv_linear_amp.argtypes = [C.POINTER(LinearDesc), P, P, P, P, P, P]
    lib.euv_wait_probe.argtypes = [P, ll, P, P]
    lib.euv_cnn_blob_bytes.restype = sz
    lib.euv_cnn_blob_bytes.argtypes = [i, i]
    lib.euv_cnn_pack.restype = i
    lib.euv_cnn_pack.argtypes = [i, C.POINTER(CnnModelWeights), i, d, P, sz, P]
    lib.euv_cnn_workspace_bytes.restype = sz
    lib.euv_cnn_workspace_bytes.argtypes = [i, i, i]
    lib.euv_cnn_predict.restype = i
    lib.euv_cnn_predict.argtypes = [C.POINTER(CnnDesc), P, P, P, P, sz, P]
    lib.euv_cnn_downsample.restype = i
    lib.euv_cnn_downsample.argtypes = [i, P, P, P]
    lib.euv_tune_set.restype = i
    lib.euv_tune_set.argtypes = [i, i, i, i]
    lib.euv_tune_get.restype = i
    lib.euv_tune_get.argtypes = [i, i, i]
    lib.euv_tune_clear.restype = None
    lib.euv_tune_clear.argtypes = []
    PP = C.POINTER(P)
    lib.euv_config_reference.restype = None
    lib.euv_config_reference.argtypes = [C.POINTER(Config)]
    lib.euv_plan_create.restype = i
    lib.euv_plan_create.argtypes = [C.POINTER(Config), PP]
    lib.euv_plan_destroy.restype = None
    lib.euv_plan_destroy.argtypes = [P]
    lib.euv_plan_get_info.restype = i
    lib.euv_plan_get_info.argtypes = [P, C.POINTER(PlanInfo)]
    for fn, n in (("euv_plan_get_orders", 2), ("euv_plan_get_pupil", 3),
                  ("euv_plan_get_sources", 5), ("euv_plan_get_na_sources", 2)):
        getattr(lib, fn).restype = i
        getattr(lib, fn).argtypes = [P] + [P] * n
    lib.euv_plan_get_abbe_table.restype = i
    lib.euv_plan_get_abbe_table.argtypes = [P, i, P, P]
    lib.euv_plan_device_bytes.restype = sz
    lib.euv_plan_device_bytes.argtypes = [P, i]
    lib.euv_plan_upload.restype = i
    lib.euv_plan_upload.argtypes = [P, i, P, sz, P]
    lib.euv_plan_check.restype = i
    lib.euv_plan_check.argtypes = [P, P, P]
    for fn in ("euv_plan_intensity_workspace_bytes", "euv_plan_amp_workspace_bytes",
               "euv_plan_m3d_workspace_bytes"):
        getattr(lib, fn).restype = sz
        getattr(lib, fn).argtypes = [P, i, i]
    lib.euv_plan_intensity.restype = i
    lib.euv_plan_intensity.argtypes = [P, P, i, i, P, P, sz, P]
    lib.euv_plan_amp.restype = i
    lib.euv_plan_amp.argtypes = [P, i, d, d, P, i, i, P, P, sz, P]
    lib.euv_plan_m3d.restype = i
    lib.euv_plan_m3d.argtypes = [P, P, i, i, P, P, P, P, sz, P]


def lib() -> C.CDLL:
    """Load the shared library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libeuvl_b200.so not found at %s; build it with `python -m euvlitho_b200.build`"
                % LIB_PATH)
        l = C.CDLL(LIB_PATH)
        _declare(l)
        _lib = l
    return _lib


def check(fn: str, rc: int) -> None:
    if rc != EUV_OK:
        raise EuvError(fn, rc, lib().euv_last_error().decode(errors="replace"))


def call(fn: str, *args) -> None:
    check(fn, getattr(lib(), fn)(*args))


_STATUS_TEXT = (
    (EUV_STATUS_TIMEOUT, "a bounded device wait gave up (results incomplete)"),
    (EUV_STATUS_STEPS_CLAMPED, "a unit needed more double-angle steps than m_max"),
    (EUV_STATUS_SINGULAR, "an LU met an exactly zero pivot"),
    (EUV_STATUS_NOT_CONVERGED, "an eigensolver stopped at its sweep limit"),
)


def status_message(bits: int) -> Optional[str]:
    """Text for the EUV_STATUS_* bits of a device status word (None if clear)."""
    if not bits:
        return None
    parts = [t for b, t in _STATUS_TEXT if bits & b]
    rest = bits & ~sum(b for b, _ in _STATUS_TEXT)
    if rest:
        parts.append("unknown bits 0x%x" % rest)
    return "; ".join(parts)


def check_status(where: str, bits: int) -> None:
    """Raise EuvError if a device status word has any bit set."""
    msg = status_message(int(bits))
    if msg is not None:
        code = EUV_ERR_TIMEOUT if bits & EUV_STATUS_TIMEOUT else (
            EUV_ERR_SINGULAR if bits & EUV_STATUS_SINGULAR else EUV_ERR_CUDA)
        raise EuvError(where, code, "device status 0x%x: %s" % (int(bits), msg))


_ORDER_KIND = {"diamond": EUV_ORDERS_DIAMOND, "ellipse": EUV_ORDERS_ELLIPSE, "box": EUV_ORDERS_BOX}


def config_struct(cfg, pols=("X",), precision: int = EUV_PREC_FP64) -> Config:
    """euv_config of a SimConfig (the same fields; permittivities as given)."""
    c = Config()
    c.ndivx, c.ndivy, c.delta, c.wavelength = cfg.ndivx, cfg.ndivy, cfg.delta, cfg.wavelength
    c.theta0, c.azimuth, c.na, c.mx, c.my = cfg.theta0, cfg.azimuth, cfg.na, cfg.mx, cfg.my
    c.illum_type, c.sigma1, c.sigma2 = cfg.illum_type, cfg.sigma1, cfg.sigma2
    c.openangle, c.sigmadiv = cfg.openangle, cfg.sigmadiv
    c.ndivs = 0 if cfg.ndivs is None else int(cfg.ndivs)
    c.max_sources = 0 if cfg.max_sources is None else int(cfg.max_sources)
    c.n_slices = cfg.nabs
    for n in range(cfg.nabs):
        c.eabs[n] = c64.of(cfg.eabs[n])
        c.dabs[n] = float(cfg.dabs[n])
    c.z0_offset = cfg.z0_offset
    st = cfg.stack
    c.stack = Stack(c64.of(st.n_mo ** 2), c64.of(st.n_si ** 2), c64.of(st.n_ru ** 2),
                    c64.of(st.n_mosi2 ** 2), c64.of(st.n_rusi ** 2), c64.of(st.n_sio2 ** 2),
                    st.d_mo, st.d_mosi, st.d_si, st.d_simo, st.d_siru, st.d_ru, st.nml)
    c.refresh_sigma = 1 if cfg.refresh_sigma else 0
    c.order_kind = _ORDER_KIND[cfg.order_kind]
    c.cut, c.lbox, c.mbox, c.z = cfg.cut, cfg.lbox, cfg.mbox, float(cfg.z)
    c.yflip_offset = cfg.yflip_offset
    c.n_pols = len(pols)
    for i, p in enumerate(pols):
        c.pols[i] = {"X": 0, "Y": 1}[p]
    c.precision = precision
    return c
