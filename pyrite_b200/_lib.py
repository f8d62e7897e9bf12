"""ctypes binding of ``libpyrite_b200.so`` (the C ABI in ``include/pyrite_b200.h``).

The structures below mirror the header field for field. Loading fails loudly
when the shared library is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libpyrite_b200.so"

PB_OK = 0
PB_ERR_INVALID, PB_ERR_CUDA, PB_ERR_UNSUPPORTED, PB_ERR_CAPACITY = 1, 2, 3, 4
PB_RNG_SPLITMIX, PB_RNG_PHILOX = 0, 1
PB_FP64, PB_MIXED = 0, 1
PB_BEAM_EXPLICIT, PB_BEAM_SPOT, PB_BEAM_TWISS = 0, 1, 2
PB_QUAD_NODE, PB_QUAD_BINMEAN = 0, 1
PB_DEV_STEP_LIMIT, PB_DEV_ROW_OVERFLOW, PB_DEV_QUEUE_OVERFLOW = 1, 2, 4
PB_DEV_WAIT_TIMEOUT, PB_DEV_BAD_INPUT = 8, 16
PB_ELASTIC_SR, PB_ELASTIC_ELSEPA = 0, 2

_vp = C.c_void_p
_i32, _i64, _u64, _f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_double


class PbLayers(C.Structure):
    _fields_ = [
        ("n_layers", _i32), ("max_el", _i32), ("z_top", _vp), ("z_bot", _vp), ("n_el", _vp),
        ("J", _vp), ("k", _vp), ("coeff", _vp), ("E_cross", _vp), ("sr_rate_numer", _vp),
        ("sr_joy_numer", _vp),
    ]


class PbLut(C.Structure):
    _fields_ = [
        ("n_energy", _i32), ("elem_bytes", _i32), ("log_E_min", _f64), ("inv_dlogE", _f64),
        ("base", _vp), ("total_bytes", _i64), ("off_total_rate", _i64), ("off_dEds", _i64),
        ("off_inv_beta", _i64), ("off_cdf", _i64), ("off_alpha", _i64),
    ]


class PbBeam(C.Structure):
    _fields_ = [
        ("mode", _i32), ("tilted", _i32), ("E0_keV", _f64), ("beam_dir", _f64 * 3),
        ("e_x", _f64 * 3), ("e_y", _f64 * 3), ("basis", _f64 * 9), ("sigma_x_ang", _f64),
        ("sigma_y_ang", _f64), ("twiss_x", _f64 * 3), ("twiss_y", _f64 * 3), ("root", _u64),
        ("pos0", _vp), ("dir0", _vp), ("E0", _vp),
    ]


class PbRows(C.Structure):
    _fields_ = [
        ("r_mid", _vp), ("v_hat", _vp), ("L", _vp), ("E_start", _vp), ("E_end", _vp),
        ("t_start", _vp), ("t_end", _vp), ("elec_id", _vp), ("layer", _vp), ("flight", _vp),
        ("event", _vp),
    ]


class PbSegments(C.Structure):
    _fields_ = [
        ("capacity", _i64), ("count", _vp), ("r_mid", _vp), ("v_hat", _vp), ("L", _vp),
        ("E_repr", _vp), ("elec_id", _vp), ("layer", _vp),
    ]


class PbTallies(C.Structure):
    _fields_ = [
        ("fates", _vp), ("exit_E", _vp), ("n_E", _i32), ("E_lo", _f64), ("E_hi", _f64),
        ("exit_theta", _vp), ("n_theta", _i32), ("theta_lo", _f64), ("theta_hi", _f64),
        ("deposit", _vp),
    ]


class PbElsepa(C.Structure):
    _fields_ = [
        ("n_mu", _i32), ("cells", _i32), ("start", _vp), ("length", _vp), ("logE", _vp), ("log_rate", _vp),
        ("cdf", _vp), ("pdf", _vp), ("mu", _vp), ("guide", _vp),
    ]


class PbStopping(C.Structure):
    _fields_ = [("width", _i32), ("count", _vp), ("logE", _vp), ("logS", _vp)]


class PbTransportArgs(C.Structure):
    _fields_ = [
        ("rng", _i32), ("precision", _i32), ("use_lut", _i32), ("block_threads", _i32),
        ("seed", _u64), ("e_start", _i64), ("n", _i64), ("E_cut_keV", _f64), ("max_steps", _i64),
        ("layers", PbLayers), ("lut", PbLut), ("beam", PbBeam), ("cap", _i64), ("rows", PbRows),
        ("seg_count", _vp), ("exit_code", _vp), ("final_pos", _vp), ("final_dir", _vp),
        ("final_E", _vp), ("seg", PbSegments), ("tallies", PbTallies), ("work_counter", _vp),
        ("status", _vp), ("straggling", _i32), ("Z", _vp), ("elastic_model", _i32), ("elsepa", PbElsepa),
        ("stopping", PbStopping),
    ]


class PbCxrTables(C.Structure):
    _fields_ = [
        ("n_g", _i32), ("G", _vp), ("ES", _vp), ("EP", _vp), ("WM", _vp), ("row_table", _vp),
        ("n_tab", _i32), ("E_tab", _vp), ("chi_re", _vp), ("chi_im", _vp), ("u_re", _vp),
        ("u_im", _vp), ("n_mu", _i32), ("log_mu", _vp), ("delta", _vp), ("lo_keep", _f64),
        ("hi_keep", _f64), ("tab_log0", _f64), ("tab_log_step", _f64),
        ("delta_tail_absmax", _vp),
    ]


class PbCxrArgs(C.Structure):
    _fields_ = [
        ("precision", _i32), ("quadrature", _i32), ("n_dir", _i32), ("n_hat", _vp),
        ("thickness", _f64), ("Ne", _i64), ("n_seg", _i64), ("r_mid", _vp), ("v_hat", _vp),
        ("L", _vp), ("E_keV", _vp), ("elec_id", _vp), ("n_seg_device", _vp),
        ("tables", PbCxrTables), ("n_E", _i32), ("E_grid", _vp), ("edges", _vp),
        ("exact_widths", _f64), ("far_pad", _i32), ("spec", _vp), ("far_moments", _vp),
        ("line_capacity", _i64), ("line_count", _vp), ("line_E", _vp), ("line_a", _vp),
        ("line_w", _vp), ("line_dir", _vp), ("pair_E", _vp), ("pair_a", _vp), ("pair_w", _vp),
        ("pair_good", _vp), ("status", _vp), ("line_seg", _vp),
        ("n_layer", _i32), ("z_top", _vp), ("z_bot", _vp), ("mu_off", _vp), ("mu_knot", _vp),
        ("mu_value", _vp), ("mu_slope", _vp), ("seg_layer", _vp), ("emit_layer", _i32), ("counters", _vp),
    ]


class PbBremArgs(C.Structure):
    _fields_ = [
        ("precision", _i32), ("n_dir", _i32), ("n_hat", _vp), ("thickness", _f64), ("Ne", _i64),
        ("n_seg", _i64), ("r_mid", _vp), ("v_hat", _vp), ("L", _vp), ("E_keV", _vp),
        ("elec_id", _vp), ("n_seg_device", _vp), ("n_el", _i32), ("Z", _vp), ("n_ang3", _vp),
        ("n_E", _i32), ("E_grid", _vp), ("mu", _vp), ("spec", _vp), ("status", _vp),
        ("n_layer", _i32), ("z_top", _vp), ("z_bot", _vp), ("mu_layer", _vp), ("seg_layer", _vp),
        ("emit_layer", _i32), ("work", _vp), ("work_bytes", _i64),
    ]


class PbCharArgs(C.Structure):
    _fields_ = [
        ("precision", _i32), ("n_dir", _i32), ("n_hat", _vp), ("thickness", _f64), ("n_layer", _i32),
        ("z_top", _vp), ("z_bot", _vp), ("Ne", _i64), ("n_seg", _i64), ("r_mid", _vp), ("v_hat", _vp),
        ("L", _vp), ("E_keV", _vp), ("elec_id", _vp), ("n_seg_device", _vp), ("n_atoms", _f64),
        ("n_shell", _i32), ("shell_E", _vp), ("shell_sigma", _vp), ("shell_offset", _vp), ("n_line", _i32),
        ("response", _vp), ("mu", _vp), ("line_yield", _vp), ("status", _vp),
        ("seg_layer", _vp), ("emit_layer", _i32),
    ]


class PbMlpGemmArgs(C.Structure):
    _fields_ = [
        ("M", _i32), ("N", _i32), ("K", _i32), ("A", _vp), ("lda", _i64), ("B", _vp), ("ldb", _i64),
        ("bias", _vp), ("act", _i32), ("dsilu_z", _vp), ("ldz", _i64), ("out_f32", _vp), ("ldc", _i64),
        ("beta", C.c_float), ("out_bf16", _vp), ("ldh", _i64), ("out_bf16_t", _vp), ("ldt", _i64), ("status", _vp),
    ]


class PbMlpInferArgs(C.Structure):
    _fields_ = [
        ("n_dir", _i32), ("dir_uv", _vp), ("e_x", _f64 * 3), ("e_y", _f64 * 3), ("theta_max", _f64),
        ("E_lo_MeV", _f64), ("E_hi_MeV", _f64), ("thickness", _f64), ("Ne", _i64), ("n_seg", _i64),
        ("r_mid", _vp), ("v_hat", _vp), ("L", _vp), ("E_keV", _vp), ("elec_id", _vp), ("n_seg_device", _vp),
        ("w1_packed", _vp), ("w_packed", _vp * 3), ("bias", _vp * 4), ("hsum", _vp), ("lsum", _vp),
        ("status", _vp),
    ]


class PbCoherentArgs(C.Structure):
    _fields_ = [
        ("n_row", _i32), ("n_E", _i32), ("n_line", _i64), ("row_off", _vp), ("row_weight", _vp),
        ("E", _vp), ("delta_omega", _vp), ("E_vac", _vp), ("a_vac", _vp), ("phase_slope", _vp),
        ("g_phase", _vp), ("cs_re", _vp), ("cs_im", _vp), ("cp_re", _vp), ("cp_im", _vp), ("L_esc", _vp),
        ("half_dL", _vp), ("apb", _vp), ("bma", _vp), ("q", _vp), ("scale", _f64), ("sinc_cutoff", _f64), ("spec", _vp),
        ("work", _vp), ("work_bytes", _u64), ("status", _vp),
    ]


class PbCoherentRecordsArgs(C.Structure):
    _fields_ = [
        ("cxr", PbCxrArgs), ("t_start", _vp), ("capacity", _i64), ("E_vac", _vp), ("a_vac", _vp),
        ("phase_slope", _vp), ("g_phase", _vp), ("cs_re", _vp), ("cs_im", _vp), ("cp_re", _vp), ("cp_im", _vp),
        ("L_esc", _vp), ("half_dL", _vp), ("apb", _vp), ("bma", _vp), ("q", _vp), ("row_off", _vp),
        ("work", _vp), ("work_bytes", _u64), ("status", _vp), ("elec_out", _vp),
    ]


class PbTransportScoreArgs(C.Structure):
    _fields_ = [
        ("transport", PbTransportArgs), ("n_cxr", _i32), ("n_brem", _i32), ("n_char", _i32), ("pad_", _i32),
        ("cxr", C.POINTER(PbCxrArgs)), ("brem", C.POINTER(PbBremArgs)), ("chars", C.POINTER(PbCharArgs)),
    ]


class PbCoherentStreamArgs(C.Structure):
    _fields_ = [("base", PbCoherentArgs), ("elec_id", _vp), ("fields", _vp), ("power", _vp)]


class PbDecoherenceArgs(C.Structure):
    _fields_ = [
        ("n_row", _i32), ("n_pop", _i32), ("n_E", _i32), ("pad_", _i32), ("G", _vp), ("A_pop", _vp),
        ("xy0_pop", _vp), ("omega", _vp), ("F", _vp),
    ]


class PbCoherentBlendArgs(C.Structure):
    _fields_ = [("base", PbCoherentArgs), ("elec_id", _vp), ("F_row", _vp)]


# Exported symbols declared by include/pyrite_b200.h, checked by the tests.
EXPORTS = (
    "pb_abi_version",
    "pb_last_error",
    "pb_device_count",
    "pb_transport",
    "pb_cxr_score",
    "pb_brem_score",
    "pb_brem_work_size",
    "pb_copy_segments",
    "pb_cxr_score_noalloc",
    "pb_char_yields",
    "pb_char_spectrum",
    "pb_mlp_gemm",
    "pb_mlp_mse_grad",
    "pb_mlp_group_mse_grad",
    "pb_mlp_colsum",
    "pb_mlp_adam",
    "pb_mlp_pack",
    "pb_mlp_infer",
    "pb_segments_sample",
    "pb_mlp_head",
    "pb_mlp_pack_umma",
    "pb_mlp_features",
    "pb_cxr_bin_lines",
    "pb_coherent_work_size",
    "pb_coherent_reduce",
    "pb_coherent_records_work_size",
    "pb_coherent_records",
    "pb_decoherence_factor",
    "pb_transport_score",
    "pb_coherent_accumulate",
    "pb_coherent_finalize",
    "pb_coherent_blend_work_size",
    "pb_coherent_blend",
)

_lib = None


class PyriteB200Error(RuntimeError):
    """A pyrite_b200 C-ABI call returned a non-zero status."""


ABI_VERSION = 6  # PB_ABI_VERSION of include/pyrite_b200.h


def load(path: Path | None = None):
    """Load the shared library (once); raise if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.is_file():
        raise PyriteB200Error(
            f"{p} is missing: build the CUDA extension first (python -m pyrite_b200.build)"
        )
    lib = C.CDLL(str(p))
    lib.pb_abi_version.restype = C.c_int
    if lib.pb_abi_version() != ABI_VERSION:
        raise PyriteB200Error(
            f"{p} has ABI {lib.pb_abi_version()}, this binding expects {ABI_VERSION}: rebuild it"
        )
    lib.pb_last_error.restype = C.c_char_p
    lib.pb_device_count.argtypes = [C.POINTER(C.c_int)]
    lib.pb_transport.argtypes = [C.POINTER(PbTransportArgs), _vp]
    lib.pb_cxr_score.argtypes = [C.POINTER(PbCxrArgs), _vp]
    lib.pb_brem_score.argtypes = [C.POINTER(PbBremArgs), _vp]
    lib.pb_brem_work_size.argtypes = [C.POINTER(PbBremArgs), C.POINTER(_i64)]
    lib.pb_copy_segments.argtypes = [_i32, _vp, _vp]
    lib.pb_cxr_score_noalloc.argtypes = [C.POINTER(PbCxrArgs), _vp]
    lib.pb_char_yields.argtypes = [C.POINTER(PbCharArgs), _vp]
    lib.pb_char_spectrum.argtypes = [_i32, _i32, _i32, _vp, _vp, _vp, _vp]
    _f32 = C.c_float
    lib.pb_mlp_gemm.argtypes = [C.POINTER(PbMlpGemmArgs), _vp]
    lib.pb_mlp_mse_grad.argtypes = [_i32, _i32, _vp, _vp, _i64, _f32, _f32, _vp, _vp, _i64, _vp, _vp]
    lib.pb_mlp_colsum.argtypes = [_i32, _i32, _vp, _i64, _vp, _vp]
    lib.pb_mlp_group_mse_grad.argtypes = [_i32, _i32, _i32, _vp, _vp, _i64, _vp, _f32, _f32, _vp, _vp, _i64, _vp, _vp]
    lib.pb_mlp_adam.argtypes = [_i64, _vp, _vp, _vp, _vp, _f32, _f32, _f32, _f32, _f32, _f32, _f32, _vp]
    lib.pb_mlp_pack.argtypes = [_i32, _i32, _vp, _vp, _i32, _vp, _i32, _i32, _vp]
    lib.pb_mlp_infer.argtypes = [C.POINTER(PbMlpInferArgs), _vp]
    lib.pb_segments_sample.argtypes = [C.POINTER(PbSegments), _i64, C.POINTER(PbSegments), _vp, _vp]
    lib.pb_mlp_features.argtypes = [C.POINTER(PbMlpInferArgs), _vp, _vp, _vp]
    lib.pb_mlp_head.argtypes = [_i32, _i32, _vp, _vp, _vp, _vp, _f64, _vp, _vp]
    lib.pb_mlp_pack_umma.argtypes = [_i32, _i32, _vp, _vp, _vp]
    lib.pb_cxr_bin_lines.argtypes = [_i64, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _i64, _f64, _f64, _i32, _vp, _vp]
    lib.pb_coherent_work_size.argtypes = [_i32, _i64, _i32, C.POINTER(_u64)]
    lib.pb_coherent_reduce.argtypes = [C.POINTER(PbCoherentArgs), _vp]
    lib.pb_coherent_records_work_size.argtypes = [_i64, _i32, C.POINTER(_u64)]
    lib.pb_coherent_records.argtypes = [C.POINTER(PbCoherentRecordsArgs), _vp]
    lib.pb_decoherence_factor.argtypes = [C.POINTER(PbDecoherenceArgs), _vp]
    lib.pb_transport_score.argtypes = [C.POINTER(PbTransportScoreArgs), _vp]
    lib.pb_coherent_accumulate.argtypes = [C.POINTER(PbCoherentStreamArgs), _vp]
    lib.pb_coherent_finalize.argtypes = [_i32, _i32, _vp, _vp, _vp, _vp, _f64, _vp, _vp]
    lib.pb_coherent_blend_work_size.argtypes = [_i32, _i64, _i32, C.POINTER(_u64)]
    lib.pb_coherent_blend.argtypes = [C.POINTER(PbCoherentBlendArgs), _vp]
    if path is None:
        _lib = lib
    return lib


def check(status: int, what: str) -> None:
    if status != PB_OK:
        msg = load().pb_last_error().decode(errors="replace")
        raise PyriteB200Error(f"{what} failed with status {status}: {msg}")
