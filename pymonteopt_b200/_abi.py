"""ctypes mirror of ``include/pmo_b200.h``.

The constants and struct layouts here must match the C header; a CPU test
parses the header and compares every ``#define`` and field.
"""
from __future__ import annotations

import ctypes as C

PMO_ABI_VERSION = 1

# status codes
PMO_OK = 0
PMO_ERR_ARG = 1
PMO_ERR_GEOMETRY = 2
PMO_ERR_LABEL = 3
PMO_ERR_STEP_CAP = 4
PMO_ERR_CUDA = 5
PMO_ERR_WORKSPACE = 6
PMO_ERR_TIMEOUT = 7
PMO_ERR_NUMERIC = 8

PMO_FP32 = 0
PMO_FP64 = 1

PMO_SRC_PENCIL = 0
PMO_SRC_GAUSSIAN = 1
PMO_SRC_STATE = 2

PMO_PROPS_LABEL = 0
PMO_PROPS_VOXEL = 1

PMO_FLU_NONE = 0
PMO_FLU_GLOBAL = 1
PMO_FLU_SHARED = 2
PMO_ABSORBED_SHIFT = 32

PMO_L_WINIT = 0
PMO_L_RD = 1
PMO_L_TT = 2
PMO_L_EXIT0 = 3
PMO_L_ABS = 4
PMO_L_RGAIN = 5
PMO_L_RLOSS = 6
PMO_L_ERRW = 7
PMO_L_RD_TOP = 8
PMO_L_TT_BOTTOM = 9
PMO_L_SPEC = 10
PMO_LEDGER_N = 16

PMO_C_PHOTONS = 0
PMO_C_INTERACT = 1
PMO_C_CROSS = 2
PMO_C_FRESNEL = 3
PMO_C_REFLECT = 4
PMO_C_ROULETTE = 5
PMO_C_EXITS = 6
PMO_C_ERR_GEOM = 7
PMO_C_ERR_LABEL = 8
PMO_C_ERR_CAP = 9
PMO_C_ERR_NUM = 10
PMO_C_SAMECROSS = 11
PMO_C_XDRAWS = 12
PMO_COUNTERS_N = 16

PMO_RR_TOP = 0
PMO_RR_BOTTOM = 1
PMO_RR_LAT_NEG = 2
PMO_RR_LAT_POS = 3
PMO_RR_CATS = 4

PMO_FLAG_EXPORT_EXITS = 1
PMO_FLAG_PHOTON_STATS = 2
PMO_FLAG_SCORE_RECORD = 4

PMO_G_REPLAYED = 0
PMO_G_SKIPPED = 1
PMO_G_MISMATCH = 2
PMO_G_COUNTERS_N = 4
PMO_FD_MAX = 32

PMO_WS_LEDGER_OFFSET = 64
PMO_STATIC_WORKSPACE_BYTES = 512
PMO_VOXEL_WORDS_SCRATCH = 5
PMO_WS_COUNTERS_OFFSET = 256

STATUS_NAMES = {
    PMO_OK: "ok",
    PMO_ERR_ARG: "bad argument",
    PMO_ERR_GEOMETRY: "photon stepped outside the volume",
    PMO_ERR_LABEL: "photon entered a label without optical properties",
    PMO_ERR_STEP_CAP: "photon exceeded its event cap",
    PMO_ERR_CUDA: "CUDA runtime error",
    PMO_ERR_WORKSPACE: "workspace missing or too small",
    PMO_ERR_TIMEOUT: "bounded device wait timed out",
    PMO_ERR_NUMERIC: "non-finite weight or direction",
}

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_up = C.POINTER(C.c_uint32)


class PmoProblem(C.Structure):
    _fields_ = [
        ("labels", C.c_void_p),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("voxel_space", C.c_float),
        ("voxel_words", C.c_void_p),
        ("end_label", C.c_int32),
        ("props_mode", C.c_int32),
        ("n_labels", C.c_int32),
        ("ma", C.c_void_p), ("ms", C.c_void_p), ("g", C.c_void_p), ("n", C.c_void_p),
        ("vox_ma", C.c_void_p), ("vox_ms", C.c_void_p),
        ("source", C.c_int32),
        ("src_ix", C.c_int32), ("src_iy", C.c_int32), ("src_iz", C.c_int32),
        ("src_p", C.c_float * 3), ("src_v", C.c_float * 3),
        ("src_w0", C.c_float),
        ("beam_sigma", C.c_float),
        ("spec_prob", C.c_float),
        ("spec_v", C.c_float * 3),
        ("center_ix", C.c_int32), ("center_iy", C.c_int32),
        ("state_add", C.c_void_p), ("state_p", C.c_void_p),
        ("state_v", C.c_void_p), ("state_w", C.c_void_p),
        ("seed", C.c_uint64),
        ("photon_begin", C.c_uint64), ("photon_count", C.c_uint64),
        ("max_events", C.c_uint32),
        ("precision", C.c_int32),
        ("flags", C.c_uint32),
    ]


class PmoTallies(C.Structure):
    _fields_ = [
        ("ledger", C.c_void_p),
        ("counters", C.c_void_p),
        ("rr", C.c_void_p),
        ("nr", C.c_int32),
        ("dr", C.c_float),
        ("fluence_mode", C.c_int32),
        ("absorbed", C.c_void_p),
        ("win_lo", C.c_int32 * 3),
        ("win_dim", C.c_int32 * 3),
        ("exit_add", C.c_void_p), ("exit_p", C.c_void_p),
        ("exit_v", C.c_void_p), ("exit_w", C.c_void_p),
        ("ph_interact", C.c_void_p), ("ph_cross", C.c_void_p), ("ph_fresnel", C.c_void_p),
        ("score_bin", C.c_void_p), ("score_w", C.c_void_p),
        ("ang", C.c_void_p),
        ("n_ang", C.c_int32),
        ("line", C.c_void_p),
        ("n_line", C.c_int32),
        ("line_dr", C.c_float),
        ("line_y_range", C.c_float),
    ]


class PmoGrad(C.Structure):
    _fields_ = [
        ("coef", C.c_void_p),
        ("nr", C.c_int32),
        ("dr", C.c_float),
        ("score_bin", C.c_void_p), ("score_w", C.c_void_p),
        ("d_ma_voxel", C.c_void_p), ("d_ms_voxel", C.c_void_p),
        ("d_ma_label", C.c_void_p), ("d_ms_label", C.c_void_p),
        ("counters", C.c_void_p),
        ("fd_target", C.c_void_p),
        ("fd_n", C.c_int32),
        ("fd_param", C.c_int32),
        ("fd_h", C.c_float),
        ("fd_out", C.c_void_p),
    ]


PMO_BS_RD, PMO_BS_RD_L, PMO_BS_RD_N, PMO_BS_TT, PMO_BS_TT_L, PMO_BS_TT_N = 0, 1, 2, 3, 4, 5
PMO_BS_ABS, PMO_BS_WINIT, PMO_BS_RGAIN, PMO_BS_RLOSS, PMO_BS_ERRW, PMO_BS_INTER = 6, 7, 8, 9, 10, 11
PMO_BS_N = 16
PMO_BT_THREAD, PMO_BT_GLOBAL = 0, 1
PMO_BR_RD, PMO_BR_TT, PMO_BR_A = 0, 1, 2
PMO_BR_DRD_DMA, PMO_BR_DRD_DMS, PMO_BR_DTT_DMA, PMO_BR_DTT_DMS = 3, 4, 5, 6
PMO_BR_BALANCE = 7
PMO_BR_N = 8


class PmoSlab(C.Structure):
    _fields_ = [("ma", C.c_float), ("ms", C.c_float), ("g", C.c_float),
                ("n_tissue", C.c_float), ("n_ambient", C.c_float), ("thickness", C.c_float),
                ("dr", C.c_float), ("photons", C.c_uint32)]


class PmoBatchItem(C.Structure):
    _fields_ = [("problem", C.c_uint32), ("begin", C.c_uint32), ("count", C.c_uint32)]


class PmoBatch(C.Structure):
    _fields_ = [
        ("slabs", C.c_void_p), ("n_problems", C.c_int32),
        ("items", C.c_void_p), ("n_items", C.c_int32),
        ("seed", C.c_uint64), ("nr", C.c_int32),
        ("sums", C.c_void_p), ("bins", C.c_void_p),
        ("remaining", C.c_void_p), ("t_done", C.c_void_p),
        ("precision", C.c_int32), ("max_events", C.c_uint32),
        ("tally_mode", C.c_int32),
    ]


PMO_MAX_LAYERS = 8
PMO_SS_RD, PMO_SS_TT, PMO_SS_ABS, PMO_SS_WINIT = 0, 1, 2, 3
PMO_SS_RGAIN, PMO_SS_RLOSS, PMO_SS_ERRW, PMO_SS_INTER = 4, 5, 6, 7
PMO_SS_LAYER0 = 8
PMO_SS_N = 40
PMO_SR_RD, PMO_SR_TT, PMO_SR_A, PMO_SR_BALANCE = 0, 1, 2, 3
PMO_SR_LAYER0 = 4
PMO_SR_N = 36
PMO_SB_N = 17


class PmoLayer(C.Structure):
    _fields_ = [("ma", C.c_float), ("ms", C.c_float), ("g", C.c_float), ("n", C.c_float),
                ("thickness", C.c_float)]


class PmoStack(C.Structure):
    _fields_ = [("first_layer", C.c_uint32), ("n_layers", C.c_uint32),
                ("n_ambient", C.c_float), ("dr", C.c_float), ("photons", C.c_uint32)]


class PmoStackBatch(C.Structure):
    _fields_ = [
        ("stacks", C.c_void_p), ("n_problems", C.c_int32),
        ("layers", C.c_void_p), ("n_layer_rows", C.c_int32),
        ("items", C.c_void_p), ("n_items", C.c_int32),
        ("seed", C.c_uint64), ("nr", C.c_int32),
        ("sums", C.c_void_p), ("bins", C.c_void_p),
        ("remaining", C.c_void_p), ("t_done", C.c_void_p),
        ("precision", C.c_int32), ("max_events", C.c_uint32),
    ]


class PmoObdParams(C.Structure):
    _fields_ = [
        ("outer_d1", C.c_double), ("ct1", C.c_double), ("r1", C.c_double),
        ("n1", C.c_double), ("bfl1", C.c_double),
        ("outer_d2", C.c_double), ("ct2", C.c_double), ("r2", C.c_double),
        ("n2", C.c_double), ("bfl2", C.c_double),
        ("slit_d", C.c_double), ("slit_width", C.c_double), ("slit_thickness", C.c_double),
        ("distance_2slits", C.c_double),
        ("d_pd", C.c_double), ("pd_correction", C.c_double),
        ("ld_fix_part", C.c_int32), ("side", C.c_int32),
        ("side_dz", C.c_double), ("side_tan", C.c_double),
        ("z", C.c_void_p), ("n_z", C.c_int32),
        ("seed", C.c_uint64),
        ("fixed_u", C.c_double),
    ]


class PmoLaunch(C.Structure):
    _fields_ = [("block_threads", C.c_int32), ("blocks_per_sm", C.c_int32)]
