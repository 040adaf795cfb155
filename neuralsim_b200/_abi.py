"""ctypes mirror of include/neuralsim.h and include/neuralsim_gen.h.

Loads the in-tree libneuralsim.so. There is no fallback: if the library is
missing or cannot be loaded the import fails with the loader's message.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libneuralsim.so")

NS_OK = 0
STATUS_NAMES = {
    0: "NS_OK", 1: "NS_ERR_INVALID_ARG", 2: "NS_ERR_NULL_HANDLE", 3: "NS_ERR_CSR",
    4: "NS_ERR_OOM", 5: "NS_ERR_CUDA", 6: "NS_ERR_DEVICE_TIMEOUT", 7: "NS_ERR_STATE",
    8: "NS_ERR_UNSUPPORTED", 9: "NS_ERR_NONFINITE", 10: "NS_ERR_SPIKE_LOG_FULL",
    11: "NS_ERR_NO_DEVICE",
}

MODEL_LIF, MODEL_IZHIKEVICH, MODEL_HH = 0, 1, 2
INPUT_DIRECT_DECAY, INPUT_DELTA_V, INPUT_RESET_EACH_STEP = 0, 1, 2
INPUT_CONDUCTANCE_REF, INPUT_CONDUCTANCE_FRESH = 3, 4
HH_EULER_REF, HH_RUSH_LARSEN = 0, 1
WEIGHT_F32, WEIGHT_BF16 = 0, 1
SYN_AMPA, SYN_GABA, SYN_GABA_B, SYN_NMDA = 0, 1, 2, 3
DRIVE_NONE, DRIVE_REF_UNIFORM, DRIVE_POISSON_KICK, DRIVE_GAUSS, DRIVE_POISSON_CONDUCTANCE = 0, 1, 2, 3, 4
GEN_W_SCALED, GEN_W_UNIFORM, GEN_W_LOGNORMAL = 0, 1, 2


class NsConfig(C.Structure):
    _fields_ = [
        ("model", C.c_uint32), ("input_mode", C.c_uint32), ("hh_integrator", C.c_uint32),
        ("weight_format", C.c_uint32), ("dt_ms", C.c_double), ("delay_steps", C.c_uint32),
        ("device", C.c_int32), ("seed", C.c_uint64), ("current_decay", C.c_double),
        ("stdp_enabled", C.c_int32), ("tau_plus", C.c_double), ("tau_minus", C.c_double),
        ("a_plus", C.c_double), ("a_minus", C.c_double), ("w_min", C.c_double),
        ("w_max", C.c_double), ("homeostasis_enabled", C.c_int32),
        ("homeostatic_target_rate", C.c_double), ("homeostatic_tau", C.c_double),
        ("contribution_tau", C.c_double), ("spike_log_capacity", C.c_uint64),
        ("spike_log_steps", C.c_uint32), ("graph_chunk", C.c_uint32),
        ("step_schedule", C.c_uint32), ("window_steps", C.c_uint32),
        ("rstdp_enabled", C.c_int32), ("rstdp_lr", C.c_double), ("rstdp_w_min", C.c_double),
        ("rstdp_w_max", C.c_double), ("eligibility_tau", C.c_double),
        ("reward_threshold", C.c_uint64), ("reward_decay", C.c_double),
        ("reward_signal", C.c_double), ("consolidation_enabled", C.c_int32),
        ("consolidation_tau", C.c_double), ("consolidation_target", C.c_double),
        ("consolidation_drift", C.c_double), ("track_rates", C.c_uint32),
    ]


class NsDrive(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32), ("p", C.c_float), ("amplitude", C.c_float),
        ("sigma_exc", C.c_float), ("sigma_inh", C.c_float), ("kick_chance", C.c_float),
        ("kick_strength", C.c_float), ("kick_min", C.c_uint32), ("kick_max", C.c_uint32),
    ]


class NsNeuronSoa(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("v", C.c_void_p), ("u", C.c_void_p), ("refractory", C.c_void_p),
        ("current", C.c_void_p), ("hh_m", C.c_void_p), ("hh_h", C.c_void_p),
        ("hh_n", C.c_void_p), ("params", C.c_void_p), ("params_per_neuron", C.c_uint32),
        ("inhibitory", C.c_void_p), ("is_output", C.c_void_p), ("pre_trace", C.c_void_p),
        ("post_trace", C.c_void_p), ("last_spike_step", C.c_void_p),
        ("pending_input", C.c_void_p), ("conductance", C.c_void_p),
        ("firing_rate", C.c_void_p),
    ]


class NsNetDesc(C.Structure):
    _fields_ = [
        ("neurons", C.POINTER(NsNeuronSoa)), ("m", C.c_uint64), ("row_ptr", C.c_void_p),
        ("col", C.c_void_p), ("w", C.c_void_p), ("syn_type", C.c_void_p),
        ("plastic", C.c_void_p), ("seed", C.c_uint64),
    ]


class NsStepStats(C.Structure):
    _fields_ = [
        ("steps_done", C.c_uint64), ("spikes", C.c_uint64), ("output_spikes", C.c_uint64),
        ("events", C.c_uint64), ("last_step_spikes", C.c_uint64), ("sim_time_ms", C.c_double),
        ("max_step_spikes", C.c_uint64),
    ]


# every symbol the public headers declare, with (restype, argtypes)
_P = C.c_void_p
_U64P = C.POINTER(C.c_uint64)
SIGNATURES = {
    "ns_config_default": (None, [C.POINTER(NsConfig)]),
    "ns_create": (C.c_int32, [C.POINTER(NsConfig), C.POINTER(_P)]),
    "ns_destroy": (C.c_int32, [_P]),
    "ns_last_error": (C.c_char_p, [_P]),
    "ns_status_string": (C.c_char_p, [C.c_int32]),
    "ns_device_count": (C.c_int32, [C.POINTER(C.c_int)]),
    "ns_upload_neurons": (C.c_int32, [_P, C.POINTER(NsNeuronSoa)]),
    "ns_upload_csr": (C.c_int32, [_P, C.c_uint64, C.c_uint64, _P, _P, _P, _P, _P]),
    "ns_set_drive": (C.c_int32, [_P, C.POINTER(NsDrive)]),
    "ns_upload_batch": (C.c_int32, [_P, C.c_uint32, C.POINTER(NsNetDesc), _P]),
    "ns_get_window": (C.c_int32, [_P, _P, _P, _P]),
    "ns_get_walk_shape": (C.c_int32, [_P, _P, _P, _P, _P, _P]),
    "ns_set_window_plan": (C.c_int32, [_P, C.c_uint32, C.c_uint32, C.c_uint32]),
    "ns_network_rates": (C.c_int32, [_P, C.c_uint64, C.c_uint32, _P]),
    # neuralsim_surrogate.h
    "ns_sur_create": (C.c_int32, [C.c_int32, _P, C.c_float, C.c_uint32, C.c_uint64, C.POINTER(_P)]),
    "ns_sur_destroy": (C.c_int32, [_P]),
    "ns_sur_last_error": (C.c_char_p, [_P]),
    "ns_sur_set_data": (C.c_int32, [_P, _P, C.c_uint64, _P]),
    "ns_sur_set_norm": (C.c_int32, [_P, _P, _P, _P, _P]),
    "ns_sur_train": (C.c_int32, [_P, C.c_uint32, C.c_float, C.c_float, _P]),
    "ns_sur_gradient": (C.c_int32, [_P, _P, _P, _P, _P]),
    "ns_sur_get_params": (C.c_int32, [_P, _P]),
    "ns_sur_set_params": (C.c_int32, [_P, _P]),
    "ns_sur_predict": (C.c_int32, [_P, _P, C.c_uint64, _P]),
    "ns_sur_set_sample_seed": (C.c_int32, [_P, C.c_uint64]),
    "ns_sur_grad_step": (C.c_int32, [_P, _P, _P]),
    "ns_sur_apply_gradient": (C.c_int32, [_P, _P, C.c_float, C.c_float]),
    "ns_tc_gemm_bf16": (C.c_int32, [_P, _P, _P, _P, _P, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32, _P]),
    "ns_set_surrogate": (C.c_int32, [_P, _P, C.c_float, C.c_float, C.c_float]),
    "ns_set_macro_step_mode": (C.c_int32, [_P, C.c_int32]),
    "ns_surrogate_counts": (C.c_int32, [_P, _U64P, _U64P]),
    "ns_step": (C.c_int32, [_P, C.c_uint32, C.POINTER(NsStepStats)]),
    "ns_read_spikes": (C.c_int32, [_P, C.c_uint64, C.c_uint32, _P, _P, C.c_uint64, _U64P]),
    "ns_clear_spike_log": (C.c_int32, [_P]),
    "ns_spike_log_range": (C.c_int32, [_P, _U64P, _U64P]),
    "ns_download_state": (C.c_int32, [_P, C.POINTER(NsNeuronSoa), _P]),
    "ns_upload_state": (C.c_int32, [_P, C.POINTER(NsNeuronSoa), _P, C.c_uint64]),
    "ns_get_step": (C.c_int32, [_P, _U64P]),
    "ns_download_rates": (C.c_int32, [_P, _P]),
    "ns_weight_stats": (C.c_int32, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ns_get_lfp": (C.c_int32, [_P, C.POINTER(C.c_double)]),
    "ns_add_input_current": (C.c_int32, [_P, C.c_uint64, C.c_void_p, C.c_void_p]),
    "ns_upload_eligibility": (C.c_int32, [_P, C.c_void_p, C.c_void_p]),
    "ns_download_eligibility": (C.c_int32, [_P, C.c_void_p]),
    "ns_download_contributions": (C.c_int32, [_P, C.c_void_p]),
    "ns_upload_contributions": (C.c_int32, [_P, C.c_void_p]),
    "ns_apply_reward": (C.c_int32, [_P, C.c_double]),
    "ns_get_reward": (C.c_int32, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ns_set_reward": (C.c_int32, [_P, C.c_double]),
    "ns_upload_stp": (C.c_int32, [_P, C.c_void_p, C.c_void_p]),
    "ns_shard_range": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64)]),
    "ns_shard_configure": (C.c_int32, [_P, C.c_uint32, C.c_uint32]),
    "ns_shard_nccl_unique_id": (C.c_int32, [C.c_void_p]),
    "ns_shard_nccl_init": (C.c_int32, [_P, C.c_void_p]),
    "ns_shard_step_begin": (C.c_int32, [_P]),
    "ns_shard_copy_bitmap": (C.c_int32, [_P, _P]),
    "ns_shard_step_end": (C.c_int32, [_P]),
    "ns_step_traced": (C.c_int32, [_P, _P, C.c_uint64, _U64P]),
    "ns_launch_count": (C.c_int32, [_P, _U64P]),
    "ns_get_schedule": (C.c_int32, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_double)]),
    "ns_get_stream": (C.c_int32, [_P, C.POINTER(_P)]),
    "ns_counters": (C.c_int32, [_P, _U64P]),
    "ns_profile_steps": (C.c_int32, [_P, C.c_uint32, C.POINTER(C.c_double), _U64P]),
    "ns_izhikevich_step_noalloc": (C.c_int32, [C.c_uint64, _P, _P, _P, _P, _P, _P, _P,
                                               C.c_float, _P, _P, _P]),
    "ns_gen_topology": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_uint64, _P, _P, _P, C.c_int32]),
    "ns_gen_weights": (C.c_int32, [C.c_uint32, C.c_uint64, C.c_uint64, _P, C.c_uint64,
                                   C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double,
                                   _P, _P, _P, C.c_int32, C.c_int32]),
}

_lib = None


def load():
    """Loads libneuralsim.so once and binds every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m neuralsim_b200.build` "
            "(the CUDA library is required; there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class NsError(RuntimeError):
    """A non-zero ns_status from the C ABI."""

    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


def check(status, handle=None):
    if status != NS_OK:
        lib = load()
        msg = lib.ns_last_error(handle)
        raise NsError(status, msg.decode() if msg else "")
