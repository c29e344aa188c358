"""ctypes binding of libstarkgpu.so (the C ABI in include/starkgpu.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstarkgpu.so")

SG_OK, SG_ERR_INVALID, SG_ERR_CUDA, SG_ERR_OOM, SG_ERR_BUDGET, SG_ERR_UNSUPPORTED = range(6)
_ERR_NAMES = {1: "SG_ERR_INVALID", 2: "SG_ERR_CUDA", 3: "SG_ERR_OOM", 4: "SG_ERR_BUDGET", 5: "SG_ERR_UNSUPPORTED"}


class SgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class LeafLayout(C.Structure):
    _fields_ = [("rows_per_leaf", C.c_uint32), ("little_endian", C.c_uint32),
                ("col_start", C.c_uint64), ("col_end", C.c_uint64)]


class TableDesc(C.Structure):
    _fields_ = [("trace", C.c_void_p), ("trace_on_device", C.c_int), ("n", C.c_uint64), ("row_u64", C.c_uint64),
                ("blowup", C.c_uint32), ("weights_on_device", C.c_int), ("weights", C.c_void_p),
                ("layout", LeafLayout)]


class PassRecord(C.Structure):
    _fields_ = [("log_len", C.c_uint32), ("cols", C.c_uint32), ("inverse", C.c_uint32), ("reps", C.c_uint32),
                ("pre", C.c_uint32), ("post", C.c_uint32), ("canon", C.c_uint32), ("pad_", C.c_uint32),
                ("tiles", C.c_uint64), ("m", C.c_uint64), ("ms", C.c_float), ("pad2_", C.c_float)]


class Rv64Info(C.Structure):
    _fields_ = [("cycles", C.c_uint64), ("a0", C.c_uint64), ("shifts", C.c_uint64), ("cells", C.c_uint64),
                ("keccak_calls", C.c_uint64), ("chips", C.c_uint32), ("reserved", C.c_uint32)]


class VerifyTable(C.Structure):
    _fields_ = [("log_n", C.c_uint32), ("log_N", C.c_uint32), ("m", C.c_uint32), ("aux_cols", C.c_uint32),
                ("queries", C.c_uint32), ("fri_layers", C.c_uint32), ("total_folds", C.c_uint32),
                ("terminal_log", C.c_uint32), ("num_coeffs", C.c_uint32), ("pad_", C.c_uint32),
                ("coset_offset", C.c_uint64), ("omega_N", C.c_uint64), ("terminal_offset", C.c_uint64),
                ("omega_T", C.c_uint64), ("consts", C.c_void_p), ("roots", C.c_void_p), ("iotas", C.c_void_p),
                ("open_main", C.c_void_p), ("open_aux", C.c_void_p), ("open_parts", C.c_void_p),
                ("path_main", C.c_void_p), ("path_aux", C.c_void_p), ("path_parts", C.c_void_p),
                ("fri_open", C.c_void_p), ("fri_paths", C.c_void_p)]


class LdeInfo(C.Structure):
    _fields_ = [("d_lde", C.c_void_p), ("lde_rows", C.c_uint64), ("row_u64", C.c_uint64),
                ("d_nodes", C.c_void_p), ("leaves_len", C.c_uint64), ("root", C.c_uint8 * 32)]


u64, u32, i32, vp = C.c_uint64, C.c_uint32, C.c_int, C.c_void_p


class DeviceProgram(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("num_nodes", C.c_uint32), ("base_consts", C.c_void_p),
                ("num_base_consts", C.c_uint32), ("ext_consts", C.c_void_p), ("num_ext_consts", C.c_uint32),
                ("roots", C.c_void_p), ("num_roots", C.c_uint32), ("num_base_slots", C.c_uint32),
                ("num_ext_slots", C.c_uint32), ("node_roots", C.c_void_p), ("hand_kernel", C.c_uint32),
                ("hand_roots", C.c_uint32), ("logup", C.c_void_p), ("logup_root", C.c_uint32)]


class Composition(C.Structure):
    _fields_ = [("beta_trans", C.c_void_p), ("d_z_inv", C.c_void_p), ("z_len", C.c_uint64),
                ("num_boundary", C.c_uint32), ("b_col", C.c_void_p), ("b_is_aux", C.c_void_p),
                ("b_value", C.c_void_p), ("b_beta", C.c_void_p), ("d_b_z_inv", C.c_void_p)]


class LogupDesc(C.Structure):
    _fields_ = [("num_interactions", C.c_uint32), ("bus_ids", C.c_void_p), ("elem_offsets", C.c_void_p),
                ("elem_alpha_idx", C.c_void_p), ("elem_consts", C.c_void_p), ("term_offsets", C.c_void_p),
                ("term_coefs", C.c_void_p), ("term_cols", C.c_void_p), ("num_out_cols", C.c_uint32),
                ("out_col_offsets", C.c_void_p), ("out_col_interactions", C.c_void_p), ("mult_consts", C.c_void_p),
                ("mult_term_offsets", C.c_void_p), ("mult_term_coefs", C.c_void_p), ("mult_term_cols", C.c_void_p),
                ("num_committed", C.c_uint32)]
class TableJob(C.Structure):
    _fields_ = [("d_trace", C.c_void_p), ("d_main_lde", C.c_void_p), ("d_main_nodes", C.c_void_p),
                ("main_leaves_len", C.c_uint64), ("n", C.c_uint64), ("m", C.c_uint64), ("blowup", C.c_uint32),
                ("coset_offset", C.c_uint64), ("d_weights", C.c_void_p), ("d_comp_weights", C.c_void_p),
                ("d_z_inv", C.c_void_p), ("d_b_z_inv", C.c_void_p), ("d_inv2x", C.c_void_p), ("d_pts_n", C.c_void_p),
                ("d_pts_N", C.c_void_p), ("d_tw0", C.c_void_p), ("logup", C.c_void_p), ("program", C.c_void_p),
                ("num_boundary", C.c_uint32), ("b_col", C.c_void_p), ("b_is_aux", C.c_void_p),
                ("b_value", C.c_void_p), ("lookup_challenges", C.c_void_p), ("alpha_pows", C.c_void_p),
                ("n_alpha", C.c_uint32), ("queries", C.c_uint32), ("grinding", C.c_uint32),
                ("final_log_degree", C.c_uint32)]


class ProofShape(C.Structure):
    _fields_ = [("aux_cols", C.c_uint64), ("total_folds", C.c_uint32), ("fri_layers", C.c_uint32),
                ("terminal_coeffs", C.c_uint32), ("depth", C.c_uint32), ("fri_path_bytes", C.c_uint64)]


class TableProof(C.Structure):
    _fields_ = [(nm, C.c_void_p) for nm in ("aux_root", "comp_root", "table_contribution", "trace_ood", "parts_ood",
                                            "fri_roots", "fri_final", "nonce", "iotas", "open_main", "open_aux",
                                            "open_parts", "path_main", "path_aux", "path_parts", "fri_open",
                                            "fri_paths")]


PROTOTYPES = {
    "sg_ctx_create": (i32, [i32, u64, C.POINTER(vp)]),
    "sg_ctx_destroy": (None, [vp]),
    "sg_last_error": (C.c_char_p, []),
    "sg_ctx_memory": (i32, [vp, C.POINTER(u64), C.POINTER(u64)]),
    "sg_ctx_launches": (u64, [vp]),
    "sg_ctx_budget": (u64, [vp]),
    "sg_ctx_fail_alloc_after": (i32, [vp, C.c_int64]),
    "sg_dev_alloc": (i32, [vp, vp, u64, C.POINTER(vp)]),
    "sg_dev_free": (i32, [vp, vp, vp, u64]),
    "sg_memcpy_h2d": (i32, [vp, vp, vp, vp, u64]),
    "sg_memcpy_d2h": (i32, [vp, vp, vp, vp, u64]),
    "sg_stream_sync": (i32, [vp, vp]),
    "sg_stream_create": (i32, [vp, C.POINTER(vp)]),
    "sg_stream_create_priority": (i32, [vp, C.c_int, C.POINTER(vp)]),
    "sg_stream_priority_range": (i32, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "sg_stream_destroy": (i32, [vp, vp]),
    "sg_host_alloc": (i32, [u64, C.POINTER(vp)]),
    "sg_host_free": (i32, [vp]),
    "sg_ntt_forward": (i32, [vp, vp, vp, u64, u64]),
    "sg_ntt_inverse": (i32, [vp, vp, vp, u64, u64]),
    "sg_coset_lde": (i32, [vp, vp, vp, u64, u64, u32, vp, vp]),
    "sg_keccak_leaves": (i32, [vp, vp, vp, u64, u64, C.POINTER(LeafLayout), vp]),
    "sg_merkle_build": (i32, [vp, vp, vp, u64, vp, vp]),
    "sg_merkle_leaves_len": (u64, [u64]),
    "sg_merkle_gather_paths": (i32, [vp, vp, vp, u64, vp, u32, vp]),
    "sg_lde_commit": (i32, [vp, vp, vp, i32, u64, u64, u32, vp, C.POINTER(LeafLayout), vp, C.POINTER(vp), vp]),
    "sg_lde_get_info": (i32, [vp, C.POINTER(LdeInfo)]),
    "sg_lde_free": (None, [vp, vp]),
    "sg_lde_free_async": (None, [vp, vp, vp]),
    "sg_lde_commit_split": (i32, [vp, vp, vp, i32, u64, u64, u32, vp, u64, i32, vp, vp, vp, vp, vp]),
    "sg_fri_begin": (i32, [vp, vp, vp, i32, vp, i32, u64, vp]),
    "sg_fri_fold_commit_layer": (i32, [vp, vp, vp, vp]),
    "sg_fri_fold_final": (i32, [vp, vp, vp]),
    "sg_fri_num_layers": (u32, [vp]),
    "sg_fri_layer": (i32, [vp, u32, vp, vp, vp, vp]),
    "sg_fri_free": (None, [vp]),
    "sg_field_ops": (i32, [vp, vp, u32, vp, vp, vp, u64]),
    "sg_batch_commit": (i32, [vp, vp, vp, u32, u32, vp, vp]),
    "sg_batch_commit_fused": (i32, [vp, vp, vp, u32, u32, vp, vp]),
    "sg_table_proof_shape": (i32, [vp, vp]),
    "sg_ctx_dft_tiles": (i32, [vp, u32, u32]),
    "sg_ctx_dft_tuning": (i32, [vp, vp, u32, vp, vp, vp]),
    "sg_prove_table": (i32, [vp, vp, vp, vp, vp]),
    "sg_grind": (i32, [vp, vp, vp, C.c_uint8, C.POINTER(u64)]),
    "sg_coset_lde_static": (i32, [vp, vp, u64, u64, u32, vp, vp]),
    "sg_transcript_new": (vp, [vp, u64]),
    "sg_transcript_clone": (vp, [vp]),
    "sg_transcript_free": (None, [vp]),
    "sg_transcript_append": (None, [vp, vp, u64]),
    "sg_transcript_append_base": (None, [vp, u64]),
    "sg_transcript_append_ext3": (None, [vp, vp]),
    "sg_transcript_sample": (None, [vp, vp]),
    "sg_transcript_state": (None, [vp, vp]),
    "sg_transcript_sample_base": (u64, [vp]),
    "sg_transcript_sample_ext3": (None, [vp, vp]),
    "sg_transcript_sample_u64": (u64, [vp, u64]),
    "sg_transcript_sample_z_ood": (None, [vp, u64, u64, u64, vp]),
    "sg_keccak256": (None, [vp, u64, vp]),
    "sg_batch_inverse_ext3": (i32, [vp, vp, vp, u64, vp, C.POINTER(i32)]),
    "sg_inv_denoms_ext3": (i32, [vp, vp, vp, u64, vp, u32, i32, vp, C.POINTER(i32)]),
    "sg_barycentric_sums": (i32, [vp, vp, vp, u64, u64, i32, u64, vp, vp, u64, u32, vp]),
    "sg_deep_composition": (i32, [vp, vp, vp, u64, vp, u64, vp, u64, u64, vp, vp, vp, vp, u32, vp, vp, i32, vp]),
    "sg_fri_fold_layer": (i32, [vp, vp, vp, u64, vp, vp, vp, vp, vp]),
    "sg_fri_leaves": (i32, [vp, vp, vp, u64, vp]),
    "sg_gather_rows": (i32, [vp, vp, vp, u64, u64, u64, u64, vp, u32, vp]),
    "sg_logup_aux": (i32, [vp, vp, vp, u64, u64, vp, vp, u32, vp, vp, vp]),
    "sg_eval_constraints": (i32, [vp, vp, vp, vp, u32, vp, u32, vp, vp, u64, vp, u64, u64, u64, vp, vp]),
    "sg_decompose_d2": (i32, [vp, vp, vp, u64, vp, vp]),
    "sg_synth_trace": (i32, [vp, vp, vp, u64, u64, u64, u32]),
    "sg_ctx_pass_log": (i32, [vp, i32]),
    "sg_rv64_run": (i32, [vp, u32, u64, u64, vp, vp, vp, vp, vp, vp, vp]),
    "sg_rv64_run_counted": (i32, [vp, u32, u64, u64, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "sg_rv64_cpu_table": (i32, [vp, vp, vp, u64, vp, u64, u32, vp]),
    "sg_rv64_keccak_table": (i32, [vp, vp, vp, u64, u64, vp]),
    "sg_rv64_shift_table": (i32, [vp, vp, vp, u64, u64, vp]),
    "sg_rv64_memory_table": (i32, [vp, vp, vp, u64, u64, vp]),
    "sg_rv64_exec": (i32, [vp, u32, u64, C.POINTER(vp), C.POINTER(Rv64Info)]),
    "sg_rv64_trace_part": (i32, [vp, u32, C.POINTER(vp), C.POINTER(u64)]),
    "sg_rv64_trace_free": (None, [vp]),
    "sg_verify_queries": (i32, [vp, vp, C.POINTER(VerifyTable), u32, vp]),
    "sg_ctx_pass_log_read": (i32, [vp, C.POINTER(PassRecord), u32, C.POINTER(u32)]),
    "sg_mlp_loss_grad": (i32, [vp, vp, vp, vp, u32, vp, vp, vp]),
    "sg_mlp_train": (i32, [vp, vp, vp, vp, u32, vp, u32, C.c_float, C.POINTER(C.c_float)]),
    "sg_mlp_predict": (i32, [vp, vp, vp, u32, vp, vp]),
    "sg_pass_features": (None, [u32, u64, u64, u32, u32, u32, u32, u32, u32, C.POINTER(C.c_float)]),
    "sg_ctx_set_pass_model": (i32, [vp, C.POINTER(C.c_float), u32]),
}
MLP_IN, MLP_HIDDEN = 16, 32
MLP_PARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN + 1
SG_STATIC_SCRATCH_BYTES = 32 << 20

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python lambda_vm_b200/build.py` "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != SG_OK:
        msg = lib().sg_last_error()
        raise SgError(rc, msg.decode() if msg else "")
    return rc
