"""dynaverse-b200: BN254 prover operators on B200, behind the dvgpu C-ABI.

Host-side mirror of the reference's operator plugin interface
(`OperatorBackend`, crates/protocol/src/types.rs:281-359, implemented for the
GPU by `IcicleBackend`, crates/gpu/src/icicle.rs:342-457).  Method names,
argument meaning and error behaviour follow the trait:

* results in caller order, element-identical to the CPU reference;
* inputs validated before any dispatch; errors raise DvgpuError and never
  fall back to a CPU path;
* a failed call leaves caller data untouched.

All compute runs in libdvgpu.so (hand-written sm_100a kernels); this module
only marshals bytes.  Wire formats: Fr 32-byte LE canonical, G1 64 bytes,
G2 128 bytes, infinity all zero (crates/gpu/src/codec.rs:25-111).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DVGPU_LIB_PATH", os.path.join(HERE, "lib", "libdvgpu.so"))

FR_BYTES = 32
G1_BYTES = 64
G2_BYTES = 128
R_MODULUS = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
Q_MODULUS = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47

NTT_FORWARD, NTT_INVERSE, NTT_COSET_FORWARD, NTT_COSET_INVERSE = 0, 1, 2, 3

_lib = None


class DvgpuError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"dvgpu error {status}: {message}")
        self.status = status
        self.message = message


class G2ValidationReport(ctypes.Structure):
    _fields_ = [("checked_points", ctypes.c_uint64), ("invalid_points", ctypes.c_uint64),
                ("first_invalid", ctypes.c_uint64), ("failure_mask", ctypes.c_uint32),
                ("algorithm", ctypes.c_uint32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("icicle_calls", ctypes.c_uint64), ("buffer_grows", ctypes.c_uint64),
                ("max_batch_size", ctypes.c_uint64), ("input_capacity", ctypes.c_uint64)]


class MemoryInfo(ctypes.Structure):
    _fields_ = [("free_bytes", ctypes.c_uint64), ("total_bytes", ctypes.c_uint64)]


class MsmPhaseTimes(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double * 8), ("calls", ctypes.c_uint64), ("accum_mixed_adds", ctypes.c_uint64)]


MSM_PHASE_NAMES = ["hist", "scan", "scatter", "accum", "merge", "reduce", "unused", "tail"]


class ServeResult(ctypes.Structure):
    _fields_ = [("submit_ns", ctypes.c_uint64), ("start_ns", ctypes.c_uint64), ("done_ns", ctypes.c_uint64),
                ("batch_requests", ctypes.c_uint32), ("batch_id", ctypes.c_uint32)]


class ServeStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in ("requests", "batches", "sessions", "resident_bytes",
                                                      "budget_bytes", "max_batch", "largest_batch", "busy_ns",
                                                      "pending")]


class ResidentOp(ctypes.Structure):
    _fields_ = [("opcode", ctypes.c_uint32), ("kind", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("a", ctypes.c_uint64), ("b", ctypes.c_uint64), ("c", ctypes.c_uint64),
                ("a_offset", ctypes.c_uint64), ("b_offset", ctypes.c_uint64), ("c_offset", ctypes.c_uint64),
                ("length", ctypes.c_uint64), ("rows", ctypes.c_uint64), ("cols", ctypes.c_uint64),
                ("input", ctypes.c_void_p), ("output", ctypes.c_void_p)]


class ResidentStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("h2d_bytes", "d2h_bytes", "bytes_allocated", "fr_transform_elements",
                                               "g1_transform_elements", "msm_g1_points", "msm_g2_points", "calls")]


class ResidentDiagnostics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "resident_allocations", "temporary_allocations", "temporary_peak_bytes", "journal_saved_bytes",
        "journal_saved_ranges", "journal_peak_bytes", "device_operation_ns", "device_operations",
        "physical_h2d_bytes", "physical_d2h_bytes", "explicit_d2d_bytes", "journal_metadata_capacity_bytes")]


RESIDENT_OPS = dict(ALLOC=1, LENGTH=2, KIND=3, BEGIN=4, ROLLBACK=5, WRITE=6, READ=7, COPY=8, REVERSE=9, TRANSPOSE=10,
                    TRANSFORM=11, ZIP=12, SCALE=13, MSM_G1=14, MSM_G2=15, ALLOC_BASES=16, TRANSFORM_PACKET=17)


class BatchPlanBuffers(ctypes.Structure):
    _fields_ = [("scalars", ctypes.c_void_p), ("ntt_values", ctypes.c_void_p), ("msm_results", ctypes.c_void_p),
                ("ntt_results", ctypes.c_void_p), ("scalar_bytes", ctypes.c_uint64), ("ntt_bytes", ctypes.c_uint64),
                ("msm_result_bytes", ctypes.c_uint64), ("msm_classes", ctypes.c_uint32),
                ("graph_nodes", ctypes.c_uint32), ("graph_kernels", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class SetupStats(ctypes.Structure):
    _fields_ = [("table_builds", ctypes.c_uint64 * 2), ("calls", ctypes.c_uint64 * 2),
                ("points", ctypes.c_uint64 * 2), ("table_bytes", ctypes.c_uint64),
                ("device_ns", ctypes.c_uint64 * 5), ("native_wall_ns", ctypes.c_uint64)]


class G2KernelConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("threads", "schedule", "layout", "fused")]


class G2ExperimentStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("repack_device_ns", "subgroup_kernel_ns", "logical_repack_bytes")]


class G2KernelResources(ctypes.Structure):
    _fields_ = [("registers", ctypes.c_uint32), ("block_threads", ctypes.c_uint32),
                ("active_blocks", ctypes.c_uint32), ("max_threads_per_sm", ctypes.c_uint32),
                ("local_bytes", ctypes.c_uint64), ("shared_bytes", ctypes.c_uint64),
                ("normalize_registers", ctypes.c_uint32), ("normalize_active_blocks", ctypes.c_uint32),
                ("normalize_local_bytes", ctypes.c_uint64), ("normalize_shared_bytes", ctypes.c_uint64)]


class MsmTimings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("conversion_ns", "icicle_ns", "output_ns")]


TIMELINE_PHASES, TIMELINE_KERNELS = 9, 10


class MsmTimeline(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64 * TIMELINE_PHASES) for n in ("wall_ns", "event_ns", "calls", "event_calls",
                                                                   "bytes")] + \
               [(n, ctypes.c_uint64 * TIMELINE_KERNELS) for n in ("kernel_ns", "kernel_calls")] + \
               [(n, ctypes.c_uint64) for n in ("instrumentation_inclusive_ns", "instrumentation_total_ns", "c",
                                               "bitsize", "windows", "buckets")]


class ResidentProfile(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "native_wall_ns", "journal_host_ns", "conversion_host_ns", "operation_host_ns", "wait_host_ns",
        "event_total_ns", "event_journal_ns", "event_operation_ns", "event_mask", "h2d_bytes", "d2h_bytes",
        "d2d_bytes")]


class DynaverseParamsInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint64), ("m", ctypes.c_uint64), ("rebuild_interval", ctypes.c_uint64),
                ("resident_bytes", ctypes.c_uint64), ("g1_generator", ctypes.c_uint8 * 64),
                ("multiplication_vanishing_g1", ctypes.c_uint8 * 64), ("vk_g2", (ctypes.c_uint8 * 128) * 19)]


class DynaverseResult(ctypes.Structure):
    _fields_ = [("submit_ns", ctypes.c_uint64), ("start_ns", ctypes.c_uint64), ("done_ns", ctypes.c_uint64),
                ("batch_requests", ctypes.c_uint32), ("batch_id", ctypes.c_uint32), ("rebuilt", ctypes.c_uint32),
                ("pad", ctypes.c_uint32)]


class DynaverseStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("requests", "batches", "sessions", "resident_bytes", "budget_bytes",
                                              "max_batch", "largest_batch", "busy_ns", "pending", "sparse_proofs",
                                              "rebuilds", "launches", "msm_fme", "host_ns", "device_wait_ns",
                                              "dense_accum_ns", "dense_accum_adds", "allocations",
                                              "allocation_ns", "enqueue_ns", "slowest_alloc_ns",
                                              "slowest_alloc_bytes", "slowest_alloc_pinned")]


# (name, restype, argtypes)
_P = ctypes.c_void_p
_B = ctypes.c_char_p
_SZ = ctypes.c_size_t
_E = [ctypes.c_char_p, ctypes.c_size_t]
SIGNATURES = [
    ("dvgpu_backend_create", ctypes.c_int, [ctypes.POINTER(_P)] + _E),
    ("dvgpu_backend_create_with_large_bucket_factor", ctypes.c_int, [ctypes.c_uint32, ctypes.POINTER(_P)] + _E),
    ("dvgpu_backend_destroy", None, [_P]),
    ("dvgpu_backend_device_identity", ctypes.c_int, [_P, _B, _SZ] + _E),
    ("dvgpu_backend_memory_info", ctypes.c_int, [_P, ctypes.POINTER(MemoryInfo)] + _E),
    ("dvgpu_backend_batch_stats", ctypes.c_int, [_P, ctypes.POINTER(BatchStats)]),
    ("dvgpu_bn254_msm", ctypes.c_int, [_P, _P, _P, _SZ, _B] + _E),
    ("dvgpu_bn254_g2_msm", ctypes.c_int, [_P, _P, _P, _SZ, _B] + _E),
    ("dvgpu_bn254_msm_batch", ctypes.c_int, [_P, _P, _P, _SZ, _SZ, _B] + _E),
    ("dvgpu_bn254_ntt", ctypes.c_int, [_P, _P, _SZ, ctypes.c_int, _B, _B] + _E),
    ("dvgpu_setup_mode", ctypes.c_int, [_P, ctypes.c_int]),
    ("dvgpu_setup_stats", ctypes.c_int, [_P, ctypes.POINTER(SetupStats)]),
    ("dvgpu_bn254_g2_validation_inspect", ctypes.c_int,
     [_P, _P, _SZ, ctypes.c_uint32, _P, ctypes.POINTER(G2ValidationReport)] + _E),
    ("dvgpu_g2_validation_stats", ctypes.c_int, [_P, _P]),
    ("dvgpu_g2_validation_traffic", ctypes.c_int, [_P, _P]),
    ("dvgpu_g2_kernel_config_set", ctypes.c_int, [_P, ctypes.POINTER(G2KernelConfig)]),
    ("dvgpu_g2_kernel_config_get", ctypes.c_int, [_P, ctypes.POINTER(G2KernelConfig)]),
    ("dvgpu_g2_kernel_resources", ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(G2KernelResources)]),
    ("dvgpu_g2_experiment_stats", ctypes.c_int, [_P, ctypes.POINTER(G2ExperimentStats)]),
    ("dvgpu_bn254_tower_inspect", ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _P, _SZ, _P,
                                                  _SZ, _P, _SZ, _P, _SZ] + _E),
    ("dvgpu_bn254_lines_inspect", ctypes.c_int, [_P, _P, _SZ, _P, _SZ, _P, _SZ, _P, _SZ] + _E),
    ("dvgpu_bn254_miller_inspect", ctypes.c_int, [_P, _P, _SZ, _P, _SZ, _P, _SZ, _P, _SZ] + _E),
    ("dvgpu_g2_psi_probe", ctypes.c_int, [_P, _P, _SZ, _P] + _E),
    ("dvgpu_g2_test_corrupt_next", ctypes.c_int, [_P, ctypes.c_uint64]),
    ("dvgpu_bn254_msm_timeline", ctypes.c_int, [_P, _P, _P, _SZ, _B, _B, ctypes.POINTER(MsmTimings),
                                                 ctypes.POINTER(MsmTimeline)] + _E),
    ("dvgpu_bn254_fixed_base_g2_checked", ctypes.c_int,
     [_P, _P, _SZ, ctypes.c_uint32, _B, ctypes.POINTER(G2ValidationReport)] + _E),
    ("dvgpu_bn254_fixed_base", ctypes.c_int, [_P, _P, _SZ, ctypes.c_int, _B] + _E),
    ("dvgpu_reserve_batch", ctypes.c_int, [_P, _SZ] + _E),
    ("dvgpu_bn254_msm_profiled", ctypes.c_int, [_P, _P, _P, _SZ, _B, _P] + _E),
    ("dvgpu_bn254_ntt_ex", ctypes.c_int, [_P, _P, _SZ, ctypes.c_int, _B] + _E),
    ("dvgpu_bn254_msm_batch_uneven", ctypes.c_int, [_P, _P, _P, _P, _SZ, _B] + _E),
    ("dvgpu_bases_register", ctypes.c_int, [_P, _P, _SZ, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_bases_release", ctypes.c_int, [_P, ctypes.c_uint64]),
    ("dvgpu_bases_precompute", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_int)] + _E),
    ("dvgpu_bn254_msm_sparse_batch", ctypes.c_int, [_P, ctypes.c_uint64, _P, _P, _P, _SZ, _B] + _E),
    ("dvgpu_bn254_msm_device", ctypes.c_int, [_P, _P, _P, _SZ, ctypes.c_int, _B, _P] + _E),
    ("dvgpu_bn254_msm_sparse_device", ctypes.c_int, [_P, ctypes.c_uint64, _P, _P, _P, _SZ, _B, _P] + _E),
    ("dvgpu_bn254_msm_resident", ctypes.c_int, [_P, ctypes.c_uint64, _P, _SZ, _B, _P] + _E),
    ("dvgpu_bn254_msm_resident_host", ctypes.c_int, [_P, ctypes.c_uint64, _P, _SZ, _B] + _E),
    ("dvgpu_bn254_ntt_device", ctypes.c_int, [_P, _P, _SZ, ctypes.c_int, _P, _P] + _E),
    ("dvgpu_bn254_fixed_base_device", ctypes.c_int, [_P, _P, _SZ, ctypes.c_int, _P, _P] + _E),
    ("dvgpu_bn254_g2_check_device", ctypes.c_int,
     [_P, _P, _SZ, ctypes.c_uint32, _P, ctypes.POINTER(G2ValidationReport), _P] + _E),
    ("dvgpu_msm_set_window", ctypes.c_int, [_P, ctypes.c_int]),
    ("dvgpu_msm_get_window", ctypes.c_int, [_P, _SZ, ctypes.POINTER(ctypes.c_int)]),
    ("dvgpu_probe_imad_rate", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double)] + _E),
    ("dvgpu_launch_count", ctypes.c_uint64, []),
    ("dvgpu_bn254_ntt_noalloc", ctypes.c_int, [_P, _SZ, ctypes.c_int, _P, _P] + _E),
    ("dvgpu_msm_autotune", ctypes.c_int, [_P, _SZ, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _B, _SZ] + _E),
    ("dvgpu_msm_timeline", ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(MsmPhaseTimes)]),
    ("dvgpu_random_fr_device", ctypes.c_int, [_P, ctypes.c_uint64, _SZ, _P, _P] + _E),
    ("dvgpu_fr_powers_device", ctypes.c_int, [_P, _P, _SZ, _P, _P] + _E),
    ("dvgpu_g2_random_twist_device", ctypes.c_int, [_P, ctypes.c_uint64, _SZ, _P, _P] + _E),
    ("dvgpu_bn254_g1_ntt_rows", ctypes.c_int, [_P, _P, _SZ, _SZ, ctypes.c_int, _B] + _E),
    ("dvgpu_bn254_g1_ntt_rows_device", ctypes.c_int, [_P, _P, _SZ, _SZ, ctypes.c_int, _P, _P] + _E),
    ("dvgpu_bn254_pairing_check", ctypes.c_int, [_P, _B, _B, _P, _SZ, _B] + _E),
    ("dvgpu_bn254_pairing", ctypes.c_int, [_P, _B, _B, _SZ, _B] + _E),
    ("dvgpu_bn254_g2_prepare", ctypes.c_int, [_P, _B, _SZ, ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_bn254_g2_prepared_release", ctypes.c_int, [_P, ctypes.c_uint64] + _E),
    ("dvgpu_bn254_pairing_check_prepared", ctypes.c_int, [_P, _B, ctypes.c_uint64, _P, _P, _SZ, _B] + _E),
    ("dvgpu_bn254_poly_multiply", ctypes.c_int, [_P, _B, _SZ, _B, _SZ, _B, _SZ, ctypes.POINTER(_SZ)] + _E),
    ("dvgpu_bn254_poly_divide_exact", ctypes.c_int, [_P, _B, _SZ, _B, _SZ, _B, _SZ, ctypes.POINTER(_SZ)] + _E),
    ("dvgpu_bn254_tree_create", ctypes.c_int, [_P, _B, _SZ, ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_bn254_tree_destroy", ctypes.c_int, [_P, ctypes.c_uint64] + _E),
    ("dvgpu_bn254_tree_vanishing", ctypes.c_int, [_P, ctypes.c_uint64, _B, _SZ, ctypes.POINTER(_SZ)] + _E),
    ("dvgpu_bn254_tree_inverse_derivatives", ctypes.c_int, [_P, ctypes.c_uint64, _B, _SZ] + _E),
    ("dvgpu_bn254_tree_evaluate", ctypes.c_int, [_P, ctypes.c_uint64, _B, _SZ, _SZ, _B] + _E),
    ("dvgpu_bn254_tree_interpolate", ctypes.c_int, [_P, ctypes.c_uint64, _B, _SZ, _SZ, _B, ctypes.POINTER(_SZ)] + _E),
    ("dvgpu_bn254_tree_cauchy_sums", ctypes.c_int, [_P, ctypes.c_uint64, _B, _SZ, _SZ, _B] + _E),
    ("dvgpu_bn254_ntt_batch", ctypes.c_int, [_P, _P, _P, _P, _SZ, _B] + _E),
    ("dvgpu_bn254_ntt_batch_device", ctypes.c_int, [_P, _P, _P, _P, _SZ, _P, _P] + _E),
    ("dvgpu_batch_plan_create", ctypes.c_int,
     [_P, ctypes.c_uint64, _P, _SZ, _P, _P, _SZ, ctypes.POINTER(ctypes.c_uint64), _B, _SZ] + _E),
    ("dvgpu_batch_plan_buffers", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.POINTER(BatchPlanBuffers)] + _E),
    ("dvgpu_batch_plan_launch", ctypes.c_int, [_P, ctypes.c_uint64, _P] + _E),
    ("dvgpu_batch_plan_check", ctypes.c_int, [_P, ctypes.c_uint64] + _E),
    ("dvgpu_batch_plan_run", ctypes.c_int, [_P, ctypes.c_uint64, _P, _P, _B, _B] + _E),
    ("dvgpu_batch_plan_destroy", ctypes.c_int, [_P, ctypes.c_uint64] + _E),
    ("dvgpu_resident_configure", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint64, _P] + _E),
    ("dvgpu_resident_call", ctypes.c_int, [_P, ctypes.POINTER(ResidentOp), ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_resident_seal", None, [_P]),
    ("dvgpu_resident_commit", None, [_P]),
    ("dvgpu_resident_stats", ctypes.c_int, [_P, ctypes.POINTER(ResidentStats)]),
    ("dvgpu_resident_diagnostics", ctypes.c_int, [_P, ctypes.POINTER(ResidentDiagnostics)]),
    ("dvgpu_resident_call_profiled", ctypes.c_int, [_P, ctypes.POINTER(ResidentOp), ctypes.POINTER(ctypes.c_uint64),
                                                    ctypes.POINTER(ResidentProfile)] + _E),
    ("dvgpu_serve_create", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_P)] + _E),
    ("dvgpu_serve_destroy", None, [_P]),
    ("dvgpu_serve_open_session", ctypes.c_int, [_P, _P, _P, _SZ, ctypes.POINTER(ctypes.c_uint64), _B] + _E),
    ("dvgpu_serve_close_session", ctypes.c_int, [_P, ctypes.c_uint64] + _E),
    ("dvgpu_serve_submit", ctypes.c_int, [_P, ctypes.c_uint64, _P, _P, _SZ, ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_serve_wait", ctypes.c_int, [_P, ctypes.c_uint64, _B, ctypes.POINTER(ServeResult)] + _E),
    ("dvgpu_serve_set_max_batch", ctypes.c_int, [_P, ctypes.c_uint32]),
    ("dvgpu_serve_stats", ctypes.c_int, [_P, ctypes.POINTER(ServeStats)]),
    ("dvgpu_dynaverse_create", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_P)] + _E),
    ("dvgpu_dynaverse_destroy", None, [_P]),
    ("dvgpu_dynaverse_params_create", ctypes.c_int, [_P, _SZ, _B, _B, ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_dynaverse_params_destroy", ctypes.c_int, [_P, ctypes.c_uint64] + _E),
    ("dvgpu_dynaverse_params_info", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.POINTER(DynaverseParamsInfo)] + _E),
    ("dvgpu_dynaverse_session_open", ctypes.c_int,
     [_P, ctypes.c_uint64, _P, _P, ctypes.POINTER(ctypes.c_uint64), _B] + _E),
    ("dvgpu_dynaverse_session_close", ctypes.c_int, [_P, ctypes.c_uint64] + _E),
    ("dvgpu_dynaverse_session_state", ctypes.c_int,
     [_P, ctypes.c_uint64, _B, _B, _B, ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_dynaverse_submit", ctypes.c_int,
     [_P, ctypes.c_uint64, _P, _P, _SZ, _P, _P, _SZ, ctypes.POINTER(ctypes.c_uint64)] + _E),
    ("dvgpu_dynaverse_wait", ctypes.c_int, [_P, ctypes.c_uint64, _B, ctypes.POINTER(DynaverseResult)] + _E),
    ("dvgpu_dynaverse_update", ctypes.c_int, [_P, ctypes.c_uint64, _P, _P, _SZ, _P, _P, _SZ, _B] + _E),
    ("dvgpu_dynaverse_verify", ctypes.c_int, [_P, ctypes.c_uint64, _P, _P, _B] + _E),
    ("dvgpu_dynaverse_set_max_batch", ctypes.c_int, [_P, ctypes.c_uint32]),
    ("dvgpu_dynaverse_stats", ctypes.c_int, [_P, ctypes.POINTER(DynaverseStats)]),
]


def lib():
    """Load libdvgpu.so.  Fails loudly when the CUDA library is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libdvgpu.so not built ({LIB_PATH}); run zkp-dynaverse_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(data):
    """Pointer to a bytes / bytearray / numpy buffer (None for empty)."""
    if data is None:
        return None
    if isinstance(data, np.ndarray):
        return data.ctypes.data if data.size else None
    if isinstance(data, (bytes, bytearray, memoryview)):
        if len(data) == 0:
            return None
        arr = np.frombuffer(data, dtype=np.uint8)
        return arr.ctypes.data
    raise TypeError(f"unsupported buffer type {type(data)}")


def _as_bytes(data):
    if isinstance(data, np.ndarray):
        return data.tobytes()
    return bytes(data)


def encode_fr(v: int) -> bytes:
    if not 0 <= v < R_MODULUS:
        raise ValueError("scalar out of range")
    return v.to_bytes(32, "little")


def decode_fr(b: bytes) -> int:
    """Rejects non-canonical encodings (crates/gpu/src/codec.rs:43-49)."""
    if len(b) != FR_BYTES:
        raise ValueError("scalar must be exactly 32 bytes")
    v = int.from_bytes(b, "little")
    if v >= R_MODULUS:
        raise ValueError("non-canonical or invalid scalar bytes")
    return v


def ntt_noalloc(d_values: int, n: int, kind: int, d_result: int, stream=None):
    """Allocation-free NTT on device buffers (dvgpu_bn254_ntt_noalloc): for
    callers that cannot allocate device memory at call time; n <= 65536.
    Its working memory is a static device array shared by all calls, so
    calls must not overlap on the GPU."""
    err = ctypes.create_string_buffer(256)
    rc = lib().dvgpu_bn254_ntt_noalloc(d_values, n, kind, d_result, stream, err, len(err))
    if rc != 0:
        raise DvgpuError(rc, err.value.decode(errors="replace"))


DYNAVERSE_PROOF_BYTES = 9304


def _fr_bytes(values) -> bytes:
    """Field elements as concatenated canonical bytes (ints or bytes)."""
    if isinstance(values, (bytes, bytearray)):
        return bytes(values)
    return b"".join(encode_fr(v % R_MODULUS) for v in values)


class DynaverseEngine:
    """Dynaverse update proofs on the device (dvgpu_dynaverse_*): the
    prover behind UpdateSession (crates/protocol/src/dynaverse/session.rs)
    with every proof composed and verified on the GPU.  Parameters and
    sessions stay resident; submit() queues an update from any thread, the
    worker merges the pending updates of up to max_batch sessions into
    shared launches (continuous batching); max_batch = 1 is the per-call
    form.  Proof bytes: DYNAVERSE_PROOF_BYTES in the layout of
    include/dynaverse_gpu.h."""

    def __init__(self, hbm_budget_bytes: int, max_batch: int = 64):
        self._L = lib()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self._L.dvgpu_dynaverse_create(hbm_budget_bytes, max_batch, ctypes.byref(h), err, len(err))
        if rc != 0:
            raise DvgpuError(rc, err.value.decode(errors="replace"))
        self._h = h

    def _call(self, name, *args):
        err = ctypes.create_string_buffer(512)
        rc = getattr(self._L, name)(self._h, *args, err, len(err))
        if rc != 0:
            raise DvgpuError(rc, err.value.decode(errors="replace"))

    def params_create(self, n: int, tau_x: int, tau_y: int) -> int:
        """DynaverseParams for ToyCircuit(n) from the two trapdoors."""
        h = ctypes.c_uint64()
        self._call("dvgpu_dynaverse_params_create", n, encode_fr(tau_x % R_MODULUS), encode_fr(tau_y % R_MODULUS),
                   ctypes.byref(h))
        return h.value

    def params_destroy(self, params: int):
        self._call("dvgpu_dynaverse_params_destroy", params)

    def params_info(self, params: int) -> DynaverseParamsInfo:
        info = DynaverseParamsInfo()
        self._call("dvgpu_dynaverse_params_info", params, ctypes.byref(info))
        return info

    def open_session(self, params: int, public_inputs, witness):
        """start_update_session: returns (session, anchor proof bytes)."""
        pub, wit = _fr_bytes(public_inputs), _fr_bytes(witness)
        s = ctypes.c_uint64()
        proof = ctypes.create_string_buffer(DYNAVERSE_PROOF_BYTES)
        self._call("dvgpu_dynaverse_session_open", params, _ptr(pub), _ptr(wit), ctypes.byref(s), proof)
        return s.value, proof.raw

    def close_session(self, session: int):
        self._call("dvgpu_dynaverse_session_close", session)

    def session_state(self, session: int, n: int):
        """(witness bytes, public input bytes, proof bytes, anchor distance)."""
        w = ctypes.create_string_buffer(32 * 6 * n)
        p = ctypes.create_string_buffer(32 * n)
        proof = ctypes.create_string_buffer(DYNAVERSE_PROOF_BYTES)
        d = ctypes.c_uint64()
        self._call("dvgpu_dynaverse_session_state", session, w, p, proof, ctypes.byref(d))
        return w.raw, p.raw, proof.raw, d.value

    @staticmethod
    def _update_args(indices, values, public_indices, public_values):
        idx = np.ascontiguousarray(np.asarray(list(indices), dtype=np.uint64))
        pidx = np.ascontiguousarray(np.asarray(list(public_indices), dtype=np.uint64))
        vals, pvals = _fr_bytes(values), _fr_bytes(public_values)
        if len(vals) != 32 * idx.size or len(pvals) != 32 * pidx.size:
            raise ValueError("update indices/values length mismatch")
        return idx, vals, pidx, pvals

    def submit(self, session: int, indices, values, public_indices=(), public_values=()) -> int:
        idx, vals, pidx, pvals = self._update_args(indices, values, public_indices, public_values)
        t = ctypes.c_uint64()
        self._call("dvgpu_dynaverse_submit", session, _ptr(idx), _ptr(vals), idx.size, _ptr(pidx), _ptr(pvals),
                   pidx.size, ctypes.byref(t))
        return t.value

    def wait(self, ticket: int):
        """(proof bytes, DynaverseResult) of a submitted update."""
        proof = ctypes.create_string_buffer(DYNAVERSE_PROOF_BYTES)
        res = DynaverseResult()
        self._call("dvgpu_dynaverse_wait", ticket, proof, ctypes.byref(res))
        return proof.raw, res

    def update(self, session: int, indices, values, public_indices=(), public_values=()) -> bytes:
        """UpdateSession::update_with_public_inputs (session.rs:39-41)."""
        idx, vals, pidx, pvals = self._update_args(indices, values, public_indices, public_values)
        proof = ctypes.create_string_buffer(DYNAVERSE_PROOF_BYTES)
        self._call("dvgpu_dynaverse_update", session, _ptr(idx), _ptr(vals), idx.size, _ptr(pidx), _ptr(pvals),
                   pidx.size, proof)
        return proof.raw

    def verify(self, params: int, public_inputs, proof: bytes) -> bool:
        """DynaverseVerifyingKey::verify on the device."""
        pub = _fr_bytes(public_inputs)
        ok = ctypes.create_string_buffer(1)
        self._call("dvgpu_dynaverse_verify", params, _ptr(pub), _ptr(bytes(proof)), ok)
        return ok.raw[0] == 1

    def set_max_batch(self, m: int):
        self._L.dvgpu_dynaverse_set_max_batch(self._h, m)

    def stats(self) -> DynaverseStats:
        s = DynaverseStats()
        self._L.dvgpu_dynaverse_stats(self._h, ctypes.byref(s))
        return s

    def close(self):
        if getattr(self, "_h", None):
            self._L.dvgpu_dynaverse_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class DvgpuServer:
    """Serving engine for commitment updates (dvgpu_serve_*): resident
    sessions, continuous batching across sessions; max_batch = 1 is the
    per-call form.  submit() may be called from any thread."""

    def __init__(self, hbm_budget_bytes: int, max_batch: int = 64):
        self._L = lib()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self._L.dvgpu_serve_create(hbm_budget_bytes, max_batch, ctypes.byref(h), err, len(err))
        if rc != 0:
            raise DvgpuError(rc, err.value.decode(errors="replace"))
        self.handle = h

    def _call(self, name, *args):
        err = ctypes.create_string_buffer(512)
        rc = getattr(self._L, name)(self.handle, *args, err, len(err))
        if rc != 0:
            raise DvgpuError(rc, err.value.decode(errors="replace"))

    def open_session(self, srs_g1: bytes, values: bytes):
        """Returns (session id, initial commitment: 64-byte affine G1)."""
        n = len(values) // FR_BYTES
        if len(srs_g1) != n * G1_BYTES:
            raise ValueError("SRS and value vector lengths differ")
        sid = ctypes.c_uint64()
        out = ctypes.create_string_buffer(G1_BYTES)
        self._call("dvgpu_serve_open_session", _ptr(srs_g1), _ptr(values), n, ctypes.byref(sid), out)
        return sid.value, out.raw

    def close_session(self, session: int):
        self._call("dvgpu_serve_close_session", session)

    def submit(self, session: int, indices, values: bytes) -> int:
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64))
        t = ctypes.c_uint64()
        self._call("dvgpu_serve_submit", session, idx.ctypes.data if idx.size else None, _ptr(values), len(idx),
                   ctypes.byref(t))
        return t.value

    def wait(self, ticket: int):
        """Returns (new commitment, ServeResult)."""
        out = ctypes.create_string_buffer(G1_BYTES)
        res = ServeResult()
        self._call("dvgpu_serve_wait", ticket, out, ctypes.byref(res))
        return out.raw, res

    def set_max_batch(self, m: int):
        self._L.dvgpu_serve_set_max_batch(self.handle, m)

    def stats(self) -> ServeStats:
        st = ServeStats()
        self._L.dvgpu_serve_stats(self.handle, ctypes.byref(st))
        return st

    def close(self):
        if getattr(self, "handle", None):
            self._L.dvgpu_serve_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class DvgpuBackend:
    """One native owner (crates/gpu/src/icicle.rs:98-110 IcicleBackend).

    Not thread-safe: one backend per caller thread, as in the reference."""

    def __init__(self, large_bucket_factor=0):
        self._L = lib()
        self._err = ctypes.create_string_buffer(512)
        h = ctypes.c_void_p()
        rc = self._L.dvgpu_backend_create_with_large_bucket_factor(large_bucket_factor, ctypes.byref(h),
                                                                    self._err, len(self._err))
        self._check(rc)
        if not h.value:
            raise DvgpuError(-3, "native backend returned a null owner")
        self.handle = h
        self.large_bucket_factor = large_bucket_factor

    # ------------------------------------------------------------------ plumbing
    def _check(self, rc):
        if rc != 0:
            raise DvgpuError(rc, self._err.value.decode(errors="replace"))

    def _call(self, name, *args):
        rc = getattr(self._L, name)(self.handle, *args, self._err, len(self._err))
        self._check(rc)

    def close(self):
        if getattr(self, "handle", None):
            self._L.dvgpu_backend_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ info
    def device_identity(self) -> str:
        out = ctypes.create_string_buffer(320)
        self._call("dvgpu_backend_device_identity", out, len(out))
        return out.value.decode()

    def memory_info(self):
        info = MemoryInfo()
        self._call("dvgpu_backend_memory_info", ctypes.byref(info))
        return info.free_bytes, info.total_bytes

    def batch_stats(self) -> BatchStats:
        s = BatchStats()
        rc = self._L.dvgpu_backend_batch_stats(self.handle, ctypes.byref(s))
        if rc != 0:
            raise DvgpuError(rc, "invalid native batch stats owner")
        return s

    def gpu_capabilities(self):
        return {"g1_msm": True, "fr_ntt": True, "g2_msm": True}

    # ------------------------------------------------------------------ MSM
    def msm(self, points: bytes, scalars: bytes) -> bytes:
        """G1 sum s_i P_i -> 64-byte affine (types.rs:295-299)."""
        n = len(scalars) // FR_BYTES
        if len(points) != n * G1_BYTES or len(scalars) != n * FR_BYTES:
            raise ValueError("MSM length mismatch")
        out = ctypes.create_string_buffer(G1_BYTES)
        self._call("dvgpu_bn254_msm", _ptr(points), _ptr(scalars), n, out)
        return out.raw

    def msm_with_timeline(self, points: bytes, scalars: bytes, label: bytes = b"msm"):
        """dvgpu_bn254_msm_timeline: (64-byte affine, MsmTimings, MsmTimeline)."""
        n = len(scalars) // FR_BYTES
        if len(points) != n * G1_BYTES or len(scalars) != n * FR_BYTES:
            raise ValueError("MSM length mismatch")
        out = ctypes.create_string_buffer(G1_BYTES)
        tm, tl = MsmTimings(), MsmTimeline()
        self._call("dvgpu_bn254_msm_timeline", _ptr(points), _ptr(scalars), n, out, label, ctypes.byref(tm),
                   ctypes.byref(tl))
        return out.raw, tm, tl

    def msm_g2_host(self, points: bytes, scalars: bytes) -> bytes:
        """G2 sum s_i Q_i -> 128-byte affine (types.rs:351-356)."""
        n = len(scalars) // FR_BYTES
        if len(points) != n * G2_BYTES or len(scalars) != n * FR_BYTES:
            raise ValueError("G2 MSM length mismatch")
        out = ctypes.create_string_buffer(G2_BYTES)
        self._call("dvgpu_bn254_g2_msm", _ptr(points), _ptr(scalars), n, out)
        return out.raw

    def msm_batch(self, point_sets, shared_scalars: bytes, offsets, lengths):
        """BatchMsmRequest (types.rs:254-259): set i uses point_sets[i][:lengths[i]]
        against shared_scalars[offsets[i] : offsets[i] + lengths[i]].  Uneven
        sets run in one native launch sequence, without padding."""
        count = len(point_sets)
        if len(offsets) != count or len(lengths) != count:
            raise ValueError("batch shape mismatch")
        n_sc = len(shared_scalars) // FR_BYTES
        pts, scs, set_off = [], [], [0]
        for i in range(count):
            L = lengths[i]
            if offsets[i] + L > n_sc:
                raise ValueError("scalar range out of bounds")
            if L * G1_BYTES > len(point_sets[i]):
                raise ValueError("point range out of bounds")
            pts.append(bytes(point_sets[i][:L * G1_BYTES]))
            scs.append(bytes(shared_scalars[offsets[i] * FR_BYTES:(offsets[i] + L) * FR_BYTES]))
            set_off.append(set_off[-1] + L)
        return self.msm_batch_uneven(b"".join(pts), b"".join(scs), set_off)

    def msm_batch_uneven(self, points: bytes, scalars: bytes, set_offsets):
        count = len(set_offsets) - 1
        if count <= 0:
            return []
        offs = np.ascontiguousarray(np.asarray(set_offsets, dtype=np.uint64))
        if len(points) != int(offs[-1]) * G1_BYTES or len(scalars) != int(offs[-1]) * FR_BYTES:
            raise ValueError("batch buffer length mismatch")
        out = ctypes.create_string_buffer(count * G1_BYTES)
        self._call("dvgpu_bn254_msm_batch_uneven", _ptr(points), _ptr(scalars), offs.ctypes.data, count, out)
        raw = out.raw
        return [raw[i * G1_BYTES:(i + 1) * G1_BYTES] for i in range(count)]

    def msm_batch_padded(self, points: bytes, scalars: bytes, length: int, count: int):
        """The reference's native padded batch (dvgpu_bn254_msm_batch)."""
        out = ctypes.create_string_buffer(count * G1_BYTES)
        self._call("dvgpu_bn254_msm_batch", _ptr(points), _ptr(scalars), length, count, out)
        raw = out.raw
        return [raw[i * G1_BYTES:(i + 1) * G1_BYTES] for i in range(count)]

    def msm_sparse_batch(self, requests):
        """SparseMsmRequest list (types.rs:262-345): each request is
        (bases: bytes, entries: [(index, scalar_bytes)]).  Every index is
        validated before any dispatch; results in request order."""
        lengths = []
        pts, scs, set_off = [], [], [0]
        for bases, entries in requests:
            nb = len(bases) // G1_BYTES
            for idx, _ in entries:
                if not 0 <= idx < nb:
                    raise ValueError("sparse MSM index out of range")
            for idx, val in entries:
                pts.append(bases[idx * G1_BYTES:(idx + 1) * G1_BYTES])
                scs.append(bytes(val))
            lengths.append(len(entries))
            set_off.append(set_off[-1] + len(entries))
        if not requests:
            return []
        return self.msm_batch_uneven(b"".join(pts), b"".join(scs), set_off)

    # resident bases + sparse-index MSM over them (no host gather)
    def register_bases(self, points: bytes, g2=False) -> int:
        size = G2_BYTES if g2 else G1_BYTES
        h = ctypes.c_uint64()
        self._call("dvgpu_bases_register", _ptr(points), len(points) // size, int(g2), ctypes.byref(h))
        return h.value

    def precompute_bases(self, handle: int, c: int = 0) -> int:
        """Attach precomputed window multiples to registered bases; returns c."""
        used = ctypes.c_int()
        self._call("dvgpu_bases_precompute", handle, c, ctypes.byref(used))
        return used.value

    def release_bases(self, handle: int):
        self._L.dvgpu_bases_release(self.handle, handle)

    def sparse_msm_resident(self, handle: int, indices, values: bytes, request_offsets):
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64))
        offs = np.ascontiguousarray(np.asarray(request_offsets, dtype=np.uint64))
        count = len(offs) - 1
        out = ctypes.create_string_buffer(max(1, count) * G1_BYTES)
        self._call("dvgpu_bn254_msm_sparse_batch", handle, idx.ctypes.data if idx.size else None,
                   _ptr(values), offs.ctypes.data, count, out)
        raw = out.raw
        return [raw[i * G1_BYTES:(i + 1) * G1_BYTES] for i in range(count)]

    def set_window(self, c: int):
        if self._L.dvgpu_msm_set_window(self.handle, c) != 0:
            raise DvgpuError(-1, "invalid window width")

    def autotune_msm(self, n: int, g2=False):
        """Time candidate window widths for n points; returns (best_c, log dict)."""
        import json
        c = ctypes.c_int()
        log = ctypes.create_string_buffer(8192)
        self._call("dvgpu_msm_autotune", n, int(g2), ctypes.byref(c), log, len(log))
        return c.value, json.loads(log.value.decode())

    def window_for(self, points_per_set: int) -> int:
        c = ctypes.c_int()
        self._L.dvgpu_msm_get_window(self.handle, points_per_set, ctypes.byref(c))
        return c.value

    # ------------------------------------------------------------------ NTT
    def ntt(self, values: bytes, inverse: bool) -> bytes:
        """Natural-order Fr transform, inverse includes 1/n (types.rs:347)."""
        n = len(values) // FR_BYTES
        if n == 0 or n & (n - 1) or len(values) != n * FR_BYTES:
            raise ValueError(f"ntt size {n} is not a power of two")
        out = ctypes.create_string_buffer(n * FR_BYTES)
        self._call("dvgpu_bn254_ntt_ex", _ptr(values), n, int(bool(inverse)), out)
        return out.raw

    def ntt_with_root(self, values: bytes, inverse: bool, root: bytes) -> bytes:
        """The reference ABI form with the explicit 2^20 root (icicle.rs:440-446)."""
        n = len(values) // FR_BYTES
        out = ctypes.create_string_buffer(max(1, n) * FR_BYTES)
        self._call("dvgpu_bn254_ntt", _ptr(values), n, int(bool(inverse)), root, out)
        return out.raw[:n * FR_BYTES]

    def ntt_coset(self, values: bytes, inverse: bool) -> bytes:
        n = len(values) // FR_BYTES
        if n == 0 or n & (n - 1):
            raise ValueError(f"ntt size {n} is not a power of two")
        out = ctypes.create_string_buffer(n * FR_BYTES)
        self._call("dvgpu_bn254_ntt_ex", _ptr(values), n, NTT_COSET_INVERSE if inverse else NTT_COSET_FORWARD, out)
        return out.raw

    # ------------------------------------------------------------------ fixed base
    def fixed_base_g1(self, scalars: bytes) -> bytes:
        n = len(scalars) // FR_BYTES
        out = ctypes.create_string_buffer(max(1, n) * G1_BYTES)
        self._call("dvgpu_bn254_fixed_base", _ptr(scalars), n, 0, out)
        return out.raw[:n * G1_BYTES]

    def fixed_base_g2(self, scalars: bytes) -> bytes:
        n = len(scalars) // FR_BYTES
        out = ctypes.create_string_buffer(max(1, n) * G2_BYTES)
        self._call("dvgpu_bn254_fixed_base", _ptr(scalars), n, 1, out)
        return out.raw[:n * G2_BYTES]

    def setup_stats(self) -> SetupStats:
        s = SetupStats()
        self._L.dvgpu_setup_stats(self.handle, ctypes.byref(s))
        return s

    # ------------------------------------------------------------------ G2 validation
    def inspect_g2_validation(self, wire: bytes, algorithm: int):
        """Status-only batched inspector (g2_validation.rs:124-135,191-203)."""
        if len(wire) % G2_BYTES or algorithm not in (1, 2, 3):
            raise ValueError("invalid G2 validation input")
        n = len(wire) // G2_BYTES
        masks = np.zeros(max(1, n), dtype=np.uint32)
        rep = G2ValidationReport()
        self._call("dvgpu_bn254_g2_validation_inspect", _ptr(wire), n, algorithm, masks.ctypes.data,
                   ctypes.byref(rep))
        return masks[:n], rep

    def g2_kernel_config(self, config=None):
        """Get (config None) or set the G2 check kernel configuration
        (G2KernelConfig or a (threads, schedule, layout, fused) tuple)."""
        if config is None:
            c = G2KernelConfig()
            if self._L.dvgpu_g2_kernel_config_get(self.handle, ctypes.byref(c)) != 0:
                raise DvgpuError(-1, "invalid G2 kernel config owner")
            return c
        c = config if isinstance(config, G2KernelConfig) else G2KernelConfig(*config)
        rc = self._L.dvgpu_g2_kernel_config_set(self.handle, ctypes.byref(c))
        if rc != 0:
            raise DvgpuError(rc, "invalid or retired G2 kernel config")
        return c

    def g2_kernel_resources(self, algorithm: int):
        r = G2KernelResources()
        rc = self._L.dvgpu_g2_kernel_resources(self.handle, algorithm, ctypes.byref(r))
        if rc != 0:
            raise DvgpuError(rc, "G2 kernel resource query failed")
        return r

    def g2_experiment_stats(self):
        st = G2ExperimentStats()
        if self._L.dvgpu_g2_experiment_stats(self.handle, ctypes.byref(st)) != 0:
            raise DvgpuError(-1, "invalid G2 experiment owner")
        return st

    def fixed_base_g2_checked(self, scalars: bytes, algorithm: int):
        n = len(scalars) // FR_BYTES
        out = ctypes.create_string_buffer(max(1, n) * G2_BYTES)
        rep = G2ValidationReport()
        self._call("dvgpu_bn254_fixed_base_g2_checked", _ptr(scalars), n, algorithm, out, ctypes.byref(rep))
        return out.raw[:n * G2_BYTES], rep

    # ------------------------------------------------------------------ device forms
    def msm_device(self, d_points: int, d_scalars: int, n: int, g2=False, stream=None) -> bytes:
        out = ctypes.create_string_buffer(G2_BYTES if g2 else G1_BYTES)
        self._call("dvgpu_bn254_msm_device", d_points, d_scalars, n, int(g2), out, stream)
        return out.raw

    def sparse_msm_device(self, handle: int, d_indices: int, d_values: int, request_offsets, stream=None):
        offs = np.ascontiguousarray(np.asarray(request_offsets, dtype=np.uint64))
        count = len(offs) - 1
        out = ctypes.create_string_buffer(max(1, count) * G1_BYTES)
        self._call("dvgpu_bn254_msm_sparse_device", handle, d_indices, d_values, offs.ctypes.data, count, out, stream)
        raw = out.raw
        return [raw[i * G1_BYTES:(i + 1) * G1_BYTES] for i in range(count)]

    def msm_resident_host(self, handle: int, scalars: bytes, g2=False) -> bytes:
        """MSM over registered bases with host scalars (dvgpu_bn254_msm_resident_host)."""
        out = ctypes.create_string_buffer(G2_BYTES if g2 else G1_BYTES)
        self._call("dvgpu_bn254_msm_resident_host", handle, _ptr(scalars), len(scalars) // FR_BYTES, out)
        return out.raw

    def msm_resident(self, handle: int, d_scalars: int, n: int, stream=None, g2=False) -> bytes:
        out = ctypes.create_string_buffer(G2_BYTES if g2 else G1_BYTES)
        self._call("dvgpu_bn254_msm_resident", handle, d_scalars, n, out, stream)
        return out.raw

    def ntt_device(self, d_values: int, n: int, kind: int, d_out: int, stream=None):
        self._call("dvgpu_bn254_ntt_device", d_values, n, kind, d_out, stream)

    def fixed_base_device(self, d_scalars: int, n: int, g2: bool, d_out: int, stream=None):
        self._call("dvgpu_bn254_fixed_base_device", d_scalars, n, int(g2), d_out, stream)

    def g2_check_device(self, d_wire: int, n: int, algorithm: int, d_masks: int, stream=None):
        rep = G2ValidationReport()
        self._call("dvgpu_bn254_g2_check_device", d_wire, n, algorithm, d_masks, ctypes.byref(rep), stream)
        return rep

    def launch_count(self) -> int:
        return int(self._L.dvgpu_launch_count())

    def msm_timeline(self, enable: bool) -> MsmPhaseTimes:
        t = MsmPhaseTimes()
        if self._L.dvgpu_msm_timeline(self.handle, int(enable), ctypes.byref(t)) != 0:
            raise DvgpuError(-1, "timeline unavailable")
        return t

    def random_fr_device(self, seed: int, n: int, d_out: int, stream=None):
        self._call("dvgpu_random_fr_device", seed, n, d_out, stream)

    def random_twist_device(self, seed: int, n: int, d_out: int, stream=None):
        """n random on-curve G2 twist points (wire form) outside the subgroup."""
        self._call("dvgpu_g2_random_twist_device", seed, n, d_out, stream)

    def fr_powers_device(self, d_tau: int, n: int, d_out: int, stream=None):
        self._call("dvgpu_fr_powers_device", d_tau, n, d_out, stream)

    # ------------------------------------------------------------------ G1 transform
    def g1_ntt_rows(self, points: bytes, row_len: int, inverse=False) -> bytes:
        """Rows of row_len G1 points through the Fr-domain FFT (EC-NTT),
        affine results (RebuildBackend::transform_rows, kind G1)."""
        if row_len <= 0 or len(points) % (G1_BYTES * row_len):
            raise ValueError("points must hold whole rows")
        rows = len(points) // (G1_BYTES * row_len)
        out = ctypes.create_string_buffer(max(1, len(points)))
        self._call("dvgpu_bn254_g1_ntt_rows", _ptr(points), row_len, rows, int(inverse), out)
        return out.raw[:len(points)]

    def g1_ntt_rows_device(self, d_points: int, row_len: int, rows: int, inverse: bool, d_out: int, stream=None):
        self._call("dvgpu_bn254_g1_ntt_rows_device", d_points, row_len, rows, int(inverse), d_out, stream)

    # ------------------------------------------------------------------ pairing checks
    # crates/protocol/src/verification.rs:37-144
    def pairing_check(self, g1: bytes, g2: bytes, offsets) -> list:
        """Verdicts of prod_{k in [offsets[e], offsets[e+1])} e(P_k, Q_k) == 1."""
        import numpy as np
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
        eqs = len(off) - 1
        out = ctypes.create_string_buffer(max(1, eqs))
        self._call("dvgpu_bn254_pairing_check", g1, g2, off.ctypes.data, eqs, out)
        return [bool(x) for x in out.raw[:eqs]]

    def g2_prepare(self, g2: bytes) -> int:
        """Prepared G2 points (their Miller-loop lines kept on the device)."""
        h = ctypes.c_uint64()
        self._call("dvgpu_bn254_g2_prepare", g2, len(g2) // G2_BYTES, ctypes.byref(h))
        return h.value

    def g2_prepared_release(self, handle: int):
        self._call("dvgpu_bn254_g2_prepared_release", handle)

    def pairing_check_prepared(self, g1: bytes, handle: int, q_index, offsets) -> list:
        """Verdicts with term k = (g1[k], prepared point q_index[k])."""
        import numpy as np
        qi = np.ascontiguousarray(np.asarray(q_index, dtype=np.uint32))
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
        eqs = len(off) - 1
        out = ctypes.create_string_buffer(max(1, eqs))
        self._call("dvgpu_bn254_pairing_check_prepared", g1, handle, qi.ctypes.data if qi.size else None,
                   off.ctypes.data, eqs, out)
        return [bool(x) for x in out.raw[:eqs]]

    def pairing(self, g1: bytes, g2: bytes) -> bytes:
        """e(P_i, Q_i): 384-byte GT elements (tower order, canonical)."""
        n = len(g1) // G1_BYTES
        out = ctypes.create_string_buffer(max(1, 384 * n))
        self._call("dvgpu_bn254_pairing", g1, g2, n, out)
        return out.raw[:384 * n]

    # ------------------------------------------------------------------ polynomial toolkit
    # crates/protocol/src/domain/fast.rs over canonical Fr coefficient bytes
    # (lowest degree first); results trimmed as domain.rs:339-346.
    def poly_multiply(self, left: bytes, right: bytes) -> bytes:
        """fft_multiply_with_backend (fast.rs:213-234)."""
        cap = max(1, (len(left) // FR_BYTES + len(right) // FR_BYTES - 1) if left and right else 1)
        out = ctypes.create_string_buffer(FR_BYTES * cap)
        n = ctypes.c_size_t()
        self._call("dvgpu_bn254_poly_multiply", left, len(left) // FR_BYTES, right, len(right) // FR_BYTES, out, cap,
                   ctypes.byref(n))
        return out.raw[:FR_BYTES * n.value]

    def poly_divide_exact(self, numerator: bytes, denominator: bytes) -> bytes:
        """newton_divide_exact_with_backend (fast.rs:236-240)."""
        cap = max(1, len(numerator) // FR_BYTES)
        out = ctypes.create_string_buffer(FR_BYTES * cap)
        n = ctypes.c_size_t()
        self._call("dvgpu_bn254_poly_divide_exact", numerator, len(numerator) // FR_BYTES, denominator,
                   len(denominator) // FR_BYTES, out, cap, ctypes.byref(n))
        return out.raw[:FR_BYTES * n.value]

    def tree_create(self, points: bytes) -> "SubproductTree":
        return SubproductTree(self, points)

    # ------------------------------------------------------------------ resident buffers
    # RebuildBackend (crates/protocol/src/incremental_rebuild/operators.rs) over
    # the resident ABI, with the reference binding's field encoding
    # (crates/gpu/src/resident.rs:250-402).  Values: canonical bytes (Fr 32,
    # G1 64 affine, G2 128).
    def resident_configure(self, memory_limit: int, journal_bytes: int, root: bytes):
        self._call("dvgpu_resident_configure", memory_limit, journal_bytes, _ptr(root))

    def resident_call(self, opcode: str, keep=None, **fields) -> int:
        op = ResidentOp()
        op.opcode = RESIDENT_OPS[opcode]
        for k, v in fields.items():
            setattr(op, k, v)
        r = ctypes.c_uint64()
        self._call("dvgpu_resident_call", ctypes.byref(op), ctypes.byref(r))
        return r.value

    def resident_call_profiled(self, opcode: str, **fields):
        """dvgpu_resident_call_profiled: (result, ResidentProfile)."""
        op = ResidentOp()
        op.opcode = RESIDENT_OPS[opcode]
        for k, v in fields.items():
            setattr(op, k, v)
        r = ctypes.c_uint64()
        prof = ResidentProfile()
        self._call("dvgpu_resident_call_profiled", ctypes.byref(op), ctypes.byref(r), ctypes.byref(prof))
        return r.value, prof

    def rb_alloc(self, kind: int, length: int, writable: bool) -> int:
        return self.resident_call("ALLOC", kind=kind, length=length, flags=int(writable))

    def rb_register_bases(self, points: bytes) -> int:
        buf = ctypes.create_string_buffer(points, max(1, len(points)))
        return self.resident_call("ALLOC_BASES", length=len(points) // G1_BYTES, input=ctypes.addressof(buf))

    def rb_seal(self):
        self._L.dvgpu_resident_seal(self.handle)

    def rb_commit(self):
        self._L.dvgpu_resident_commit(self.handle)

    def rb_len(self, h: int) -> int:
        return self.resident_call("LENGTH", a=h)

    def rb_kind(self, h: int) -> int:
        return self.resident_call("KIND", a=h)

    def rb_begin(self):
        self.resident_call("BEGIN")

    def rb_rollback(self):
        self.resident_call("ROLLBACK")

    def rb_write(self, h: int, offset: int, data: bytes, kind: int):
        width = FR_BYTES if kind == 0 else G1_BYTES
        buf = ctypes.create_string_buffer(data, max(1, len(data)))
        self.resident_call("WRITE", kind=kind, a=h, a_offset=offset, length=len(data) // width,
                           input=ctypes.addressof(buf))

    def rb_read(self, h: int, offset: int, length: int, kind: int, flags: int = 0) -> bytes:
        width = FR_BYTES if kind == 0 else G1_BYTES
        out = ctypes.create_string_buffer(max(1, length * width))
        self.resident_call("READ", kind=kind, a=h, a_offset=offset, length=length, flags=flags,
                           output=ctypes.addressof(out))
        return out.raw[:length * width]

    def rb_copy(self, src, src_off, dst, dst_off, length):
        self.resident_call("COPY", a=src, a_offset=src_off, c=dst, c_offset=dst_off, length=length)

    def rb_reverse(self, kind, src, src_off, dst, dst_off, length):
        self.resident_call("REVERSE", kind=kind, a=src, a_offset=src_off, c=dst, c_offset=dst_off, length=length)

    def rb_transpose(self, kind, src, dst, rows, cols, start, length, root=None):
        buf = ctypes.create_string_buffer(root if root else bytes(32), 32)
        self.resident_call("TRANSPOSE", kind=kind, a=src, c=dst, rows=rows, cols=cols, a_offset=start, length=length,
                           flags=int(root is not None), input=ctypes.addressof(buf))

    def rb_transform_rows(self, kind, src, dst, row_len, first_row, row_count, inverse):
        self.resident_call("TRANSFORM", kind=kind, a=src, c=dst, cols=row_len, rows=row_count, a_offset=first_row,
                           flags=int(inverse))

    def rb_transform_packet(self, kind, src, scratch, dst, length, inverse):
        self.resident_call("TRANSFORM_PACKET", kind=kind, a=src, b=scratch, c=dst, length=length, flags=int(inverse))

    def rb_zip(self, op: int, left, left_off, right, right_off, dst, dst_off, length):
        self.resident_call("ZIP", flags=op, a=left, a_offset=left_off, b=right, b_offset=right_off, c=dst,
                           c_offset=dst_off, length=length)

    def rb_scale(self, pts, pts_off, sc, sc_off, dst, dst_off, length):
        self.resident_call("SCALE", a=pts, a_offset=pts_off, b=sc, b_offset=sc_off, c=dst, c_offset=dst_off,
                           length=length)

    def rb_msm_g1(self, pts, pts_off, sc, sc_off, length) -> bytes:
        out = ctypes.create_string_buffer(G1_BYTES)
        self.resident_call("MSM_G1", a=pts, a_offset=pts_off, b=sc, b_offset=sc_off, length=length,
                           output=ctypes.addressof(out))
        return out.raw

    def rb_msm_g2(self, points: bytes, sc, sc_off) -> bytes:
        inp = ctypes.create_string_buffer(points, max(1, len(points)))
        out = ctypes.create_string_buffer(G2_BYTES)
        self.resident_call("MSM_G2", b=sc, b_offset=sc_off, length=len(points) // G2_BYTES,
                           input=ctypes.addressof(inp), output=ctypes.addressof(out))
        return out.raw

    def rb_stats(self) -> ResidentStats:
        st = ResidentStats()
        self._L.dvgpu_resident_stats(self.handle, ctypes.byref(st))
        return st

    def rb_diagnostics(self) -> ResidentDiagnostics:
        d = ResidentDiagnostics()
        self._L.dvgpu_resident_diagnostics(self.handle, ctypes.byref(d))
        return d

    # ------------------------------------------------------------------ batching
    def ntt_batch(self, values: bytes, log_sizes, kinds=None) -> bytes:
        """Transforms of sizes 2^log_sizes[i] (concatenated canonical
        elements) in one persistent launch; kinds as in ntt_ex (None =
        forward)."""
        logs = np.ascontiguousarray(np.asarray(log_sizes, dtype=np.uint32))
        kd = None if kinds is None else np.ascontiguousarray(np.asarray(kinds, dtype=np.int32))
        out = ctypes.create_string_buffer(max(1, len(values)))
        self._call("dvgpu_bn254_ntt_batch", _ptr(values), logs.ctypes.data if logs.size else None,
                   None if kd is None else kd.ctypes.data, len(logs), out)
        return out.raw[:len(values)]

    def ntt_batch_device(self, d_values: int, log_sizes, d_out: int, kinds=None, stream=None):
        logs = np.ascontiguousarray(np.asarray(log_sizes, dtype=np.uint32))
        kd = None if kinds is None else np.ascontiguousarray(np.asarray(kinds, dtype=np.int32))
        self._call("dvgpu_bn254_ntt_batch_device", d_values, logs.ctypes.data if logs.size else None,
                   None if kd is None else kd.ctypes.data, len(logs), d_out, stream)

    def batch_plan_create(self, bases_handle: int, msm_sizes, ntt_log_sizes=(), ntt_kinds=None):
        """CUDA-graph plan of G1 MSMs over prefixes of registered bases plus
        NTTs; returns (plan handle, autotuner log dict)."""
        import json
        sizes = np.ascontiguousarray(np.asarray(msm_sizes, dtype=np.uint64))
        logs = np.ascontiguousarray(np.asarray(ntt_log_sizes, dtype=np.uint32))
        kd = None if ntt_kinds is None else np.ascontiguousarray(np.asarray(ntt_kinds, dtype=np.int32))
        h = ctypes.c_uint64()
        log = ctypes.create_string_buffer(1 << 16)
        self._call("dvgpu_batch_plan_create", bases_handle, sizes.ctypes.data if sizes.size else None, len(sizes),
                   logs.ctypes.data if logs.size else None, None if kd is None else kd.ctypes.data, len(logs),
                   ctypes.byref(h), log, len(log))
        return h.value, json.loads(log.value.decode())

    def batch_plan_buffers(self, plan: int) -> BatchPlanBuffers:
        b = BatchPlanBuffers()
        self._call("dvgpu_batch_plan_buffers", plan, ctypes.byref(b))
        return b

    def batch_plan_launch(self, plan: int, stream=None):
        self._call("dvgpu_batch_plan_launch", plan, stream)

    def batch_plan_check(self, plan: int):
        self._call("dvgpu_batch_plan_check", plan)

    def batch_plan_run(self, plan: int, scalars, ntt_values, msm_count: int):
        """Host inputs (concatenated, request order) -> (list of 64-byte MSM
        results, concatenated NTT outputs)."""
        msm_out = ctypes.create_string_buffer(max(1, msm_count) * G1_BYTES)
        nbytes = 0 if ntt_values is None else len(ntt_values)
        ntt_out = ctypes.create_string_buffer(max(1, nbytes))
        self._call("dvgpu_batch_plan_run", plan, _ptr(scalars), _ptr(ntt_values), msm_out, ntt_out)
        raw = msm_out.raw
        return [raw[i * G1_BYTES:(i + 1) * G1_BYTES] for i in range(msm_count)], ntt_out.raw[:nbytes]

    def batch_plan_destroy(self, plan: int):
        self._call("dvgpu_batch_plan_destroy", plan)

    def probe_imad_rate(self) -> float:
        v = ctypes.c_double()
        self._call("dvgpu_probe_imad_rate", ctypes.byref(v))
        return v.value


class SubproductTree:
    """SubproductTree::new_with_backend (crates/protocol/src/domain/fast.rs:11-139)
    held on the device: distinct canonical Fr points in input order."""

    def __init__(self, backend: DvgpuBackend, points: bytes):
        self.backend = backend
        self.count = len(points) // FR_BYTES
        h = ctypes.c_uint64()
        backend._call("dvgpu_bn254_tree_create", points, self.count, ctypes.byref(h))
        self.handle = h.value

    def close(self):
        if getattr(self, "handle", None) and getattr(self.backend, "handle", None):
            self.backend._call("dvgpu_bn254_tree_destroy", self.handle)
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def vanishing(self) -> bytes:
        out = ctypes.create_string_buffer(FR_BYTES * (self.count + 1))
        n = ctypes.c_size_t()
        self.backend._call("dvgpu_bn254_tree_vanishing", self.handle, out, self.count + 1, ctypes.byref(n))
        return out.raw[:FR_BYTES * n.value]

    def inverse_derivatives(self) -> bytes:
        out = ctypes.create_string_buffer(max(1, FR_BYTES * self.count))
        self.backend._call("dvgpu_bn254_tree_inverse_derivatives", self.handle, out, self.count)
        return out.raw[:FR_BYTES * self.count]

    def multipoint_eval(self, polynomial: bytes, rows: int = 1) -> bytes:
        """Values of `rows` polynomials (equal lengths, concatenated) at the points."""
        length = len(polynomial) // (FR_BYTES * rows)
        out = ctypes.create_string_buffer(max(1, FR_BYTES * self.count * rows))
        self.backend._call("dvgpu_bn254_tree_evaluate", self.handle, polynomial, length, rows, out)
        return out.raw[:FR_BYTES * self.count * rows]

    def interpolate(self, values: bytes, rows: int = 1):
        """Trimmed coefficients of each row (a list of bytes when rows > 1)."""
        count = len(values) // (FR_BYTES * rows)
        stride = max(1, self.count)
        out = ctypes.create_string_buffer(FR_BYTES * stride * rows)
        lens = (ctypes.c_size_t * rows)()
        self.backend._call("dvgpu_bn254_tree_interpolate", self.handle, values, count, rows, out, lens)
        res = [out.raw[FR_BYTES * stride * r:FR_BYTES * (stride * r + lens[r])] for r in range(rows)]
        return res[0] if rows == 1 else res

    def cauchy_sums(self, weights: bytes, rows: int = 1) -> bytes:
        count = len(weights) // (FR_BYTES * rows)
        out = ctypes.create_string_buffer(max(1, FR_BYTES * self.count * rows))
        self.backend._call("dvgpu_bn254_tree_cauchy_sums", self.handle, weights, count, rows, out)
        return out.raw[:FR_BYTES * self.count * rows]
