"""Loads ``libcellweave_b200.so`` and declares its C ABI for ctypes.

The library is the product: there is no CPU path.  Loading fails loudly when
the shared object is missing, and every call that fails raises the error the
reference would return (``CellweaveError``, crates/core/src/error.rs:7-23).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcellweave_b200.so")

OK, ERR_CONFIG, ERR_SIMULATION, ERR_ODE, ERR_NOT_FOUND, ERR_CUDA, ERR_TIMEOUT = range(7)


class CellweaveError(RuntimeError):
    """Base of every error the library returns."""


class ConfigError(CellweaveError):
    """CellweaveError::Config."""


class SimulationError(CellweaveError):
    """CellweaveError::Simulation (for example a field that did not settle)."""


class OdeSolverError(CellweaveError):
    """CellweaveError::OdeSolver."""


class NotFoundError(CellweaveError):
    """CellweaveError::NotFound."""


class CudaError(CellweaveError):
    """A CUDA call failed, or there is no usable device."""


class TimeoutError_(CellweaveError):
    """A bounded device loop ran out of iterations."""


_ERRORS = {ERR_CONFIG: ConfigError, ERR_SIMULATION: SimulationError, ERR_ODE: OdeSolverError,
           ERR_NOT_FOUND: NotFoundError, ERR_CUDA: CudaError, ERR_TIMEOUT: TimeoutError_}


class RelaxOpts(C.Structure):
    _fields_ = [("omega", C.c_double), ("stop", C.c_int32), ("tolerance", C.c_double), ("max_sweeps", C.c_int64),
                ("precision", C.c_int32), ("inner_sweeps", C.c_int32), ("block_depth", C.c_int32),
                ("window", C.c_int32), ("error_tolerance", C.c_double)]


class RelaxStats(C.Structure):
    _fields_ = [("sweeps", C.c_int64), ("last_change", C.c_double), ("residual", C.c_double),
                ("status", C.c_int32), ("omega", C.c_double)]


class TermSpec(C.Structure):
    _fields_ = [("node", C.c_int32), ("kind", C.c_int32), ("source", C.c_char_p), ("rate", C.c_double),
                ("hill_n", C.c_double), ("hill_k", C.c_double), ("param", C.c_double), ("has_hill", C.c_int32)]


class Mutation(C.Structure):
    _fields_ = [("node", C.c_int32), ("term", C.c_int32), ("kind", C.c_int32), ("change", C.c_int32),
                ("value", C.c_double), ("source", C.c_int32), ("suppressed", C.c_int32)]


class Measurements(C.Structure):
    _fields_ = [("mcs", C.c_uint64), ("cycling", C.c_uint64), ("quiescent", C.c_uint64), ("necrotic", C.c_uint64),
                ("born", C.c_uint64), ("gone", C.c_uint64), ("vessel", C.c_uint64), ("tissue_radius", C.c_double),
                ("necrotic_radius", C.c_double), ("viable_depth", C.c_double), ("exposure", C.c_double),
                ("differentiating", C.c_uint64), ("apoptotic", C.c_uint64), ("clones", C.c_uint64),
                ("lesion", C.c_uint64)]


class FitConfig(C.Structure):
    _fields_ = [("dcoef", C.c_double), ("uptake", C.c_double * 3), ("vessel_value", C.c_double),
                ("vessel_x", C.c_int32), ("egf", C.c_double), ("signal_dcoef", C.c_double),
                ("signal_decay", C.c_double), ("secretion", C.c_double), ("steps", C.c_int32),
                ("checkpoint_every", C.c_int32), ("dt", C.c_double), ("nbins", C.c_int32), ("bin_width", C.c_double),
                ("hypoxic_level", C.c_double), ("tau", C.c_double), ("signal_weight", C.c_double),
                ("tolerance", C.c_double), ("adjoint_tolerance", C.c_double), ("precision", C.c_int32),
                ("omega", C.c_double), ("network_params", C.c_int32)]


class SimConfig(C.Structure):
    _fields_ = [("nh", C.c_uint32), ("w", C.c_void_p), ("h", C.c_void_p), ("d", C.c_void_p),
                ("ncells", C.c_void_p), ("seeds", C.c_void_p), ("temperature", C.c_double), ("K", C.c_int32),
                ("J", C.c_void_p), ("contact_order", C.c_int32), ("target_volume", C.c_int32),
                ("lambda_volume", C.c_double), ("surface_target", C.c_int32), ("lambda_surface", C.c_double),
                ("seeding", C.c_int32), ("seed_side", C.c_int32), ("nfields", C.c_int32), ("o2_dcoef", C.c_double),
                ("o2_sink_by_type", C.c_void_p), ("o2_background_sink", C.c_double), ("o2_hold", C.c_int32), ("signal_dcoef", C.c_double),
                ("signal_decay", C.c_double), ("signal_secretion", C.c_double), ("hypoxic_level", C.c_double),
                ("tolerance", C.c_double), ("precision", C.c_int32), ("omega", C.c_double),
                ("inner_sweeps", C.c_int32), ("relax_every", C.c_int32), ("dt", C.c_double), ("substeps", C.c_int32), ("sweeps", C.c_int32),
                ("death_threshold", C.c_double), ("necrotic_type", C.c_int32), ("use_graphs", C.c_int32),
                ("divide", C.c_int32), ("max_cells", C.c_int32), ("spare_cells", C.c_int32),
                ("waste_production", C.c_double), ("necrotic_production", C.c_double),
                ("necrotic_release_for", C.c_int32), ("subsweeps", C.c_int32), ("o2_uptake", C.c_double),
                ("divide_every", C.c_int32), ("vessel_radius", C.c_int32), ("stop_rule", C.c_int32),
                ("first_tolerance", C.c_double), ("cycle_median", C.c_double), ("cycle_spread", C.c_double),
                ("debris_loss", C.c_double), ("still_medium", C.c_double),
                ("exposure_intensity", C.c_double), ("exposure_uptake", C.c_double), ("exposure_start", C.c_int32),
                ("exposure_on", C.c_int32), ("exposure_off", C.c_int32), ("mutation_rate", C.c_double),
                ("rewiring", C.c_double), ("field_off", C.c_int32), ("differentiated_type", C.c_int32),
                ("apoptotic_type", C.c_int32), ("lineage", C.c_int32), ("error_tolerance", C.c_double),
                ("suppress_before", C.c_int32), ("tracing", C.c_int32), ("tracing_at", C.c_int32)]


P = C.c_void_p
U32, I32, I64, U64, D = C.c_uint32, C.c_int32, C.c_int64, C.c_uint64, C.c_double

SIGNATURES = {
    "cw_last_error": (C.c_char_p, []),
    "cw_version": (C.c_int, []),
    "cw_set_stream": (C.c_int, [P]),
    "cw_set_device": (C.c_int, [I32]),
    "cw_get_stream": (P, []),
    "cw_synchronize": (C.c_int, []),
    "cw_launch_count": (C.c_uint64, []),
    "cw_sim_clones": (C.c_int, [P, U32, U32, P]),
    "cw_sim_clone_count": (C.c_int, [P, P]),
    "cw_sim_clone_records": (C.c_int, [P, P, P, P]),
    "cw_test_faults": (C.c_int, [U64, I32, I32, I32]),
    "cw_event_record_on": (C.c_int, [P, I32]),
    "cw_lattice_set_stream": (C.c_int, [P, P]),
    "cw_field_set_stream": (C.c_int, [P, P]),
    "cw_network_set_stream": (C.c_int, [P, P]),
    "cw_sim_set_stream": (C.c_int, [P, P]),
    "cw_lattice_get_stream": (P, [P]),
    "cw_field_get_stream": (P, [P]),
    "cw_network_get_stream": (P, [P]),
    "cw_sim_get_stream": (P, [P]),
    "cw_lattice_last_error": (C.c_char_p, [P]),
    "cw_field_last_error": (C.c_char_p, [P]),
    "cw_network_last_error": (C.c_char_p, [P]),
    "cw_sim_last_error": (C.c_char_p, [P]),
    "cw_fit_last_error": (C.c_char_p, [P]),
    "cw_lattice_create": (C.c_int, [U32, P, P, P, P, D, P]),
    "cw_lattice_destroy": (C.c_int, [P]),
    "cw_lattice_count": (C.c_int, [P, P]),
    "cw_lattice_set_copy_nbhd": (C.c_int, [P, I32]),
    "cw_lattice_divide": (C.c_int, [P, U32, U32, P, P, P]),
    "cw_lattice_cell_count": (C.c_int, [P, U32, P]),
    "cw_lattice_capacity": (C.c_int, [P, U32, P]),
    "cw_lattice_pass_rounds": (C.c_int, [P, P]),
    "cw_lattice_set_contact": (C.c_int, [P, I32, P, I32]),
    "cw_lattice_set_temperature": (C.c_int, [P, D]),
    "cw_lattice_upload": (C.c_int, [P, U32, P]),
    "cw_lattice_download": (C.c_int, [P, U32, P]),
    "cw_lattice_upload_all": (C.c_int, [P, P]),
    "cw_lattice_download_all": (C.c_int, [P, P]),
    "cw_cells_set": (C.c_int, [P, U32, U32, P, P, P, P]),
    "cw_cells_get": (C.c_int, [P, U32, U32, P, P, P, P]),
    "cw_cells_set_surface": (C.c_int, [P, U32, U32, P, P]),
    "cw_cells_get_surface": (C.c_int, [P, U32, U32, P]),
    "cw_lattice_set_seed": (C.c_int, [P, U32, U64]),
    "cw_lattice_set_mcs": (C.c_int, [P, U32]),
    "cw_lattice_get_mcs": (C.c_int, [P, P]),
    "cw_lattice_mcs": (C.c_int, [P, U32]),
    "cw_lattice_delta_h_batch": (C.c_int, [P, U32, U32, P, P, P]),
    "cw_lattice_verify": (C.c_int, [P, U32, P]),
    "cw_field_create": (C.c_int, [U32, P, P, P, D, D, D, P]),
    "cw_field_destroy": (C.c_int, [P]),
    "cw_field_set_source": (C.c_int, [P, D]),
    "cw_field_set_diffusion": (C.c_int, [P, D]),
    "cw_field_set_floor": (C.c_int, [P, I32]),
    "cw_field_upload": (C.c_int, [P, U32, I32, P]),
    "cw_field_download": (C.c_int, [P, U32, I32, P]),
    "cw_field_upload_held": (C.c_int, [P, U32, P]),
    "cw_field_download_held": (C.c_int, [P, U32, P]),
    "cw_field_fill": (C.c_int, [P, D]),
    "cw_field_clear": (C.c_int, [P, I32]),
    "cw_field_release_all": (C.c_int, [P]),
    "cw_field_hold_mask": (C.c_int, [P, U32, P, D]),
    "cw_field_hold_bath": (C.c_int, [P, U32, P, D]),
    "cw_field_relax": (C.c_int, [P, P, P]),
    "cw_field_residual": (C.c_int, [P, P]),
    "cw_field_inflow": (C.c_int, [P, P]),
    "cw_field_step": (C.c_int, [P, D]),
    "cw_field_relax_noalloc": (C.c_int, [P, P, P, P, P, U32, U32, D, D, D, D, D, I64, I32, P, P]),
    "cw_field_relax_adjoint": (C.c_int, [P, P, P, P, P]),
    "cw_field_time_inner": (C.c_int, [P, I32, I32, I32, D, P, P]),
    "cw_field_inner_correction": (C.c_int, [P, U32, P]),
    "cw_couple_uptake": (C.c_int, [P, P, I32, P, I32]),
    "cw_couple_background_uptake": (C.c_int, [P, P, D]),
    "cw_couple_production": (C.c_int, [P, P, U32, U32, P]),
    "cw_couple_hold_obstacles": (C.c_int, [P, P, D]),
    "cw_couple_hold_medium_bath": (C.c_int, [P, P, D]),
    "cw_couple_hold_vessels_by": (C.c_int, [P, P, D, P]),
    "cw_couple_mean_per_cell": (C.c_int, [P, P, U32, U32, P]),
    "cw_network_compile": (C.c_int, [I32, P, P, I32, P, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                                     C.c_char_p, C.c_char_p, C.c_char_p, D, D, D, U32, P]),
    "cw_network_destroy": (C.c_int, [P]),
    "cw_network_info": (C.c_int, [P, P, P, P]),
    "cw_network_step_batch": (C.c_int, [P, I64, P, P, D, I32]),
    "cw_network_backward_batch": (C.c_int, [P, I64, P, P, D, I32, P, P, I32, P]),
    "cw_network_mechanics_batch": (C.c_int, [P, I64, P, P, P]),
    "cw_network_mutate": (C.c_int, [P, D, D, P, P]),
    "cw_lattice_bath": (C.c_int, [P, U32, P]),
    "cw_lattice_set_subsweeps": (C.c_int, [P, I32]),
    "cw_sim_measure": (C.c_int, [P, P]),
    "cw_network_rewire": (C.c_int, [P, P, P, P]),
    "cw_network_step_clones": (C.c_int, [I32, P, I64, P, P, P, D, I32]),
    "cw_sim_create": (C.c_int, [P, P, P]),
    "cw_sim_set_lesion": (C.c_int, [P, P, C.c_uint32, D, D, D]),
    "cw_sim_traced": (C.c_int, [P, C.c_uint32, C.c_uint32, P, P, P]),
    "cw_sim_destroy": (C.c_int, [P]),
    "cw_sim_step": (C.c_int, [P, U32]),
    "cw_sim_lattice": (C.c_int, [P, P]),
    "cw_sim_tuning": (C.c_int, [P, P, P, P, P, P]),
    "cw_sim_graph_info": (C.c_int, [P, P, P, P]),
    "cw_sim_field": (C.c_int, [P, I32, P]),
    "cw_sim_stats": (C.c_int, [P, P]),
    "cw_sim_network_state": (C.c_int, [P, U32, U32, P]),
    "cw_sim_cycle": (C.c_int, [P, U32, U32, P, P]),
    "cw_sim_touches_edge": (C.c_int, [P, P]),
    "cw_fit_create": (C.c_int, [P, P, P, P]),
    "cw_fit_destroy": (C.c_int, [P]),
    "cw_fit_nparams": (C.c_int, [P, P]),
    "cw_fit_get_params": (C.c_int, [P, P]),
    "cw_fit_set_params": (C.c_int, [P, P]),
    "cw_fit_set_target": (C.c_int, [P, P, P]),
    "cw_fit_forward": (C.c_int, [P, P, P, P]),
    "cw_fit_gradient": (C.c_int, [P, P, P]),
    "cw_event_record": (C.c_int, [I32]),
    "cw_profiler_start": (C.c_int, []),
    "cw_profiler_stop": (C.c_int, []),
    "cw_event_elapsed": (C.c_int, [I32, I32, P]),
}

_LIB = None


def lib():
    """The loaded library (raises ``CudaError`` when the shared object is missing)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise CudaError(f"{LIB_PATH} is not built: run cellweave_b200/build.py (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc: int) -> None:
    if rc != OK:
        msg = lib().cw_last_error().decode(errors="replace")
        raise _ERRORS.get(rc, CellweaveError)(msg)


def call(name: str, *args):
    check(getattr(lib(), name)(*args))


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
