"""ctypes prototypes for the C ABI declared in include/espp_b200.h.

``bind(lib)`` attaches argument and result types to a loaded ``ctypes.CDLL`` that
exports the ABI.  ``call(lib, name, *args)`` runs one entry point and raises
``RuntimeError`` with the library's error text on a non-zero status, the way the
reference's Boost.Python layer turns ``std::runtime_error`` into a Python exception.
"""
import ctypes
from ctypes import (POINTER, c_char_p, c_double, c_int32, c_int64, c_size_t, c_uint8,
                    c_uint64, c_void_p)

_P = c_void_p
_D = POINTER(c_double)
_I64 = POINTER(c_int64)
_I32 = POINTER(c_int32)
_U8 = POINTER(c_uint8)

PROTOTYPES = {
    "espp_abi_version": (c_int32, []),
    "espp_last_error": (c_size_t, [c_char_p, c_size_t]),
    "espp_system_create": (c_int32, [_D, c_double, _I32, c_int32, c_uint64, POINTER(c_void_p)]),
    "espp_system_destroy": (c_int32, [_P]),
    "espp_set_skin": (c_int32, [_P, c_double]),
    "espp_add_particles": (c_int32, [_P, c_int64, _I64, _I32, _D, _D, _D]),
    "espp_decompose": (c_int32, [_P]),
    "espp_num_particles": (c_int32, [_P, _I64]),
    "espp_get_particles": (c_int32, [_P, c_int64, _I64, _D, _D, _D, _I32]),
    "espp_set_particles": (c_int32, [_P, c_int64, _I64, _D, _D]),
    "espp_set_images": (c_int32, [_P, c_int64, _I64, _I32]),
    "espp_vl_create": (c_int32, [_P, c_double, c_int64, _I64]),
    "espp_vl_rebuild": (c_int32, [_P]),
    "espp_vl_size": (c_int32, [_P, _I64]),
    "espp_vl_pairs": (c_int32, [_P, c_int64, _I64, _I64]),
    "espp_vl_builds": (c_int32, [_P, _I64]),
    "espp_vl_digest": (c_int32, [_P, POINTER(c_uint64)]),
    "espp_lj_set": (c_int32, [_P, c_int32, c_int32, c_double, c_double, c_double, c_double,
                              c_double]),
    "espp_bonds_add": (c_int32, [_P, c_int64, _I64]),
    "espp_bonds_size": (c_int32, [_P, _I64]),
    "espp_bonds_clear": (c_int32, [_P]),
    "espp_fene_set": (c_int32, [_P, c_double, c_double, c_double, c_double, c_double]),
    "espp_bonds_max_sqr": (c_int32, [_P, _D]),
    "espp_bonds_reset_max": (c_int32, [_P]),
    "espp_triples_add": (c_int32, [_P, c_int64, _I64]),
    "espp_triples_size": (c_int32, [_P, _I64]),
    "espp_triples_clear": (c_int32, [_P]),
    "espp_cosine_set": (c_int32, [_P, c_double, c_double]),
    "espp_tab_read": (c_int32, [c_char_p, c_int64, _D, _D, _D, _I64]),
    "espp_tab_eval": (c_int32, [c_int32, c_int64, _D, _D, _D, c_int64, _D, _D, _D]),
    "espp_tab_pair_set": (c_int32, [_P, c_int32, c_int32, c_int32, c_int64, _D, _D, _D,
                                    c_double, c_double]),
    "espp_tab_bond_set": (c_int32, [_P, c_int32, c_int64, _D, _D, _D, c_double, c_double]),
    "espp_tab_angle_set": (c_int32, [_P, c_int32, c_int64, _D, _D, _D]),
    "espp_integrator_set": (c_int32, [_P, c_double]),
    "espp_step_get": (c_int32, [_P, _I64]),
    "espp_step_set": (c_int32, [_P, c_int64]),
    "espp_langevin_set": (c_int32, [_P, c_int32, c_double, c_double, c_int64, _I64]),
    "espp_capforce_set": (c_int32, [_P, c_int32, _D]),
    "espp_run": (c_int32, [_P, c_int64]),
    "espp_num_resorts": (c_int32, [_P, _I64]),
    "espp_dd_load": (c_int32, [_P, c_int64, _I64, _I32, _D, _D, _D, _I32, _U8]),
    "espp_dd_set_halo_positions": (c_int32, [_P, c_int64, _I64, _D]),
    "espp_dd_run_begin": (c_int32, [_P, c_int64, _D]),
    "espp_memory_space": (c_int32, [_I32]),
    "espp_dd_read_positions": (c_int32, [_P, c_int64, _I64, _D]),
    "espp_dd_write_halo": (c_int32, [_P, c_int64, _I64, _D]),
    "espp_dd_step": (c_int32, [_P, c_int32, _D]),
    "espp_dd_run_end": (c_int32, [_P]),
    "espp_timers": (c_int32, [_P, _D]),
    "espp_energy": (c_int32, [_P, c_int32, _D]),
    "espp_virial": (c_int32, [_P, c_int32, _D]),
    "espp_virial_tensor": (c_int32, [_P, c_int32, _D]),
    "espp_kinetic": (c_int32, [_P, _D, _I64]),
    "espp_kinetic_tensor": (c_int32, [_P, _D]),
    "espp_kinetic_types": (c_int32, [_P, c_uint64, _D, _I64]),
    "espp_rdf": (c_int32, [_P, c_int32, _D]),
    "espp_confs_create": (c_int32, [_P, c_int32, c_int64, _I64, POINTER(c_void_p)]),
    "espp_confs_destroy": (c_int32, [_P]),
    "espp_confs_gather": (c_int32, [_P]),
    "espp_confs_push": (c_int32, [_P, _D]),
    "espp_confs_size": (c_int32, [_P, _I32]),
    "espp_confs_clear": (c_int32, [_P]),
    "espp_confs_get": (c_int32, [_P, c_int32, _D]),
    "espp_msd": (c_int32, [_P, _D]),
    "espp_msd_chain_com": (c_int32, [_P, c_int32, _D]),
    "espp_force_acc": (c_int32, [_P, c_int32, c_int64, _I64, _D]),
    "espp_mlp_create": (c_int32, [c_double, c_double, POINTER(c_void_p)]),
    "espp_mlp_destroy": (c_int32, [_P]),
    "espp_mlp_set_mode": (c_int32, [_P, c_int32]),
    "espp_mlp_num_params": (c_int32, [_I64]),
    "espp_mlp_set_params": (c_int32, [_P, c_int64, _D]),
    "espp_mlp_get_params": (c_int32, [_P, c_int64, _D]),
    "espp_mlp_set_norm": (c_int32, [_P, _D, _D]),
    "espp_mlp_attach": (c_int32, [_P, _P]),
    "espp_mlp_descriptors": (c_int32, [_P, c_int64, _I64, _D]),
    "espp_mlp_fm_grad": (c_int32, [_P, c_int64, _I64, _D, _D, _D]),
    "espp_mlp_adam_step": (c_int32, [_P, c_double, c_double, c_double, c_double, c_double]),
    "espp_energy_noalloc": (c_int32, [_P, c_int32, _D]),
    "espp_set_profiling": (c_int32, [_P, c_int32]),
    "espp_profile": (c_int32, [_P, _D, _I64]),
    "espp_last_run_ms": (c_int32, [_P, _D]),
    "espp_select_device": (c_int32, [c_int32]),
    "espp_set_tpp": (c_int32, [_P, c_int32]),
    "espp_fp32_peak": (c_int32, [_D]),
    "espp_selftest_bounded_wait": (c_int32, [_P, c_int64, _D]),
    "espp_batch_create": (c_int32, [POINTER(c_void_p), c_int32, POINTER(c_void_p)]),
    "espp_batch_destroy": (c_int32, [_P]),
    "espp_batch_run": (c_int32, [_P, c_int64]),
    "espp_batch_last_run_ms": (c_int32, [_P, _D]),
    "espp_autotune": (c_int32, [_P, _I32, _D]),
    "espp_set_layout": (c_int32, [_P, c_int32, c_int32, _I32]),
    "espp_set_half_cell_int": (c_int32, [_P, c_int32]),
    "espp_get_layout": (c_int32, [_P, _I32]),
    "espp_autotune_layout": (c_int32, [_P, c_double, _I32, _D, c_int32, _I32]),
}

# status codes (include/espp_b200.h)
ESPP_OK = 0
PREC_FP64 = 0
PREC_MIXED = 1
IA_LJ = 0
IA_FENE = 1
IA_TAB_PAIR = 2
IA_TAB_BOND = 3
IA_MLP = 4
IA_COSINE = 5
IA_TAB_ANGLE = 6
TAB_LINEAR, TAB_AKIMA, TAB_CUBIC = 1, 2, 3
CAP_OFF, CAP_ABS, CAP_COMPONENT = 0, 1, 2
CONF_POSITION, CONF_VELOCITY, CONF_UNFOLDED = 0, 1, 2


def bind(lib, extra=None):
    protos = dict(PROTOTYPES)
    if extra:
        protos.update(extra)
    for name, (res, args) in protos.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def last_error(lib):
    n = lib.espp_last_error(None, 0)
    buf = ctypes.create_string_buffer(int(n) + 1)
    lib.espp_last_error(buf, n + 1)
    return buf.value.decode(errors="replace")


def call(lib, name, *args):
    rc = getattr(lib, name)(*args)
    if rc != ESPP_OK:
        raise RuntimeError("%s failed (status %d): %s" % (name, rc, last_error(lib)))
    return rc


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array (or None)."""
    return None if a is None else a.ctypes.data_as(_D)


def u8ptr(a):
    return None if a is None else a.ctypes.data_as(_U8)


def i64ptr(a):
    return None if a is None else a.ctypes.data_as(_I64)


def i32ptr(a):
    return None if a is None else a.ctypes.data_as(_I32)
