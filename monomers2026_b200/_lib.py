"""ctypes binding of libselm_b200.so (the C ABI declared in include/selm_b200.h).

The library is built in-tree (``monomers2026_b200/lib/``).  There is no
fallback: if the shared object is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libselm_b200.so")

# symbols declared in include/selm_b200.h (checked by the CPU test suite)
EXPORTED = [
    "selm_create", "selm_create_from_files", "selm_set_particles", "selm_set_topology",
    "selm_set_force_callback", "selm_initial", "selm_step", "selm_destroy", "selm_get_particles",
    "selm_get_field", "selm_set_field", "selm_get_info", "selm_status", "selm_set_stream",
    "selm_get_stream", "selm_synchronize", "selm_profile_enable", "selm_profile_read",
    "selm_op_interp", "selm_op_spread", "selm_op_spread_noalloc", "selm_op_fft3_r2c", "selm_op_fft3_c2r", "selm_kernel_launches",
    "selm_last_error", "selm_version",
    "selm_batch_create", "selm_batch_add", "selm_batch_remove", "selm_batch_step", "selm_batch_size",
    "selm_batch_get_stream", "selm_batch_synchronize", "selm_batch_destroy", "selm_device_bytes",
    "selm_batch_add_job", "selm_batch_poll", "selm_batch_retire",
    "selm_tune_set", "selm_tune_get", "selm_tune_default",
    "selm_dcd_open", "selm_dcd_open_sim", "selm_dcd_write", "selm_dcd_write_sim", "selm_dcd_close", "selm_case_dump",
    "selm_analysis_create", "selm_analysis_sample", "selm_analysis_msd", "selm_analysis_structure",
    "selm_analysis_kinetic", "selm_analysis_reset", "selm_analysis_device_bytes", "selm_analysis_destroy",
    "selm_get_coupling_impulse", "selm_host_register", "selm_host_unregister",
    "selm_slab_create", "selm_slab_layout", "selm_slab_buffers", "selm_slab_gather", "selm_slab_advance",
    "selm_slab_solve", "selm_slab_finish", "selm_slab_velocity",
]

SELM_OK = 0


class SelmParams(C.Structure):
    _fields_ = [
        ("num_mesh_pts", C.c_int * 3),
        ("box_lo", C.c_double), ("box_hi", C.c_double),
        ("rho", C.c_double), ("mu", C.c_double), ("KB", C.c_double), ("T", C.c_double), ("dt", C.c_double),
        ("flag_stochastic", C.c_int),
        ("seed", C.c_ulonglong),
        ("form", C.c_int), ("integrator", C.c_int), ("noise_mode", C.c_int),
    ]


class SelmTopology(C.Structure):
    _fields_ = [
        ("natoms", C.c_int), ("ntypes", C.c_int), ("type", C.c_void_p),
        ("nbonds", C.c_int), ("bond_style", C.c_int), ("nbondtypes", C.c_int),
        ("bonds", C.c_void_p), ("bond_coeff", C.c_void_p),
        ("nangles", C.c_int), ("angle_style", C.c_int), ("nangletypes", C.c_int),
        ("angles", C.c_void_p), ("angle_coeff", C.c_void_p),
        ("pair_style", C.c_int), ("pair_coeff", C.c_void_p),
        ("special_lj", C.c_double * 3), ("body_force", C.c_double * 3),
    ]


FORCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                       C.POINTER(C.c_double))

_lib = None


def load():
    """Load libselm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libselm_b200.so not built ({LIB_PATH}); run monomers2026_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    L.selm_create.argtypes = [C.POINTER(SelmParams), C.POINTER(vp)]
    L.selm_create_from_files.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.selm_set_particles.argtypes = [vp, C.c_int, dp, dp, dp]
    L.selm_set_topology.argtypes = [vp, C.POINTER(SelmTopology)]
    L.selm_set_force_callback.argtypes = [vp, FORCE_FN, vp]
    L.selm_initial.argtypes = [vp]
    L.selm_step.argtypes = [vp, C.c_int]
    L.selm_destroy.argtypes = [vp]
    L.selm_get_particles.argtypes = [vp, dp, dp, dp]
    L.selm_get_field.argtypes = [vp, C.c_int, dp]
    L.selm_set_field.argtypes = [vp, C.c_int, dp]
    L.selm_get_info.argtypes = [vp, ip, ip, C.POINTER(C.c_ulonglong)]
    L.selm_status.argtypes = [vp, C.POINTER(C.c_uint)]
    L.selm_set_stream.argtypes = [vp, vp]
    L.selm_get_stream.argtypes = [vp]
    L.selm_get_stream.restype = vp
    L.selm_synchronize.argtypes = [vp]
    L.selm_profile_enable.argtypes = [vp, C.c_int]
    L.selm_profile_read.argtypes = [vp, C.c_char_p, dp, C.POINTER(C.c_long)]
    L.selm_op_interp.argtypes = [C.c_int, ip, C.c_double, C.c_double, dp, C.c_int, dp, dp]
    L.selm_op_spread.argtypes = [C.c_int, ip, C.c_double, C.c_double, dp, C.c_int, dp, dp]
    L.selm_op_spread_noalloc.argtypes = [C.c_int, ip, C.c_double, C.c_double, vp, C.c_int, vp, vp, vp]
    L.selm_op_fft3_r2c.argtypes = [C.c_int, ip, dp, dp]
    L.selm_op_fft3_c2r.argtypes = [C.c_int, ip, dp, dp]
    L.selm_kernel_launches.argtypes = []
    L.selm_kernel_launches.restype = C.c_ulonglong
    L.selm_batch_create.argtypes = [vp, C.POINTER(vp)]
    L.selm_batch_add.argtypes = [vp, vp]
    L.selm_batch_remove.argtypes = [vp, vp]
    L.selm_batch_step.argtypes = [vp, C.c_int]
    L.selm_batch_size.argtypes = [vp]
    L.selm_batch_get_stream.argtypes = [vp]
    L.selm_batch_get_stream.restype = vp
    L.selm_batch_synchronize.argtypes = [vp]
    L.selm_batch_destroy.argtypes = [vp]
    L.selm_batch_add_job.argtypes = [vp, vp, C.c_longlong]
    L.selm_batch_poll.argtypes = [vp, C.POINTER(vp), C.c_int, C.POINTER(C.c_int)]
    L.selm_batch_retire.argtypes = [vp, vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.selm_slab_create.argtypes = [C.POINTER(SelmParams), C.c_int, C.c_int, C.POINTER(vp)]
    L.selm_slab_layout.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                   C.POINTER(C.c_longlong)]
    L.selm_slab_buffers.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(C.c_longlong)]
    for name in ("selm_slab_gather", "selm_slab_advance", "selm_slab_solve", "selm_slab_finish"):
        getattr(L, name).argtypes = [vp]
    L.selm_slab_velocity.argtypes = [vp, C.POINTER(C.c_double)]
    L.selm_device_bytes.argtypes = [vp, C.POINTER(C.c_ulonglong)]
    L.selm_host_register.argtypes = [vp, C.c_ulonglong]
    L.selm_host_unregister.argtypes = [vp]
    L.selm_tune_set.argtypes = [vp, C.c_int, C.c_int]
    L.selm_tune_get.argtypes = [vp, C.c_int, ip]
    L.selm_tune_default.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    L.selm_dcd_open.argtypes = [C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_int, dp, C.POINTER(vp)]
    L.selm_dcd_open_sim.argtypes = [C.c_char_p, vp, C.c_int, C.POINTER(vp)]
    L.selm_dcd_write.argtypes = [vp, dp]
    L.selm_dcd_write_sim.argtypes = [vp, vp]
    L.selm_dcd_close.argtypes = [vp]
    L.selm_get_coupling_impulse.argtypes = [vp, dp, dp]
    L.selm_case_dump.argtypes = [vp, ip, C.c_char_p, C.c_int]
    llp = C.POINTER(C.c_longlong)
    L.selm_analysis_create.argtypes = [vp, C.c_int, C.c_int, C.c_int, ip, C.POINTER(vp)]
    L.selm_analysis_sample.argtypes = [vp]
    L.selm_analysis_msd.argtypes = [vp, dp, llp]
    L.selm_analysis_structure.argtypes = [vp, dp, dp, llp]
    L.selm_analysis_kinetic.argtypes = [vp, dp, dp, llp]
    L.selm_analysis_reset.argtypes = [vp]
    L.selm_analysis_device_bytes.argtypes = [vp, C.POINTER(C.c_ulonglong)]
    L.selm_analysis_destroy.argtypes = [vp]
    L.selm_last_error.restype = C.c_char_p
    L.selm_version.restype = C.c_char_p
    _lib = L
    return L


class SelmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"selm error {code}: {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != SELM_OK:
        raise SelmError(rc, load().selm_last_error().decode(errors="replace"))
