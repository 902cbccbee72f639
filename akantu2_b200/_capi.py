"""ctypes declarations of libakb.so (include/akb_capi.h).

The shared library is the only compute path of this package: if it is missing
or cannot be loaded, every call raises.  There is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# AKB_BOUNDS_CHECK=1 in the environment loads the bounds-checking build
# (libakb_checked.so: every index of the step kernels checked on the device)
LIB_PATH = os.path.join(_HERE, "libakb_checked.so" if os.environ.get("AKB_BOUNDS_CHECK") == "1"
                        else "libakb.so")

AKB_OK = 0
ERRORS = {
    1: "AKB_EINVAL", 2: "AKB_ENOMEM", 3: "AKB_ECUDA", 4: "AKB_ENEGJAC", 5: "AKB_ENAN",
    6: "AKB_EPARSE", 7: "AKB_ESTATE", 8: "AKB_EUNSUPPORTED", 9: "AKB_EIO",
    10: "AKB_EMATERIAL",
}

TETRAHEDRON_4, HEXAHEDRON_8, TRIANGLE_6 = 0, 1, 2
EXPLICIT_LUMPED_MASS = 0
PRECISION_FP64, PRECISION_MIXED, PRECISION_FP64_FAST = 0, 1, 2
(DISPLACEMENT, VELOCITY, ACCELERATION, EXTERNAL_FORCE, INTERNAL_FORCE, MASS,
 BLOCKED_DOFS, CURRENT_POSITION, PREVIOUS_DISPLACEMENT, DISPLACEMENT_INCREMENT) = range(10)
(GRAD_U, STRESS, PIOLA_KIRCHHOFF_2, INELASTIC_STRAIN, ISO_HARDENING,
 PLASTIC_ENERGY, EIGEN_GRAD_U) = range(7)
# AKB_ASYNC_READS_IN_FLIGHT: asynchronous reads that can be waited on one by one
ASYNC_READS_IN_FLIGHT = 4


class AkbError(RuntimeError):
    """Error returned by libakb (status code and message)."""

    def __init__(self, code, message):
        self.code = code
        self.name = ERRORS.get(code, str(code))
        super().__init__(f"{self.name}: {message}")


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(make -C akantu2_b200/csrc, or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp, i64, c_int, c_dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double
    pp = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "akb_last_error": (ctypes.c_char_p, []),
        "akb_version": (c_int, []),
        "akb_device_count": (c_int, [ctypes.POINTER(c_int)]),
        "akb_set_device": (c_int, [c_int]),
        "akb_host_alloc": (c_int, [ctypes.c_size_t, pp]),
        "akb_host_free": (c_int, [vp]),
        "akb_mesh_read_msh": (c_int, [ctypes.c_char_p, c_int, c_int, pp]),
        "akb_mesh_sizes": (c_int, [vp, ctypes.POINTER(i64), ctypes.POINTER(i64),
                                   ctypes.POINTER(c_int)]),
        "akb_mesh_nb_groups": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_mesh_group": (c_int, [vp, c_int, ctypes.c_char_p, ctypes.c_size_t,
                                   ctypes.POINTER(c_int), ctypes.POINTER(i64), vp]),
        "akb_mesh_nb_element_names": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_mesh_element_names": (c_int, [vp, c_int, ctypes.c_char_p, ctypes.c_size_t, vp]),
        "akb_mesh_copy": (c_int, [vp, vp, vp, vp]),
        "akb_mesh_free": (None, [vp]),
        "akb_model_create": (c_int, [c_int, c_int, vp, i64, vp, i64, pp]),
        "akb_model_destroy": (c_int, [vp]),
        "akb_model_load_materials": (c_int, [vp, ctypes.c_char_p]),
        "akb_model_add_material": (c_int, [vp, ctypes.c_char_p, ctypes.c_char_p]),
        "akb_model_set_element_materials": (c_int, [vp, vp]),
        "akb_model_set_quadrature_rule": (c_int, [vp, c_int]),
        "akb_model_init_full": (c_int, [vp, c_int, c_int]),
        "akb_model_nb_materials": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_model_get_material_param": (c_int, [vp, c_int, ctypes.c_char_p,
                                                 ctypes.POINTER(c_dbl)]),
        "akb_model_get_material_name": (c_int, [vp, c_int, ctypes.c_char_p, ctypes.c_size_t]),
        "akb_model_get_fe_data": (c_int, [vp, c_int, vp, i64]),
        "akb_model_nb_quadrature_points": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_model_get_stable_time_step": (c_int, [vp, ctypes.POINTER(c_dbl)]),
        "akb_model_set_time_step": (c_int, [vp, c_dbl]),
        "akb_model_get_time_step": (c_int, [vp, ctypes.POINTER(c_dbl)]),
        "akb_model_set_nodal": (c_int, [vp, c_int, vp, i64]),
        "akb_model_get_nodal": (c_int, [vp, c_int, vp, i64]),
        "akb_model_nodal_device_pointer": (c_int, [vp, c_int, pp]),
        "akb_model_qp_field_size": (c_int, [vp, c_int, c_int, ctypes.POINTER(i64)]),
        "akb_model_get_qp_field": (c_int, [vp, c_int, c_int, vp, i64]),
        "akb_model_set_qp_field": (c_int, [vp, c_int, c_int, vp, i64]),
        "akb_model_solve_step": (c_int, [vp, i64]),
        "akb_model_set_graph_steps": (c_int, [vp, i64]),
        "akb_model_synchronize": (c_int, [vp]),
        "akb_model_time_steps": (c_int, [vp, i64, ctypes.POINTER(c_dbl)]),
        "akb_model_profile_steps": (c_int, [vp, i64, ctypes.POINTER(c_dbl),
                                            ctypes.POINTER(c_dbl)]),
        "akb_model_assemble_internal_forces": (c_int, [vp]),
        "akb_model_get_energy": (c_int, [vp, ctypes.c_char_p, ctypes.POINTER(c_dbl)]),
        "akb_model_get_status": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_stable_time_step_noalloc": (c_int, [c_int, vp, vp, i64, vp, i64, c_dbl, vp, vp]),
        "akb_model_prepare_graphs": (c_int, [vp]),
        "akb_model_autotune": (c_int, [vp, c_int]),
        "akb_model_set_stream_priority": (c_int, [vp, c_int]),
        "akb_model_set_nodal_async": (c_int, [vp, c_int, vp, i64]),
        "akb_model_get_nodal_async": (c_int, [vp, c_int, vp, i64, ctypes.POINTER(i64)]),
        "akb_model_wait_nodal_async": (c_int, [vp, i64]),
        "akb_model_set_node_shape": (c_int, [vp, c_int, c_int]),
        "akb_model_get_node_shape": (c_int, [vp, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
        "akb_model_set_dependent_launch": (c_int, [vp, c_int]),
        "akb_model_set_increment_tracking": (c_int, [vp, c_int]),
        "akb_model_set_affine_kernel": (c_int, [vp, c_int]),
        "akb_model_get_affine_kernel": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_model_get_dependent_launch": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_mesh_neumann_forces": (c_int, [c_int, vp, i64, vp, i64, vp, i64, vp, vp]),
        "akb_model_apply_neumann_stress": (c_int, [vp, vp, i64, vp]),
        "akb_partition_elements": (c_int, [c_int, vp, i64, vp, i64, c_int, vp]),
        "akb_subdomain_create": (c_int, [c_int, vp, i64, vp, i64, vp, c_int, c_int,
                                         ctypes.POINTER(vp)]),
        "akb_subdomain_sizes": (c_int, [vp, ctypes.POINTER(i64), ctypes.POINTER(i64),
                                        ctypes.POINTER(i64), ctypes.POINTER(c_int)]),
        "akb_subdomain_mesh": (c_int, [vp, vp, vp, vp, vp]),
        "akb_subdomain_neighbor": (c_int, [vp, c_int, ctypes.POINTER(c_int), ctypes.POINTER(i64),
                                           ctypes.POINTER(i64)]),
        "akb_subdomain_lists": (c_int, [vp, c_int, vp, vp]),
        "akb_subdomain_destroy": (None, [vp]),
        "akb_model_halo_pack": (c_int, [vp, vp, i64, vp]),
        "akb_model_halo_unpack": (c_int, [vp, vp, i64, vp]),
        "akb_model_set_persistent": (c_int, [vp, c_int]),
        "akb_model_persistent_active": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_model_set_prescribed_velocity_ramp": (c_int, [vp, vp, i64, c_dbl, i64]),
        "akb_model_get_launch_shape": (c_int, [vp, c_int, ctypes.POINTER(c_int),
                                               ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                               ctypes.POINTER(c_int)]),
        "akb_model_set_launch_shape": (c_int, [vp, c_int, c_int, c_int, c_int, c_int]),
        "akb_model_set_prefetch": (c_int, [vp, c_int, c_int]),
        "akb_model_get_prefetch": (c_int, [vp, c_int, ctypes.POINTER(c_int)]),
        "akb_model_set_recompute_geometry": (c_int, [vp, c_int, c_int]),
        "akb_model_get_recompute_geometry": (c_int, [vp, c_int, ctypes.POINTER(c_int)]),
        "akb_model_set_streamed_points": (c_int, [vp, c_int, c_int]),
        "akb_model_get_streamed_points": (c_int, [vp, c_int, ctypes.POINTER(c_int)]),
        "akb_model_stream": (c_int, [vp, pp]),
        "akb_model_device_bytes": (c_int, [vp, ctypes.POINTER(i64)]),
        "akb_estimate_device_bytes": (c_int, [c_int, c_int, i64, i64, c_int, c_int,
                                              ctypes.POINTER(i64)]),
        "akb_bounds_checked": (c_int, []),
        "akb_model_debug_write_index": (c_int, [vp, c_int, i64, ctypes.c_int32]),
        "akb_model_set_persistent_wait_test": (c_int, [vp, ctypes.c_uint, c_int, ctypes.c_uint]),
        "akb_exchange_create": (c_int, [vp, c_int, pp]),
        "akb_exchange_add_link": (c_int, [vp, c_int, c_int, vp, vp, i64]),
        "akb_exchange_set_graph_steps": (c_int, [vp, i64]),
        "akb_exchange_solve_step": (c_int, [vp, i64]),
        "akb_exchange_synchronize": (c_int, [vp]),
        "akb_exchange_destroy": (c_int, [vp]),
        "akb_estimate_batch_device_bytes": (c_int, [c_int, c_int, i64, i64, c_int, c_int,
                                                    c_int, ctypes.POINTER(i64)]),
        "akb_server_create": (c_int, [vp, pp]),
        "akb_server_submit": (c_int, [vp, vp, ctypes.POINTER(i64)]),
        "akb_server_poll": (c_int, [vp, vp, c_int, ctypes.POINTER(c_int), c_dbl]),
        "akb_server_get_stats": (c_int, [vp, vp]),
        "akb_server_destroy": (c_int, [vp]),
        "akb_batch_create": (c_int, [c_int, c_int, c_int, vp, vp, vp, vp, pp]),
        "akb_batch_nb_instances": (c_int, [vp, ctypes.POINTER(c_int)]),
        "akb_batch_instance_offsets": (c_int, [vp, vp, vp]),
        "akb_batch_set_instance_materials": (c_int, [vp, vp]),
        "akb_batch_set_instance_steps": (c_int, [vp, vp]),
        "akb_batch_instance_steps_left": (c_int, [vp, vp]),
        "akb_batch_copy_instance_nodal": (c_int, [vp, c_int, c_int, vp, i64]),
        "akb_batch_get_stable_time_steps": (c_int, [vp, vp]),
        "akb_batch_set_time_steps": (c_int, [vp, vp]),
        "akb_batch_get_time_steps": (c_int, [vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc):
    """Raise AkbError for a non-zero status."""
    if rc != AKB_OK:
        msg = lib().akb_last_error()
        raise AkbError(rc, msg.decode() if msg else "")
    return rc


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class PinnedArray:
    """numpy array over page-locked host memory from akb_host_alloc."""

    def __init__(self, shape, dtype=float):
        import numpy as np
        self.dtype = np.dtype(dtype)
        nbytes = int(np.prod(shape)) * self.dtype.itemsize
        self._p = ctypes.c_void_p()
        check(lib().akb_host_alloc(nbytes, ctypes.byref(self._p)))
        buf = (ctypes.c_char * max(nbytes, 1)).from_address(self._p.value)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=int(np.prod(shape))).reshape(shape)

    def __del__(self):
        if getattr(self, "_p", None) and self._p.value:
            lib().akb_host_free(self._p)
            self._p = None
