"""Serving loop over libakb's akb_server_* entry points.

Solves are submitted with a mesh, a material, an initial state and a step
count; the server admits them by device-memory footprint, keeps them resident
and advances all of them together on one GPU (include/akb_capi.h).
"""
import ctypes

import numpy as np

from . import _capi
from .mesh import Mesh, TYPE_IDS


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_active", ctypes.c_int),
                ("device_bytes", ctypes.c_int64), ("chunk_steps", ctypes.c_int64),
                ("builders", ctypes.c_int), ("short_work", ctypes.c_double),
                ("no_batching", ctypes.c_int), ("batch_max_instances", ctypes.c_int),
                ("batch_max_request_elements", ctypes.c_int64),
                ("batch_max_elements", ctypes.c_int64)]


class Request(ctypes.Structure):
    _fields_ = [("element_type", ctypes.c_int), ("quadrature_rule", ctypes.c_int),
                ("precision", ctypes.c_int), ("nb_nodes", ctypes.c_int64),
                ("nb_elements", ctypes.c_int64), ("nodes", ctypes.c_void_p),
                ("connectivity", ctypes.c_void_p), ("material_type", ctypes.c_char_p),
                ("material_params", ctypes.c_char_p), ("displacement", ctypes.c_void_p),
                ("velocity", ctypes.c_void_p), ("blocked_dofs", ctypes.c_void_p),
                ("dt_factor", ctypes.c_double), ("nb_steps", ctypes.c_int64),
                ("displacement_out", ctypes.c_void_p), ("velocity_out", ctypes.c_void_p)]


class Completion(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int),
                ("message", ctypes.c_char * 256), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_start", ctypes.c_double),
                ("t_end", ctypes.c_double), ("nb_elements", ctypes.c_int64),
                ("nb_steps", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("dt", ctypes.c_double), ("batched", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("queued", ctypes.c_int64), ("building", ctypes.c_int64),
                ("running", ctypes.c_int64), ("finishing", ctypes.c_int64),
                ("completed_unpolled", ctypes.c_int64),
                ("device_bytes_reserved", ctypes.c_int64),
                ("device_bytes_budget", ctypes.c_int64), ("now", ctypes.c_double)]


_PRECISION = {"fp64": _capi.PRECISION_FP64, "mixed": _capi.PRECISION_MIXED,
              "fp64_fast": _capi.PRECISION_FP64_FAST}


def _params_text(params):
    def fmt(v):
        if isinstance(v, (bool, np.bool_)):
            return "true" if v else "false"
        return repr(float(v)) if isinstance(v, (int, float, np.floating)) else str(v)
    return "\n".join(f"{k} = {fmt(v)}" for k, v in params.items())


class Server:
    """Continuous-batching solve server on one GPU (small solves of the same
    kind share batch models whose instances stop and report one by one).

    ``submit`` returns an id and a dict whose "displacement" (and "velocity")
    arrays are filled when the solve completes; ``poll`` returns the
    completions (id, status, timings in seconds on the server's clock)."""

    def __init__(self, device=0, max_active=64, device_bytes=0, chunk_steps=500, builders=4,
                 short_work=1e8, batching=True, batch_max_instances=256,
                 batch_max_request_elements=1 << 17, batch_max_elements=1 << 23):
        cfg = ServerConfig(device, max_active, int(device_bytes), int(chunk_steps), builders,
                           float(short_work), 0 if batching else 1, int(batch_max_instances),
                           int(batch_max_request_elements), int(batch_max_elements))
        self._h = ctypes.c_void_p()
        _capi.check(_capi.lib().akb_server_create(ctypes.byref(cfg), ctypes.byref(self._h)))
        self._outputs = {}

    @staticmethod
    def estimate_bytes(mesh, material, precision="fp64", quadrature_rule=0):
        """Device bytes the server reserves for a solve of this mesh."""
        law = {"elastic": 0, "neohookean": 1, "plastic_linear_isotropic_hardening": 2}[
            material["type"]]
        b = ctypes.c_int64()
        _capi.check(_capi.lib().akb_estimate_device_bytes(
            TYPE_IDS[mesh.element_type], quadrature_rule, mesh.getNbNodes(),
            mesh.getNbElement(), law, _PRECISION[precision], ctypes.byref(b)))
        return b.value

    def submit(self, mesh, material, steps, velocity=None, displacement=None, blocked=None,
               dt_factor=0.8, precision="fp64", want_velocity=False, quadrature_rule=0):
        if not isinstance(mesh, Mesh):
            raise TypeError("mesh must be an akantu2_b200.Mesh")
        shape = mesh.nodes.shape
        keep = {"nodes": mesh.nodes, "conn": mesh.connectivity}
        mat = dict(material)
        mtype = mat.pop("type")
        keep["params"] = _params_text(mat).encode()
        keep["type"] = mtype.encode()

        def arr(a, dtype):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dtype).reshape(shape)
            return a

        for name, a, dt in (("v", velocity, np.float64), ("u", displacement, np.float64),
                            ("b", blocked, np.uint8)):
            keep[name] = arr(a, dt)
        out = {"displacement": np.zeros(shape)}
        if want_velocity:
            out["velocity"] = np.zeros(shape)
        p = lambda a: a.ctypes.data if a is not None else None
        req = Request(TYPE_IDS[mesh.element_type], quadrature_rule, _PRECISION[precision],
                      mesh.getNbNodes(), mesh.getNbElement(), p(keep["nodes"]), p(keep["conn"]),
                      keep["type"], keep["params"], p(keep["u"]), p(keep["v"]), p(keep["b"]),
                      float(dt_factor), int(steps), p(out["displacement"]),
                      p(out.get("velocity")))
        rid = ctypes.c_int64()
        _capi.check(_capi.lib().akb_server_submit(self._h, ctypes.byref(req), ctypes.byref(rid)))
        self._outputs[rid.value] = out
        return rid.value, out

    def poll(self, wait=0.0, capacity=256):
        buf = (Completion * capacity)()
        n = ctypes.c_int()
        _capi.check(_capi.lib().akb_server_poll(self._h, buf, capacity, ctypes.byref(n),
                                                float(wait)))
        res = []
        for k in range(n.value):
            c = buf[k]
            res.append({"id": c.id, "status": c.status, "message": c.message.decode(),
                        "t_submit": c.t_submit, "t_admit": c.t_admit, "t_start": c.t_start,
                        "t_end": c.t_end, "nb_elements": c.nb_elements, "nb_steps": c.nb_steps,
                        "device_bytes": c.device_bytes, "dt": c.dt,
                        "batched": bool(c.batched),
                        "outputs": self._outputs.pop(c.id, None)})
        return res

    def stats(self):
        st = ServerStats()
        _capi.check(_capi.lib().akb_server_get_stats(self._h, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def drain(self, timeout=600.0):
        """Polls until every submitted solve has completed; returns them."""
        import time
        res, t0 = [], time.perf_counter()
        while self._outputs:
            res += self.poll(wait=0.05)
            if time.perf_counter() - t0 > timeout:
                raise TimeoutError("solves still running")
        return res

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().akb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
