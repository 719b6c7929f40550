"""Pipeline documents (*.cpipe.json, schema v0.4) on the device-resident
runner (cpipe_b200_pipeline_* in include/cpipe_b200.h).

`Pipeline` mirrors the reference's cpipe::runtime::Pipeline
(src/cpipe/runtime/Pipeline.cpp): `Pipeline(host, document)` is
Pipeline::load with its checks and status codes, `run(buffer)` runs the
planned nodes on a device buffer (the reference binds a source plugin and
walks CpuBuffers; here the caller passes the source's buffer), and the output
buffer belongs to the pipeline until the next run.
"""
import ctypes as C
import json

from . import _abi as A
from .host import Buffer, CpipeError


class _PipelineBuffer(Buffer):
    """The pipeline's output buffer: a handle the pipeline owns."""

    def __init__(self, host, handle, fmt, width, height):  # noqa: D401 (no allocation)
        self.host = host
        self.fmt = fmt
        self.width, self.height = int(width), int(height)
        self._h = handle

    def close(self):
        self._h = None


class Pipeline:
    """host None: plan only (the load checks, node order and memory plan)."""

    def __init__(self, host, document, until=None):
        text = document if isinstance(document, (str, bytes)) else json.dumps(document)
        raw = text.encode() if isinstance(text, str) else text
        st = C.c_int32()
        self.host = host
        self._h = A.lib().cpipe_b200_pipeline_load(host._h if host is not None else None, raw, len(raw),
                                                   until.encode() if until else None, C.byref(st))
        if not self._h:
            raise CpipeError(st.value, A.lib().cpipe_b200_pipeline_last_error(None).decode())
        self._out = None

    def close(self):
        if self._h:
            A.lib().cpipe_b200_pipeline_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nodes(self):
        """(id, type) of the planned nodes in execution order."""
        L = A.lib()
        n = L.cpipe_b200_pipeline_node_count(self._h)
        return [(L.cpipe_b200_pipeline_node_id(self._h, i).decode(), L.cpipe_b200_pipeline_node_type(self._h, i).decode())
                for i in range(n)]

    def memory_plan(self, width, height):
        peak, slots = C.c_uint64(), C.c_uint32()
        st = A.lib().cpipe_b200_pipeline_memory_plan(self._h, int(width), int(height), C.byref(peak), C.byref(slots))
        if st:
            raise CpipeError(st, "memory_plan")
        return peak.value, slots.value

    def last_error(self):
        return A.lib().cpipe_b200_pipeline_last_error(self._h).decode()

    def run(self, buffer):
        """Run on a host Buffer; returns the last node's buffer (owned by the
        pipeline, valid until the next run)."""
        out = C.c_void_p()
        st = A.lib().cpipe_b200_pipeline_run(self._h, buffer._h, C.byref(out))
        if st:
            raise CpipeError(st, self.last_error())
        fmt = A.lib().cpipe_b200_buffer_format(out.value)
        return _PipelineBuffer(self.host, out.value, fmt, buffer.width, buffer.height)
