"""Python mirror of the reference host interface for the raw->linear path.

The reference drives a node as registry lookup -> main_entry(create) ->
main_entry(process) with cpipe_process_ctx -> main_entry(destroy) -> freeze the
metadata builder (reference tests/unit/test_golden_isp_nodes.cpp:233-269,
src/cpipe/runtime/Pipeline.cpp:704-787), and a filter as
HalideParamFilterEntry(inputs, n, outputs, n, blob, size)
(src/cpipe/runtime/HalideFilterRegistry.hpp:18-21).  This module exposes the
same two levels over libcpipe_b200.so:

* `Registry` / `Host` / `Buffer` / `run_node` -- node level, device-resident
  buffers, metadata as the reference BufferMetadata carries it;
* `call_filter` -- filter level, numpy host buffers staged through the GPU by
  the library (the drop-in for a CPU-filter caller), or device pointers.

Everything here calls into the CUDA library; nothing computes pixels in Python.
"""
import ctypes as C
import json

import numpy as np

from . import _abi as A


class CpipeError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {A.STATUS_NAMES.get(status, status)}")


# ------------------------------------------------------------------ registry
class NodeDesc:
    def __init__(self, desc):
        self._desc = desc
        self.node_id = desc.node_id.decode()
        self.version = desc.node_version.decode()
        self.abi = (desc.abi_major, desc.abi_minor)
        self.manifest = json.loads(desc.manifest_json.decode())


class Registry:
    """Node descriptors exported by the library (reference Registry.cpp:13-35)."""

    def __init__(self):
        self._nodes = {}

    def load_builtin_nodes(self):
        n = C.c_size_t()
        base = A.lib().cpipe_b200_node_descs(C.byref(n))
        for i in range(n.value):
            d = NodeDesc(base[i])
            if d.abi[0] == 0 and d.abi[1] <= 4:  # reference ABI filter, Registry.cpp:18-23
                self._nodes[d.node_id] = d
        return len(self._nodes)

    def find(self, node_id):
        return self._nodes.get(node_id)

    def ids(self):
        return sorted(self._nodes)


# ----------------------------------------------------------------- filters
_HALIDE_TYPES = {np.dtype(np.uint16): (1, 16), np.dtype(np.float32): (2, 32), np.dtype(np.float16): (2, 16),
                 np.dtype(np.uint8): (1, 8)}


class DeviceImage:
    """A device allocation described like a numpy array (shape, dtype), for
    calling filters in place.  `ptr` is a CUDA device pointer (int)."""

    def __init__(self, ptr, shape, dtype):
        self.ptr = int(ptr)
        self.shape = tuple(shape)
        self.dtype = np.dtype(dtype)


def _halide(arr, keep):
    dims = (A.HalideDim * 3)()
    hb = A.HalideBuffer()
    code, bits = _HALIDE_TYPES[np.dtype(arr.dtype)]
    hb.type = A.HalideType(code, bits, 1)
    shape = arr.shape
    h, w = shape[0], shape[1]
    if len(shape) == 3:
        c = shape[2]
        dims[0] = A.HalideDim(0, w, c, 0)
        dims[1] = A.HalideDim(0, h, w * c, 0)
        dims[2] = A.HalideDim(0, c, 1, 0)
        hb.dimensions = 3
    else:
        dims[0] = A.HalideDim(0, w, 1, 0)
        dims[1] = A.HalideDim(0, h, w, 0)
        hb.dimensions = 2
    hb.dim = C.cast(dims, C.POINTER(A.HalideDim))
    if isinstance(arr, DeviceImage):
        hb.device = arr.ptr
    else:
        assert arr.flags["C_CONTIGUOUS"]
        hb.host = arr.ctypes.data
    keep.append(dims)
    return hb


def call_filter(aot_id, inputs, outputs, blob=None):
    """Call the CUDA filter registered under the reference `aot_id`.

    inputs/outputs: numpy arrays (HxW Bayer or HxWx4 RGBA; uint16, float32,
    float16, uint8) or DeviceImage.  blob: bytes / ctypes struct / None.
    Returns the cpipe status code."""
    L = A.lib()
    f = L.cpipe_cuda_find_filter(aot_id.encode())
    if not f:
        raise KeyError(aot_id)
    keep = []
    ins = [_halide(a, keep) for a in inputs]
    outs = [_halide(a, keep) for a in outputs]
    if f.contents.takes_params:
        if blob is None:
            bptr, bsize = None, 0
        else:
            raw = bytes(blob)
            keep.append(C.create_string_buffer(raw, len(raw)))
            bptr, bsize = C.cast(keep[-1], C.c_void_p), len(raw)
        pin = (C.POINTER(A.HalideBuffer) * max(1, len(ins)))(*[C.pointer(b) for b in ins])
        pout = (C.POINTER(A.HalideBuffer) * max(1, len(outs)))(*[C.pointer(b) for b in outs])
        fn = A.PARAM_FILTER(f.contents.entry)
        return fn(pin, len(ins), pout, len(outs), bptr, bsize)
    fn = A.PLAIN_FILTER(f.contents.entry)
    return fn(C.pointer(ins[0]), C.pointer(outs[0]))


def call_entry(symbol, inputs, outputs, blob=None):
    """Call an exported HalideParamFilterEntry-shaped function of the library by
    its symbol name (for entry points outside the aot_id table), with the same
    buffer and blob conventions as call_filter."""
    fn = getattr(A.lib(), symbol)
    keep = []
    ins = [_halide(a, keep) for a in inputs]
    outs = [_halide(a, keep) for a in outputs]
    if blob is None:
        bptr, bsize = None, 0
    else:
        raw = bytes(blob)
        keep.append(C.create_string_buffer(raw, len(raw)))
        bptr, bsize = C.cast(keep[-1], C.c_void_p), len(raw)
    pin = (C.POINTER(A.HalideBuffer) * max(1, len(ins)))(*[C.pointer(b) for b in ins])
    pout = (C.POINTER(A.HalideBuffer) * max(1, len(outs)))(*[C.pointer(b) for b in outs])
    entry = A.PARAM_FILTER(C.cast(fn, C.c_void_p).value)
    return entry(pin, len(ins), pout, len(outs), bptr, bsize)


def last_error():
    return A.lib().cpipe_cuda_last_error().decode()


# ------------------------------------------------------------------ host
_FMT_INFO = {A.FMT_R16_UINT: (np.uint16, 1), A.FMT_R32_SFLOAT: (np.float32, 1),
             A.FMT_R16G16B16A16_SFLOAT: (np.float16, 4), A.FMT_R32G32B32A32_SFLOAT: (np.float32, 4),
             A.FMT_R8G8B8A8_UNORM: (np.uint8, 4), A.FMT_R16G16B16A16_UNORM: (np.uint16, 4)}


class Buffer:
    """Device-resident Image2D buffer with reference-style metadata."""

    def __init__(self, host, fmt, width, height):
        self.host = host
        self.fmt = fmt
        self.width, self.height = int(width), int(height)
        self._h = A.lib().cpipe_b200_buffer_create(host._h, fmt, self.width, self.height)
        if not self._h:
            raise CpipeError(A.OOM, "buffer_create " + host.last_error())

    def close(self):
        if self._h:
            A.lib().cpipe_b200_buffer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def dtype(self):
        return _FMT_INFO[self.fmt][0]

    @property
    def shape(self):
        ch = _FMT_INFO[self.fmt][1]
        return (self.height, self.width) if ch == 1 else (self.height, self.width, ch)

    @property
    def device_ptr(self):
        return A.lib().cpipe_b200_buffer_device_ptr(self._h)

    def upload(self, arr):
        arr = np.ascontiguousarray(arr, dtype=self.dtype)
        assert arr.shape == self.shape, (arr.shape, self.shape)
        st = A.lib().cpipe_b200_buffer_upload(self._h, arr.ctypes.data, arr.nbytes)
        if st:
            raise CpipeError(st, "upload")
        return self

    def download(self):
        out = np.empty(self.shape, dtype=self.dtype)
        st = A.lib().cpipe_b200_buffer_download(self._h, out.ctypes.data, out.nbytes)
        if st:
            raise CpipeError(st, "download")
        return out

    # -- metadata setters (BufferMetadata / CalibrationBlock / CaptureBlock fields)
    def set_metadata(self, cfa=None, cfa_repeat=(2, 2), black_level=None, white_level=None, color_matrix1=None,
                     color_matrix2=None, forward_matrix1=None, forward_matrix2=None, illuminants=None,
                     linearization_table=None, noise_profile=None, as_shot_neutral=None, cs_role=None,
                     applied_steps=(), blobs=None):
        L = A.lib()
        if cfa is not None:
            pat = (C.c_uint8 * 16)(*list(cfa)[:16])
            rep = (C.c_uint8 * 2)(*cfa_repeat)
            L.cpipe_b200_buffer_set_cfa(self._h, rep, pat)
        if black_level is not None or white_level is not None:
            bl = (C.c_float * 4)(*(black_level or (0, 0, 0, 0)))
            L.cpipe_b200_buffer_set_levels(self._h, bl, int(white_level or 0))
        for which, m in ((1, color_matrix1), (2, color_matrix2), (3, forward_matrix1), (4, forward_matrix2)):
            if m is not None:
                L.cpipe_b200_buffer_set_matrix(self._h, which, (C.c_float * 9)(*m))
        if illuminants is not None:
            L.cpipe_b200_buffer_set_illuminants(self._h, int(illuminants[0]), int(illuminants[1]))
        if linearization_table is not None:
            t = np.ascontiguousarray(linearization_table, dtype=np.uint16)
            L.cpipe_b200_buffer_set_linearization_table(self._h, t.ctypes.data, t.size)
        if noise_profile is not None:  # [(beta, lambda), ...]
            beta = np.ascontiguousarray([p[0] for p in noise_profile], dtype=np.float32)
            lam = np.ascontiguousarray([p[1] for p in noise_profile], dtype=np.float32)
            L.cpipe_b200_buffer_set_noise_profile(self._h, beta.ctypes.data, lam.ctypes.data, beta.size)
        if as_shot_neutral is not None:
            L.cpipe_b200_buffer_set_as_shot_neutral(self._h, (C.c_float * 3)(*as_shot_neutral))
        if cs_role is not None:
            L.cpipe_b200_buffer_set_cs_role(self._h, cs_role.encode())
        for s in applied_steps:
            L.cpipe_b200_buffer_add_applied_step(self._h, s.encode())
        for k, v in (blobs or {}).items():
            raw = bytes(v)
            L.cpipe_b200_buffer_set_blob(self._h, k.encode(), raw, len(raw))
        return self

    def has_step(self, step):
        return bool(A.lib().cpipe_b200_buffer_has_applied_step(self._h, step.encode()))

    @property
    def cs_role(self):
        return A.lib().cpipe_b200_buffer_cs_role(self._h).decode()

    def blob(self, key):
        p, n = C.c_void_p(), C.c_size_t()
        if A.lib().cpipe_b200_buffer_get_blob(self._h, key.encode(), C.byref(p), C.byref(n)):
            return None
        return C.string_at(p, n.value)

    def cfa(self):
        has = C.c_int()
        rep = (C.c_uint8 * 2)()
        pat = (C.c_uint8 * 16)()
        A.lib().cpipe_b200_buffer_get_cfa(self._h, C.byref(has), rep, pat)
        return bool(has.value), tuple(rep), tuple(pat)


class Params:
    def __init__(self, values=None):
        self._h = A.lib().cpipe_b200_params_create()
        for k, v in (values or {}).items():
            self.set(k, v)

    def set(self, key, value):
        L = A.lib()
        if isinstance(value, bool):
            L.cpipe_b200_params_set_bool(self._h, key.encode(), int(value))
        elif isinstance(value, (int, float)):
            L.cpipe_b200_params_set_double(self._h, key.encode(), float(value))
        else:
            L.cpipe_b200_params_set_string(self._h, key.encode(), str(value).encode())

    def __del__(self):
        try:
            A.lib().cpipe_b200_params_destroy(self._h)
        except Exception:
            pass


class Host:
    """Host runtime with the reference suites over device buffers (one CUDA stream)."""

    def __init__(self, memory_cap=0):
        self._h = A.lib().cpipe_b200_host_create()
        if not self._h:
            raise CpipeError(A.INTERNAL_ERROR, "host_create (no usable CUDA device?)")
        if memory_cap:
            A.lib().cpipe_b200_host_set_memory_cap(self._h, int(memory_cap))

    def close(self):
        if self._h:
            A.lib().cpipe_b200_host_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def buffer(self, fmt, width, height):
        return Buffer(self, fmt, width, height)

    def last_error(self):
        return A.lib().cpipe_b200_host_last_error(self._h).decode() if self._h else ""

    def run_node(self, node_id, inputs, outputs, params=None):
        """create -> process -> destroy; returns the cpipe status."""
        p = params if isinstance(params, Params) else Params(params or {})
        ins = (C.c_void_p * max(1, len(inputs)))(*[b._h for b in inputs])
        outs = (C.c_void_p * max(1, len(outputs)))(*[b._h for b in outputs])
        return A.lib().cpipe_b200_run_node(self._h, node_id.encode(), p._h, ins, len(inputs), outs, len(outputs))


def process_single_input_node(host, node_id, input_buffer, output_fmt, params=None):
    """The reference golden-test harness shape (test_golden_isp_nodes.cpp:233-269):
    allocate the output with the manifest's format, run the node, return
    (status, output buffer)."""
    out = host.buffer(output_fmt, input_buffer.width, input_buffer.height)
    st = host.run_node(node_id, [input_buffer], [out], params)
    return st, out
