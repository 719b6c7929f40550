"""DNG ingest over the C ABI: the host-side mirror of cpipe::ingest::dng::DngReader
(src/cpipe/ingest/dng/DngReader.cpp:190-232) and of the metadata that
OpcodeListParser::parse extracts (src/cpipe/ingest/dng_opcode/OpcodeListParser.cpp:330-515).

    result = DngReader.read("frame.dng")     # or bytes of a DNG
    result.status, result.buffer (torch uint16 (h, w) on the current CUDA device),
    result.metadata (dict), result.message

The parse runs on the host; the strip unpack runs on the GPU.  There is no CPU
decode path: without the library or a GPU the read fails.
"""
import ctypes as C
from dataclasses import dataclass, field

import torch

from . import _abi


def _blob(data, off, n):
    return bytes(data[off:off + n]) if n else b""


def info_to_metadata(info, data):
    """ParsedDngMetadata-shaped dict from a cpipe_DngInfo and the file bytes."""
    rep = list(info.cfa_repeat)
    lin = b""
    if info.linearization_count:
        lin = _blob(data, info.linearization_offset, 2 * info.linearization_count)
    names = ("color_matrix1", "color_matrix2", "forward_matrix1", "forward_matrix2")
    return {
        "width": info.width, "height": info.height, "bits_per_sample": info.bits_per_sample,
        "compression": info.compression, "strip_offset": info.strip_offset,
        "strip_byte_count": info.strip_byte_count, "make": info.make.decode("latin-1"),
        "model": info.model.decode("latin-1"),
        "cs_role": "raw_camera",
        "calibration": {
            "cfa": {"repeat": rep, "pattern": list(info.cfa_pattern)[:rep[0] * rep[1]]},
            "black_level": list(info.black_level), "white_level": info.white_level,
            "linearization_table": list(memoryview(lin).cast("H")) if lin else None,
            "calibration_illuminant1": info.calibration_illuminant[0],
            "calibration_illuminant2": info.calibration_illuminant[1],
            **{n: (list(info.matrix[m]) if info.has_matrix[m] else None) for m, n in enumerate(names)},
        },
        "capture": {
            "camera_id": info.make.decode("latin-1"), "physical_camera_id": info.model.decode("latin-1"),
            "iso": info.iso, "exposure_time_ns": info.exposure_time_ns, "lens_aperture": info.lens_aperture,
            "lens_focal_length_mm": info.lens_focal_length_mm, "orientation": info.orientation,
            "as_shot_neutral": list(info.as_shot_neutral),
        },
        "active_area": (dict(zip(("x", "y", "width", "height"), info.active_area))
                        if info.has_active_area else None),
        "exif_blob": _blob(data, info.exif_offset, info.exif_bytes),
        "xmp_blob": _blob(data, info.xmp_offset, info.xmp_bytes),
        "icc_blob": _blob(data, info.icc_offset, info.icc_bytes),
        "ext_blobs": {f"com.cpipe.dng.opcode_list_{i + 1}_bytes": _blob(data, info.opcode_list_offset[i],
                                                                       info.opcode_list_bytes[i])
                      for i in range(3) if info.opcode_list_bytes[i]},
    }


def parse(data):
    """(status, cpipe_DngInfo) from DNG bytes; host only."""
    data = bytes(data)
    info = _abi.DngInfo()
    st = _abi.lib().cpipe_dng_parse(data, len(data), C.byref(info))
    return st, info


@dataclass
class DngReadResult:
    status: int
    buffer: torch.Tensor = None
    metadata: dict = field(default_factory=dict)
    message: str = ""


class DngReader:
    @staticmethod
    def read(source, device=None):
        """Decode a DNG file (path or bytes) into an R16 plane on the GPU."""
        if isinstance(source, (bytes, bytearray, memoryview)):
            data = bytes(source)
        else:
            try:
                with open(source, "rb") as f:
                    data = f.read()
            except OSError as e:
                return DngReadResult(_abi.FAILED, message=f"failed to open DNG: {e}")
        L = _abi.lib()
        st, info = parse(data)
        if st != _abi.OK:
            msg = L.cpipe_cuda_last_error().decode()
            return DngReadResult(_abi.FAILED if st == _abi.UNSUPPORTED else st, message=msg)
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        out = torch.empty((info.height, info.width), dtype=torch.uint16, device=dev)
        with torch.cuda.device(dev):
            L.cpipe_cuda_set_stream(C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
            st = L.cpipe_cuda_dng_decode(data, len(data), C.c_void_p(out.data_ptr()), out.numel() * 2,
                                         C.byref(info))
        if st != _abi.OK:
            return DngReadResult(st, message=L.cpipe_cuda_last_error().decode())
        return DngReadResult(_abi.OK, out, info_to_metadata(info, data))
