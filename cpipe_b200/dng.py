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


def _main():
    """Times cpipe_cuda_dng_decode of a synthetic lossless-JPEG DNG: the 12 MP
    benchmark frame's 10-bit mosaic in 256x256 tiles.

        python -m cpipe_b200.dng --tables per_component --reps 5
    """
    import argparse
    import time

    import numpy as np

    from .chain import ChainConfig
    from .dng_synth import build_dng, lj92_tiles
    ap = argparse.ArgumentParser(description=_main.__doc__.split("\n")[0])
    ap.add_argument("--tables", choices=["per_component", "fixed"], default="per_component")
    ap.add_argument("--tile", type=int, default=256)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    L = _abi.lib()
    raw = ChainConfig.full_12mp().make_raw()
    h, w = raw.shape
    data = build_dng(width=w, height=h, bits=10, tile=(a.tile, a.tile),
                     segments=lj92_tiles(raw, 10, a.tile, a.tile, 2, a.tables))
    out = torch.empty((h, w), dtype=torch.int16, device="cuda")
    ms = []
    for _ in range(a.reps):
        t = time.perf_counter()
        st = L.cpipe_cuda_dng_decode(data, len(data), C.c_void_p(out.data_ptr()), out.numel() * 2, None)
        ms.append((time.perf_counter() - t) * 1e3)
        assert st == 0, L.cpipe_cuda_last_error().decode()
    fig = (C.c_uint64 * 9)()
    L.cpipe_cuda_lj92_last_stats(fig, 9)
    exact = bool(np.array_equal(out.cpu().numpy().view(np.uint16), raw))
    print(f"lossless-JPEG DNG {w}x{h} ({len(data)} bytes, tables {a.tables}): best {min(ms):.3f} ms "
          f"from host memory; exact {exact}; figures {list(fig)}")


if __name__ == "__main__":
    _main()
