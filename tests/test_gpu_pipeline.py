"""The device-resident pipeline runner (cpipe_b200_pipeline_*) on the GPU.

A document in the fused chain's node order returns, bit for bit, what the
fused chain returns (which equals the nodes run one by one); the classic
raw->display document's device prefix equals its nodes run one by one through
the host; slots stay allocated between runs of one extent; a memory cap below
the plan's peak is CPIPE_OOM."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest
from cpipe_b200 import _abi as A
from cpipe_b200 import blobs as BL
from cpipe_b200.chain import CAMERA_TO_XYZ, COLOR_MATRIX1, COLOR_MATRIX2, Chain, ChainConfig
from cpipe_b200.host import CpipeError, Host
from cpipe_b200.pipeline import Pipeline
from pipeline_docs import classic, fused_chain_order

pytestmark = pytest.mark.gpu


def raw_input(host, cfg, raw, lin_table=False):
    b = cfg.blobs()
    buf = host.buffer(A.FMT_R16_UINT, cfg.width, cfg.height).upload(raw)
    blob_meta = {}
    if "opcode_list_2" in b:
        blob_meta["com.cpipe.dng.opcode_list_2_bytes"] = b["opcode_list_2"]
    if "opcode_list_3" in b:
        blob_meta["com.cpipe.dng.opcode_list_3_bytes"] = b["opcode_list_3"]
    meta = dict(cfa=cfg.cfa, black_level=[cfg.black] * 4, white_level=cfg.white, cs_role="raw_camera",
                illuminants=(17, 21), as_shot_neutral=list(cfg.neutral), noise_profile=[(cfg.noise_b, cfg.noise_a)],
                color_matrix1=COLOR_MATRIX1, color_matrix2=COLOR_MATRIX2, forward_matrix1=CAMERA_TO_XYZ,
                forward_matrix2=CAMERA_TO_XYZ, blobs=blob_meta)
    if lin_table:
        meta["linearization_table"] = np.arange(1 << cfg.bits, dtype=np.uint16)
    buf.set_metadata(**meta)
    return buf, b


@pytest.fixture
def cube(tmp_path):
    def make(values):
        path = str(tmp_path / "look.cube")
        BL.write_cube(path, 33, values)
        return path
    return make


@pytest.mark.parametrize("w,h", [(160, 120), (97, 63), (4032, 3024)])
def test_runner_equals_fused_chain(host, cube, w, h):
    cfg = ChainConfig.small(w, h) if w < 4032 else ChainConfig.full_12mp()
    raw = cfg.make_raw()
    buf, b = raw_input(host, cfg, raw)
    p = Pipeline(host, fused_chain_order(cube(b["lut_values"]), cfg.guided_radius, cfg.guided_eps))
    got = p.run(buf).download()
    chain = Chain(cfg)
    want = chain.run_host(raw)
    chain.close()
    np.testing.assert_array_equal(got.view(np.uint16), want.view(np.uint16))
    p.close()
    buf.close()


def test_runner_classic_prefix_equals_nodes(host, cube):
    """qbc (a Bayer frame passes through) -> linearize -> GainMap -> black level
    -> RCD -> OpcodeList3 -> WB -> colormatrix -> BM3D -> wavelet -> filmic ->
    LUT -> sharpen -> sRGB display, against the same nodes one by one."""
    cfg = ChainConfig.small(128, 96)
    raw = cfg.make_raw()
    buf, b = raw_input(host, cfg, raw, lin_table=True)
    lut = cube(b["lut_values"])
    doc = classic(lut)
    p = Pipeline(host, doc, until="display")
    got = p.run(buf).download()
    cur = buf
    keep = []
    for node in doc["nodes"][:-1]:
        t = node["type"]
        fmt = {"com.cpipe.demosaic.quad_bayer_remosaic": A.FMT_R16_UINT,
               "com.cpipe.color.scene_linear_to_display": A.FMT_R8G8B8A8_UNORM}.get(t)
        if fmt is None:
            fmt = A.FMT_R32_SFLOAT if t in ("com.cpipe.linearize.dng_lut", "com.cpipe.lens.shading_gainmap",
                                            "com.cpipe.blacklevel.dng_levels") else A.FMT_R16G16B16A16_SFLOAT
        nxt = host.buffer(fmt, cfg.width, cfg.height)
        keep.append(nxt)
        st = host.run_node(t, [cur], [nxt], node["params"])
        assert st == 0, (t, host.last_error())
        cur = nxt
    np.testing.assert_array_equal(got, cur.download())
    p.close()


def test_runner_keeps_slots_between_runs(host, cube):
    cfg = ChainConfig.small(256, 192)
    raw = cfg.make_raw()
    buf, b = raw_input(host, cfg, raw)
    p = Pipeline(host, fused_chain_order(cube(b["lut_values"]), cfg.guided_radius, cfg.guided_eps))
    first = p.run(buf).download()
    L = A.lib()
    free0 = C.c_uint64()
    assert L.cpipe_cuda_memory_stats(None, None, C.byref(free0), None) == 0
    for _ in range(3):
        again = p.run(buf).download()
        np.testing.assert_array_equal(again.view(np.uint16), first.view(np.uint16))
    free1 = C.c_uint64()
    assert L.cpipe_cuda_memory_stats(None, None, C.byref(free1), None) == 0
    assert free1.value == free0.value  # no allocation once the slots exist
    peak, slots = p.memory_plan(256, 192)
    assert slots == 2 and peak == 256 * 192 * 2 + 2 * 256 * 192 * 8
    # another extent re-plans
    cfg2 = ChainConfig.small(130, 70)
    raw2 = cfg2.make_raw()
    buf2, b2 = raw_input(host, cfg2, raw2)
    p2 = Pipeline(host, fused_chain_order(cube(b2["lut_values"]), cfg2.guided_radius, cfg2.guided_eps))
    small = p2.run(buf2).download()
    chain = Chain(cfg2)
    np.testing.assert_array_equal(small.view(np.uint16), chain.run_host(raw2).view(np.uint16))
    chain.close()
    for x in (p, p2, buf, buf2):
        x.close()


def test_runner_memory_cap_is_oom(cube):
    cfg = ChainConfig.small(64, 48)
    raw = cfg.make_raw()
    h = Host(memory_cap=64 * 48 * 2 + 10)  # room for the input buffer only
    buf, b = raw_input(h, cfg, raw)
    p = Pipeline(h, fused_chain_order(cube(b["lut_values"]), cfg.guided_radius, cfg.guided_eps))
    with pytest.raises(CpipeError) as e:
        p.run(buf)
    assert e.value.status == A.OOM
    p.close()
    buf.close()
    h.close()


def test_runner_refuses_wrong_input_format(host, cube):
    cfg = ChainConfig.small(32, 24)
    buf = host.buffer(A.FMT_R32_SFLOAT, 32, 24)
    p = Pipeline(host, fused_chain_order(cube(cfg.lut_values()), cfg.guided_radius, cfg.guided_eps))
    with pytest.raises(CpipeError) as e:
        p.run(buf)
    assert e.value.status == A.BAD_PRECISION
    p.close()
