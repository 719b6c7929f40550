"""The pipeline runner's load-time planning on the CPU (host None: plan
only): node order, implicit precision converts, memory slots, and the
reference Pipeline::load status for every rejection
(src/cpipe/runtime/Pipeline.cpp:368-601, PrecisionPlanner::auto_insert)."""
import copy
import json

import pytest
from cpipe_b200 import _abi as A
from cpipe_b200.host import CpipeError
from cpipe_b200.pipeline import Pipeline
from pipeline_docs import chain, classic, document, fused_chain_order


def plan(doc, until=None):
    return Pipeline(None, doc, until=until)


def status_of(doc, until=None):
    try:
        plan(doc, until).close()
        return A.OK
    except CpipeError as e:
        return e.status


def test_classic_prefix_plans_in_document_order():
    p = plan(classic("x.cube"), until="display")
    assert [n for n, _ in p.nodes] == ["qbc", "lin", "gain", "bl", "dem", "op3", "wb", "cm", "bm3d", "wavelet",
                                       "tone", "lut", "sharp", "display"]
    # two planner slots suffice for a linear document (each output lives until the next node)
    peak, slots = p.memory_plan(4032, 3024)
    assert slots == 2
    rgba16 = 4032 * 3024 * 8
    assert peak == 4032 * 3024 * 2 + 2 * rgba16


def test_whole_classic_document_needs_the_heif_writer():
    """The HEIF writer is not a node of this library (the reference's
    registry has it): loading the whole document is CPIPE_BAD_INDEX."""
    assert status_of(classic("x.cube")) == A.BAD_INDEX


def test_implicit_precision_convert_inserted():
    # the R16_UINT input reaches the black level (f32) through an implicit converter
    p = plan(fused_chain_order("x.cube"))
    assert [t for _, t in p.nodes][:2] == ["com.cpipe.precision_convert", "com.cpipe.blacklevel.dng_levels"]
    assert p.nodes[0][0].startswith("__precision_convert_input_")
    # an edge whose precisions do not meet (u16 remosaic -> f32 GainMap)
    doc = chain([("qbc", "com.cpipe.demosaic.quad_bayer_remosaic", {}, "qbc", "bayer"),
                 ("gain", "com.cpipe.lens.shading_gainmap", {}, "linear_bayer", "corrected_bayer")])
    p = plan(doc)
    assert [t for _, t in p.nodes] == ["com.cpipe.demosaic.quad_bayer_remosaic", "com.cpipe.precision_convert",
                                       "com.cpipe.lens.shading_gainmap"]
    assert p.nodes[1][0].startswith("__precision_convert_")
    # matching precisions need none
    doc = chain([("lin", "com.cpipe.linearize.dng_lut", {}, "raw", "bayer"),
                 ("bl", "com.cpipe.blacklevel.dng_levels", {}, "bayer", "bayer"),
                 ("dem", "com.cpipe.demosaic.bilinear", {}, "bayer", "rgba"),
                 ("wb", "com.cpipe.wb.dual_illuminant", {}, "rgb", "rgb")])
    assert "com.cpipe.precision_convert" not in [t for _, t in plan(doc).nodes]


def test_memory_plan_reuses_slots_on_a_branch():
    """A branch keeps its producer live until both consumers ran: three slots."""
    doc = document([("dem", "com.cpipe.demosaic.bilinear", {}), ("wb", "com.cpipe.wb.dual_illuminant", {}),
                    ("cm", "com.cpipe.colormatrix.dng_to_working", {}), ("gw", "com.cpipe.wb.greyworld_auto", {})],
                   [("dem.rgba", "wb.rgb"), ("wb.rgb", "cm.rgb"), ("dem.rgba", "gw.rgb")], "R32_SFLOAT")
    p = plan(doc)
    assert p.memory_plan(64, 48)[1] == 3


@pytest.mark.parametrize("mutate,status", [
    (lambda d: d.update(version="0.3"), A.FAILED),
    (lambda d: d.pop("edges"), A.FAILED),
    (lambda d: d["nodes"][0].update(type="com.cpipe.nope"), A.BAD_INDEX),
    (lambda d: d["nodes"][0].update(type="com.cpipe.precision_convert"), A.BAD_INDEX),
    (lambda d: d["nodes"][4]["params"].update(bogus=1), A.BAD_INDEX),
    (lambda d: d["nodes"][4]["params"].update(algorithm="fancy"), A.BAD_INDEX),
    (lambda d: d["nodes"][8]["params"].update(sigma=5.0), A.BAD_INDEX),
    (lambda d: d["nodes"][8]["params"].update(sigma="high"), A.BAD_INDEX),
    (lambda d: d["edges"].append({"from": "nobody.x", "to": "lin.raw"}), A.BAD_INDEX),
    (lambda d: d["edges"].append({"from": "cm.rgb", "to": "op3.scene_rgb"}), A.FAILED),  # cycle
])
def test_load_rejections(mutate, status):
    doc = copy.deepcopy(classic("x.cube"))
    mutate(doc)
    assert status_of(doc, until="display") == status


def test_missing_step_and_role_mismatch():
    # filmic straight after the demosaic: its input requires the wavelet step
    doc = chain([("bl", "com.cpipe.blacklevel.dng_levels", {}, "bayer", "bayer"),
                 ("dem", "com.cpipe.demosaic.rcd", {}, "bayer", "rgba"),
                 ("tone", "com.cpipe.tone.filmic_rgb", {}, "rgb", "rgb")], "R32_SFLOAT")
    assert status_of(doc) == A.NEED_METADATA
    # colormatrix output (scene linear) into a white balance (raw camera)
    doc = chain([("dem", "com.cpipe.demosaic.rcd", {}, "bayer", "rgba"),
                 ("wb", "com.cpipe.wb.dual_illuminant", {}, "rgb", "rgb"),
                 ("cm", "com.cpipe.colormatrix.dng_to_working", {}, "rgb", "rgb"),
                 ("wb2", "com.cpipe.wb.dual_illuminant", {}, "rgb", "rgb")], "R32_SFLOAT")
    assert status_of(doc) == A.NEED_METADATA


def test_precision_mismatch_without_direct_conversion():
    # an RGBA16F output into a single-channel f32 port has no direct conversion
    doc = chain([("dem", "com.cpipe.demosaic.bilinear", {}, "bayer", "rgba"),
                 ("gain", "com.cpipe.lens.shading_gainmap", {}, "linear_bayer", "corrected_bayer")], "R32_SFLOAT")
    assert status_of(doc) == A.BAD_PRECISION


def test_malformed_json_and_unknown_until():
    assert status_of("{not json") == A.FAILED
    assert status_of(classic("x.cube"), until="nope") == A.BAD_INDEX
    assert status_of(json.dumps(classic("x.cube")), until="bm3d") == A.OK
