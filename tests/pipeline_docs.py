"""Pipeline documents (schema v0.4) for the runner tests, built here from node
lists: the classic raw->display layout (a Quad-Bayer remosaic, linearize,
GainMap, black level, RCD, OpcodeList3, WB, colormatrix, denoise, tone, LUT,
sharpen, display, HEIF writer) and the fused chain's node order."""


def document(nodes, edges, input_format="R16_UINT", version="0.4", doc_id="test"):
    return {"$schema": "https://schemas.cpipe.dev/pipeline/v0.4.json", "version": version, "id": doc_id,
            "inputs": [{"port": "raw", "kind": "Image2D", "format": input_format}],
            "nodes": [{"id": i, "type": t, "params": p} for i, t, p in nodes],
            "edges": [{"from": f, "to": t} for f, t in edges]}


def chain(nodes, input_format="R16_UINT"):
    """A linear document: nodes = [(id, type, params, in_port, out_port)]."""
    edges = [(f"{a[0]}.{a[4]}", f"{b[0]}.{b[3]}") for a, b in zip(nodes, nodes[1:])]
    return document([(n[0], n[1], n[2]) for n in nodes], edges, input_format)


def classic(lut_path, display="sRGB"):
    return chain([
        ("qbc", "com.cpipe.demosaic.quad_bayer_remosaic", {}, "qbc", "bayer"),
        ("lin", "com.cpipe.linearize.dng_lut", {}, "raw", "bayer"),
        ("gain", "com.cpipe.lens.shading_gainmap", {}, "linear_bayer", "corrected_bayer"),
        ("bl", "com.cpipe.blacklevel.dng_levels", {}, "bayer", "bayer"),
        ("dem", "com.cpipe.demosaic.rcd", {}, "bayer", "rgba"),
        ("op3", "com.cpipe.lens.dng_opcode_list_3", {}, "scene_rgb", "corrected_rgb"),
        ("wb", "com.cpipe.wb.dual_illuminant", {}, "rgb", "rgb"),
        ("cm", "com.cpipe.colormatrix.dng_to_working", {}, "rgb", "rgb"),
        ("bm3d", "com.cpipe.denoise.bm3d", {}, "rgb", "rgb"),
        ("wavelet", "com.cpipe.denoise.wavelet_bayes_shrink", {}, "rgb", "rgb"),
        ("tone", "com.cpipe.tone.filmic_rgb", {}, "rgb", "rgb"),
        ("lut", "com.cpipe.color.3d_lut", {"lut_path": lut_path}, "rgb", "rgb"),
        ("sharp", "com.cpipe.sharpen.edge_aware_usm", {}, "rgb", "rgb"),
        ("display", "com.cpipe.color.scene_linear_to_display", {"target": display}, "rgb", "display"),
        ("out", "com.cpipe.output.heif_sdr", {}, "rgb", ""),
    ])


def fused_chain_order(lut_path, guided_radius=8, guided_eps=1e-3, demosaic="rcd"):
    """The fused chain's node order; the raw input reaches the black level
    through an implicit precision_convert."""
    return chain([
        ("bl", "com.cpipe.blacklevel.dng_levels", {}, "bayer", "bayer"),
        ("gain", "com.cpipe.lens.shading_gainmap", {}, "linear_bayer", "corrected_bayer"),
        ("dem", f"com.cpipe.demosaic.{demosaic}", {}, "bayer", "rgba"),
        ("op3", "com.cpipe.lens.dng_opcode_list_3", {}, "scene_rgb", "corrected_rgb"),
        ("wb", "com.cpipe.wb.dual_illuminant", {}, "rgb", "rgb"),
        ("cm", "com.cpipe.colormatrix.dng_to_working", {}, "rgb", "rgb"),
        ("bm3d", "com.cpipe.denoise.bm3d", {}, "rgb", "rgb"),
        ("guided", "com.cpipe.denoise.guided_filter", {"radius": guided_radius, "eps": guided_eps}, "rgb", "rgb"),
        ("wavelet", "com.cpipe.denoise.wavelet_bayes_shrink", {"chroma_strength": 1.0}, "rgb", "rgb"),
        ("tone", "com.cpipe.tone.filmic_rgb", {}, "rgb", "rgb"),
        ("lut", "com.cpipe.color.3d_lut", {"lut_path": lut_path}, "rgb", "rgb"),
    ])
