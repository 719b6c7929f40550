"""The CPU legs of bench.py build the chain's filter blobs without the product
library (oracle/oracle_blobs.py, from the reference's POD layouts and its own
white-balance helpers).  They must be the bytes the library's host preparation
produces, and the reference CPU chain must compute what the oracle chain does."""
import numpy as np
import oracle
import oracle_blobs
import pytest
from chain_oracle import run_chain_oracle, run_reference_chain
from cpipe_b200.chain import ChainConfig

CFGS = [ChainConfig.full_12mp(), ChainConfig.small_frame(), ChainConfig.small(97, 63, cfa=(2, 1, 1, 0)),
        ChainConfig.qbc_50mp(), ChainConfig.small(64, 48, cfa=(1, 0, 2, 1), warp=(1.0, -0.1, 0.0, 0.01, 0.001, 0.0))]


@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: c.name)
def test_blobs_equal_library_preparation(cfg):
    if oracle.ref_lib() is None:
        pytest.skip("reference build absent")
    mine = oracle_blobs.chain_blobs(cfg)
    lib = cfg.blobs()
    for key in ("blacklevel", "gainmap", "opcode3", "wb", "colormatrix"):
        assert (key in mine) == (key in lib), key
        if key in lib:
            assert mine[key] == lib[key], key
    assert mine["colormatrix_t"] == lib["colormatrix_t"]


@pytest.mark.parametrize("cfg", [ChainConfig.small(97, 63), ChainConfig.small(130, 70, cfa=(1, 0, 2, 1)),
                                 ChainConfig.small_frame(200, 150), ChainConfig.small(96, 64, quad_bayer=True)],
                         ids=lambda c: c.name)
def test_reference_chain_equals_oracle_chain(cfg):
    if oracle.ref_lib() is None:
        pytest.skip("reference build absent")
    raw = cfg.make_raw()
    a = run_reference_chain(cfg, raw, oracle_blobs.chain_blobs(cfg))
    b = run_chain_oracle(cfg, raw)
    np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
