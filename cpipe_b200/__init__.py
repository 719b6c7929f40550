"""cpipe_b200: B200 (sm_100a) CUDA kernels for the cpipe raw->linear node chain,
behind the reference's filter (HalideParamFilterEntry) and plugin (main_entry)
interfaces.  See include/cpipe_b200.h for the C ABI."""
from ._abi import lib  # noqa: F401  (raises if libcpipe_b200.so is not built)
from .host import (Buffer, CpipeError, DeviceImage, Host, Params, Registry, call_entry, call_filter,  # noqa: F401
                   last_error, process_single_input_node)
