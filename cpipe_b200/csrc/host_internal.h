// Internal hooks of the host runtime (host_runtime.cpp) for the pipeline
// runner (pipeline_runtime.cpp).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/cpipe_b200.h"

// A buffer handle over device memory the caller keeps (no allocation; destroy
// frees only the handle).
cpipe_b200_buffer* cpb_buffer_view(cpipe_b200_host* h, int format, uint32_t w, uint32_t hgt, void* dev);
size_t cpb_format_bytes(int format);
int cpb_buffer_format(const cpipe_b200_buffer* b);
void cpb_buffer_extent(const cpipe_b200_buffer* b, uint32_t* w, uint32_t* h);
// dst takes src's metadata (shared, frozen).
void cpb_buffer_share_metadata(cpipe_b200_buffer* dst, const cpipe_b200_buffer* src);
cudaStream_t cpb_host_stream(cpipe_b200_host* h);
uint64_t cpb_host_memory_cap(cpipe_b200_host* h);  // 0 = none
void cpb_host_set_error(cpipe_b200_host* h, const std::string& e);
const std::string& cpb_host_error(cpipe_b200_host* h);
// Builtin-node access to this library's own host (the reference's builtin
// dng_input replaces its output's buffer object the same privileged way).
bool cpb_is_own_host(const cpipe_host_t* h);
cudaStream_t cpb_abi_host_stream(cpipe_host_t* h);
void* cpb_buffer_device(const cpipe_buffer_t* b);
struct cpipe_DngInfo;
int cpb_builder_set_dng(cpipe_metadata_builder_t* builder, const struct cpipe_DngInfo* info, const uint8_t* file,
                        size_t file_bytes);
int cpb_run_node(cpipe_b200_host* h, const cpipe_plugin_desc_t* desc, const cpipe_b200_params* params,
                 cpipe_b200_buffer* const* inputs, size_t n_in, cpipe_b200_buffer* const* outputs, size_t n_out,
                 bool sync);
