/* Halide runtime buffer descriptor, restated so the filter seam can be called
 * by a host that hands out `halide_buffer_t*` exactly as the reference runtime
 * does (`src/cpipe/runtime/HalideBufferAdapter.cpp:37-76`).
 *
 * Layout: the public `halide_buffer_t` struct of the Halide v21 runtime
 * (`HalideRuntime.h`, a third-party header that is not part of the reference
 * tree).  The struct fields are an ABI, so they are kept in the same order.
 *
 * Device convention of this library: when `device != 0` the buffer is CUDA
 * device memory (a CUdeviceptr, the same convention Halide's own CUDA device
 * interface uses) and kernels read/write it in place; otherwise `host` is used
 * and the library stages the pixels through device memory.
 */
#ifndef CPIPE_HALIDE_ABI_H
#define CPIPE_HALIDE_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef HALIDE_HALIDERUNTIME_H
typedef enum {
    halide_type_int = 0,
    halide_type_uint = 1,
    halide_type_float = 2,
    halide_type_handle = 3,
    halide_type_bfloat = 4
} halide_type_code_t;

struct halide_type_t {
    uint8_t code;
    uint8_t bits;
    uint16_t lanes;
};

typedef struct halide_dimension_t {
    int32_t min;
    int32_t extent;
    int32_t stride;
    uint32_t flags;
} halide_dimension_t;

struct halide_device_interface_t;

typedef struct halide_buffer_t {
    uint64_t device;
    const struct halide_device_interface_t* device_interface;
    uint8_t* host;
    uint64_t flags;
    struct halide_type_t type;
    int32_t dimensions;
    halide_dimension_t* dim;
    void* padding;
} halide_buffer_t;

enum { halide_buffer_flag_host_dirty = 1, halide_buffer_flag_device_dirty = 2 };
#endif

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CPIPE_HALIDE_ABI_H */
