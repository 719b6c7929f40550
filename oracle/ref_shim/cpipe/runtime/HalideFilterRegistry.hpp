/* Stand-in for the reference's HalideFilterRegistry.hpp used only when the
 * reference's filter sources are compiled into the oracle's reference build:
 * the two registration macros record (aot_id, entry) pairs in a table that
 * oracle/ref_glue.cpp exposes through a C function.  Test infrastructure only. */
#pragma once
#include <HalideRuntime.h>
#include <cstddef>

using RefFilterEntry = int (*)(halide_buffer_t*, halide_buffer_t*);
using RefParamFilterEntry = int (*)(halide_buffer_t* const*, std::size_t, halide_buffer_t* const*,
                                    std::size_t, const void*, std::size_t);
void cpipe_ref_register_filter(const char* aot_id, RefFilterEntry entry);
void cpipe_ref_register_param_filter(const char* aot_id, RefParamFilterEntry entry);

#define CPIPE_REF_CAT2(a, b) a##b
#define CPIPE_REF_CAT(a, b) CPIPE_REF_CAT2(a, b)
#define CPIPE_REGISTER_HALIDE_FILTER(aot_id_literal, entry_ptr)                              \
    namespace {                                                                              \
    const int CPIPE_REF_CAT(cpipe_ref_reg_, __COUNTER__) =                                   \
        (cpipe_ref_register_filter(aot_id_literal, entry_ptr), 0);                           \
    }
#define CPIPE_REGISTER_HALIDE_PARAM_FILTER(aot_id_literal, entry_ptr)                        \
    namespace {                                                                              \
    const int CPIPE_REF_CAT(cpipe_ref_reg_, __COUNTER__) =                                   \
        (cpipe_ref_register_param_filter(aot_id_literal, entry_ptr), 0);                     \
    }
