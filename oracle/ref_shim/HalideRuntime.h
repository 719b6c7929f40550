/* Minimal stand-in for the Halide runtime header, so the reference's plain-C++
 * filters can be compiled as the oracle's reference build.  Only the public
 * buffer structs are needed; the layout comes from include/cpipe_halide_abi.h.
 * Test infrastructure only. */
#pragma once
#include "../../include/cpipe_halide_abi.h"
template <class T> struct halide_type_of_impl;
template <> struct halide_type_of_impl<float> {
    static halide_type_t get() { return halide_type_t{halide_type_float, 32, 1}; }
};
template <class T> inline halide_type_t halide_type_of() { return halide_type_of_impl<T>::get(); }
