/* Minimal stand-in for the reference SDK header, sufficient for compiling the
 * reference's header-only white-balance helpers (src/cpipe/nodes/wb/WbMetadata.hpp)
 * into the oracle's reference build.  Only the types those helpers name are
 * declared.  Test infrastructure only. */
#pragma once
#include <array>
#include <cpipe/sdk/cpipe_node.h>
#include <cstddef>
#include <cstdint>
#include <optional>
#include <span>
#include <string>
#include <string_view>
#include <utility>
#include <variant>

namespace tl {
template <class E> struct unexpected {
    E value;
    explicit unexpected(E e) : value(std::move(e)) {}
};
}  // namespace tl

namespace cpipe::sdk {
struct Error {
    int code{0};
    std::string message;
};
template <class T> class Result {
public:
    Result(T v) : v_(std::move(v)) {}
    template <class E> Result(tl::unexpected<E> e) : v_(Error{e.value}) {}
    explicit operator bool() const { return v_.index() == 0; }
    const T& operator*() const { return std::get<0>(v_); }
    const T* operator->() const { return &std::get<0>(v_); }
    Error error() const { return std::get<1>(v_); }
private:
    std::variant<T, Error> v_;
};
template <> class Result<void> {
public:
    Result() = default;
    template <class E> Result(tl::unexpected<E> e) : err_(Error{e.value}), ok_(false) {}
    explicit operator bool() const { return ok_; }
    Error error() const { return err_; }
private:
    Error err_{};
    bool ok_{true};
};
struct CalibrationView {
    std::optional<std::array<float, 9>> color_matrix1;
    std::optional<std::array<float, 9>> color_matrix2;
    std::optional<std::array<float, 9>> forward_matrix1;
    std::optional<std::array<float, 9>> forward_matrix2;
    std::uint16_t calibration_illuminant1{0};
    std::uint16_t calibration_illuminant2{0};
};
struct MetadataBuilder {
    Result<void> set_blob(std::string_view, std::span<const std::byte>) { return {}; }
};
}  // namespace cpipe::sdk
