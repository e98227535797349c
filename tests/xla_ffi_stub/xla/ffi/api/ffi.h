// A compile-only stand-in for XLA's typed FFI header (xla/ffi/api/ffi.h), used by
// tests/test_xla_ffi.py to compile gradsolve_b200/csrc/gs_xla_ffi.cc where JAX is not installed.
// It declares the subset of the API the handlers use, with XLA's names and shapes, and makes
// XLA_FFI_DEFINE_HANDLER_SYMBOL check at compile time that each binding decodes to exactly the
// parameter types of its handler (Ctx<PlatformStream<T>> -> T, Arg<T> -> T, Ret<T> ->
// Result<T>, Attr<T> -> T, in order).  Nothing here runs.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <tuple>
#include <type_traits>

struct XLA_FFI_Error;
struct XLA_FFI_CallFrame;

namespace xla::ffi {

enum class DataType : uint8_t { S32, S64, F32, F64 };
inline constexpr DataType S32 = DataType::S32;
inline constexpr DataType S64 = DataType::S64;
inline constexpr DataType F32 = DataType::F32;
inline constexpr DataType F64 = DataType::F64;

template <DataType>
struct NativeTypeOf;
template <> struct NativeTypeOf<DataType::S32> { using type = int32_t; };
template <> struct NativeTypeOf<DataType::S64> { using type = int64_t; };
template <> struct NativeTypeOf<DataType::F32> { using type = float; };
template <> struct NativeTypeOf<DataType::F64> { using type = double; };
template <DataType d>
using NativeType = typename NativeTypeOf<d>::type;

template <typename T>
struct Span {
  const T* data_;
  size_t size_;
  size_t size() const { return size_; }
  const T& operator[](size_t i) const { return data_[i]; }
  const T& back() const { return data_[size_ - 1]; }
};

inline constexpr size_t kDynamicRank = static_cast<size_t>(-1);

template <DataType dtype, size_t rank = kDynamicRank>
class Buffer {
 public:
  NativeType<dtype>* typed_data() const;
  Span<const int64_t> dimensions() const;
  size_t element_count() const;
};

template <typename T>
class Result {
 public:
  T* operator->() const;
  T& operator*() const;
};

template <DataType dtype, size_t rank = kDynamicRank>
using ResultBuffer = Result<Buffer<dtype, rank>>;

class Error {
 public:
  static Error Success();
  static Error Internal(std::string message);
  static Error InvalidArgument(std::string message);
};

template <typename T>
struct PlatformStream {};

template <typename T>
struct CtxDecoding;
template <typename T>
struct CtxDecoding<PlatformStream<T>> {
  using type = T;
};

template <typename Fn>
struct HandlerParams;
template <typename R, typename... As>
struct HandlerParams<R (*)(As...)> {
  using result = R;
  using params = std::tuple<As...>;
};

template <typename... Ts>
class Binding {
 public:
  template <typename T>
  Binding<Ts..., typename CtxDecoding<T>::type> Ctx() const;
  template <typename T>
  Binding<Ts..., T> Arg() const;
  template <typename T>
  Binding<Ts..., Result<T>> Ret() const;
  template <typename T>
  Binding<Ts..., T> Attr(const char* name) const;
  // true when a handler of type Fn takes exactly the decoded types, in order, returning Error
  template <typename Fn>
  static constexpr bool binds() {
    using H = HandlerParams<Fn>;
    return std::is_same_v<typename H::params, std::tuple<Ts...>> &&
           std::is_same_v<typename H::result, Error>;
  }
};

class Ffi {
 public:
  static Binding<> Bind();
};

}  // namespace xla::ffi

#define XLA_FFI_DEFINE_HANDLER_SYMBOL(fn, impl, binding)                                    \
  static_assert(std::decay_t<decltype(binding)>::template binds<decltype(&impl)>(),          \
                "the FFI binding of " #fn " does not match the parameters of " #impl);       \
  extern "C" XLA_FFI_Error* fn(XLA_FFI_CallFrame*) { return nullptr; }
