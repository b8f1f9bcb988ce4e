// Minimal stand-in for absl::StatusOr<T> where no absl installation exists.
#pragma once

#include <cassert>
#include <optional>
#include <type_traits>
#include <utility>

#include "absl/status/status.h"

namespace absl {

template <typename T>
class StatusOr {
 public:
  StatusOr() : status_(StatusCode::kUnknown, {}) {}
  StatusOr(const Status& status) : status_(status) {}  // NOLINT: implicit like absl
  StatusOr(Status&& status) : status_(std::move(status)) {}  // NOLINT
  StatusOr(const T& value) : value_(value) {}  // NOLINT
  StatusOr(T&& value) : value_(std::move(value)) {}  // NOLINT
  template <typename U,
            typename = std::enable_if_t<std::is_constructible_v<T, U&&> && !std::is_same_v<std::decay_t<U>, T> &&
                                        !std::is_same_v<std::decay_t<U>, Status> &&
                                        !std::is_same_v<std::decay_t<U>, StatusOr<T>>>>
  StatusOr(U&& value) : value_(T(std::forward<U>(value))) {}  // NOLINT
  StatusOr(const StatusOr&) = default;
  StatusOr(StatusOr&&) = default;
  StatusOr& operator=(const StatusOr&) = default;
  StatusOr& operator=(StatusOr&&) = default;

  bool ok() const { return value_.has_value(); }
  const Status& status() const& { return status_; }
  Status status() && { return status_; }
  T& value() & { return *value_; }
  const T& value() const& { return *value_; }
  T&& value() && { return std::move(*value_); }
  T& operator*() & { return *value_; }
  const T& operator*() const& { return *value_; }
  T&& operator*() && { return std::move(*value_); }
  T* operator->() { return &*value_; }
  const T* operator->() const { return &*value_; }
  template <typename U>
  T value_or(U&& fallback) const& { return ok() ? *value_ : static_cast<T>(std::forward<U>(fallback)); }

 private:
  Status status_;
  std::optional<T> value_;
};

}  // namespace absl
