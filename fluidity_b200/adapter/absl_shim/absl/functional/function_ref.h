// Minimal stand-in for absl::FunctionRef where no absl installation exists
// (a non-owning callable reference is approximated with std::function).
#pragma once

#include <functional>

namespace absl {
template <typename Signature>
using FunctionRef = std::function<Signature>;
}  // namespace absl
