// Minimal stand-in for absl::FunctionRef used by the oracle build only
// (a non-owning callable reference is approximated with std::function).
#pragma once

#include <functional>

namespace absl {
template <typename Signature>
using FunctionRef = std::function<Signature>;
}  // namespace absl
