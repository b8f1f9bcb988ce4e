// Minimal stand-in for absl::Cleanup where no absl installation exists (the
// backend adapter and the reference's CPU operators built in this repository;
// inside the reference's own tree its absl is used instead): a move-only scope
// guard that runs its callback on destruction unless cancelled.
#pragma once

#include <utility>

namespace absl {

template <typename Callback>
class Cleanup {
 public:
  Cleanup(Callback callback) : callback_(std::move(callback)) {}
  Cleanup(Cleanup&& other) noexcept : callback_(std::move(other.callback_)), armed_(other.armed_) {
    other.armed_ = false;
  }
  Cleanup(const Cleanup&) = delete;
  Cleanup& operator=(const Cleanup&) = delete;
  ~Cleanup() {
    if (armed_) callback_();
  }
  void Cancel() && { armed_ = false; }
  void Invoke() && {
    if (armed_) {
      armed_ = false;
      callback_();
    }
  }

 private:
  Callback callback_;
  bool armed_ = true;
};

template <typename Callback>
Cleanup(Callback) -> Cleanup<Callback>;

template <typename Callback>
Cleanup<Callback> MakeCleanup(Callback callback) {
  return Cleanup<Callback>(std::move(callback));
}

}  // namespace absl
